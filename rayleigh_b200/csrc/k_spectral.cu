// Spectral-space stages of the step:
//   cheb_synthesis_kernel  d^k/dr^k on the collocation grid of the solved
//                          Chebyshev coefficients (K5 + K7 fused: the derivative
//                          recursion of Cheby_Deriv_Buffer_4D followed by
//                          From_Spectral4D equals one product with the derivative
//                          matrices dcheby(:,:,k); Chebyshev_Polynomials.F90:299-351,
//                          450-644), parity split about the mid-shell.
//   post_assemble_kernel   Add_Derivative x16 + Set_All_RHS + Transpose_1a2a
//                          (Sphere_Spectral_Space.F90:204-410, Linear_Solve.F90:758-796).
//   rlm_a_kernel           rlm_spacea algebra (Sphere_Hybrid_Space.F90:64-355).
//   rlm_b_kernel           rlm_spaceb algebra + Transpose_2b1b (Sphere_Hybrid_Space.F90:127-222).
// The per-l implicit solves that follow (Implicit_Solve, LU_Decompose_Matrices)
// are in k_solve.cu.
#include <cmath>

#include "ra_internal.h"
#include "gemm_f64.cuh"

namespace ra {

__device__ __forceinline__ int ell_of_lm(long lm) {
    int l = (int)floor((sqrt(8.0 * (double)lm + 1.0) - 1.0) * 0.5);
    while ((long)(l + 1) * (l + 2) / 2 <= lm) ++l;
    while ((long)l * (l + 1) / 2 > lm) --l;
    return l;
}

// ---------------------------------------------------------------------------
// Chebyshev synthesis of the 12 grid outputs (W W' W'' W''' P P' T T' T'' Z Z' Z'')
// ---------------------------------------------------------------------------

// One CTA per (field, 128-column tile).  D(n_r - 1 - r, k) = (-1)^(k+d) D(r, k),
// so rows r < n_r/2 give both halves of the grid:
//   g(r) = E + O,  g(n_r - 1 - r) = (-1)^d (E - O),
// E / O the products over even / odd k.  Dpar[d][par][r][k'] = D_d(r, 2k' + par).
// Per (derivative order, 32-row block: the n_r/2 = 96 half-grid rows in three
// full blocks) the CTA computes E, parks it in shared memory (each thread its
// own accumulator slots, so no barrier), computes O in the same registers and
// writes both halves.  The coefficients stream through the tile engine's own
// double-buffered stage from L2: one accumulator and no coefficient stage keep
// a CTA at about 75 KB of shared memory and 168 registers, three CTAs per SM.
struct ChebField { int o0, nd, var; };
__constant__ ChebField kChebField[6] = {{G_W0, 4, 0}, {G_P0, 2, 1}, {G_T0, 3, 2}, {G_Z0, 3, 3},
                                        {G_C0, 3, 4}, {G_A0, 3, 5}};   // C and A with magnetism

using ChebShape = Wide;   // 32 x 128 tiles: 32-row blocks cover the n_r/2 = 96 half-grid rows exactly
struct ChebSmem {
    GemmSmemT<1, 4> g;
    double park[32][GEMM_THREADS];   // E of the thread's 32 accumulator slots
};

__global__ void __launch_bounds__(GEMM_THREADS, 3) cheb_synthesis_kernel(const double* __restrict__ Dpar,
                                                                         const double* __restrict__ sol_wpt,
                                                                         const double* __restrict__ sol_z,
                                                                         const double* __restrict__ sol_c,
                                                                         const double* __restrict__ sol_a,
                                                                         double* __restrict__ g, int nr, int kc,
                                                                         long ncols) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ChebSmem& sm = *reinterpret_cast<ChebSmem*>(smem_raw);
    const int kh = (kc + 1) / 2;   // coefficients per parity (the odd plane has one fewer when kc is odd)
    const ChebField cf = kChebField[blockIdx.y];
    const long c0 = (long)blockIdx.x * ChebShape::BN;
    const int nr2 = nr / 2;
    const double* src;
    long cstride;
    if (cf.var < 3) {
        src = sol_wpt + (long)cf.var * nr;
        cstride = 3L * nr;
    } else {
        src = cf.var == 3 ? sol_z : (cf.var == 4 ? sol_c : sol_a);
        cstride = nr;
    }
    const int t = threadIdx.x;
    for (int dd = 0; dd < cf.nd; ++dd) {
        const int o = cf.o0 + dd;
        const double sgn = (dd & 1) ? -1.0 : 1.0;
        double* out = g + (long)o * ncols * nr;
        for (int r0 = 0; r0 < nr2; r0 += ChebShape::BM) {
            Acc acc;
#pragma unroll 1
            for (int par = 0; par < 2; ++par) {
                const double* Dp = Dpar + (((long)dd * 2 + par) * nr2) * kh;
                auto fa = [&](int k, int x) -> double {
                    const int r = r0 + x;
                    return (k < kh && r < nr2) ? __ldg(Dp + (long)r * kh + k) : 0.0;
                };
                auto fb = [&](int k, int y) -> double {   // coefficient 2k + par of column c0 + y
                    const long col = c0 + y;
                    const int kk = 2 * k + par;
                    return (kk < kc && col < ncols) ? __ldg(src + col * cstride + kk) : 0.0;
                };
                acc.zero();
                gemm_tile<false, false, 1, 4>(acc, fa, fb, kh, sm.g);
                if (par == 0) {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j)
#pragma unroll
                            for (int q = 0; q < 2; ++q) sm.park[(i * 4 + j) * 2 + q][t] = acc.v[i][j][q];
                }
            }
            int slot = 0;
            acc_foreach<1, 4>(acc, [&](int x, int y, double od) {
                const double e = sm.park[slot++][t];
                const int r = r0 + x;
                const long col = c0 + y;
                if (r < nr2 && col < ncols) {
                    out[col * nr + r] = e + od;
                    out[col * nr + (nr - 1 - r)] = sgn * (e - od);
                }
            });
        }
    }
}

// The finite-difference radial mode's synthesis: the state holds grid values, and every grid
// output is one banded operator (I, D_1, D_2, D_3 of Finite_Difference.F90, or D_1 D_1 for the
// deriv_cluge plane) applied to a field's radial columns (d_by_dx3d3, Post_Solve_FD,
// Sphere_Spectral_Space.F90:37-176).  Each output point is its row's stencil (at most fd_w
// coefficients) against the column: one thread per point, r fastest, so that the column
// reads and the plane writes are coalesced and each field is read from HBM about once; all
// outputs in one launch (grid y = output).
struct FdOuts {
    int n;
    int o[NG_MAG + 1], var[NG_MAG + 1], mat[NG_MAG + 1];
};

__global__ void __launch_bounds__(256) fd_synthesis_kernel(const double* __restrict__ band, int w,
                                                           const double* __restrict__ sol_wpt,
                                                           const double* __restrict__ sol_z,
                                                           const double* __restrict__ sol_c,
                                                           const double* __restrict__ sol_a,
                                                           double* __restrict__ g, int nr, long ncols, FdOuts outs) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (column, r), r fastest
    if (i >= ncols * nr) return;
    const int oi = blockIdx.y;
    const int var = outs.var[oi];
    const long col = i / nr;
    const int r = (int)(i - col * nr);
    const double* src;
    long cstride;
    if (var < 3) {
        src = sol_wpt + (long)var * nr;
        cstride = 3L * nr;
    } else {
        src = var == 3 ? sol_z : (var == 4 ? sol_c : sol_a);
        cstride = nr;
    }
    const double* row = band + ((long)outs.mat[oi] * nr + r) * (w + 1);
    const int first = (int)__ldg(row);   // first + w <= nr
    const double* x = src + col * cstride + first;
    double s = 0.0;
    for (int j = 0; j < w; ++j) s += __ldg(row + 1 + j) * __ldg(x + j);
    g[(long)outs.o[oi] * ncols * nr + i] = s;
}

static void launch_fd_synthesis(Ctx& c) {
    const long ncols = 2 * c.d.nlm;
    FdOuts outs{};
    auto add = [&](int o, int var, int mat) {
        outs.o[outs.n] = o;
        outs.var[outs.n] = var;
        outs.mat[outs.n] = mat;
        ++outs.n;
    };
    for (int d = 0; d < 4; ++d) add(G_W0 + d, 0, d);
    for (int d = 0; d < 2; ++d) add(G_P0 + d, 1, d);
    for (int d = 0; d < 3; ++d) add(G_T0 + d, 2, d);
    for (int d = 0; d < 3; ++d) add(G_Z0 + d, 3, d);
    if (c.mag) {
        for (int d = 0; d < 3; ++d) add(G_C0 + d, 4, d);
        for (int d = 0; d < 3; ++d) add(G_A0 + d, 5, d);
    }
    add(c.ng, 0, 4);   // the deriv_cluge plane: D_1 D_1 W
    const long total = ncols * c.d.nr;
    dim3 grid((unsigned)((total + 255) / 256), (unsigned)outs.n);
    fd_synthesis_kernel<<<grid, 256, 0, c.stream>>>(c.d_Dfd, c.fd_w, c.d_sol_wpt, c.d_sol_z, c.d_sol_c, c.d_sol_a,
                                                    c.d_g, c.d.nr, ncols, outs);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

void launch_cheb_synthesis(Ctx& c) {
    if (!c.cfg.chebyshev) {
        launch_fd_synthesis(c);
        return;
    }
    const long ncols = 2 * c.d.nlm;
    const size_t smem = sizeof(ChebSmem);
    // the limit is per device: set it on every launch (a host-side call, also legal during capture)
    RA_CUDA(cudaFuncSetAttribute(cheb_synthesis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((ncols + ChebShape::BN - 1) / ChebShape::BN), c.mag ? 6 : 4);
    cheb_synthesis_kernel<<<grid, GEMM_THREADS, smem, c.stream>>>(c.d_Dpar, c.d_sol_wpt, c.d_sol_z, c.d_sol_c,
                                                                   c.d_sol_a, c.d_g, c.d.nr, c.d.kc, ncols);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// ---------------------------------------------------------------------------
// RHS assembly + transpose to the m-major spectral layout
// ---------------------------------------------------------------------------
// the RHS terms (equation, grid source) as compile-time functions, so that
// unrolled loops index register arrays with constants (same table as kSlots)
__host__ __device__ constexpr int slot_eq(int s) {
    constexpr int e[NSLOT] = {EQ_W, EQ_W, EQ_W, EQ_W, EQ_W, EQ_P, EQ_P, EQ_P,
                              EQ_P, EQ_P, EQ_T, EQ_T, EQ_T, EQ_Z, EQ_Z, EQ_Z};
    return e[s];
}
__host__ __device__ constexpr int slot_g(int s) {
    constexpr int g[NSLOT] = {G_W0, G_W1, G_W2, G_P1, G_T0, G_W0, G_W1, G_W2,
                              G_W3, G_P0, G_T0, G_T1, G_T2, G_Z0, G_Z1, G_Z2};
    return g[s];
}
static_assert(slot_eq(3) == kSlots[3].eq && slot_g(8) == kSlots[8].g && slot_g(15) == kSlots[15].g, "slot table");

// w2s (finite-difference mode only, else NULL): the plane of d/dr (dW/dr) that Post_Solve_FD's
// deriv_cluge sends on to rlm_spacea in place of d2W/dr2 (Sphere_Spectral_Space.F90:96-98).
__global__ void post_assemble_kernel(const double* __restrict__ g, const double* __restrict__ ab,
                                     const double* __restrict__ coef, double* __restrict__ rhs_wpt,
                                     double* __restrict__ rhs_z, double* __restrict__ s2a, long nlm, int nr,
                                     int L, double old_ab, const double* __restrict__ w2s) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (lm, r), r fastest; both re/im
    if (idx >= nlm * nr) return;
    const int r = (int)(idx % nr);
    const long lm = idx / nr;
    const int l = ell_of_lm(lm);
    const int m = (int)(lm - (long)l * (l + 1) / 2);
    const long plane = nlm * 2 * nr;    // one field of g / ab
    const long i0 = lm * 2 * nr + r;    // (lm, re, r); (lm, im, r) is nr further
    double gv[NG][2];
#pragma unroll
    for (int o = 0; o < NG; ++o) {
        gv[o][0] = g[o * plane + i0];
        gv[o][1] = g[o * plane + i0 + nr];
    }
    double acc[4][2];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        acc[e][0] = ab[e * plane + i0] * old_ab;
        acc[e][1] = ab[e * plane + i0 + nr] * old_ab;
    }
    const double* cf = coef + (long)l * NSLOT * nr + r;
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) {
        const double c = cf[s * nr];
        acc[slot_eq(s)][0] += c * gv[slot_g(s)][0];   // compile-time indices (unrolled)
        acc[slot_eq(s)][1] += c * gv[slot_g(s)][1];
    }
#pragma unroll
    for (int ri = 0; ri < 2; ++ri) {
        const long base = (lm * 2 + ri) * 3L * nr;
        rhs_wpt[base + r] = acc[EQ_W][ri];
        rhs_wpt[base + nr + r] = acc[EQ_P][ri];
        rhs_wpt[base + 2 * nr + r] = acc[EQ_T][ri];
        rhs_z[(lm * 2 + ri) * nr + r] = acc[EQ_Z][ri];
    }
    // s2a[row][f][r][ri] with f = W T Z W' T' Z' W''
    const long row = row_index(m, l, L);
    double* o = s2a + row * (long)NS2A * nr * 2 + (long)r * 2;
    const long fs = 2L * nr;
    constexpr int kOut[NS2A] = {G_W0, G_T0, G_Z0, G_W1, G_T1, G_Z1, G_W2};
#pragma unroll
    for (int f = 0; f < NS2A - 1; ++f)
        *reinterpret_cast<double2*>(o + f * fs) = make_double2(gv[kOut[f]][0], gv[kOut[f]][1]);
    const double2 w2 = w2s ? make_double2(w2s[i0], w2s[i0 + nr]) : make_double2(gv[G_W2][0], gv[G_W2][1]);
    *reinterpret_cast<double2*>(o + (NS2A - 1) * fs) = w2;
}

void launch_post_assemble(Ctx& c, double old_ab) {
    const long total = c.d.nlm * c.d.nr;
    const double* w2s = c.cfg.chebyshev ? nullptr : c.d_g + (size_t)c.ng * c.d.nlm * 2 * c.d.nr;
    post_assemble_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(
        c.d_g, c.d_ab, c.d_coef, c.d_rhs_wpt, c.d_rhs_z, c.d_s2a, c.d.nlm, c.d.nr, c.d.L, old_ab, w2s);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// The C and A parts of Post_Solve (Sphere_Spectral_Space.F90:268-297, 370-384): their
// right-hand sides, and the fields rlm_spacea's magnetic part reads, m-major.
__global__ void post_assemble_mag_kernel(const double* __restrict__ g, const double* __restrict__ ab,
                                         const double* __restrict__ coefm, double* __restrict__ rhs_c,
                                         double* __restrict__ rhs_a, double* __restrict__ s2am, long nlm, int nr,
                                         int L, double old_ab) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (lm, r)
    if (idx >= nlm * nr) return;
    const int r = (int)(idx % nr);
    const long lm = idx / nr;
    const int l = ell_of_lm(lm);
    const int m = (int)(lm - (long)l * (l + 1) / 2);
    const long plane = nlm * 2 * nr;
    const long i0 = lm * 2 * nr + r;
    const double* cf = coefm + (long)l * NMSLOT * nr + r;
    const double c0 = cf[MS_C0 * nr], c2 = cf[MS_C2 * nr];
    const double a0 = cf[MS_A0 * nr], a1 = cf[MS_A1 * nr], a2 = cf[MS_A2 * nr];
    double gv[6][2];
#pragma unroll
    for (int o = 0; o < 6; ++o) {
        gv[o][0] = g[(G_C0 + o) * plane + i0];
        gv[o][1] = g[(G_C0 + o) * plane + i0 + nr];
    }
#pragma unroll
    for (int ri = 0; ri < 2; ++ri) {
        const long o = i0 + ri * nr;
        // p1b = old_ab * p1b, then Add_Derivative in the reference's order: A'' (from the
        // ctemp buffer), then A, A' and C'', C
        double ra = ab[5 * plane + o] * old_ab;
        double rc = ab[4 * plane + o] * old_ab;
        ra += a2 * gv[G_A2 - G_C0][ri];
        ra += a0 * gv[G_A0 - G_C0][ri];
        ra += a1 * gv[G_A1 - G_C0][ri];
        rc += c2 * gv[G_C2 - G_C0][ri];
        rc += c0 * gv[G_C0 - G_C0][ri];
        rhs_a[o] = ra;
        rhs_c[o] = rc;
    }
    const long row = row_index(m, l, L);
    double* so = s2am + row * (long)NS2AM * nr * 2 + (long)r * 2;
    const long fs = 2L * nr;
    constexpr int kOut[NS2AM] = {G_C0, G_A0, G_C1, G_A1, G_C2};
#pragma unroll
    for (int f = 0; f < NS2AM; ++f)
        *reinterpret_cast<double2*>(so + f * fs) = make_double2(gv[kOut[f] - G_C0][0], gv[kOut[f] - G_C0][1]);
}

void launch_post_assemble_mag(Ctx& c, double old_ab) {
    const long total = c.d.nlm * c.d.nr;
    post_assemble_mag_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(
        c.d_g, c.d_ab, c.d_coef_mag, c.d_rhs_c, c.d_rhs_a, c.d_s2am, c.d.nlm, c.d.nr, c.d.L, old_ab);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// ---------------------------------------------------------------------------
// rlm_spacea: 7 spectral fields -> the 11 fields the inverse transform carries
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dth_c1(int l, int m) {   // sin(theta) d/dtheta, l-1 coefficient
    const double num = (double)(l + m) * (l - m), den = (double)(2 * l + 1) * (2 * l - 1);
    return (l - 1) * sqrt(num / den);
}
__device__ __forceinline__ double dth_c2(int l, int m) {   // l+1 coefficient
    const double num = (double)(l + 1 + m) * (l + 1 - m), den = (double)(2 * l + 1) * (2 * l + 3);
    return -(l + 2) * sqrt(num / den);
}
__device__ __forceinline__ double sdth_c1(int l, int m) {
    const double num = (double)(l + m) * (l - m), den = (double)(2 * l + 1) * (2 * l - 1);
    return (l + 1) * sqrt(num / den);
}
__device__ __forceinline__ double sdth_c2(int l, int m) {
    const double num = (double)(l + 1 + m) * (l + 1 - m), den = (double)(2 * l + 1) * (2 * l + 3);
    return -l * sqrt(num / den);
}

constexpr int RLM_A_THREADS = 256;

// (m, l) of a row of the m-major, parity-split row order (row_index inverted):
// m_off(m) <= row < m_off(m + 1), then the even-l rows of m before the odd-l ones.
__device__ __forceinline__ void ml_of_row(long row, int L, int& m, int& l) {
    const double b = 2.0 * L + 1.0;
    int mm = (int)floor((b - sqrt(b * b - 8.0 * (double)row)) * 0.5);
    mm = max(0, min(mm, L - 1));
    while (mm > 0 && m_off(mm, L) > row) --mm;
    while (mm + 1 < L && m_off(mm + 1, L) <= row) ++mm;
    const int p = (int)(row - m_off(mm, L));
    const int ne = n_even(mm, L);
    m = mm;
    l = mm + (p < ne ? 2 * p : 2 * (p - ne) + 1);
}

// Compute_BandCurlB (Sphere_Hybrid_Space.F90:357-435): B and curl B in (l, m) space from
// C, A, C', A', C'' (the l_max mode zeroed on entry and exit, as for the hydrodynamic fields):
//   B_r = l(l+1) C / r^2,  (curl B)_r = l(l+1) A / r^2,  X = C'' - B_r,
//   r sin(theta) (curl B)_theta = d_theta A' - d_phi X,  r sin(theta) (curl B)_phi = d_phi A' + d_theta X,
//   r sin(theta) B_theta = d_phi A + d_theta C',          r sin(theta) B_phi = d_phi C' - d_theta A,
// with d_theta = sin(theta) d/dtheta through the l -+ 1 couplings (fields A_BR .. A_BP).
__device__ __forceinline__ void band_curl_b(const double* __restrict__ s2am, const double* __restrict__ radial,
                                            int nr, int L, int l, int m, int r, double (*out)[2]) {
    const int lmax = L - 1;
    const long fsz = 2L * nr;
    const long rsz = (long)NS2AM * fsz;
    auto get2 = [&](int f, int ll) -> double2 {
        if (ll < m || ll >= lmax) return make_double2(0.0, 0.0);
        return __ldg(reinterpret_cast<const double2*>(s2am + row_index(m, ll, L) * rsz + f * fsz + r * 2));
    };
    const double orsq = radial[R_OVER_RSQ * nr + r];
    const double c1 = dth_c1(l, m), c2 = dth_c2(l, m);
    const double llp1 = (double)l * (l + 1);
    const double llm = (double)(l - 1) * l, llq = (double)(l + 1) * (l + 2);
    const double2 C = get2(SM_C, l), A = get2(SM_A, l), C1 = get2(SM_C1, l), A1 = get2(SM_A1, l);
    const double2 C2 = get2(SM_C2, l);
    const double2 Cm = get2(SM_C, l - 1), Cp = get2(SM_C, l + 1), C2m = get2(SM_C2, l - 1), C2p = get2(SM_C2, l + 1);
    const double2 Am = get2(SM_A, l - 1), Ap = get2(SM_A, l + 1), A1m = get2(SM_A1, l - 1), A1p = get2(SM_A1, l + 1);
    const double2 C1m = get2(SM_C1, l - 1), C1p = get2(SM_C1, l + 1);
    auto c = [](double2 v, int ri) { return ri ? v.y : v.x; };
#pragma unroll
    for (int ri = 0; ri < 2; ++ri) {
        const double sg = ri ? (double)m : -(double)m;   // d/dphi: (re, im) -> (-m im, m re)
        const int rj = 1 - ri;
        const double br = llp1 * c(C, ri) * orsq;
        const double xj = c(C2, rj) - llp1 * c(C, rj) * orsq;    // X at l, the other part
        const double xm = c(C2m, ri) - llm * c(Cm, ri) * orsq;   // X at l - 1, l + 1
        const double xp = c(C2p, ri) - llq * c(Cp, ri) * orsq;
        out[0][ri] = br;
        out[1][ri] = llp1 * c(A, ri) * orsq;
        out[2][ri] = (c(A1m, ri) * c1 + c(A1p, ri) * c2) - sg * xj;
        out[3][ri] = sg * c(A1, rj) + (xm * c1 + xp * c2);
        out[4][ri] = sg * c(A, rj) + (c(C1m, ri) * c1 + c(C1p, ri) * c2);
        out[5][ri] = sg * c(C1, rj) - (c(Am, ri) * c1 + c(Ap, ri) * c2);
    }
}

// MAG: the magnetic fields are formed by the same thread (band_curl_b) and stored with the
// hydrodynamic ones, the 17 fields of a radius as one contiguous record.
template <bool MAG>
__global__ void __launch_bounds__(MAG ? 128 : RLM_A_THREADS, MAG ? 3 : 1) rlm_a_kernel(const double* __restrict__ s2a,
                                                             const double* __restrict__ s2am,
                                                             double* __restrict__ s2o,
                                                             const double* __restrict__ radial, long nlm, int nr,
                                                             int L, int nfa) {
    constexpr int NF = MAG ? (int)NP2A_MAG : (int)NP2A;
    constexpr int NT = MAG ? 128 : RLM_A_THREADS;
    __shared__ double2 stage[NT * NF];   // the block's outputs, re-read for coalesced stores
    const long total = nlm * nr;
    const long idx0 = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (row, r)
    const bool valid = idx0 < total;
    const long idx = valid ? idx0 : total - 1;   // tail lanes compute a copy, store nothing
    const int r = (int)(idx % nr);
    int l, m;   // threads run in row order: input and output rows stream, the l +- 1 rows are near
    ml_of_row(idx / nr, L, m, l);
    const int lmax = L - 1;
    const long fsz = 2L * nr;   // one field of one row
    const long rsz = (long)NS2A * fsz;
    // (re, im) of field f at (ll, m, r) in one load
    auto get2 = [&](int f, int ll) -> double2 {
        if (ll < m || ll >= lmax) return make_double2(0.0, 0.0);   // l_max zeroed on entry (Sphere_Hybrid_Space.F90:73-75)
        return __ldg(reinterpret_cast<const double2*>(s2a + row_index(m, ll, L) * rsz + f * fsz + r * 2));
    };
    const double2 cW = get2(S_W, l), cT = get2(S_T, l), cZ = get2(S_Z, l), cW1 = get2(S_W1, l);
    const double2 cT1 = get2(S_T1, l), cZ1 = get2(S_Z1, l), cW2 = get2(S_W2, l);
    const double2 mW = get2(S_W, l - 1), pW = get2(S_W, l + 1), mW1 = get2(S_W1, l - 1), pW1 = get2(S_W1, l + 1);
    const double2 mZ = get2(S_Z, l - 1), pZ = get2(S_Z, l + 1), mW2 = get2(S_W2, l - 1), pW2 = get2(S_W2, l + 1);
    const double2 mZ1 = get2(S_Z1, l - 1), pZ1 = get2(S_Z1, l + 1), mT = get2(S_T, l - 1), pT = get2(S_T, l + 1);
    auto c = [](double2 v, int ri) { return ri ? v.y : v.x; };
    auto get = [&](int f, int ll, int ri) -> double {
        const int dl = ll - l;
        switch (f) {
            case S_W: return c(dl < 0 ? mW : (dl > 0 ? pW : cW), ri);
            case S_T: return c(dl < 0 ? mT : (dl > 0 ? pT : cT), ri);
            case S_Z: return c(dl < 0 ? mZ : (dl > 0 ? pZ : cZ), ri);
            case S_W1: return c(dl < 0 ? mW1 : (dl > 0 ? pW1 : cW1), ri);
            case S_T1: return c(cT1, ri);
            case S_Z1: return c(dl < 0 ? mZ1 : (dl > 0 ? pZ1 : cZ1), ri);
            default: return c(dl < 0 ? mW2 : (dl > 0 ? pW2 : cW2), ri);
        }
    };
    const double orsq = radial[R_OVER_RHORSQ * nr + r];
    const double orr = radial[R_OVER_RHOR * nr + r];
    const double drho = radial[R_DRHO_TERM * nr + r];
    const double two_r = radial[R_TWO_OVER_R * nr + r];
    const double dlnrho = radial[R_DLNRHO * nr + r];
    const double c1 = dth_c1(l, m), c2 = dth_c2(l, m);
    const double llp1 = (double)l * (l + 1);
    const double llm = (double)(l - 1) * l, llq = (double)(l + 1) * (l + 2);
    double out[NF][2];
    if constexpr (MAG) band_curl_b(s2am, radial, nr, L, l, m, r, out + NP2A);
#pragma unroll
    for (int ri = 0; ri < 2; ++ri) {
        const double sg = ri ? (double)m : -(double)m;   // d/dphi: (re, im) -> (-m im, m re)
        const int rj = 1 - ri;
        const double W = get(S_W, l, ri), T = get(S_T, l, ri), Z = get(S_Z, l, ri);
        const double W1 = get(S_W1, l, ri), T1 = get(S_T1, l, ri);
        const double vr = llp1 * W * orsq;
        double dvrdr = llp1 * W1 * orsq;
        dvrdr = dvrdr - vr * two_r;
        dvrdr = dvrdr - vr * dlnrho;
        const double vrm = llm * get(S_W, l - 1, ri) * orsq;
        const double vrp = llq * get(S_W, l + 1, ri) * orsq;
        const double dth_w1 = get(S_W1, l - 1, ri) * c1 + get(S_W1, l + 1, ri) * c2;
        const double dth_z = get(S_Z, l - 1, ri) * c1 + get(S_Z, l + 1, ri) * c2;
        const double dth_w2 = get(S_W2, l - 1, ri) * c1 + get(S_W2, l + 1, ri) * c2;
        const double dth_z1 = get(S_Z1, l - 1, ri) * c1 + get(S_Z1, l + 1, ri) * c2;
        const double vt = (dth_w1 + sg * get(S_Z, l, rj)) * orr;
        const double vp = (sg * get(S_W1, l, rj) - dth_z) * orr;
        double dvtdr = (dth_w2 + sg * get(S_Z1, l, rj)) * orr;
        dvtdr = dvtdr - vt * drho;
        double dvpdr = (sg * get(S_W2, l, rj) - dth_z1) * orr;
        dvpdr = dvpdr - vp * drho;
        out[A_VR][ri] = vr;
        out[A_T][ri] = T;
        out[A_OMR][ri] = llp1 * Z * orsq;
        out[A_DVRDR][ri] = dvrdr;
        out[A_DTDR][ri] = T1;
        out[A_DVRDT][ri] = vrm * c1 + vrp * c2;
        out[A_DTDT][ri] = get(S_T, l - 1, ri) * c1 + get(S_T, l + 1, ri) * c2;
        out[A_VT][ri] = vt;
        out[A_VP][ri] = vp;
        out[A_DVTDR][ri] = dvtdr;
        out[A_DVPDR][ri] = dvpdr;
    }
    const bool zero = (l == lmax);   // Sphere_Hybrid_Space.F90:100-102
    // s2a11[row][r][field][re, im]: a thread's 11 fields are 176 contiguous
    // bytes, and a warp's lanes of one row are contiguous in r.  The warp
    // stages its outputs in shared memory and stores them as consecutive
    // 16-byte chunks, so each store instruction covers a few whole lines.
    const int lane = threadIdx.x & 31;
    double2* st = stage + (threadIdx.x - lane) * NF;
#pragma unroll
    for (int f = 0; f < NF; ++f)
        st[lane * NF + f] = zero ? make_double2(0.0, 0.0) : make_double2(out[f][0], out[f][1]);
    __syncwarp();
    const long obase = row_index(m, l, L) * (long)nfa * fsz + (long)r * (2 * nfa);   // nfa == NF fields per radius
#pragma unroll
    for (int i = 0; i < NF; ++i) {
        const int ci = i * 32 + lane, sl = ci / NF, f = ci - sl * NF;
        const long b = __shfl_sync(0xffffffffu, obase, sl);
        const int ok = __shfl_sync(0xffffffffu, (int)valid, sl);
        if (ok) *reinterpret_cast<double2*>(s2o + b + f * 2) = st[ci];
    }
}

void launch_rlm_a(Ctx& c) {
    const long total = c.d.nlm * c.d.nr;
    if (c.mag) {
        rlm_a_kernel<true><<<(unsigned)((total + 127) / 128), 128, 0, c.stream>>>(
            c.d_s2a, c.d_s2am, c.d_s2a11, c.d_radial, c.d.nlm, c.d.nr, c.d.L, c.nfa);
    } else {
        rlm_a_kernel<false><<<(unsigned)((total + RLM_A_THREADS - 1) / RLM_A_THREADS), RLM_A_THREADS, 0, c.stream>>>(
            c.d_s2a, nullptr, c.d_s2a11, c.d_radial, c.d.nlm, c.d.nr, c.d.L, c.nfa);
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// ---------------------------------------------------------------------------
// rlm_spaceb: curl algebra on the transformed NL terms, written l-major (p1b)
// ---------------------------------------------------------------------------
__global__ void rlm_b_kernel(const double* __restrict__ s2b, double* __restrict__ ab, double* __restrict__ rhs_wpt,
                             double* __restrict__ rhs_z, long nlm, int nr, int L, double new_ab, double bc_top,
                             double bc_bot, const double* __restrict__ bcv, int* __restrict__ status, int nfb) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (lm, r)
    if (idx >= nlm * nr) return;
    const int r = (int)(idx % nr);
    const long lm = idx / nr;
    const int l = ell_of_lm(lm);
    const int m = (int)(lm - (long)l * (l + 1) / 2);
    const int lmax = L - 1;
    const long rsz = 2L * nfb * nr;   // s2b[row][r][field][re, im]
    auto get2 = [&](int f, int ll) -> double2 {
        if (ll < m || ll > lmax) return make_double2(0.0, 0.0);
        return __ldg(reinterpret_cast<const double2*>(s2b + row_index(m, ll, L) * rsz + r * (2 * nfb) + f * 2));
    };
    const double2 cW = get2(0, l), cP = get2(1, l), cT = get2(2, l), cZ = get2(3, l);
    const double2 mP = get2(1, l - 1), pP = get2(1, l + 1), mZ = get2(3, l - 1), pZ = get2(3, l + 1);
    auto get = [&](int f, int ll, int ri) -> double {   // f, ll - l are compile-time after unrolling
        const int dl = ll - l;
        const double2 v = f == 0 ? cW : f == 2 ? cT
                        : f == 1 ? (dl < 0 ? mP : (dl > 0 ? pP : cP))
                                 : (dl < 0 ? mZ : (dl > 0 ? pZ : cZ));
        return ri ? v.y : v.x;
    };
    const double ollp1 = (l > 0) ? 1.0 / ((double)l * (l + 1)) : 1.0;
    const double c1 = sdth_c1(l, m), c2 = sdth_c2(l, m);
    const long plane = nlm * 2 * nr;
    const bool edge = (r == 0 || r == nr - 1);
#pragma unroll
    for (int ri = 0; ri < 2; ++ri) {
        const double sg = ri ? (double)m : -(double)m;
        const int rj = 1 - ri;
        double W = get(0, l, ri) * ollp1;
        const double T = get(2, l, ri);
        const double sd_z = get(3, l - 1, ri) * c1 + get(3, l + 1, ri) * c2;
        const double sd_p = get(1, l - 1, ri) * c1 + get(1, l + 1, ri) * c2;
        const double dphi_p = sg * get(1, l, rj);
        const double dphi_z = sg * get(3, l, rj);
        double Z = (dphi_p - sd_z) * ollp1;
        double P = (sd_p + dphi_z) * ollp1;
        double Tt = T;
        if (l == 0) {   // m = 0 here: W, P and Z of l = 0 carry no RHS (:186-193)
            W = 0.0;
            P = 0.0;
            Z = 0.0;
        }
        if (l == lmax) {   // :205-208
            W = P = Tt = Z = 0.0;
        }
        if (!(isfinite(W) && isfinite(P) && isfinite(Tt) && isfinite(Z))) atomicOr(status, RA_STATUS_NONFINITE);
        const long col = lm * 2 + ri;
        const long o = col * nr + r;
        ab[0 * plane + o] = W;
        ab[1 * plane + o] = P;
        ab[2 * plane + o] = Tt;
        ab[3 * plane + o] = Z;
        // AdvanceTime: Add_To_All_RHS(p1b, new_ab) then Apply_Boundary_Mask
        // (Sphere_Spectral_Space.F90:427-428, Linear_Solve.F90:401-418, 733-754)
        double* rw = rhs_wpt + col * 3L * nr + r;
        if (edge) {
            if (bcv) {   // the caller's bc_values(top/bottom, re/im, lm, equation)
                const double* bv = bcv + (lm * 2 + ri) * 2 + (r == 0 ? 0 : 1);
                rw[0] = bv[0];
                rw[nr] = bv[4 * nlm];
                rw[2 * nr] = bv[8 * nlm];
                rhs_z[o] = bv[12 * nlm];
            } else {
                const double tb = (col == 0) ? (r == 0 ? bc_top : bc_bot) : 0.0;   // only l = 0 T carries a value
                rw[0] = 0.0;
                rw[nr] = 0.0;
                rw[2 * nr] = tb;
                rhs_z[o] = 0.0;
            }
        } else {
            rw[0] += new_ab * W;
            rw[nr] += new_ab * P;
            rw[2 * nr] += new_ab * Tt;
            rhs_z[o] += new_ab * Z;
        }
    }
}

static void bc_values(const Ctx& c, double& top, double& bot) {
    // bc_values for l = 0 T (BoundaryConditions.F90:383-418): sqrt(4 pi) x value
    const double s4pi = std::sqrt(4.0 * M_PI);
    top = (c.cfg.fix_tvar_top ? c.cfg.t_top : c.cfg.dtdr_top) * s4pi;
    bot = (c.cfg.fix_tvar_bottom ? c.cfg.t_bottom : c.cfg.dtdr_bottom) * s4pi;
}

// Diagnostics of the pressure: the P and dP/dr grids g[G_P0], g[G_P1] into the
// T and dT/dr fields of s2a, so that rlm_spacea and the inverse Legendre
// transform form P and dP/dr on the physical grid in the places of T and dT/dr
// (those s2a fields are the grids copied unchanged).
__global__ void pressure_to_s2a_kernel(const double* __restrict__ g, double* __restrict__ s2a, long nlm, int nr,
                                       int L) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (lm, r)
    if (idx >= nlm * nr) return;
    const int r = (int)(idx % nr);
    const long lm = idx / nr;
    const int l = ell_of_lm(lm);
    const int m = (int)(lm - (long)l * (l + 1) / 2);
    const long plane = nlm * 2 * nr;   // g[o][lm][ri][r]
    double* dst = s2a + row_index(m, l, L) * (NS2A * 2L * nr) + S_T * (2L * nr) + 2L * r;
    dst[0] = g[G_P0 * plane + (lm * 2) * nr + r];
    dst[1] = g[G_P0 * plane + (lm * 2 + 1) * nr + r];
    double* dst1 = dst + (S_T1 - S_T) * (2L * nr);
    dst1[0] = g[G_P1 * plane + (lm * 2) * nr + r];
    dst1[1] = g[G_P1 * plane + (lm * 2 + 1) * nr + r];
}

void launch_pressure_to_s2a(Ctx& c) {
    const long total = c.d.nlm * c.d.nr;
    pressure_to_s2a_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(c.d_g, c.d_s2a, c.d.nlm, c.d.nr,
                                                                                   c.d.L);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

void launch_rlm_b(Ctx& c, double new_ab) {
    const long total = c.d.nlm * c.d.nr;
    double top, bot;
    bc_values(c, top, bot);
    rlm_b_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(c.d_s2b, c.d_ab, c.d_rhs_wpt, c.d_rhs_z,
                                                                        c.d.nlm, c.d.nr, c.d.L, new_ab, top, bot,
                                                                        c.d_bcval, c.d_status, c.nfb);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// Adjust_Emf (Sphere_Hybrid_Space.F90:557-602) and the first half of Finalize_EMF: the C
// right-hand side from the radial curl of the EMF,
//   N_C = (sd_theta EMF_phi - d_phi EMF_theta) / l(l+1),
// the A one's EMF_r part, and X = (d_phi EMF_phi + sd_theta EMF_theta) / l(l+1), whose
// radial derivative emf_radial_kernel adds (1 / l(l+1) -> 1 at l = 0, l_max zeroed).
// Then AB history, Add_To_All_RHS and the (zero) magnetic boundary rows for C.
__global__ void rlm_b_mag_kernel(const double* __restrict__ s2b, double* __restrict__ ab,
                                 double* __restrict__ rhs_c, double* __restrict__ xemf, long nlm, int nr, int L,
                                 double new_ab, int nfb, int* __restrict__ status) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (lm, r)
    if (idx >= nlm * nr) return;
    const int r = (int)(idx % nr);
    const long lm = idx / nr;
    const int l = ell_of_lm(lm);
    const int m = (int)(lm - (long)l * (l + 1) / 2);
    const int lmax = L - 1;
    const long rsz = 2L * nfb * nr;
    auto get2 = [&](int f, int ll) -> double2 {
        if (ll < m || ll > lmax) return make_double2(0.0, 0.0);
        return __ldg(reinterpret_cast<const double2*>(s2b + row_index(m, ll, L) * rsz + r * (2 * nfb) + f * 2));
    };
    const double2 et = get2(B_EMFT, l), er = get2(B_EMFR, l), ep = get2(B_EMFP, l);
    const double2 etm = get2(B_EMFT, l - 1), etp = get2(B_EMFT, l + 1);
    const double2 epm = get2(B_EMFP, l - 1), epp = get2(B_EMFP, l + 1);
    auto c = [](double2 v, int ri) { return ri ? v.y : v.x; };
    const double ollp1 = (l > 0) ? 1.0 / ((double)l * (l + 1)) : 1.0;
    const double c1 = sdth_c1(l, m), c2 = sdth_c2(l, m);
    const long plane = nlm * 2 * nr;
    const bool edge = (r == 0 || r == nr - 1);
#pragma unroll
    for (int ri = 0; ri < 2; ++ri) {
        const double sg = ri ? (double)m : -(double)m;
        const int rj = 1 - ri;
        double nc = ((c(epm, ri) * c1 + c(epp, ri) * c2) - sg * c(et, rj)) * ollp1;
        double x = (sg * c(ep, rj) + (c(etm, ri) * c1 + c(etp, ri) * c2)) * ollp1;
        double na = c(er, ri);
        if (l == lmax) nc = x = na = 0.0;
        if (!(isfinite(nc) && isfinite(x) && isfinite(na))) atomicOr(status, RA_STATUS_NONFINITE);
        const long o = (lm * 2 + ri) * nr + r;
        ab[4 * plane + o] = nc;
        ab[5 * plane + o] = na;   // emf_radial_kernel adds d/dr X
        xemf[o] = x;
        rhs_c[o] = edge ? 0.0 : rhs_c[o] + new_ab * nc;
    }
}

// Finalize_EMF's radial derivative (Sphere_Spectral_Space.F90:436-488) as one product with
// the grid operator M (to_spectral, d/dr, dealias, from_spectral): N_A = EMF_r + M X per
// (l, m, re/im) column, on the FP64 tensor-core tile engine; then the A history, the A
// right-hand side and its (zero) boundary rows.
__global__ void __launch_bounds__(GEMM_THREADS, 4) emf_radial_kernel(const double* __restrict__ M,
                                                                  const double* __restrict__ xemf,
                                                                  double* __restrict__ ab_a,
                                                                  double* __restrict__ rhs_a, int nr, long ncols,
                                                                  double new_ab) {
    __shared__ GemmSmem sm;
    const int r0 = blockIdx.y * Sq::BM;
    const long c0 = (long)blockIdx.x * Sq::BN;
    auto fa = [&](int k, int x) -> double {   // M(r0 + x, k)
        const int rr = r0 + x;
        return (k < nr && rr < nr) ? __ldg(M + (long)rr * nr + k) : 0.0;
    };
    auto fb = [&](int k, int y) -> double {   // X(k, c0 + y)
        const long col = c0 + y;
        return (k < nr && col < ncols) ? __ldg(xemf + col * nr + k) : 0.0;
    };
    Acc acc;
    acc.zero();
    gemm_tile<false, false>(acc, fa, fb, nr, sm);
    acc_foreach(acc, [&](int x, int y, double v) {
        const int rr = r0 + x;
        const long col = c0 + y;
        if (rr < nr && col < ncols) {
            const long o = col * nr + rr;
            const double na = ab_a[o] + v;
            ab_a[o] = na;
            rhs_a[o] = (rr == 0 || rr == nr - 1) ? 0.0 : rhs_a[o] + new_ab * na;
        }
    });
}

// The same in the finite-difference mode, where the grid operator is D_1 (Finalize_EMF's FD
// branch): its band (operator 1 of the synthesis bands) per point, one thread per point with
// r fastest, and the same epilogue.
__global__ void __launch_bounds__(256) emf_band_kernel(const double* __restrict__ band, int w,
                                                       const double* __restrict__ xemf, double* __restrict__ ab_a,
                                                       double* __restrict__ rhs_a, int nr, long ncols,
                                                       double new_ab) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (column, r), r fastest
    if (i >= ncols * nr) return;
    const long col = i / nr;
    const int rr = (int)(i - col * nr);
    const double* row = band + ((long)nr + rr) * (w + 1);
    const int first = (int)__ldg(row);   // first + w <= nr
    const double* x = xemf + col * nr + first;
    double v = 0.0;
    for (int j = 0; j < w; ++j) v += __ldg(row + 1 + j) * __ldg(x + j);
    const double na = ab_a[i] + v;
    ab_a[i] = na;
    rhs_a[i] = (rr == 0 || rr == nr - 1) ? 0.0 : rhs_a[i] + new_ab * na;
}

void launch_rlm_b_mag(Ctx& c, double new_ab) {
    const long total = c.d.nlm * c.d.nr;
    rlm_b_mag_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(
        c.d_s2b, c.d_ab, c.d_rhs_c, c.d_xemf, c.d.nlm, c.d.nr, c.d.L, new_ab, c.nfb, c.d_status);
    RA_CUDA(cudaGetLastError());
    const long ncols = 2 * c.d.nlm;
    double* ab_a = c.d_ab + 5 * c.d.nlm * 2 * c.d.nr;
    if (c.cfg.chebyshev) {
        dim3 grid((unsigned)((ncols + Sq::BN - 1) / Sq::BN), (unsigned)((c.d.nr + Sq::BM - 1) / Sq::BM));
        emf_radial_kernel<<<grid, GEMM_THREADS, 0, c.stream>>>(c.d_Memf, c.d_xemf, ab_a, c.d_rhs_a, c.d.nr, ncols,
                                                             new_ab);
    } else {
        const long total = ncols * c.d.nr;
        emf_band_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(c.d_Dfd, c.fd_w, c.d_xemf, ab_a,
                                                                             c.d_rhs_a, c.d.nr, ncols, new_ab);
    }
    RA_CUDA(cudaGetLastError());
    c.launches += 2;
}

}  // namespace ra
