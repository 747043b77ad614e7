// Legendre path: P_l^m table generation and the two Legendre transforms.
//
//  * plm_kernel  restates Compute_Plms + Parity_Resort
//    (src/Math_Layer/Legendre_Polynomials.F90:146-331) in double-double
//    arithmetic (the reference computes in REAL*16) with a carried binary
//    exponent for the sin^m(theta) underflow.
//  * lt_inverse_kernel restates StP_4d_dgp2 (Legendre_Transforms.F90:968-1074):
//    per m, an even-l and an odd-l product, then the equatorial mirror
//    (south = e + o, north = e - o).
//  * lt_forward_kernel restates PtS_4d_dgpv3 (Legendre_Transforms.F90:1077-1175):
//    equatorial fold (f_even = s + n, f_odd = s - n) in the operand load, then
//    the per-parity product with the weighted tables.
//  All m share one launch; K (the number of l of one parity) is ragged and the
//  grid is ordered by m so that the long products start first.
#include "ra_internal.h"
#include "gemm_f64.cuh"

namespace ra {

// Double-double arithmetic (an unevaluated sum hi + lo, |lo| <= ulp(hi)/2, about
// 106 significant bits) for the table recurrence, so that the tables come out
// correctly rounded from a computation at least as precise as the reference's
// REAL*16 one.  Error-free transformations: Knuth's two-sum, the FMA two-product.
struct dd {
    double hi, lo;
};
__device__ __forceinline__ dd dd_two_sum(double a, double b) {
    const double s = a + b, bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ dd dd_fast(double a, double b) {   // |a| >= |b|
    const double s = a + b;
    return {s, b - (s - a)};
}
__device__ __forceinline__ dd dd_mul(dd a, dd b) {
    const double p = a.hi * b.hi;
    const double e = fma(a.hi, b.hi, -p) + (a.hi * b.lo + a.lo * b.hi);
    return dd_fast(p, e);
}
__device__ __forceinline__ dd dd_mul_d(dd a, double b) {
    const double p = a.hi * b;
    return dd_fast(p, fma(a.hi, b, -p) + a.lo * b);
}
__device__ __forceinline__ dd dd_sub(dd a, dd b) {
    dd s = dd_two_sum(a.hi, -b.hi);
    const dd t = dd_two_sum(a.lo, -b.lo);
    s = dd_fast(s.hi, s.lo + t.hi);
    return dd_fast(s.hi, s.lo + t.lo);
}
__device__ __forceinline__ dd dd_div(dd a, dd b) {
    const double q1 = a.hi / b.hi;
    const dd r = dd_sub(a, dd_mul_d(b, q1));
    const double q2 = r.hi / b.hi;
    const dd r2 = dd_sub(r, dd_mul_d(b, q2));
    return dd_fast(dd_fast(q1, q2).hi, dd_fast(q1, q2).lo + r2.hi / b.hi);
}
// n / d for integers exactly representable in double
__device__ __forceinline__ dd dd_ratio(double n, double d) { return dd_div(dd{n, 0.0}, dd{d, 0.0}); }
__device__ __forceinline__ dd dd_sqrt(dd a) {
    const double s = sqrt(a.hi);
    const double e = fma(-s, s, a.hi);   // a.hi - s^2, exact
    return dd_fast(s, (e + a.lo) / (2.0 * s));
}

// Compute_Plms + Parity_Resort in double-double: P_m^m from its closed form
// (Legendre_Polynomials.F90:190-212), the three-term recurrence in l
// (:215-226), the normalisations 1 / 1/2 (p_lm) and 2 pi w times the
// double-precision constants 1/(2 N_theta), 1/N_theta (ip_lm, :270-276); a
// carried binary exponent keeps sin^m(theta) from underflowing.  x, s = sin,
// and 2 pi w come as hi/lo pairs made from the host's long-double values.
__global__ void plm_kernel(const double* __restrict__ xhl, const double* __restrict__ shl,
                           const double* __restrict__ whl, int L, int nth, double* __restrict__ Ptab,
                           double* __restrict__ iPtab) {
    const int nth2 = nth / 2;
    const int th = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (th >= nth2 || m >= L) return;
    const int lmax = L - 1;
    const dd xv{xhl[th], xhl[nth2 + th]}, sv{shl[th], shl[nth2 + th]}, wt{whl[th], whl[nth2 + th]};
    const double stp = (m == 0) ? 1.0 : 0.5;
    const double pts = (m == 0) ? 1.0 / (2.0 * nth) : 1.0 / (double)nth;   // double-precision constants
    const double TWO600 = 0x1p600, TWOM600 = 0x1p-600;
    const dd twopi{6.283185307179586232e+00, 2.449293598294706414e-16};
    // P_m^m = (-1)^m sqrt((m+1/2)/(2 pi)) prod_{i<=m} sqrt((i-1/2)/i) sin^m(theta)
    dd p = dd_sqrt(dd_div(dd{m + 0.5, 0.0}, twopi));
    int e = 0;
    for (int i = 1; i <= m; ++i) {
        p = dd_mul(dd_mul(p, dd_sqrt(dd_ratio(2.0 * i - 1.0, 2.0 * i))), sv);
        if (fabs(p.hi) < TWOM600) {
            p.hi *= TWO600;
            p.lo *= TWO600;
            e -= 600;
        }
    }
    if (m & 1) p = dd{-p.hi, -p.lo};
    auto store = [&](int l, dd v) {
        const long row = row_index(m, l, L);
        Ptab[row * nth2 + th] = ldexp(v.hi, e) * stp;
        const dd vw = dd_mul_d(dd_mul(v, wt), pts);
        iPtab[row * nth2 + th] = ldexp(vw.hi, e);
    };
    store(m, p);
    if (m == lmax) return;
    dd p1 = dd_mul(dd_mul(p, xv), dd_sqrt(dd{2.0 * m + 3.0, 0.0}));   // P_{m+1}^m
    dd p0 = p;
    store(m + 1, p1);
    for (int l = m + 2; l <= lmax; ++l) {
        const double lm1 = (double)(l - 1);
        const dd a = dd_sqrt(dd_ratio(lm1 * lm1 - (double)m * m, 4.0 * lm1 * lm1 - 1.0));
        const dd t = dd_sub(dd_mul(p1, xv), dd_mul(a, p0));
        const dd b = dd_sqrt(dd_ratio(4.0 * (double)l * l - 1.0, (double)l * l - (double)m * m));
        const dd pn = dd_mul(t, b);
        p0 = p1;
        p1 = pn;
        if (e < 0 && fabs(p1.hi) > TWO600) {
            p1.hi *= TWOM600;
            p1.lo *= TWOM600;
            p0.hi *= TWOM600;
            p0.lo *= TWOM600;
            e += 600;
        }
        store(l, p1);
    }
}

void launch_plm(Ctx& c, const double* d_x, const double* d_w) {
    // d_x holds [x hi | x lo | s hi | s lo] (nth2 each); d_w holds [2 pi w hi | lo]
    const int nth2 = c.d.nth2;
    dim3 grid((nth2 + 127) / 128, c.d.L);
    plm_kernel<<<grid, 128, 0, c.stream>>>(d_x, d_x + 2 * nth2, d_w, c.d.L, c.d.nth, c.d_Ptab, c.d_iPtab);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// ---------------------------------------------------------------------------
// Inverse transform, per (m, parity):
//   p2[theta_h][m][par][col] = sum_l P_par(l, theta_h) s2[row(m, l)][col]
// (E for par = 0, O for par = 1; the physical-space kernel forms E +- O).
// theta_h is the slowest index so that the physical-space kernel, which reads
// every (m, parity) of one theta_h, touches one contiguous block.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(GEMM_THREADS) lt_inverse_kernel(const double* __restrict__ Ptab,
                                                                  const double* __restrict__ s2,
                                                                  double* __restrict__ p2, int L, int nth,
                                                                  int ncol) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GemmSmem& sm = *reinterpret_cast<GemmSmem*>(smem_raw);
    const int m = blockIdx.z >> 1, par = blockIdx.z & 1;
    const int th0 = blockIdx.y * BM;
    const int c0 = blockIdx.x * BN;
    const int nth2 = nth / 2;
    const int ne = n_even(m, L);
    const int nl = par ? n_odd(m, L) : ne;
    const long roff = m_off(m, L) + (par ? ne : 0);
    const double* pa = Ptab + roff * nth2;
    const double* pb = s2 + roff * ncol;
    Acc acc;
    acc.zero();
    auto fa = [&](int k, int x) -> double {
        const int th = th0 + x;
        return (k < nl && th < nth2) ? __ldg(pa + (long)k * nth2 + th) : 0.0;
    };
    auto fb = [&](int k, int y) -> double {
        const int col = c0 + y;
        return (k < nl && col < ncol) ? __ldg(pb + (long)k * ncol + col) : 0.0;
    };
    gemm_tile<true, true>(acc, fa, fb, nl, sm);
    double* out = p2 + (long)blockIdx.z * ncol;
    const long th_stride = 2L * L * ncol;
    acc_foreach(acc, [&](int x, int y, double v) {
        const int th = th0 + x, col = c0 + y;
        if (th < nth2 && col < ncol) out[(long)th * th_stride + col] = v;
    });
}

void launch_lt_inverse(Ctx& c, const double* s2, double* p2, int ncol) {
    dim3 grid((ncol + BN - 1) / BN, (c.d.nth2 + BM - 1) / BM, 2 * c.d.L);
    lt_inverse_kernel<<<grid, GEMM_THREADS, sizeof(GemmSmem), c.stream>>>(c.d_Ptab, s2, p2, c.d.L, c.d.nth, ncol);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// ---------------------------------------------------------------------------
// Forward transform, per (m, parity), on the equatorially folded input
// p2[m][par][theta_h][col] (f_even, f_odd):
//   s2[row(m, l)][col] = sum_th iP_par(l, th) p2[m][par][th][col]
// tiles: (m, parity, l-tile) in descending-K order
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(GEMM_THREADS) lt_forward_kernel(const double* __restrict__ iPtab,
                                                                  const double* __restrict__ p2,
                                                                  double* __restrict__ s2,
                                                                  const int4* __restrict__ tiles, int L,
                                                                  int nth, int ncol) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GemmSmem& sm = *reinterpret_cast<GemmSmem*>(smem_raw);
    const int4 tl = tiles[blockIdx.y];
    const int m = tl.x, par = tl.y, l0 = tl.z * BM;
    const int c0 = blockIdx.x * BN;
    const int nth2 = nth / 2;
    const int ne = n_even(m, L);
    const int nl = par ? n_odd(m, L) : ne;
    const long roff = m_off(m, L) + (par ? ne : 0) + l0;
    const double* pa = iPtab + roff * nth2;
    const double* pm = p2 + ((long)m * 2 + par) * nth2 * ncol;
    Acc acc;
    acc.zero();
    auto fa = [&](int k, int x) -> double {
        return (l0 + x < nl && k < nth2) ? __ldg(pa + (long)x * nth2 + k) : 0.0;
    };
    auto fb = [&](int k, int y) -> double {
        const int col = c0 + y;
        return (k < nth2 && col < ncol) ? __ldg(pm + (long)k * ncol + col) : 0.0;
    };
    gemm_tile<false, true>(acc, fa, fb, nth2, sm);
    double* out = s2 + roff * ncol;
    acc_foreach(acc, [&](int x, int y, double v) {
        const int col = c0 + y;
        if (l0 + x < nl && col < ncol) out[(long)x * ncol + col] = v;
    });
}

static std::vector<int> forward_tiles(int L) {
    std::vector<int> t;
    for (int m = 0; m < L; ++m) {
        for (int par = 0; par < 2; ++par) {
            const int nl = par ? n_odd(m, L) : n_even(m, L);
            for (int lt = 0; lt * BM < nl; ++lt) {
                t.push_back(m);
                t.push_back(par);
                t.push_back(lt);
                t.push_back(0);
            }
        }
    }
    return t;
}

// The forward transform's tile list, built once at set-up (no allocation may
// run while the step is captured into a graph).
void lt_forward_prepare(Ctx& c) {
    if (!c.d_fwd_tiles) {
        std::vector<int> t = forward_tiles(c.d.L);
        c.n_fwd_tiles = (int)(t.size() / 4);
        RA_CUDA(cudaMalloc(&c.d_fwd_tiles, t.size() * sizeof(int)));
        RA_CUDA(cudaMemcpy(c.d_fwd_tiles, t.data(), t.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
}

void launch_lt_forward(Ctx& c, const double* p2, double* s2, int ncol) {
    if (!c.d_fwd_tiles) throw ArgError("forward-transform tiles not prepared (lt_forward_prepare runs at set-up)");
    dim3 grid((ncol + BN - 1) / BN, c.n_fwd_tiles);
    lt_forward_kernel<<<grid, GEMM_THREADS, sizeof(GemmSmem), c.stream>>>(
        c.d_iPtab, p2, s2, reinterpret_cast<const int4*>(c.d_fwd_tiles), c.d.L, c.d.nth, ncol);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

}  // namespace ra
