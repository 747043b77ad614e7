// Per-l implicit solves on the device: LU_Decompose_full (DGETRF) and
// LU_Solve_full (DGETRS) of Linear_Solve.F90:1028-1036, 1088-1110, called by
// LU_Decompose_Matrices (:459-480) and Implicit_Solve (:423-457).
//
//   lu_factor_kernel    DGETRF: blocked right-looking LU with partial (row)
//                       pivoting, one CTA per matrix; 32-column panels are
//                       factored in shared memory, the trailing matrix is
//                       updated in 128-column chunks (FP64 FMA, 8 x 4
//                       register tiles); pivot ties go to the first row (as
//                       IDAMAX), a zero or non-finite pivot marks the
//                       matrix singular (DGETRF's INFO > 0).  A threshold
//                       relative to |A| is not used: the anelastic matrices
//                       in cgs units (the Jones et al. benchmark polytrope)
//                       have pivots below n 2^-53 of their largest entries,
//                       even after row and column equilibration, and LAPACK
//                       factors and solves them.
//   lu_diag_inv_kernel  the factors rewritten for block substitution with
//   lu_offdiag_kernel   64-row blocks: M_ij = -L_ii^-1 L_ij (j < i),
//                       M_ij = -U_ii^-1 U_ij (j > i), M_ii = L_ii^-1 (strictly
//                       lower part, unit diagonal implied) + U_ii^-1 (upper
//                       part).  Then y_i = L_ii^-1 (Pb)_i + sum_{j<i} M_ij y_j
//                       and x_i = U_ii^-1 y_i + sum_{j>i} M_ij x_j are plain
//                       products, and the substitution runs on the tensor cores.
//   lu_solve_kernel     DGETRS: one CTA per (system, l, NC right-hand-side
//                       columns); the permuted columns stay in shared memory
//                       for both sweeps, the rows of M stream through a
//                       3-stage cp.async ring, and every block product is an
//                       FP64 tensor-core product (mma.sync.m8n8k4.f64).
//   lu_refine_kernel    FP32 block substitution (the same M rounded to FP32)
//                       with FP64 residuals b - A x, iterated until the update
//                       reaches the rounding level of the solution or stops
//                       shrinking (iterative refinement), one CTA per (l,
//                       column tile) in one launch.
//
// The block substitution differs from DGETRS only in the order of the
// roundings: for the per-l matrices of the headline radial size (N_r = 192,
// condition numbers up to ~1e11) it agrees with LAPACK's DGETRS to ~1e-14
// per field after ten steps, where the explicit inverse A^-1 b loses 3e-11.
#include <algorithm>
#include <vector>

#include "ra_internal.h"

namespace ra {

// ---------------------------------------------------------------------------
// Factorisation
// ---------------------------------------------------------------------------
constexpr int LU_THREADS = 256;
constexpr int LU_CW = 128;   // trailing-update column chunk

template <int PW>
struct LuFactorSmem {
    static constexpr int PS = PW + 1;   // odd row stride: column walks of the panel are conflict-free
    static size_t bytes(int n) { return ((size_t)n * PS + (size_t)PW * LU_CW) * sizeof(double); }
};

__device__ __forceinline__ void block_max_index(double& v, int& idx, double* red_v, int* red_i) {
    // max |value|, ties to the smallest index (IDAMAX); NaN never wins
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, v, o);
        const int oi = __shfl_down_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) {
            v = ov;
            idx = oi;
        }
    }
    if (lane == 0) {
        red_v[w] = v;
        red_i[w] = idx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q)
            if (red_v[q] > red_v[0] || (red_v[q] == red_v[0] && red_i[q] < red_i[0])) {
                red_v[0] = red_v[q];
                red_i[0] = red_i[q];
            }
    }
    __syncthreads();
    v = red_v[0];
    idx = red_i[0];
}

template <int PW>
__global__ void __launch_bounds__(LU_THREADS) lu_factor_kernel(double* __restrict__ mats, int n,
                                                               const int* __restrict__ skip, int* __restrict__ perm_all,
                                                               int* __restrict__ status) {
    constexpr int PS = LuFactorSmem<PW>::PS;
    extern __shared__ __align__(16) double fsm[];
    double* P = fsm;                    // panel rows k0 .. n-1, [pr][PS]
    double* U = fsm + (size_t)n * PS;   // U12 chunk [PW][LU_CW]
    __shared__ double red_v[LU_THREADS / 32];
    __shared__ int red_i[LU_THREADS / 32];
    __shared__ int s_piv[PW];
    __shared__ int s_bad;
    const int mat = blockIdx.x, t = threadIdx.x;
    double* A = mats + (size_t)mat * n * n;
    int* perm = perm_all + (size_t)mat * n;
    if (skip && skip[mat]) {   // an equation not solved for this l: identity
        for (long e = t; e < (long)n * n; e += LU_THREADS) A[e] = (e / n == e % n) ? 1.0 : 0.0;
        for (int i = t; i < n; i += LU_THREADS) perm[i] = i;
        if (t == 0) status[mat] = 0;
        return;
    }
    for (int i = t; i < n; i += LU_THREADS) perm[i] = i;
    if (t == 0) s_bad = 0;
    __syncthreads();
    for (int k0 = 0; k0 < n; k0 += PW) {
        const int pw = min(PW, n - k0), pr = n - k0;
        for (int e = t; e < pr * PW; e += LU_THREADS) {
            const int i = e / PW, j = e % PW;
            P[i * PS + j] = (j < pw) ? A[(size_t)(k0 + i) * n + k0 + j] : 0.0;
        }
        __syncthreads();
        // ---- panel: unblocked LU of rows k0.., columns k0 .. k0+pw-1 ----
        for (int j = 0; j < pw; ++j) {
            double bv = -1.0;
            int bi = 0x7fffffff;
            for (int i = j + t; i < pr; i += LU_THREADS) {
                const double v = fabs(P[i * PS + j]);
                if (v > bv) {
                    bv = v;
                    bi = i;
                }
            }
            block_max_index(bv, bi, red_v, red_i);
            if (!(bv > 0.0)) {   // zero or NaN pivot
                if (t == 0) s_bad = 1;
                break;
            }
            if (t == 0) s_piv[j] = bi;
            if (bi != j && t < PW) {
                const double a = P[j * PS + t];
                P[j * PS + t] = P[bi * PS + t];
                P[bi * PS + t] = a;
            }
            __syncthreads();
            const double rinv = 1.0 / P[j * PS + j];
            for (int i = j + 1 + t; i < pr; i += LU_THREADS) {
                const double lij = P[i * PS + j] * rinv;
                P[i * PS + j] = lij;
                for (int q = j + 1; q < pw; ++q) P[i * PS + q] = fma(-lij, P[j * PS + q], P[i * PS + q]);
            }
            __syncthreads();
        }
        __syncthreads();
        if (s_bad) break;
        for (int e = t; e < pr * pw; e += LU_THREADS) {
            const int i = e / pw, j = e % pw;
            A[(size_t)(k0 + i) * n + k0 + j] = P[i * PS + j];
        }
        // ---- the panel's row interchanges on the other columns, then U12 = L11^-1 A12 ----
        for (int c = t; c < n; c += LU_THREADS) {   // one thread per column: no two threads touch one element
            if (c >= k0 && c < k0 + pw) continue;
            for (int j = 0; j < pw; ++j) {
                const int p = s_piv[j];
                if (p != j) {
                    double* x = A + (size_t)(k0 + j) * n + c;
                    double* y = A + (size_t)(k0 + p) * n + c;
                    const double tmp = *x;
                    *x = *y;
                    *y = tmp;
                }
            }
            if (c >= k0 + pw) {
                double u[PW];
#pragma unroll
                for (int j = 0; j < PW; ++j) u[j] = (j < pw) ? A[(size_t)(k0 + j) * n + c] : 0.0;
#pragma unroll
                for (int j = 1; j < PW; ++j) {
                    double s = u[j];
#pragma unroll
                    for (int q = 0; q < j; ++q) s = fma(-P[j * PS + q], u[q], s);
                    u[j] = s;
                }
#pragma unroll
                for (int j = 0; j < PW; ++j)
                    if (j < pw) A[(size_t)(k0 + j) * n + c] = u[j];
            }
        }
        if (t == 0)
            for (int j = 0; j < pw; ++j) {
                const int p = k0 + s_piv[j];
                const int a = perm[k0 + j];
                perm[k0 + j] = perm[p];
                perm[p] = a;
            }
        __syncthreads();
        // ---- trailing update A22 -= L21 U12 ----
        const int r0 = pw;   // first panel row below the diagonal block
        for (int cb = k0 + pw; cb < n; cb += LU_CW) {
            const int cw = min(LU_CW, n - cb);
            for (int e = t; e < PW * LU_CW; e += LU_THREADS) {
                const int q = e / LU_CW, cc = e % LU_CW;
                U[e] = (q < pw && cc < cw) ? A[(size_t)(k0 + q) * n + cb + cc] : 0.0;
            }
            __syncthreads();
            const int cg = t & 31, rg = t >> 5;   // 4 columns cg + 32 s, 8 rows per pass
            for (int ib = r0 + rg * 8; ib < pr; ib += 8 * (LU_THREADS / 32)) {
                double acc[8][4];
#pragma unroll
                for (int r = 0; r < 8; ++r)
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        const int i = ib + r, cc = cg + 32 * s;
                        acc[r][s] = (i < pr && cc < cw) ? A[(size_t)(k0 + i) * n + cb + cc] : 0.0;
                    }
                for (int q = 0; q < pw; ++q) {
                    double a[8], b[4];
#pragma unroll
                    for (int r = 0; r < 8; ++r) a[r] = (ib + r < pr) ? P[(ib + r) * PS + q] : 0.0;
#pragma unroll
                    for (int s = 0; s < 4; ++s) b[s] = U[q * LU_CW + cg + 32 * s];
#pragma unroll
                    for (int r = 0; r < 8; ++r)
#pragma unroll
                        for (int s = 0; s < 4; ++s) acc[r][s] = fma(-a[r], b[s], acc[r][s]);
                }
#pragma unroll
                for (int r = 0; r < 8; ++r)
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        const int i = ib + r, cc = cg + 32 * s;
                        if (i < pr && cc < cw) A[(size_t)(k0 + i) * n + cb + cc] = acc[r][s];
                    }
            }
            __syncthreads();
        }
    }
    if (t == 0) status[mat] = s_bad;
}

// ---------------------------------------------------------------------------
// Block-substitution form of the factors
// ---------------------------------------------------------------------------
constexpr int SB = 64;         // block rows of the substitution
constexpr int SBP = SB + 1;    // padded shared row stride

// Inverses of the diagonal blocks: W[mat][ib][0] = L_ii^-1, W[mat][ib][1] = U_ii^-1 (64 x 64 each).
__global__ void __launch_bounds__(128) lu_diag_inv_kernel(const double* __restrict__ mats, int n,
                                                          double* __restrict__ W) {
    extern __shared__ __align__(16) double dsm[];
    double* D = dsm;                 // [SB][SBP]
    double* Li = D + SB * SBP;
    double* Ui = Li + SB * SBP;
    const int mat = blockIdx.x, ib = blockIdx.y, t = threadIdx.x;
    const int nblk = (n + SB - 1) / SB, i0 = ib * SB, bs = min(SB, n - i0);
    const double* A = mats + (size_t)mat * n * n;
    for (int e = t; e < SB * SB; e += blockDim.x) {
        const int r = e / SB, c = e % SB;
        D[r * SBP + c] = (r < bs && c < bs) ? A[(size_t)(i0 + r) * n + i0 + c] : (r == c ? 1.0 : 0.0);
        Li[r * SBP + c] = 0.0;
        Ui[r * SBP + c] = 0.0;
    }
    __syncthreads();
    if (t < SB) {          // column t of L^-1 (unit lower): x_r = [r == t] - sum_{q<r} L(r, q) x_q
        const int c = t;
        for (int r = 0; r < SB; ++r) {
            double s = (r == c) ? 1.0 : 0.0;
            for (int q = 0; q < r; ++q) s = fma(-D[r * SBP + q], Li[q * SBP + c], s);
            Li[r * SBP + c] = (r >= c) ? s : 0.0;
        }
    } else {               // column t - 64 of U^-1: x_r = ([r == c] - sum_{q>r} U(r, q) x_q) / U(r, r)
        const int c = t - SB;
        for (int r = SB - 1; r >= 0; --r) {
            double s = (r == c) ? 1.0 : 0.0;
            for (int q = r + 1; q < SB; ++q) s = fma(-D[r * SBP + q], Ui[q * SBP + c], s);
            Ui[r * SBP + c] = (r <= c) ? s / D[r * SBP + r] : 0.0;
        }
    }
    __syncthreads();
    double* out = W + ((size_t)mat * nblk + ib) * 2 * SB * SB;
    for (int e = t; e < SB * SB; e += blockDim.x) {
        const int r = e / SB, c = e % SB;
        out[e] = Li[r * SBP + c];
        out[SB * SB + e] = Ui[r * SBP + c];
    }
}

// M_ij = -inv_i X_ij for j != i (X from the factors, in place), packed diagonal blocks for j == i.
__global__ void __launch_bounds__(256) lu_offdiag_kernel(double* __restrict__ mats, int n,
                                                         const double* __restrict__ W) {
    extern __shared__ __align__(16) double osm[];
    double* Iv = osm;              // [SB][SBP]
    double* X = osm + SB * SBP;    // [SB][SBP]
    const int mat = blockIdx.x, ib = blockIdx.y, jb = blockIdx.z, t = threadIdx.x;
    const int nblk = (n + SB - 1) / SB;
    const int i0 = ib * SB, j0 = jb * SB, bi = min(SB, n - i0), bj = min(SB, n - j0);
    double* A = mats + (size_t)mat * n * n;
    const double* w = W + ((size_t)mat * nblk + ib) * 2 * SB * SB;
    if (ib == jb) {
        for (int e = t; e < bi * bi; e += blockDim.x) {
            const int r = e / bi, c = e % bi;
            A[(size_t)(i0 + r) * n + i0 + c] = (c < r) ? w[r * SB + c] : w[SB * SB + r * SB + c];
        }
        return;
    }
    const double* inv = w + (jb < ib ? 0 : SB * SB);
    for (int e = t; e < SB * SB; e += blockDim.x) {
        const int r = e / SB, c = e % SB;
        Iv[r * SBP + c] = inv[e];
        X[r * SBP + c] = (r < bi && c < bj) ? A[(size_t)(i0 + r) * n + j0 + c] : 0.0;
    }
    __syncthreads();
    const int tr = t >> 4, tc = t & 15;
    double acc[4][4] = {};
    for (int q = 0; q < SB; ++q) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = Iv[(tr * 4 + i) * SBP + q];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = X[q * SBP + tc * 4 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = tr * 4 + i, c = tc * 4 + j;
            if (r < bi && c < bj) A[(size_t)(i0 + r) * n + j0 + c] = -acc[i][j];
        }
}

// ---------------------------------------------------------------------------
// Block substitution (DGETRS)
// ---------------------------------------------------------------------------
// One CTA per (system, l, NC right-hand-side columns), 8 warps.  The CTA's
// columns (P b) sit in shared memory for both sweeps.  For block row i the
// product over its K range is split between two warp groups (K chunks of 16
// dealt alternately); warp w owns rows 16 (w mod 4) .. +16 of the block row and
// all NC columns (2 x NC/8 tensor-core tiles, 2 NC/8 x 2 mma per k-step), and
// streams ITS OWN rows of M through a private 3-stage cp.async ring, so no
// CTA-wide barrier is needed until the block row ends: the second group then
// hands its partial sums to the first through shared memory, which writes the
// block row's result over its right-hand side.
constexpr int LS_KC = 16;                 // K per chunk
constexpr int LS_RS = LS_KC + 4;          // ring row stride (doubles): conflict-free A fragments
constexpr int LS_STAGES = 3;
constexpr int LS_WARPS = 8, LS_THREADS = 32 * LS_WARPS;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// The column block in shared memory, [row][NC] with the columns of row i
// permuted by XOR with h(i) = 8 (i mod 2) + (i/2 mod 8): over a warp, a B
// fragment (rows k..k+3, k = 0 mod 4, 8 columns) and a walk down 32
// consecutive rows of one column both touch every 8-byte bank exactly twice.
// (A layout that is also conflict-free per half warp, h(i) = 4 (i mod 4) +
// (i/4 mod 4), measured 35 % slower: 0.92 against 0.68 ms at l_max = 127,
// N_r = 192, with a third of the shared wavefronts.)
template <int NC>
__device__ __forceinline__ int xs_index(int i, int c) {
    return i * NC + (c ^ (((i & 1) << 3) | ((i >> 1) & 7)));
}

// chunk j of block row ib (both sweeps): K start
__device__ __forceinline__ int chunk_k0(bool backward, int ib, int j) {
    return backward ? ib * SB + j * LS_KC : j * LS_KC;
}

template <int NC>
struct LuSolveShape {
    static size_t smem(int n) {
        const int nrow = (n + SB - 1) / SB * SB;
        return ((size_t)nrow * NC + (size_t)LS_WARPS * LS_STAGES * 16 * LS_RS + (size_t)SB * NC) * sizeof(double);
    }
};

template <int NC>
__global__ void __launch_bounds__(LS_THREADS) lu_solve_kernel(const int4* __restrict__ tiles, LuSys S, int mode,
                                                              int ncols_fixed) {
    constexpr int NT = NC / 8;               // n-tiles per warp
    extern __shared__ __align__(16) double ssm[];
    const int4 tl = tiles[blockIdx.x];
    const int l = tl.y, c0 = tl.z * NC, n = S.n;
    const int nblk = (n + SB - 1) / SB, nrow = nblk * SB;
    double* Xs = ssm;                                      // [nrow][NC]
    double* ring_all = Xs + (size_t)nrow * NC;             // [warp][stage][16][LS_RS]
    double* red = ring_all + LS_WARPS * LS_STAGES * 16 * LS_RS;   // [SB][NC] second group's partial sums
    const double* M = S.M + (size_t)l * n * n;
    const int* perm = S.perm + (size_t)l * n;
    const double* rhs = nullptr;
    double* sol;
    int ncol;
    if (mode == LU_MODE_STEP) {
        const long lstart = (long)l * (l + 1) / 2;
        rhs = S.rhs + 2 * lstart * n;
        sol = S.sol + 2 * lstart * n;
        ncol = 2 * (l + 1);
    } else if (mode == LU_MODE_INVERSE) {
        sol = S.sol + (size_t)l * n * n;
        ncol = n;
    } else {
        rhs = S.rhs + (size_t)l * ncols_fixed * n;
        sol = S.sol + (size_t)l * ncols_fixed * n;
        ncol = ncols_fixed;
    }
    const int t = threadIdx.x;
    // permuted right-hand sides (P b), zero past n and past the last column; threads walk rows
    for (int c = 0; c < NC; ++c) {
        const int col = c0 + c;
        for (int i = t; i < nrow; i += LS_THREADS) {
            double v = 0.0;
            if (i < n && col < ncol)
                v = (mode == LU_MODE_INVERSE) ? (perm[i] == col ? 1.0 : 0.0) : rhs[(size_t)col * n + perm[i]];
            Xs[xs_index<NC>(i, c)] = v;
        }
    }
    const int lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int rgp = warp & 3, grp = warp >> 2;             // row group (16 rows), K group
    double* ring = ring_all + warp * LS_STAGES * 16 * LS_RS;
    // this warp's chunks in order over both sweeps: (block row q-th, chunk j = grp, grp + 2, ...)
    // forward block ib has 4 (ib + 1) chunks; backward block ib has 4 (nblk - ib)
    auto nchunks = [&](bool bw, int ib) { return bw ? 4 * (nblk - ib) : 4 * (ib + 1); };
    // issue the copy of the warp's chunk number s (its 16 rows x 16 k of M)
    int f_bw = 0, f_q = 0, f_j = grp;                      // fetch cursor: sweep, block row ordinal, chunk
    auto fetch_next = [&](int stage) {
        if (f_bw < 2) {
            const bool bw = f_bw == 1;
            const int ib = bw ? nblk - 1 - f_q : f_q;
            const int k0 = chunk_k0(bw, ib, f_j);
            double* dst = ring + stage * 16 * LS_RS;
#pragma unroll
            for (int p = 0; p < 4; ++p) {           // 16 rows x 8 pieces of 16 bytes = 128 pieces, 4 per lane
                const int e = lane + 32 * p, r = e >> 3, pc = e & 7;
                const int gr = ib * SB + rgp * 16 + r, gk = k0 + 2 * pc;
                const bool ok = gr < n && gk < n;
                cp_async16(dst + r * LS_RS + 2 * pc, ok ? (const void*)(M + (size_t)gr * n + gk) : (const void*)M,
                           ok ? 16 : 0);
            }
            f_j += 2;
            if (f_j >= nchunks(bw, ib)) {
                f_j = grp;
                if (++f_q == nblk) {
                    f_q = 0;
                    ++f_bw;
                }
            }
        }
        cp_async_commit();
    };
    __syncthreads();   // Xs complete
#pragma unroll
    for (int st = 0; st < LS_STAGES - 1; ++st) fetch_next(st);
    int stage = 0;
    for (int bwi = 0; bwi < 2; ++bwi) {
        const bool bw = bwi == 1;
        for (int q = 0; q < nblk; ++q) {
            const int ib = bw ? nblk - 1 - q : q;
            const int nch = nchunks(bw, ib);
            double acc[2][NT][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < NT; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
            for (int j = grp; j < nch; j += 2) {
                cp_async_wait<LS_STAGES - 2>();
                __syncwarp();
                fetch_next((stage + LS_STAGES - 1) % LS_STAGES);
                const double* a_st = ring + stage * 16 * LS_RS;
                const int k0 = chunk_k0(bw, ib, j);
                const bool diag = k0 >= ib * SB && k0 < ib * SB + SB;
#pragma unroll
                for (int kk = 0; kk < LS_KC; kk += 4) {
                    const int kg = k0 + kk + tig;
                    double a[2], b[NT];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi) {
                        const int r = mi * 8 + g;
                        double v = a_st[r * LS_RS + kk + tig];
                        if (diag) {
                            const int rg = ib * SB + rgp * 16 + r;
                            v = bw ? (kg >= rg ? v : 0.0) : (kg < rg ? v : (kg == rg ? 1.0 : 0.0));
                        }
                        a[mi] = v;
                    }
#pragma unroll
                    for (int ni = 0; ni < NT; ++ni) b[ni] = Xs[xs_index<NC>(kg, ni * 8 + g)];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                        for (int ni = 0; ni < NT; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
                }
                stage = (stage + 1) % LS_STAGES;
            }
            // the second K group hands over its partial sums; the first writes the block row
            if (grp == 1) {
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < NT; ++ni)
#pragma unroll
                        for (int h = 0; h < 2; ++h)
                            red[(rgp * 16 + mi * 8 + g) * NC + ni * 8 + 2 * tig + h] = acc[mi][ni][h];
            }
            __syncthreads();   // partials parked; every warp is done reading this block row's Xs rows
            if (grp == 0) {
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < NT; ++ni)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int r = rgp * 16 + mi * 8 + g, c = ni * 8 + 2 * tig + h;
                            Xs[xs_index<NC>(ib * SB + r, c)] = acc[mi][ni][h] + red[r * NC + c];
                        }
            }
            __syncthreads();
        }
    }
    cp_async_wait<0>();
    for (int c = 0; c < NC && c0 + c < ncol; ++c)
        for (int i = t; i < n; i += LS_THREADS) sol[(size_t)(c0 + c) * n + i] = Xs[xs_index<NC>(i, c)];
}

// ---------------------------------------------------------------------------
// FP32 substitution + FP64 residual iterative refinement
// ---------------------------------------------------------------------------
constexpr int RF_NC = 16, RF_THREADS = 256, RF_MAXIT = 30;

__global__ void __launch_bounds__(RF_THREADS) lu_refine_kernel(const int4* __restrict__ tiles, LuSys S,
                                                               const float* __restrict__ Mf_all,
                                                               const double* __restrict__ A_all, int ncols,
                                                               int* __restrict__ iters) {
    extern __shared__ __align__(16) double rsm[];
    const int n = S.n, nblk = (n + SB - 1) / SB, nrow = nblk * SB;
    double* xs = rsm;                                   // [nrow][RF_NC] solution (FP64)
    float* rs = reinterpret_cast<float*>(xs + (size_t)nrow * RF_NC);   // [nrow][RF_NC] residual / update
    float* ys = rs + (size_t)nrow * RF_NC;              // [SB][RF_NC] block result
    __shared__ int s_done;
    __shared__ unsigned long long s_dmax[RF_NC], s_xmax[RF_NC];
    __shared__ double s_dprev[RF_NC];
    const int4 tl = tiles[blockIdx.x];
    const int l = tl.y, c0 = tl.z * RF_NC, t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const double* A = A_all + (size_t)l * n * n;
    const float* Mf = Mf_all + (size_t)l * n * n;
    const int* perm = S.perm + (size_t)l * n;
    const double* b = S.rhs + (size_t)l * ncols * n;
    double* x = S.sol + (size_t)l * ncols * n;
    for (int e = t; e < nrow * RF_NC; e += RF_THREADS) xs[e] = 0.0;
    __syncthreads();
    int it = 0;
    for (; it < RF_MAXIT; ++it) {
        // r = P (b - A x): one warp per row, lane = (k parity, column), the two k halves joined by a shuffle
        for (int i = warp; i < nrow; i += RF_THREADS / 32) {
            const int c = lane & (RF_NC - 1), kh = lane >> 4;
            double sacc = 0.0;
            if (i < n) {
                const double* arow = A + (size_t)perm[i] * n;
                for (int k = kh; k < n; k += 2) sacc = fma(arow[k], xs[k * RF_NC + c], sacc);
            }
            sacc += __shfl_xor_sync(0xffffffffu, sacc, 16);
            if (kh == 0) {
                const int col = c0 + c;
                double v = 0.0;
                if (i < n && col < ncols) v = b[(size_t)col * n + perm[i]] - sacc;
                rs[i * RF_NC + c] = (float)v;
            }
        }
        __syncthreads();
        // forward then backward block substitution in FP32 on rs
        for (int sweep = 0; sweep < 2; ++sweep)
            for (int q = 0; q < nblk; ++q) {
                const int ib = sweep ? nblk - 1 - q : q;
                const int kb = sweep ? ib * SB : 0, ke = sweep ? nrow : ib * SB + SB;
                for (int e = t; e < SB * RF_NC; e += RF_THREADS) {
                    const int r = e / RF_NC, c = e % RF_NC, rg = ib * SB + r;
                    float acc = 0.f;
                    if (rg < n) {
                        const float* mrow = Mf + (size_t)rg * n;
                        for (int k = kb; k < min(ke, n); ++k) {
                            float a = mrow[k];
                            if (k >= ib * SB && k < ib * SB + SB)
                                a = sweep ? (k >= rg ? a : 0.f) : (k < rg ? a : (k == rg ? 1.f : 0.f));
                            acc = fmaf(a, rs[k * RF_NC + c], acc);
                        }
                    }
                    ys[e] = acc;
                }
                __syncthreads();
                for (int e = t; e < SB * RF_NC; e += RF_THREADS) rs[(ib * SB) * RF_NC + e] = ys[e];
                __syncthreads();
            }
        // x += d; stop when every column's update is below 2^-52 of its largest entry
        if (t < RF_NC) {
            s_dmax[t] = 0ull;
            s_xmax[t] = 0ull;
        }
        __syncthreads();
        for (int e = t; e < n * RF_NC; e += RF_THREADS) {
            const double d = (double)rs[e];
            const double xn = xs[e] + d;
            xs[e] = xn;
            atomicMax(&s_dmax[e % RF_NC], (unsigned long long)__double_as_longlong(fabs(d)));
            atomicMax(&s_xmax[e % RF_NC], (unsigned long long)__double_as_longlong(fabs(xn)));
        }
        __syncthreads();
        if (t == 0) {
            // a column is done when its update is at the rounding level of the solution
            // (<= 2^-50 of its largest entry) or stopped shrinking (no longer halved:
            // the FP64 residual's own rounding is reached)
            int done = 1;
            for (int c = 0; c < RF_NC; ++c) {
                const double dm = __longlong_as_double((long long)s_dmax[c]);
                const double xm = __longlong_as_double((long long)s_xmax[c]);
                const bool conv = dm <= 0x1p-50 * xm || (it > 0 && dm > 0.5 * s_dprev[c]);
                if (!conv) done = 0;
                s_dprev[c] = dm;
            }
            s_done = done;
        }
        __syncthreads();
        if (s_done) {
            ++it;
            break;
        }
    }
    for (int e = t; e < n * RF_NC; e += RF_THREADS) {
        const int c = e / n, i = e % n, col = c0 + c;
        if (col < ncols) x[(size_t)col * n + i] = xs[i * RF_NC + c];
    }
    if (t == 0) iters[blockIdx.x] = it;
}

__global__ void to_float_kernel(const double* __restrict__ in, float* __restrict__ out, long count) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = (float)in[i];
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <class F>
static void set_smem(F* kern, size_t bytes) {
    RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

int lu_nc_for(int n) {
    return LuSolveShape<32>::smem(n) <= (size_t)(227 << 10) ? 32 : 16;
}

void lu_workspace(LuWork& w, int n, int count) {
    const int nblk = (n + SB - 1) / SB;
    if (w.cap_n >= n && w.cap_count >= count) return;
    lu_workspace_free(w);
    RA_CUDA(cudaMalloc(&w.d_status, (size_t)count * sizeof(int)));
    RA_CUDA(cudaMalloc(&w.d_inv, (size_t)count * nblk * 2 * SB * SB * sizeof(double)));
    w.cap_n = n;
    w.cap_count = count;
}

void lu_workspace_free(LuWork& w) {
    if (w.d_status) cudaFree(w.d_status);
    if (w.d_inv) cudaFree(w.d_inv);
    w = LuWork{};
}

int lu_factor_batch(cudaStream_t st, LuWork& w, double* d_mats, int* d_perm, int n, int count, const int* d_skip,
                    long* launches) {
    if (n < 2 || (n & 1)) throw ArgError("per-l matrices must have an even order >= 2");
    lu_workspace(w, n, count);
    const int nblk = (n + SB - 1) / SB;
    if (LuFactorSmem<32>::bytes(n) <= (size_t)(227 << 10)) {
        set_smem(lu_factor_kernel<32>, LuFactorSmem<32>::bytes(n));
        lu_factor_kernel<32><<<count, LU_THREADS, LuFactorSmem<32>::bytes(n), st>>>(d_mats, n, d_skip, d_perm,
                                                                                   w.d_status);
    } else if (LuFactorSmem<16>::bytes(n) <= (size_t)(227 << 10)) {
        set_smem(lu_factor_kernel<16>, LuFactorSmem<16>::bytes(n));
        lu_factor_kernel<16><<<count, LU_THREADS, LuFactorSmem<16>::bytes(n), st>>>(d_mats, n, d_skip, d_perm,
                                                                                   w.d_status);
    } else {
        throw ArgError("per-l matrix order " + std::to_string(n) + " exceeds the factorisation's shared-memory panel");
    }
    RA_CUDA(cudaGetLastError());
    std::vector<int> stt(count);
    RA_CUDA(cudaMemcpyAsync(stt.data(), w.d_status, count * sizeof(int), cudaMemcpyDeviceToHost, st));
    RA_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < count; ++i)
        if (stt[i]) return i + 1;
    const size_t dsm = 3 * SB * SBP * sizeof(double), osm = 2 * SB * SBP * sizeof(double);
    set_smem(lu_diag_inv_kernel, dsm);
    set_smem(lu_offdiag_kernel, osm);
    lu_diag_inv_kernel<<<dim3(count, nblk), 128, dsm, st>>>(d_mats, n, w.d_inv);
    RA_CUDA(cudaGetLastError());
    lu_offdiag_kernel<<<dim3(count, nblk, nblk), 256, osm, st>>>(d_mats, n, w.d_inv);
    RA_CUDA(cudaGetLastError());
    if (launches) *launches += 3;
    return 0;
}

void launch_lu_solve(cudaStream_t st, const int* d_tiles, int ntiles, const LuSys& sys, int mode, int ncols_fixed,
                     int nc) {
    if (ntiles == 0) return;
    if (nc == 32) {
        const size_t sm = LuSolveShape<32>::smem(sys.n);
        set_smem(lu_solve_kernel<32>, sm);
        lu_solve_kernel<32><<<ntiles, LS_THREADS, sm, st>>>(reinterpret_cast<const int4*>(d_tiles), sys, mode,
                                                            ncols_fixed);
    } else {
        const size_t sm = LuSolveShape<16>::smem(sys.n);
        if (sm > (size_t)(227 << 10)) throw ArgError("per-l matrix order too large for the block substitution");
        set_smem(lu_solve_kernel<16>, sm);
        lu_solve_kernel<16><<<ntiles, LS_THREADS, sm, st>>>(reinterpret_cast<const int4*>(d_tiles), sys, mode,
                                                            ncols_fixed);
    }
    RA_CUDA(cudaGetLastError());
}

// Tiles (system, l, column tile, 0) of one system, l descending.
void lu_append_tiles(std::vector<int>& t, int sys, int L, const std::vector<int>& ncols_of_l, int nc) {
    for (int l = L - 1; l >= 0; --l)
        for (int ct = 0; ct * nc < ncols_of_l[l]; ++ct) {
            t.push_back(sys);
            t.push_back(l);
            t.push_back(ct);
            t.push_back(0);
        }
}

void launch_lu_refine(cudaStream_t st, const int* d_tiles, int ntiles, const LuSys& s, const float* d_mf,
                      const double* d_a, int ncols, int* d_iters) {
    const int nrow = (s.n + SB - 1) / SB * SB;
    const size_t sm = (size_t)nrow * RF_NC * sizeof(double) + (size_t)nrow * RF_NC * sizeof(float) +
                      (size_t)SB * RF_NC * sizeof(float);
    if (sm > (size_t)(227 << 10)) throw ArgError("per-l matrix order too large for the refinement kernel");
    set_smem(lu_refine_kernel, sm);
    lu_refine_kernel<<<ntiles, RF_THREADS, sm, st>>>(reinterpret_cast<const int4*>(d_tiles), s, d_mf, d_a, ncols,
                                                     d_iters);
    RA_CUDA(cudaGetLastError());
}

void launch_to_float(cudaStream_t st, const double* in, float* out, long count) {
    to_float_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(in, out, count);
    RA_CUDA(cudaGetLastError());
}

int lu_refine_tile_cols() { return RF_NC; }

// ---------------------------------------------------------------------------
// The context's implicit solves
// ---------------------------------------------------------------------------
template <class T>
static T* upload_vec(Ctx& c, const std::vector<T>& v) {
    T* d = nullptr;
    RA_CUDA(cudaMalloc(&d, v.size() * sizeof(T)));
    RA_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c.stream));
    return d;
}

// Tile lists of the step's substitution (one launch per system) and, in the
// mixed form, of the explicit inverses; built once at set-up, since no
// allocation may run while a step is captured.
void solve_prepare(Ctx& c) {
    c.solve_nc = lu_nc_for(3 * c.d.nr);
    c.solve_nc_z = lu_nc_for(c.d.nr);
    rebuild_solve_tiles(c);
}

// (re)builds the missing tile lists for the current column-block choices
void rebuild_solve_tiles(Ctx& c) {
    const int L = c.d.L, nr = c.d.nr;
    auto make = [&](int*& d, int& cnt, const std::vector<int>& ncols, int nc) {
        if (d) return;
        std::vector<int> t;
        lu_append_tiles(t, 0, L, ncols, nc);
        cnt = (int)(t.size() / 4);
        d = upload_vec(c, t);
    };
    std::vector<int> step_cols(L);
    for (int l = 0; l < L; ++l) step_cols[l] = 2 * (l + 1);
    make(c.d_solve_tiles, c.n_solve_tiles, step_cols, c.solve_nc);
    make(c.d_solve_tiles_z, c.n_solve_tiles_z, step_cols, c.solve_nc_z);
    if (c.mixed_solve) {
        make(c.d_inv_sol_tiles, c.n_inv_sol_tiles, std::vector<int>(L, 3 * nr), c.solve_nc);
        make(c.d_inv_sol_tiles_z, c.n_inv_sol_tiles_z, std::vector<int>(L, nr), c.solve_nc_z);
    }
    RA_CUDA(cudaStreamSynchronize(c.stream));
}

// LU_Decompose_Matrices (Linear_Solve.F90:459-480): the assembled matrices in
// d_Awpt / d_Az are factored in place into the block-substitution form; the
// mixed form also forms the explicit inverses (transposed) for its split
// products.
void factor_matrices(Ctx& c) {
    const int L = c.d.L, nr = c.d.nr;
    int bad = lu_factor_batch(c.stream, c.lu_work, c.d_Awpt, c.d_perm_wpt, 3 * nr, L, nullptr, &c.launches);
    if (bad) throw SingularError("singular W-P-T matrix at l = " + std::to_string(bad - 1));
    bad = lu_factor_batch(c.stream, c.lu_work, c.d_Az, c.d_perm_z, nr, L, c.d_skip_z, &c.launches);
    if (bad) throw SingularError("singular Z matrix at l = " + std::to_string(bad - 1));
    if (c.mag) {   // C and A: no equation at l = 0, as for Z
        bad = lu_factor_batch(c.stream, c.lu_work, c.d_Ac, c.d_perm_c, nr, L, c.d_skip_z, &c.launches);
        if (bad) throw SingularError("singular C matrix at l = " + std::to_string(bad - 1));
        bad = lu_factor_batch(c.stream, c.lu_work, c.d_Aa, c.d_perm_a, nr, L, c.d_skip_z, &c.launches);
        if (bad) throw SingularError("singular A matrix at l = " + std::to_string(bad - 1));
    }
    if (c.mixed_solve) {
        const LuSys s0{c.d_Awpt, c.d_perm_wpt, nullptr, c.d_Ainv_wpt, 3 * nr};
        const LuSys s1{c.d_Az, c.d_perm_z, nullptr, c.d_Ainv_z, nr};
        launch_lu_solve(c.stream, c.d_inv_sol_tiles, c.n_inv_sol_tiles, s0, LU_MODE_INVERSE, 0, c.solve_nc);
        launch_lu_solve(c.stream, c.d_inv_sol_tiles_z, c.n_inv_sol_tiles_z, s1, LU_MODE_INVERSE, 0, c.solve_nc_z);
        c.launches += 2;
        if (c.mag) {   // the C and A systems go through the split products too
            const LuSys sc{c.d_Ac, c.d_perm_c, nullptr, c.d_Ainv_c, nr};
            const LuSys sa{c.d_Aa, c.d_perm_a, nullptr, c.d_Ainv_a, nr};
            launch_lu_solve(c.stream, c.d_inv_sol_tiles_z, c.n_inv_sol_tiles_z, sc, LU_MODE_INVERSE, 0, c.solve_nc_z);
            launch_lu_solve(c.stream, c.d_inv_sol_tiles_z, c.n_inv_sol_tiles_z, sa, LU_MODE_INVERSE, 0, c.solve_nc_z);
            c.launches += 2;
        }
    }
    RA_CUDA(cudaStreamSynchronize(c.stream));
}

// Implicit_Solve (Linear_Solve.F90:423-457): x = A_l^-1 b for every (system, l).
void launch_solve(Ctx& c) {
    if (!c.d_solve_tiles) throw ArgError("solve tiles not prepared (solve_prepare runs at set-up)");
    const int nr = c.d.nr;
    const LuSys s0{c.d_Awpt, c.d_perm_wpt, c.d_rhs_wpt, c.d_sol_wpt, 3 * nr};
    const LuSys s1{c.d_Az, c.d_perm_z, c.d_rhs_z, c.d_sol_z, nr};
    launch_lu_solve(c.stream, c.d_solve_tiles, c.n_solve_tiles, s0, LU_MODE_STEP, 0, c.solve_nc);
    launch_lu_solve(c.stream, c.d_solve_tiles_z, c.n_solve_tiles_z, s1, LU_MODE_STEP, 0, c.solve_nc_z);
    c.launches += 2;
}

// The C and A equations of the magnetic set (both precision forms): FP64 LU substitution
// with the Z system's tile list (same size, same columns per l; l = 0 is the identity).
void launch_solve_mag(Ctx& c) {
    if (!c.d_solve_tiles_z) throw ArgError("solve tiles not prepared (solve_prepare runs at set-up)");
    const int nr = c.d.nr;
    const LuSys sc{c.d_Ac, c.d_perm_c, c.d_rhs_c, c.d_sol_c, nr};
    const LuSys sa{c.d_Aa, c.d_perm_a, c.d_rhs_a, c.d_sol_a, nr};
    launch_lu_solve(c.stream, c.d_solve_tiles_z, c.n_solve_tiles_z, sc, LU_MODE_STEP, 0, c.solve_nc_z);
    launch_lu_solve(c.stream, c.d_solve_tiles_z, c.n_solve_tiles_z, sa, LU_MODE_STEP, 0, c.solve_nc_z);
    c.launches += 2;
}

}  // namespace ra
