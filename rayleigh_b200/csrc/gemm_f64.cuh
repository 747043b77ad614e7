// FP64 tile engine: a 64x64 CTA tile of C += A B computed with the FP64
// tensor-core instruction mma.sync.m8n8k4.f64 (4 warps, 32x32 per warp).
//
// Operands are read through functors, so the same engine serves the Legendre
// transforms (ragged K per m, parity split, equatorial fold), the Chebyshev
// synthesis and the per-l implicit solves.  Tiles of A (BK x BM) and B
// (BK x BN) are staged in shared memory, double buffered, with the next
// k-tile prefetched into registers while the current one is multiplied.
#pragma once

#include <cuda_runtime.h>

namespace ra {

constexpr int BK = 16, GEMM_THREADS = 128;
constexpr int SPAD = 4;  // row padding (doubles): conflict-free fragment reads

// Tile shape: WM x WN warps of 32x32 (WM * WN == 4), CTA tile BM x BN.
template <int WM, int WN>
struct Shape {
    static constexpr int BM = 32 * WM, BN = 32 * WN;
    static constexpr int NA = BK * BM / GEMM_THREADS, NB = BK * BN / GEMM_THREADS;
};
using Sq = Shape<2, 2>;     // 64 x 64
using Wide = Shape<1, 4>;   // 32 x 128
constexpr int BM = Sq::BM, BN = Sq::BN;

template <int WM, int WN>
struct GemmSmemT {
    double A[2][BK][32 * WM + SPAD];
    double B[2][BK][32 * WN + SPAD];
};
using GemmSmem = GemmSmemT<2, 2>;

struct Acc {
    double v[4][4][2];
    __device__ void zero() {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) v[i][j][0] = v[i][j][1] = 0.0;
    }
};

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// Element (k, x) of a BK x BX tile handled by thread t in slot i.
// MC = true: consecutive threads walk x (operand stored x-contiguous in memory);
// MC = false: consecutive threads walk k.
template <bool MC, int BX>
__device__ __forceinline__ void tile_coord(int t, int i, int& k, int& x) {
    int e = t + GEMM_THREADS * i;
    if (MC) {
        k = e / BX;
        x = e % BX;
    } else {
        x = e / BK;
        k = e % BK;
    }
}

// acc += sum_{k < K} A(k, m) B(k, n) for the CTA's BM x BN tile.
// fa(k, m) and fb(k, n) must return 0 outside the problem.
template <bool AMC, bool BNC, int WM = 2, int WN = 2, class FA, class FB>
__device__ __forceinline__ void gemm_tile(Acc& acc, const FA& fa, const FB& fb, int K, GemmSmemT<WM, WN>& sm) {
    using S = Shape<WM, WN>;
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = warp % WM, wn = warp / WM;
    double ra[S::NA], rb[S::NB];
    const int nk = (K + BK - 1) / BK;
    if (nk == 0) return;
    auto fetch = [&](int kt) {
#pragma unroll
        for (int i = 0; i < S::NA; ++i) {
            int k, x;
            tile_coord<AMC, S::BM>(t, i, k, x);
            ra[i] = fa(kt * BK + k, x);
        }
#pragma unroll
        for (int i = 0; i < S::NB; ++i) {
            int k, x;
            tile_coord<BNC, S::BN>(t, i, k, x);
            rb[i] = fb(kt * BK + k, x);
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int i = 0; i < S::NA; ++i) {
            int k, x;
            tile_coord<AMC, S::BM>(t, i, k, x);
            sm.A[buf][k][x] = ra[i];
        }
#pragma unroll
        for (int i = 0; i < S::NB; ++i) {
            int k, x;
            tile_coord<BNC, S::BN>(t, i, k, x);
            sm.B[buf][k][x] = rb[i];
        }
    };
    fetch(0);
    stash(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) fetch(kt + 1);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sm.A[buf][kk + tig][wm * 32 + i * 8 + g];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sm.B[buf][kk + tig][wn * 32 + j * 8 + g];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc.v[i][j], a[i], b[j]);
        }
        if (kt + 1 < nk) stash(buf ^ 1);
        __syncthreads();
    }
}

// Visit the accumulator: f(m, n, value) with (m, n) local to the CTA tile.
template <int WM = 2, int WN = 2, class F>
__device__ __forceinline__ void acc_foreach(const Acc& acc, const F& f) {
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = warp % WM, wn = warp / WM;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 2; ++q) f(wm * 32 + i * 8 + g, wn * 32 + j * 8 + 2 * tig + q, acc.v[i][j][q]);
}

template <int WM = 2, int WN = 2, class F>
__device__ __forceinline__ void acc_foreach2(const Acc& a, const Acc& b, const F& f) {
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = warp % WM, wn = warp / WM;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 2; ++q)
                f(wm * 32 + i * 8 + g, wn * 32 + j * 8 + 2 * tig + q, a.v[i][j][q], b.v[i][j][q]);
}

}  // namespace ra
