// Split-precision products on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// A double-precision product C = A B (A: M x K, B: K x N) is evaluated as an
// Ozaki-type sum of exact integer products.  Every row of A and every column
// of B is scaled by a power of two 2^e so that its largest entry lies in
// [1/4, 1/2), rounded to a 39-bit integer v = rint(x 2^{39-e}) and cut into
// S = 5 balanced base-256 digits (int8, the low bytes taken as signed):
//     x = 2^e sum_{s<S} q_s 2^{-(8s+7)} + r,   |r| <= 2^{e-40}.
// The digit products qa_s qb_t with s + t <= S-1 (15 of them) are accumulated
// over K in int32 by tcgen05.mma.kind::i8, one TMEM accumulator per diagonal
// d = s + t (exact for K < 20000), and the epilogue forms
//     c_ij = 2^{ea_i + eb_j} sum_d D_d[i,j] 2^{-(8d+14)}
// exactly in int64 and rounds it once to FP64 (all scalings are powers of two).  The relative error of a
// Legendre transform is ~1e-11 (vs ~1e-6 for one FP32-accumulated product).
//
// The product kernel is persistent (one CTA per SM, tiles dealt round-robin
// from a list ordered longest-K first) and warp-specialised:
//   warp 0      producer: one bulk copy (cp.async.bulk, no multicast) per
//               operand per K-step into a shared-memory ring of OZ_NST stages;
//   warp 1      MMA issuer: 15 tcgen05.mma per K-step, committed to the
//               stage's "empty" barrier and, after the last K-step, to the
//               accumulator's "full" barrier;
//   warps 2-13  epilogue: three warps per TMEM lane quadrant, each taking a
//               third of the tile's columns: tcgen05.ld of the 5 diagonals (one
//               wait per 8 columns), exact int64 recombination, scaled stores.
// Output tiles are 128 x 96: one accumulator set of 5 x 96 of the 512
// tensor-memory columns.  A 96-wide tile reads each A K-step once for 96
// output columns (the operands stream from L2 and bound the kernel), at the
// price of the next tile's MMAs waiting while the epilogue reads the set out
// of tensor memory (the stores and the FP64 sum over segments come after the
// set is released).  Every wait is bounded: when a limit runs out the CTA raises the
// device error word, drains its own copies and MMAs (bounded again), frees
// its tensor memory and returns.
#include <cstdint>
#include <cstdio>
#include <algorithm>

#include "ra_internal.h"
#include "ozaki.h"

namespace ra {

constexpr int OZ_STAGE = OZ_ABLK + OZ_BBLK;  // 35840 bytes
constexpr int OZ_NST = (232448 - 1024) / OZ_STAGE;   // operand ring stages that fit in 227 KB (6)
constexpr int OZ_EPI_WARPS = 12;                           // three per TMEM lane quadrant
constexpr int OZ_THREADS = 32 * (2 + OZ_EPI_WARPS);
constexpr int OZ_EPI_COLS = OZ_HB / (OZ_EPI_WARPS / 4);   // columns per epilogue warp (32)
static_assert(OZ_EPI_COLS % 8 == 0 && OZ_EPI_COLS <= 32, "epilogue column split");
constexpr int OZ_TMEM_COLS = 512;
// accumulator sets in tensor memory (two when 2 x 5 x HB columns fit, at a 256-column stride)
constexpr int OZ_NACC = (2 * OZ_S * OZ_HB <= OZ_TMEM_COLS) ? 2 : 1;
constexpr int OZ_ACC_STRIDE = 256;
static_assert(OZ_NACC == 2 ? OZ_S * OZ_HB <= OZ_ACC_STRIDE : OZ_S * OZ_HB <= OZ_TMEM_COLS,
              "accumulator sets exceed tensor memory");
constexpr long OZ_SPIN_LIMIT = 1L << 25;     // bounded waits: ~seconds, then the error word is set
static_assert(OZ_STAGE % 128 == 0, "stage size");

struct OzSmem {
    alignas(128) int8_t stage[OZ_NST][OZ_STAGE];
    alignas(8) uint64_t full[OZ_NST];
    uint64_t empty[OZ_NST];
    uint64_t acc_full[OZ_NACC];
    uint64_t acc_empty[OZ_NACC];
    uint64_t drain;
    uint32_t tmem_base;
    int abort;
};
static_assert(sizeof(OzSmem) <= 232448, "operand ring exceeds the 227 KB of shared memory per block");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle matrix descriptor (sm_100 version 1): start address,
// leading byte offset (between 16-byte K chunks), stride byte offset (between
// 8-row groups), all in 16-byte units.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// kind::i8 instruction descriptor: D s32, A/B signed int8, K-major both, N, M
__host__ __device__ constexpr uint32_t idesc_i8(int m, int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(smem_u32(bar)));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity));
    return ok != 0;
}

// bounded wait for the completion of the phase with the given parity;
// false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (long i = 0; i < OZ_SPIN_LIMIT; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > 16) __nanosleep(64);
    }
    return false;
}

// global -> shared bulk copy (no multicast), completion counted on bar
__device__ __forceinline__ void bulk_g2s(void* sdst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(sdst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// 2^e as a double (exact; ldexp outside the normal exponent range)
__device__ __forceinline__ double pow2(int e) {
    return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

__device__ __forceinline__ int vload(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// the 5 balanced base-256 digits of an integer v (|v| <= 2^38), most
// significant first in q[0]
__device__ __forceinline__ void oz_digits(long long v, int8_t (&q)[OZ_S]) {
#pragma unroll
    for (int s = OZ_S - 1; s > 0; --s) {
        const int8_t lo = (int8_t)(v & 0xFF);
        q[s] = lo;
        v = (v - lo) >> 8;
    }
    q[0] = (int8_t)v;
}

__global__ void __launch_bounds__(OZ_THREADS, 1) ozaki_gemm_kernel(const OzProblem* __restrict__ probs,
                                                                   const int4* __restrict__ tiles, int ntiles,
                                                                   int* __restrict__ status) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    OzSmem& sm = *reinterpret_cast<OzSmem*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < OZ_NST; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < OZ_NACC; ++b) {
            mbar_init(&sm.acc_full[b], 1);
            mbar_init(&sm.acc_empty[b], OZ_EPI_WARPS);
        }
        mbar_init(&sm.drain, 1);
        sm.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = sm.tmem_base;

    if (warp == 0) {
        // ---------------- producer ----------------
        // the next tile's descriptor is loaded while the current one streams
        int it = 0;
        int t = blockIdx.x;
        int4 tl = (t < ntiles) ? tiles[t] : make_int4(0, 0, 0, 0);
        OzProblem pb = probs[tl.x];
        for (; t < ntiles; t += gridDim.x) {
            if (vload(&sm.abort)) break;
            const int tn = t + gridDim.x;
            const int4 tl_n = (tn < ntiles) ? tiles[tn] : tl;
            const int8_t* a = pb.A + (long)tl.y * pb.a_tile;
            const int8_t* b = pb.B + (long)tl.z * pb.b_tile;
            const int nks = tl.w & 0xFFFF;
            bool ok = true;
            for (int ks = 0; ks < nks; ++ks, ++it) {
                const int st = it % OZ_NST;
                const uint32_t ph = (uint32_t)(it / OZ_NST) & 1u;
                if (!__all_sync(0xffffffffu, mbar_wait(&sm.empty[st], ph ^ 1u))) {
                    ok = false;
                    break;
                }
                if (lane == 0) {
                    mbar_expect_tx(&sm.full[st], (uint32_t)OZ_STAGE);
                    bulk_g2s(&sm.stage[st][0], a + (long)ks * OZ_ABLK, OZ_ABLK, &sm.full[st]);
                    bulk_g2s(&sm.stage[st][OZ_ABLK], b + (long)ks * OZ_BBLK, OZ_BBLK, &sm.full[st]);
                }
                __syncwarp();
            }
            if (!ok) {
                sm.abort = 1;
                break;
            }
            tl = tl_n;
            pb = probs[tl.x];
        }
        // copies still in flight after an abort: wait (bounded) for the last ones
        if (vload(&sm.abort)) {
            for (int j = (it > OZ_NST ? it - OZ_NST : 0); j < it; ++j)
                mbar_wait(&sm.full[j % OZ_NST], (uint32_t)(j / OZ_NST) & 1u);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        const uint32_t idesc = idesc_i8(OZ_HA, OZ_HB);
        // stage-0 descriptors; every stage and digit slice is an offset from these
        // (shared addresses stay below 2^18, so the 14-bit start field cannot overflow)
        const uint64_t adesc0 = umma_desc(smem_u32(&sm.stage[0][0]), OZ_HA * 16, 128);
        const uint64_t bdesc0 = umma_desc(smem_u32(&sm.stage[0][OZ_ABLK]), OZ_HB * 16, 128);
        int it = 0, tl_i = 0;   // tl_i counts accumulator uses (segments)
        int tw_n = (blockIdx.x < ntiles) ? tiles[blockIdx.x].w : 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            if (vload(&sm.abort)) break;
            const int nks = tw_n & 0xFFFF, nseg = tw_n >> 16;
            if (t + (int)gridDim.x < ntiles) tw_n = tiles[t + gridDim.x].w;
            const int kseg = nks / nseg;
            for (int sg = 0; sg < nseg && ok; ++sg, ++tl_i) {
                const int buf = tl_i % OZ_NACC;
                const uint32_t aph = (uint32_t)(tl_i / OZ_NACC) & 1u;
                ok = __all_sync(0xffffffffu, mbar_wait(&sm.acc_empty[buf], aph ^ 1u));
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t dacc = tmem + (uint32_t)(buf * OZ_ACC_STRIDE);
                for (int ks = 0; ks < kseg && ok; ++ks, ++it) {
                    const int st = it % OZ_NST;
                    const uint32_t ph = (uint32_t)(it / OZ_NST) & 1u;
                    if (!__all_sync(0xffffffffu, mbar_wait(&sm.full[st], ph))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    if (lane == 0) {
                        // descriptors of this stage: the start-address field (16-byte units) advanced
                        const uint64_t ast = adesc0 + (uint64_t)((st * OZ_STAGE) >> 4);
                        const uint64_t bst = bdesc0 + (uint64_t)((st * OZ_STAGE) >> 4);
#pragma unroll
                        for (int d = 0; d < OZ_S; ++d) {
#pragma unroll
                            for (int s = 0; s <= d; ++s) {
                                mma_i8(dacc + (uint32_t)(d * OZ_HB), ast + (uint64_t)((s * OZ_HA * OZ_BK) >> 4),
                                       bst + (uint64_t)(((d - s) * OZ_HB * OZ_BK) >> 4), idesc,
                                       (ks > 0 || s > 0) ? 1u : 0u);
                            }
                        }
                        umma_commit(&sm.empty[st]);
                    }
                    __syncwarp();
                }
                if (!ok) break;
                if (lane == 0) umma_commit(&sm.acc_full[buf]);
                __syncwarp();
            }
        }
        if (!ok) sm.abort = 1;
        // all MMAs of this CTA finished before the tensor memory is released
        if (lane == 0) umma_commit(&sm.drain);
        __syncwarp();
        if (!__all_sync(0xffffffffu, mbar_wait(&sm.drain, 0))) sm.abort = 1;
    } else {
        // ---------------- epilogue (warps 2..13): lane quadrant warp % 4, column third (warp - 2) / 4 ----------------
        const int q = warp & 3;
        const int cbeg = ((warp - 2) >> 2) * OZ_EPI_COLS;
        int tl_i = 0;   // accumulator uses (segments), as the MMA warp counts them
        int4 tl_n = (blockIdx.x < ntiles) ? tiles[blockIdx.x] : make_int4(0, 0, 0, 0);
        OzProblem pb_n = probs[tl_n.x];
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            if (vload(&sm.abort)) break;
            const int4 tl = tl_n;
            const OzProblem pb = pb_n;   // by value: stores to C cannot alias it
            if (t + (int)gridDim.x < ntiles) {
                tl_n = tiles[t + gridDim.x];
                pb_n = probs[tl_n.x];
            }
            const int nseg = tl.w >> 16;
            const int row = tl.y * OZ_HA + q * 32 + lane;
            const bool rok = row < pb.M;
            const int colw = tl.z * OZ_HB + cbeg + lane;
            const bool cok = lane < OZ_EPI_COLS && colw < pb.N;
            double part[OZ_EPI_COLS];   // FP64 sum over the segments
#pragma unroll
            for (int j = 0; j < OZ_EPI_COLS; ++j) part[j] = 0.0;
            for (int sg = 0; sg < nseg; ++sg, ++tl_i) {
                const int buf = tl_i % OZ_NACC;
                const uint32_t aph = (uint32_t)(tl_i / OZ_NACC) & 1u;
                // row scale with the combined weight 2^-46 of S below folded in; the
                // column scales of this warp's columns, one per lane, shared by shuffle
                // (loaded before the wait for the accumulator, which hides their latency)
                const int ea_v = rok ? pb.ea[sg * pb.ea_seg + row] : 0;
                const int eb_v = cok ? __ldg(pb.eb + sg * pb.eb_seg + colw) : 0;
                if (!mbar_wait(&sm.acc_full[buf], aph)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const double sa = rok ? pow2(ea_v - 46) : 0.0;
                const double sbl = cok ? pow2(eb_v) : 0.0;
                const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * OZ_ACC_STRIDE);
#pragma unroll
                for (int c8 = 0; c8 < OZ_EPI_COLS; c8 += 8) {
                    uint32_t v[OZ_S][8];
#pragma unroll
                    for (int d = 0; d < OZ_S; ++d)
                        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                                     : "=r"(v[d][0]), "=r"(v[d][1]), "=r"(v[d][2]), "=r"(v[d][3]), "=r"(v[d][4]),
                                       "=r"(v[d][5]), "=r"(v[d][6]), "=r"(v[d][7])
                                     : "r"(tbase + (uint32_t)(d * OZ_HB + cbeg + c8)));
                    asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        // S = sum_d D_d 2^(8(4-d)) is exact in int64 (|S| < 2^59 for K <= 20000);
                        // the value is S 2^-46 2^(ea + eb), rounded once per segment
                        long long S = (long long)(int)v[0][j];
#pragma unroll
                        for (int d = 1; d < OZ_S; ++d) S = S * 256 + (long long)(int)v[d][j];
                        const double sb = __shfl_sync(0xffffffffu, sbl, c8 + j);
                        part[c8 + j] += (__ll2double_rn(S) * sa) * sb;
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;");
                __syncwarp();
                if (lane == 0) mbar_arrive(&sm.acc_empty[buf]);
            }
            if (!ok) break;
            if (rok) {
                double* crow = pb.C + (long)row * pb.c_m;
                const int cb = tl.z * OZ_HB + cbeg;
#pragma unroll
                for (int j = 0; j < OZ_EPI_COLS; ++j)
                    if (cb + j < pb.N) crow[(long)(cb + j) * pb.c_n] = part[j];
            }
        }
        if (!ok) sm.abort = 1;
    }

    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (threadIdx.x == 0 && sm.abort) atomicOr(status, RA_STATUS_TIMEOUT);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(OZ_TMEM_COLS));
    }
}

// ---------------------------------------------------------------------------
// Splitting into tiled digits (a batch of jobs).  Block = 16 rows of one job:
// a max pass over K, then per K-step a 16 x 32 tile of X through shared
// memory (read along whichever index is contiguous), digits transposed into
// the [s][kc][row][16] block layout and written as 16-byte rows.
// ---------------------------------------------------------------------------
// Split of a job whose K runs are contiguous (sk == 1): 16 rows per CTA,
// staged through shared memory so that each store is 16 rows x 16 bytes.
__global__ void __launch_bounds__(256) ozaki_split_kernel(const OzSplitJob* __restrict__ jobs) {
    const OzSplitJob& jb = jobs[blockIdx.y];
    if (jb.sk != 1) return;   // ozaki_split_rows_kernel
    const int r0 = blockIdx.x * 16;
    if (r0 >= jb.nrt * jb.H) return;
    __shared__ double xs[16][33];
    __shared__ double red[16][17];
    __shared__ int ex_s[16];
    __shared__ __align__(16) int8_t dig[OZ_S][2][16][16];
    const int tid = threadIdx.x;
    const bool kmajor = (jb.sk == 1);
    // pass 1: row maxima (thread: row lr, K offset lk, stride 16) and the row
    // shifts 39 - e: the digits are those of the integer rint(x 2^(39-e))
    const int lr = kmajor ? (tid >> 4) : (tid & 15);
    const int lk = kmajor ? (tid & 15) : (tid >> 4);
    const int r = r0 + lr;
    double mx = 0.0;
    if (r < jb.R)
        for (int k = lk; k < jb.K; k += 16) mx = fmax(mx, fabs(jb.X[(long)r * jb.sr + (long)k * jb.sk]));
    red[lr][lk] = mx;
    __syncthreads();
    if (tid < 16) {
        double m = red[tid][0];
#pragma unroll
        for (int i = 1; i < 16; ++i) m = fmax(m, red[tid][i]);
        const int ex = (m > 0.0) ? ilogb(m) + 2 : 0;
        ex_s[tid] = 39 - ex;
        if (r0 + tid < jb.R) jb.e[r0 + tid] = ex;
    }
    const int rt = r0 / jb.H, rin = r0 - rt * jb.H;
    const long blk = (long)OZ_S * jb.H * OZ_BK;
    const int kstride = jb.kstride > 0 ? jb.kstride : jb.nks;
    for (int ks = 0; ks < jb.nks; ++ks) {
        const int k0 = ks * OZ_BK;
        __syncthreads();   // ex_s ready / previous tile consumed
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int idx = tid + 256 * i;
            const int row = kmajor ? (idx >> 5) : (idx & 15);
            const int kk = kmajor ? (idx & 31) : (idx >> 4);
            const int rr = r0 + row, k = k0 + kk;
            xs[row][kk] = (rr < jb.R && k < jb.K) ? jb.X[(long)rr * jb.sr + (long)k * jb.sk] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int idx = tid + 256 * i;
            const int row = idx >> 5, kk = idx & 31;
            const int sh = ex_s[row];
            const double a = (sh <= 1023 && sh >= -1022) ? xs[row][kk] * pow2(sh) : ldexp(xs[row][kk], sh);
            int8_t qd[OZ_S];
            oz_digits(__double2ll_rn(a), qd);
#pragma unroll
            for (int s = 0; s < OZ_S; ++s) dig[s][kk >> 4][row][kk & 15] = qd[s];
        }
        __syncthreads();
        if (tid < OZ_S * 32) {
            const int s = tid >> 5, kc = (tid >> 4) & 1, row = tid & 15;
            int8_t* dst = jb.out + ((long)rt * kstride + jb.ks0 + ks) * blk + (long)s * jb.H * OZ_BK + (long)kc * jb.H * 16 +
                          (long)(rin + row) * 16;
            *reinterpret_cast<int4*>(dst) = *reinterpret_cast<const int4*>(&dig[s][kc][row][0]);
        }
    }
}

// Split of a job whose rows are contiguous (sk != 1; the transposed operands
// s2a11^T, p2b^T): 64 rows per CTA, four threads per row taking every fourth
// k (pass 1) and every fourth 16-wide K chunk (pass 2).  A warp is 32
// consecutive rows of one K lane, so its loads cover 256 contiguous bytes; each
// thread packs the digits of 16 consecutive k into one 16-byte chunk per digit
// plane, and a warp's chunks are 512 contiguous bytes of the tiled layout.  A
// CTA reads its 64 x K block twice (maxima, then digits); the blocks of all
// resident CTAs fit in L2, so the second pass does not go back to HBM.
constexpr int OZ_ROWS_THREADS = 256;
constexpr int OZ_ROWS_PER_CTA = 64;
constexpr int OZ_KLANES = OZ_ROWS_THREADS / OZ_ROWS_PER_CTA;

__global__ void __launch_bounds__(OZ_ROWS_THREADS) ozaki_split_rows_kernel(const OzSplitJob* __restrict__ jobs) {
    const OzSplitJob& jb = jobs[blockIdx.y];
    if (jb.sk == 1) return;   // ozaki_split_kernel
    const int r0 = blockIdx.x * OZ_ROWS_PER_CTA;
    if (r0 >= jb.nrt * jb.H) return;
    __shared__ double red[OZ_KLANES][OZ_ROWS_PER_CTA];
    const int lrow = threadIdx.x % OZ_ROWS_PER_CTA, kl = threadIdx.x / OZ_ROWS_PER_CTA;
    const int r = r0 + lrow;
    const bool pad = r >= jb.nrt * jb.H;   // past the last row tile: no work
    const bool live = r < jb.R;            // rows R .. nrt*H - 1 are padding: zero digits
    const long sk = jb.sk;
    const int K = jb.K;
    const double* __restrict__ xr = jb.X + (long)(live ? r : 0) * jb.sr;
    // eight loads in flight per thread: this pass streams the operand from HBM
    double mm[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) mm[i] = 0.0;
    if (live) {
        int k = kl;
        for (; k + 7 * OZ_KLANES < K; k += 8 * OZ_KLANES) {
            double v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = __ldg(xr + (long)(k + i * OZ_KLANES) * sk);
#pragma unroll
            for (int i = 0; i < 8; ++i) mm[i] = fmax(mm[i], fabs(v[i]));
        }
        for (; k < K; k += OZ_KLANES) mm[0] = fmax(mm[0], fabs(__ldg(xr + (long)k * sk)));
    }
    red[kl][lrow] = fmax(fmax(fmax(mm[0], mm[1]), fmax(mm[2], mm[3])), fmax(fmax(mm[4], mm[5]), fmax(mm[6], mm[7])));
    __syncthreads();
    double mx = red[0][lrow];
#pragma unroll
    for (int i = 1; i < OZ_KLANES; ++i) mx = fmax(mx, red[i][lrow]);
    if (pad) return;
    const int ex = (mx > 0.0) ? ilogb(mx) + 2 : 0;   // digits of the integer rint(x 2^(39-e))
    if (live && kl == 0) jb.e[r] = ex;
    const int sh = 39 - ex;
    const bool direct = (sh <= 1023 && sh >= -1022);
    const double sc = direct ? pow2(sh) : 1.0;
    const int rt = r / jb.H, rin = r - rt * jb.H;
    const long blk = (long)OZ_S * jb.H * OZ_BK;
    const int kstride = jb.kstride > 0 ? jb.kstride : jb.nks;
#pragma unroll 1
    for (int ch = kl; ch < 2 * jb.nks; ch += OZ_KLANES) {   // 16-wide K chunk ch = (K-step, half)
        const int ks = ch >> 1, kc = ch & 1;
        const int k0 = ch * 16;
        double v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = (live && k0 + i < K) ? __ldg(xr + (long)(k0 + i) * sk) : 0.0;
        unsigned w[OZ_S][4];
#pragma unroll
        for (int s = 0; s < OZ_S; ++s) w[s][0] = w[s][1] = w[s][2] = w[s][3] = 0u;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const double a = direct ? v[i] * sc : ldexp(v[i], sh);
            int8_t qd[OZ_S];
            oz_digits(__double2ll_rn(a), qd);
#pragma unroll
            for (int s = 0; s < OZ_S; ++s) w[s][i >> 2] |= (unsigned)(uint8_t)qd[s] << (8 * (i & 3));
        }
        int8_t* base = jb.out + ((long)rt * kstride + jb.ks0 + ks) * blk + (long)kc * jb.H * 16 + (long)rin * 16;
#pragma unroll
        for (int s = 0; s < OZ_S; ++s)
            *reinterpret_cast<int4*>(base + (long)s * jb.H * OZ_BK) =
                make_int4((int)w[s][0], (int)w[s][1], (int)w[s][2], (int)w[s][3]);
    }
}

int oz_split_kinds(const OzSplitJob* jobs, int njobs) {
    int kinds = 0;
    for (int i = 0; i < njobs; ++i) kinds |= (jobs[i].sk == 1) ? OZ_SPLIT_KMAJOR : OZ_SPLIT_ROWS;
    return kinds;
}

void ozaki_split(Ctx& c, const OzSplitJob* d_jobs, int njobs, int max_rows, int kinds) {
    if (njobs == 0 || max_rows == 0) return;
    if (kinds & OZ_SPLIT_KMAJOR) {
        dim3 grid((max_rows + 15) / 16, njobs);
        ozaki_split_kernel<<<grid, 256, 0, c.stream>>>(d_jobs);
        RA_CUDA(cudaGetLastError());
        ++c.launches;
    }
    if (kinds & OZ_SPLIT_ROWS) {
        dim3 grid((max_rows + OZ_ROWS_PER_CTA - 1) / OZ_ROWS_PER_CTA, njobs);
        ozaki_split_rows_kernel<<<grid, OZ_ROWS_THREADS, 0, c.stream>>>(d_jobs);
        RA_CUDA(cudaGetLastError());
        ++c.launches;
    }
}

// SM count of the current device (asked on every call: one process may drive several devices)
static int oz_sm_count() {
    int dev = 0, n = 0;
    RA_CUDA(cudaGetDevice(&dev));
    RA_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

void ozaki_gemm(Ctx& c, const OzProblem* d_probs, const int* d_tiles, int ntiles, int* d_status) {
    if (ntiles == 0) return;
    // the limit is per device: set it on every launch
    RA_CUDA(cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(OzSmem)));
    const int grid = std::min(ntiles, oz_sm_count());
    ozaki_gemm_kernel<<<grid, OZ_THREADS, sizeof(OzSmem), c.stream>>>(
        d_probs, reinterpret_cast<const int4*>(d_tiles), ntiles, d_status);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// Tile list (problem, m-tile, n-tile, K-steps | segments << 16), longest K
// first so that the ragged products finish together; products with K = 0 get
// no tiles.
std::vector<int> ozaki_tiles(const std::vector<OzProblem>& probs) {
    std::vector<int> order(probs.size());
    for (size_t p = 0; p < probs.size(); ++p) order[p] = (int)p;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return probs[a].nks > probs[b].nks; });
    std::vector<int> t;
    for (int p : order) {
        const OzProblem& q = probs[p];
        if (q.nks == 0) continue;
        for (int mt = 0; mt * OZ_HA < q.M; ++mt)
            for (int nt = 0; nt * OZ_HB < q.N; ++nt) {
                t.push_back(p);
                t.push_back(mt);
                t.push_back(nt);
                t.push_back(q.nks | ((q.nseg > 0 ? q.nseg : 1) << 16));
            }
    }
    return t;
}

// ---------------------------------------------------------------------------
// Allocation-free form of the split-precision product (ra_mixed_gemm_noalloc).
//
// All scratch lives in one file-scope device array of fixed size; its device
// address is looked up on every call (cudaGetSymbolAddress with the caller's
// device current: one lookup per call, nothing cached between calls, so no
// host-side state is shared by threads).  Scratch layout, every piece
// 256-byte aligned:
//   [0]        int        status word    (set to zero by oz_static_prepare_kernel)
//   [256]      OzProblem                 (written by oz_static_prepare_kernel)
//   [512]      OzSplitJob[2]             (written by oz_static_prepare_kernel)
//   [1024]     int4       tiles[ntiles]  (written by oz_static_prepare_kernel)
//   then       int        ea[mp], eb[np] (written by the split kernel)
//   then       int8       A digits (mp x kp x 5), B digits (np x kp x 5) (split kernel)
// Nothing else needs to start at zero: the split kernel writes every padded
// digit and every exponent the product reads.  Calls on one device share the
// array, so calls that overlap in time (two host threads, or two streams)
// race on it.
// ---------------------------------------------------------------------------
constexpr size_t OZ_STATIC_BYTES = (size_t)16 << 20;   // 16 MiB
static __device__ __align__(256) unsigned char oz_static_scratch[OZ_STATIC_BYTES];

static size_t oz_align256(size_t x) { return (x + 255) & ~(size_t)255; }

__global__ void oz_static_prepare_kernel(OzProblem pr, OzSplitJob ja, OzSplitJob jb, OzProblem* __restrict__ dprob,
                                         OzSplitJob* __restrict__ djobs, int4* __restrict__ tiles, int ntm, int ntn,
                                         int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        *dprob = pr;
        djobs[0] = ja;
        djobs[1] = jb;
        *status = 0;
    }
    if (i < ntm * ntn) tiles[i] = make_int4(0, i / ntn, i % ntn, pr.nks | (1 << 16));
}

}  // namespace ra

static void oz_set_msg(char* msg, int len, const char* text) {
    if (!msg || len <= 0) return;
    int i = 0;
    for (; text[i] && i < len - 1; ++i) msg[i] = text[i];
    msg[i] = 0;
}

extern "C" int ra_mixed_gemm_noalloc(const double* d_a, const double* d_b, double* d_c, int m, int n, int k,
                                     void* stream, char* msg, int msg_len) {
    using namespace ra;
    oz_set_msg(msg, msg_len, "");
    if (!d_a || !d_b || !d_c || m <= 0 || n <= 0 || k <= 0) {
        oz_set_msg(msg, msg_len, "ra_mixed_gemm_noalloc: null pointer or non-positive size");
        return RA_ERR_ARG;
    }
    if (k > OZ_MAX_K) {
        oz_set_msg(msg, msg_len, "ra_mixed_gemm_noalloc: k exceeds the exact int32 accumulation limit (20000)");
        return RA_ERR_ARG;
    }
    const int ntm = oz_tiles_of(m, OZ_HA), ntn = oz_tiles_of(n, OZ_HB), ntiles = ntm * ntn;
    const int mp = ntm * OZ_HA, np = ntn * OZ_HB, nks = oz_ksteps(k), kp = nks * OZ_BK;
    const size_t off_prob = 256, off_jobs = 512, off_tiles = 1024;
    const size_t off_ea = off_tiles + oz_align256((size_t)ntiles * sizeof(int4));
    const size_t off_eb = off_ea + oz_align256((size_t)mp * sizeof(int));
    const size_t off_sa = off_eb + oz_align256((size_t)np * sizeof(int));
    const size_t off_sb = off_sa + oz_align256((size_t)OZ_S * mp * kp);
    const size_t need = off_sb + oz_align256((size_t)OZ_S * np * kp);
    if (need > OZ_STATIC_BYTES) {
        char text[200];
        snprintf(text, sizeof(text),
                 "ra_mixed_gemm_noalloc: m=%d n=%d k=%d needs %zu bytes of scratch; the static limit is %zu bytes (16 MiB)",
                 m, n, k, need, OZ_STATIC_BYTES);
        oz_set_msg(msg, msg_len, text);
        return RA_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0) {
        oz_set_msg(msg, msg_len, "ra_mixed_gemm_noalloc: no usable current device");
        return RA_ERR_CUDA;
    }
    // the array's device address on the current device (the host-side name is not one)
    void* scratch = nullptr;
    e = cudaGetSymbolAddress(&scratch, oz_static_scratch);
    if (e != cudaSuccess || !scratch) {
        oz_set_msg(msg, msg_len, cudaGetErrorString(e));
        return RA_ERR_CUDA;
    }
    int nsm = 0;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || nsm <= 0) {
        oz_set_msg(msg, msg_len, "ra_mixed_gemm_noalloc: cannot read the SM count");
        return RA_ERR_CUDA;
    }
    unsigned char* base = static_cast<unsigned char*>(scratch);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int* d_status = reinterpret_cast<int*>(base);
    OzProblem* d_prob = reinterpret_cast<OzProblem*>(base + off_prob);
    OzSplitJob* d_jobs = reinterpret_cast<OzSplitJob*>(base + off_jobs);
    int4* d_tiles = reinterpret_cast<int4*>(base + off_tiles);
    int* ea = reinterpret_cast<int*>(base + off_ea);
    int* eb = reinterpret_cast<int*>(base + off_eb);
    int8_t* sa = reinterpret_cast<int8_t*>(base + off_sa);
    int8_t* sb = reinterpret_cast<int8_t*>(base + off_sb);

    const OzSplitJob ja{d_a, (long)k, 1L, m, k, OZ_HA, ntm, nks, sa, ea};
    const OzSplitJob jbj{d_b, 1L, (long)n, n, k, OZ_HB, ntn, nks, sb, eb};
    const OzProblem pr{sa, sb, (long)nks * OZ_ABLK, (long)nks * OZ_BBLK, ea, eb, m, n, nks, d_c, (long)n, 1L};
    oz_static_prepare_kernel<<<(ntiles + 127) / 128, 128, 0, st>>>(pr, ja, jbj, d_prob, d_jobs, d_tiles, ntm, ntn,
                                                                     d_status);
    ozaki_split_kernel<<<dim3((std::max(mp, np) + 15) / 16, 2), 256, 0, st>>>(d_jobs);
    ozaki_split_rows_kernel<<<dim3((std::max(mp, np) + OZ_ROWS_PER_CTA - 1) / OZ_ROWS_PER_CTA, 2), OZ_ROWS_THREADS,
                              0, st>>>(d_jobs);
    e = cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(OzSmem));
    if (e == cudaSuccess) {
        ozaki_gemm_kernel<<<std::min(ntiles, nsm), OZ_THREADS, sizeof(OzSmem), st>>>(d_prob, d_tiles, ntiles, d_status);
        e = cudaGetLastError();
    }
    int status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        oz_set_msg(msg, msg_len, cudaGetErrorString(e));
        return RA_ERR_CUDA;
    }
    if (status) {
        oz_set_msg(msg, msg_len, "ra_mixed_gemm_noalloc: tensor-core product timed out waiting on its pipeline barrier");
        return RA_ERR_CUDA;
    }
    return RA_OK;
}
