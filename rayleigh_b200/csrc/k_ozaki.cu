// Split-precision products on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// A double-precision product C = A B (A: M x K, B: K x N) is evaluated as an
// Ozaki-type sum of exact integer products.  Every row of A and every column
// of B is scaled by a power of two so that its largest entry lies in [1/2, 1),
// then cut into S signed 7-bit digits (int8):
//     a_ik = 2^{ea_i} sum_{s<S} qa_s[i,k] 2^{-7(s+1)},  b_kj = 2^{eb_j} sum_{t<S} qb_t[j,k] 2^{-7(t+1)}.
// The products qa_s qb_t with s + t <= S-1 are accumulated over K in int32 by
// tcgen05.mma.kind::i8, one TMEM accumulator per diagonal d = s + t (exact: no
// rounding at all until the epilogue), and the epilogue forms
//     c_ij = 2^{ea_i + eb_j} sum_d D_d[i,j] 2^{-7(d+2)}
// in FP64.  With S = 6 (21 products) the relative error of a Legendre
// transform is ~1e-11 (measured against the FP64 product), against ~1e-6 for
// a single FP32-accumulated product.
//
// Kernel layout: one CTA (4 warps) per 128 x 64 output tile; operand tiles of
// 32 int8 columns (one MMA K-step) per slice are staged in shared memory in
// the K-major "core matrix" layout (8 rows x 16 bytes contiguous, no swizzle)
// by cp.async, 4 stages deep; thread 0 issues the 21 MMAs of a stage and
// commits them to the stage's mbarrier; the accumulators (6 x 64 columns of
// int32) live in tensor memory and are read back with tcgen05.ld.
#include <cstdint>
#include <cstdio>

#include "ra_internal.h"
#include "ozaki.h"

namespace ra {

constexpr int OZ_BM = 128, OZ_BN = 64, OZ_BK = 32, OZ_NST = 4, OZ_THREADS = 128;
constexpr int OZ_TMEM_COLS = 512;
constexpr long OZ_SPIN_LIMIT = 1L << 26;   // bounded waits: ~seconds, then the error word is set

struct OzSmem {
    alignas(128) int8_t A[OZ_NST][OZ_S][OZ_BM * OZ_BK];
    alignas(128) int8_t B[OZ_NST][OZ_S][OZ_BN * OZ_BK];
    alignas(8) uint64_t mbar[OZ_NST];
    uint32_t tmem_base;
    int abort;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle matrix descriptor (sm_100 version 1)
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

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity));
    return ok != 0;
}

// bounded wait; returns false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (long i = 0; i < OZ_SPIN_LIMIT; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > 64) __nanosleep(32);
    }
    return false;
}

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sdst)), "l"(gsrc));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }

// core-matrix offset of (row, 16-byte chunk kc) in a tile of R rows x 32 bytes
__device__ __forceinline__ int cm_off(int row, int kc, int R) { return kc * (R / 8) * 128 + (row >> 3) * 128 + (row & 7) * 16; }

__global__ void __launch_bounds__(OZ_THREADS, 1) ozaki_gemm_kernel(const OzProblem* __restrict__ probs,
                                                                   const int4* __restrict__ tiles,
                                                                   int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    OzSmem& sm = *reinterpret_cast<OzSmem*>(smem_raw);
    const int4 tl = tiles[blockIdx.x];
    const OzProblem pb = probs[tl.x];
    const int m0 = tl.y * OZ_BM, n0 = tl.z * OZ_BN;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nk = pb.kpad / OZ_BK;

    if (nk == 0) {   // empty product: the tile is zero
        for (int e = tid; e < OZ_BM * OZ_BN; e += OZ_THREADS) {
            const int i = m0 + e / OZ_BN, j = n0 + e % OZ_BN;
            if (i < pb.M && j < pb.N) pb.C[(long)i * pb.c_m + (long)j * pb.c_n] = 0.0;
        }
        return;
    }
    if (tid == 0) {
        for (int s = 0; s < OZ_NST; ++s) mbar_init(&sm.mbar[s], 1);
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

    auto load_stage = [&](int kstep, int st) {
        const long k0 = (long)kstep * OZ_BK;
        // A: S slices x 128 rows x 2 chunks
        for (int e = tid; e < OZ_S * OZ_BM * 2; e += OZ_THREADS) {
            const int s = e / (OZ_BM * 2), rem = e % (OZ_BM * 2);
            const int row = rem >> 1, kc = rem & 1;
            const int8_t* src = pb.A + s * pb.a_slice + (long)(m0 + row) * pb.kpad + k0 + kc * 16;
            cp_async16(&sm.A[st][s][cm_off(row, kc, OZ_BM)], src);
        }
        for (int e = tid; e < OZ_S * OZ_BN * 2; e += OZ_THREADS) {
            const int s = e / (OZ_BN * 2), rem = e % (OZ_BN * 2);
            const int row = rem >> 1, kc = rem & 1;
            const int8_t* src = pb.B + s * pb.b_slice + (long)(n0 + row) * pb.kpad + k0 + kc * 16;
            cp_async16(&sm.B[st][s][cm_off(row, kc, OZ_BN)], src);
        }
    };

    const uint32_t idesc = idesc_i8(OZ_BM, OZ_BN);
    bool ok = true;
    int issued = 0;   // steps whose MMAs were issued and committed
    // prologue: stages 0 .. NST-2
    for (int p = 0; p < OZ_NST - 1; ++p) {
        if (p < nk) load_stage(p, p);
        cp_async_commit();
    }
    for (int k = 0; k < nk; ++k) {
        const int st = k % OZ_NST;
        cp_async_wait<OZ_NST - 2>();
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int d = 0; d < OZ_S; ++d) {
#pragma unroll
                for (int s = 0; s <= d; ++s) {
                    const int t = d - s;
                    const uint64_t ad = umma_desc(smem_u32(&sm.A[st][s][0]), (OZ_BM / 8) * 128, 128);
                    const uint64_t bd = umma_desc(smem_u32(&sm.B[st][t][0]), (OZ_BN / 8) * 128, 128);
                    mma_i8(tmem + (uint32_t)(d * OZ_BN), ad, bd, idesc, (k > 0 || s > 0) ? 1u : 0u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&sm.mbar[st])));
        }
        ++issued;
        // refill the buffer that the MMAs of step k-1 read
        const int kn = k + OZ_NST - 1;
        if (kn < nk) {
            if (k >= 1) {
                const int pb_ = (k - 1) % OZ_NST;
                if (!mbar_wait(&sm.mbar[pb_], (uint32_t)(((k - 1) / OZ_NST) & 1))) {
                    ok = false;
                }
            }
            if (ok) load_stage(kn, kn % OZ_NST);
        }
        cp_async_commit();
        if (!ok) {
            sm.abort = 1;
        }
        __syncthreads();
        if (sm.abort) break;
    }
    cp_async_wait<0>();
    // wait (bounded) for the last committed MMAs, on the normal and the abort path alike
    if (issued > 0) {
        const int kl = issued - 1;
        if (!mbar_wait(&sm.mbar[kl % OZ_NST], (uint32_t)((kl / OZ_NST) & 1))) sm.abort = 1;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!sm.abort) {
        // epilogue: warp w owns tile rows 32w .. 32w+31 (TMEM lanes)
        const int row = m0 + warp * 32 + lane;
        const int ea = (row < pb.M) ? pb.ea[row] : 0;
        for (int c0 = 0; c0 < OZ_BN; c0 += 16) {
            double acc[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = 0.0;
#pragma unroll
            for (int d = 0; d < OZ_S; ++d) {
                uint32_t v[16];
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(d * OZ_BN + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;");
                const double sc = ldexp(1.0, -7 * (d + 2));
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[j] += (double)(int32_t)v[j] * sc;
            }
            if (row < pb.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + c0 + j;
                    if (col < pb.N) pb.C[(long)row * pb.c_m + (long)col * pb.c_n] = ldexp(acc[j], ea + pb.eb[col]);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(status, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(OZ_TMEM_COLS));
}

// ---------------------------------------------------------------------------
// Splitting: rows of X (element (i, k) at X[i*si + k*sk], i < R, k < K) into
// S int8 digit slices out[s][i][kpad] (rows padded to rpad, columns to kpad)
// and exponents e[i] (e = 0 for an all-zero row).  One warp per row.
// ---------------------------------------------------------------------------
__global__ void ozaki_split_kernel(const double* __restrict__ X, long si, long sk, int R, int K, int rpad, int kpad,
                                   int8_t* __restrict__ out, long slice, int* __restrict__ e) {
    const int warps = blockDim.x / 32;
    const int row = blockIdx.x * warps + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= rpad) return;
    double mx = 0.0;
    if (row < R)
        for (int k = lane; k < K; k += 32) mx = fmax(mx, fabs(X[(long)row * si + (long)k * sk]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const int ex = (mx > 0.0) ? ilogb(mx) + 1 : 0;
    if (lane == 0 && row < R) e[row] = ex;
    const double scale = ldexp(1.0, -ex);
    for (int k = lane; k < kpad; k += 32) {
        double a = (row < R && k < K) ? X[(long)row * si + (long)k * sk] * scale : 0.0;
        int8_t* o = out + (long)row * kpad + k;
#pragma unroll
        for (int s = 0; s < OZ_S; ++s) {
            a *= 128.0;
            const double q = trunc(a);
            a -= q;
            o[s * slice] = (int8_t)(int)q;
        }
    }
}

void ozaki_split(Ctx& c, const double* X, long si, long sk, int R, int K, int rpad, int kpad, int8_t* out, long slice,
                 int* e) {
    const int warps = 8;
    ozaki_split_kernel<<<(rpad + warps - 1) / warps, warps * 32, 0, c.stream>>>(X, si, sk, R, K, rpad, kpad, out, slice, e);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

void ozaki_gemm(Ctx& c, const OzProblem* d_probs, const int* d_tiles, int ntiles, int* d_status) {
    static bool attr = false;
    if (!attr) {
        RA_CUDA(cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(OzSmem)));
        attr = true;
    }
    ozaki_gemm_kernel<<<ntiles, OZ_THREADS, sizeof(OzSmem), c.stream>>>(d_probs, reinterpret_cast<const int4*>(d_tiles),
                                                                         d_status);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

std::vector<int> ozaki_tiles(const std::vector<OzProblem>& probs) {
    std::vector<int> t;
    for (size_t p = 0; p < probs.size(); ++p) {
        const OzProblem& q = probs[p];
        for (int mt = 0; mt * OZ_BM < q.M; ++mt)
            for (int nt = 0; nt * OZ_BN < q.N; ++nt) {
                t.push_back((int)p);
                t.push_back(mt);
                t.push_back(nt);
                t.push_back(0);
            }
    }
    return t;
}

int oz_round_m(int m) { return (m + OZ_BM - 1) / OZ_BM * OZ_BM; }
int oz_round_n(int n) { return (n + OZ_BN - 1) / OZ_BN * OZ_BN; }
int oz_round_k(int k) { return (k + OZ_BK - 1) / OZ_BK * OZ_BK; }

// ---------------------------------------------------------------------------
// Allocation-free form of the split-precision product (ra_mixed_gemm_noalloc).
//
// All scratch lives in one file-scope device array of fixed size; its device
// address is looked up once per device (cudaGetSymbolAddress, with that device
// current) on the first call made on that device.  Scratch layout, every piece
// 256-byte aligned:
//   [0]        int   status word      (set to zero by oz_static_prepare_kernel)
//   [256]      OzProblem              (written by oz_static_prepare_kernel)
//   [512]      int4  tiles[ntiles]    (written by oz_static_prepare_kernel)
//   then       int   ea[mp], eb[np]   (written by the split kernel)
//   then       int8  A digits [S][mp][kp], B digits [S][np][kp] (split kernel)
// Nothing else needs to start at zero: the split kernel writes every padded
// digit and every exponent the product reads.  Calls on one device share the
// array, so calls that overlap in time (two host threads, or two streams)
// race on it.
// ---------------------------------------------------------------------------
constexpr size_t OZ_STATIC_BYTES = (size_t)16 << 20;   // 16 MiB
static __device__ __align__(256) unsigned char oz_static_scratch[OZ_STATIC_BYTES];

constexpr int OZ_MAX_DEVICES = 64;
static unsigned char* oz_static_ptr[OZ_MAX_DEVICES] = {};

static size_t oz_align256(size_t x) { return (x + 255) & ~(size_t)255; }

__global__ void oz_static_prepare_kernel(OzProblem pr, OzProblem* __restrict__ dprob, int4* __restrict__ tiles,
                                         int ntm, int ntn, int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        *dprob = pr;
        *status = 0;
    }
    if (i < ntm * ntn) tiles[i] = make_int4(0, i / ntn, i % ntn, 0);
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
    const int mp = oz_round_m(m), np = oz_round_n(n), kp = oz_round_k(k);
    const int ntm = mp / 128, ntn = np / 64, ntiles = ntm * ntn;
    const size_t off_prob = 256, off_tiles = 512;
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
    if (e != cudaSuccess || dev < 0 || dev >= OZ_MAX_DEVICES) {
        oz_set_msg(msg, msg_len, "ra_mixed_gemm_noalloc: no usable current device");
        return RA_ERR_CUDA;
    }
    if (!oz_static_ptr[dev]) {   // first call on this device: resolve the scratch address
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, oz_static_scratch);
        if (e != cudaSuccess || !p) {
            oz_set_msg(msg, msg_len, cudaGetErrorString(e));
            return RA_ERR_CUDA;
        }
        oz_static_ptr[dev] = static_cast<unsigned char*>(p);
    }
    unsigned char* base = oz_static_ptr[dev];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int* d_status = reinterpret_cast<int*>(base);
    OzProblem* d_prob = reinterpret_cast<OzProblem*>(base + off_prob);
    int4* d_tiles = reinterpret_cast<int4*>(base + off_tiles);
    int* ea = reinterpret_cast<int*>(base + off_ea);
    int* eb = reinterpret_cast<int*>(base + off_eb);
    int8_t* sa = reinterpret_cast<int8_t*>(base + off_sa);
    int8_t* sb = reinterpret_cast<int8_t*>(base + off_sb);

    OzProblem pr{sa, sb, (long)mp * kp, (long)np * kp, ea, eb, m, n, kp, d_c, n, 1};
    oz_static_prepare_kernel<<<(ntiles + 127) / 128, 128, 0, st>>>(pr, d_prob, d_tiles, ntm, ntn, d_status);
    ozaki_split_kernel<<<(mp + 7) / 8, 256, 0, st>>>(d_a, k, 1, m, k, mp, kp, sa, (long)mp * kp, ea);
    ozaki_split_kernel<<<(np + 7) / 8, 256, 0, st>>>(d_b, 1, n, n, k, np, kp, sb, (long)np * kp, eb);
    e = cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(OzSmem));
    if (e == cudaSuccess) {
        ozaki_gemm_kernel<<<ntiles, OZ_THREADS, sizeof(OzSmem), st>>>(d_prob, d_tiles, d_status);
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

