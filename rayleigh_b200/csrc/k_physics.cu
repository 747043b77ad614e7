// Physical-space stage, fused per (r, theta) row:
//   Phi_Derivatives           (Sphere_Physical_Space.F90:745-759) in the spectrum load,
//   fft_to_physical  (c2r)    (Fourier_Transform.F90:142-183), 14 fields,
//   sintheta_div + NL terms   (Sphere_Physical_Space.F90:98-224, 303-700),
//   Find_MyMinDT (CFL max)    (:784-813),
//   fft_to_spectral (r2c)     (Fourier_Transform.F90:100-140), 4 fields,
//   equatorial fold of PtS    (Legendre_Transforms.F90:1109-1122),
// reading the inverse Legendre output p2a[theta_h][m][par][f][r][re/im] (E, O) and
// writing the folded p2b[m][par][theta_h][f][r][re/im] for m <= l_max.  The
// reference materialises the packed (n_phi+2, r, theta, f) buffers p3a/p3b
// between these steps; here the 18 phi rows of one (r, theta) point never
// leave the SM.
//
// One CTA (256 threads, two per SM) handles one row; the rows theta and
// pi - theta are the two CTAs of a cluster, which fold their spectra through
// distributed shared memory.  The 14 input fields go through the FFT two at a
// time; the four nonlinear outputs accumulate in shared memory (each thread
// owns its points), the velocity in registers.
//
// FFT: a real length-2N transform through one complex length-N transform
// (N = n_theta = 2^a 3^b), Stockham autosort, radix 8/4/2/3, in shared memory;
// unnormalised like FFTW (the normalisation lives in the Legendre tables).
#include <cmath>

#include <cooperative_groups.h>

#include "ra_internal.h"

namespace ra {

struct FFTPlan {
    int n;
    int npass;
    int radix[16];
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// exp(sign * 2 pi i e / N) from wr[k] = exp(2 pi i k / (2N)), k < N
__device__ __forceinline__ double2 twiddle(const double2* wr, int N, int e, int sign) {
    double2 w = (2 * e < N) ? wr[2 * e] : make_double2(-wr[2 * e - N].x, -wr[2 * e - N].y);
    if (sign < 0) w.y = -w.y;
    return w;
}

__device__ __forceinline__ void dft4(double2& u0, double2& u1, double2& u2, double2& u3, int sign) {
    const double2 t0 = cadd(u0, u2), t1 = csub(u0, u2);
    const double2 t2 = cadd(u1, u3), d = csub(u1, u3);
    // w = sign * i : w * (x + i y) = sign * (-y + i x)
    const double2 wd = make_double2(-sign * d.y, sign * d.x);
    u0 = cadd(t0, t2);
    u2 = csub(t0, t2);
    u1 = cadd(t1, wd);
    u3 = csub(t1, wd);
}

__device__ __forceinline__ void dft_small(int R, double2* u, int sign) {
    if (R == 2) {
        const double2 a = u[0], b = u[1];
        u[0] = cadd(a, b);
        u[1] = csub(a, b);
    } else if (R == 4) {
        dft4(u[0], u[1], u[2], u[3], sign);
    } else if (R == 8) {
        const double H = 0.70710678118654752440;   // sqrt(2)/2
        double2 a0 = cadd(u[0], u[4]), a1 = cadd(u[1], u[5]), a2 = cadd(u[2], u[6]), a3 = cadd(u[3], u[7]);
        double2 b0 = csub(u[0], u[4]), b1 = csub(u[1], u[5]), b2 = csub(u[2], u[6]), b3 = csub(u[3], u[7]);
        // b_j *= exp(sign i pi j / 4)
        b1 = make_double2(H * (b1.x - sign * b1.y), H * (b1.y + sign * b1.x));
        b2 = make_double2(-sign * b2.y, sign * b2.x);
        b3 = make_double2(H * (-b3.x - sign * b3.y), H * (-b3.y + sign * b3.x));
        dft4(a0, a1, a2, a3, sign);
        dft4(b0, b1, b2, b3, sign);
        u[0] = a0; u[2] = a1; u[4] = a2; u[6] = a3;
        u[1] = b0; u[3] = b1; u[5] = b2; u[7] = b3;
    } else {  // R == 3
        const double S3 = 0.86602540378443864676;
        const double2 t = cadd(u[1], u[2]), d = csub(u[1], u[2]);
        const double2 a = make_double2(u[0].x - 0.5 * t.x, u[0].y - 0.5 * t.y);
        const double2 sd = make_double2(-sign * S3 * d.y, sign * S3 * d.x);
        u[0] = cadd(u[0], t);
        u[1] = cadd(a, sd);
        u[2] = csub(a, sd);
    }
}

// Runs nb independent FFTs of length N stored at a + b*N (b < nb), scratch at
// bb + b*N; returns the buffer base holding the results.  Must be entered with
// a synchronised input; leaves the result synchronised.
__device__ double2* fft_run(double2* a, double2* bb, int nb, const FFTPlan& pl, const double2* wr, int sign) {
    const int N = pl.n;
    int p = 1;
    double2* src = a;
    double2* dst = bb;
    for (int ps = 0; ps < pl.npass; ++ps) {
        const int R = pl.radix[ps];
        const int T = N / R;
        const int stride = N / (p * R);
        for (int g = threadIdx.x; g < T * nb; g += blockDim.x) {
            const int b = g / T, bi = g - b * T;
            const double2* sb = src + b * N;
            double2* db = dst + b * N;
            const int k = bi % p;
            double2 u[8];
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (r < R) u[r] = sb[bi + r * T];
#pragma unroll
            for (int r = 1; r < 8; ++r)
                if (r < R) u[r] = cmul(u[r], twiddle(wr, N, r * k * stride, sign));
            dft_small(R, u, sign);
            const int j = (bi - k) * R + k;
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (r < R) db[j + r * p] = u[r];
        }
        __syncthreads();
        double2* t = src;
        src = dst;
        dst = t;
        p *= R;
    }
    return src;
}

// ---- compile-time plans: the same greedy radix order as make_plan (8, 4, 2, 3) ----
__host__ __device__ constexpr int radix_at(int n, int i) {
    int m = n, k = 0;
    while (m % 8 == 0) { if (k == i) return 8; m /= 8; ++k; }
    while (m % 4 == 0) { if (k == i) return 4; m /= 4; ++k; }
    while (m % 2 == 0) { if (k == i) return 2; m /= 2; ++k; }
    while (m % 3 == 0) { if (k == i) return 3; m /= 3; ++k; }
    return 0;
}
__host__ __device__ constexpr int npass_of(int n) {
    int k = 0;
    while (radix_at(n, k) != 0) ++k;
    return k;
}
__host__ __device__ constexpr int pprod(int n, int i) {
    int p = 1;
    for (int j = 0; j < i; ++j) p *= radix_at(n, j);
    return p;
}

// Shared-memory index swizzle for the FFT buffers: permutes the 8 complex
// values of each aligned group by XOR with the next 3 index bits, which makes the
// stride-R writes of the first Stockham passes bank-conflict free.
__device__ __forceinline__ int SW(int i) { return i ^ ((i >> 3) & 7); }

// Stride between the fields of a batched buffer: a multiple of 64, so that a
// field's swizzled indices stay inside the field whatever buffer it sits in.
__host__ __device__ constexpr int fstride(int n) { return (n + 63) / 64 * 64; }

// Offsets of the per-pass twiddle tables tw[(r-1) P + k] = exp(2 pi i r k STRIDE / N).
__host__ __device__ constexpr int tw_off(int n, int ps) {
    int o = 0;
    for (int j = 0; j < ps; ++j) o += (radix_at(n, j) - 1) * pprod(n, j);
    return o;
}
__host__ __device__ constexpr int tw_size(int n) { return tw_off(n, npass_of(n)); }

// Builds the per-pass tables from the global table wr[k] = exp(2 pi i k / 2N).
template <int N, int NT, int PS = 0>
__device__ __forceinline__ void build_twiddles(double2* tw, const double2* __restrict__ wrg) {
    if constexpr (PS < npass_of(N)) {
        constexpr int R = radix_at(N, PS), P = pprod(N, PS), STRIDE = N / (P * R);
        for (int idx = threadIdx.x; idx < (R - 1) * P; idx += NT) {
            const int r = idx / P + 1, k = idx - (r - 1) * P;
            const int e = (r * k * STRIDE) % N;
            tw[tw_off(N, PS) + idx] = (2 * e < N) ? wrg[2 * e] : make_double2(-wrg[2 * e - N].x, -wrg[2 * e - N].y);
        }
        build_twiddles<N, NT, PS + 1>(tw, wrg);
    }
}

template <int N, int NB, int NT, int PS>
__device__ __forceinline__ void fft_pass_t(const double2* __restrict__ src, double2* __restrict__ dst,
                                           const double2* __restrict__ tw, int sign, int tid) {
    constexpr int R = radix_at(N, PS);
    constexpr int P = pprod(N, PS);
    constexpr int T = N / R;
    constexpr int TO = tw_off(N, PS);
#pragma unroll 1
    for (int g = tid; g < T * NB; g += NT) {
        const int b = g / T, bi = g - b * T;
        const int base = b * fstride(N);
        const int k = bi % P;
        double2 u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = src[SW(base + bi + r * T)];
        if (P > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                double2 w = tw[TO + (r - 1) * P + k];
                if (sign < 0) w.y = -w.y;
                u[r] = cmul(u[r], w);
            }
        }
        dft_small(R, u, sign);
        const int j = (bi - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[SW(base + j + r * P)] = u[r];
    }
}

template <int N, int NB, int NT, int PS = 0>
__device__ __forceinline__ double2* fft_run_t(double2* a, double2* b, const double2* tw, int sign, int tid) {
    if constexpr (PS < npass_of(N)) {
        fft_pass_t<N, NB, NT, PS>(a, b, tw, sign, tid);
        __syncthreads();
        return fft_run_t<N, NB, NT, PS + 1>(b, a, tw, sign, tid);
    } else {
        return a;
    }
}

struct PhysParams {
    const double* p2a;
    double* p2b;
    const double* radial;   // packed radial profiles
    const double* trig;     // [4][nth]: cos, sin, csc, cot
    const double2* wr;      // [nth] exp(2 pi i k / n_phi)
    unsigned long long* cfl;
    int L, nth, nr, ncola, ncolb;
    double coriolis;
    int rotation;
    double llmax;
};

// One CTA = one (theta, r) row; the rows theta and pi - theta of a pair form a
// 2-CTA cluster that folds its spectra through distributed shared memory.
constexpr int ROW_THREADS = 256;
constexpr int FB = 2;   // fields per batched FFT

// Shared memory of a row CTA (double2 units): two FFT ping-pong buffers of FB
// fields, the four nonlinear outputs (W, P, T, Z; each thread owns its points),
// the per-pass twiddle tables.
template <int N>
struct RowSmem {
    static constexpr int FS = fstride(N);
    static constexpr int A = 0, B = FB * FS, ACC = 2 * FB * FS, TW = ACC + 4 * FS;
    static constexpr int SIZE = TW + tw_size(N);
};

// Runs the Stockham passes PS .. PE-1 (ping-pong a -> b -> a ...); returns the
// buffer holding the result.
template <int N, int NB, int NT, int PS, int PE>
__device__ __forceinline__ double2* fft_range(double2* a, double2* b, const double2* tw, int sign, int tid) {
    if constexpr (PS < PE) {
        fft_pass_t<N, NB, NT, PS>(a, b, tw, sign, tid);
        __syncthreads();
        return fft_range<N, NB, NT, PS + 1, PE>(b, a, tw, sign, tid);
    } else {
        return a;
    }
}

// One spectrum value of this row: X = E + O (south, h = 0) or E - O (north,
// h = 1), as StP_4d_dgp2 reflects the even-l / odd-l products
// (Legendre_Transforms.F90:1030-1064); d/dphi (i m X) when dp; Im X_0 = 0 as
// FFTW's c2r ignores it; X_m = 0 for m >= L.
__device__ __forceinline__ double2 spec_value(const double* __restrict__ base, long mstride, long ostride, int m,
                                              int L, int h, bool dp) {
    if (m >= L) return make_double2(0.0, 0.0);
    const double2 e = __ldg(reinterpret_cast<const double2*>(base + m * mstride));
    const double2 o = __ldg(reinterpret_cast<const double2*>(base + m * mstride + ostride));
    double2 x = h ? csub(e, o) : cadd(e, o);
    if (dp) x = make_double2(-m * x.y, m * x.x);
    if (m == 0) x.y = 0.0;
    return x;
}

// Half-length complex input of the real transform:
//   Z_k = (X_k + conj X_{N-k}) + i w^k (X_k - conj X_{N-k}),  w = exp(2 pi i / 2N).
__device__ __forceinline__ double2 zform(double2 xk, double2 xn, double2 wk) {
    const double2 e = cadd(xk, cconj(xn));
    const double2 d = csub(xk, cconj(xn));
    const double2 wd = cmul(wk, d);
    return make_double2(e.x - wd.y, e.y + wd.x);
}

// Whether the last Stockham pass leaves, per thread t, the outputs n = t + q*ROW_THREADS
// of every field (then it is run straight into registers).
template <int N>
__host__ __device__ constexpr bool last_pass_in_regs() {
    return N / radix_at(N, npass_of(N) - 1) == ROW_THREADS;
}

// Forms the half-length complex FFT input Z_k (zform) of FB fields of this row
// in buffer A straight from the spectra in p2a (spec_value): one work item is
// the pair (k, N-k), whose two Z values need the same two spectrum values.
template <int N>
__device__ __forceinline__ void c2r_stage(const PhysParams& P, const double* __restrict__ rowbase, int h, int f0,
                                          bool d0, int f1, bool d1, double2* bA, int t) {
    constexpr int FS = fstride(N);
    constexpr int NI = N / 2 + 1;                                   // k = 0 .. N/2
    constexpr int QI = (FB * NI + ROW_THREADS - 1) / ROW_THREADS;   // items per thread
    const int L = P.L;
    const long ostride = (long)P.ncola;   // E -> O within p2a[theta_h][m][par][col]
    const long mstride = 2L * P.ncola;
    double2 xk[QI], xn[QI];
#pragma unroll
    for (int q = 0; q < QI; ++q) {
        const int g = t + q * ROW_THREADS;
        xk[q] = xn[q] = make_double2(0.0, 0.0);
        if (g < FB * NI) {
            const int b = g / NI, k = g - b * NI;
            const double* base = rowbase + (long)(b ? f1 : f0) * P.nr * 2;
            const bool dp = b ? d1 : d0;
            xk[q] = spec_value(base, mstride, ostride, k, L, h, dp);
            xn[q] = spec_value(base, mstride, ostride, N - k, L, h, dp);   // N - k >= L for k = 0
        }
    }
#pragma unroll
    for (int q = 0; q < QI; ++q) {
        const int g = t + q * ROW_THREADS;
        if (g < FB * NI) {
            const int b = g / NI, k = g - b * NI;
            bA[SW(b * FS + k)] = zform(xk[q], xn[q], __ldg(P.wr + k));
            if (k != 0 && 2 * k != N) bA[SW(b * FS + N - k)] = zform(xn[q], xk[q], __ldg(P.wr + N - k));
        }
    }
    __syncthreads();
}

// c2r of FB fields of this row: y[b][q] = (y[2n], y[2n+1]) of field b at n = t + q*ROW_THREADS.
template <int N, int ZPT>
__device__ __forceinline__ void row_c2r(const PhysParams& P, const double* __restrict__ rowbase, int h, int f0,
                                        bool d0, int f1, bool d1, double2* sm, const double2* tw, int t,
                                        double2 (&y)[FB][ZPT]) {
    constexpr int FS = fstride(N), NP = npass_of(N);
    double2* bA = sm + RowSmem<N>::A;
    double2* bB = sm + RowSmem<N>::B;
    c2r_stage<N>(P, rowbase, h, f0, d0, f1, d1, bA, t);
    if constexpr (last_pass_in_regs<N>()) {
        const double2* src = fft_range<N, FB, ROW_THREADS, 0, NP - 1>(bA, bB, tw, +1, t);
        constexpr int PS = NP - 1, R = radix_at(N, PS), PP = pprod(N, PS), TO = tw_off(N, PS);
        static_assert(R == ZPT, "last radix must equal the points per thread");
#pragma unroll
        for (int b = 0; b < FB; ++b) {
            double2 u[R];
#pragma unroll
            for (int r = 0; r < R; ++r) u[r] = src[SW(b * FS + t + r * ROW_THREADS)];
            if (PP > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) u[r] = cmul(u[r], tw[TO + (r - 1) * PP + t]);
            }
            dft_small(R, u, +1);
#pragma unroll
            for (int r = 0; r < R; ++r) y[b][r] = u[r];
        }
    } else {
        const double2* res = fft_range<N, FB, ROW_THREADS, 0, NP>(bA, bB, tw, +1, t);
#pragma unroll
        for (int b = 0; b < FB; ++b)
#pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                const int n = t + q * ROW_THREADS;
                y[b][q] = (n < N) ? res[SW(b * FS + n)] : make_double2(0.0, 0.0);
            }
    }
}

// r2c of two of the accumulated outputs (acc fields a0, a0+1): Z = FFT(y[2n] + i y[2n+1]),
// X_k = e - i conj(w^k) d with e, d the half sums/differences of Z_k, conj Z_{N-k};
// X_k (k < L) is written back over the two acc fields.
template <int N>
__device__ __forceinline__ void row_r2c_pair(const PhysParams& P, int a0, double2* sm, const double2* tw, int t) {
    constexpr int FS = fstride(N);
    double2* acc = sm + RowSmem<N>::ACC + a0 * FS;
    double2* bA = sm + RowSmem<N>::A;
    double2* bB = sm + RowSmem<N>::B;
    fft_pass_t<N, FB, ROW_THREADS, 0>(acc, bA, tw, -1, t);
    __syncthreads();
    const double2* Z = fft_run_t<N, FB, ROW_THREADS, 1>(bA, bB, tw, -1, t);
    const int L = P.L;
    for (int g = t; g < FB * L; g += ROW_THREADS) {
        const int f = g / L, k = g - f * L;
        const double2 zk = Z[SW(f * FS + k)];
        const double2 zn = cconj(Z[SW(f * FS + (N - k) % N)]);
        const double2 e = make_double2(0.5 * (zk.x + zn.x), 0.5 * (zk.y + zn.y));
        const double2 d = make_double2(0.5 * (zk.x - zn.x), 0.5 * (zk.y - zn.y));
        const double2 wd = cmul(cconj(__ldg(P.wr + k)), d);
        double2 Xk = make_double2(e.x + wd.y, e.y - wd.x);
        if (k == 0) Xk.y = 0.0;
        acc[SW(f * FS + k)] = Xk;
    }
    __syncthreads();
}

template <int NTH>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(ROW_THREADS, 2) physics_kernel(PhysParams P) {
    constexpr int N = NTH;
    constexpr int FS = fstride(N);
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    double2* tw = sm + RowSmem<N>::TW;
    double2* acc = sm + RowSmem<N>::ACC;
    __shared__ double red[ROW_THREADS / 32];
    const int t = threadIdx.x;
    const int h = (int)cluster.block_rank();        // 0: theta (south half), 1: pi - theta
    build_twiddles<N, ROW_THREADS>(tw, P.wr);
    const int nr = P.nr;
    const int pair = blockIdx.x >> 1;
    const int r = pair % nr;
    const int thh = pair / nr;
    const int th = h ? (N - 1 - thh) : thh;
    const double rad = P.radial[R_RADIUS * nr + r];
    const double orad = P.radial[R_OVER_R * nr + r];
    const double rho = P.radial[R_DENSITY * nr + r];
    const double dlnrho = P.radial[R_DLNRHO * nr + r];
    const double dr = P.radial[R_DELTA_R * nr + r];
    const double cs = P.trig[th], sn = P.trig[N + th], csc = P.trig[2 * N + th], cot = P.trig[3 * N + th];
    const double cor = P.rotation ? P.coriolis : 0.0;
    const double c2r = csc * csc * orad;
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * 2;
    __syncthreads();

    double2 vr[ZPT], vt[ZPT], vp[ZPT];
    double2 y[FB][ZPT];
    auto acc_at = [&](int f, int q) -> double2& { return acc[SW(f * FS + t + q * ROW_THREADS)]; };
    auto live = [&](int q) { return t + q * ROW_THREADS < N; };
    // B1: v_r, v_theta
    row_c2r<N, ZPT>(P, rowbase, h, A_VR, false, A_VT, false, sm, tw, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        vr[q] = y[0][q];
        vt[q] = y[1][q];
        vt[q].x *= csc;
        vt[q].y *= csc;
    }
    __syncthreads();
    // B2: v_phi, dv_r/dr: the quadratic, Coriolis and radial-advection terms
    row_c2r<N, ZPT>(P, rowbase, h, A_VP, false, A_DVRDR, false, sm, tw, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        vp[q] = y[0][q];
        vp[q].x *= csc;
        vp[q].y *= csc;
        const double2 x = y[1][q];
        auto w0 = [&](double a, double b, double c, double xx) {
            return rho * (rad * b * b + rad * c * c + cor * sn * rad * rad * c) - rho * rad * rad * a * xx;
        };
        auto p0 = [&](double a, double b, double c, double xx) {
            return -b * b * cot * orad - b * a * orad - b * a * dlnrho - c * c * cot * orad - cor * cs * c - b * xx;
        };
        auto z0 = [&](double a, double b, double c) { return c * a * orad + cor * (cs * b + sn * a); };
        if (live(q)) {
            acc_at(0, q) = make_double2(w0(vr[q].x, vt[q].x, vp[q].x, x.x), w0(vr[q].y, vt[q].y, vp[q].y, x.y));
            acc_at(1, q) = make_double2(p0(vr[q].x, vt[q].x, vp[q].x, x.x), p0(vr[q].y, vt[q].y, vp[q].y, x.y));
            acc_at(2, q) = make_double2(0.0, 0.0);
            acc_at(3, q) = make_double2(z0(vr[q].x, vt[q].x, vp[q].x), z0(vr[q].y, vt[q].y, vp[q].y));
        }
    }
    __syncthreads();
    // B3: dv_r/dtheta, dv_r/dphi
    row_c2r<N, ZPT>(P, rowbase, h, A_DVRDT, false, A_VR, true, sm, tw, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        if (!live(q)) continue;
        const double2 a = y[0][q], b = y[1][q];
        double2& w = acc_at(0, q);
        w.x += -rho * rad * vt[q].x * a.x * csc - rho * rad * csc * vp[q].x * b.x;
        w.y += -rho * rad * vt[q].y * a.y * csc - rho * rad * csc * vp[q].y * b.y;
    }
    __syncthreads();
    // B4: dv_theta/dr, dv_theta/dphi
    row_c2r<N, ZPT>(P, rowbase, h, A_DVTDR, false, A_VT, true, sm, tw, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        if (!live(q)) continue;
        const double2 c = y[0][q], d = y[1][q];
        double2& pp = acc_at(1, q);
        double2& z = acc_at(3, q);
        pp.x += vr[q].x * c.x * csc + vp[q].x * d.x * c2r;
        pp.y += vr[q].y * c.y * csc + vp[q].y * d.y * c2r;
        z.x += vt[q].x * d.x * c2r;
        z.y += vt[q].y * d.y * c2r;
    }
    __syncthreads();
    // B5: dv_phi/dr, dv_phi/dphi
    row_c2r<N, ZPT>(P, rowbase, h, A_DVPDR, false, A_VP, true, sm, tw, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        if (!live(q)) continue;
        const double2 a = y[0][q], b = y[1][q];
        double2& pp = acc_at(1, q);
        double2& z = acc_at(3, q);
        z.x += vr[q].x * a.x * csc + vp[q].x * b.x * c2r;
        z.y += vr[q].y * a.y * csc + vp[q].y * b.y * c2r;
        pp.x += -vt[q].x * b.x * c2r;
        pp.y += -vt[q].y * b.y * c2r;
    }
    __syncthreads();
    // B6: omega_r, dT/dr
    row_c2r<N, ZPT>(P, rowbase, h, A_OMR, false, A_DTDR, false, sm, tw, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        if (!live(q)) continue;
        const double2 c = y[0][q], d = y[1][q];
        double2& z = acc_at(3, q);
        double2& tt = acc_at(2, q);
        z.x += vt[q].x * c.x;
        z.y += vt[q].y * c.y;
        tt.x += -vr[q].x * d.x;
        tt.y += -vr[q].y * d.y;
    }
    __syncthreads();
    // B7: dT/dtheta, dT/dphi
    row_c2r<N, ZPT>(P, rowbase, h, A_DTDT, false, A_T, true, sm, tw, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        if (!live(q)) continue;
        const double2 a = y[0][q], b = y[1][q];
        double2& tt = acc_at(2, q);
        tt.x += -a.x * csc * vt[q].x * orad - vp[q].x * b.x * csc * orad;
        tt.y += -a.y * csc * vt[q].y * orad - vp[q].y * b.y * csc * orad;
    }
    // CFL (Find_MyMinDT) and the rho r sin(theta) factor of the P and Z terms
    double cmax = 0.0;
    const double hfac = P.llmax * orad * orad, rfac = 1.0 / (dr * dr);
    const double sfac = rho * rad * csc;
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        if ((t + q * ROW_THREADS) < N) {
            cmax = fmax(cmax, (vt[q].x * vt[q].x + vp[q].x * vp[q].x) * hfac);
            cmax = fmax(cmax, (vt[q].y * vt[q].y + vp[q].y * vp[q].y) * hfac);
            cmax = fmax(cmax, vr[q].x * vr[q].x * rfac);
            cmax = fmax(cmax, vr[q].y * vr[q].y * rfac);
            double2& pp = acc_at(1, q);
            double2& z = acc_at(3, q);
            pp.x *= sfac; pp.y *= sfac;
            z.x *= sfac; z.y *= sfac;
        }
    }
    __syncthreads();
    // r2c of W, P and of T, Z; the spectra X_k (k < L) replace the accumulators
    row_r2c_pair<N>(P, 0, sm, tw, t);
    row_r2c_pair<N>(P, 2, sm, tw, t);
    // equatorial fold of PtS_4d_dgpv3 (Legendre_Transforms.F90:1109-1122) with the
    // partner row: f_even = X(theta) + X(pi - theta) (written by rank 0),
    // f_odd = X(theta) - X(pi - theta) (written by rank 1)
    cluster.sync();
    {
        const double2* mine = acc;
        const double2* peer = cluster.map_shared_rank(acc, h ^ 1);
        const int L = P.L;
        const long mstride = 2L * (P.nth / 2) * P.ncolb;   // p2b[m][par][theta_h][col]
        double* obase = P.p2b + (long)h * (P.nth / 2) * P.ncolb + (long)thh * P.ncolb + (long)r * 2;
        for (int g = t; g < 4 * L; g += ROW_THREADS) {
            const int f = g / L, k = g - f * L;
            const double2 a = mine[SW(f * FS + k)], b = peer[SW(f * FS + k)];
            const double2 v = h ? csub(b, a) : cadd(a, b);
            *reinterpret_cast<double2*>(obase + k * mstride + (long)f * P.nr * 2) = v;
        }
    }
    // CFL max over the row
    for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_down_sync(0xffffffffu, cmax, o));
    if ((t & 31) == 0) red[t >> 5] = cmax;
    cluster.sync();   // the partner has finished reading this CTA's spectra
    if (t == 0) {
        double v = red[0];
        for (int i = 1; i < ROW_THREADS / 32; ++i) v = fmax(v, red[i]);
        atomicMax(P.cfl, (unsigned long long)__double_as_longlong(v));
    }
}

FFTPlan make_plan(int n) {
    FFTPlan p{};
    p.n = n;
    int m = n;
    while (m % 8 == 0) { p.radix[p.npass++] = 8; m /= 8; }
    while (m % 4 == 0) { p.radix[p.npass++] = 4; m /= 4; }
    while (m % 2 == 0) { p.radix[p.npass++] = 2; m /= 2; }
    while (m % 3 == 0) { p.radix[p.npass++] = 3; m /= 3; }
    if (m != 1) throw ArgError("n_theta must be of the form 2^a 3^b for the phi FFT");
    return p;
}

void launch_physics(Ctx& c) {
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.p2b = c.d_p2b;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.cfl = c.d_cfl;
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = NP2A * c.d.nr * 2;
    P.ncolb = NP2B * c.d.nr * 2;
    P.coriolis = c.rad.coriolis;
    P.rotation = c.cfg.rotation;
    P.llmax = (double)c.d.lmax * (c.d.lmax + 1);
    make_plan(c.d.nth);   // validates n_theta = 2^a 3^b
    const unsigned grid = 2u * (unsigned)c.d.nth2 * (unsigned)c.d.nr;   // clusters of 2 rows
    auto go = [&](auto kern, int n, size_t smem_units) {
        const size_t smem = smem_units * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, ROW_THREADS, smem, c.stream>>>(P);
        (void)n;
    };
    switch (c.d.nth) {
        case 24: go(physics_kernel<24>, 24, RowSmem<24>::SIZE); break;
        case 32: go(physics_kernel<32>, 32, RowSmem<32>::SIZE); break;
        case 48: go(physics_kernel<48>, 48, RowSmem<48>::SIZE); break;
        case 64: go(physics_kernel<64>, 64, RowSmem<64>::SIZE); break;
        case 96: go(physics_kernel<96>, 96, RowSmem<96>::SIZE); break;
        case 128: go(physics_kernel<128>, 128, RowSmem<128>::SIZE); break;
        case 192: go(physics_kernel<192>, 192, RowSmem<192>::SIZE); break;
        case 256: go(physics_kernel<256>, 256, RowSmem<256>::SIZE); break;
        case 384: go(physics_kernel<384>, 384, RowSmem<384>::SIZE); break;
        case 512: go(physics_kernel<512>, 512, RowSmem<512>::SIZE); break;
        case 768: go(physics_kernel<768>, 768, RowSmem<768>::SIZE); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) +
                                " has no physical-space kernel instance (24..768 of the form 2^a or 3*2^a)");
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

__global__ void fft_rows_kernel(double* x, long howmany, const double2* wrg, FFTPlan plan, int inverse) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = plan.n;
    double2* a = reinterpret_cast<double2*>(smem_raw);
    double2* b = a + N;
    double2* wr = b + N;
    for (int k = threadIdx.x; k < N; k += blockDim.x) wr[k] = wrg[k];
    double* row = x + (long)blockIdx.x * (2 * N + 2);
    __syncthreads();
    if (inverse) {
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            double2 xk = make_double2(row[2 * k], row[2 * k + 1]);
            double2 xn = make_double2(row[2 * (N - k)], row[2 * (N - k) + 1]);
            if (k == 0) { xk.y = 0.0; xn.y = 0.0; }
            if (k == 0) xn = make_double2(row[2 * N], 0.0);
            const double2 e = cadd(xk, cconj(xn));
            const double2 d = csub(xk, cconj(xn));
            const double2 wd = cmul(wr[k], d);
            a[k] = make_double2(e.x - wd.y, e.y + wd.x);
        }
        __syncthreads();
        double2* res = fft_run(a, b, 1, plan, wr, +1);
        for (int n = threadIdx.x; n < N; n += blockDim.x) {
            row[2 * n] = res[n].x;
            row[2 * n + 1] = res[n].y;
        }
        __syncthreads();
        if (threadIdx.x == 0) { row[2 * N] = 0.0; row[2 * N + 1] = 0.0; }
    } else {
        for (int n = threadIdx.x; n < N; n += blockDim.x) a[n] = make_double2(row[2 * n], row[2 * n + 1]);
        __syncthreads();
        double2* Z = fft_run(a, b, 1, plan, wr, -1);
        for (int k = threadIdx.x; k <= N; k += blockDim.x) {
            const double2 zk = Z[k % N];
            const double2 zn = cconj(Z[(N - k) % N]);
            const double2 e = make_double2(0.5 * (zk.x + zn.x), 0.5 * (zk.y + zn.y));
            const double2 d = make_double2(0.5 * (zk.x - zn.x), 0.5 * (zk.y - zn.y));
            double2 w = (k < N) ? cconj(wr[k]) : make_double2(-1.0, 0.0);
            const double2 wd = cmul(w, d);
            double2 X = make_double2(e.x + wd.y, e.y - wd.x);
            if (k == 0 || k == N) X.y = 0.0;
            row[2 * k] = X.x;
            row[2 * k + 1] = X.y;
        }
    }
}

void launch_fft_rows(Ctx& c, double* d_x, long howmany, int inverse) {
    FFTPlan plan = make_plan(c.d.nth);
    const size_t smem = 3 * (size_t)c.d.nth * sizeof(double2);
    RA_CUDA(cudaFuncSetAttribute(fft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fft_rows_kernel<<<(unsigned)howmany, 256, smem, c.stream>>>(d_x, howmany, reinterpret_cast<const double2*>(c.d_twid),
                                                              plan, inverse);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

}  // namespace ra
