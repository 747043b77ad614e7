// Physical-space stage, fused per (r, theta) row:
//   Phi_Derivatives           (Sphere_Physical_Space.F90:745-759) in the spectrum load,
//   fft_to_physical  (c2r)    (Fourier_Transform.F90:142-183), 14 fields,
//   sintheta_div + NL terms   (Sphere_Physical_Space.F90:98-224, 303-700),
//   Find_MyMinDT (CFL max)    (:784-813),
//   fft_to_spectral (r2c)     (Fourier_Transform.F90:100-140), 4 fields,
//   equatorial fold of PtS    (Legendre_Transforms.F90:1109-1122),
// reading the inverse Legendre output p2a[theta_h][m][par][r][f][re/im] (E, O) and
// writing the folded p2b[m][par][theta_h][r][f][re/im] for m <= l_max.  The
// reference materialises the packed (n_phi+2, r, theta, f) buffers p3a/p3b
// between these steps; here the 18 phi rows of one (r, theta) point never
// leave the SM.
//
// One CTA (384 threads, two per SM) handles one row; the rows theta and
// pi - theta are the two CTAs of a cluster, which fold their spectra through
// distributed shared memory.  The 14 input fields go through the FFT in
// batches of four, four, four and two; the four nonlinear outputs accumulate
// in shared memory (each thread owns its points), the velocity in registers,
// the row's radial and colatitude factors in shared memory.  The same c2r
// serves the output-iteration diagnostics (kinetic energy, shell slices).
//
// FFT: a real length-2N transform through one complex length-N transform
// (N = n_theta = 2^a 3^b), in place in shared memory: decimation in frequency
// (radix 8, 4, 2, 3 passes) for the c2r, which leaves the physical points in
// a digit-reversed order; the nonlinear terms are pointwise in phi, so they
// are formed in that order, and the r2c runs the passes in reverse
// (decimation in time) back to natural order.  One twiddle table load per
// butterfly, the other powers by complex products; two passes deal their
// butterflies over pairs of fields so that shared accesses avoid bank
// conflicts (butterfly_of).  Unnormalised like FFTW (the normalisation lives
// in the Legendre tables).
#include <cmath>
#include <vector>
#include <algorithm>

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

// The same from a table in global memory (read-only path).
__device__ __forceinline__ double2 twiddle_g(const double2* __restrict__ wr, int N, int e, int sign) {
    double2 w;
    if (2 * e < N) {
        w = __ldg(wr + 2 * e);
    } else {
        const double2 v = __ldg(wr + 2 * e - N);
        w = make_double2(-v.x, -v.y);
    }
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
    } else if (R == 16) {
        // 16 = 4 x 4: DFT-4 over the elements q + 4p, twiddle w16^(q k1), DFT-4 over q;
        // output k1 + 4 k2
        const double C1 = 0.92387953251128675613, S1 = 0.38268343236508977173;   // cos, sin pi/8
        const double H = 0.70710678118654752440;                                  // cos pi/4
#pragma unroll
        for (int q = 0; q < 4; ++q) dft4(u[q], u[q + 4], u[q + 8], u[q + 12], sign);
        // element (q, k1) sits at u[q + 4 k1]; w16^e = (cos, sign sin)(2 pi e / 16)
        auto tw16 = [&](double2 a, int e) -> double2 {
            double c, sn;
            switch (e) {
                case 1: c = C1; sn = S1; break;
                case 2: c = H; sn = H; break;
                case 3: c = S1; sn = C1; break;
                case 4: c = 0.0; sn = 1.0; break;
                case 6: c = -H; sn = H; break;
                case 9: c = -C1; sn = -S1; break;
                default: c = 1.0; sn = 0.0; break;
            }
            sn *= sign;
            return make_double2(a.x * c - a.y * sn, a.x * sn + a.y * c);
        };
#pragma unroll
        for (int q = 1; q < 4; ++q)
#pragma unroll
            for (int k1 = 1; k1 < 4; ++k1) u[q + 4 * k1] = tw16(u[q + 4 * k1], q * k1);
        double2 v[16];
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            double2 a0 = u[0 + 4 * k1], a1 = u[1 + 4 * k1], a2 = u[2 + 4 * k1], a3 = u[3 + 4 * k1];
            dft4(a0, a1, a2, a3, sign);
            v[k1 + 0] = a0;
            v[k1 + 4] = a1;
            v[k1 + 8] = a2;
            v[k1 + 12] = a3;
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) u[k] = v[k];
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

// ---- compile-time plans of the in-place FFT: greedy radix order 16, 8, 4, 2, 3 ----
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

// Shared-memory index of a buffer position.  The in-place passes' strides
// (96, 12, 3, 1 at N = 768) conflict least with the identity map: an XOR
// swizzle of bits 3-5 cost 1.67 wavefronts per ideal one over all passes
// (the stride-1 radix-3 pass 2.5), the identity 1.33.
__device__ __forceinline__ int SW(int i) { return i; }

// Stride between the fields of a batched buffer (16-byte slots): 2 mod 8, so
// that the spectrum writes, whose lanes run over the batch's fields first, hit
// eight different bank groups per quarter warp (n is a multiple of 8).
__host__ __device__ constexpr int fstride(int n) { return n + 2; }

struct PhysParams {
    const double* p2a;
    double* p2b;
    const double* radial;   // packed radial profiles
    const double* trig;     // [4][nth]: cos, sin, csc, cot
    const double2* wr;      // [nth] exp(2 pi i k / n_phi)
    const double2* twp;     // per-pass FFT twiddles (ip_tw_off; one load per butterfly, twiddle_apply)
    unsigned long long* cfl;
    int L, nth, nr, ncola, ncolb;
    double coriolis;
    int rotation;
    double llmax;
    int nfa, nfb;           // fields per radius of p2a / p2b
    double lorentz;         // Lorentz_Coeff (magnetism)
};

// One CTA = one (theta, r) row; the rows theta and pi - theta of a pair form a
// 2-CTA cluster that folds its spectra through distributed shared memory.
constexpr int ROW_THREADS = 384;
enum { RC_RAD, RC_ORAD, RC_RHO, RC_DLNRHO, RC_DR, RC_CS, RC_SN, RC_CSC, RC_COT, RC_COR, RC_C2R, RC_HSF, RC_VH, RC_OH,
       RC_COUNT };
constexpr int FB = 4;   // fields per batched FFT

// Shared memory of a row CTA (double2 units): one in-place FFT buffer of FB
// fields and the four nonlinear outputs (W, P, T, Z; each thread owns its
// points; the r2c runs in place on them).
template <int N>
struct RowSmem {
    static constexpr int FS = fstride(N);
    static constexpr int BUF = 0, ACC = FB * FS;
    static constexpr int SIZE = ACC + 4 * FS;
};

// In-place mixed-radix FFT passes (field f at f*FS).  Pass s:
// sub-transform length LS = N / (R_0 ... R_{s-1}), radix R = R_s, stride
// SS = LS / R; butterfly (b, j) takes the elements b*LS + j + m*SS.
// Decimation in frequency (c2r, sign +1): DFT_R, then twiddle w_LS^{jk}; after
// all passes position p holds the output of a fixed digit-reversed index.
// Decimation in time (r2c, sign -1, passes in reverse order): twiddle
// w_LS^{-jm}, then DFT_R; it takes the digit-reversed arrangement back to
// natural order.  The nonlinear terms are pointwise in phi, so the physical
// points may stay digit-reversed between the two.
// The twiddles of pass s are the table entries tw[off(s) + (k-1)*SS + j] =
// exp(2 pi i j k / LS), k = 1 .. R-1, j < SS (conjugated for sign -1).
__host__ __device__ constexpr int ip_ls(int n, int ps) { return n / pprod(n, ps); }
__host__ __device__ constexpr int ip_tw_off(int n, int ps) {
    int o = 0;
    for (int j = 0; j < ps; ++j) o += (radix_at(n, j) - 1) * (ip_ls(n, j) / radix_at(n, j));
    return o;
}
__host__ __device__ constexpr int ip_tw_size(int n) { return ip_tw_off(n, npass_of(n)); }

// u[k] *= w^k, k = 1 .. R-1, for the butterfly's one table twiddle w: the
// powers are complex products (at most three deep, a few units in the last
// place) formed in the order they are used, w^2 = w w, w^3 = w^2 w,
// w^4 = w^2 w^2, w^5 = w^4 w, w^6 = w^4 w^2, w^7 = w^4 w^3, so that no more
// than four of them are live next to the butterfly's R values.
template <int R>
__device__ __forceinline__ void twiddle_apply(double2 (&u)[R], double2 w1) {
    static_assert(R == 2 || R == 3 || R == 4 || R == 8, "radix");
    u[1] = cmul(u[1], w1);
    if constexpr (R >= 3) {
        const double2 w2 = cmul(w1, w1);
        u[2] = cmul(u[2], w2);
        if constexpr (R >= 4) {
            const double2 w3 = cmul(w2, w1);
            u[3] = cmul(u[3], w3);
            if constexpr (R == 8) {
                const double2 w4 = cmul(w2, w2);
                u[4] = cmul(u[4], w4);
                u[5] = cmul(u[5], cmul(w4, w1));
                u[6] = cmul(u[6], cmul(w4, w2));
                u[7] = cmul(u[7], cmul(w4, w3));
            }
        }
    }
}

// Butterfly g of a pass -> (field f, block b, offset j).  The plain order runs
// over (f, b, j).  A 16-byte shared access is served in 8-lane phases, one
// wavefront per phase when its 8 slots fall in 8 different bank groups
// (slot mod 8); the field stride (2 mod 8) shifts a field's slots by 2.  In
// two passes the plain order puts two slots of a phase in one group, and
// these passes deal their butterflies out over pairs of fields instead:
//   R = 8, SS = 12 (slot = 2f + j mod 8): fields f and f + 2 together; per b,
//     j 0-7 of f, j 0-7 of f + 2, then j 8-11 of both: every phase conflict-free;
//   R = 4, SS = 3 (slot = 2f + 4b + j mod 8): fields f and f + 1 together; per
//     four b, the six butterflies of (b0, b0+1) of f with the j = 1 ones of
//     (b0+2, b0+3) of f + 1, the same with the fields swapped, then the
//     j = 0, 2 ones of (b0+2, b0+3) of both: 4 wavefronts per 24 butterflies
//     instead of 6 (the fewest: j = 1 gives the only odd slots).
// The mapping only changes which thread computes which butterfly.
template <int N, int NB, int R, int LS, int SS, int T>
__device__ __forceinline__ void butterfly_of(int g, int& f, int& b, int& j) {
    if constexpr (R == 8 && SS == 12 && NB >= 3) {
        constexpr int NPAIR = NB == 4 ? 2 : 1;   // fields (0, 2), (1, 3)
        if (g < NPAIR * 2 * T) {
            const int p = g / (2 * T), rem = g - p * 2 * T;
            b = rem / 24;
            const int w = rem - b * 24, qi = w >> 3, l8 = w & 7;
            if (qi < 2) {
                f = p + 2 * qi;
                j = l8;
            } else {
                f = (l8 < 4) ? p : p + 2;
                j = 8 + (l8 & 3);
            }
            return;
        }
        const int bi = g - NPAIR * 2 * T;   // NB = 3: field 1 alone
        f = 1;
        b = bi / SS;
        j = bi - b * SS;
        return;
    } else if constexpr (R == 4 && SS == 3 && (N / LS) % 4 == 0 && NB >= 2) {
        constexpr int NPAIR = NB / 2;   // fields (0, 1), (2, 3)
        if (g < NPAIR * 2 * T) {
            const int fp = g / (2 * T), rem = g - fp * 2 * T;
            const int blk = rem / 24, w = rem - blk * 24, qi = w >> 3, l8 = w & 7;
            const int f0 = 2 * fp, b0 = 4 * blk;
            if (qi == 2) {
                f = f0 + (l8 >> 2);
                b = b0 + 2 + ((l8 & 3) >> 1);
                j = (l8 & 1) * 2;
            } else if (l8 < 6) {
                f = f0 + qi;
                b = b0 + l8 / 3;
                j = l8 - (l8 / 3) * 3;
            } else {
                f = f0 + 1 - qi;
                b = b0 + 2 + (l8 - 6);
                j = 1;
            }
            return;
        }
        const int bi = g - NPAIR * 2 * T;   // NB = 3: field 2 alone
        f = 2 * NPAIR;
        b = bi / SS;
        j = bi - b * SS;
        return;
    }
    f = g / T;
    const int bi = g - f * T;
    b = bi / SS;
    j = bi - b * SS;
}

template <int N, int NB, int NT, int PS, bool DIT>
__device__ __forceinline__ void fft_pass_ip(double2* __restrict__ buf, const double2* __restrict__ twp, int sign,
                                            int tid) {
    constexpr int R = radix_at(N, PS), LS = ip_ls(N, PS), SS = LS / R, T = N / R, FS = fstride(N);
    const double2* __restrict__ tw = twp + ip_tw_off(N, PS);
    auto butterfly = [&](int g) {
        int f, b, j;
        butterfly_of<N, NB, R, LS, SS, T>(g, f, b, j);
        const int base = f * FS + b * LS + j;
        double2 u[R];
#pragma unroll
        for (int m = 0; m < R; ++m) u[m] = buf[SW(base + m * SS)];
        if constexpr (SS > 1) {
            double2 w1 = __ldg(tw + j);   // exp(2 pi i j / LS), conjugated for the r2c
            if (DIT) {
                w1.y = -w1.y;
                twiddle_apply<R>(u, w1);
                dft_small(R, u, sign);
            } else {
                dft_small(R, u, sign);
                twiddle_apply<R>(u, w1);
            }
        } else {
            dft_small(R, u, sign);
        }
#pragma unroll
        for (int m = 0; m < R; ++m) buf[SW(base + m * SS)] = u[m];
    };
    // two independent butterflies per iteration for instruction-level parallelism
    // (one for radix 16, whose butterfly alone fills the registers)
    if constexpr (R >= 16 || NT > 256) {
#pragma unroll 1
        for (int g = tid; g < T * NB; g += NT) butterfly(g);
    } else {
#pragma unroll 1
        for (int g = tid; g < T * NB; g += 2 * NT) {
            butterfly(g);
            if (g + NT < T * NB) butterfly(g + NT);
        }
    }
}

template <int N, int NB, int NT, int PS = 0>
__device__ __forceinline__ void fft_dif(double2* buf, const double2* twp, int tid) {
    if constexpr (PS < npass_of(N)) {
        fft_pass_ip<N, NB, NT, PS, false>(buf, twp, +1, tid);
        __syncthreads();
        fft_dif<N, NB, NT, PS + 1>(buf, twp, tid);
    }
}

template <int N, int NB, int NT, int PS = npass_of(N) - 1>
__device__ __forceinline__ void fft_dit(double2* buf, const double2* twp, int tid) {
    if constexpr (PS >= 0) {
        fft_pass_ip<N, NB, NT, PS, true>(buf, twp, -1, tid);
        __syncthreads();
        fft_dit<N, NB, NT, PS - 1>(buf, twp, tid);
    }
}

// One spectrum value of this row: X = E + O (south, h = 0) or E - O (north,
// h = 1), as StP_4d_dgp2 reflects the even-l / odd-l products
// (Legendre_Transforms.F90:1030-1064); d/dphi (i m X) when dp; Im X_0 = 0 as
// FFTW's c2r ignores it; X_m = 0 for m >= L.
// mpart (diagnostics): 0 the field, 1 its fluctuating part (m > 0), 2 its azimuthal mean (m = 0)
__device__ __forceinline__ double2 spec_value(const double* __restrict__ base, long mstride, long ostride, int m,
                                              int L, int h, bool dp, int mpart = 0) {
    if (m >= L || (mpart == 1 && m == 0) || (mpart == 2 && m != 0)) return make_double2(0.0, 0.0);
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

// a[b] for a runtime b without a local-memory array
template <class T, int NB>
__device__ __forceinline__ T pick(const T (&a)[NB], int b) {
    T v = a[0];
#pragma unroll
    for (int i = 1; i < NB; ++i)
        if (b == i) v = a[i];
    return v;
}

// c2r of NB fields of this row (fields fo[b], d/dphi where dp[b]; mpart as in spec_value,
// 0 in the time step): the input Z is formed straight from the spectrum loads (one (k, N-k)
// pair per work item), then the DIF passes.  On return y[b][q] holds the physical pair
// (y[2n], y[2n+1]) of field b at the buffer position t + q*ROW_THREADS.
template <int N, int NB, int ZPT>
__device__ __forceinline__ void row_c2r(const PhysParams& P, const double* __restrict__ rowbase, int h,
                                        const int (&fo)[NB], const bool (&dp)[NB], double2* sm, int t,
                                        double2 (&y)[FB][ZPT], int mpart = 0) {
    constexpr int FS = fstride(N);
    constexpr int NI = N / 2 + 1;                                   // k = 0 .. N/2
    constexpr int QI = (NB * NI + ROW_THREADS - 1) / ROW_THREADS;   // items per thread
    double2* buf = sm + RowSmem<N>::BUF;
    const int L = P.L;
    const long ostride = (long)P.ncola;   // E -> O within p2a[theta_h][m][par][r][field][2]
    const long mstride = 2L * P.ncola;
    __syncthreads();   // the buffer is free (previous batch read)
    constexpr int QC = 3;   // items whose loads are in flight together
    // item g = (k, b), b fastest: a quarter warp reads the batch's adjacent
    // fields of two wavenumbers (NB = 4).  For NB = 2 a quarter warp takes the
    // wavenumbers k0 + {0, 1, 4, 5} (then k0 + {2, 3, 6, 7}) of both fields, so
    // that its Z writes (slot 2b + k mod 8) fall in distinct bank groups.
    auto item = [](int g, int& k, int& b) {
        if constexpr (NB == 2 && (N / 2) % 8 == 0) {
            const int l8 = g & 7, kk = l8 >> 1;
            b = l8 & 1;
            k = (g >> 4) * 8 + ((g >> 3) & 1) * 2 + (kk & 1) + ((kk >> 1) << 2);
        } else {
            k = g / NB;
            b = g - k * NB;
        }
    };
#pragma unroll 1
    for (int q0 = 0; q0 < QI; q0 += QC) {
        double2 xk[QC], xn[QC];
#pragma unroll
        for (int qq = 0; qq < QC; ++qq) {
            const int g = t + (q0 + qq) * ROW_THREADS;
            xk[qq] = xn[qq] = make_double2(0.0, 0.0);
            if (q0 + qq < QI && g < NB * NI) {
                int k, b;
                item(g, k, b);
                const double* base = rowbase + (long)pick(fo, b) * 2;
                const bool d = pick(dp, b);
                xk[qq] = spec_value(base, mstride, ostride, k, L, h, d, mpart);
                xn[qq] = spec_value(base, mstride, ostride, N - k, L, h, d, mpart);   // N - k >= L for k = 0
            }
        }
#pragma unroll
        for (int qq = 0; qq < QC; ++qq) {
            const int g = t + (q0 + qq) * ROW_THREADS;
            if (q0 + qq < QI && g < NB * NI) {
                int k, b;
                item(g, k, b);
                const double2 wk = __ldg(P.wr + k);   // w^(N-k) = -conj(w^k), w = exp(2 pi i / 2N)
                buf[SW(b * FS + k)] = zform(xk[qq], xn[qq], wk);
                if (k != 0 && 2 * k != N) buf[SW(b * FS + N - k)] = zform(xn[qq], xk[qq], make_double2(-wk.x, wk.y));
            }
        }
    }
    __syncthreads();
    fft_dif<N, NB, ROW_THREADS>(buf, P.twp, t);
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int q = 0; q < ZPT; ++q) {
            const int n = t + q * ROW_THREADS;
            y[b][q] = (n < N) ? buf[SW(b * FS + n)] : make_double2(0.0, 0.0);
        }
}

// X_k of the real transform from the complex r2c output Z (in place, one (k, N-k) pair per
// work item): X_k = e - i conj(w^k) d with e, d the half sums / differences of Z_k and
// conj Z_{N-k}, each times hs(f); Im X_0 = 0; only k < L is kept.
template <int N, class HS>
__device__ __forceinline__ void r2c_finish(double2* a, int nf, int L, const double2* __restrict__ wr, int t,
                                           const HS& hsf) {
    constexpr int FS = fstride(N);
    constexpr int NI = N / 2 + 1;
    for (int g = t; g < nf * NI; g += ROW_THREADS) {
        const int f = g / NI, k = g - f * NI;
        const double2 zk = a[SW(f * FS + k)];
        const double2 zn = a[SW(f * FS + (N - k) % N)];
        const double2 wk = __ldg(wr + k);   // w^(N-k) = -conj(w^k)
        const double hs = hsf(f);
        auto xval = [&](double2 p, double2 q, double2 w, bool zero_im) {   // X from Z_kk = p, Z_{N-kk} = q
            const double2 qn = cconj(q);
            const double2 e = make_double2(hs * (p.x + qn.x), hs * (p.y + qn.y));
            const double2 d = make_double2(hs * (p.x - qn.x), hs * (p.y - qn.y));
            const double2 wd = cmul(cconj(w), d);
            double2 X = make_double2(e.x + wd.y, e.y - wd.x);
            if (zero_im) X.y = 0.0;
            return X;
        };
        if (k < L) a[SW(f * FS + k)] = xval(zk, zn, wk, k == 0);
        if (k != 0 && 2 * k != N && N - k < L) a[SW(f * FS + N - k)] = xval(zn, zk, make_double2(-wk.x, wk.y), false);
    }
}

template <int NTH, bool MAG, bool HEAT>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(ROW_THREADS, 2) physics_kernel(PhysParams P) {
    constexpr int N = NTH;
    constexpr int FS = fstride(N);
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    double2* acc = sm + RowSmem<N>::ACC;
    __shared__ double red[ROW_THREADS / 32];
    const int t = threadIdx.x;
    const int h = (int)cluster.block_rank();        // 0: theta (south half), 1: pi - theta
    const int nr = P.nr;
    const int pair = blockIdx.x >> 1;
    const int r = pair % nr;
    const int thh = pair / nr;
    const int th = h ? (N - 1 - thh) : thh;
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    // The row's radial and colatitude factors live in shared memory and are read
    // where they are used, so that they hold no registers across the FFTs.
    __shared__ double rowc[RC_COUNT];
    if (t == 0) {
        const double csc = P.trig[2 * N + th], orad = P.radial[R_OVER_R * nr + r];
        rowc[RC_RAD] = P.radial[R_RADIUS * nr + r];
        rowc[RC_ORAD] = orad;
        rowc[RC_RHO] = P.radial[R_DENSITY * nr + r];
        rowc[RC_DLNRHO] = P.radial[R_DLNRHO * nr + r];
        rowc[RC_DR] = P.radial[R_DELTA_R * nr + r];
        rowc[RC_CS] = P.trig[th];
        rowc[RC_SN] = P.trig[N + th];
        rowc[RC_CSC] = csc;
        rowc[RC_COT] = P.trig[3 * N + th];
        rowc[RC_COR] = P.rotation ? P.coriolis : 0.0;
        rowc[RC_C2R] = csc * csc * orad;
        rowc[RC_HSF] = 0.5 * (P.radial[R_DENSITY * nr + r] * P.radial[R_RADIUS * nr + r] * csc);
        rowc[RC_VH] = P.radial[R_VISC_HEAT * nr + r];
        rowc[RC_OH] = P.radial[R_OHM_HEAT * nr + r];
    }   // read after row_c2r's first barrier

    double2 vr[ZPT], vt[ZPT], vp[ZPT];
    double2 y[FB][ZPT];
    auto acc_at = [&](int f, int q) -> double2& { return acc[SW(f * FS + t + q * ROW_THREADS)]; };
    auto live = [&](int q) { return t + q * ROW_THREADS < N; };
    if constexpr (HEAT) {
        // The anelastic form: the same terms, with the viscous heating
        // (Compute_Viscous_Heating, Sphere_Physical_Space.F90:337-443) in T's accumulator.
        // Its strain-rate components are products across fields, so the batches are
        // regrouped for each component to complete inside one batch:
        //   H1: v_r, v_theta, v_phi
        //   H2: dv_r/dtheta, dv_r/dphi, dv_theta/dr, dv_phi/dr  -> 2 e_r_theta, 2 e_r_phi
        //   H3: dv_phi/dphi, omega_r, dv_theta/dphi, dv_r/dr    -> e_rr, e_theta_theta,
        //       e_phi_phi, 2 e_phi_theta (dv_theta/dtheta, dv_phi/dtheta as :226-248 form them)
        //   H4: dT/dr, dT/dtheta, dT/dphi
        {
            const int fo[3] = {A_VR, A_VT, A_VP};
            const bool dp[3] = {false, false, false};
            row_c2r<N, 3, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double rad = rowc[RC_RAD], orad = rowc[RC_ORAD], rho = rowc[RC_RHO], dlnrho = rowc[RC_DLNRHO];
            const double cs = rowc[RC_CS], sn = rowc[RC_SN], csc = rowc[RC_CSC], cot = rowc[RC_COT], cor = rowc[RC_COR];
#pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                vr[q] = y[0][q];
                vt[q] = make_double2(y[1][q].x * csc, y[1][q].y * csc);
                vp[q] = make_double2(y[2][q].x * csc, y[2][q].y * csc);
                auto w0 = [&](double b, double c) { return rho * (rad * b * b + rad * c * c + cor * sn * rad * rad * c); };
                auto p0 = [&](double a, double b, double c) {
                    return -b * b * cot * orad - b * a * orad - b * a * dlnrho - c * c * cot * orad - cor * cs * c;
                };
                auto z0 = [&](double a, double b, double c) { return c * a * orad + cor * (cs * b + sn * a); };
                if (live(q)) {
                    acc_at(0, q) = make_double2(w0(vt[q].x, vp[q].x), w0(vt[q].y, vp[q].y));
                    acc_at(1, q) = make_double2(p0(vr[q].x, vt[q].x, vp[q].x), p0(vr[q].y, vt[q].y, vp[q].y));
                    acc_at(3, q) = make_double2(z0(vr[q].x, vt[q].x, vp[q].x), z0(vr[q].y, vt[q].y, vp[q].y));
                }
            }
        }
        {
            const int fo[4] = {A_DVRDT, A_VR, A_DVTDR, A_DVPDR};
            const bool dp[4] = {false, true, false, false};
            row_c2r<N, 4, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double rad = rowc[RC_RAD], orad = rowc[RC_ORAD], rho = rowc[RC_RHO], csc = rowc[RC_CSC];
            const double dlnrho = rowc[RC_DLNRHO], vh = rowc[RC_VH];
#pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                if (!live(q)) continue;
                double2& w = acc_at(0, q);
                double2& pp = acc_at(1, q);
                double2& z = acc_at(3, q);
                // a = sin(theta) dv_r/dtheta, b = dv_r/dphi, c = sin(theta) dv_theta/dr, d = sin(theta) dv_phi/dr
                auto terms = [&](double a, double b, double c, double d, double vrr, double vtt, double vpp, double& wv,
                                 double& pv, double& zv) {
                    wv += -rho * rad * vtt * a * csc - rho * rad * csc * vpp * b;
                    pv += vrr * c * csc;
                    zv += vrr * d * csc;
                    const double erth = (a * csc - vtt) * orad + c * csc;   // 2 e_r_theta
                    const double erph = (b * csc - vpp) * orad + d * csc;   // 2 e_r_phi
                    const double dv = -vrr * dlnrho;                        // div u
                    return vh * (erth * erth * 0.5 + erph * erph * 0.5 - dv * dv * (1.0 / 3.0));
                };
                const double hx = terms(y[0][q].x, y[1][q].x, y[2][q].x, y[3][q].x, vr[q].x, vt[q].x, vp[q].x, w.x,
                                        pp.x, z.x);
                const double hy = terms(y[0][q].y, y[1][q].y, y[2][q].y, y[3][q].y, vr[q].y, vt[q].y, vp[q].y, w.y,
                                        pp.y, z.y);
                acc_at(2, q) = make_double2(hx, hy);
            }
        }
        {
            const int fo[4] = {A_VP, A_OMR, A_VT, A_DVRDR};
            const bool dp[4] = {true, false, true, false};
            row_c2r<N, 4, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double rad = rowc[RC_RAD], orad = rowc[RC_ORAD], rho = rowc[RC_RHO], csc = rowc[RC_CSC];
            const double cot = rowc[RC_COT], c2r = rowc[RC_C2R], dlnrho = rowc[RC_DLNRHO], vh = rowc[RC_VH];
            const double csc2 = csc * csc;
#pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                if (!live(q)) continue;
                double2& w = acc_at(0, q);
                double2& pp = acc_at(1, q);
                double2& tt = acc_at(2, q);
                double2& z = acc_at(3, q);
                // a = sin(theta) dv_phi/dphi, b = omega_r, c = sin(theta) dv_theta/dphi, x = dv_r/dr
                auto terms = [&](double a, double b, double c, double x, double vrr, double vtt, double vpp, double& wv,
                                 double& pv, double& zv) {
                    wv += -rho * rad * rad * vrr * x;
                    pv += -vtt * x + vpp * c * c2r - vtt * a * c2r;
                    zv += vtt * c * c2r + vpp * a * c2r + vtt * b;
                    const double dvtdt = -vrr * (rad * dlnrho + 2.0) - rad * x - vtt * cot - a * csc2;
                    const double dvpdt = rad * b + c * csc2 - vpp * cot;
                    const double eff = (a * csc2 + vrr + vtt * cot) * orad;     // e_phi_phi
                    const double ett = (dvtdt + vrr) * orad;                    // e_theta_theta
                    const double eph = (dvpdt + c * csc2 - vpp * cot) * orad;   // 2 e_phi_theta
                    return vh * (x * x + eff * eff + ett * ett + eph * eph * 0.5);
                };
                tt.x += terms(y[0][q].x, y[1][q].x, y[2][q].x, y[3][q].x, vr[q].x, vt[q].x, vp[q].x, w.x, pp.x, z.x);
                tt.y += terms(y[0][q].y, y[1][q].y, y[2][q].y, y[3][q].y, vr[q].y, vt[q].y, vp[q].y, w.y, pp.y, z.y);
            }
        }
        {
            const int fo[3] = {A_DTDR, A_DTDT, A_T};
            const bool dp[3] = {false, false, true};
            row_c2r<N, 3, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double csc = rowc[RC_CSC], orad = rowc[RC_ORAD];
#pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                if (!live(q)) continue;
                const double2 d = y[0][q], a = y[1][q], b = y[2][q];
                double2& tt = acc_at(2, q);
                tt.x += -vr[q].x * d.x - a.x * csc * vt[q].x * orad - vp[q].x * b.x * csc * orad;
                tt.y += -vr[q].y * d.y - a.y * csc * vt[q].y * orad - vp[q].y * b.y * csc * orad;
            }
        }
    } else {
        // B1: v_r, v_theta, v_phi, dv_r/dr: the quadratic, Coriolis and radial-advection terms
        {
            const int fo[4] = {A_VR, A_VT, A_VP, A_DVRDR};
            const bool dp[4] = {false, false, false, false};
            row_c2r<N, 4, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double rad = rowc[RC_RAD], orad = rowc[RC_ORAD], rho = rowc[RC_RHO], dlnrho = rowc[RC_DLNRHO];
            const double cs = rowc[RC_CS], sn = rowc[RC_SN], csc = rowc[RC_CSC], cot = rowc[RC_COT], cor = rowc[RC_COR];
    #pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                vr[q] = y[0][q];
                vt[q] = y[1][q];
                vp[q] = y[2][q];
                vt[q].x *= csc;
                vt[q].y *= csc;
                vp[q].x *= csc;
                vp[q].y *= csc;
                const double2 x = y[3][q];
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
                    acc_at(3, q) = make_double2(z0(vr[q].x, vt[q].x, vp[q].x), z0(vr[q].y, vt[q].y, vp[q].y));
                }
            }
        }
        // B2: dv_r/dtheta, dv_r/dphi, dv_theta/dr, dv_theta/dphi
        {
            const int fo[4] = {A_DVRDT, A_VR, A_DVTDR, A_VT};
            const bool dp[4] = {false, true, false, true};
            row_c2r<N, 4, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double rad = rowc[RC_RAD], rho = rowc[RC_RHO], csc = rowc[RC_CSC], c2r = rowc[RC_C2R];
    #pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                if (!live(q)) continue;
                const double2 a = y[0][q], b = y[1][q], c = y[2][q], d = y[3][q];
                double2& w = acc_at(0, q);
                double2& pp = acc_at(1, q);
                double2& z = acc_at(3, q);
                w.x += -rho * rad * vt[q].x * a.x * csc - rho * rad * csc * vp[q].x * b.x;
                w.y += -rho * rad * vt[q].y * a.y * csc - rho * rad * csc * vp[q].y * b.y;
                pp.x += vr[q].x * c.x * csc + vp[q].x * d.x * c2r;
                pp.y += vr[q].y * c.y * csc + vp[q].y * d.y * c2r;
                z.x += vt[q].x * d.x * c2r;
                z.y += vt[q].y * d.y * c2r;
            }
        }
        // B3: dv_phi/dr, dv_phi/dphi, omega_r, dT/dr (the T term's first part, written)
        {
            const int fo[4] = {A_DVPDR, A_VP, A_OMR, A_DTDR};
            const bool dp[4] = {false, true, false, false};
            row_c2r<N, 4, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double csc = rowc[RC_CSC], c2r = rowc[RC_C2R];
    #pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                if (!live(q)) continue;
                const double2 a = y[0][q], b = y[1][q], c = y[2][q], d = y[3][q];
                double2& pp = acc_at(1, q);
                double2& z = acc_at(3, q);
                z.x += vr[q].x * a.x * csc + vp[q].x * b.x * c2r + vt[q].x * c.x;
                z.y += vr[q].y * a.y * csc + vp[q].y * b.y * c2r + vt[q].y * c.y;
                pp.x += -vt[q].x * b.x * c2r;
                pp.y += -vt[q].y * b.y * c2r;
                acc_at(2, q) = make_double2(-vr[q].x * d.x, -vr[q].y * d.y);
            }
        }
        // B4: dT/dtheta, dT/dphi
        {
            const int fo[2] = {A_DTDT, A_T};
            const bool dp[2] = {false, true};
            row_c2r<N, 2, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double csc = rowc[RC_CSC], orad = rowc[RC_ORAD];
    #pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                if (!live(q)) continue;
                const double2 a = y[0][q], b = y[1][q];
                double2& tt = acc_at(2, q);
                tt.x += -a.x * csc * vt[q].x * orad - vp[q].x * b.x * csc * orad;
                tt.y += -a.y * csc * vt[q].y * orad - vp[q].y * b.y * csc * orad;
            }
        }
    }
    // CFL (Find_MyMinDT); the rho r / sin(theta) factor of the P and Z terms is a
    // row constant, applied to their spectra after the r2c (RC_HSF)
    double cmax = 0.0;
    const double orad = rowc[RC_ORAD], dr = rowc[RC_DR];
    const double hfac = P.llmax * orad * orad, rfac = 1.0 / (dr * dr);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        if (live(q)) {
            cmax = fmax(cmax, (vt[q].x * vt[q].x + vp[q].x * vp[q].x) * hfac);
            cmax = fmax(cmax, (vt[q].y * vt[q].y + vp[q].y * vp[q].y) * hfac);
            cmax = fmax(cmax, vr[q].x * vr[q].x * rfac);
            cmax = fmax(cmax, vr[q].y * vr[q].y * rfac);
        }
    }
    if constexpr (MAG) {
        // M1: B_r, B_theta, B_phi, (curl B)_r.  The EMF u x B (Compute_EMF,
        // Sphere_Physical_Space.F90:534-581) replaces them in the FFT buffer and goes through
        // its own r2c and fold into p2b fields B_EMFT, B_EMFR, B_EMFP; B stays in registers
        // for the Lorentz force, which M2 ((curl B)_theta, (curl B)_phi) completes.
        double2 br[ZPT], bt[ZPT], bp[ZPT], cbr[ZPT];
        double2* buf = sm + RowSmem<N>::BUF;
        {
            const int fo[4] = {A_BR, A_BT, A_BP, A_CBR};
            const bool dp[4] = {false, false, false, false};
            row_c2r<N, 4, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double csc = rowc[RC_CSC], rad = rowc[RC_RAD], rho = rowc[RC_RHO];
            // the Alfven speed (:798-806)
            const double hfb = P.llmax * orad * orad / rho * P.lorentz, rfb = P.lorentz / (dr * dr * rho);
#pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                br[q] = y[0][q];
                bt[q] = make_double2(y[1][q].x * csc * orad, y[1][q].y * csc * orad);   // rsintheta_div
                bp[q] = make_double2(y[2][q].x * csc * orad, y[2][q].y * csc * orad);
                cbr[q] = y[3][q];
                if (!live(q)) continue;
                if constexpr (HEAT) {   // Compute_Ohmic_Heating (:446-466), the (curl B)_r part
                    const double oh = rowc[RC_OH];
                    acc_at(2, q).x += cbr[q].x * cbr[q].x * oh;
                    acc_at(2, q).y += cbr[q].y * cbr[q].y * oh;
                }
                cmax = fmax(cmax, (bt[q].x * bt[q].x + bp[q].x * bp[q].x) * hfb);
                cmax = fmax(cmax, (bt[q].y * bt[q].y + bp[q].y * bp[q].y) * hfb);
                cmax = fmax(cmax, br[q].x * br[q].x * rfb);
                cmax = fmax(cmax, br[q].y * br[q].y * rfb);
                auto emft = [&](double a, double c, double b_r, double b_p) { return (-a * b_p + c * b_r) * csc * rad; };
                auto emfr = [&](double b, double c, double b_t, double b_p) { return b * b_p - c * b_t; };
                auto emfp = [&](double a, double b, double b_r, double b_t) { return (a * b_t - b * b_r) * csc * rad; };
                const int n = t + q * ROW_THREADS;
                buf[SW(0 * FS + n)] = make_double2(emft(vr[q].x, vp[q].x, br[q].x, bp[q].x),
                                                   emft(vr[q].y, vp[q].y, br[q].y, bp[q].y));
                buf[SW(1 * FS + n)] = make_double2(emfr(vt[q].x, vp[q].x, bt[q].x, bp[q].x),
                                                   emfr(vt[q].y, vp[q].y, bt[q].y, bp[q].y));
                buf[SW(2 * FS + n)] = make_double2(emfp(vr[q].x, vt[q].x, br[q].x, bt[q].x),
                                                   emfp(vr[q].y, vt[q].y, br[q].y, bt[q].y));
            }
        }
        __syncthreads();
        fft_dit<N, 3, ROW_THREADS>(buf, P.twp, t);
        r2c_finish<N>(buf, 3, P.L, P.wr, t, [](int) { return 0.5; });
        cluster.sync();
        {
            const double2* peer = cluster.map_shared_rank(buf, h ^ 1);
            const int L = P.L;
            const long mstride = 2L * (P.nth / 2) * P.ncolb;
            double* obase = P.p2b + (long)h * (P.nth / 2) * P.ncolb + (long)thh * P.ncolb + (long)r * (2 * P.nfb) +
                            2 * B_EMFT;
            for (int g = t; g < 3 * L; g += ROW_THREADS) {
                const int k = g / 3, f = g - 3 * k;
                const double2 a = buf[SW(f * FS + k)], b = peer[SW(f * FS + k)];
                *reinterpret_cast<double2*>(obase + k * mstride + f * 2) = h ? csub(b, a) : cadd(a, b);
            }
        }
        cluster.sync();   // the partner has read this CTA's EMF spectra
        // M2: (curl B)_theta, (curl B)_phi -> the Lorentz force (:512-519, 635-641, 712-718)
        {
            const int fo[2] = {A_CBT, A_CBP};
            const bool dp[2] = {false, false};
            row_c2r<N, 2, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
            const double csc = rowc[RC_CSC], rad = rowc[RC_RAD], rho = rowc[RC_RHO];
            const double lc = P.lorentz, r2lc = rad * rad * lc, lcr = lc / rho;
#pragma unroll
            for (int q = 0; q < ZPT; ++q) {
                if (!live(q)) continue;
                const double2 cbt = make_double2(y[0][q].x * csc * orad, y[0][q].y * csc * orad);
                const double2 cbp = make_double2(y[1][q].x * csc * orad, y[1][q].y * csc * orad);
                double2& w = acc_at(0, q);
                double2& pp = acc_at(1, q);
                double2& z = acc_at(3, q);
                w.x += r2lc * (cbt.x * bp[q].x - cbp.x * bt[q].x);
                w.y += r2lc * (cbt.y * bp[q].y - cbp.y * bt[q].y);
                pp.x -= lcr * (cbp.x * br[q].x - cbr[q].x * bp[q].x);
                pp.y -= lcr * (cbp.y * br[q].y - cbr[q].y * bp[q].y);
                z.x -= lcr * (cbr[q].x * bt[q].x - cbt.x * br[q].x);
                z.y -= lcr * (cbr[q].y * bt[q].y - cbt.y * br[q].y);
                if constexpr (HEAT) {   // the (curl B)_theta and (curl B)_phi parts
                    const double oh = rowc[RC_OH];
                    acc_at(2, q).x += (cbt.x * cbt.x + cbp.x * cbp.x) * oh;
                    acc_at(2, q).y += (cbt.y * cbt.y + cbp.y * cbp.y) * oh;
                }
            }
        }
    }
    __syncthreads();
    // r2c of W, P, T, Z in place on the accumulators: Z = FFT(y[2n] + i y[2n+1]), then
    // X_k = e - i conj(w^k) d with e, d the half sums/differences of Z_k, conj Z_{N-k},
    // one (k, N-k) pair per work item, in place
    fft_dit<N, 4, ROW_THREADS>(acc, P.twp, t);
    {
        const double hsf_pz = rowc[RC_HSF];   // P and Z (f = 1, 3) take the row factor
        r2c_finish<N>(acc, 4, P.L, P.wr, t, [&](int f) { return (f & 1) ? hsf_pz : 0.5; });
    }
    // equatorial fold of PtS_4d_dgpv3 (Legendre_Transforms.F90:1109-1122) with the
    // partner row: f_even = X(theta) + X(pi - theta) (written by rank 0),
    // f_odd = X(theta) - X(pi - theta) (written by rank 1)
    cluster.sync();
    {
        const double2* mine = acc;
        const double2* peer = cluster.map_shared_rank(acc, h ^ 1);
        const int L = P.L;
        const long mstride = 2L * (P.nth / 2) * P.ncolb;   // p2b[m][par][theta_h][r][field][2]
        double* obase = P.p2b + (long)h * (P.nth / 2) * P.ncolb + (long)thh * P.ncolb + (long)r * (2 * P.nfb);
        for (int g = t; g < 4 * L; g += ROW_THREADS) {   // g = (k, f), f fastest: 64 contiguous bytes per k
            const int k = g >> 2, f = g & 3;
            const double2 a = mine[SW(f * FS + k)], b = peer[SW(f * FS + k)];
            const double2 v = h ? csub(b, a) : cadd(a, b);
            *reinterpret_cast<double2*>(obase + k * mstride + f * 2) = v;
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

// Per-pass twiddles exp(2 pi i j k / LS) of the in-place FFT, in long
// double, built once at set-up: the step may be captured into a CUDA graph on
// its first launch (a context restored at a later iteration), where no
// allocation or blocking copy may run.
static bool p3_supported(int n);

void physics_prepare(Ctx& c) {
    if (!c.d_twp) {
        const int n = c.d.nth;
        std::vector<double> tw(2 * (size_t)ip_tw_size(n));
        const long double PI = 3.141592653589793238462643383279502884L;
        for (int ps = 0; ps < npass_of(n); ++ps) {
            const int R = radix_at(n, ps), LS = ip_ls(n, ps), SS = LS / R, off = ip_tw_off(n, ps);
            for (int k = 1; k < R; ++k)
                for (int j = 0; j < SS; ++j) {
                    const long double a = 2.0L * PI * (long double)j * k / LS;
                    tw[2 * (off + (k - 1) * SS + j)] = (double)cosl(a);
                    tw[2 * (off + (k - 1) * SS + j) + 1] = (double)sinl(a);
                }
        }
        RA_CUDA(cudaMalloc(&c.d_twp, std::max<size_t>(tw.size(), 2) * sizeof(double)));
        RA_CUDA(cudaMemcpy(c.d_twp, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    c.physics3_ok = p3_supported(c.d.nth);
    // default: all passes in shared memory where that kernel exists (20.7 against 21.5 ms at
    // n_theta = 768, N_r = 192); the autotuner measures both
    c.physics_form = physics_form1_supported(c.d.nth) ? 1 : 0;
    if (!c.physics3_ok && !physics_form1_supported(c.d.nth))
        throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no physical-space kernel instance");
    if (c.mag && !physics_form1_supported(c.d.nth))   // the magnetic terms live in that kernel only
        throw ArgError("magnetism needs n_theta in 24..768 (2^a or 3*2^a); got " + std::to_string(c.d.nth));
    if (c.rad.heating && !physics_form1_supported(c.d.nth))   // and so do the heating terms
        throw ArgError("viscous / ohmic heating needs n_theta in 24..768 (2^a or 3*2^a); got " +
                       std::to_string(c.d.nth));
}

// ---------------------------------------------------------------------------
// Physical-space kernel with the last FFT pass in registers (N = n_theta with
// a final radix-3 pass: 384, 768, 1536; N/3 threads per row).
//
// The c2r runs the in-place passes of physics_kernel except the last one; the
// last (radix-3, stride-1) pass is done in registers by thread t on the three
// points 3t, 3t+1, 3t+2 of every field, the same points in every batch, so
// the nonlinear terms are formed where the transform leaves them, and the
// r2c's first (radix-3) pass is done on the same registers.  Per field this
// saves the last pass's write and the read-back of the physical values in the
// c2r, and the first pass's read in the r2c; the velocity stays in registers
// (nine complex values per thread).  Shared layout and butterfly dealing are
// physics_kernel's.
// ---------------------------------------------------------------------------
template <int N>
struct P3 {
    static constexpr int NT = N / 3;
    static constexpr int NP = npass_of(N);     // passes; the last one (radix 3) runs in registers
    static_assert(radix_at(N, npass_of(N) - 1) == 3, "the last pass must be radix 3");
    static constexpr int FS = fstride(N);
    static constexpr int SIZE = 8 * FS;        // 4-field FFT buffer + 4 accumulators (double2)
    static __host__ __device__ constexpr int slot(int p) { return p; }
};

template <int N, int NB, int NT, int PS = 0>
__device__ __forceinline__ void fft_dif_upto_last(double2* buf, const double2* twp, int tid) {
    if constexpr (PS < npass_of(N) - 1) {
        fft_pass_ip<N, NB, NT, PS, false>(buf, twp, +1, tid);
        __syncthreads();
        fft_dif_upto_last<N, NB, NT, PS + 1>(buf, twp, tid);
    }
}

template <int N, int NB, int NT, int PS = npass_of(N) - 2>
__device__ __forceinline__ void fft_dit_from_second(double2* buf, const double2* twp, int tid) {
    if constexpr (PS >= 0) {
        fft_pass_ip<N, NB, NT, PS, true>(buf, twp, -1, tid);
        __syncthreads();
        fft_dit_from_second<N, NB, NT, PS - 1>(buf, twp, tid);
    }
}

// c2r of NB fields of this row (fo, dp as in row_c2r); on return y[b][m] holds
// the physical pair at buffer position 3t + m of field b.
template <int N, int NB>
__device__ __forceinline__ void p3_c2r(const PhysParams& P, const double* __restrict__ rowbase, int h,
                                       const int (&fo)[NB], const bool (&dp)[NB], double2* buf, int t,
                                       double2 (&y)[4][3]) {
    using S = P3<N>;
    constexpr int NI = N / 2 + 1;
    const int L = P.L;
    const long ostride = (long)P.ncola, mstride = 2L * P.ncola;
    __syncthreads();   // the buffer is free
    auto item = [](int g, int& k, int& b) {
        if constexpr (NB == 2 && (N / 2) % 8 == 0) {
            const int l8 = g & 7, kk = l8 >> 1;
            b = l8 & 1;
            k = (g >> 4) * 8 + ((g >> 3) & 1) * 2 + (kk & 1) + ((kk >> 1) << 2);
        } else {
            k = g / NB;
            b = g - k * NB;
        }
    };
    constexpr int QI = (NB * NI + S::NT - 1) / S::NT;
    constexpr int QC = 3;
#pragma unroll 1
    for (int q0 = 0; q0 < QI; q0 += QC) {
        double2 xk[QC], xn[QC];
#pragma unroll
        for (int qq = 0; qq < QC; ++qq) {
            const int g = t + (q0 + qq) * S::NT;
            xk[qq] = xn[qq] = make_double2(0.0, 0.0);
            if (q0 + qq < QI && g < NB * NI) {
                int k, b;
                item(g, k, b);
                const double* base = rowbase + (long)pick(fo, b) * 2;
                const bool d = pick(dp, b);
                xk[qq] = spec_value(base, mstride, ostride, k, L, h, d);
                xn[qq] = spec_value(base, mstride, ostride, N - k, L, h, d);
            }
        }
#pragma unroll
        for (int qq = 0; qq < QC; ++qq) {
            const int g = t + (q0 + qq) * S::NT;
            if (q0 + qq < QI && g < NB * NI) {
                int k, b;
                item(g, k, b);
                const double2 wk = __ldg(P.wr + k);
                buf[b * S::FS + k] = zform(xk[qq], xn[qq], wk);
                if (k != 0 && 2 * k != N) buf[b * S::FS + N - k] = zform(xn[qq], xk[qq], make_double2(-wk.x, wk.y));
            }
        }
    }
    __syncthreads();
    fft_dif_upto_last<N, NB, S::NT>(buf, P.twp, t);
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        double2 u[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) u[m] = buf[b * S::FS + 3 * t + m];
        dft_small(3, u, +1);
#pragma unroll
        for (int m = 0; m < 3; ++m) y[b][m] = u[m];
    }
}

template <int N, int MINB>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(P3<N>::NT, MINB) physics3_kernel(PhysParams P) {
    using S = P3<N>;
    constexpr int FS = S::FS, NT = S::NT;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    double2* acc = buf + 4 * FS;
    __shared__ double red[NT / 32];
    __shared__ double rowc[RC_COUNT];
    const int t = threadIdx.x;
    const int h = (int)cluster.block_rank();
    const int nr = P.nr;
    const int pair = blockIdx.x >> 1;
    const int r = pair % nr;
    const int thh = pair / nr;
    const int th = h ? (N - 1 - thh) : thh;
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    if (t == 0) {
        const double csc = P.trig[2 * N + th], orad = P.radial[R_OVER_R * nr + r];
        rowc[RC_RAD] = P.radial[R_RADIUS * nr + r];
        rowc[RC_ORAD] = orad;
        rowc[RC_RHO] = P.radial[R_DENSITY * nr + r];
        rowc[RC_DLNRHO] = P.radial[R_DLNRHO * nr + r];
        rowc[RC_DR] = P.radial[R_DELTA_R * nr + r];
        rowc[RC_CS] = P.trig[th];
        rowc[RC_SN] = P.trig[N + th];
        rowc[RC_CSC] = csc;
        rowc[RC_COT] = P.trig[3 * N + th];
        rowc[RC_COR] = P.rotation ? P.coriolis : 0.0;
        rowc[RC_C2R] = csc * csc * orad;
        rowc[RC_HSF] = 0.5 * (P.radial[R_DENSITY * nr + r] * P.radial[R_RADIUS * nr + r] * csc);
    }   // read after p3_c2r's first barrier
    double2 vr[3], vt[3], vp[3];
    double2 y[4][3];
    auto acc_at = [&](int f, int m) -> double2& { return acc[f * FS + S::slot(3 * t + m)]; };
    // B1: v_r, v_theta, v_phi, dv_r/dr
    {
        const int fo[4] = {A_VR, A_VT, A_VP, A_DVRDR};
        const bool dp[4] = {false, false, false, false};
        p3_c2r<N, 4>(P, rowbase, h, fo, dp, buf, t, y);
        const double rad = rowc[RC_RAD], orad = rowc[RC_ORAD], rho = rowc[RC_RHO], dlnrho = rowc[RC_DLNRHO];
        const double cs = rowc[RC_CS], sn = rowc[RC_SN], csc = rowc[RC_CSC], cot = rowc[RC_COT], cor = rowc[RC_COR];
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            vr[m] = y[0][m];
            vt[m] = make_double2(y[1][m].x * csc, y[1][m].y * csc);
            vp[m] = make_double2(y[2][m].x * csc, y[2][m].y * csc);
            const double2 x = y[3][m];
            auto w0 = [&](double a, double b, double c, double xx) {
                return rho * (rad * b * b + rad * c * c + cor * sn * rad * rad * c) - rho * rad * rad * a * xx;
            };
            auto p0 = [&](double a, double b, double c, double xx) {
                return -b * b * cot * orad - b * a * orad - b * a * dlnrho - c * c * cot * orad - cor * cs * c - b * xx;
            };
            auto z0 = [&](double a, double b, double c) { return c * a * orad + cor * (cs * b + sn * a); };
            acc_at(0, m) = make_double2(w0(vr[m].x, vt[m].x, vp[m].x, x.x), w0(vr[m].y, vt[m].y, vp[m].y, x.y));
            acc_at(1, m) = make_double2(p0(vr[m].x, vt[m].x, vp[m].x, x.x), p0(vr[m].y, vt[m].y, vp[m].y, x.y));
            acc_at(3, m) = make_double2(z0(vr[m].x, vt[m].x, vp[m].x), z0(vr[m].y, vt[m].y, vp[m].y));
        }
    }
    // B2: dv_r/dtheta, dv_r/dphi, dv_theta/dr, dv_theta/dphi
    {
        const int fo[4] = {A_DVRDT, A_VR, A_DVTDR, A_VT};
        const bool dp[4] = {false, true, false, true};
        p3_c2r<N, 4>(P, rowbase, h, fo, dp, buf, t, y);
        const double rad = rowc[RC_RAD], rho = rowc[RC_RHO], csc = rowc[RC_CSC], c2r = rowc[RC_C2R];
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const double2 a = y[0][m], b = y[1][m], c = y[2][m], d = y[3][m];
            double2& w = acc_at(0, m);
            double2& pp = acc_at(1, m);
            double2& z = acc_at(3, m);
            w.x += -rho * rad * vt[m].x * a.x * csc - rho * rad * csc * vp[m].x * b.x;
            w.y += -rho * rad * vt[m].y * a.y * csc - rho * rad * csc * vp[m].y * b.y;
            pp.x += vr[m].x * c.x * csc + vp[m].x * d.x * c2r;
            pp.y += vr[m].y * c.y * csc + vp[m].y * d.y * c2r;
            z.x += vt[m].x * d.x * c2r;
            z.y += vt[m].y * d.y * c2r;
        }
    }
    // B3: dv_phi/dr, dv_phi/dphi, omega_r, dT/dr (the T term's first part, written)
    {
        const int fo[4] = {A_DVPDR, A_VP, A_OMR, A_DTDR};
        const bool dp[4] = {false, true, false, false};
        p3_c2r<N, 4>(P, rowbase, h, fo, dp, buf, t, y);
        const double csc = rowc[RC_CSC], c2r = rowc[RC_C2R];
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const double2 a = y[0][m], b = y[1][m], c = y[2][m], d = y[3][m];
            double2& pp = acc_at(1, m);
            double2& z = acc_at(3, m);
            z.x += vr[m].x * a.x * csc + vp[m].x * b.x * c2r + vt[m].x * c.x;
            z.y += vr[m].y * a.y * csc + vp[m].y * b.y * c2r + vt[m].y * c.y;
            pp.x += -vt[m].x * b.x * c2r;
            pp.y += -vt[m].y * b.y * c2r;
            acc_at(2, m) = make_double2(-vr[m].x * d.x, -vr[m].y * d.y);
        }
    }
    // B4: dT/dtheta, dT/dphi; then the r2c's first (radix-3, stride-1) pass on the
    // thread's own points of W, P, T, Z, in registers
    {
        const int fo[2] = {A_DTDT, A_T};
        const bool dp[2] = {false, true};
        p3_c2r<N, 2>(P, rowbase, h, fo, dp, buf, t, y);
        const double csc = rowc[RC_CSC], orad = rowc[RC_ORAD];
        double2 u[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const double2 a = y[0][m], b = y[1][m];
            const double2 tt = acc_at(2, m);
            u[m] = make_double2(tt.x - a.x * csc * vt[m].x * orad - vp[m].x * b.x * csc * orad,
                                tt.y - a.y * csc * vt[m].y * orad - vp[m].y * b.y * csc * orad);
        }
        dft_small(3, u, -1);
#pragma unroll
        for (int m = 0; m < 3; ++m) acc_at(2, m) = u[m];
#pragma unroll
        for (int f = 0; f < 4; f += (f == 1 ? 2 : 1)) {   // W, P, Z
#pragma unroll
            for (int m = 0; m < 3; ++m) u[m] = acc_at(f, m);
            dft_small(3, u, -1);
#pragma unroll
            for (int m = 0; m < 3; ++m) acc_at(f, m) = u[m];
        }
    }
    // CFL (Find_MyMinDT)
    double cmax = 0.0;
    {
        const double orad = rowc[RC_ORAD], dr = rowc[RC_DR];
        const double hfac = P.llmax * orad * orad, rfac = 1.0 / (dr * dr);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            cmax = fmax(cmax, (vt[m].x * vt[m].x + vp[m].x * vp[m].x) * hfac);
            cmax = fmax(cmax, (vt[m].y * vt[m].y + vp[m].y * vp[m].y) * hfac);
            cmax = fmax(cmax, vr[m].x * vr[m].x * rfac);
            cmax = fmax(cmax, vr[m].y * vr[m].y * rfac);
        }
    }
    __syncthreads();
    // the r2c's remaining passes (reverse order, decimation in time) in shared memory
    fft_dit_from_second<N, 4, NT>(acc, P.twp, t);
    {
        constexpr int NI = N / 2 + 1;
        const int L = P.L;
        for (int g = t; g < 4 * NI; g += NT) {
            const int f = g / NI, k = g - f * NI;
            const double2 zk = acc[f * FS + S::slot(k)];
            const double2 zn = acc[f * FS + S::slot((N - k) % N)];
            const double2 wk = __ldg(P.wr + k);
            const double hs = (f & 1) ? rowc[RC_HSF] : 0.5;
            auto xval = [&](double2 a, double2 b, double2 w, bool zero_im) {
                const double2 bn = cconj(b);
                const double2 e = make_double2(hs * (a.x + bn.x), hs * (a.y + bn.y));
                const double2 d = make_double2(hs * (a.x - bn.x), hs * (a.y - bn.y));
                const double2 wd = cmul(cconj(w), d);
                double2 X = make_double2(e.x + wd.y, e.y - wd.x);
                if (zero_im) X.y = 0.0;
                return X;
            };
            // both values are read before either is written: k and N - k belong to this item only
            const bool wk_ok = k < L, wn_ok = k != 0 && 2 * k != N && N - k < L;
            const double2 xk = xval(zk, zn, wk, k == 0);
            const double2 xn = xval(zn, zk, make_double2(-wk.x, wk.y), false);
            if (wk_ok) acc[f * FS + S::slot(k)] = xk;
            if (wn_ok) acc[f * FS + S::slot(N - k)] = xn;
        }
    }
    cluster.sync();
    {
        const double2* peer = cluster.map_shared_rank(acc, h ^ 1);
        const int L = P.L;
        const long mstride = 2L * (P.nth / 2) * P.ncolb;
        double* obase = P.p2b + (long)h * (P.nth / 2) * P.ncolb + (long)thh * P.ncolb + (long)r * (2 * P.nfb);
        for (int g = t; g < 4 * L; g += NT) {
            const int k = g >> 2, f = g & 3;
            const double2 a = acc[f * FS + S::slot(k)], b = peer[f * FS + S::slot(k)];
            const double2 v = h ? csub(b, a) : cadd(a, b);
            *reinterpret_cast<double2*>(obase + k * mstride + f * 2) = v;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_down_sync(0xffffffffu, cmax, o));
    if ((t & 31) == 0) red[t >> 5] = cmax;
    cluster.sync();
    if (t == 0) {
        double v = red[0];
        for (int i = 1; i < NT / 32; ++i) v = fmax(v, red[i]);
        atomicMax(P.cfl, (unsigned long long)__double_as_longlong(v));
    }
}

// the register-last-pass kernel serves the n_theta whose plan ends in radix 3
static bool p3_supported(int n) { return n == 384 || n == 768 || n == 1536; }

// n_theta with an instance of physics_kernel (all passes in shared memory)
bool physics_form1_supported(int n) {
    switch (n) {
        case 24: case 32: case 48: case 64: case 96: case 128: case 192: case 256: case 384: case 512: case 768:
            return true;
        default:
            return false;
    }
}

void launch_physics(Ctx& c) {
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.p2b = c.d_p2b;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    if (!c.d_twp) throw ArgError("physics tables not prepared (physics_prepare runs at set-up)");
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.cfl = c.d_cfl;
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    P.ncolb = c.nfb * c.d.nr * 2;
    P.coriolis = c.rad.coriolis;
    P.rotation = c.cfg.rotation;
    P.llmax = (double)c.d.lmax * (c.d.lmax + 1);
    P.lorentz = c.cfg.magnetism ? c.rad.lorentz : 0.0;
    make_plan(c.d.nth);   // validates n_theta = 2^a 3^b
    if (c.d.L > (2 * c.d.nth) / 3 + 1)
        throw ArgError("n_theta must be at least 3 (l_max + 1) / 2 for the physical-space kernel");
    const unsigned grid = 2u * (unsigned)c.d.nth2 * (unsigned)c.d.nr;   // clusters of 2 rows
    if (c.physics3_ok && c.physics_form != 1 && !c.mag && !c.rad.heating) {   // last pass in registers (form 0: two CTAs per SM, 2: one)
        auto go3 = [&](auto kern, int nt, size_t units) {
            const size_t smem = units * sizeof(double2);
            RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            kern<<<grid, nt, smem, c.stream>>>(P);
        };
        const bool two = c.physics_form == 0;
        switch (c.d.nth) {
            case 384:
                if (two) go3(physics3_kernel<384, 2>, P3<384>::NT, P3<384>::SIZE);
                else go3(physics3_kernel<384, 1>, P3<384>::NT, P3<384>::SIZE);
                break;
            case 768:
                if (two) go3(physics3_kernel<768, 2>, P3<768>::NT, P3<768>::SIZE);
                else go3(physics3_kernel<768, 1>, P3<768>::NT, P3<768>::SIZE);
                break;
            default:   // 1536: 512 threads and 197 KB of shared memory, one CTA per SM
                go3(physics3_kernel<1536, 1>, P3<1536>::NT, P3<1536>::SIZE);
                break;
        }
        RA_CUDA(cudaGetLastError());
        ++c.launches;
        return;
    }
    auto go = [&](auto kern, int n, size_t smem_units) {
        const size_t smem = smem_units * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, ROW_THREADS, smem, c.stream>>>(P);
        (void)n;
    };
#define RA_PHYS_CASE(NN)                                                   \
    case NN:                                                               \
        if (c.mag && heat)                                                 \
            go(physics_kernel<NN, true, true>, NN, RowSmem<NN>::SIZE);     \
        else if (c.mag)                                                    \
            go(physics_kernel<NN, true, false>, NN, RowSmem<NN>::SIZE);    \
        else if (heat)                                                     \
            go(physics_kernel<NN, false, true>, NN, RowSmem<NN>::SIZE);    \
        else                                                               \
            go(physics_kernel<NN, false, false>, NN, RowSmem<NN>::SIZE);   \
        break;
    const bool heat = c.rad.heating;
    switch (c.d.nth) {
        RA_PHYS_CASE(24)
        RA_PHYS_CASE(32)
        RA_PHYS_CASE(48)
        RA_PHYS_CASE(64)
        RA_PHYS_CASE(96)
        RA_PHYS_CASE(128)
        RA_PHYS_CASE(192)
        RA_PHYS_CASE(256)
        RA_PHYS_CASE(384)
        RA_PHYS_CASE(512)
        RA_PHYS_CASE(768)
#undef RA_PHYS_CASE
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


// Benchmark_Checkup's volume-averaged kinetic energy (Benchmarking.F90:645-656,
// 733-736) of the velocity in p2a.  One CTA per (theta, r) row forms v_r,
// v_theta, v_phi on the phi grid with the physics kernel's c2r and writes the
// row's share w_theta w_r rho / 2 * mean_phi |u|^2; kew holds the theta weights
// (Gauss-Legendre weight / 2 / n_phi, ComputeEll0) and then the radial
// integration weights (Compute_Radial_Average).  No cluster: each row reads
// its own hemisphere's reflection of the even and odd parts.
template <int N, bool ME>
__global__ void __launch_bounds__(ROW_THREADS) kinetic_energy_rows_kernel(PhysParams P, const double* __restrict__ kew,
                                                                          double* __restrict__ rows) {
    // ME: |B|^2 from B_r and r sin(theta) B_theta, B_phi (Benchmarking.F90:689-696), else rho |u|^2 / 2
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    __shared__ double red[ROW_THREADS / 32];
    const int t = threadIdx.x;
    const int h = (int)(blockIdx.x & 1);
    const int nr = P.nr;
    const int pair = (int)(blockIdx.x >> 1);
    const int r = pair % nr;
    const int thh = pair / nr;
    const int th = h ? (N - 1 - thh) : thh;
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    int fo[3] = {A_VR, A_VT, A_VP};
    if (ME) {
        fo[0] = A_BR;
        fo[1] = A_BT;
        fo[2] = A_BP;
    }
    const bool dp[3] = {false, false, false};
    double2 y[FB][ZPT];
    row_c2r<N, 3, ZPT>(P, rowbase, h, fo, dp, sm, t, y);
    const double csc = ME ? P.trig[2 * N + th] * P.radial[R_OVER_R * nr + r] : P.trig[2 * N + th];
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < ZPT; ++q)
        if (t + q * ROW_THREADS < N) {
            const double2 a = y[0][q];
            const double2 b = make_double2(y[1][q].x * csc, y[1][q].y * csc);
            const double2 c = make_double2(y[2][q].x * csc, y[2][q].y * csc);
            s += (a.x * a.x + b.x * b.x + c.x * c.x) + (a.y * a.y + b.y * b.y + c.y * c.y);
        }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((t & 31) == 0) red[t >> 5] = s;
    __syncthreads();
    if (t == 0) {
        double v = red[0];
        for (int i = 1; i < ROW_THREADS / 32; ++i) v += red[i];
        const double w = ME ? 1.0 : 0.5 * P.radial[R_DENSITY * nr + r];
        rows[(long)th * nr + r] = w * v * kew[th] * kew[N + r];
    }
}

// Sum of the row shares in a fixed order (one CTA): the result is the same on
// every call for the same state.
__global__ void __launch_bounds__(1024) kinetic_energy_sum_kernel(const double* __restrict__ rows, long n,
                                                                  double* __restrict__ out) {
    __shared__ double red[32];
    const int t = threadIdx.x;
    double s = 0.0;
    for (long i = t; i < n; i += 1024) s += rows[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((t & 31) == 0) red[t >> 5] = s;
    __syncthreads();
    if (t == 0) {
        double v = red[0];
        for (int i = 1; i < 32; ++i) v += red[i];
        *out = v;
    }
}

void launch_kinetic_energy(Ctx& c, bool magnetic) {
    if (magnetic && !c.mag) throw ArgError("the magnetic energy needs a context created with magnetism");
    if (!c.d_twp || !c.d_kew || !c.d_ke_rows) throw ArgError("diagnostic tables not prepared at set-up");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const unsigned grid = 2u * (unsigned)c.d.nth2 * (unsigned)c.d.nr;
    auto go = [&](auto kern, int n) {
        const size_t smem = (size_t)3 * fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, ROW_THREADS, smem, c.stream>>>(P, c.d_kew, c.d_ke_rows);
    };
    switch (c.d.nth) {
        case 24: if (magnetic) go(kinetic_energy_rows_kernel<24, true>, 24); else go(kinetic_energy_rows_kernel<24, false>, 24); break;
        case 32: if (magnetic) go(kinetic_energy_rows_kernel<32, true>, 32); else go(kinetic_energy_rows_kernel<32, false>, 32); break;
        case 48: if (magnetic) go(kinetic_energy_rows_kernel<48, true>, 48); else go(kinetic_energy_rows_kernel<48, false>, 48); break;
        case 64: if (magnetic) go(kinetic_energy_rows_kernel<64, true>, 64); else go(kinetic_energy_rows_kernel<64, false>, 64); break;
        case 96: if (magnetic) go(kinetic_energy_rows_kernel<96, true>, 96); else go(kinetic_energy_rows_kernel<96, false>, 96); break;
        case 128: if (magnetic) go(kinetic_energy_rows_kernel<128, true>, 128); else go(kinetic_energy_rows_kernel<128, false>, 128); break;
        case 192: if (magnetic) go(kinetic_energy_rows_kernel<192, true>, 192); else go(kinetic_energy_rows_kernel<192, false>, 192); break;
        case 256: if (magnetic) go(kinetic_energy_rows_kernel<256, true>, 256); else go(kinetic_energy_rows_kernel<256, false>, 256); break;
        case 384: if (magnetic) go(kinetic_energy_rows_kernel<384, true>, 384); else go(kinetic_energy_rows_kernel<384, false>, 384); break;
        case 512: if (magnetic) go(kinetic_energy_rows_kernel<512, true>, 512); else go(kinetic_energy_rows_kernel<512, false>, 512); break;
        case 768: if (magnetic) go(kinetic_energy_rows_kernel<768, true>, 768); else go(kinetic_energy_rows_kernel<768, false>, 768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no kinetic-energy kernel instance");
    }
    RA_CUDA(cudaGetLastError());
    kinetic_energy_sum_kernel<<<1, 1024, 0, c.stream>>>(c.d_ke_rows, (long)c.d.nth * c.d.nr,
                                                        c.d_ke_rows + (long)c.d.nth * c.d.nr);
    RA_CUDA(cudaGetLastError());
    c.launches += 2;
}

// Natural phi index of buffer position p after the in-place DIF passes: with
// p = sum_s d_s SS_s (SS_s the stride of pass s), n = d_0 + R_0 (d_1 + R_1 (d_2 + ...)).
template <int N>
__device__ __forceinline__ int natural_index(int p) {
    int n = 0, mul = 1;
#pragma unroll
    for (int s = 0; s < npass_of(N); ++s) {
        const int R = radix_at(N, s), SS = ip_ls(N, s) / R;
        n += ((p / SS) % R) * mul;
        mul *= R;
    }
    return n;
}

// One buffer-field sum C (DiagCombo) on the row into e[.]: a c2r per term.
template <int N, int ZPT>
__device__ __forceinline__ void row_combo(const PhysParams& P, const DiagCombo& C, const double* rowbase, int h,
                                          int th, int r, double2* sm, int t, double2 (&y)[FB][ZPT],
                                          double2 (&e)[ZPT]) {
    const double csc = P.trig[2 * N + th], cot = P.trig[3 * N + th];
    const double rad = P.radial[R_RADIUS * P.nr + r], orad = P.radial[R_OVER_R * P.nr + r];
    const double rdl = rad * P.radial[R_DLNRHO * P.nr + r] + 2.0;
#pragma unroll
    for (int q = 0; q < ZPT; ++q) e[q] = make_double2(0.0, 0.0);
#pragma unroll 1
    for (int j = 0; j < C.nt; ++j) {
        const DiagTerm T = C.t[j];
        const int fo[1] = {T.field};
        const bool dp[1] = {T.dphi != 0};
        row_c2r<N, 1, ZPT>(P, rowbase, h, fo, dp, sm, t, y, C.mpart);
        const double tf = T.th == 1 ? csc : (T.th == 2 ? cot : (T.th == 3 ? csc * cot : (T.th == 4 ? csc * csc : 1.0)));
        const double rf = T.rad == 1 ? orad : (T.rad == 2 ? rad : (T.rad == 3 ? rdl : 1.0));
        const double cs = T.c * tf * rf;
#pragma unroll
        for (int q = 0; q < ZPT; ++q) {
            e[q].x += cs * y[0][q].x;
            e[q].y += cs * y[0][q].y;
        }
    }
}

// The diagnostic quantity S on the row (theta index th, radial index r) into y[0][.]: one
// field through the c2r (d/dphi in the spectrum, its fluctuating or mean part by mpart), or
// a sum of products of buffer-field sums (the vorticity components, the energy densities,
// enstrophy, helicity, J.J: SliceSpec.nprod), times 1, rho(r) / 2, a constant, rho(r) T(r),
// its square or rho(r).  Returns the
// factor the caller still applies: the single field's 1/sin(theta) and 1/r, 1 for a product.
template <int N, int ZPT>
__device__ __forceinline__ double row_quantity(const PhysParams& P, const SliceSpec& S, const double* rowbase,
                                               int h, int th, int r, double2* sm, int t, double2 (&y)[FB][ZPT]) {
    const double csc = P.trig[2 * N + th], orad = P.radial[R_OVER_R * P.nr + r];
    if (S.nprod == 0) {
        const int fo[1] = {S.field};
        const bool dp[1] = {S.dphi != 0};
        row_c2r<N, 1, ZPT>(P, rowbase, h, fo, dp, sm, t, y, S.mpart);
        return (S.csc ? csc : 1.0) * (S.orad ? orad : 1.0);
    }
    double2 acc[ZPT], a[ZPT], b[ZPT];
#pragma unroll
    for (int q = 0; q < ZPT; ++q) acc[q] = make_double2(0.0, 0.0);
#pragma unroll 1
    for (int i = 0; i < S.nprod; ++i) {
        row_combo<N, ZPT>(P, S.a[i], rowbase, h, th, r, sm, t, y, a);
        if (S.bsame[i]) {
#pragma unroll
            for (int q = 0; q < ZPT; ++q) b[q] = a[q];
        } else if (S.b[i].nt == 0) {
#pragma unroll
            for (int q = 0; q < ZPT; ++q) b[q] = make_double2(1.0, 1.0);
        } else {
            row_combo<N, ZPT>(P, S.b[i], rowbase, h, th, r, sm, t, y, b);
        }
#pragma unroll
        for (int q = 0; q < ZPT; ++q) {
            acc[q].x += a[q].x * b[q].x;
            acc[q].y += a[q].y * b[q].y;
        }
    }
    const double rt = P.radial[R_RHO_T * P.nr + r];
    const double rho = P.radial[R_DENSITY * P.nr + r];
    const double c = S.coef == 1 ? 0.5 * rho
                                 : (S.coef == 2 ? S.cval
                                                : (S.coef == 3 ? rt : (S.coef == 4 ? rt * rt : (S.coef == 5 ? rho : 1.0))));
#pragma unroll
    for (int q = 0; q < ZPT; ++q) y[0][q] = make_double2(acc[q].x * c, acc[q].y * c);
    return 1.0;
}

// Shell slices (Spherical_IO.F90 Shell_Slices) of one diagnostic quantity: one
// CTA per (theta, level) row forms the quantity on the phi grid from p2a with
// the physics kernel's c2r (d/dphi in the spectrum, 1/sin(theta) where the
// physical-space stage divides by it) and writes the row in natural phi order:
// out[level][theta][phi].
template <int N>
__global__ void __launch_bounds__(ROW_THREADS) shell_slice_kernel(PhysParams P, SliceSpec S, double* __restrict__ out) {
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    const int t = threadIdx.x;
    const int h = (int)(blockIdx.x & 1);
    const int thh = (int)(blockIdx.x >> 1);
    const int th = h ? (N - 1 - thh) : thh;
    const int lv = (int)blockIdx.y;
    const int r = S.level[lv];
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    double2 y[FB][ZPT];
    const double scale = row_quantity<N, ZPT>(P, S, rowbase, h, th, r, sm, t, y);
    double2* row = reinterpret_cast<double2*>(out + ((long)lv * N + th) * (2L * N));
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        const int p = t + q * ROW_THREADS;
        if (p < N) row[natural_index<N>(p)] = make_double2(y[0][q].x * scale, y[0][q].y * scale);
    }
}

void launch_shell_slice(Ctx& c, const SliceSpec& S, double* out) {
    if (!c.d_twp) throw ArgError("physics tables not prepared (physics_prepare runs at set-up)");
    if (S.nl < 1 || S.nl > SliceSpec::MAXL) throw ArgError("shell slice: 1 .. 64 levels per launch");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const dim3 grid(2u * (unsigned)c.d.nth2, (unsigned)S.nl);
    auto go = [&](auto kern, int n) {
        const size_t smem = (size_t)fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, out);
    };
    switch (c.d.nth) {
        case 24: go(shell_slice_kernel<24>, 24); break;
        case 32: go(shell_slice_kernel<32>, 32); break;
        case 48: go(shell_slice_kernel<48>, 48); break;
        case 64: go(shell_slice_kernel<64>, 64); break;
        case 96: go(shell_slice_kernel<96>, 96); break;
        case 128: go(shell_slice_kernel<128>, 128); break;
        case 192: go(shell_slice_kernel<192>, 192); break;
        case 256: go(shell_slice_kernel<256>, 256); break;
        case 384: go(shell_slice_kernel<384>, 384); break;
        case 512: go(shell_slice_kernel<512>, 512); break;
        case 768: go(shell_slice_kernel<768>, 768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no shell-slice kernel instance");
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// Shell averages (Spherical_IO.F90 Shell_Averages, ComputeEll0 :1350-1391) of
// one diagnostic quantity: one CTA per (theta, r) row forms the quantity on the
// phi grid (as shell_slice_kernel) and writes its theta-weighted phi sum:
// MOMENTS = false, sum q (the mean's share, slot 0); MOMENTS = true, the sums
// of (q - mean(r))^m for m = 2, 3, 4 (slots 1-3).  rows[slot][theta][r];
// kew[theta] = Gauss-Legendre weight / 2 / n_phi.
template <int N, bool MOMENTS>
__global__ void __launch_bounds__(ROW_THREADS) shell_moment_rows_kernel(PhysParams P, SliceSpec S,
                                                                        const double* __restrict__ kew,
                                                                        const double* __restrict__ mean,
                                                                        double* __restrict__ rows) {
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    __shared__ double red[3][ROW_THREADS / 32];
    const int t = threadIdx.x;
    const int h = (int)(blockIdx.x & 1);
    const int thh = (int)(blockIdx.x >> 1);
    const int th = h ? (N - 1 - thh) : thh;
    const int r = (int)blockIdx.y;
    const int nr = P.nr;
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    double2 y[FB][ZPT];
    const double scale = row_quantity<N, ZPT>(P, S, rowbase, h, th, r, sm, t, y);
    const double mu = MOMENTS ? mean[r] : 0.0;
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
    for (int q = 0; q < ZPT; ++q)
        if (t + q * ROW_THREADS < N) {
            const double a = y[0][q].x * scale - mu, b = y[0][q].y * scale - mu;
            if (MOMENTS) {
                const double a2 = a * a, b2 = b * b;
                s1 += a2 + b2;
                s2 += a2 * a + b2 * b;
                s3 += a2 * a2 + b2 * b2;
            } else {
                s1 += a + b;
            }
        }
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        if (MOMENTS) {
            s2 += __shfl_down_sync(0xffffffffu, s2, o);
            s3 += __shfl_down_sync(0xffffffffu, s3, o);
        }
    }
    if ((t & 31) == 0) {
        red[0][t >> 5] = s1;
        red[1][t >> 5] = s2;
        red[2][t >> 5] = s3;
    }
    __syncthreads();
    if (t < (MOMENTS ? 3 : 1)) {
        double v = red[t][0];
        for (int i = 1; i < ROW_THREADS / 32; ++i) v += red[t][i];
        const int slot = MOMENTS ? 1 + t : 0;
        rows[((long)slot * N + th) * nr + r] = v * kew[th];
    }
}

// out[slot][r] = sum over theta of rows[slot][theta][r], in a fixed order (one
// CTA per (r, slot)).
__global__ void __launch_bounds__(256) shell_reduce_kernel(const double* __restrict__ rows, int nth, int nr,
                                                           int slot0, double* __restrict__ out) {
    __shared__ double red[8];
    const int r = (int)blockIdx.x, slot = slot0 + (int)blockIdx.y, t = threadIdx.x;
    double s = 0.0;
    for (int th = t; th < nth; th += 256) s += rows[((long)slot * nth + th) * nr + r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((t & 31) == 0) red[t >> 5] = s;
    __syncthreads();
    if (t == 0) {
        double v = red[0];
        for (int i = 1; i < 8; ++i) v += red[i];
        out[(long)slot * nr + r] = v;
    }
}

// The four shell moments of one quantity into out[4][nr] (device): mean, then
// the theta-phi averages of (q - mean)^2, ^3, ^4.  rows: 4 nth nr scratch.
void launch_shell_moments(Ctx& c, const SliceSpec& S, double* rows, double* out) {
    if (!c.d_twp || !c.d_kew) throw ArgError("diagnostic tables not prepared at set-up");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const dim3 grid(2u * (unsigned)c.d.nth2, (unsigned)c.d.nr);
    auto go = [&](auto k0, auto k1, int n) {
        const size_t smem = (size_t)fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        RA_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k0<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, c.d_kew, out, rows);
        RA_CUDA(cudaGetLastError());
        shell_reduce_kernel<<<dim3((unsigned)c.d.nr, 1), 256, 0, c.stream>>>(rows, c.d.nth, c.d.nr, 0, out);
        RA_CUDA(cudaGetLastError());
        k1<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, c.d_kew, out, rows);   // reads the mean, out[0][r]
        RA_CUDA(cudaGetLastError());
        shell_reduce_kernel<<<dim3((unsigned)c.d.nr, 3), 256, 0, c.stream>>>(rows, c.d.nth, c.d.nr, 1, out);
        RA_CUDA(cudaGetLastError());
    };
#define RA_MOM(n) go(shell_moment_rows_kernel<n, false>, shell_moment_rows_kernel<n, true>, n)
    switch (c.d.nth) {
        case 24: RA_MOM(24); break;
        case 32: RA_MOM(32); break;
        case 48: RA_MOM(48); break;
        case 64: RA_MOM(64); break;
        case 96: RA_MOM(96); break;
        case 128: RA_MOM(128); break;
        case 192: RA_MOM(192); break;
        case 256: RA_MOM(256); break;
        case 384: RA_MOM(384); break;
        case 512: RA_MOM(512); break;
        case 768: RA_MOM(768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no shell-average kernel instance");
    }
#undef RA_MOM
    c.launches += 4;
}

// Azimuthal averages (AZ_Avgs) of one quantity: the phi mean of every
// (theta, r) row into rows[theta][r] (the shell-moment row kernel with the
// weights 1 / n_phi).
void launch_azimuthal_average(Ctx& c, const SliceSpec& S, double* rows) {
    if (!c.d_twp || !c.d_kaz) throw ArgError("diagnostic tables not prepared at set-up");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const dim3 grid(2u * (unsigned)c.d.nth2, (unsigned)c.d.nr);
    auto go = [&](auto k0, int n) {
        const size_t smem = (size_t)fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k0<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, c.d_kaz, nullptr, rows);
    };
#define RA_AZ(n) go(shell_moment_rows_kernel<n, false>, n)
    switch (c.d.nth) {
        case 24: RA_AZ(24); break;
        case 32: RA_AZ(32); break;
        case 48: RA_AZ(48); break;
        case 64: RA_AZ(64); break;
        case 96: RA_AZ(96); break;
        case 128: RA_AZ(128); break;
        case 192: RA_AZ(192); break;
        case 256: RA_AZ(256); break;
        case 384: RA_AZ(384); break;
        case 512: RA_AZ(512); break;
        case 768: RA_AZ(768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no azimuthal-average kernel instance");
    }
#undef RA_AZ
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// Shell spectra (Shell_Spectra output; Parallel_IO.F90 Spectral_Prep
// :973-1047): the quantity on the phi grid (as shell_slice_kernel), its
// unnormalised r2c (FFT_To_Spectral) and the equatorial fold of PtS with the
// partner row (theta, pi - theta in one cluster, as physics_kernel), written
// into the p2b layout at the column slot slot0 + level index; the forward
// Legendre transform of that buffer then gives the (l, m) coefficients.
template <int N>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(ROW_THREADS)
    spectra_rows_kernel(PhysParams P, SliceSpec S, int slot0, double* __restrict__ p2b) {
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    constexpr int NI = N / 2 + 1;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    const int t = threadIdx.x;
    const int h = (int)cluster.block_rank();
    const int thh = (int)(blockIdx.x >> 1);
    const int th = h ? (N - 1 - thh) : thh;
    const int lv = (int)blockIdx.y;
    const int r = S.level[lv];
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    double2 y[FB][ZPT];
    const double scale = row_quantity<N, ZPT>(P, S, rowbase, h, th, r, buf, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {   // each thread rewrites the positions it read
        const int p = t + q * ROW_THREADS;
        if (p < N) buf[p] = make_double2(y[0][q].x * scale, y[0][q].y * scale);
    }
    __syncthreads();
    fft_dit<N, 1, ROW_THREADS>(buf, P.twp, t);
    const int L = P.L;
    for (int k = t; k < NI; k += ROW_THREADS) {   // r2c steps, one (k, N - k) pair per item, in place
        const double2 zk = buf[k];
        const double2 zn = buf[(N - k) % N];
        const double2 wk = __ldg(P.wr + k);
        auto xval = [&](double2 a, double2 b, double2 w, bool zero_im) {
            const double2 bn = cconj(b);
            const double2 e = make_double2(0.5 * (a.x + bn.x), 0.5 * (a.y + bn.y));
            const double2 d = make_double2(0.5 * (a.x - bn.x), 0.5 * (a.y - bn.y));
            const double2 wd = cmul(cconj(w), d);
            double2 X = make_double2(e.x + wd.y, e.y - wd.x);
            if (zero_im) X.y = 0.0;
            return X;
        };
        if (k < L) buf[k] = xval(zk, zn, wk, k == 0);
        if (k != 0 && 2 * k != N && N - k < L) buf[N - k] = xval(zn, zk, make_double2(-wk.x, wk.y), false);
    }
    cluster.sync();
    {
        const double2* peer = cluster.map_shared_rank(buf, h ^ 1);
        const long ncolb = (long)P.nfb * P.nr * 2;
        const long mstride = 2L * (N / 2) * ncolb;   // p2b[m][par][theta_h][col]
        double* obase = p2b + (long)h * (N / 2) * ncolb + (long)thh * ncolb + (long)(slot0 + lv) * 2;
        for (int k = t; k < L; k += ROW_THREADS) {
            const double2 a = buf[k], b = peer[k];
            *reinterpret_cast<double2*>(obase + k * mstride) = h ? csub(b, a) : cadd(a, b);
        }
    }
    cluster.sync();   // the partner has finished reading this CTA's spectrum
}

// (l, m) coefficients of ns consecutive column slots of the forward transform's
// output s2[row][slot][re/im] into out[slot][re/im][m][l] (zero for l < m).
__global__ void spectra_gather_kernel(const double* __restrict__ s2, int L, int nslots, long rowlen,
                                      double* __restrict__ out) {
    const long total = (long)nslots * 2 * L * L;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int l = (int)(i % L);
        const long rest = i / L;
        const int m = (int)(rest % L);
        const int ri = (int)((rest / L) % 2);
        const int s = (int)(rest / (2L * L));
        out[i] = (l >= m) ? s2[row_index(m, l, L) * rowlen + (long)s * 2 + ri] : 0.0;
    }
}

void launch_spectra_rows(Ctx& c, const SliceSpec& S, int slot0, double* p2b) {
    if (!c.d_twp) throw ArgError("physics tables not prepared (physics_prepare runs at set-up)");
    if (S.nl < 1 || S.nl > SliceSpec::MAXL) throw ArgError("shell spectra: 1 .. 64 levels per launch");
    if (slot0 < 0 || slot0 + S.nl > c.nfb * c.d.nr) throw ArgError("shell spectra: column slots out of range");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const dim3 grid(2u * (unsigned)c.d.nth2, (unsigned)S.nl);
    auto go = [&](auto kern, int n) {
        const size_t smem = (size_t)fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, slot0, p2b);
    };
    switch (c.d.nth) {
        case 24: go(spectra_rows_kernel<24>, 24); break;
        case 32: go(spectra_rows_kernel<32>, 32); break;
        case 48: go(spectra_rows_kernel<48>, 48); break;
        case 64: go(spectra_rows_kernel<64>, 64); break;
        case 96: go(spectra_rows_kernel<96>, 96); break;
        case 128: go(spectra_rows_kernel<128>, 128); break;
        case 192: go(spectra_rows_kernel<192>, 192); break;
        case 256: go(spectra_rows_kernel<256>, 256); break;
        case 384: go(spectra_rows_kernel<384>, 384); break;
        case 512: go(spectra_rows_kernel<512>, 512); break;
        case 768: go(spectra_rows_kernel<768>, 768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no shell-spectra kernel instance");
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

void launch_spectra_gather(Ctx& c, const double* s2, int nslots, double* out) {
    const long total = (long)nslots * 2 * c.d.L * c.d.L;
    const unsigned blocks = (unsigned)std::min<long>((total + 255) / 256, 148L * 16);
    spectra_gather_kernel<<<blocks, 256, 0, c.stream>>>(s2, c.d.L, nslots, (long)c.nfb * c.d.nr * 2, out);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// Equatorial slices (Spherical_IO.F90:394-398: the theta rows n_theta/2 and
// n_theta/2 + 1, weights 1/2 each): the pair of rows nearest the equator is one
// cluster (theta_h = n_theta/2 - 1); each CTA forms its row on the phi grid (as
// shell_slice_kernel) and rank 0 averages the two through distributed shared
// memory into out[r][phi] (natural phi order).  One cluster per radius.
template <int N>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(ROW_THREADS)
    equatorial_slice_kernel(PhysParams P, SliceSpec S, double* __restrict__ out) {
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    const int t = threadIdx.x;
    const int h = (int)cluster.block_rank();
    const int thh = N / 2 - 1;
    const int th = h ? (N - 1 - thh) : thh;
    const int r = (int)blockIdx.y;
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    double2 y[FB][ZPT];
    const double scale = row_quantity<N, ZPT>(P, S, rowbase, h, th, r, buf, t, y);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {   // each thread rewrites the positions it read
        const int p = t + q * ROW_THREADS;
        if (p < N) buf[p] = make_double2(y[0][q].x * scale, y[0][q].y * scale);
    }
    cluster.sync();
    if (h == 0) {
        const double2* peer = cluster.map_shared_rank(buf, 1);
        double2* row = reinterpret_cast<double2*>(out + (long)r * (2L * N));
        for (int p = t; p < N; p += ROW_THREADS) {
            const double2 a = buf[p], b = peer[p];
            row[natural_index<N>(p)] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
        }
    }
    cluster.sync();   // the partner has finished reading this CTA's row
}

void launch_equatorial_slice(Ctx& c, const SliceSpec& S, double* out) {
    if (!c.d_twp) throw ArgError("physics tables not prepared (physics_prepare runs at set-up)");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const dim3 grid(2u, (unsigned)c.d.nr);
    auto go = [&](auto kern, int n) {
        const size_t smem = (size_t)fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, out);
    };
    switch (c.d.nth) {
        case 24: go(equatorial_slice_kernel<24>, 24); break;
        case 32: go(equatorial_slice_kernel<32>, 32); break;
        case 48: go(equatorial_slice_kernel<48>, 48); break;
        case 64: go(equatorial_slice_kernel<64>, 64); break;
        case 96: go(equatorial_slice_kernel<96>, 96); break;
        case 128: go(equatorial_slice_kernel<128>, 128); break;
        case 192: go(equatorial_slice_kernel<192>, 192); break;
        case 256: go(equatorial_slice_kernel<256>, 256); break;
        case 384: go(equatorial_slice_kernel<384>, 384); break;
        case 512: go(equatorial_slice_kernel<512>, 512); break;
        case 768: go(equatorial_slice_kernel<768>, 768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no equatorial-slice kernel instance");
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// Meridional slices (Spherical_IO.F90:384-387, 467-473): the quantity at
// chosen phi indices (S.level[0 .. S.nl) holds them here) at every (theta, r);
// one CTA per row forms the row on the phi grid, puts it in natural order in
// shared memory and writes the chosen points to out[j][theta][r].
template <int N>
__global__ void __launch_bounds__(ROW_THREADS) meridional_slice_kernel(PhysParams P, SliceSpec S,
                                                                       double* __restrict__ out) {
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    const int t = threadIdx.x;
    const int h = (int)(blockIdx.x & 1);
    const int thh = (int)(blockIdx.x >> 1);
    const int th = h ? (N - 1 - thh) : thh;
    const int r = (int)blockIdx.y;
    const int nr = P.nr;
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    double2 y[FB][ZPT];
    const double scale = row_quantity<N, ZPT>(P, S, rowbase, h, th, r, buf, t, y);
    __syncthreads();   // every thread has read its points out of the buffer
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        const int p = t + q * ROW_THREADS;
        if (p < N) buf[natural_index<N>(p)] = make_double2(y[0][q].x * scale, y[0][q].y * scale);
    }
    __syncthreads();
    const double* row = reinterpret_cast<const double*>(buf);   // natural phi order
    for (int j = t; j < S.nl; j += ROW_THREADS) out[((long)j * N + th) * nr + r] = row[S.level[j]];
}

void launch_meridional_slice(Ctx& c, const SliceSpec& S, double* out) {
    if (!c.d_twp) throw ArgError("physics tables not prepared (physics_prepare runs at set-up)");
    if (S.nl < 1 || S.nl > SliceSpec::MAXL) throw ArgError("meridional slices: 1 .. 64 phi indices");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const dim3 grid(2u * (unsigned)c.d.nth2, (unsigned)c.d.nr);
    auto go = [&](auto kern, int n) {
        const size_t smem = (size_t)fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, out);
    };
    switch (c.d.nth) {
        case 24: go(meridional_slice_kernel<24>, 24); break;
        case 32: go(meridional_slice_kernel<32>, 32); break;
        case 48: go(meridional_slice_kernel<48>, 48); break;
        case 64: go(meridional_slice_kernel<64>, 64); break;
        case 96: go(meridional_slice_kernel<96>, 96); break;
        case 128: go(meridional_slice_kernel<128>, 128); break;
        case 192: go(meridional_slice_kernel<192>, 192); break;
        case 256: go(meridional_slice_kernel<256>, 256); break;
        case 384: go(meridional_slice_kernel<384>, 384); break;
        case 512: go(meridional_slice_kernel<512>, 512); break;
        case 768: go(meridional_slice_kernel<768>, 768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no meridional-slice kernel instance");
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// out[0] = sum_r w[r] v[r] in a fixed order (one warp).
__global__ void radial_dot_kernel(const double* __restrict__ v, const double* __restrict__ w, int nr,
                                  double* __restrict__ out) {
    double s = 0.0;
    for (int r = threadIdx.x; r < nr; r += 32) s += w[r] * v[r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = s;
}

// Global average (G_Avgs; Compute_Radial_Average, Spherical_IO.F90:1436-1470)
// of one quantity into out[0]: the spherical means per radius (the shell-moment
// row kernel and the theta reduction) weighted by the radial integration
// weights.  rows: nth nr scratch; mean: nr scratch.
void launch_global_average(Ctx& c, const SliceSpec& S, double* rows, double* mean, double* out) {
    if (!c.d_twp || !c.d_kew) throw ArgError("diagnostic tables not prepared at set-up");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const dim3 grid(2u * (unsigned)c.d.nth2, (unsigned)c.d.nr);
    auto go = [&](auto k0, int n) {
        const size_t smem = (size_t)fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k0<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, c.d_kew, nullptr, rows);
    };
#define RA_GA(n) go(shell_moment_rows_kernel<n, false>, n)
    switch (c.d.nth) {
        case 24: RA_GA(24); break;
        case 32: RA_GA(32); break;
        case 48: RA_GA(48); break;
        case 64: RA_GA(64); break;
        case 96: RA_GA(96); break;
        case 128: RA_GA(128); break;
        case 192: RA_GA(192); break;
        case 256: RA_GA(256); break;
        case 384: RA_GA(384); break;
        case 512: RA_GA(512); break;
        case 768: RA_GA(768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no global-average kernel instance");
    }
#undef RA_GA
    RA_CUDA(cudaGetLastError());
    shell_reduce_kernel<<<dim3((unsigned)c.d.nr, 1), 256, 0, c.stream>>>(rows, c.d.nth, c.d.nr, 0, mean);
    RA_CUDA(cudaGetLastError());
    radial_dot_kernel<<<1, 32, 0, c.stream>>>(mean, c.d_kew + c.d.nth, c.d.nr, out);
    RA_CUDA(cudaGetLastError());
    c.launches += 3;
}

// Point probes (Spherical_IO.F90:379-382: tensor products of radial, theta and
// phi index lists): one CTA per chosen (theta, r) row forms the row on the phi
// grid, in natural order in shared memory, and writes the chosen phi points to
// out[r_i][theta_j][phi_k].
template <int N>
__global__ void __launch_bounds__(ROW_THREADS) point_probe_kernel(PhysParams P, SliceSpec S, ProbeSet Q,
                                                                  double* __restrict__ out) {
    constexpr int ZPT = (N + ROW_THREADS - 1) / ROW_THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    const int t = threadIdx.x;
    const int jt = (int)blockIdx.x, ir = (int)blockIdx.y;
    const int th = Q.theta[jt], r = Q.r[ir];
    const int h = th >= N / 2 ? 1 : 0;
    const int thh = h ? (N - 1 - th) : th;
    const double* rowbase = P.p2a + (long)thh * (2L * P.L * P.ncola) + (long)r * (2 * P.nfa);
    double2 y[FB][ZPT];
    const double scale = row_quantity<N, ZPT>(P, S, rowbase, h, th, r, buf, t, y);
    __syncthreads();   // every thread has read its points out of the buffer
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        const int p = t + q * ROW_THREADS;
        if (p < N) buf[natural_index<N>(p)] = make_double2(y[0][q].x * scale, y[0][q].y * scale);
    }
    __syncthreads();
    const double* row = reinterpret_cast<const double*>(buf);
    for (int k = t; k < Q.nphi; k += ROW_THREADS)
        out[((long)ir * Q.ntheta + jt) * Q.nphi + k] = row[Q.phi[k]];
}

void launch_point_probes(Ctx& c, const SliceSpec& S, const ProbeSet& Q, double* out) {
    if (!c.d_twp) throw ArgError("physics tables not prepared (physics_prepare runs at set-up)");
    PhysParams P{};
    P.p2a = c.d_p2a;
    P.radial = c.d_radial;
    P.trig = c.d_costh;
    P.wr = reinterpret_cast<const double2*>(c.d_twid);
    P.twp = reinterpret_cast<const double2*>(c.d_twp);
    P.L = c.d.L;
    P.nth = c.d.nth;
    P.nr = c.d.nr;
    P.ncola = c.nfa * c.d.nr * 2;
    P.nfa = c.nfa;
    P.nfb = c.nfb;
    const dim3 grid((unsigned)Q.ntheta, (unsigned)Q.nr);
    auto go = [&](auto kern, int n) {
        const size_t smem = (size_t)fstride(n) * sizeof(double2);
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, ROW_THREADS, smem, c.stream>>>(P, S, Q, out);
    };
    switch (c.d.nth) {
        case 24: go(point_probe_kernel<24>, 24); break;
        case 32: go(point_probe_kernel<32>, 32); break;
        case 48: go(point_probe_kernel<48>, 48); break;
        case 64: go(point_probe_kernel<64>, 64); break;
        case 96: go(point_probe_kernel<96>, 96); break;
        case 128: go(point_probe_kernel<128>, 128); break;
        case 192: go(point_probe_kernel<192>, 192); break;
        case 256: go(point_probe_kernel<256>, 256); break;
        case 384: go(point_probe_kernel<384>, 384); break;
        case 512: go(point_probe_kernel<512>, 512); break;
        case 768: go(point_probe_kernel<768>, 768); break;
        default: throw ArgError("n_theta " + std::to_string(c.d.nth) + " has no point-probe kernel instance");
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

}  // namespace ra
