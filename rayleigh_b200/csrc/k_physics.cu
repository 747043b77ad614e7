// Physical-space stage, fused per (r, theta) row:
//   Phi_Derivatives           (Sphere_Physical_Space.F90:745-759) in the spectrum load,
//   fft_to_physical  (c2r)    (Fourier_Transform.F90:142-183), 14 fields,
//   sintheta_div + NL terms   (Sphere_Physical_Space.F90:98-224, 303-700),
//   Find_MyMinDT (CFL max)    (:784-813),
//   fft_to_spectral (r2c)     (Fourier_Transform.F90:100-140), 4 fields,
// reading the inverse Legendre output p2a[m][theta][f][r][re/im] and writing
// p2b[m][theta][f][r][re/im] for m <= l_max.  The reference materialises the
// packed (n_phi+2, r, theta, f) buffers p3a/p3b between these steps; here the
// 18 phi rows of one (r, theta) point never leave the SM.
//
// FFT: a real length-2N transform through one complex length-N transform
// (N = n_theta = 2^a 3^b), Stockham autosort, radix 4/2/3, in shared memory;
// unnormalised like FFTW (the normalisation lives in the Legendre tables).
#include <cmath>

#include "ra_internal.h"

namespace ra {

constexpr int PHYS_THREADS = 256;

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

__device__ __forceinline__ void dft_small(int R, double2* u, int sign) {
    if (R == 2) {
        const double2 a = u[0], b = u[1];
        u[0] = cadd(a, b);
        u[1] = csub(a, b);
    } else if (R == 4) {
        const double2 t0 = cadd(u[0], u[2]), t1 = csub(u[0], u[2]);
        const double2 t2 = cadd(u[1], u[3]), d = csub(u[1], u[3]);
        // w = sign * i : w * (x + i y) = sign * (-y + i x)
        const double2 wd = make_double2(-sign * d.y, sign * d.x);
        u[0] = cadd(t0, t2);
        u[2] = csub(t0, t2);
        u[1] = cadd(t1, wd);
        u[3] = csub(t1, wd);
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

// Runs the FFT on the data in a (b is scratch); returns the buffer holding the result.
// Must be entered with a synchronised input; leaves the result synchronised.
__device__ double2* fft_run(double2* a, double2* b, const FFTPlan& pl, const double2* wr, int sign) {
    const int N = pl.n;
    int p = 1;
    double2* src = a;
    double2* dst = b;
    for (int ps = 0; ps < pl.npass; ++ps) {
        const int R = pl.radix[ps];
        const int T = N / R;
        const int stride = N / (p * R);
        for (int bi = threadIdx.x; bi < T; bi += blockDim.x) {
            const int k = bi % p;
            double2 u[4];
            for (int r = 0; r < R; ++r) u[r] = src[bi + r * T];
            for (int r = 1; r < R; ++r) u[r] = cmul(u[r], twiddle(wr, N, r * k * stride, sign));
            dft_small(R, u, sign);
            const int j = (bi - k) * R + k;
            for (int r = 0; r < R; ++r) dst[j + r * p] = u[r];
        }
        __syncthreads();
        double2* t = src;
        src = dst;
        dst = t;
        p *= R;
    }
    return src;
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
    FFTPlan plan;
};

// c2r of one field of the row into a (real pairs y[2n], y[2n+1] at index n).
template <int ZPT>
__device__ __forceinline__ void row_c2r(const PhysParams& P, int th, int r, int f, bool dphi, double2* bufA,
                                        double2* bufB, const double2* wr, double2 (&out)[ZPT]) {
    const int N = P.nth, L = P.L;
    const long mstride = (long)P.nth * P.ncola;
    const double* base = P.p2a + (long)th * P.ncola + ((long)f * P.nr + r) * 2;
    for (int q = 0; q < ZPT; ++q) {
        const int k = threadIdx.x + q * PHYS_THREADS;
        if (k >= N) break;
        double2 xk = make_double2(0.0, 0.0), xn = make_double2(0.0, 0.0);
        if (k < L) xk = *reinterpret_cast<const double2*>(base + k * mstride);
        const int kn = N - k;   // X_{N-k}; X_N (Nyquist) is zero since L <= N
        if (kn < L) xn = *reinterpret_cast<const double2*>(base + kn * mstride);
        if (dphi) {
            xk = make_double2(-k * xk.y, k * xk.x);
            xn = make_double2(-kn * xn.y, kn * xn.x);
        }
        if (k == 0) xk.y = 0.0;   // c2r ignores Im X_0 (FFTW's Hermitian convention)
        // Z_k = (X_k + conj X_{N-k}) + i w^k (X_k - conj X_{N-k}),  w = exp(2 pi i / 2N)
        const double2 e = cadd(xk, cconj(xn));
        const double2 d = csub(xk, cconj(xn));
        const double2 wd = cmul(wr[k], d);
        bufA[k] = make_double2(e.x - wd.y, e.y + wd.x);
    }
    __syncthreads();
    double2* res = fft_run(bufA, bufB, P.plan, wr, +1);
    for (int q = 0; q < ZPT; ++q) {
        const int n = threadIdx.x + q * PHYS_THREADS;
        out[q] = (n < N) ? res[n] : make_double2(0.0, 0.0);
    }
    __syncthreads();
}

// r2c of one output row (values in regs as (y[2n], y[2n+1])) -> p2b for m < L.
template <int ZPT>
__device__ __forceinline__ void row_r2c(const PhysParams& P, int th, int r, int f, const double2 (&v)[ZPT],
                                        double2* bufA, double2* bufB, const double2* wr) {
    const int N = P.nth, L = P.L;
    for (int q = 0; q < ZPT; ++q) {
        const int n = threadIdx.x + q * PHYS_THREADS;
        if (n < N) bufA[n] = v[q];
    }
    __syncthreads();
    double2* Z = fft_run(bufA, bufB, P.plan, wr, -1);
    const long mstride = (long)P.nth * P.ncolb;
    double* base = P.p2b + (long)th * P.ncolb + ((long)f * P.nr + r) * 2;
    for (int k = threadIdx.x; k < L; k += blockDim.x) {
        const double2 zk = Z[k];
        const double2 zn = cconj(Z[(N - k) % N]);
        const double2 e = make_double2(0.5 * (zk.x + zn.x), 0.5 * (zk.y + zn.y));
        const double2 d = make_double2(0.5 * (zk.x - zn.x), 0.5 * (zk.y - zn.y));
        // X_k = e - i conj(w^k) d
        const double2 wc = cconj(wr[k]);
        const double2 wd = cmul(wc, d);
        double2 X = make_double2(e.x + wd.y, e.y - wd.x);
        if (k == 0) X.y = 0.0;
        *reinterpret_cast<double2*>(base + k * mstride) = X;
    }
    __syncthreads();
}

template <int ZPT>
__global__ void __launch_bounds__(PHYS_THREADS) physics_kernel(PhysParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = P.nth;
    double2* bufA = reinterpret_cast<double2*>(smem_raw);
    double2* bufB = bufA + N;
    double2* wr = bufB + N;
    __shared__ double red[PHYS_THREADS / 32];
    for (int k = threadIdx.x; k < N; k += blockDim.x) wr[k] = P.wr[k];
    const int r = blockIdx.x % P.nr;
    const int th = blockIdx.x / P.nr;
    const int nr = P.nr;
    const double rad = P.radial[R_RADIUS * nr + r];
    const double orad = P.radial[R_OVER_R * nr + r];
    const double rho = P.radial[R_DENSITY * nr + r];
    const double dlnrho = P.radial[R_DLNRHO * nr + r];
    const double dr = P.radial[R_DELTA_R * nr + r];
    const double cs = P.trig[th], sn = P.trig[N + th], csc = P.trig[2 * N + th], cot = P.trig[3 * N + th];
    const double cor = P.rotation ? P.coriolis : 0.0;
    __syncthreads();

    double2 vr[ZPT], vt[ZPT], vp[ZPT], x[ZPT];
    double2 oW[ZPT], oP[ZPT], oT[ZPT], oZ[ZPT];
    row_c2r<ZPT>(P, th, r, A_VR, false, bufA, bufB, wr, vr);
    row_c2r<ZPT>(P, th, r, A_VT, false, bufA, bufB, wr, vt);
    row_c2r<ZPT>(P, th, r, A_VP, false, bufA, bufB, wr, vp);
    double cmax = 0.0;
    const double hfac = P.llmax * orad * orad, rfac = 1.0 / (dr * dr);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        vt[q].x *= csc; vt[q].y *= csc;
        vp[q].x *= csc; vp[q].y *= csc;
        const bool live = (threadIdx.x + q * PHYS_THREADS) < N;
        if (live) {
            cmax = fmax(cmax, (vt[q].x * vt[q].x + vp[q].x * vp[q].x) * hfac);
            cmax = fmax(cmax, (vt[q].y * vt[q].y + vp[q].y * vp[q].y) * hfac);
            cmax = fmax(cmax, vr[q].x * vr[q].x * rfac);
            cmax = fmax(cmax, vr[q].y * vr[q].y * rfac);
        }
        // velocity-only terms
        auto w0 = [&](double a, double b, double c) {   // vr, vt, vp
            return rho * (rad * b * b + rad * c * c + cor * sn * rad * rad * c);
        };
        auto p0 = [&](double a, double b, double c) {
            return -b * b * cot * orad - b * a * orad - b * a * dlnrho - c * c * cot * orad - cor * cs * c;
        };
        auto z0 = [&](double a, double b, double c) { return c * a * orad + cor * (cs * b + sn * a); };
        oW[q] = make_double2(w0(vr[q].x, vt[q].x, vp[q].x), w0(vr[q].y, vt[q].y, vp[q].y));
        oP[q] = make_double2(p0(vr[q].x, vt[q].x, vp[q].x), p0(vr[q].y, vt[q].y, vp[q].y));
        oZ[q] = make_double2(z0(vr[q].x, vt[q].x, vp[q].x), z0(vr[q].y, vt[q].y, vp[q].y));
        oT[q] = make_double2(0.0, 0.0);
    }
#define RA_ACC(dst, expr_x, expr_y)   \
    {                                 \
        dst[q].x += (expr_x);         \
        dst[q].y += (expr_y);         \
    }
    // dvrdr
    row_c2r<ZPT>(P, th, r, A_DVRDR, false, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        RA_ACC(oW, -rho * rad * rad * vr[q].x * x[q].x, -rho * rad * rad * vr[q].y * x[q].y);
        RA_ACC(oP, -vt[q].x * x[q].x, -vt[q].y * x[q].y);
    }
    // dvrdt (sin theta d vr / d theta)
    row_c2r<ZPT>(P, th, r, A_DVRDT, false, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) RA_ACC(oW, -rho * rad * vt[q].x * x[q].x * csc, -rho * rad * vt[q].y * x[q].y * csc);
    // dvrdp
    row_c2r<ZPT>(P, th, r, A_VR, true, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) RA_ACC(oW, -rho * rad * csc * vp[q].x * x[q].x, -rho * rad * csc * vp[q].y * x[q].y);
    // dvtdr
    row_c2r<ZPT>(P, th, r, A_DVTDR, false, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) RA_ACC(oP, vr[q].x * x[q].x * csc, vr[q].y * x[q].y * csc);
    // dvtdp
    row_c2r<ZPT>(P, th, r, A_VT, true, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        const double sx = x[q].x * csc * csc * orad, sy = x[q].y * csc * csc * orad;
        RA_ACC(oP, vp[q].x * sx, vp[q].y * sy);
        RA_ACC(oZ, vt[q].x * sx, vt[q].y * sy);
    }
    // dvpdr
    row_c2r<ZPT>(P, th, r, A_DVPDR, false, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) RA_ACC(oZ, vr[q].x * x[q].x * csc, vr[q].y * x[q].y * csc);
    // dvpdp
    row_c2r<ZPT>(P, th, r, A_VP, true, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        const double sx = x[q].x * csc * csc * orad, sy = x[q].y * csc * csc * orad;
        RA_ACC(oP, -vt[q].x * sx, -vt[q].y * sy);
        RA_ACC(oZ, vp[q].x * sx, vp[q].y * sy);
    }
    // omega_r
    row_c2r<ZPT>(P, th, r, A_OMR, false, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) RA_ACC(oZ, vt[q].x * x[q].x, vt[q].y * x[q].y);
    // dTdr
    row_c2r<ZPT>(P, th, r, A_DTDR, false, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) RA_ACC(oT, -vr[q].x * x[q].x, -vr[q].y * x[q].y);
    // dTdt (sin theta dT/dtheta)
    row_c2r<ZPT>(P, th, r, A_DTDT, false, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) RA_ACC(oT, -x[q].x * csc * vt[q].x * orad, -x[q].y * csc * vt[q].y * orad);
    // dTdp
    row_c2r<ZPT>(P, th, r, A_T, true, bufA, bufB, wr, x);
#pragma unroll
    for (int q = 0; q < ZPT; ++q) RA_ACC(oT, -vp[q].x * x[q].x * csc * orad, -vp[q].y * x[q].y * csc * orad);
#undef RA_ACC
    const double sfac = rho * rad * csc;
#pragma unroll
    for (int q = 0; q < ZPT; ++q) {
        oP[q].x *= sfac; oP[q].y *= sfac;
        oZ[q].x *= sfac; oZ[q].y *= sfac;
    }
    row_r2c<ZPT>(P, th, r, 0, oW, bufA, bufB, wr);
    row_r2c<ZPT>(P, th, r, 1, oP, bufA, bufB, wr);
    row_r2c<ZPT>(P, th, r, 2, oT, bufA, bufB, wr);
    row_r2c<ZPT>(P, th, r, 3, oZ, bufA, bufB, wr);
    // CFL max over the row
    for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_down_sync(0xffffffffu, cmax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = red[0];
        for (int i = 1; i < PHYS_THREADS / 32; ++i) v = fmax(v, red[i]);
        atomicMax(P.cfl, (unsigned long long)__double_as_longlong(v));
    }
}

FFTPlan make_plan(int n) {
    FFTPlan p{};
    p.n = n;
    int m = n;
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
    P.plan = make_plan(c.d.nth);
    const size_t smem = 3 * (size_t)c.d.nth * sizeof(double2);
    const unsigned grid = (unsigned)c.d.nth * c.d.nr;
    const int zpt = (c.d.nth + PHYS_THREADS - 1) / PHYS_THREADS;
    auto go = [&](auto kern) {
        RA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, PHYS_THREADS, smem, c.stream>>>(P);
    };
    switch (zpt) {
        case 1: go(physics_kernel<1>); break;
        case 2: go(physics_kernel<2>); break;
        case 3: go(physics_kernel<3>); break;
        case 4: go(physics_kernel<4>); break;
        case 6: go(physics_kernel<6>); break;
        default: throw ArgError("unsupported n_theta for the physical-space kernel");
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

// ---------------------------------------------------------------------------
// Standalone in-place row FFTs on x(n_phi+2, howmany) (unit-level operator)
// ---------------------------------------------------------------------------
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
        double2* res = fft_run(a, b, plan, wr, +1);
        for (int n = threadIdx.x; n < N; n += blockDim.x) {
            row[2 * n] = res[n].x;
            row[2 * n + 1] = res[n].y;
        }
        __syncthreads();
        if (threadIdx.x == 0) { row[2 * N] = 0.0; row[2 * N + 1] = 0.0; }
    } else {
        for (int n = threadIdx.x; n < N; n += blockDim.x) a[n] = make_double2(row[2 * n], row[2 * n + 1]);
        __syncthreads();
        double2* Z = fft_run(a, b, plan, wr, -1);
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
