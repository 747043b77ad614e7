// Device-resident spherical-harmonic transforms of an arbitrary batch of fields
// (ra_transform_dev): the Legendre transform of the step (StP_4d_dgp2 /
// PtS_4d_dgpv3, Legendre_Transforms.F90:968-1175) in either precision form, the
// relayout between its E/O (theta, pi - theta) blocks and phi rows, and the phi
// FFTs (FFT_To_Physical / FFT_To_Spectral, Fourier_Transform.F90:100-183) on
// rows of n_phi + 2 doubles.  The step fuses the last two into its
// physical-space kernel; this path serves batches of arbitrary fields (the
// transform sweep) with the operands in device memory.
#include <cmath>

#include "ra_internal.h"

namespace ra {

constexpr int TT = 32;   // transpose tile (complex entries)

// p2[theta_h][m][par][fr] (E, O; fr = (field, r) complex columns) -> rows[theta][fr][k],
// k = 0 .. n_phi/2: X_m = E + O on the south row theta_h, E - O on the north row
// n_theta - 1 - theta_h (Legendre_Transforms.F90:1030-1064), zero for m >= L.
__global__ void p2_to_rows_kernel(const double2* __restrict__ p2, double2* __restrict__ rows, int L, int nth,
                                  int nfr, int nk) {
    __shared__ double2 tile[TT][TT + 1];
    const int th = blockIdx.z, nth2 = nth / 2;
    const bool north = th >= nth2;
    const int thh = north ? nth - 1 - th : th;
    const int k0 = blockIdx.y * TT, c0 = blockIdx.x * TT;
    for (int j = threadIdx.y; j < TT; j += blockDim.y) {
        const int k = k0 + j, fr = c0 + threadIdx.x;
        double2 v = make_double2(0.0, 0.0);
        if (k < L && fr < nfr) {
            const double2 e = p2[((size_t)(thh * L + k) * 2 + 0) * nfr + fr];
            const double2 o = p2[((size_t)(thh * L + k) * 2 + 1) * nfr + fr];
            v = north ? make_double2(e.x - o.x, e.y - o.y) : make_double2(e.x + o.x, e.y + o.y);
        }
        tile[j][threadIdx.x] = v;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < TT; j += blockDim.y) {
        const int fr = c0 + j, k = k0 + threadIdx.x;
        if (fr < nfr && k < nk) rows[((size_t)th * nfr + fr) * nk + k] = tile[threadIdx.x][j];
    }
}

// rows[theta][fr][k] (the r2c output) -> the folded p2[m][par][theta_h][fr] of PtS_4d_dgpv3
// (Legendre_Transforms.F90:1109-1122): even = X(theta_h) + X(n_theta - 1 - theta_h), odd the
// difference, m < L.
__global__ void rows_to_p2_kernel(const double2* __restrict__ rows, double2* __restrict__ p2, int L, int nth,
                                  int nfr, int nk) {
    __shared__ double2 te[TT][TT + 1], to[TT][TT + 1];
    const int thh = blockIdx.z, nth2 = nth / 2;
    const int k0 = blockIdx.y * TT, c0 = blockIdx.x * TT;
    for (int j = threadIdx.y; j < TT; j += blockDim.y) {
        const int fr = c0 + j, k = k0 + threadIdx.x;
        double2 a = make_double2(0.0, 0.0), b = a;
        if (fr < nfr && k < nk) {
            a = rows[((size_t)thh * nfr + fr) * nk + k];
            b = rows[((size_t)(nth - 1 - thh) * nfr + fr) * nk + k];
        }
        te[threadIdx.x][j] = make_double2(a.x + b.x, a.y + b.y);
        to[threadIdx.x][j] = make_double2(a.x - b.x, a.y - b.y);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < TT; j += blockDim.y) {
        const int k = k0 + j, fr = c0 + threadIdx.x;
        if (k < L && fr < nfr) {
            p2[(((size_t)k * 2 + 0) * nth2 + thh) * nfr + fr] = te[j][threadIdx.x];
            p2[(((size_t)k * 2 + 1) * nth2 + thh) * nfr + fr] = to[j][threadIdx.x];
        }
    }
}

static void launch_relayout(Ctx& c, bool to_rows, double* p2, double* rows, int nfr) {
    const int L = c.d.L, nth = c.d.nth, nk = c.d.nphi / 2 + 1;
    const dim3 blk(TT, 8);
    if (to_rows) {
        const dim3 grid((nfr + TT - 1) / TT, (nk + TT - 1) / TT, nth);
        p2_to_rows_kernel<<<grid, blk, 0, c.stream>>>(reinterpret_cast<const double2*>(p2),
                                                      reinterpret_cast<double2*>(rows), L, nth, nfr, nk);
    } else {
        const dim3 grid((nfr + TT - 1) / TT, (L + TT - 1) / TT, nth / 2);
        rows_to_p2_kernel<<<grid, blk, 0, c.stream>>>(reinterpret_cast<const double2*>(rows),
                                                      reinterpret_cast<double2*>(p2), L, nth, nfr, nk);
    }
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

void transform_dev(Ctx& c, int direction, int precision, double* spec, double* grid, double* work, int nfr,
                   double* stage_ms) {
    const int ncol = 2 * nfr;
    const long rows = (long)c.d.nth * nfr;
    cudaEvent_t ev[4];
    for (auto& e : ev) RA_CUDA(cudaEventCreate(&e));
    auto product = [&] {
        if (direction == 0) {
            if (precision == RA_PREC_MIXED)
                launch_lt_unit_mixed(c, 1, spec, work, ncol);
            else
                launch_lt_inverse(c, spec, work, ncol);
        } else {
            if (precision == RA_PREC_MIXED)
                launch_lt_unit_mixed(c, 0, work, spec, ncol);
            else
                launch_lt_forward(c, work, spec, ncol);
        }
    };
    // event order: [0] start, [1] after the first stage, [2] after the second, [3] end
    if (direction == 0) {   // spectral -> physical: StP, relayout, c2r
        RA_CUDA(cudaEventRecord(ev[0], c.stream));
        product();
        RA_CUDA(cudaEventRecord(ev[1], c.stream));
        launch_relayout(c, true, work, grid, nfr);
        RA_CUDA(cudaEventRecord(ev[2], c.stream));
        launch_fft_rows(c, grid, rows, 1);
        RA_CUDA(cudaEventRecord(ev[3], c.stream));
    } else {                // physical -> spectral: r2c, fold, PtS
        RA_CUDA(cudaEventRecord(ev[0], c.stream));
        launch_fft_rows(c, grid, rows, 0);
        RA_CUDA(cudaEventRecord(ev[1], c.stream));
        launch_relayout(c, false, work, grid, nfr);
        RA_CUDA(cudaEventRecord(ev[2], c.stream));
        product();
        RA_CUDA(cudaEventRecord(ev[3], c.stream));
    }
    RA_CUDA(cudaStreamSynchronize(c.stream));
    if (stage_ms) {
        float t[3];
        for (int i = 0; i < 3; ++i) RA_CUDA(cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]));
        // [0] Legendre product (with the digit split in the mixed form), [1] relayout, [2] FFT
        stage_ms[0] = direction == 0 ? t[0] : t[2];
        stage_ms[1] = t[1];
        stage_ms[2] = direction == 0 ? t[2] : t[0];
    }
    for (auto& e : ev) cudaEventDestroy(e);
}

}  // namespace ra
