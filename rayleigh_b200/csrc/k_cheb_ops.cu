// Unit-level Chebyshev operators on columns f(n_r, ncols) (one thread per column):
//   mode 0  To_Spectral4D          (Chebyshev_Polynomials.F90:375-448), parity fold, alpha = 2/N
//   mode 1  From_Spectral4D        (:450-558), all N coefficients, minus c_0/2
//   mode 2  Cheby_Deriv_Buffer_4D  (:560-644), backward recursion, times scaling^order
// The time step itself uses the fused synthesis in k_spectral.cu.
#include "ra_internal.h"

namespace ra {

__global__ void cheb_columns_kernel(const double* __restrict__ D0, const double* __restrict__ in,
                                    double* __restrict__ out, long ncols, int n, int mode, int order,
                                    double scaling) {
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncols) return;
    const double* x = in + col * n;
    double* y = out + col * n;
    if (mode == 0) {
        const double alpha = 2.0 / n;
        const int nx = (n + 1) / 2;
        for (int k = 0; k < n; ++k) {
            double s = 0.0;
            for (int i = 0; i < nx; ++i) {
                const double fe = (k & 1) ? (x[i] - x[n - 1 - i]) : (x[i] + x[n - 1 - i]);
                const double t = D0[(long)i * n + k] + (k == 0 ? 0.5 : 0.0);
                s += t * fe;
            }
            y[k] = alpha * s;
        }
    } else if (mode == 1) {
        for (int r = 0; r < n; ++r) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += D0[(long)r * n + k] * x[k];
            y[r] = s;
        }
    } else {
        for (int k = 0; k < n; ++k) y[k] = x[k];
        for (int o = 0; o < order; ++o) {
            // y holds the previous order; build the next in place from the top down
            double d2 = 0.0, d1 = 0.0;   // d(i+2), d(i+1)
            double cprev = y[n - 1];
            y[n - 1] = 0.0;
            d1 = 0.0;
            double nxt = 2.0 * (n - 1) * cprev;   // d(n-2)
            double cur_c = y[n - 2];
            y[n - 2] = nxt;
            d2 = d1;
            d1 = nxt;
            for (int i = n - 3; i >= 0; --i) {
                const double ci1 = cur_c;        // c(i+1) of the previous order
                cur_c = y[i];
                const double di = d2 + 2.0 * (i + 1) * ci1;
                y[i] = di;
                d2 = d1;
                d1 = di;
            }
        }
        double s = 1.0;
        for (int o = 0; o < order; ++o) s *= scaling;
        for (int k = 0; k < n; ++k) y[k] *= s;
    }
}

void launch_cheb_columns(Ctx& c, const double* d_in, double* d_out, long ncols, int mode, int order) {
    cheb_columns_kernel<<<(unsigned)((ncols + 127) / 128), 128, 0, c.stream>>>(c.d_D, d_in, d_out, ncols, c.d.nr,
                                                                               mode, order, c.deriv_scaling);
    RA_CUDA(cudaGetLastError());
    ++c.launches;
}

}  // namespace ra
