// C ABI of the batched per-l solver on its own (no transform context): the
// reference's LU_Decompose_full / LU_Solve_full (Linear_Solve.F90:1028-1036,
// 1088-1110) for any set of equally sized matrices, in two forms:
//   RA_SOLVE_FP64    block substitution with the FP64 factors (k_solve.cu)
//   RA_SOLVE_REFINE  FP32 substitution with FP64 residuals, iterated to FP64
//                    accuracy (iterative refinement), one persistent launch.
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ra_internal.h"

using namespace ra;

struct ra_lu {
    int n = 0, count = 0, device = 0;
    cudaStream_t stream = nullptr;
    double* d_a = nullptr;     // the matrices as given (row-major), kept for the refinement residuals
    double* d_m = nullptr;     // factors in block-substitution form
    float* d_mf = nullptr;     // the same in FP32 (refinement form)
    int* d_perm = nullptr;
    int* d_tiles = nullptr;
    int ntiles = 0, tiles_ncols = 0, tiles_nc = 0;
    int* d_iters = nullptr;
    double* d_b = nullptr;     // right-hand sides / solutions on the device
    double* d_x = nullptr;
    size_t cap_rhs = 0;
    bool factored = false;
    LuWork work;
    std::string err;
};

namespace {

template <class F>
int lu_guarded(ra_lu* lu, F f) {
    try {
        if (lu && lu->stream) RA_CUDA(cudaSetDevice(lu->device));
        f();
        return RA_OK;
    } catch (const ArgError& e) {
        if (lu) lu->err = e.what;
        return RA_ERR_ARG;
    } catch (const SingularError& e) {
        if (lu) lu->err = e.what;
        return RA_ERR_SINGULAR;
    } catch (const NonFiniteError& e) {
        if (lu) lu->err = e.what;
        return RA_ERR_NONFINITE;
    } catch (const CudaError& e) {
        if (lu) lu->err = e.what;
        return e.code == cudaErrorMemoryAllocation ? RA_ERR_NOMEM : RA_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        if (lu) lu->err = "host allocation failed";
        return RA_ERR_NOMEM;
    }
}

void lu_free(ra_lu* lu) {
    void* bufs[] = {lu->d_a, lu->d_m, lu->d_mf, lu->d_perm, lu->d_tiles, lu->d_iters, lu->d_b, lu->d_x};
    for (void* b : bufs)
        if (b) cudaFree(b);
    lu_workspace_free(lu->work);
    if (lu->stream) cudaStreamDestroy(lu->stream);
}

__global__ void lu_transpose_kernel(const double* __restrict__ in, double* __restrict__ out, int n) {
    __shared__ double tile[32][33];
    const size_t b = blockIdx.z;
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, i = i0 + threadIdx.x;
        if (j < n && i < n) tile[r][threadIdx.x] = in[b * n * n + (size_t)j * n + i];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, j = j0 + threadIdx.x;
        if (i < n && j < n) out[b * n * n + (size_t)i * n + j] = tile[threadIdx.x][r];
    }
}

}  // namespace

extern "C" {

int ra_lu_create(ra_lu** out, int n, int count, int device) {
    if (!out) return RA_ERR_ARG;
    *out = nullptr;
    ra_lu* lu = new (std::nothrow) ra_lu();
    if (!lu) return RA_ERR_NOMEM;
    const int rc = lu_guarded(lu, [&] {
        if (n < 2 || (n & 1)) throw ArgError("n must be even and >= 2");
        if (count < 1) throw ArgError("count must be >= 1");
        // the refinement kernel's shared column block (FP64 solution + FP32 residual) bounds n
        if (n > 1152) throw ArgError("n must be <= 1152 (the substitution keeps its columns in shared memory)");
        lu->n = n;
        lu->count = count;
        lu->device = device;
        RA_CUDA(cudaSetDevice(device));
        RA_CUDA(cudaStreamCreateWithFlags(&lu->stream, cudaStreamNonBlocking));
        const size_t nn = (size_t)count * n * n;
        RA_CUDA(cudaMalloc(&lu->d_a, nn * sizeof(double)));
        RA_CUDA(cudaMalloc(&lu->d_m, nn * sizeof(double)));
        RA_CUDA(cudaMalloc(&lu->d_perm, (size_t)count * n * sizeof(int)));
    });
    if (rc != RA_OK) {
        std::string msg = lu->err;
        lu_free(lu);
        *lu = ra_lu();
        lu->err = msg;
    }
    *out = lu;
    return rc;
}

int ra_lu_destroy(ra_lu* lu) {
    if (!lu) return RA_OK;
    if (lu->stream) cudaSetDevice(lu->device);
    lu_free(lu);
    delete lu;
    return RA_OK;
}

int ra_lu_last_error(const ra_lu* lu, char* msg, int len) {
    if (!lu || !msg || len <= 0) return RA_ERR_ARG;
    std::strncpy(msg, lu->err.c_str(), (size_t)len - 1);
    msg[len - 1] = 0;
    return RA_OK;
}

int ra_lu_factor(ra_lu* lu, const double* a, double* ms) {
    if (!lu || !lu->stream) return RA_ERR_STATE;
    if (!a) return RA_ERR_ARG;
    return lu_guarded(lu, [&] {
        const int n = lu->n, count = lu->count;
        const size_t nn = (size_t)count * n * n;
        for (size_t i = 0; i < nn; ++i)
            if (!std::isfinite(a[i])) throw NonFiniteError("matrix entry " + std::to_string(i) + " is not finite");
        lu->factored = false;
        // the caller's matrices are column-major per l (the reference's lhs(n, n)): transpose to row-major
        RA_CUDA(cudaMemcpyAsync(lu->d_m, a, nn * sizeof(double), cudaMemcpyHostToDevice, lu->stream));
        dim3 grid((n + 31) / 32, (n + 31) / 32, count);
        lu_transpose_kernel<<<grid, dim3(32, 8), 0, lu->stream>>>(lu->d_m, lu->d_a, n);
        RA_CUDA(cudaGetLastError());
        RA_CUDA(cudaMemcpyAsync(lu->d_m, lu->d_a, nn * sizeof(double), cudaMemcpyDeviceToDevice, lu->stream));
        cudaEvent_t e0, e1;
        RA_CUDA(cudaEventCreate(&e0));
        RA_CUDA(cudaEventCreate(&e1));
        RA_CUDA(cudaEventRecord(e0, lu->stream));
        const int bad = lu_factor_batch(lu->stream, lu->work, lu->d_m, lu->d_perm, n, count, nullptr, nullptr);
        RA_CUDA(cudaEventRecord(e1, lu->stream));
        RA_CUDA(cudaEventSynchronize(e1));
        float t = 0.f;
        RA_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms) *ms = t;
        if (bad) throw SingularError("singular matrix " + std::to_string(bad - 1) +
                                     " (a zero pivot)");
        if (lu->d_mf) {
            cudaFree(lu->d_mf);
            lu->d_mf = nullptr;
        }
        lu->factored = true;
    });
}

int ra_lu_solve(ra_lu* lu, const double* b, double* x, int ncols, int mode, int* iters, double* ms) {
    if (!lu || !lu->stream) return RA_ERR_STATE;
    if (!b || !x || ncols < 1) return RA_ERR_ARG;
    return lu_guarded(lu, [&] {
        if (!lu->factored) throw ArgError("ra_lu_factor must succeed before ra_lu_solve");
        if (mode != RA_SOLVE_FP64 && mode != RA_SOLVE_REFINE) throw ArgError("unknown solve mode");
        const int n = lu->n, count = lu->count;
        const size_t nb = (size_t)count * ncols * n;
        if (nb > lu->cap_rhs) {
            if (lu->d_b) cudaFree(lu->d_b);
            if (lu->d_x) cudaFree(lu->d_x);
            lu->d_b = lu->d_x = nullptr;
            lu->cap_rhs = 0;
            RA_CUDA(cudaMalloc(&lu->d_b, nb * sizeof(double)));
            RA_CUDA(cudaMalloc(&lu->d_x, nb * sizeof(double)));
            lu->cap_rhs = nb;
        }
        const int nc = mode == RA_SOLVE_FP64 ? lu_nc_for(n) : lu_refine_tile_cols();
        if (lu->tiles_ncols != ncols || lu->tiles_nc != nc) {
            std::vector<int> t;
            lu_append_tiles(t, 0, count, std::vector<int>(count, ncols), nc);
            if (lu->d_tiles) cudaFree(lu->d_tiles);
            if (lu->d_iters) cudaFree(lu->d_iters);
            lu->d_tiles = nullptr;
            lu->d_iters = nullptr;
            lu->tiles_ncols = 0;
            RA_CUDA(cudaMalloc(&lu->d_tiles, t.size() * sizeof(int)));
            RA_CUDA(cudaMemcpy(lu->d_tiles, t.data(), t.size() * sizeof(int), cudaMemcpyHostToDevice));
            lu->ntiles = (int)(t.size() / 4);
            RA_CUDA(cudaMalloc(&lu->d_iters, (size_t)lu->ntiles * sizeof(int)));
            lu->tiles_ncols = ncols;
            lu->tiles_nc = nc;
        }
        if (mode == RA_SOLVE_REFINE && !lu->d_mf) {
            RA_CUDA(cudaMalloc(&lu->d_mf, (size_t)count * n * n * sizeof(float)));
            launch_to_float(lu->stream, lu->d_m, lu->d_mf, (long)count * n * n);
        }
        RA_CUDA(cudaMemcpyAsync(lu->d_b, b, nb * sizeof(double), cudaMemcpyHostToDevice, lu->stream));
        cudaEvent_t e0, e1;
        RA_CUDA(cudaEventCreate(&e0));
        RA_CUDA(cudaEventCreate(&e1));
        RA_CUDA(cudaEventRecord(e0, lu->stream));
        const LuSys s{lu->d_m, lu->d_perm, lu->d_b, lu->d_x, n};
        if (mode == RA_SOLVE_FP64)
            launch_lu_solve(lu->stream, lu->d_tiles, lu->ntiles, s, LU_MODE_FIXED, ncols, nc);
        else
            launch_lu_refine(lu->stream, lu->d_tiles, lu->ntiles, s, lu->d_mf, lu->d_a, ncols, lu->d_iters);
        RA_CUDA(cudaEventRecord(e1, lu->stream));
        RA_CUDA(cudaMemcpyAsync(x, lu->d_x, nb * sizeof(double), cudaMemcpyDeviceToHost, lu->stream));
        RA_CUDA(cudaStreamSynchronize(lu->stream));
        float t = 0.f;
        RA_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms) *ms = t;
        if (iters) {   // per (matrix, column tile), matrices in order (the launch runs them last first)
            const int ntc = lu->ntiles / count;
            std::vector<int> it(lu->ntiles, 1);
            if (mode == RA_SOLVE_REFINE)
                RA_CUDA(cudaMemcpy(it.data(), lu->d_iters, (size_t)lu->ntiles * sizeof(int), cudaMemcpyDeviceToHost));
            for (int l = 0; l < count; ++l)
                for (int ct = 0; ct < ntc; ++ct) iters[l * ntc + ct] = it[(size_t)(count - 1 - l) * ntc + ct];
        }
    });
}

int ra_lu_tiles(const ra_lu* lu, int ncols, int mode) {
    if (!lu || lu->n == 0 || ncols < 1) return RA_ERR_ARG;
    const int nc = mode == RA_SOLVE_REFINE ? lu_refine_tile_cols() : lu_nc_for(lu->n);
    return lu->count * ((ncols + nc - 1) / nc);
}

}  // extern "C"
