// FP64 kernels of the defect-correction (mixed-precision) Jacobi solver for lap(u) = f.
//
// No counterpart kernel in the reference: pyheat3d solves the Poisson problem by plain Jacobi
// with an additive source (src/pyheat3d/validation.py:135-147, b = -h^2 f / (2d),
// src/pyheat3d/problem.py:15-16) in one precision. Here the outer loop keeps the solution and
// the residual in FP64 on the GPU while the inner Jacobi sweeps on the correction run with
// 16-bit storage and fp32 arithmetic (the stencil kernels of this library, with a source):
//
//   r = f - A u,        A u = (S(u) - 2d u) / h^2      (FP64, interior; r = 0 on the boundary)
//   b = -h^2 (r / s) / (2d)   (fp32 source of the scaled correction equation A e = r / s)
//   e <- Jacobi sweeps (16-bit storage, fp32 math, e = 0 on the boundary)
//   u <- u + s e        (FP64)
// The scale s is a power of two near the residual's RMS, chosen by the host, so the correction
// stays inside the 16-bit exponent range (fp16 would otherwise flush it to zero) and scaling is
// exact.
//
// Every FP64 operation is an explicitly rounded __dadd_rn / __dmul_rn in a fixed order, so the
// NumPy oracle reproduces residual and update bit for bit. Reductions are two-pass and
// deterministic: a fixed grid of blocks writes one partial sum each into caller-provided
// scratch, one block sums the partials in a fixed tree order.
#include "ph3_common.cuh"
#include "ph3_internal.h"

namespace ph3 {

namespace {

constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] = __dadd_rn(sh[t], sh[t + s]);
        __syncthreads();
    }
    return sh[0];
}

template <int DIMS>
__global__ void __launch_bounds__(kRedThreads)
dc_residual_kernel(const double* __restrict__ u, const double* __restrict__ f, int nz, int ny,
                   int nx, double inv_h2, double bscale, float* __restrict__ b,
                   double* __restrict__ partial) {
    __shared__ double sh[kRedThreads];
    const int64_t P = int64_t(nx) * ny;
    const int64_t n = P * (DIMS == 3 ? nz : 1);
    double acc = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int x = int(i % nx);
        const int y = int((i / nx) % ny);
        const int z = DIMS == 3 ? int(i / P) : 0;
        const bool interior = x > 0 && x < nx - 1 && y > 0 && y < ny - 1 &&
                              (DIMS == 2 || (z > 0 && z < nz - 1));
        double r = 0.0;
        if (interior) {
            double s = __dadd_rn(__dadd_rn(u[i - 1], u[i + 1]), __dadd_rn(u[i - nx], u[i + nx]));
            if (DIMS == 3) s = __dadd_rn(s, __dadd_rn(u[i - P], u[i + P]));
            const double au = __dmul_rn(__dadd_rn(s, -__dmul_rn(2.0 * DIMS, u[i])), inv_h2);
            r = __dadd_rn(f[i], -au);
        }
        if (b != nullptr) b[i] = __double2float_rn(__dmul_rn(bscale, r));
        acc = __fma_rn(r, r, acc);
    }
    const double tot = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kRedThreads)
dot_kernel(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
           double* __restrict__ partial) {
    __shared__ double sh[kRedThreads];
    double acc = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        acc = __fma_rn(x[i], y[i], acc);
    const double tot = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kRedThreads)
finish_kernel(const double* __restrict__ partial, int nparts, double* __restrict__ out) {
    __shared__ double sh[kRedThreads];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc = __dadd_rn(acc, partial[i]);
    const double tot = block_sum(acc, sh);
    if (threadIdx.x == 0) *out = tot;
}

template <typename T>
__global__ void correct_kernel(double* __restrict__ u, const T* __restrict__ e, double scale,
                               int64_t n) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        u[i] = __dadd_rn(u[i], __dmul_rn(scale, double(to_f(e[i]))));
}

}  // namespace

cudaError_t launch_dc_residual(int dims, int nz, int ny, int nx, const double* u, const double* f,
                               double h, double b_scale, float* b, double* out, double* scratch,
                               cudaStream_t stream) {
    const double inv_h2 = 1.0 / (h * h);
    const double bscale = (-(h * h) / (2.0 * dims)) * b_scale;
    if (dims == 3)
        dc_residual_kernel<3><<<kReductionParts, kRedThreads, 0, stream>>>(
            u, f, nz, ny, nx, inv_h2, bscale, b, scratch);
    else
        dc_residual_kernel<2><<<kReductionParts, kRedThreads, 0, stream>>>(
            u, f, 1, ny, nx, inv_h2, bscale, b, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    finish_kernel<<<1, kRedThreads, 0, stream>>>(scratch, kReductionParts, out);
    return cudaGetLastError();
}

cudaError_t launch_dot(const double* x, const double* y, int64_t n, double* out, double* scratch,
                       cudaStream_t stream) {
    dot_kernel<<<kReductionParts, kRedThreads, 0, stream>>>(x, y, n, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    finish_kernel<<<1, kRedThreads, 0, stream>>>(scratch, kReductionParts, out);
    return cudaGetLastError();
}

cudaError_t launch_dc_correct(double* u, const void* e, int storage, double scale, int64_t n,
                              cudaStream_t stream) {
    const int blocks = 4 * (sm_count() > 0 ? sm_count() : 148);
    switch (storage) {
        case kF32:
            correct_kernel<<<blocks, 256, 0, stream>>>(u, static_cast<const float*>(e), scale, n);
            break;
        case kF16:
            correct_kernel<<<blocks, 256, 0, stream>>>(u, static_cast<const __half*>(e), scale, n);
            break;
        case kBF16:
            correct_kernel<<<blocks, 256, 0, stream>>>(u, static_cast<const __nv_bfloat16*>(e),
                                                      scale, n);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace ph3
