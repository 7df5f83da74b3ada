// C ABI of the pyheat3d B200 stencil backend: argument checking, dispatch, error reporting.
// Declarations and conventions: include/ph3b200.h.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/ph3b200.h"
#include "ph3_internal.h"

namespace ph3 {

// Per-device status word written by kernels whose bounded waits expire.
__device__ int g_status_word;

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(PH3_ECUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

constexpr int kMaxDev = 64;

int* status_ptr() {
    static int* ptrs[kMaxDev] = {nullptr};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (ptrs[dev] == nullptr) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_status_word) == cudaSuccess) ptrs[dev] = static_cast<int*>(p);
    }
    return ptrs[dev];
}

int check_grid(int dims, int nz, int ny, int nx, int storage, int bc) {
    if (dims != 2 && dims != 3) return fail(PH3_EINVAL, "dims must be 2 or 3, got %d", dims);
    if (dims == 2 && nz != 1) return fail(PH3_EINVAL, "2D grids take nz == 1, got %d", nz);
    // base.py:45-46: every axis needs at least 3 points
    if (ny < 3 || nx < 3 || (dims == 3 && nz < 3))
        return fail(PH3_EINVAL, "every axis needs at least 3 points, got (%d, %d, %d)", nz, ny, nx);
    if (storage < PH3_FLOAT32 || storage > PH3_BFLOAT16)
        return fail(PH3_EINVAL, "storage must be 0 (fp32), 1 (fp16) or 2 (bf16), got %d", storage);
    if (bc != PH3_DIRICHLET && bc != PH3_PERIODIC)
        return fail(PH3_EINVAL, "bc must be 0 (dirichlet) or 1 (periodic), got %d", bc);
    const long long cells = 1LL * nz * ny * nx;
    if (cells > (1LL << 40)) return fail(PH3_EUNSUPPORTED, "grid of %lld cells too large", cells);
    return PH3_OK;
}

int check_ptrs(const void* u, const void* out, const float* src) {
    if (u == nullptr || out == nullptr) return fail(PH3_EINVAL, "u and out must be non-null");
    if (u == out) return fail(PH3_EINVAL, "u and out must be distinct buffers (ping-pong)");
    if (src != nullptr && (static_cast<const void*>(src) == out))
        return fail(PH3_EINVAL, "src must not alias out");
    return PH3_OK;
}

Launch make(int dims, int nz, int ny, int nx, int storage, int bc, float c0, float c1,
            const void* u, void* out, const float* src, int k, int chunk, void* stream) {
    Launch L;
    L.u = u; L.out = out; L.src = src;
    L.dims = dims; L.nz = dims == 2 ? 1 : nz; L.ny = ny; L.nx = nx;
    L.periodic = bc == PH3_PERIODIC; L.storage = storage;
    L.c0 = c0; L.c1 = c1; L.k = k; L.chunk = chunk;
    L.stream = static_cast<cudaStream_t>(stream);
    L.err = status_ptr();
    return L;
}

int finish(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return cuda_fail(e, what);
    g_err[0] = '\0';
    return PH3_OK;
}

cudaError_t launch_single(const Launch& L, int variant) {
    if (variant == PH3_VARIANT_NAIVE) return launch_naive(L);
    if (L.dims == 3 && zmarch_tma_supported(L)) return launch_zmarch_tma(L);
    return launch_march_k1(L);
}

}  // namespace

int sm_count() {
    static int counts[kMaxDev] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return 0;
    if (counts[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        counts[dev] = n;
    }
    return counts[dev];
}

}  // namespace ph3

using namespace ph3;

extern "C" {

int ph3_version(void) { return 1 * 10000 + 0 * 100 + 0; }

const char* ph3_last_error(void) { return g_err; }

int ph3_sm_count(void) {
    const int n = sm_count();
    if (n == 0) fail(PH3_ECUDA, "no CUDA device");
    return n;
}

int ph3_device_status(int* code, int clear) {
    if (code == nullptr) return fail(PH3_EINVAL, "code must be non-null");
    int* p = status_ptr();
    if (p == nullptr) return fail(PH3_ECUDA, "no CUDA device / status word unavailable");
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
    e = cudaMemcpy(code, p, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "read status word");
    if (clear) {
        e = cudaMemset(p, 0, sizeof(int));
        if (e != cudaSuccess) return cuda_fail(e, "clear status word");
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
    }
    return PH3_OK;
}

int ph3_naive2d(const void* u, void* out, const float* src, int ny, int nx, float c0, float c1,
                int storage, int bc, void* stream) {
    int rc = check_grid(2, 1, ny, nx, storage, bc);
    if (rc == PH3_OK) rc = check_ptrs(u, out, src);
    if (rc != PH3_OK) return rc;
    return finish(launch_naive(make(2, 1, ny, nx, storage, bc, c0, c1, u, out, src, 1, 0, stream)),
                  "naive2d launch");
}

int ph3_naive3d(const void* u, void* out, const float* src, int nz, int ny, int nx, float c0,
                float c1, int storage, int bc, void* stream) {
    int rc = check_grid(3, nz, ny, nx, storage, bc);
    if (rc == PH3_OK) rc = check_ptrs(u, out, src);
    if (rc != PH3_OK) return rc;
    return finish(
        launch_naive(make(3, nz, ny, nx, storage, bc, c0, c1, u, out, src, 1, 0, stream)),
        "naive3d launch");
}

int ph3_zmarch3d(const void* u, void* out, const float* src, int nz, int ny, int nx, float c0,
                 float c1, int storage, int bc, int chunk, void* stream) {
    int rc = check_grid(3, nz, ny, nx, storage, bc);
    if (rc == PH3_OK) rc = check_ptrs(u, out, src);
    if (rc != PH3_OK) return rc;
    return finish(launch_single(make(3, nz, ny, nx, storage, bc, c0, c1, u, out, src, 1, chunk,
                                     stream),
                                PH3_VARIANT_MARCH),
                  "zmarch3d launch");
}

int ph3_ymarch2d(const void* u, void* out, const float* src, int ny, int nx, float c0, float c1,
                 int storage, int bc, int chunk, void* stream) {
    int rc = check_grid(2, 1, ny, nx, storage, bc);
    if (rc == PH3_OK) rc = check_ptrs(u, out, src);
    if (rc != PH3_OK) return rc;
    return finish(
        launch_march_k1(make(2, 1, ny, nx, storage, bc, c0, c1, u, out, src, 1, chunk, stream)),
        "ymarch2d launch");
}

static int tb_common(int dims, const void* u, void* out, const float* src, int nz, int ny, int nx,
                     int k, float c0, float c1, int storage, int bc, int chunk, void* stream) {
    int rc = check_grid(dims, nz, ny, nx, storage, bc);
    if (rc == PH3_OK) rc = check_ptrs(u, out, src);
    if (rc != PH3_OK) return rc;
    if (k != 2 && k != 3 && k != 4 && k != 8)
        return fail(PH3_EINVAL, "tb k must be one of 2, 3, 4, 8, got %d", k);
    return finish(
        launch_tb(make(dims, nz, ny, nx, storage, bc, c0, c1, u, out, src, k, chunk, stream)),
        dims == 3 ? "tb3d launch" : "tb2d launch");
}

int ph3_tb3d(const void* u, void* out, const float* src, int nz, int ny, int nx, int k, float c0,
             float c1, int storage, int bc, int chunk, void* stream) {
    return tb_common(3, u, out, src, nz, ny, nx, k, c0, c1, storage, bc, chunk, stream);
}

int ph3_tb2d(const void* u, void* out, const float* src, int ny, int nx, int k, float c0,
             float c1, int storage, int bc, int chunk, void* stream) {
    return tb_common(2, u, out, src, 1, ny, nx, k, c0, c1, storage, bc, chunk, stream);
}

int ph3_advance(int dims, int nz, int ny, int nx, int storage, int bc, float c0, float c1,
                int variant, int k, void* a, void* b, const float* src, int64_t nsteps,
                void* stream, int* in_b) {
    int rc = check_grid(dims, nz, ny, nx, storage, bc);
    if (rc == PH3_OK) rc = check_ptrs(a, b, src);
    if (rc != PH3_OK) return rc;
    if (in_b == nullptr) return fail(PH3_EINVAL, "in_b must be non-null");
    if (nsteps < 0) return fail(PH3_EINVAL, "nsteps must be >= 0");
    if (variant < PH3_VARIANT_NAIVE || variant > PH3_VARIANT_TB)
        return fail(PH3_EINVAL, "unknown variant %d", variant);
    if (variant == PH3_VARIANT_TB) {
        if (k != 1 && k != 2 && k != 3 && k != 4 && k != 8)
            return fail(PH3_EINVAL, "tb k must be one of 1, 2, 3, 4, 8, got %d", k);
    } else if (k != 1) {
        return fail(PH3_EINVAL, "k must be 1 for single-step variants, got %d", k);
    }
    Launch L = make(dims, nz, ny, nx, storage, bc, c0, c1, a, b, src, k, 0, stream);
    const int single = variant == PH3_VARIANT_NAIVE ? PH3_VARIANT_NAIVE : PH3_VARIANT_MARCH;
    const void* cur = a;
    void* nxt = b;
    int swaps = 0;
    const int64_t passes = k > 1 ? nsteps / k : 0;
    const int64_t rest = k > 1 ? nsteps % k : nsteps;
    for (int64_t i = 0; i < passes; ++i) {
        L.u = cur; L.out = nxt;
        cudaError_t e = launch_tb(L);
        if (e != cudaSuccess) return cuda_fail(e, "tb launch");
        void* t = const_cast<void*>(cur); cur = nxt; nxt = t; swaps ^= 1;
    }
    L.k = 1;
    for (int64_t i = 0; i < rest; ++i) {
        L.u = cur; L.out = nxt;
        cudaError_t e = launch_single(L, single);
        if (e != cudaSuccess) return cuda_fail(e, "single-step launch");
        void* t = const_cast<void*>(cur); cur = nxt; nxt = t; swaps ^= 1;
    }
    *in_b = swaps;
    g_err[0] = '\0';
    return PH3_OK;
}

}  // extern "C"
