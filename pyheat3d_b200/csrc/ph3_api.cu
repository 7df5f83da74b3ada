// C ABI of the pyheat3d B200 stencil backend: argument checking, dispatch, error reporting.
// Declarations and conventions: include/ph3b200.h.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/ph3b200.h"
#include "ph3_common.cuh"
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

// ------------------------------------------------------------------------ tuning table
constexpr int kMaxK = 8;
std::atomic<int> g_tune_cfg[kNumFamilies][2][3][kMaxK + 1];
std::atomic<int> g_tune_chunk[kNumFamilies][2][3][kMaxK + 1];
std::once_flag g_tune_once;

void tune_init() {
    std::call_once(g_tune_once, [] {
        for (int f = 0; f < kNumFamilies; ++f)
            for (int d = 0; d < 2; ++d)
                for (int s = 0; s < 3; ++s)
                    for (int k = 0; k <= kMaxK; ++k) {
                        g_tune_cfg[f][d][s][k].store(-1);
                        g_tune_chunk[f][d][s][k].store(0);
                    }
    });
}

int family_count(int family, int dims, int k, const char** names, int max) {
    switch (family) {
        case kFamZmarch: return dims == 3 && k == 1 ? zmarch_configs(names, max) : 0;
        case kFamMarch: return k == 1 ? march_configs(dims, names, max) : 0;
        case kFamTb: return tb_configs(dims, k, names, max);
        case kFamBatch: return k == 1 ? batch_configs(names, max) : 0;
        default: return 0;
    }
}

// Fill cfg / chunk of a launch from the table (an explicit chunk argument wins).
void apply_tune(Launch& L, int family) {
    tune_init();
    const int d = L.dims - 2, s = L.storage, k = L.k < 0 || L.k > kMaxK ? 0 : L.k;
    L.cfg = g_tune_cfg[family][d][s][k].load(std::memory_order_relaxed);
    if (L.chunk <= 0) L.chunk = g_tune_chunk[family][d][s][k].load(std::memory_order_relaxed);
}

Launch make(int dims, int nz, int ny, int nx, int storage, int bc, float c0, float c1,
            const void* u, void* out, const float* src, int k, int chunk, void* stream) {
    Launch L;
    L.u = u; L.out = out; L.src = src;
    L.dims = dims; L.nz = dims == 2 ? 1 : nz; L.ny = ny; L.nx = nx;
    L.periodic = bc == PH3_PERIODIC; L.storage = storage;
    L.c0 = c0; L.c1 = c1; L.k = k; L.chunk = chunk; L.cfg = -1;
    L.zb = 0; L.ze = 0;
    L.stream = static_cast<cudaStream_t>(stream);
    L.err = status_ptr();
    L.geo = nullptr;
    return L;
}

int finish(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return cuda_fail(e, what);
    g_err[0] = '\0';
    return PH3_OK;
}

cudaError_t launch_single(Launch L, int variant) {
    if (variant == PH3_VARIANT_NAIVE) return launch_naive(L);
    if (L.dims == 3 && zmarch_tma_supported(L)) {
        apply_tune(L, kFamZmarch);
        return launch_zmarch_tma(L);
    }
    apply_tune(L, kFamMarch);
    return launch_march_k1(L);
}

cudaError_t launch_tb_tuned(Launch L) {
    apply_tune(L, kFamTb);
    return launch_tb(L);
}

}  // namespace

int sm_count() {
    // concurrent first calls may both query the device; they store the same value atomically
    static std::atomic<int> counts[kMaxDev];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return 0;
    int n = counts[dev].load(std::memory_order_acquire);
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        counts[dev].store(n, std::memory_order_release);
    }
    return n;
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

namespace ph3 {
__global__ void wait_flag_kernel(const int* flag, int target, uint32_t limit, int* err) {
    if (threadIdx.x == 0) wait_flag_geq(flag, target, limit, err, nullptr);
}
}  // namespace ph3

int ph3_wait_flag(const int* flag, int target, unsigned int spin_limit, void* stream) {
    if (flag == nullptr) return fail(PH3_EINVAL, "flag must be non-null");
    if (reinterpret_cast<uintptr_t>(flag) % alignof(int) != 0)
        return fail(PH3_EINVAL, "flag must be 4-byte aligned");
    if (spin_limit == 0 || spin_limit > kSpinLimit)
        return fail(PH3_EINVAL, "spin_limit must be in [1, %u], got %u", kSpinLimit, spin_limit);
    int* err = status_ptr();
    if (err == nullptr) return fail(PH3_ECUDA, "no CUDA device / status word unavailable");
    ph3::wait_flag_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(flag, target, spin_limit,
                                                                       err);
    return finish(cudaGetLastError(), "wait_flag launch");
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

int ph3_zmarch3d_planes(const void* u, void* out, const float* src, int nz, int ny, int nx,
                        int z0, int z1, float c0, float c1, int storage, int bc, int chunk,
                        void* stream) {
    int rc = check_grid(3, nz, ny, nx, storage, bc);
    if (rc == PH3_OK) rc = check_ptrs(u, out, src);
    if (rc != PH3_OK) return rc;
    if (z0 < 1 || z1 > nz - 1 || z0 > z1)
        return fail(PH3_EINVAL, "planes [%d, %d) must satisfy 1 <= z0 <= z1 <= nz-1 = %d", z0, z1,
                    nz - 1);
    if (z0 == z1) return finish(cudaSuccess, "");
    Launch L = make(3, nz, ny, nx, storage, bc, c0, c1, u, out, src, 1, chunk, stream);
    L.zb = z0;
    L.ze = z1;
    return finish(launch_single(L, PH3_VARIANT_MARCH), "zmarch3d_planes launch");
}

int ph3_ymarch2d(const void* u, void* out, const float* src, int ny, int nx, float c0, float c1,
                 int storage, int bc, int chunk, void* stream) {
    int rc = check_grid(2, 1, ny, nx, storage, bc);
    if (rc == PH3_OK) rc = check_ptrs(u, out, src);
    if (rc != PH3_OK) return rc;
    return finish(
        launch_single(make(2, 1, ny, nx, storage, bc, c0, c1, u, out, src, 1, chunk, stream),
                      PH3_VARIANT_MARCH),
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
        launch_tb_tuned(make(dims, nz, ny, nx, storage, bc, c0, c1, u, out, src, k, chunk, stream)),
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

int ph3_tb_tile(int dims, int nz, int ny, int nx, int storage, int bc, int k, int* tx, int* ty,
                int* chunk) {
    int rc = check_grid(dims, dims == 2 ? 1 : nz, ny, nx, storage, bc);
    if (rc != PH3_OK) return rc;
    if (k != 2 && k != 3 && k != 4 && k != 8)
        return fail(PH3_EINVAL, "tb k must be one of 2, 3, 4, 8, got %d", k);
    if (tx == nullptr || ty == nullptr || chunk == nullptr)
        return fail(PH3_EINVAL, "tx, ty and chunk must be non-null");
    int geo[3] = {0, 0, 0};
    Launch L = make(dims, nz, ny, nx, storage, bc, 0.f, 0.f, nullptr, nullptr, nullptr, k, 0,
                    nullptr);
    L.geo = geo;
    rc = finish(launch_tb_tuned(L), "tb geometry");
    if (rc != PH3_OK) return rc;
    *tx = geo[0];
    *ty = geo[1];
    *chunk = geo[2];
    return PH3_OK;
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
        cudaError_t e = launch_tb_tuned(L);
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

int64_t ph3_reduction_scratch_len(void) { return kReductionParts; }

int ph3_dc_residual(int dims, int nz, int ny, int nx, const double* u, const double* f, double h,
                    double b_scale, float* b, double* rnorm2, double* scratch,
                    int64_t scratch_len, void* stream) {
    int rc = check_grid(dims, dims == 2 ? 1 : nz, ny, nx, PH3_FLOAT32, PH3_DIRICHLET);
    if (rc != PH3_OK) return rc;
    if (u == nullptr || f == nullptr || rnorm2 == nullptr || scratch == nullptr)
        return fail(PH3_EINVAL, "u, f, rnorm2 and scratch must be non-null");
    if (scratch_len < kReductionParts)
        return fail(PH3_EINVAL, "scratch needs %d doubles, got %lld", kReductionParts,
                    (long long)scratch_len);
    if (!(h > 0.0)) return fail(PH3_EINVAL, "h must be > 0");
    return finish(launch_dc_residual(dims, nz, ny, nx, u, f, h, b_scale, b, rnorm2, scratch,
                                     static_cast<cudaStream_t>(stream)),
                  "dc_residual launch");
}

int ph3_dot_f64(const double* x, const double* y, int64_t n, double* out, double* scratch,
                int64_t scratch_len, void* stream) {
    if (x == nullptr || y == nullptr || out == nullptr || scratch == nullptr)
        return fail(PH3_EINVAL, "x, y, out and scratch must be non-null");
    if (n < 0) return fail(PH3_EINVAL, "n must be >= 0");
    if (scratch_len < kReductionParts)
        return fail(PH3_EINVAL, "scratch needs %d doubles, got %lld", kReductionParts,
                    (long long)scratch_len);
    return finish(launch_dot(x, y, n, out, scratch, static_cast<cudaStream_t>(stream)),
                  "dot launch");
}

int ph3_dc_correct(double* u, const void* e, int storage, double e_scale, int64_t n,
                   void* stream) {
    if (u == nullptr || e == nullptr) return fail(PH3_EINVAL, "u and e must be non-null");
    if (storage < PH3_FLOAT32 || storage > PH3_BFLOAT16)
        return fail(PH3_EINVAL, "storage must be 0, 1 or 2, got %d", storage);
    if (n < 0) return fail(PH3_EINVAL, "n must be >= 0");
    return finish(launch_dc_correct(u, e, storage, e_scale, n, static_cast<cudaStream_t>(stream)),
                  "dc_correct launch");
}

int64_t ph3_batch_workspace_bytes(const ph3_problem* problems, int n) {
    if (n < 0 || (n > 0 && problems == nullptr)) {
        fail(PH3_EINVAL, "problems must be non-null and n >= 0");
        return -1;
    }
    return batch_workspace_bytes(problems, n);
}

int ph3_batch_prepare(const ph3_problem* problems, int n, void* ws, int64_t ws_bytes,
                      void* stream) {
    if (n < 0 || (n > 0 && problems == nullptr) || ws == nullptr)
        return fail(PH3_EINVAL, "problems and ws must be non-null and n >= 0");
    for (int i = 0; i < n; ++i) {
        const ph3_problem& p = problems[i];
        int rc = check_grid(p.dims, p.dims == 2 ? 1 : p.nz, p.ny, p.nx, p.storage, p.bc);
        if (rc == PH3_OK) rc = check_ptrs(p.a, p.b, p.src);
        if (rc != PH3_OK) {
            char msg[512];
            snprintf(msg, sizeof(msg), "%s", g_err);
            return fail(rc, "problem %d: %s", i, msg);
        }
        if (p.steps < 0) return fail(PH3_EINVAL, "problem %d: steps must be >= 0", i);
        if (p.k != 0 && p.k != 1 && p.k != 2 && p.k != 4)
            return fail(PH3_EINVAL, "problem %d: k must be 0, 1, 2 or 4, got %d", i, p.k);
        if (p.k > 1 && p.dims != 2)
            return fail(PH3_EINVAL, "problem %d: k = %d needs a 2D problem", i, p.k);
    }
    const long long need = batch_workspace_bytes(problems, n);
    if (ws_bytes < need)
        return fail(PH3_EINVAL, "workspace needs %lld bytes, got %lld", need, (long long)ws_bytes);
    tune_init();  // the batch family's entry (keyed dims 3, fp32, k 1) picks the tile config
    const int cfg = g_tune_cfg[kFamBatch][1][PH3_FLOAT32][1].load();
    return finish(batch_prepare(problems, n, ws, ws_bytes, static_cast<cudaStream_t>(stream),
                                nullptr, cfg),
                  "batch prepare");
}

int ph3_batch_launch(void* ws, int n, void* stream) {
    if (ws == nullptr || n < 0) return fail(PH3_EINVAL, "ws must be non-null and n >= 0");
    tune_init();
    const int cfg = g_tune_cfg[kFamBatch][1][PH3_FLOAT32][1].load();
    return finish(batch_launch(ws, n, status_ptr(), static_cast<cudaStream_t>(stream), cfg),
                  "batch launch");
}

int ph3_batch_run_static(const ph3_problem* problems, int n, void* stream) {
    if (n < 0 || (n > 0 && problems == nullptr))
        return fail(PH3_EINVAL, "problems must be non-null and n >= 0");
    for (int i = 0; i < n; ++i) {
        const ph3_problem& p = problems[i];
        int rc = check_grid(p.dims, p.dims == 2 ? 1 : p.nz, p.ny, p.nx, p.storage, p.bc);
        if (rc == PH3_OK) rc = check_ptrs(p.a, p.b, p.src);
        if (rc != PH3_OK) {
            char msg[512];
            snprintf(msg, sizeof(msg), "%s", g_err);
            return fail(rc, "problem %d: %s", i, msg);
        }
        if (p.steps < 0) return fail(PH3_EINVAL, "problem %d: steps must be >= 0", i);
        if (p.k != 0 && p.k != 1 && p.k != 2 && p.k != 4)
            return fail(PH3_EINVAL, "problem %d: k must be 0, 1, 2 or 4, got %d", i, p.k);
        if (p.k > 1 && p.dims != 2)
            return fail(PH3_EINVAL, "problem %d: k = %d needs a 2D problem", i, p.k);
    }
    long long need = 0;
    tune_init();
    const int cfg = g_tune_cfg[kFamBatch][1][PH3_FLOAT32][1].load();
    const cudaError_t e = batch_run_static(problems, n, status_ptr(),
                                           static_cast<cudaStream_t>(stream), &need, cfg);
    if (e == cudaErrorInvalidValue && need > batch_static_capacity())
        return fail(PH3_EINVAL,
                    "batch plan needs %lld bytes; the static workspace holds %lld bytes "
                    "(use ph3_batch_prepare with a larger workspace)",
                    need, batch_static_capacity());
    return finish(e, "batch run (static workspace)");
}

static thread_local char g_name[64];

static int check_tune_key(int kernel, int dims, int storage, int k) {
    if (kernel < 0 || kernel >= kNumFamilies) return fail(PH3_EINVAL, "unknown kernel %d", kernel);
    if (dims != 2 && dims != 3) return fail(PH3_EINVAL, "dims must be 2 or 3, got %d", dims);
    if (storage < PH3_FLOAT32 || storage > PH3_BFLOAT16)
        return fail(PH3_EINVAL, "storage must be 0, 1 or 2, got %d", storage);
    if (k < 1 || k > kMaxK) return fail(PH3_EINVAL, "k must be in 1..%d, got %d", kMaxK, k);
    return PH3_OK;
}

int ph3_tune_count(int kernel, int dims, int k) {
    if (check_tune_key(kernel, dims, PH3_FLOAT32, k) != PH3_OK) return 0;
    return family_count(kernel, dims, k, nullptr, 0);
}

const char* ph3_tune_name(int kernel, int dims, int k, int cfg) {
    g_name[0] = '\0';
    if (check_tune_key(kernel, dims, PH3_FLOAT32, k) != PH3_OK) return g_name;
    const char* names[16] = {nullptr};
    const int n = family_count(kernel, dims, k, names, 16);
    if (cfg < 0 || cfg >= n || cfg >= 16 || names[cfg] == nullptr) {
        fail(PH3_EINVAL, "configuration %d out of range (%d)", cfg, n);
        return g_name;
    }
    snprintf(g_name, sizeof(g_name), "%s", names[cfg]);
    return g_name;
}

int ph3_tune_set(int kernel, int dims, int storage, int k, int cfg, int chunk) {
    int rc = check_tune_key(kernel, dims, storage, k);
    if (rc != PH3_OK) return rc;
    const int n = family_count(kernel, dims, k, nullptr, 0);
    if (cfg >= n) return fail(PH3_EINVAL, "configuration %d out of range (%d)", cfg, n);
    if (chunk < 0) return fail(PH3_EINVAL, "chunk must be >= 0");
    tune_init();
    g_tune_cfg[kernel][dims - 2][storage][k].store(cfg < 0 ? -1 : cfg);
    g_tune_chunk[kernel][dims - 2][storage][k].store(chunk);
    g_err[0] = '\0';
    return PH3_OK;
}

int ph3_tune_get(int kernel, int dims, int storage, int k, int* cfg, int* chunk) {
    int rc = check_tune_key(kernel, dims, storage, k);
    if (rc != PH3_OK) return rc;
    if (cfg == nullptr || chunk == nullptr) return fail(PH3_EINVAL, "cfg and chunk must be non-null");
    tune_init();
    *cfg = g_tune_cfg[kernel][dims - 2][storage][k].load();
    *chunk = g_tune_chunk[kernel][dims - 2][storage][k].load();
    return PH3_OK;
}

}  // extern "C"
