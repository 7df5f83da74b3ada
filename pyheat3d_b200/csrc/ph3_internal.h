// Host-side declarations shared by the kernel translation units and the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ph3b200.h"

namespace ph3 {

enum Storage : int { kF32 = 0, kF16 = 1, kBF16 = 2 };

// One stencil launch: out = step^k(u) for a ping-pong pair (u and out never alias).
struct Launch {
    const void* u;
    void* out;
    const float* src;   // optional Jacobi source b (fp32, same shape), nullptr if none
    int dims;           // 2 or 3
    int nz, ny, nx;     // nz == 1 in 2D
    bool periodic;
    int storage;        // Storage
    float c0, c1;
    int k;              // fused time steps (1 for single-step kernels)
    int chunk;          // march chunk length (planes in 3D, rows in 2D); <= 0 picks a default
    int cfg;            // compiled tile configuration of the family; < 0 picks the default
    int zb, ze;         // 3D single step: update only planes zb .. ze-1, no wrap in z (ze > 0;
                        // 1 <= zb <= ze <= nz-1); ze == 0: every plane the boundary allows
    cudaStream_t stream;
    int* err;           // device status word for bounded waits (may be null)
    int* geo;           // tb<k> only: when set, the launcher writes the extended tile width,
                        // height (1 in 2D) and chunk of its work items here and launches nothing
};

// Kernel families (ph3_stencil.cu, ph3_zmarch.cu). Each returns the launch status.
cudaError_t launch_naive(const Launch& L);
cudaError_t launch_march_k1(const Launch& L);   // register march, k = 1, any shape
cudaError_t launch_tb(const Launch& L);         // temporal blocking, k in {2,3,4,8}
cudaError_t launch_zmarch_tma(const Launch& L); // 3D TMA z-march, k = 1, aligned shapes
bool zmarch_tma_supported(const Launch& L);
// 3D single step for any nx from 1D tensor copies of row boxes (ph3_zmarch.cu); variant 0..2
cudaError_t launch_ring3d(const Launch& L, int variant);
bool ring3d_supported(const Launch& L);
cudaError_t launch_tbbulk(const Launch& L);     // 3D tb with a bulk-copy ring, aligned shapes
bool tbbulk_supported(const Launch& L);
int tbbulk_configs(int k, const char** names, int max);
cudaError_t launch_tb2d(const Launch& L);       // 2D tb, two-row wavefront (any shape)
int tb2d_configs(int k, const char** names, int max);
cudaError_t launch_tb3d_planes(const Launch& L);  // 3D tb, shared-memory level planes (any shape)

// Kernel families with selectable compiled configurations (the tuning table's first index).
enum Family : int {
    kFamZmarch = 0, kFamMarch = 1, kFamTb = 2, kFamNaive = 3, kFamBatch = 4, kNumFamilies = 5
};

// Names of the compiled configurations of a family for (dims, k); returns how many there are.
// names may be null. Implemented by the translation unit that owns the family.
int zmarch_configs(const char** names, int max);
int march_configs(int dims, const char** names, int max);
int tb_configs(int dims, int k, const char** names, int max);

// FP64 defect-correction kernels and deterministic reductions (ph3_dc.cu). The reductions
// write kReductionParts partial sums into caller-provided scratch, then sum them in one block.
constexpr int kReductionParts = 1024;
cudaError_t launch_dc_residual(int dims, int nz, int ny, int nx, const double* u, const double* f,
                               double h, double b_scale, float* b, double* out, double* scratch,
                               cudaStream_t stream);
cudaError_t launch_dot(const double* x, const double* y, int64_t n, double* out, double* scratch,
                       cudaStream_t stream);
cudaError_t launch_dc_correct(double* u, const void* e, int storage, double scale, int64_t n,
                              cudaStream_t stream);

// Batched persistent launch (ph3_batch.cu).
long long batch_workspace_bytes(const ph3_problem* p, int n);
cudaError_t batch_prepare(const ph3_problem* p, int n, void* ws, long long ws_bytes,
                          cudaStream_t stream, long long* total_items, int cfg);
int batch_configs(const char** names, int max);
// cfg: the tuning table's batch configuration (>= 3: the two-blocks-per-SM kernel); the tile
// geometry comes from the plan the workspace holds
cudaError_t batch_launch(void* ws, int n, int* err, cudaStream_t stream, int cfg);
long long batch_static_capacity();
cudaError_t batch_run_static(const ph3_problem* p, int n, int* err, cudaStream_t stream,
                             long long* need_bytes, int cfg);

// Number of streaming multiprocessors of the current device (cached per device).
int sm_count();

// Default march chunk: split the marching axis so that at least `target_ctas` blocks exist,
// never shorter than `min_len` planes; the result is clamped to [1, n_march].
int default_chunk(int n_march, long long tiles, int min_len, long long target_ctas);

}  // namespace ph3
