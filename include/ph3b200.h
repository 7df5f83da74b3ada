/*
 * ph3b200.h — C ABI of the pyheat3d B200 stencil backend (libph3b200.so, sm_100a).
 *
 * Conventions
 * - The caller owns all memory: every pointer is a device pointer the caller allocated
 *   (cudaMalloc, torch, ...). Entry points allocate nothing on the device.
 * - Arrays are C-ordered (z, y, x) in 3D and (y, x) in 2D with x contiguous. Storage is fp32,
 *   fp16 or bf16 (PH3_FLOAT32 / PH3_FLOAT16 / PH3_BFLOAT16); arithmetic is always fp32 and every
 *   result is bit-identical to pyheat3d's NumPy reference in the canonical summation order.
 * - `src` (optional, may be NULL) is the additive Jacobi source b, fp32, same shape as u.
 * - `u` and `out` must not alias (ping-pong). With PH3_DIRICHLET the outer layer of `out` is
 *   never written, so both buffers must carry the same boundary values.
 * - `stream` is a cudaStream_t (NULL = legacy default stream). Launches are asynchronous; no
 *   entry point synchronises the device unless its comment says so.
 * - Every function returns PH3_OK (0) or an error code; ph3_last_error() then gives a message
 *   (thread-local). Entry points are re-entrant.
 *
 * Reference interfaces replaced (pyheat3d, paths relative to the project root):
 *   src/pyheat3d/backends/stencil.cu        the NVRTC kernels naive2d/naive3d/zmarch3d/tb3d/tb2d
 *   src/pyheat3d/backends/cupy_backend.py   CupyStepper._launch / step (launch + remainder rule)
 */
#ifndef PH3B200_H
#define PH3B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* return codes */
#define PH3_OK 0
#define PH3_EINVAL 1       /* invalid argument (shape, pointer, storage, k, ...) */
#define PH3_ECUDA 2        /* a CUDA runtime call failed (message has the CUDA error string) */
#define PH3_EUNSUPPORTED 3 /* valid request this library cannot serve (e.g. grid too large) */
#define PH3_EDEVICE 4      /* a kernel reported an expired bounded wait (see ph3_device_status) */

/* storage types (stencil.cu:16-30 STORAGE macro: 0 fp32, 1 fp16, 2 bf16) */
#define PH3_FLOAT32 0
#define PH3_FLOAT16 1
#define PH3_BFLOAT16 2

/* boundary conditions (problem.py:18-21; stencil.cu PERIODIC macro) */
#define PH3_DIRICHLET 0
#define PH3_PERIODIC 1

/* kernel families for ph3_advance */
#define PH3_VARIANT_NAIVE 0 /* one site per thread (stencil.cu:43-93) */
#define PH3_VARIANT_MARCH 1 /* single-step march: TMA z-march in 3D, y-march in 2D */
#define PH3_VARIANT_TB 2    /* temporal blocking, k fused steps per pass */

/* kernel families of the tuning table */
#define PH3_KERNEL_ZMARCH 0 /* 3D TMA z-march, k = 1 */
#define PH3_KERNEL_MARCH 1  /* plain-load single-step march (2D y-march, 3D unaligned) */
#define PH3_KERNEL_TB 2     /* temporal blocking, k in {2, 3, 4, 8} */
#define PH3_KERNEL_NAIVE 3  /* one site per thread (no configurations) */
#define PH3_KERNEL_BATCH 4  /* batch tiles; one entry, keyed dims 3, PH3_FLOAT32, k 1 */

/* Library version (major*10000 + minor*100 + patch). */
int ph3_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* ph3_last_error(void);

/* Number of SMs of the current device (0 and an error message if no device). */
int ph3_sm_count(void);

/*
 * Read the current device's kernel status word into *code (0 = no expired wait) and reset it
 * when `clear` is nonzero. Synchronises the current device.
 */
int ph3_device_status(int* code, int clear);

/*
 * One update, one site per thread.
 * Replaces stencil.cu:43-64 naive2d(u, o, ny, nx, c0, c1) / :66-93 naive3d(u, o, nz, ny, nx,
 * c0, c1), where STORAGE and PERIODIC were NVRTC macros; here they are arguments.
 */
int ph3_naive2d(const void* u, void* out, const float* src, int ny, int nx, float c0, float c1,
                int storage, int bc, void* stream);
int ph3_naive3d(const void* u, void* out, const float* src, int nz, int ny, int nx, float c0,
                float c1, int storage, int bc, void* stream);

/*
 * One update by the 3D z-march. Replaces stencil.cu:101-161 zmarch3d(u, o, nz, ny, nx, c0, c1)
 * (BX/BY/ZCH macros -> `chunk`, the z-planes per work item; <= 0 picks a default). Uses TMA
 * plane staging when nx*sizeof(storage) is a multiple of 16 bytes and the buffers are 16-byte
 * aligned, otherwise a plain-load register march; the results are identical.
 */
int ph3_zmarch3d(const void* u, void* out, const float* src, int nz, int ny, int nx, float c0,
                 float c1, int storage, int bc, int chunk, void* stream);

/*
 * One update of the planes z0 .. z1-1 only (1 <= z0 <= z1 <= nz-1), reading planes z0-1 .. z1:
 * the z-march of ph3_zmarch3d restricted to a range of planes, with no wrap in z; `bc` applies
 * to x and y (Dirichlet also leaves the outer rows and columns of every plane unwritten). This
 * is the kernel of a z-slab split of one grid over several GPUs: a rank's array holds its slab
 * between two halo planes that the caller refreshes before each step (with periodic x / y for a
 * periodic grid). Planes outside the range are not written. No counterpart in the reference,
 * which runs one grid on one GPU (cupy_backend.py:188-194).
 */
int ph3_zmarch3d_planes(const void* u, void* out, const float* src, int nz, int ny, int nx,
                        int z0, int z1, float c0, float c1, int storage, int bc, int chunk,
                        void* stream);

/*
 * One update by the 2D y-march. Replaces stencil.cu:289-385 tb2d with K = 1 ("ymarch",
 * cupy_backend.py:63-70). `chunk` = rows per block (<= 0: default).
 */
int ph3_ymarch2d(const void* u, void* out, const float* src, int ny, int nx, float c0, float c1,
                 int storage, int bc, int chunk, void* stream);

/*
 * k fused updates in one pass (temporal blocking), k in {2, 3, 4, 8}; intermediate levels stay
 * in fp32 and are rounded to storage once per pass. Replaces stencil.cu:178-281
 * tb3d(u, o, nz, ny, nx, c0, c1) and :289-385 tb2d(u, o, ny, nx, c0, c1) (K macro -> k).
 */
int ph3_tb3d(const void* u, void* out, const float* src, int nz, int ny, int nx, int k, float c0,
             float c1, int storage, int bc, int chunk, void* stream);
int ph3_tb2d(const void* u, void* out, const float* src, int ny, int nx, int k, float c0,
             float c1, int storage, int bc, int chunk, void* stream);

/*
 * Geometry of the pass ph3_tb2d / ph3_tb3d make on this grid (the tuning table applied; 16-byte
 * aligned buffers assumed): the extended tile of one work item, *tx columns by *ty rows (*ty = 1
 * in 2D), and its chunk *chunk (planes in 3D, rows in 2D). Launches nothing; needs a device.
 * These are the inputs of pyheat3d's halo-traffic model of overlapped tiling, which
 * src/pyheat3d/benchmark.py:219-230 reads from the CuPy stepper's `tile` (traffic.py:38-50).
 */
int ph3_tb_tile(int dims, int nz, int ny, int nx, int storage, int bc, int k, int* tx, int* ty,
                int* chunk);

/*
 * Advance `nsteps` time steps / Jacobi sweeps on the ping-pong pair (a, b), starting from the
 * state in `a`: nsteps / k passes of the variant's main kernel, then nsteps % k single steps
 * (cupy_backend.py:188-194). *in_b is set to 1 when the final state is in `b`, else 0.
 * nz must be 1 when dims == 2. k must be 1 for the naive and march variants.
 */
int ph3_advance(int dims, int nz, int ny, int nx, int storage, int bc, float c0, float c1,
                int variant, int k, void* a, void* b, const float* src, int64_t nsteps,
                void* stream, int* in_b);

/*
 * Mixed-precision defect correction for lap(u) = f (Dirichlet, grid spacing h). No counterpart
 * in the reference, which runs plain Jacobi in one precision (validation.py:135-147).
 *
 * ph3_reduction_scratch_len: doubles of scratch the reductions below need (a constant).
 * ph3_dc_residual: FP64 residual r = f - A u, A u = (S(u) - 2d u) / h^2 on the interior
 *   (r = 0 on the boundary layer), written as the fp32 Jacobi source
 *   b = ((-h^2 / (2d)) * b_scale) * r of the scaled correction equation A e = b_scale * r
 *   (b may be NULL; b_scale is normally 1/s for a power of two s), and *rnorm2 = sum(r^2)
 *   (a device pointer). u, f: FP64 arrays of the grid's shape; nz = 1 in 2D.
 * ph3_dot_f64: *out = sum(x * y) over n FP64 values (device pointer out).
 * ph3_dc_correct: u += e_scale * e over n values; u FP64, e in `storage` (the correction).
 * Sums are deterministic for a given input (fixed partition and summation order).
 */
int64_t ph3_reduction_scratch_len(void);
int ph3_dc_residual(int dims, int nz, int ny, int nx, const double* u, const double* f, double h,
                    double b_scale, float* b, double* rnorm2, double* scratch, int64_t scratch_len,
                    void* stream);
int ph3_dot_f64(const double* x, const double* y, int64_t n, double* out, double* scratch,
                int64_t scratch_len, void* stream);
int ph3_dc_correct(double* u, const void* e, int storage, double e_scale, int64_t n,
                   void* stream);

/*
 * Batched solves: many independent grids of any sizes advanced in ONE persistent launch (no
 * counterpart in the reference, which launches every grid and step separately,
 * cupy_backend.py:183-194). Results equal the single-grid entry points bit for bit.
 *
 * Each ph3_problem names a ping-pong pair (a holds the initial state; with PH3_DIRICHLET, b must
 * hold the same boundary values), the grid, the coefficients, the number of steps and `k`: 0 or 1
 * advance the problem by single steps; 2 or 4 (2D problems only) by steps / k passes of k
 * fused steps each and then steps % k single steps (temporal blocking: 16-bit storage rounds
 * once per pass, as ph3_advance with a tb variant). After the launch a problem's state is in `a`
 * when its number of passes (steps, or steps / k + steps % k) is even, else in `b`.
 *
 * ph3_batch_workspace_bytes: device workspace (plan + counters) the problem list needs.
 * ph3_batch_prepare: validate the problems, build the plan and upload it into `ws` (synchronises
 *   `stream`; not capturable). The problem buffers must stay allocated until the launches end.
 * ph3_batch_launch: reset the counters and run the persistent kernel on `stream` (capturable in
 *   a CUDA graph; may be launched again after re-initialising the fields).
 */
typedef struct ph3_problem {
    void* a;
    void* b;
    const float* src; /* optional fp32 source b (NULL) */
    int32_t dims, nz, ny, nx;
    int32_t bc, storage;
    float c0, c1;
    int32_t steps;
    int32_t k; /* fused steps per pass: 0 or 1, or 2 / 4 for 2D problems */
} ph3_problem;

int64_t ph3_batch_workspace_bytes(const ph3_problem* problems, int n);
int ph3_batch_prepare(const ph3_problem* problems, int n, void* ws, int64_t ws_bytes,
                      void* stream);
int ph3_batch_launch(void* ws, int n, void* stream);

/*
 * ph3_batch_run_static: prepare and launch a batch without any device allocation — for hosts
 * that cannot call cudaMalloc where they run batches (a serving loop that must not allocate in
 * steady state, since an allocation can synchronise the device or fail under memory pressure;
 * a foreign host that hands over field buffers but owns no CUDA allocator). No counterpart in
 * the reference. The plan and counters live in a fixed 1 MiB device array inside the library
 * (every GPU that loads the library holds it until exit); problem lists whose plan needs more
 * (ph3_batch_workspace_bytes > 1 MiB, roughly 8000 problems or 100000 steps) are rejected with
 * PH3_EINVAL. Every call shares the array: the counters are cleared and the plan rewritten on
 * each call, and calls that overlap on the GPU race, so the caller must serialise them. The
 * first call on a device looks up the array's device address (make it before any stream
 * capture); each call synchronises `stream` after uploading the plan. The array used is the
 * current device's, so `stream` must belong to the current device. Results equal
 * ph3_batch_prepare + ph3_batch_launch bit for bit.
 */
int ph3_batch_run_static(const ph3_problem* problems, int n, void* stream);

/*
 * ph3_wait_flag: the bounded wait every persistent kernel of this library uses, run alone on
 * `stream` by one thread: poll *flag (device memory, acquire ordering) until it reaches `target`
 * or `spin_limit` polls (1 .. 4194304, each backing off about 0.25 us) have passed. A wait that
 * runs out records code 2 (dependency timeout) in the status word (ph3_device_status) and the
 * kernel returns, leaving the context usable. It is the host-visible check of the watchdog
 * path: a test points it at a flag that nothing sets and reads the status back. No counterpart
 * in the reference, whose only failure handling is on the host (registry.py:185-189
 * availability(), benchmark.py:289-293).
 */
int ph3_wait_flag(const int* flag, int target, unsigned int spin_limit, void* stream);

/*
 * Tuning table (no counterpart in the reference, whose tile constants are module globals that
 * bench/tune.py monkey-patches, cupy_backend.py:50-70). Every family has a few compiled tile
 * configurations; the table holds, per (kernel, dims, storage, k), the configuration index and
 * the march chunk (planes per work item in 3D, rows per block in 2D) that the launches use.
 * -1 / 0 mean "built-in default". The table is process-wide and applies to all devices.
 *
 * ph3_tune_count: number of configurations of (kernel, dims, k); 0 if none.
 * ph3_tune_name:  name of configuration `cfg` ("" and an error if out of range).
 * ph3_tune_set / ph3_tune_get: write / read one table entry.
 */
int ph3_tune_count(int kernel, int dims, int k);
const char* ph3_tune_name(int kernel, int dims, int k, int cfg);
int ph3_tune_set(int kernel, int dims, int storage, int k, int cfg, int chunk);
int ph3_tune_get(int kernel, int dims, int storage, int k, int* cfg, int* chunk);

#ifdef __cplusplus
}
#endif

#endif /* PH3B200_H */
