// Stencil kernels for any grid shape (sm_100a): naive single-site kernels and register marches
// for one time step; the dispatch of the temporal-blocking (tb<k>) families, whose kernels live
// in ph3_tb2d.cu (2D), ph3_tbbulk.cu (3D, aligned rows) and ph3_tbsmem.cu (3D, any rows).
//
// Functional spec (what, not how): pyheat3d src/pyheat3d/backends/stencil.cu
//   naive2d/naive3d :43-93, zmarch3d :101-161, tb2d with K = 1 (the y-march) :289-385,
// with the launch/remainder semantics of src/pyheat3d/backends/cupy_backend.py:141-194.
//
// Layout: C order, (z, y, x) / (y, x), x contiguous; storage fp32, fp16 or bf16; fp32 math.
// Dirichlet: the outer layer is never written. Periodic: every cell, wrap-around neighbours.
#include <algorithm>

#include "ph3_common.cuh"
#include "ph3_internal.h"
#include "ph3_march.cuh"
#include "ph3_tile3d.cuh"

namespace ph3 {

// ------------------------------------------------------------------------------------------
// naive: one lattice site per thread; every operand through L1/L2. The site's offset is formed
// once; the neighbours are signed deltas from it (+-1, +-nx, +-nx*ny), replaced by the wrapped
// delta only on the periodic boundary, so a site costs seven loads, the update and one store.
// Index arithmetic is in I: 32-bit whenever the field has fewer than 2^31 elements (one 32-bit
// offset per site, one wide address per load), 64-bit otherwise. The block shape is a
// compile-time constant.
// ------------------------------------------------------------------------------------------
constexpr int kNaive2X = 32, kNaive2Y = 8;
constexpr int kNaive3X = 32, kNaive3Y = 4, kNaive3Z = 2;

template <typename T, bool PER, bool SRC, typename I>
__global__ void __launch_bounds__(256)
naive2d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int ny,
               int nx, float c0, float c1) {
    const int i = blockIdx.x * kNaive2X + threadIdx.x;
    const int j = blockIdx.y * kNaive2Y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    if constexpr (!PER) {
        if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1) return;
    }
    const I c = I(j) * nx + i;
    I xm = -1, xp = 1, ym = -I(nx), yp = nx;
    if constexpr (PER) {
        xm = i == 0 ? I(nx - 1) : xm;
        xp = i == nx - 1 ? I(1 - nx) : xp;
        ym = j == 0 ? I(ny - 1) * nx : ym;
        yp = j == ny - 1 ? -I(ny - 1) * nx : yp;
    }
    const T* p = u + c;
    float v = upd2(c0, c1, ldg1(p), ldg1(p + xm), ldg1(p + xp), ldg1(p + ym), ldg1(p + yp));
    if constexpr (SRC) v = __fadd_rn(v, __ldg(b + c));
    o[c] = from_f<T>(v);
}

template <typename T, bool PER, bool SRC, typename I>
__global__ void __launch_bounds__(256)
naive3d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int nz,
               int ny, int nx, float c0, float c1) {
    const int i = blockIdx.x * kNaive3X + threadIdx.x;
    const int j = blockIdx.y * kNaive3Y + threadIdx.y;
    const int k = blockIdx.z * kNaive3Z + threadIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    if constexpr (!PER) {
        if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1) return;
    }
    const I P = I(nx) * ny;
    const I c = I(k) * P + I(j) * nx + i;
    I xm = -1, xp = 1, ym = -I(nx), yp = nx, zm = -P, zp = P;
    if constexpr (PER) {
        xm = i == 0 ? I(nx - 1) : xm;
        xp = i == nx - 1 ? I(1 - nx) : xp;
        ym = j == 0 ? P - nx : ym;
        yp = j == ny - 1 ? nx - P : yp;
        zm = k == 0 ? I(nz - 1) * P : zm;
        zp = k == nz - 1 ? -I(nz - 1) * P : zp;
    }
    const T* p = u + c;
    float v = upd3(c0, c1, ldg1(p), ldg1(p + xm), ldg1(p + xp), ldg1(p + ym), ldg1(p + yp),
                   ldg1(p + zm), ldg1(p + zp));
    if constexpr (SRC) v = __fadd_rn(v, __ldg(b + c));
    o[c] = from_f<T>(v);
}

template <typename T, bool PER, int V, int W, int RB>
__global__ void __launch_bounds__(32 * W)
march2d_k1_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b,
                  int ny, int nx, float c0, float c1, int ych, int vec_i) {
    march2d_item<T, PER, V, W, RB, false>(u, o, b, ny, nx, c0, c1, blockIdx.x * W, blockIdx.y,
                                          ych, vec_i != 0);
}

template <typename T, bool PER, int W, int RB>
__global__ void __launch_bounds__(32 * W)
march2d_raw_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b,
                   int ny, int nx, float c0, float c1, int ych) {
    march2d_raw_item<T, PER, RB, false>(u, o, b, ny, nx, c0, c1, blockIdx.x * W + (threadIdx.x >> 5),
                                        blockIdx.y, ych);
}

template <typename T, bool PER, int V, int R, int W>
__global__ void __launch_bounds__(32 * W)
march3d_k1_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b,
                  int nz, int ny, int nx, float c0, float c1, int zch, int vec_i) {
    __shared__ __align__(16) float edge[2 * W * 32 * V];
    march3d_item<T, PER, V, R, W, false>(u, o, b, nz, ny, nx, c0, c1, blockIdx.x, blockIdx.y,
                                         blockIdx.z, zch, vec_i != 0, edge);
}

template <typename T, bool PER, int R, int W, bool SRC = true>
__global__ void __launch_bounds__(32 * W)
lite3d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int nz,
              int ny, int nx, float c0, float c1, int zch, int zb, int ze) {
    const int w = threadIdx.x >> 5;
    const int z0 = zb + blockIdx.z * zch;
    lite3d_item<T, PER, R, false, SRC>(u, o, b, nz, ny, nx, c0, c1, blockIdx.x,
                                       (blockIdx.y * W + w) * R, z0, min(z0 + zch, ze));
}

template <typename T, bool PER, bool SRC>
__global__ void __launch_bounds__(32 * Tile3::W)
tile3d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int nz,
              int ny, int nx, float c0, float c1, int zch) {
    __shared__ __align__(16) float sm[Tile3::SMEM / 4];
    const int z0 = blockIdx.z * zch;
    tile3d_item<T, PER, SRC, false>(u, o, b, nz, ny, nx, c0, c1, blockIdx.x, blockIdx.y, z0,
                                    min(z0 + zch, nz), sm);
}

template <typename T, bool PER, int R, int W>
__global__ void __launch_bounds__(32 * W)
avec3d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int nz,
              int ny, int nx, float c0, float c1, int zch, int zb, int ze) {
    const int w = threadIdx.x >> 5;
    const int z0 = zb + blockIdx.z * zch;
    avec3d_item<T, PER, R, false>(u, o, b, nz, ny, nx, c0, c1, blockIdx.x,
                                  (blockIdx.y * W + w) * R, z0, min(z0 + zch, ze));
}

template <typename T, bool PER, int RB, int W, bool SRC = true>
__global__ void __launch_bounds__(32 * W)
lite2d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int ny,
              int nx, float c0, float c1, int ych) {
    const int y0 = blockIdx.y * ych;
    lite2d_item<T, PER, RB, false, SRC>(u, o, b, ny, nx, c0, c1,
                                        blockIdx.x * W + (threadIdx.x >> 5), y0,
                                        min(y0 + ych, ny));
}

// ------------------------------------------------------------------------------------------
// host launchers
// ------------------------------------------------------------------------------------------
static inline int cdiv(long long a, long long b) { return int((a + b - 1) / b); }

static bool aligned_to(const void* p, size_t bytes) {
    return p == nullptr || (reinterpret_cast<uintptr_t>(p) % bytes) == 0;
}

int default_chunk(int n_march, long long tiles, int min_len, long long target_ctas) {
    long long want = (target_ctas + tiles - 1) / std::max(1LL, tiles);
    want = std::max(1LL, want);
    int len = cdiv(n_march, want);
    len = std::max(len, min_len);
    return std::min(std::max(len, 1), n_march);
}

template <typename T, bool PER, typename I>
static cudaError_t naive_launch(const Launch& L) {
    const T* u = static_cast<const T*>(L.u);
    T* o = static_cast<T*>(L.out);
    if (L.dims == 2) {
        dim3 blk(kNaive2X, kNaive2Y), grd(cdiv(L.nx, kNaive2X), cdiv(L.ny, kNaive2Y));
        if (grd.y > 65535) return cudaErrorInvalidConfiguration;
        if (L.src != nullptr)
            naive2d_kernel<T, PER, true, I><<<grd, blk, 0, L.stream>>>(u, o, L.src, L.ny, L.nx,
                                                                       L.c0, L.c1);
        else
            naive2d_kernel<T, PER, false, I><<<grd, blk, 0, L.stream>>>(u, o, nullptr, L.ny, L.nx,
                                                                        L.c0, L.c1);
    } else {
        dim3 blk(kNaive3X, kNaive3Y, kNaive3Z);
        dim3 grd(cdiv(L.nx, kNaive3X), cdiv(L.ny, kNaive3Y), cdiv(L.nz, kNaive3Z));
        if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
        if (L.src != nullptr)
            naive3d_kernel<T, PER, true, I><<<grd, blk, 0, L.stream>>>(u, o, L.src, L.nz, L.ny,
                                                                       L.nx, L.c0, L.c1);
        else
            naive3d_kernel<T, PER, false, I><<<grd, blk, 0, L.stream>>>(u, o, nullptr, L.nz, L.ny,
                                                                        L.nx, L.c0, L.c1);
    }
    return cudaGetLastError();
}

template <typename T, bool PER>
static cudaError_t naive_t(const Launch& L) {
    const long long n = 1LL * (L.dims == 2 ? 1 : L.nz) * L.ny * L.nx;
    // 32-bit offsets when every offset and wrapped delta (|delta| < n) fits
    if (n < (1LL << 31)) return naive_launch<T, PER, int>(L);
    return naive_launch<T, PER, int64_t>(L);
}

template <typename T, bool PER, int V>
static bool vec_ok(const Launch& L) {
    return L.nx % V == 0 && aligned_to(L.u, sizeof(T) * V) && aligned_to(L.out, sizeof(T) * V) &&
           aligned_to(L.src, sizeof(float) * V);
}

template <typename T, bool PER>
static cudaError_t march_k1_t(const Launch& L) {
    const T* u = static_cast<const T*>(L.u);
    T* o = static_cast<T*>(L.out);
    const long long target = 8LL * sm_count();
    // defaults measured on a B200: in 3D the lean one-column-per-lane march (2.1-2.4x the
    // vector march on unaligned grids); in 2D the raw-row march, 8 rows per step for fp32 and
    // 6 for 16-bit storage (16384^2: fp32 805 vs 674 GLUPS for the float-window march, bf16
    // 1289 vs 547)
    int cfg = L.cfg >= 0 ? L.cfg : (L.dims == 3 ? 0 : (sizeof(T) == 4 ? 3 : 4));
    if (L.dims == 3 && cfg >= 4 && cfg <= 6) {
        // row boxes by 1D tensor copies into per-warp shared-memory rings
        if (ring3d_supported(L)) return launch_ring3d(L, cfg - 4);
        cfg = 0;
    }
    if (L.dims == 3 && (cfg == 2 || cfg == 3)) {
        // any-alignment lane vectors: 4 columns per lane; array bases aligned to 4 elements
        if (aligned_to(L.u, 4 * sizeof(T)) && aligned_to(L.out, 4 * sizeof(T)) &&
            aligned_to(L.src, 16)) {
            constexpr int W = 4;
            const int R = cfg == 2 ? 4 : 2;
            const int zb = L.ze > 0 ? L.zb : 0, ze = L.ze > 0 ? L.ze : L.nz;
            const long long tiles = 1LL * cdiv(L.nx, 128) * cdiv(L.ny, W * R);
            const int zch = L.chunk > 0 ? L.chunk : default_chunk(ze - zb, tiles, 16, 2 * target);
            dim3 grd(cdiv(L.nx, 128), cdiv(L.ny, W * R), cdiv(ze - zb, zch));
            if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
            if (cfg == 2)
                avec3d_kernel<T, PER, 4, W><<<grd, 32 * W, 0, L.stream>>>(
                    u, o, L.src, L.nz, L.ny, L.nx, L.c0, L.c1, zch, zb, ze);
            else
                avec3d_kernel<T, PER, 2, W><<<grd, 32 * W, 0, L.stream>>>(
                    u, o, L.src, L.nz, L.ny, L.nx, L.c0, L.c1, zch, zb, ze);
            return cudaGetLastError();
        }
        cfg = 0;
    }
    if (L.ze > 0) cfg = 0;  // z ranges: the lean march or the lane-vector march above
    if (L.dims == 3 && cfg == 7) {
        // block-wide shared-memory plane tiles, 64 x 32 columns
        const long long tiles = 1LL * cdiv(L.nx, Tile3::OX) * cdiv(L.ny, Tile3::OY);
        const int zch = L.chunk > 0 ? L.chunk : default_chunk(L.nz, tiles, 16, 2 * target);
        dim3 grd(cdiv(L.nx, Tile3::OX), cdiv(L.ny, Tile3::OY), cdiv(L.nz, zch));
        if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
        if (int64_t(L.nx) * L.ny >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
        if (L.src != nullptr)
            tile3d_kernel<T, PER, true><<<grd, 32 * Tile3::W, 0, L.stream>>>(
                u, o, L.src, L.nz, L.ny, L.nx, L.c0, L.c1, zch);
        else
            tile3d_kernel<T, PER, false><<<grd, 32 * Tile3::W, 0, L.stream>>>(
                u, o, nullptr, L.nz, L.ny, L.nx, L.c0, L.c1, zch);
        return cudaGetLastError();
    }
    if (cfg == 0) {
        if (L.dims == 2) {
            constexpr int W = 4, RB = 4;
            const int strips = cdiv(L.nx, 32);
            const int ych = L.chunk > 0 ? L.chunk
                                        : default_chunk(L.ny, cdiv(strips, W), 8 * RB, 2 * target);
            dim3 grd(cdiv(strips, W), cdiv(L.ny, ych));
            if (grd.y > 65535) return cudaErrorInvalidConfiguration;
            if (L.src != nullptr)
                lite2d_kernel<T, PER, RB, W, true><<<grd, 32 * W, 0, L.stream>>>(
                    u, o, L.src, L.ny, L.nx, L.c0, L.c1, ych);
            else
                lite2d_kernel<T, PER, RB, W, false><<<grd, 32 * W, 0, L.stream>>>(
                    u, o, nullptr, L.ny, L.nx, L.c0, L.c1, ych);
        } else {
            constexpr int R = 4, W = 4;
            // planes zb .. ze-1 (a z range never wraps: its neighbour planes are in the array)
            const int zb = L.ze > 0 ? L.zb : 0, ze = L.ze > 0 ? L.ze : L.nz;
            const long long tiles = 1LL * cdiv(L.nx, 32) * cdiv(L.ny, W * R);
            const int zch = L.chunk > 0 ? L.chunk : default_chunk(ze - zb, tiles, 16, 2 * target);
            dim3 grd(cdiv(L.nx, 32), cdiv(L.ny, W * R), cdiv(ze - zb, zch));
            if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
            if (L.src != nullptr)
                lite3d_kernel<T, PER, R, W, true><<<grd, 32 * W, 0, L.stream>>>(
                    u, o, L.src, L.nz, L.ny, L.nx, L.c0, L.c1, zch, zb, ze);
            else
                lite3d_kernel<T, PER, R, W, false><<<grd, 32 * W, 0, L.stream>>>(
                    u, o, nullptr, L.nz, L.ny, L.nx, L.c0, L.c1, zch, zb, ze);
        }
        return cudaGetLastError();
    }
    if (L.dims == 2 && cfg >= 2 && vec_ok<T, PER, 16 / sizeof(T)>(L)) {
        // raw-row march: 2 -> 4 rows per step, 3 -> 8, 4 -> 6 (4 warps per block)
        constexpr int V = 16 / sizeof(T), W = 4;
        const int rb = cfg == 2 ? 4 : (cfg == 4 ? 6 : 8);
        const int strips = cdiv(L.nx, 32 * V);
        // many short row chunks (about 64 rows at 16384^2, the measured best) keep more blocks
        // and loads in flight than one chunk per resident block
        const int ych = L.chunk > 0 ? L.chunk
                                    : default_chunk(L.ny, cdiv(strips, W), 4 * rb, 8 * target);
        dim3 grd(cdiv(strips, W), cdiv(L.ny, ych));
        if (grd.y > 65535) return cudaErrorInvalidConfiguration;
        if (cfg == 2)
            march2d_raw_kernel<T, PER, W, 4><<<grd, 32 * W, 0, L.stream>>>(u, o, L.src, L.ny, L.nx,
                                                                         L.c0, L.c1, ych);
        else if (cfg == 4)
            march2d_raw_kernel<T, PER, W, 6><<<grd, 32 * W, 0, L.stream>>>(u, o, L.src, L.ny, L.nx,
                                                                         L.c0, L.c1, ych);
        else
            march2d_raw_kernel<T, PER, W, 8><<<grd, 32 * W, 0, L.stream>>>(u, o, L.src, L.ny, L.nx,
                                                                         L.c0, L.c1, ych);
        return cudaGetLastError();
    }
    if (L.dims == 2) {
        constexpr int V = 16 / sizeof(T), W = 4, RB = sizeof(T) == 4 ? 4 : 2;
        const int strips = cdiv(L.nx, 32 * V);
        const int ych = L.chunk > 0 ? L.chunk
                                    : default_chunk(L.ny, cdiv(strips, W), 4 * RB, target);
        dim3 grd(cdiv(strips, W), cdiv(L.ny, ych));
        if (grd.y > 65535) return cudaErrorInvalidConfiguration;
        march2d_k1_kernel<T, PER, V, W, RB><<<grd, 32 * W, 0, L.stream>>>(
            u, o, L.src, L.ny, L.nx, L.c0, L.c1, ych, vec_ok<T, PER, V>(L) ? 1 : 0);
    } else {
        constexpr int V = 16 / sizeof(T), R = 2, W = 8;
        const long long tiles = 1LL * cdiv(L.nx, 32 * V) * cdiv(L.ny, W * R);
        const int zch = L.chunk > 0 ? L.chunk : default_chunk(L.nz, tiles, 8, target);
        dim3 grd(cdiv(L.nx, 32 * V), cdiv(L.ny, W * R), cdiv(L.nz, zch));
        if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
        march3d_k1_kernel<T, PER, V, R, W><<<grd, 32 * W, 0, L.stream>>>(
            u, o, L.src, L.nz, L.ny, L.nx, L.c0, L.c1, zch, vec_ok<T, PER, V>(L) ? 1 : 0);
    }
    return cudaGetLastError();
}

#define PH3_DISPATCH(fn, L)                                                               \
    do {                                                                                  \
        switch ((L).storage) {                                                            \
            case kF32: return (L).periodic ? fn<float, true>(L) : fn<float, false>(L);    \
            case kF16: return (L).periodic ? fn<__half, true>(L) : fn<__half, false>(L);  \
            case kBF16:                                                                   \
                return (L).periodic ? fn<__nv_bfloat16, true>(L)                          \
                                    : fn<__nv_bfloat16, false>(L);                        \
            default: return cudaErrorInvalidValue;                                        \
        }                                                                                 \
    } while (0)

cudaError_t launch_naive(const Launch& L) { PH3_DISPATCH(naive_t, L); }
cudaError_t launch_march_k1(const Launch& L) { PH3_DISPATCH(march_k1_t, L); }

cudaError_t launch_tb(const Launch& L) {
    if (L.dims == 2) return launch_tb2d(L);
    if (tbbulk_supported(L)) return launch_tbbulk(L);
    return launch_tb3d_planes(L);
}

// 2D: 0 lean one-column-per-lane march, 1 float-window vector march, 2 / 3 / 4 raw-row vector
// march with 4 / 8 / 6 rows per step (shapes without whole 16-byte rows fall back to 1). 3D: 0 lean,
// 1 vector march, 2 / 3 any-alignment lane vectors with 4 / 2 rows per warp, 4 / 5 / 6 row boxes
// by 1D tensor copies into per-warp rings (rows per warp, ring stages: 2/3, 2/4, 4/3), 7 block-wide
// shared-memory plane tiles of 64 x 32 columns.
int march_configs(int dims, const char** names, int max) {
    static const char* k2[] = {"lane1_W4_RB4", "V16B_W4_RB4", "raw16B_W4_RB4", "raw16B_W4_RB8",
                               "raw16B_W4_RB6"};
    static const char* k3[] = {"lane1_R4_W4", "V16B_R2_W8", "V4any_R4_W4", "V4any_R2_W4",
                               "ring1d_R2_W4_S3", "ring1d_R2_W4_S4", "ring1d_R4_W4_S3",
                               "smem_tile_64x32"};
    const int n = dims == 2 ? 5 : 8;
    for (int i = 0; i < n && names != nullptr && i < max; ++i) names[i] = dims == 2 ? k2[i] : k3[i];
    return n;
}

int tb_configs(int dims, int k, const char** names, int max) {
    return dims == 3 ? tbbulk_configs(k, names, max) : tb2d_configs(k, names, max);
}

}  // namespace ph3
