// Stencil kernels for any grid shape (sm_100a): naive single-site kernels, register marches
// for one time step, and temporal-blocking (tb<k>) wavefront kernels.
//
// Functional spec (what, not how): pyheat3d src/pyheat3d/backends/stencil.cu
//   naive2d/naive3d :43-93, zmarch3d :101-161, tb3d :178-281, tb2d (K=1 -> ymarch) :289-385,
// with the launch/remainder semantics of src/pyheat3d/backends/cupy_backend.py:141-194.
//
// Layout: C order, (z, y, x) / (y, x), x contiguous; storage fp32, fp16 or bf16; fp32 math.
// Dirichlet: the outer layer is never written. Periodic: every cell, wrap-around neighbours.
#include <algorithm>

#include "ph3_common.cuh"
#include "ph3_internal.h"
#include "ph3_march.cuh"

namespace ph3 {

// ------------------------------------------------------------------------------------------
// naive: one lattice site per thread; every operand through L1/L2
// ------------------------------------------------------------------------------------------
template <typename T, bool PER>
__global__ void __launch_bounds__(256)
naive2d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int ny,
               int nx, float c0, float c1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    int im, ip, jm, jp;
    if constexpr (PER) {
        im = i == 0 ? nx - 1 : i - 1; ip = i == nx - 1 ? 0 : i + 1;
        jm = j == 0 ? ny - 1 : j - 1; jp = j == ny - 1 ? 0 : j + 1;
    } else {
        if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1) return;
        im = i - 1; ip = i + 1; jm = j - 1; jp = j + 1;
    }
    const int64_t r = int64_t(j) * nx;
    float v = upd2(c0, c1, ldg1(u + r + i), ldg1(u + r + im), ldg1(u + r + ip),
                   ldg1(u + int64_t(jm) * nx + i), ldg1(u + int64_t(jp) * nx + i));
    if (b != nullptr) v = __fadd_rn(v, __ldg(b + r + i));
    o[r + i] = from_f<T>(v);
}

template <typename T, bool PER>
__global__ void __launch_bounds__(256)
naive3d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int nz,
               int ny, int nx, float c0, float c1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    int im, ip, jm, jp, km, kp;
    if constexpr (PER) {
        im = i == 0 ? nx - 1 : i - 1; ip = i == nx - 1 ? 0 : i + 1;
        jm = j == 0 ? ny - 1 : j - 1; jp = j == ny - 1 ? 0 : j + 1;
        km = k == 0 ? nz - 1 : k - 1; kp = k == nz - 1 ? 0 : k + 1;
    } else {
        if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1) return;
        im = i - 1; ip = i + 1; jm = j - 1; jp = j + 1; km = k - 1; kp = k + 1;
    }
    const int64_t P = int64_t(nx) * ny;
    const int64_t c = int64_t(k) * P + int64_t(j) * nx;
    float v = upd3(c0, c1, ldg1(u + c + i), ldg1(u + c + im), ldg1(u + c + ip),
                   ldg1(u + int64_t(k) * P + int64_t(jm) * nx + i),
                   ldg1(u + int64_t(k) * P + int64_t(jp) * nx + i),
                   ldg1(u + int64_t(km) * P + int64_t(j) * nx + i),
                   ldg1(u + int64_t(kp) * P + int64_t(j) * nx + i));
    if (b != nullptr) v = __fadd_rn(v, __ldg(b + c + i));
    o[c + i] = from_f<T>(v);
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

// ------------------------------------------------------------------------------------------
// temporal blocking, 3D: k fused steps per pass, (z, t) wavefront with overlapped tiling.
// The block's extended xy tile is 32*V x W*R sites (lane l: V columns, warp w: R rows); the
// valid region shrinks by one site per level and only the centre OX x OY sites are stored.
// Level s (1..K) of plane iz-s is computed while plane iz+1 is in flight; each level keeps a
// 3-plane register queue. The x halo is rounded up to whole vectors so loads and stores stay
// aligned vectors.
// ------------------------------------------------------------------------------------------
template <typename T, bool PER, int K, int V, int R, int W>
__global__ void __launch_bounds__(32 * W)
tb3d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int nz,
            int ny, int nx, float c0, float c1, int zch, int vec_i) {
    constexpr int KX = ((K + V - 1) / V) * V;
    constexpr int EX = 32 * V, OX = EX - 2 * KX;
    constexpr int EY = W * R, OY = EY - 2 * K;
    static_assert(OX > 0 && OY > 0, "tile too small for k");
    __shared__ __align__(16) float edge[2][2][W][EX];  // [buffer][first/last][warp][column]
    const bool vec = vec_i != 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gx = blockIdx.x * OX - KX + lane * V;
    const int gy0 = blockIdx.y * OY - K + w * R;
    const int z0 = blockIdx.z * zch, z1 = min(z0 + zch, nz);
    const int64_t P = int64_t(nx) * ny;

    Cols<PER, V> cols;
    cols.init(gx, nx, vec);
    int64_t roff[R];
#pragma unroll
    for (int r = 0; r < R; ++r) roff[r] = int64_t(fix_near<PER>(gy0 + r, ny)) * nx;
    uint32_t fixx = 0, fixy = 0;  // Dirichlet: boundary or outside sites keep their value
    if constexpr (!PER) {
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gx + j <= 0 || gx + j >= nx - 1) fixx |= 1u << j;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (gy0 + r <= 0 || gy0 + r >= ny - 1) fixy |= 1u << r;
    }
    const int lx = lane * V;
    const bool xwriter = lx >= KX && lx < KX + OX;

    float q[K][3][R][V];
#pragma unroll
    for (int s = 0; s < K; ++s)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int j = 0; j < V; ++j) q[s][a][r][j] = 0.f;

    float pre[R][V];
    auto load_plane = [&](int z, float (&dst)[R][V]) {
        const T* pl = u + int64_t(fix_near<PER>(z, nz)) * P;
#pragma unroll
        for (int r = 0; r < R; ++r) cols.load(pl + roff[r], vec, dst[r]);
    };
    load_plane(z0 - K, pre);
    int buf = 0;

    for (int iz = z0 - K; iz < z1 + K; ++iz) {
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int j = 0; j < V; ++j) {
                q[0][0][r][j] = q[0][1][r][j];
                q[0][1][r][j] = q[0][2][r][j];
                q[0][2][r][j] = pre[r][j];
            }
        if (iz + 1 < z1 + K) load_plane(iz + 1, pre);
        float res[R][V];
#pragma unroll
        for (int s = 1; s <= K; ++s) {
            const int c = iz - s;
            float up[V], dn[V];
            if constexpr (W > 1) {
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    edge[buf][0][w][lx + j] = q[s - 1][1][0][j];
                    edge[buf][1][w][lx + j] = q[s - 1][1][R - 1][j];
                }
                __syncthreads();
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    up[j] = w > 0 ? edge[buf][1][w - 1][lx + j] : q[s - 1][1][0][j];
                    dn[j] = w < W - 1 ? edge[buf][0][w + 1][lx + j] : q[s - 1][1][R - 1][j];
                }
                buf ^= 1;
            } else {
#pragma unroll
                for (int j = 0; j < V; ++j) { up[j] = q[s - 1][1][0][j]; dn[j] = q[s - 1][1][R - 1][j]; }
            }
            const bool zfix = !PER && (c <= 0 || c >= nz - 1);
            const float* bpl = b != nullptr ? b + int64_t(fix_near<PER>(c, nz)) * P : nullptr;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float left = __shfl_up_sync(kFull, q[s - 1][1][r][V - 1], 1);
                const float right = __shfl_down_sync(kFull, q[s - 1][1][r][0], 1);
                float bv[V];
                if (bpl != nullptr) cols.load_src(bpl + roff[r], vec, bv);
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    const float ctr = q[s - 1][1][r][j];
                    const float xm = j > 0 ? q[s - 1][1][r][j - 1] : left;
                    const float xp = j < V - 1 ? q[s - 1][1][r][j + 1] : right;
                    const float ym = r > 0 ? q[s - 1][1][r - 1][j] : up[j];
                    const float yp = r < R - 1 ? q[s - 1][1][r + 1][j] : dn[j];
                    float v = upd3(c0, c1, ctr, xm, xp, ym, yp, q[s - 1][0][r][j], q[s - 1][2][r][j]);
                    if (bpl != nullptr) v = __fadd_rn(v, bv[j]);
                    if constexpr (!PER) {
                        if (zfix || ((fixy >> r) & 1u) || ((fixx >> j) & 1u)) v = ctr;
                    }
                    res[r][j] = v;
                }
            }
            if (s < K) {
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int j = 0; j < V; ++j) {
                        q[s][0][r][j] = q[s][1][r][j];
                        q[s][1][r][j] = q[s][2][r][j];
                        q[s][2][r][j] = res[r][j];
                    }
            }
        }
        const int c = iz - K;
        const bool zok = c >= z0 && c < z1 && (PER || (c > 0 && c < nz - 1));
        if (zok && xwriter) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int row = w * R + r, gy = gy0 + r;
                if (row >= K && row < K + OY && gy < ny && !((fixy >> r) & 1u))
                    store_cols<T, V>(o + int64_t(c) * P + int64_t(gy) * nx, gx, nx, vec, fixx,
                                     res[r]);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// temporal blocking, 2D: warp-synchronous; each warp owns an extended strip of 32*V columns
// and walks a chunk of rows with a K-level 3-row register queue. No shared memory, no block
// sync. Strips overlap by 2*KX columns.
// ------------------------------------------------------------------------------------------
template <typename T, bool PER, int K, int V, int W>
__global__ void __launch_bounds__(32 * W)
tb2d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int ny,
            int nx, float c0, float c1, int ych, int vec_i) {
    constexpr int KX = ((K + V - 1) / V) * V;
    constexpr int EX = 32 * V, OX = EX - 2 * KX;
    static_assert(OX > 0, "strip too narrow for k");
    const bool vec = vec_i != 0;
    const int lane = threadIdx.x & 31;
    const int strip = blockIdx.x * W + (threadIdx.x >> 5);
    if (strip * OX >= nx) return;  // warp-uniform; no block sync in this kernel
    const int gx = strip * OX - KX + lane * V;
    const int y0 = blockIdx.y * ych, y1 = min(y0 + ych, ny);

    Cols<PER, V> cols;
    cols.init(gx, nx, vec);
    uint32_t fixx = 0;
    if constexpr (!PER) {
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gx + j <= 0 || gx + j >= nx - 1) fixx |= 1u << j;
    }
    const int lx = lane * V;
    const bool xwriter = lx >= KX && lx < KX + OX;

    float q[K][3][V];
#pragma unroll
    for (int s = 0; s < K; ++s)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int j = 0; j < V; ++j) q[s][a][j] = 0.f;
    float pre[V];
    cols.load(u + int64_t(fix_near<PER>(y0 - K, ny)) * nx, vec, pre);

    for (int iy = y0 - K; iy < y1 + K; ++iy) {
#pragma unroll
        for (int j = 0; j < V; ++j) {
            q[0][0][j] = q[0][1][j];
            q[0][1][j] = q[0][2][j];
            q[0][2][j] = pre[j];
        }
        if (iy + 1 < y1 + K) cols.load(u + int64_t(fix_near<PER>(iy + 1, ny)) * nx, vec, pre);
        float res[V];
#pragma unroll
        for (int s = 1; s <= K; ++s) {
            const int c = iy - s;
            const bool yfix = !PER && (c <= 0 || c >= ny - 1);
            const float left = __shfl_up_sync(kFull, q[s - 1][1][V - 1], 1);
            const float right = __shfl_down_sync(kFull, q[s - 1][1][0], 1);
            float bv[V];
            if (b != nullptr) cols.load_src(b + int64_t(fix_near<PER>(c, ny)) * nx, vec, bv);
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const float ctr = q[s - 1][1][j];
                const float xm = j > 0 ? q[s - 1][1][j - 1] : left;
                const float xp = j < V - 1 ? q[s - 1][1][j + 1] : right;
                float v = upd2(c0, c1, ctr, xm, xp, q[s - 1][0][j], q[s - 1][2][j]);
                if (b != nullptr) v = __fadd_rn(v, bv[j]);
                if constexpr (!PER) {
                    if (yfix || ((fixx >> j) & 1u)) v = ctr;
                }
                res[j] = v;
            }
            if (s < K) {
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    q[s][0][j] = q[s][1][j];
                    q[s][1][j] = q[s][2][j];
                    q[s][2][j] = res[j];
                }
            }
        }
        const int c = iy - K;
        const bool yok = c >= y0 && c < y1 && (PER || (c > 0 && c < ny - 1));
        if (yok && xwriter) store_cols<T, V>(o + int64_t(c) * nx, gx, nx, vec, fixx, res);
    }
}

template <typename T, bool PER, int R, int W>
__global__ void __launch_bounds__(32 * W)
lite3d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int nz,
              int ny, int nx, float c0, float c1, int zch, int zb, int ze) {
    const int w = threadIdx.x >> 5;
    const int z0 = zb + blockIdx.z * zch;
    lite3d_item<T, PER, R, false>(u, o, b, nz, ny, nx, c0, c1, blockIdx.x,
                                  (blockIdx.y * W + w) * R, z0, min(z0 + zch, ze));
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

template <typename T, bool PER, int RB, int W>
__global__ void __launch_bounds__(32 * W)
lite2d_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b, int ny,
              int nx, float c0, float c1, int ych) {
    const int y0 = blockIdx.y * ych;
    lite2d_item<T, PER, RB, false>(u, o, b, ny, nx, c0, c1, blockIdx.x * W + (threadIdx.x >> 5),
                                   y0, min(y0 + ych, ny));
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

template <typename T, bool PER>
static cudaError_t naive_t(const Launch& L) {
    const T* u = static_cast<const T*>(L.u);
    T* o = static_cast<T*>(L.out);
    if (L.dims == 2) {
        dim3 blk(32, 8), grd(cdiv(L.nx, 32), cdiv(L.ny, 8));
        if (grd.y > 65535) return cudaErrorInvalidConfiguration;
        naive2d_kernel<T, PER><<<grd, blk, 0, L.stream>>>(u, o, L.src, L.ny, L.nx, L.c0, L.c1);
    } else {
        dim3 blk(32, 4, 2), grd(cdiv(L.nx, 32), cdiv(L.ny, 4), cdiv(L.nz, 2));
        if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
        naive3d_kernel<T, PER><<<grd, blk, 0, L.stream>>>(u, o, L.src, L.nz, L.ny, L.nx, L.c0,
                                                          L.c1);
    }
    return cudaGetLastError();
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
    if (cfg == 0) {
        if (L.dims == 2) {
            constexpr int W = 4, RB = 4;
            const int strips = cdiv(L.nx, 32);
            const int ych = L.chunk > 0 ? L.chunk
                                        : default_chunk(L.ny, cdiv(strips, W), 8 * RB, 2 * target);
            dim3 grd(cdiv(strips, W), cdiv(L.ny, ych));
            if (grd.y > 65535) return cudaErrorInvalidConfiguration;
            lite2d_kernel<T, PER, RB, W><<<grd, 32 * W, 0, L.stream>>>(u, o, L.src, L.ny, L.nx,
                                                                      L.c0, L.c1, ych);
        } else {
            constexpr int R = 4, W = 4;
            // planes zb .. ze-1 (a z range never wraps: its neighbour planes are in the array)
            const int zb = L.ze > 0 ? L.zb : 0, ze = L.ze > 0 ? L.ze : L.nz;
            const long long tiles = 1LL * cdiv(L.nx, 32) * cdiv(L.ny, W * R);
            const int zch = L.chunk > 0 ? L.chunk : default_chunk(ze - zb, tiles, 16, 2 * target);
            dim3 grd(cdiv(L.nx, 32), cdiv(L.ny, W * R), cdiv(ze - zb, zch));
            if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
            lite3d_kernel<T, PER, R, W><<<grd, 32 * W, 0, L.stream>>>(
                u, o, L.src, L.nz, L.ny, L.nx, L.c0, L.c1, zch, zb, ze);
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

template <typename T, bool PER, int K, int V, int R, int W>
static cudaError_t tb3d_t(const Launch& L) {
    constexpr int KX = ((K + V - 1) / V) * V, OX = 32 * V - 2 * KX, OY = W * R - 2 * K;
    const long long tiles = 1LL * cdiv(L.nx, OX) * cdiv(L.ny, OY);
    const int zch = L.chunk > 0 ? L.chunk
                                : default_chunk(L.nz, tiles, std::max(8, 4 * K), 4LL * sm_count());
    dim3 grd(cdiv(L.nx, OX), cdiv(L.ny, OY), cdiv(L.nz, zch));
    if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
    tb3d_kernel<T, PER, K, V, R, W><<<grd, 32 * W, 0, L.stream>>>(
        static_cast<const T*>(L.u), static_cast<T*>(L.out), L.src, L.nz, L.ny, L.nx, L.c0, L.c1,
        zch, vec_ok<T, PER, V>(L) ? 1 : 0);
    return cudaGetLastError();
}

template <typename T, bool PER, int K, int V, int W>
static cudaError_t tb2d_t(const Launch& L) {
    constexpr int KX = ((K + V - 1) / V) * V, OX = 32 * V - 2 * KX;
    const int strips = cdiv(L.nx, OX);
    const int ych = L.chunk > 0 ? L.chunk
                                : default_chunk(L.ny, cdiv(strips, W), std::max(16, 8 * K),
                                                8LL * sm_count());
    dim3 grd(cdiv(strips, W), cdiv(L.ny, ych));
    if (grd.y > 65535) return cudaErrorInvalidConfiguration;
    tb2d_kernel<T, PER, K, V, W><<<grd, 32 * W, 0, L.stream>>>(
        static_cast<const T*>(L.u), static_cast<T*>(L.out), L.src, L.ny, L.nx, L.c0, L.c1, ych,
        vec_ok<T, PER, V>(L) ? 1 : 0);
    return cudaGetLastError();
}

template <typename T, bool PER>
static cudaError_t tb_t(const Launch& L) {
    if (L.dims == 2) {
        switch (L.k) {
            case 2: return tb2d_t<T, PER, 2, 4, 4>(L);
            case 3: return tb2d_t<T, PER, 3, 4, 4>(L);
            case 4: return tb2d_t<T, PER, 4, 4, 4>(L);
            case 8: return tb2d_t<T, PER, 8, 4, 4>(L);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (L.k) {
        case 2: return tb3d_t<T, PER, 2, 4, 2, 16>(L);
        case 3: return tb3d_t<T, PER, 3, 4, 2, 16>(L);
        case 4: return tb3d_t<T, PER, 4, 2, 2, 16>(L);
        case 8: return tb3d_t<T, PER, 8, 2, 1, 32>(L);
        default: return cudaErrorInvalidValue;
    }
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

static cudaError_t launch_tb_plain(const Launch& L) { PH3_DISPATCH(tb_t, L); }

cudaError_t launch_tb(const Launch& L) {
    if (L.dims == 3 && tbbulk_supported(L)) return launch_tbbulk(L);
    return launch_tb_plain(L);
}

// 2D: 0 lean one-column-per-lane march, 1 float-window vector march, 2 / 3 / 4 raw-row vector
// march with 4 / 8 / 6 rows per step (shapes without whole 16-byte rows fall back to 1). 3D: 0 lean,
// 1 vector march, 2 / 3 any-alignment lane vectors with 4 / 2 rows per warp, 4 / 5 / 6 row boxes
// by 1D tensor copies into per-warp rings (rows per warp, ring stages: 2/3, 2/4, 4/3).
int march_configs(int dims, const char** names, int max) {
    static const char* k2[] = {"lane1_W4_RB4", "V16B_W4_RB4", "raw16B_W4_RB4", "raw16B_W4_RB8",
                               "raw16B_W4_RB6"};
    static const char* k3[] = {"lane1_R4_W4", "V16B_R2_W8", "V4any_R4_W4", "V4any_R2_W4",
                               "ring1d_R2_W4_S3", "ring1d_R2_W4_S4", "ring1d_R4_W4_S3"};
    const int n = dims == 2 ? 5 : 7;
    for (int i = 0; i < n && names != nullptr && i < max; ++i) names[i] = dims == 2 ? k2[i] : k3[i];
    return n;
}

int tb_configs(int dims, int k, const char** names, int max) {
    if (dims == 3) return tbbulk_configs(k, names, max);
    if (k != 2 && k != 3 && k != 4 && k != 8) return 0;
    if (names != nullptr && max > 0) names[0] = "V4_W4";
    return 1;
}

}  // namespace ph3
