// 3D temporal blocking for grids whose rows are not whole 16-byte vectors (sm_100a).
//
// Functional spec: pyheat3d src/pyheat3d/backends/stencil.cu:178-281 (tb3d) — k updates per DRAM
// pass by a (z, t) wavefront over overlapped xy tiles; intermediate levels stay in fp32 and are
// rounded to the storage type once per pass (src/pyheat3d/validation.py:168-183).
//
// Design: every level lives in shared memory. A block owns an extended EX x EY tile and one
// chunk of planes; level s (0 .. k-1) keeps its three most recent planes of the tile in a
// shared-memory ring of fp32 planes. Per step of the march the block
//   1. stores level-0 plane iz (loaded element by element from global memory one plane ahead,
//      so any row alignment works; periodic wrap / Dirichlet clamp per element),
//   2. for s = 1 .. k computes plane iz - s of level s from level s-1's planes iz-s-1 .. iz-s+1,
//      every thread a fixed set of sites, x- and y-neighbours read from the same plane in
//      shared memory (consecutive lanes read consecutive words: no bank conflicts),
//   3. writes level k's plane to global memory, stored region only.
// A block barrier separates the levels. The valid region shrinks by one site per level on
// every side; sites near the tile edge compute from stale neighbours and are never stored.
// Aligned grids take the bulk-copy register wavefront (ph3_tbbulk.cu) instead; this kernel
// trades speed for generality.
#include <algorithm>
#include <atomic>

#include "ph3_common.cuh"
#include "ph3_internal.h"

namespace ph3 {

namespace {

struct TsGeom {
    int nz, ny, nx;
    int ntx, nty;  // tiles of OX x OY stored sites
    int zch;       // planes per chunk
    int nitems;
};

template <int K, int EX, int EY>
struct TsCfg {
    static constexpr int OX = EX - 2 * K, OY = EY - 2 * K;
    static constexpr int THREADS = 256;
    static constexpr int PLANE = EX * EY;             // fp32 words per plane
    static constexpr int SITES = PLANE / THREADS;     // sites per thread and plane
    static constexpr int SMEM = K * 3 * PLANE * 4;    // level planes 0 .. k-1, three each
    static_assert(EX % 32 == 0 && PLANE % THREADS == 0 && OX > 0 && OY > 0, "tile shape");
};

template <typename T, bool PER, int K, int EX, int EY>
__global__ void __launch_bounds__(256)
tb3d_planes_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b,
                   TsGeom g, float c0, float c1) {
    using C = TsCfg<K, EX, EY>;
    constexpr int PLANE = C::PLANE, SITES = C::SITES;
    extern __shared__ __align__(16) float lv[];  // [level][slot][EY][EX]
    const int item = blockIdx.x;
    const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty, ch = item / (g.ntx * g.nty);
    const int xs = tx * C::OX - K, ys = ty * C::OY - K;
    const int z0 = ch * g.zch, z1 = min(z0 + g.zch, g.nz);
    const int64_t P = int64_t(g.nx) * g.ny;

    // this thread's sites: index i = threadIdx.x + j * THREADS over the EY x EX tile
    int off[SITES];      // global row-column offset (wrapped / clamped) of the site
    uint32_t inner = 0;  // bit j: not on the tile edge (has all four in-plane neighbours)
    uint32_t fixed = 0;  // bit j: Dirichlet boundary column / row (keeps its value)
    uint32_t store = 0;  // bit j: in the stored region and inside the domain
#pragma unroll
    for (int j = 0; j < SITES; ++j) {
        const int i = threadIdx.x + j * C::THREADS;
        const int ly = i / EX, lx = i % EX;
        const int gy = ys + ly, gx = xs + lx;
        const int wy = PER ? wrap_near(gy, g.ny) : clamp_idx(gy, 0, g.ny - 1);
        const int wx = PER ? wrap_near(gx, g.nx) : clamp_idx(gx, 0, g.nx - 1);
        off[j] = wy * g.nx + wx;
        if (lx > 0 && lx < EX - 1 && ly > 0 && ly < EY - 1) inner |= 1u << j;
        if (!PER && (gy <= 0 || gy >= g.ny - 1 || gx <= 0 || gx >= g.nx - 1)) fixed |= 1u << j;
        if (lx >= K && lx < K + C::OX && ly >= K && ly < K + C::OY && gx < g.nx && gy < g.ny &&
            !((fixed >> j) & 1u))
            store |= 1u << j;
    }
    auto plane_ptr = [&](int lev, int c) { return lv + (lev * 3 + ((c % 3) + 3) % 3) * PLANE; };
    auto wz = [&](int z) { return PER ? wrap_near(z, g.nz) : clamp_idx(z, 0, g.nz - 1); };

    float pre[SITES];
    auto load = [&](int z) {
        const T* pl = u + int64_t(wz(z)) * P;
#pragma unroll
        for (int j = 0; j < SITES; ++j) pre[j] = ldg1(pl + off[j]);
    };
    load(z0 - K);

    for (int iz = z0 - K; iz < z1 + K; ++iz) {
        float* l0 = plane_ptr(0, iz);
#pragma unroll
        for (int j = 0; j < SITES; ++j) l0[threadIdx.x + j * C::THREADS] = pre[j];
        if (iz + 1 < z1 + K) load(iz + 1);
        __syncthreads();
#pragma unroll
        for (int s = 1; s <= K; ++s) {
            const int c = iz - s;
            const float* dn = plane_ptr(s - 1, c - 1);
            const float* md = plane_ptr(s - 1, c);
            const float* up = plane_ptr(s - 1, c + 1);
            const bool zfix = !PER && (c <= 0 || c >= g.nz - 1);
            const float* bpl = b != nullptr ? b + int64_t(wz(c)) * P : nullptr;
            const bool out_plane = s == K && c >= z0 && c < z1;
            float* dst = s < K ? plane_ptr(s, c) : nullptr;
#pragma unroll
            for (int j = 0; j < SITES; ++j) {
                if (!((inner >> j) & 1u)) continue;
                const int i = threadIdx.x + j * C::THREADS;
                const float ctr = md[i];
                float v = upd3(c0, c1, ctr, md[i - 1], md[i + 1], md[i - EX], md[i + EX], dn[i],
                               up[i]);
                if (bpl != nullptr) v = __fadd_rn(v, __ldg(bpl + off[j]));
                if (zfix || ((fixed >> j) & 1u)) v = ctr;
                if (s < K) {
                    dst[i] = v;
                } else if (out_plane && ((store >> j) & 1u) && !zfix) {
                    o[int64_t(c) * P + off[j]] = from_f<T>(v);
                }
            }
            __syncthreads();
        }
    }
}

template <typename T, bool PER, int K, int EX, int EY>
cudaError_t ts_launch(const Launch& L) {
    using C = TsCfg<K, EX, EY>;
    auto kern = tb3d_planes_kernel<T, PER, K, EX, EY>;
    static std::atomic<int> blocks_per_sm[64];  // per device; first calls may race harmlessly
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    int nbl = blocks_per_sm[dev].load(std::memory_order_acquire);
    if (nbl == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             C::SMEM);
        if (e != cudaSuccess) return e;
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, C::THREADS, C::SMEM);
        if (e != cudaSuccess) return e;
        if (nb < 1) return cudaErrorInvalidConfiguration;
        nbl = nb;
        blocks_per_sm[dev].store(nbl, std::memory_order_release);
    }
    if (int64_t(L.nx) * L.ny >= (int64_t(1) << 31)) return cudaErrorInvalidValue;  // int offsets
    TsGeom g;
    g.nz = L.nz; g.ny = L.ny; g.nx = L.nx;
    g.ntx = (L.nx + C::OX - 1) / C::OX;
    g.nty = (L.ny + C::OY - 1) / C::OY;
    const long long tiles = 1LL * g.ntx * g.nty;
    const long long slots = 1LL * sm_count() * nbl;
    g.zch = L.chunk > 0 ? std::min(L.chunk, L.nz)
                        : default_chunk(L.nz, tiles, std::max(8, 4 * K), 2 * slots);
    const long long items = tiles * ((L.nz + g.zch - 1) / g.zch);
    if (items > (1LL << 31) - 1) return cudaErrorInvalidValue;
    g.nitems = int(items);
    if (L.geo != nullptr) {
        L.geo[0] = EX; L.geo[1] = EY; L.geo[2] = g.zch;
        return cudaSuccess;
    }
    kern<<<int(items), C::THREADS, C::SMEM, L.stream>>>(
        static_cast<const T*>(L.u), static_cast<T*>(L.out), L.src, g, L.c0, L.c1);
    return cudaGetLastError();
}

template <typename T, bool PER>
cudaError_t ts_dispatch(const Launch& L) {
    switch (L.k) {
        case 2: return ts_launch<T, PER, 2, 64, 32>(L);
        case 3: return ts_launch<T, PER, 3, 64, 32>(L);
        case 4: return ts_launch<T, PER, 4, 64, 32>(L);
        case 8: return ts_launch<T, PER, 8, 64, 32>(L);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_tb3d_planes(const Launch& L) {
    switch (L.storage) {
        case kF32: return L.periodic ? ts_dispatch<float, true>(L) : ts_dispatch<float, false>(L);
        case kF16: return L.periodic ? ts_dispatch<__half, true>(L) : ts_dispatch<__half, false>(L);
        case kBF16:
            return L.periodic ? ts_dispatch<__nv_bfloat16, true>(L)
                              : ts_dispatch<__nv_bfloat16, false>(L);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ph3
