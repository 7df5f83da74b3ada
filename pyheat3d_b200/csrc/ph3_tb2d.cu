// 2D temporal blocking: k fused updates per pass (sm_100a).
//
// Functional spec: pyheat3d src/pyheat3d/backends/stencil.cu:289-385 (tb2d) — k updates per DRAM
// pass over overlapped column strips; intermediate levels stay in fp32 and are rounded to the
// storage type once per pass (src/pyheat3d/validation.py:168-183 emulates this).
//
// Design for B200:
// * A work item is one column strip of EX = 32 lanes x V columns and one chunk of rows; strips
//   overlap by KX columns on each side (K rounded up to a 16-byte granule), so OX = EX - 2 KX
//   columns are stored. One warp owns one item; warps never wait for each other (no block
//   barrier anywhere in the kernel).
// * The wavefront advances TWO rows per iteration. Level 0 rows arrive as row pairs in a
//   per-warp shared-memory ring, filled by untiled cp.async.bulk copies that complete on the
//   stage's mbarrier. The row extent of a strip splits into the same contiguous pieces for every
//   row (at the periodic seam, or at the array edge for Dirichlet), so each lane owns at most
//   one piece, computed once per item, and a row pair is issued by one predicated copy per lane
//   and row.
// * Level s keeps one row pair in registers. In an iteration it produces the pair two rows
//   further on from its predecessor level's kept pair and new pair (four consecutive rows);
//   the new pair goes to the second of two register sets, and the two sets trade roles every
//   iteration (the loop body is the two iterations), so no row is ever copied.
// * Arithmetic in packed f32x2 (neighbour sums, products), the final c0*u + c1*S as scalar
//   non-contracting adds: bit-identical to the scalar canonical chain. x-neighbours across
//   lanes by two shuffles per row.
// * Rows without whole 16-byte vectors (or unaligned buffers) take the same wavefront with
//   level 0 loaded element by element from global memory (one pair ahead in registers).
// * Waits are bounded: an expired wait records the error in the status word, the warp stops
//   storing, waits (bounded) for the copies it issued and returns.
#include <algorithm>
#include <atomic>

#include "ph3_common.cuh"
#include "ph3_internal.h"
#include "ph3_tb2d.cuh"

namespace ph3 {

namespace {

struct T2Geom {
    int ny, nx;
    int nstrips;  // strips of OX stored columns
    int ych;      // rows per chunk
    int nitems;   // nstrips * chunks
};

template <typename T, bool PER, bool SRC, bool BULK, int K, int V, int STAGES, int W, int MINB>
__global__ void __launch_bounds__(32 * W, MINB)
tb2d_pair_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b,
                 T2Geom g, float c0, float c1, int* err) {
    using C = T2Cfg<T, K, V, STAGES>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int item = blockIdx.x * W + warp;
    if (item >= g.nitems) return;  // warp-uniform; the kernel has no block barrier
    T* ring = reinterpret_cast<T*>(smem + warp * C::RING_BYTES);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + W * C::RING_BYTES) + warp * STAGES;
    const int strip = item % g.nstrips, chunk = item / g.nstrips;
    const int y0 = chunk * g.ych, y1 = min(y0 + g.ych, g.ny);
    tb2d_pair_item<T, PER, SRC, BULK, K, V, STAGES>(u, o, b, g.ny, g.nx, strip, y0, y1, c0, c1,
                                                    err, ring, bar);
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

// Rows per chunk (even) minimising the critical path ceil(items / slots) * (pairs + k) over the
// warps resident at once.
int t2_chunk(int ny, int nstrips, long long slots, int k) {
    int best = ny + (ny & 1);
    double best_cost = 1e300;
    const int max_nch = std::max(1, ny / std::max(4 * k, 16));
    for (int nch = 1; nch <= max_nch; ++nch) {
        int ych = (ny + nch - 1) / nch;
        ych += ych & 1;
        const long long items = 1LL * nstrips * ((ny + ych - 1) / ych);
        const double waves = double((items + slots - 1) / slots);
        const double cost = waves * (ych / 2 + k);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = ych;
        }
    }
    return best;
}

template <typename T, bool PER, bool SRC, bool BULK, int K, int V, int STAGES, int W, int MINB>
cudaError_t t2_launch(const Launch& L) {
    using C = T2Cfg<T, K, V, STAGES>;
    auto kern = tb2d_pair_kernel<T, PER, SRC, BULK, K, V, STAGES, W, MINB>;
    constexpr int SMEM = BULK ? W * (C::RING_BYTES + STAGES * 8) : 0;
    static std::atomic<int> blocks_per_sm[64];  // per device; first calls may race harmlessly
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    int nbl = blocks_per_sm[dev].load(std::memory_order_acquire);
    if (nbl == 0) {
        if (SMEM > 48 * 1024) {
            cudaError_t e =
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
            if (e != cudaSuccess) return e;
        }
        int nb = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * W, SMEM);
        if (e != cudaSuccess) return e;
        nbl = std::max(1, nb);
        blocks_per_sm[dev].store(nbl, std::memory_order_release);
    }
    T2Geom g;
    g.ny = L.ny;
    g.nx = L.nx;
    g.nstrips = (L.nx + C::OX - 1) / C::OX;
    const long long slots = 1LL * sm_count() * nbl * W;
    g.ych = L.chunk > 0 ? std::min(L.chunk + (L.chunk & 1), L.ny + (L.ny & 1))
                        : t2_chunk(L.ny, g.nstrips, slots, K);
    const long long items = 1LL * g.nstrips * ((L.ny + g.ych - 1) / g.ych);
    if (items > (1LL << 30)) return cudaErrorInvalidValue;
    if (L.geo != nullptr) {
        L.geo[0] = C::EX; L.geo[1] = 1; L.geo[2] = g.ych;
        return cudaSuccess;
    }
    g.nitems = int(items);
    const int grid = int((items + W - 1) / W);
    kern<<<grid, 32 * W, SMEM, L.stream>>>(static_cast<const T*>(L.u), static_cast<T*>(L.out),
                                           L.src, g, L.c0, L.c1, L.err);
    return cudaGetLastError();
}

// Whole 16-byte rows, 16-byte aligned buffers and enough columns that a strip's row splits
// into fewer than 32 pieces (one per lane).
template <typename T, int V>
bool t2_bulk_ok(const Launch& L) {
    auto al = [](const void* p) { return p == nullptr || reinterpret_cast<uintptr_t>(p) % 16 == 0; };
    const int G = 16 / int(sizeof(T));
    return (size_t(L.nx) * sizeof(T)) % 16 == 0 && L.nx >= std::max(G, (32 * V) / 28 + 1) &&
           al(L.u) && al(L.out) && al(L.src);
}

// The Jacobi source is a compile-time choice: the kernel without it carries neither its loads
// nor the branches around them (the loop body stays small enough for the instruction cache).
template <typename T, bool PER, int K, int V, int STAGES, int W, int MINB>
cudaError_t t2_pick(const Launch& L) {
    const bool bulk = t2_bulk_ok<T, V>(L);
    if (L.src != nullptr)
        return bulk ? t2_launch<T, PER, true, true, K, V, STAGES, W, MINB>(L)
                    : t2_launch<T, PER, true, false, K, V, STAGES, W, MINB>(L);
    return bulk ? t2_launch<T, PER, false, true, K, V, STAGES, W, MINB>(L)
                : t2_launch<T, PER, false, false, K, V, STAGES, W, MINB>(L);
}

// Compiled configurations per k: values per lane (EX = 32 V) and the register budget of a
// thread (128: 16 resident warps per SM; 168: 12). 0 is the default for k <= 4, 1 for k = 8,
// where the kept row pairs of the eight levels need more than 128 registers.
constexpr int kT2Cfgs = 3;
const char* kT2Names[kT2Cfgs] = {"pair_V4_R128", "pair_V4_R168", "pair_V2_R128"};

template <typename T, bool PER, int K, int STAGES>
cudaError_t t2_cfg(const Launch& L) {
    const int cfg = L.cfg < 0 ? (K >= 8 ? 1 : 0) : L.cfg;
    switch (cfg) {
        case 1: return t2_pick<T, PER, K, 4, STAGES, 4, 3>(L);
        case 2: return t2_pick<T, PER, K, 2, STAGES, 4, 4>(L);
        default: return t2_pick<T, PER, K, 4, STAGES, 4, 4>(L);
    }
}

template <typename T, bool PER>
cudaError_t t2_dispatch(const Launch& L) {
    switch (L.k) {
        case 2: return t2_cfg<T, PER, 2, 6>(L);
        case 3: return t2_cfg<T, PER, 3, 6>(L);
        case 4: return t2_cfg<T, PER, 4, 6>(L);
        case 8: return t2_cfg<T, PER, 8, 4>(L);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int tb2d_configs(int k, const char** names, int max) {
    if (k != 2 && k != 3 && k != 4 && k != 8) return 0;
    for (int i = 0; i < kT2Cfgs && names != nullptr && i < max; ++i) names[i] = kT2Names[i];
    return kT2Cfgs;
}

cudaError_t launch_tb2d(const Launch& L) {
    switch (L.storage) {
        case kF32: return L.periodic ? t2_dispatch<float, true>(L) : t2_dispatch<float, false>(L);
        case kF16: return L.periodic ? t2_dispatch<__half, true>(L) : t2_dispatch<__half, false>(L);
        case kBF16:
            return L.periodic ? t2_dispatch<__nv_bfloat16, true>(L)
                              : t2_dispatch<__nv_bfloat16, false>(L);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ph3
