// Batched solves: many independent grids of uneven sizes advanced in ONE persistent launch.
//
// No counterpart in the reference (one launch per grid and step, cupy_backend.py:183-194). Each
// problem is cut into tiles (the single-step march tiles of ph3_march.cuh); a work item is
// (problem P, step s, tile t). Items are numbered round by round — round s holds step s of every
// problem that still has steps left, problems in descending step count — so every item's
// predecessors (all tiles of step s-1 of the same problem) come earlier in the numbering.
// Persistent blocks take items in order from a global counter, wait (bounded) until the
// problem's step counter reaches s * tiles, run the tile, and count it done. A block only ever
// waits for items handed out before its own, which are held by running blocks that never wait
// for later items, so the launch always makes progress.
//
// Tiles are the lean one-column-per-lane marches of ph3_march.cuh (any row alignment, no block
// barrier inside a tile). A 2D problem with k > 1 advances by passes of k fused steps instead:
// its items are (problem, pass, tile) and its tiles are eight warps of the 2D temporal-blocking
// wavefront (ph3_tb2d.cuh, element loads), one overlapped column strip and a chunk of rows per
// warp, followed by steps % k single-step passes over the same strips; the round numbering then
// counts passes. Field reads go through L2 only (__ldcg): other
// blocks of the same launch write the fields.
// The item list is implicit: a plan in device memory (problem descriptors, the problems sorted
// by steps, prefix sums of their tile counts and per-round item offsets) lets a block decode an
// item number with two binary searches.
//
// Workspace layout (caller-allocated device memory, ph3_batch_workspace_bytes):
//   [counters: u64 next item | i32 abort | i32 pad | u64 done[n]]  (rounded up to 256 bytes)
//   [header][descriptors][order (i32)][tile prefix (i64)][round offsets (i64)]
// The per-problem done counters are 64-bit: a problem counts steps x tiles completions, which
// exceeds 2^31 for a large grid run for many steps.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "../../include/ph3b200.h"
#include "ph3_common.cuh"
#include "ph3_internal.h"
#include "ph3_march.cuh"
#include "ph3_tb2d.cuh"
#include "ph3_tile3d.cuh"

namespace ph3 {

namespace {

struct BatchDesc {
    void* a;
    void* b;
    const float* src;
    int dims, nz, ny, nx, periodic, storage;
    float c0, c1;
    int steps;
    int k;       // fused steps per pass (1: single steps)
    int fused;   // leading passes of k fused steps: steps / k
    int passes;  // rounds this problem takes part in: steps / k, then steps % k single steps
    int ntx, nty, ntz, ntiles;
};

struct BatchHeader {
    int n;
    int max_steps;  // most passes of any problem (the number of rounds)
    int cfg;  // tile configuration the descriptors' tile counts were computed for
    int pad;
    long long total_items;
    long long off_desc, off_order, off_tilepre, off_round;
};

constexpr int kW = 8;  // warps per block
constexpr int kTbRows = 256;  // rows per chunk of a 2D temporal-blocking tile

// Lane widths of the batch's 2D temporal-blocking tiles (the batch kernel's register budget):
// k = 2 takes 4 values per lane, k = 4 takes 2. The x halo is whole 16-byte granules, one granule
// for every k up to 4 (and for the single-step remainder passes, which therefore cut a problem
// into the same strips as its fused passes).
template <int K> struct TbLane { static constexpr int V = K == 2 ? 4 : 2; };
template <typename T, int K>
__host__ __device__ constexpr int tb_strip_width() {  // stored columns per strip
    return 32 * TbLane<K>::V - 2 * (((K + 16 / int(sizeof(T)) - 1) / (16 / int(sizeof(T)))) *
                                    (16 / int(sizeof(T))));
}
static_assert(T2Cfg<float, 1, 4, 2>::OX == tb_strip_width<float, 2>() &&
                  T2Cfg<float, 1, 2, 2>::OX == tb_strip_width<float, 4>() &&
                  T2Cfg<__half, 1, 4, 2>::OX == tb_strip_width<__half, 2>() &&
                  T2Cfg<__half, 1, 2, 2>::OX == tb_strip_width<__half, 4>(),
              "remainder passes must cut the same strips as the fused passes");

// Compiled tile configurations (the tuning table's batch family): rows per warp and planes per
// 3D tile, rows per iteration and rows per 2D tile. The plan records which one it was built for.
// S3: 3D tiles are the block-wide shared-memory plane tiles of ph3_tile3d.cuh (64 x 32 columns)
// instead of one lean march per warp (32 columns x 8 R rows).
template <int CFG> struct BCfg;
template <> struct BCfg<0> { static constexpr int R = 4, ZCH = 32, RB2 = 4, YCH = 128; static constexpr bool S3 = false; };
template <> struct BCfg<1> { static constexpr int R = 2, ZCH = 16, RB2 = 4, YCH = 64; static constexpr bool S3 = false; };
template <> struct BCfg<2> { static constexpr int R = 8, ZCH = 64, RB2 = 8, YCH = 256; static constexpr bool S3 = false; };
template <> struct BCfg<3> { static constexpr int R = 4, ZCH = 256, RB2 = 8, YCH = 256; static constexpr bool S3 = true; };
template <> struct BCfg<4> { static constexpr int R = 4, ZCH = 128, RB2 = 8, YCH = 256; static constexpr bool S3 = true; };
template <> struct BCfg<5> { static constexpr int R = 4, ZCH = 64, RB2 = 8, YCH = 256; static constexpr bool S3 = true; };
// Configurations kBatchTiles .. 2 kBatchTiles - 1 are the same tile sets with the kernel compiled
// for two blocks per SM instead of three (128 registers per thread instead of 80: the tile bodies
// no longer spill).
constexpr int kBatchTiles = 6;
constexpr int kBatchCfgs = 2 * kBatchTiles;
const char* kBatchNames[kBatchCfgs] = {
    "R4_Z32_Y128",    "R2_Z16_Y64",    "R8_Z64_Y256",    "S64x32_Z256_Y256",   "S64x32_Z128_Y256",
    "S64x32_Z64_Y256", "R4_Z32_Y128_B2", "R2_Z16_Y64_B2", "R8_Z64_Y256_B2", "S64x32_Z256_Y256_B2",
    "S64x32_Z128_Y256_B2", "S64x32_Z64_Y256_B2"};

// shared-memory plane ring of the 3D tiles of tile sets with S3 (one per block)
__shared__ __align__(16) float g_tile_sm[Tile3::SMEM / 4];

struct Geo { int R, ZCH, YCH; bool S3; };
template <int CFG> Geo geo_t() { return {BCfg<CFG>::R, BCfg<CFG>::ZCH, BCfg<CFG>::YCH, BCfg<CFG>::S3}; }
Geo geo_of(int cfg) {
    switch (cfg) {
        case 1: return geo_t<1>();
        case 2: return geo_t<2>();
        case 3: return geo_t<3>();
        case 4: return geo_t<4>();
        case 5: return geo_t<5>();
        default: return geo_t<0>();
    }
}
constexpr int kThreads = 32 * kW;
constexpr int kSmemTilePre = 1024;  // tile prefix sums kept in shared memory (n < 1024)
static_assert(Tile3::W == kW, "3D plane tiles take the whole block");

__host__ __device__ __forceinline__ long long counter_bytes(int n) {
    return ((16LL + 8LL * n + 255) / 256) * 256;
}
long long align256(long long x) { return ((x + 255) / 256) * 256; }

// Not inlined: each tile body (storage, boundary, tile shape, with or without a Jacobi source)
// keeps its own register allocation instead of the kernel carrying the union of all of them.
template <typename T, bool PER, int ZCH, bool SRC>
__device__ __noinline__ void run_plane_tile3(const BatchDesc& d, int s, int t) {
    const T* src = static_cast<const T*>((s & 1) ? d.b : d.a);
    T* dst = static_cast<T*>((s & 1) ? d.a : d.b);
    const int tx = t % d.ntx, ty = (t / d.ntx) % d.nty, tz = t / (d.ntx * d.nty);
    const int z0 = tz * ZCH, z1 = min(z0 + ZCH, d.nz);
    tile3d_item<T, PER, SRC, true>(src, dst, SRC ? d.src : nullptr, d.nz, d.ny, d.nx, d.c0, d.c1,
                                   tx, ty, z0, z1, g_tile_sm);
}

template <typename T, bool PER, int R, int ZCH, bool SRC>
__device__ __noinline__ void run_lean_tile3(const BatchDesc& d, int s, int t) {
    const T* src = static_cast<const T*>((s & 1) ? d.b : d.a);
    T* dst = static_cast<T*>((s & 1) ? d.a : d.b);
    const int w = threadIdx.x >> 5;
    const int tx = t % d.ntx, ty = (t / d.ntx) % d.nty, tz = t / (d.ntx * d.nty);
    const int z0 = tz * ZCH, z1 = min(z0 + ZCH, d.nz), y0 = (ty * kW + w) * R;
    lite3d_item<T, PER, R, true, SRC>(src, dst, SRC ? d.src : nullptr, d.nz, d.ny, d.nx, d.c0,
                                      d.c1, tx, y0, z0, z1);
}

template <typename T, bool PER, int RB2, int YCH, bool SRC>
__device__ __noinline__ void run_lean_tile2(const BatchDesc& d, int s, int t) {
    const T* src = static_cast<const T*>((s & 1) ? d.b : d.a);
    T* dst = static_cast<T*>((s & 1) ? d.a : d.b);
    const int w = threadIdx.x >> 5;
    const int tx = t % d.ntx, ty = t / d.ntx;
    const int y0 = ty * YCH, y1 = min(y0 + YCH, d.ny);
    lite2d_item<T, PER, RB2, true, SRC>(src, dst, SRC ? d.src : nullptr, d.ny, d.nx, d.c0, d.c1,
                                        tx * kW + w, y0, y1);
}

// problems without a Jacobi source take tiles compiled without it
template <typename T, bool PER, int CFG>
__device__ __forceinline__ void run_tile(const BatchDesc& d, int s, int t) {
    using C = BCfg<CFG>;
    const bool src = d.src != nullptr;
    if (d.dims == 3 && C::S3) {
        if (src) run_plane_tile3<T, PER, C::ZCH, true>(d, s, t);
        else run_plane_tile3<T, PER, C::ZCH, false>(d, s, t);
    } else if (d.dims == 3) {
        if (src) run_lean_tile3<T, PER, C::R, C::ZCH, true>(d, s, t);
        else run_lean_tile3<T, PER, C::R, C::ZCH, false>(d, s, t);
    } else {
        if (src) run_lean_tile2<T, PER, C::RB2, C::YCH, true>(d, s, t);
        else run_lean_tile2<T, PER, C::RB2, C::YCH, false>(d, s, t);
    }
}

// One item of a 2D problem with temporal blocking: eight strips (one per warp) of one chunk of
// rows, pass s from buffer s % 2 into the other. KP fused steps in this pass (k, or 1 for the
// remainder passes), lanes V wide as the problem's k sets.
template <typename T, bool PER, int KP, int V, int KPROB>
__device__ __noinline__ void run_tb2d_tile(const BatchDesc& d, int s, int t) {
    const T* src = static_cast<const T*>((s & 1) ? d.b : d.a);
    T* dst = static_cast<T*>((s & 1) ? d.a : d.b);
    const int w = threadIdx.x >> 5;
    const int tx = t % d.ntx, ty = t / d.ntx;
    const int strip = tx * kW + w;
    constexpr int OX = tb_strip_width<T, KPROB>();
    const int nstrips = (d.nx + OX - 1) / OX;
    if (strip >= nstrips) return;  // warp-uniform
    const int y0 = ty * kTbRows, y1 = min(y0 + kTbRows, d.ny);
    if (d.src != nullptr)
        tb2d_pair_item<T, PER, true, false, KP, V, 2, true>(src, dst, d.src, d.ny, d.nx, strip, y0,
                                                           y1, d.c0, d.c1, nullptr, nullptr,
                                                           nullptr);
    else
        tb2d_pair_item<T, PER, false, false, KP, V, 2, true>(src, dst, nullptr, d.ny, d.nx, strip,
                                                            y0, y1, d.c0, d.c1, nullptr, nullptr,
                                                            nullptr);
}

template <typename T, bool PER, int CFG>
__device__ __forceinline__ void run_problem_tile(const BatchDesc& d, int s, int t) {
    if (d.k == 2) {
        if (s < d.fused) run_tb2d_tile<T, PER, 2, TbLane<2>::V, 2>(d, s, t);
        else run_tb2d_tile<T, PER, 1, TbLane<2>::V, 2>(d, s, t);
    } else if (d.k == 4) {
        if (s < d.fused) run_tb2d_tile<T, PER, 4, TbLane<4>::V, 4>(d, s, t);
        else run_tb2d_tile<T, PER, 1, TbLane<4>::V, 4>(d, s, t);
    } else {
        run_tile<T, PER, CFG>(d, s, t);
    }
}

template <int CFG>
__device__ __forceinline__ void run_any(const BatchDesc& d, int s, int t) {
    switch (d.storage * 2 + d.periodic) {
        case 0: run_problem_tile<float, false, CFG>(d, s, t); break;
        case 1: run_problem_tile<float, true, CFG>(d, s, t); break;
        case 2: run_problem_tile<__half, false, CFG>(d, s, t); break;
        case 3: run_problem_tile<__half, true, CFG>(d, s, t); break;
        case 4: run_problem_tile<__nv_bfloat16, false, CFG>(d, s, t); break;
        default: run_problem_tile<__nv_bfloat16, true, CFG>(d, s, t); break;
    }
}

__device__ __forceinline__ long long upper_bound_i64(const long long* a, int n, long long key) {
    int lo = 0, hi = n;  // first index with a[i] > key
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
batch_kernel(unsigned char* __restrict__ ws, int n, int* err) {
    __shared__ int s_p, s_s, s_t;
    __shared__ long long s_item;
    unsigned long long* next = reinterpret_cast<unsigned long long*>(ws);
    int* abort_flag = reinterpret_cast<int*>(ws + 8);
    unsigned long long* done = reinterpret_cast<unsigned long long*>(ws + 16);
    const BatchHeader* hd = reinterpret_cast<const BatchHeader*>(ws + counter_bytes(n));
    const unsigned char* base = reinterpret_cast<const unsigned char*>(hd);
    const BatchDesc* desc = reinterpret_cast<const BatchDesc*>(base + hd->off_desc);
    const int* order = reinterpret_cast<const int*>(base + hd->off_order);
    const long long* tilepre = reinterpret_cast<const long long*>(base + hd->off_tilepre);
    const long long* round_off = reinterpret_cast<const long long*>(base + hd->off_round);
    const long long total = hd->total_items;
    const int max_steps = hd->max_steps;
    const int cfg = hd->cfg % kBatchTiles;
    // the tile prefix sums of short problem lists live in shared memory for the item decode
    __shared__ long long s_tilepre[kSmemTilePre];
    const bool tp_shared = n + 1 <= kSmemTilePre;
    if (tp_shared)
        for (int i = threadIdx.x; i <= n; i += blockDim.x) s_tilepre[i] = tilepre[i];
    __syncthreads();
    const long long* tp = tp_shared ? s_tilepre : tilepre;
    int s_prev = 0;  // thread 0: round of its previous item (a block's items only increase)

    for (;;) {
        if (threadIdx.x == 0) {
            long long item = static_cast<long long>(atomicAdd(next, 1ULL));
            if (item >= total || *reinterpret_cast<volatile int*>(abort_flag) != 0) {
                item = -1;
            } else {
                int s = s_prev;  // round_off[s] <= item; most items stay in the same round
                if (round_off[s + 1] <= item)
                    s += int(upper_bound_i64(round_off + s, max_steps + 1 - s, item)) - 1;
                s_prev = s;
                const long long j = item - round_off[s];
                const int q = int(upper_bound_i64(tp, n + 1, j)) - 1;
                const int p = order[q];
                s_p = p;
                s_s = s;
                s_t = int(j - tp[q]);
                const unsigned long long need =
                    static_cast<unsigned long long>(s) * static_cast<unsigned long long>(desc[p].ntiles);
                if (!wait_u64_geq(&done[p], need, kSpinLimit, err, abort_flag)) {
                    atomicExch(abort_flag, 1);
                    item = -1;
                }
                __threadfence();
            }
            s_item = item;
        }
        __syncthreads();
        if (s_item < 0) break;
        const BatchDesc d = desc[s_p];
        const int s = s_s, t = s_t;
        switch (cfg) {
            case 1: run_any<1>(d, s, t); break;
            case 2: run_any<2>(d, s, t); break;
            case 3: run_any<3>(d, s, t); break;
            case 4: run_any<4>(d, s, t); break;
            case 5: run_any<5>(d, s, t); break;
            default: run_any<0>(d, s, t); break;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&done[s_p], 1ULL);
        }
    }
}

template <int MINB>
int blocks_per_sm_cached() {
    // per device; concurrent first calls may both query, and store the same value atomically
    static std::atomic<int> nb[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
    int v = nb[dev].load(std::memory_order_acquire);
    if (v == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, batch_kernel<MINB>, kThreads, 0) !=
                cudaSuccess ||
            v < 1)
            v = 1;
        nb[dev].store(v, std::memory_order_release);
    }
    return v;
}

int cdiv(long long a, long long b) { return int((a + b - 1) / b); }

// Geometry of one problem's tiles (must match run_tile / the item functions).
void tiles_of(BatchDesc& d, int cfg) {
    const Geo g = geo_of(cfg % kBatchTiles);
    d.k = d.k > 1 ? d.k : 1;
    d.fused = d.steps / d.k;
    d.passes = d.fused + d.steps % d.k;
    if (d.k > 1) {  // 2D temporal blocking: eight strips x one row chunk per item
        int ox = 0;
        const bool wide = d.storage == kF32;
        if (d.k == 2) ox = wide ? tb_strip_width<float, 2>() : tb_strip_width<__half, 2>();
        else ox = wide ? tb_strip_width<float, 4>() : tb_strip_width<__half, 4>();
        d.ntx = cdiv(cdiv(d.nx, ox), kW);
        d.nty = cdiv(d.ny, kTbRows);
        d.ntz = 1;
        d.ntiles = d.ntx * d.nty;
        return;
    }
    if (d.dims == 3 && g.S3) {
        d.ntx = cdiv(d.nx, Tile3::OX);
        d.nty = cdiv(d.ny, Tile3::OY);
        d.ntz = cdiv(d.nz, g.ZCH);
    } else if (d.dims == 3) {
        d.ntx = cdiv(d.nx, 32);
        d.nty = cdiv(d.ny, kW * g.R);
        d.ntz = cdiv(d.nz, g.ZCH);
    } else {
        d.ntx = cdiv(cdiv(d.nx, 32), kW);
        d.nty = cdiv(d.ny, g.YCH);
        d.ntz = 1;
    }
    d.ntiles = d.ntx * d.nty * d.ntz;
}

struct Layout {
    long long cnt, header, desc, order, tilepre, round, total;
};

Layout layout_of(int n, int max_steps) {
    Layout L;
    L.cnt = counter_bytes(n);
    L.header = L.cnt;
    L.desc = align256(sizeof(BatchHeader));
    L.order = L.desc + align256(sizeof(BatchDesc) * (long long)n);
    L.tilepre = L.order + align256(4LL * n);
    L.round = L.tilepre + align256(8LL * (n + 1));
    L.total = L.cnt + L.round + align256(8LL * (max_steps + 1));
    return L;
}

}  // namespace

// -------------------------------------------------------------------------------- host API
cudaError_t batch_launch(void* ws, int n, int* err, cudaStream_t stream, int cfg);

// Passes of a problem: its steps, or steps / k fused passes and steps % k single steps.
int passes_of(const ph3_problem& p) {
    return p.k > 1 ? p.steps / p.k + p.steps % p.k : p.steps;
}

long long batch_workspace_bytes(const ph3_problem* p, int n) {
    int max_steps = 0;
    for (int i = 0; i < n; ++i) max_steps = std::max(max_steps, passes_of(p[i]));
    return layout_of(n, max_steps).total;
}

cudaError_t batch_prepare(const ph3_problem* p, int n, void* ws, long long ws_bytes,
                          cudaStream_t stream, long long* total_items, int cfg) {
    if (cfg < 0 || cfg >= kBatchCfgs) cfg = 0;
    std::vector<BatchDesc> d(n);
    int max_steps = 0;
    for (int i = 0; i < n; ++i) {
        BatchDesc& x = d[i];
        x.a = p[i].a; x.b = p[i].b; x.src = p[i].src;
        x.dims = p[i].dims; x.nz = p[i].dims == 2 ? 1 : p[i].nz; x.ny = p[i].ny; x.nx = p[i].nx;
        x.periodic = p[i].bc == PH3_PERIODIC ? 1 : 0;
        x.storage = p[i].storage;
        x.c0 = p[i].c0; x.c1 = p[i].c1;
        x.steps = p[i].steps;
        x.k = p[i].k;
        tiles_of(x, cfg);
        max_steps = std::max(max_steps, x.passes);
    }
    const Layout L = layout_of(n, max_steps);
    if (ws_bytes < L.total) return cudaErrorInvalidValue;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return d[a].passes > d[b].passes; });
    std::vector<long long> tilepre(n + 1, 0);
    for (int q = 0; q < n; ++q) tilepre[q + 1] = tilepre[q] + d[order[q]].ntiles;
    std::vector<long long> round(max_steps + 1, 0);
    int active = n;
    for (int s = 0; s < max_steps; ++s) {
        while (active > 0 && d[order[active - 1]].passes <= s) --active;
        round[s + 1] = round[s] + tilepre[active];
    }
    BatchHeader h;
    h.n = n;
    h.max_steps = max_steps;
    h.cfg = cfg;
    h.pad = 0;
    h.total_items = round[max_steps];
    h.off_desc = L.desc;
    h.off_order = L.order;
    h.off_tilepre = L.tilepre;
    h.off_round = L.round;
    std::vector<unsigned char> img(L.total - L.header, 0);
    std::memcpy(img.data(), &h, sizeof(h));
    std::memcpy(img.data() + L.desc, d.data(), sizeof(BatchDesc) * n);
    std::memcpy(img.data() + L.order, order.data(), 4 * n);
    std::memcpy(img.data() + L.tilepre, tilepre.data(), 8 * (n + 1));
    std::memcpy(img.data() + L.round, round.data(), 8 * (max_steps + 1));
    cudaError_t e = cudaMemcpyAsync(static_cast<unsigned char*>(ws) + L.header, img.data(),
                                    img.size(), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);  // the staging image is freed on return
    if (total_items != nullptr) *total_items = h.total_items;
    return e;
}

// ---------------------------------------------------------------------------------------------
// Allocation-free variant (ph3_batch_run_static). Some hosts cannot allocate device memory at
// the point where they want to run a batch: a serving loop that must not allocate once it is in
// steady state (an allocation can synchronise the device or fail under memory pressure), or a
// foreign host (Go, Java, a plugin) that hands over field buffers but owns no CUDA allocator.
// For them the plan and counters live in this file-scope device array: 1 MiB on every GPU that
// loads the library, held until the process exits. Every call shares it, so calls that overlap
// on the GPU (two streams, two host threads) race and must be serialised by the caller; the
// counters are cleared on every call, the plan is rewritten on every call.
// ---------------------------------------------------------------------------------------------
constexpr long long kStaticWsBytes = 1LL << 20;
static __device__ __align__(256) unsigned char g_static_ws[kStaticWsBytes];

namespace {

std::mutex g_static_mu;                          // serialises the host-side plan image
unsigned char g_static_img[kStaticWsBytes];      // host staging of the plan (no heap use)

// Device address of g_static_ws on the current device, looked up once per device.
// Concurrent first calls on one device may both look it up; they store the same address
// atomically.
unsigned char* static_ws_device(cudaError_t* err) {
    static std::atomic<unsigned char*> ptrs[64];
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= 64) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    unsigned char* ptr = ptrs[dev].load(std::memory_order_acquire);
    if (ptr == nullptr) {
        void* p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_static_ws);
        if (*err != cudaSuccess) return nullptr;
        ptr = static_cast<unsigned char*>(p);
        ptrs[dev].store(ptr, std::memory_order_release);
    }
    return ptr;
}

}  // namespace

long long batch_static_capacity() { return kStaticWsBytes; }

int batch_configs(const char** names, int max) {
    for (int i = 0; i < kBatchCfgs && names != nullptr && i < max; ++i) names[i] = kBatchNames[i];
    return kBatchCfgs;
}

cudaError_t batch_run_static(const ph3_problem* p, int n, int* err, cudaStream_t stream,
                             long long* need_bytes, int cfg) {
    if (cfg < 0 || cfg >= kBatchCfgs) cfg = 0;
    int max_steps = 0;
    for (int i = 0; i < n; ++i) max_steps = std::max(max_steps, passes_of(p[i]));
    const Layout L = layout_of(n, max_steps);
    if (need_bytes != nullptr) *need_bytes = L.total;
    if (L.total > kStaticWsBytes) return cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    unsigned char* ws = static_ws_device(&e);
    if (ws == nullptr) return e;
    std::lock_guard<std::mutex> lk(g_static_mu);
    unsigned char* img = g_static_img;
    std::memset(img, 0, size_t(L.total - L.header));
    BatchDesc* d = reinterpret_cast<BatchDesc*>(img + L.desc);
    for (int i = 0; i < n; ++i) {
        BatchDesc& x = d[i];
        x.a = p[i].a; x.b = p[i].b; x.src = p[i].src;
        x.dims = p[i].dims; x.nz = p[i].dims == 2 ? 1 : p[i].nz; x.ny = p[i].ny; x.nx = p[i].nx;
        x.periodic = p[i].bc == PH3_PERIODIC ? 1 : 0;
        x.storage = p[i].storage;
        x.c0 = p[i].c0; x.c1 = p[i].c1;
        x.steps = p[i].steps;
        x.k = p[i].k;
        tiles_of(x, cfg);
    }
    int* order = reinterpret_cast<int*>(img + L.order);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order, order + n, [&](int a, int b) {
        return d[a].passes != d[b].passes ? d[a].passes > d[b].passes : a < b;
    });
    long long* tilepre = reinterpret_cast<long long*>(img + L.tilepre);
    tilepre[0] = 0;
    for (int q = 0; q < n; ++q) tilepre[q + 1] = tilepre[q] + d[order[q]].ntiles;
    long long* round = reinterpret_cast<long long*>(img + L.round);
    round[0] = 0;
    int active = n;
    for (int s = 0; s < max_steps; ++s) {
        while (active > 0 && d[order[active - 1]].passes <= s) --active;
        round[s + 1] = round[s] + tilepre[active];
    }
    BatchHeader* h = reinterpret_cast<BatchHeader*>(img);
    h->n = n;
    h->max_steps = max_steps;
    h->cfg = cfg;
    h->total_items = round[max_steps];
    h->off_desc = L.desc;
    h->off_order = L.order;
    h->off_tilepre = L.tilepre;
    h->off_round = L.round;
    e = cudaMemcpyAsync(ws + L.header, img, size_t(L.total - L.header), cudaMemcpyHostToDevice,
                        stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);  // the staging image is reused by the next call
    if (e != cudaSuccess) return e;
    return batch_launch(ws, n, err, stream, cfg);
}

cudaError_t batch_launch(void* ws, int n, int* err, cudaStream_t stream, int cfg) {
    cudaError_t e = cudaMemsetAsync(ws, 0, counter_bytes(n), stream);
    if (e != cudaSuccess) return e;
    unsigned char* w = static_cast<unsigned char*>(ws);
    if (cfg >= kBatchTiles) {
        batch_kernel<2><<<sm_count() * blocks_per_sm_cached<2>(), kThreads, 0, stream>>>(w, n, err);
    } else {
        batch_kernel<3><<<sm_count() * blocks_per_sm_cached<3>(), kThreads, 0, stream>>>(w, n, err);
    }
    return cudaGetLastError();
}

}  // namespace ph3
