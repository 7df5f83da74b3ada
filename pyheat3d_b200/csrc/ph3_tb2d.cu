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

namespace ph3 {

namespace {

constexpr unsigned kAll = 0xffffffffu;

struct T2Geom {
    int ny, nx;
    int nstrips;  // strips of OX stored columns
    int ych;      // rows per chunk
    int nitems;   // nstrips * chunks
};

template <typename T, int K, int V, int STAGES>
struct T2Cfg {
    static constexpr int G = 16 / int(sizeof(T));     // 16-byte granule in elements
    static constexpr int KX = ((K + G - 1) / G) * G;  // x halo, whole granules
    static constexpr int EX = 32 * V, OX = EX - 2 * KX;
    static constexpr int NP = V / 2;
    static constexpr int ROW_BYTES = EX * int(sizeof(T));
    static constexpr int STAGE_BYTES = 2 * ROW_BYTES;
    static constexpr int RING_BYTES = STAGES * STAGE_BYTES;  // per warp
    static_assert(OX > 0 && V % 2 == 0, "strip too narrow for k");
    static_assert(ROW_BYTES % 16 == 0, "ring rows must stay 16-byte aligned");
};

// x-neighbour sums (xm + xp) of one row held as NP float2 pairs per lane (columns lane*V ..).
template <int NP>
__device__ __forceinline__ void xsum_row(const float2 (&r)[NP], float2 (&sx)[NP]) {
    const float left = __shfl_up_sync(kAll, r[NP - 1].y, 1);
    const float right = __shfl_down_sync(kAll, r[0].x, 1);
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const float xl = p > 0 ? r[p - 1].y : left;
        const float xr = p < NP - 1 ? r[p + 1].x : right;
        sx[p] = make_float2(__fadd_rn(xl, r[p].y), __fadd_rn(r[p].x, xr));
    }
}

// V fp32 values (16-byte aligned p when V >= 4, 8-byte when V == 2) through the read-only path
template <int V>
__device__ __forceinline__ void ldg_floats(const float* p, float (&f)[V]) {
    if constexpr (V % 4 == 0) {
#pragma unroll
        for (int q = 0; q < V / 4; ++q) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(p) + q);
            f[4 * q] = t.x; f[4 * q + 1] = t.y; f[4 * q + 2] = t.z; f[4 * q + 3] = t.w;
        }
    } else {
        static_assert(V == 2, "V is 2 or a multiple of 4");
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        f[0] = t.x; f[1] = t.y;
    }
}

// storage <-> float2 pairs for one lane's V values
template <typename T, int V>
__device__ __forceinline__ void lds_pairs(const T* p, float2 (&v)[V / 2]) {
    float f[V];
    ld_vec_shared<T, V>(p, f);
#pragma unroll
    for (int q = 0; q < V / 2; ++q) v[q] = make_float2(f[2 * q], f[2 * q + 1]);
}

template <typename T, bool PER, bool SRC, bool BULK, int K, int V, int STAGES, int W, int MINB>
__global__ void __launch_bounds__(32 * W, MINB)
tb2d_pair_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b,
                 T2Geom g, float c0, float c1, int* err) {
    using C = T2Cfg<T, K, V, STAGES>;
    constexpr int NP = C::NP, EX = C::EX, KX = C::KX, OX = C::OX;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int item = blockIdx.x * W + warp;
    if (item >= g.nitems) return;  // warp-uniform; the kernel has no block barrier

    T* ring = reinterpret_cast<T*>(smem + warp * C::RING_BYTES);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + W * C::RING_BYTES) + warp * STAGES;

    const int strip = item % g.nstrips, chunk = item / g.nstrips;
    const int y0 = chunk * g.ych, y1 = min(y0 + g.ych, g.ny);
    const int xs = strip * OX - KX;  // first column of the extended strip
    const int lx = lane * V, gx = xs + lx;
    const int nit = K + (y1 - y0 + 1) / 2;  // iterations: K warm-up pairs + the stored pairs
    const int ybase = y0 - K;               // level-0 row of pair t: ybase + 2t

    // ---- level-0 source
    // bulk ring: this lane's piece of the extended row (destination column, source column,
    // length); every row splits the same way
    int pc_dst = 0, pc_src = 0, pc_len = 0;
    // direct loads: this lane's V columns, wrapped (periodic) or clamped (Dirichlet)
    int col[V];
    float pre[2][V];
    if constexpr (BULK) {
        if (lane == 0) {
            for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
            fence_mbar_init();
        }
        int done = 0, j = 0;
        while (done < EX) {
            const int x = xs + done;
            int src, len;
            if (PER) {
                src = wrap_near(x, g.nx);
                len = min(EX - done, g.nx - src);
            } else if (x < 0) {  // outside the array: any in-range data (never used)
                src = 0;
                len = min(min(EX - done, -x), g.nx);
            } else if (x >= g.nx) {
                src = 0;
                len = min(EX - done, g.nx);
            } else {
                src = x;
                len = min(EX - done, g.nx - x);
            }
            if (j == lane) { pc_dst = done; pc_src = src; pc_len = len; }
            done += len;
            ++j;
        }
        __syncwarp();
    } else {
#pragma unroll
        for (int j = 0; j < V; ++j)
            col[j] = PER ? wrap_near(gx + j, g.nx) : clamp_idx(gx + j, 0, g.nx - 1);
    }
    auto row_of = [&](int r) { return PER ? wrap_near(r, g.ny) : clamp_idx(r, 0, g.ny - 1); };
    auto issue = [&](int t) {  // bulk: copy level-0 pair t into its stage
        const int s = t % STAGES;
        if (lane == 0) mbar_arrive_expect_tx(&bar[s], C::STAGE_BYTES);
        __syncwarp();
        if (pc_len > 0) {
            T* dst = ring + s * (2 * EX) + pc_dst;
            const int r = ybase + 2 * t;
            bulk_load(dst, u + int64_t(row_of(r)) * g.nx + pc_src, uint32_t(pc_len) * sizeof(T),
                      &bar[s]);
            bulk_load(dst + EX, u + int64_t(row_of(r + 1)) * g.nx + pc_src,
                      uint32_t(pc_len) * sizeof(T), &bar[s]);
        }
    };
    auto load_direct = [&](int t) {  // direct: level-0 pair t into `pre`
        const int r = ybase + 2 * t;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const T* row = u + int64_t(row_of(r + i)) * g.nx;
#pragma unroll
            for (int j = 0; j < V; ++j) pre[i][j] = ldg1(row + col[j]);
        }
    };

    // ---- Dirichlet: columns 0 and nx-1 keep their values at every level
    uint32_t fixx = 0;
    if constexpr (!PER) {
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gx + j == 0 || gx + j == g.nx - 1) fixx |= 1u << j;
    }
    const bool writer = lx >= KX && lx < KX + OX && gx < g.nx;
    const bool vec_store = BULK && gx + V <= g.nx;  // whole aligned vector inside the row
    // the source row of a lane as one vector when its V columns are contiguous in the array
    const int bcol = PER ? wrap_near(gx, g.nx) : gx;
    const bool bvec = BULK && bcol >= 0 && bcol + V <= g.nx;

    const float2 c0v = make_float2(c0, c0), c1v = make_float2(c1, c1);
    bool ok = true;
    int waited = 0, issued = 0;

    if constexpr (BULK) {
        const int pro = min(STAGES - 1, nit);
        for (int t = 0; t < pro; ++t) issue(t);
        issued = pro;
    } else {
        load_direct(0);
    }

    // level s (0..K-1): the kept pair and the new pair, trading roles every iteration
    float2 A[K][2][NP], B[K][2][NP];
#pragma unroll
    for (int s = 0; s < K; ++s)
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int p = 0; p < NP; ++p) A[s][i][p] = B[s][i][p] = make_float2(0.f, 0.f);

    // one row of level s from its centre row, its y-neighbours and the centre's x-sums
    auto level_row = [&](const float2 (&ctr)[NP], const float2 (&ym)[NP], const float2 (&yp)[NP],
                         int c, float2 (&res)[NP]) {
        float2 sx[NP];
        xsum_row<NP>(ctr, sx);
        float2 bv[NP];
        if constexpr (SRC) {  // Jacobi source, added last
            const float* brow = b + int64_t(row_of(c)) * g.nx;
            float f[V];
            if (bvec) {
                ldg_floats<V>(brow + bcol, f);
            } else {
#pragma unroll
                for (int j = 0; j < V; ++j)
                    f[j] = __ldg(brow + (PER ? wrap_near(gx + j, g.nx)
                                             : clamp_idx(gx + j, 0, g.nx - 1)));
            }
#pragma unroll
            for (int p = 0; p < NP; ++p) bv[p] = make_float2(f[2 * p], f[2 * p + 1]);
        }
        const bool rowfix = !PER && (c <= 0 || c >= g.ny - 1);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            float2 v = lin2(c0v, c1v, ctr[p], add2(sx[p], add2(ym[p], yp[p])));
            if constexpr (SRC) v = add2(v, bv[p]);
            if constexpr (!PER) {
                if (rowfix || ((fixx >> (2 * p)) & 1u)) v.x = ctr[p].x;
                if (rowfix || ((fixx >> (2 * p + 1)) & 1u)) v.y = ctr[p].y;
            }
            res[p] = v;
        }
    };

    auto store_row = [&](int c, const float2 (&v)[NP]) {
        if (!ok || !writer || c < y0 || c >= y1) return;
        if (!PER && (c == 0 || c == g.ny - 1)) return;
        T* dst = o + int64_t(c) * g.nx + gx;
        if (vec_store && fixx == 0) {
            float f[V];
#pragma unroll
            for (int p = 0; p < NP; ++p) { f[2 * p] = v[p].x; f[2 * p + 1] = v[p].y; }
            st_vec<T, V>(dst, f);
        } else {
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int j = 2 * p;
                if (gx + j < g.nx && !((fixx >> j) & 1u)) dst[j] = from_f<T>(v[p].x);
                if (gx + j + 1 < g.nx && !((fixx >> (j + 1)) & 1u)) dst[j + 1] = from_f<T>(v[p].y);
            }
        }
    };

    // One iteration: level-0 pair t becomes New[0]; level s = 1..K makes rows (r0-s, r0-s+1)
    // from level s-1's kept pair Old (rows r0-s-1, r0-s) and new pair New (r0-s+1, r0-s+2).
    auto iter = [&](float2 (&Old)[K][2][NP], float2 (&New)[K][2][NP], int t) {
        const int r0 = ybase + 2 * t;
        if constexpr (BULK) {
            if (ok && issued < nit && issued <= t + STAGES - 1) {
                issue(issued);
                ++issued;
            }
            const int s = t % STAGES;
            if (ok) {
                if (mbar_wait(&bar[s], uint32_t(t / STAGES) & 1u, err)) ++waited;
                else ok = false;
            }
            const T* st = ring + s * (2 * EX) + lx;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                if (ok) {
                    lds_pairs<T, V>(st + i * EX, New[0][i]);
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p) New[0][i][p] = make_float2(0.f, 0.f);
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int p = 0; p < NP; ++p) New[0][i][p] = make_float2(pre[i][2 * p], pre[i][2 * p + 1]);
            if (t + 1 < nit) load_direct(t + 1);
        }
#pragma unroll
        for (int s = 1; s <= K; ++s) {
            float2 ra[NP], rb[NP];
            const int ca = r0 - s;
            level_row(Old[s - 1][1], Old[s - 1][0], New[s - 1][0], ca, ra);
            level_row(New[s - 1][0], Old[s - 1][1], New[s - 1][1], ca + 1, rb);
            if (s < K) {
#pragma unroll
                for (int p = 0; p < NP; ++p) { New[s][0][p] = ra[p]; New[s][1][p] = rb[p]; }
            } else {
                store_row(ca, ra);
                store_row(ca + 1, rb);
            }
        }
    };

    for (int t = 0; t < nit; t += 2) {
        iter(A, B, t);
        if (t + 1 >= nit) break;
        iter(B, A, t + 1);
    }

    if constexpr (BULK) {
        // copies still in flight (after an expired wait) must land before the warp leaves
        if (lane == 0) {
            for (int t = waited; t < issued; ++t)
                if (!mbar_wait(&bar[t % STAGES], uint32_t(t / STAGES) & 1u, err)) break;
        }
        __syncwarp();
    }
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
