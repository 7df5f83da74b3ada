// 3D single-step z-march with TMA plane staging (sm_100a).
//
// Functional spec: pyheat3d src/pyheat3d/backends/stencil.cu:101-161 (zmarch3d) — one update of
// the 7-point stencil per pass, marching along z. This kernel is a new design for B200:
//
// * Persistent blocks walk a static list of work items (tile_x, tile_y, z-chunk), ordered with
//   the chunk slowest so that blocks running at the same time work on neighbouring tiles of the
//   same planes (halo rows and chunk-edge planes then come from L2, not HBM).
// * One producer warp streams the planes of each item into a STAGES-deep shared-memory ring with
//   cp.async.bulk.tensor loads that complete on an mbarrier (transaction bytes): per plane one
//   TX x TY body box, two TX x 1 halo rows and two HX x TY halo columns, all at wrapped
//   coordinates for periodic grids (TMA does not wrap; out-of-range Dirichlet halos read zeros
//   that are never used).
// * NWC consumer warps keep a register queue along z (below / centre / above), take the
//   x-neighbours from warp shuffles (lanes 0 and 31 read the halo columns) and the y-neighbours
//   from registers or the staged plane, and store 16-byte vectors straight to global memory.
// * Every mbarrier wait is bounded; on expiry the error word is set and the block drains the
//   loads it issued before returning.
//
// Requirements (else the caller uses the plain-load march): nx * sizeof(T) % 16 == 0 and 16-byte
// aligned buffers.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "ph3_common.cuh"
#include "ph3_internal.h"
#include "ph3_march.cuh"

namespace ph3 {

namespace {

constexpr unsigned kFullMask = 0xffffffffu;

template <typename T, int TY, int NWC, int STAGES, int LB = 16>
struct ZmCfg {
    static constexpr int V = LB / int(sizeof(T));  // values per lane (one LB-byte vector)
    static constexpr int TX = 32 * V;              // tile width: 32 * LB bytes per row
    static constexpr int HX = 16 / int(sizeof(T)); // halo column box: 16 bytes
    static constexpr int RW = TY / NWC;            // rows per consumer warp
    static_assert(TY % NWC == 0, "rows must split evenly over the consumer warps");
    static constexpr int BODY_BYTES = (TY + 2) * TX * int(sizeof(T));
    static constexpr int SIDE_BYTES = TY * HX * int(sizeof(T));
    static constexpr int STAGE_BYTES = ((BODY_BYTES + 2 * SIDE_BYTES + 127) / 128) * 128;
    static constexpr int TX_BYTES = BODY_BYTES + 2 * SIDE_BYTES;  // bytes landed per plane
    static constexpr int SMEM = STAGES * STAGE_BYTES + 2 * STAGES * 8 + 16;
    // every box lands at a 128-byte aligned shared-memory address (the tensor-copy destination
    // rule): rows are 512 bytes, and the second side box starts SIDE_BYTES after the first
    static_assert(SIDE_BYTES % 128 == 0, "TY must be a multiple of 8");
    static constexpr int THREADS = 32 * (NWC + 1);
};

struct ZmGeom {
    int nz, ny, nx;
    int ntx, nty;      // tiles in x and y
    int zbase, nzi;    // first marched plane and number of marched planes
    int zch, nchunks;  // chunk length and count
    int nitems;
};

// One lane's source values of one plane (RW rows x V fp32 values, as float4s). The consumers
// load them one plane ahead, so the Jacobi source never stalls a plane on DRAM latency.
template <int RW, int V>
struct SrcRows {
    float4 v[RW][V / 4];
    __device__ __forceinline__ void load(const float* __restrict__ b, int64_t zoff,
                                         const int (&boff)[RW]) {
#pragma unroll
        for (int r = 0; r < RW; ++r)
#pragma unroll
            for (int q = 0; q < V / 4; ++q)
                v[r][q] = __ldg(reinterpret_cast<const float4*>(b + zoff + boff[r]) + q);
    }
};

// Blocks per SM the register budget is sized for (the ring's shared memory allows as many).
template <typename T, int TY, int NWC, int LB = 16>
constexpr int zm_min_blocks() {
    constexpr int RW = TY / NWC;
    if (LB == 8) return 2;  // 4 values per lane: half the registers of a 16-byte lane
    if (NWC >= 16) return sizeof(T) == 4 ? 2 : 1;
    if (sizeof(T) == 4) return RW >= 4 ? 2 : 3;
    return RW >= 2 ? 1 : 3;
}

// Producer (one thread): streams the planes zlo-1 .. zhi of every item of this block into the
// ring, in the order the consumers take them. Stage s of plane number `it` is reused once all
// NWC consumer warps released its previous use (the empty barrier's phase).
template <typename T, bool PER, int TY, int NWC, int STAGES, int LB = 16>
__device__ __forceinline__ void zm_produce(const CUtensorMap* tm_body, const CUtensorMap* tm_row,
                                           const CUtensorMap* tm_side, const ZmGeom& g,
                                           unsigned char* smem, uint64_t* full, uint64_t* empty,
                                           volatile int* issued, int* err) {
    using C = ZmCfg<T, TY, NWC, STAGES, LB>;
    constexpr int TX = C::TX, HX = C::HX;
    prefetch_tmap(tm_body);
    prefetch_tmap(tm_row);
    prefetch_tmap(tm_side);
    uint32_t it = 0;
    for (int item = blockIdx.x; item < g.nitems; item += gridDim.x) {
        const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty;
        const int ch = item / (g.ntx * g.nty);
        const int x0 = tx * TX, y0 = ty * TY;
        const int zlo = g.zbase + ch * g.zch;
        const int zhi = min(zlo + g.zch, g.zbase + g.nzi);
        int ytop = y0 - 1, ybot = y0 + TY, xl = x0 - HX, xr = x0 + TX;
        if constexpr (PER) {
            ytop = y0 == 0 ? g.ny - 1 : y0 - 1;
            ybot = y0 + TY >= g.ny ? 0 : y0 + TY;
            xl = x0 == 0 ? g.nx - HX : x0 - HX;
            xr = x0 + TX >= g.nx ? 0 : x0 + TX;
        }
        for (int p = zlo - 1; p <= zhi; ++p, ++it) {
            const int s = it % STAGES;
            const uint32_t n = it / STAGES;
            if (n > 0 && !mbar_wait(&empty[s], (n & 1u) ^ 1u, err)) return;
            int pz = p;
            if constexpr (PER) pz = p < 0 ? p + g.nz : (p >= g.nz ? p - g.nz : p);
            unsigned char* st = smem + s * C::STAGE_BYTES;
            constexpr int ROW = TX * int(sizeof(T));
            mbar_arrive_expect_tx(&full[s], C::TX_BYTES);
            tma_load_3d(st, tm_row, x0, ytop, pz, &full[s]);
            tma_load_3d(st + ROW, tm_body, x0, y0, pz, &full[s]);
            tma_load_3d(st + (TY + 1) * ROW, tm_row, x0, ybot, pz, &full[s]);
            tma_load_3d(st + C::BODY_BYTES, tm_side, xl, y0, pz, &full[s]);
            tma_load_3d(st + C::BODY_BYTES + C::SIDE_BYTES, tm_side, xr, y0, pz, &full[s]);
            *issued = int(it + 1);
        }
    }
}

template <typename T, bool PER, int TY, int NWC, int STAGES, bool PACKED, int LB = 16,
          bool SRC = true, bool ROT = false>
__global__ void __launch_bounds__(32 * (NWC + 1), zm_min_blocks<T, TY, NWC, LB>())
zmarch_tma_kernel(const __grid_constant__ CUtensorMap tm_body,
                  const __grid_constant__ CUtensorMap tm_row,
                  const __grid_constant__ CUtensorMap tm_side, T* __restrict__ o,
                  const float* __restrict__ b, ZmGeom g, float c0, float c1, int* err) {
    using C = ZmCfg<T, TY, NWC, STAGES, LB>;
    constexpr int V = C::V, TX = C::TX, HX = C::HX, RW = C::RW;
    static_assert(V % 2 == 0, "lanes hold whole float2 pairs");
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * C::STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    volatile int* issued = reinterpret_cast<volatile int*>(empty + STAGES);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NWC);
        }
        *issued = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const int64_t P = int64_t(g.nx) * g.ny;

    if (warp == NWC) {
        if (lane == 0)
            zm_produce<T, PER, TY, NWC, STAGES, LB>(&tm_body, &tm_row, &tm_side, g, smem, full,
                                                    empty, issued, err);
        return;
    }

    // --------------------------------------------------------------------- consumer warps
    using PK = PackLane<T, LB>;
    using LW = typename PK::W;  // one lane's vector
    constexpr int NP = PK::NP;  // float2 pairs per lane (V / 2)
    const int r0 = warp * RW;   // first tile row of this warp
    const float2 c0v = make_float2(c0, c0), c1v = make_float2(c1, c1);
    uint32_t it = 0;        // planes consumed
    int nxt_s = 0;          // stage of the next plane to consume
    uint32_t nxt_ph = 0;    // its mbarrier phase parity
    auto take = [&](int& s, uint32_t& ph) {
        s = nxt_s;
        ph = nxt_ph;
        if (++nxt_s == STAGES) { nxt_s = 0; nxt_ph ^= 1u; }
        ++it;
    };
    bool ok = true;
    auto stage_row = [&](int s, int row) -> const LW* {
        return reinterpret_cast<const LW*>(smem + s * C::STAGE_BYTES + row * TX * int(sizeof(T))) +
               lane;
    };
    auto side = [&](int s, int right) -> const T* {
        return reinterpret_cast<const T*>(smem + s * C::STAGE_BYTES + C::BODY_BYTES +
                                          right * C::SIDE_BYTES);
    };
    auto release = [&](int s) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    };

    for (int item = blockIdx.x; item < g.nitems && ok; item += gridDim.x) {
        const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty;
        const int ch = item / (g.ntx * g.nty);
        const int x0 = tx * TX, y0 = ty * TY;
        const int zlo = g.zbase + ch * g.zch;
        const int zhi = min(zlo + g.zch, g.zbase + g.nzi);
        const int gx = x0 + lane * V;
        // masks of sites this thread must not write
        uint32_t skipx = 0, skipy = 0;
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gx + j >= g.nx || (!PER && (gx + j == 0 || gx + j == g.nx - 1))) skipx |= 1u << j;
#pragma unroll
        for (int r = 0; r < RW; ++r) {
            const int gy = y0 + r0 + r;
            if (gy >= g.ny || (!PER && (gy == 0 || gy == g.ny - 1))) skipy |= 1u << r;
        }
        // periodic wrap inside a partial tile: the site after column nx-1 / row ny-1 is the
        // halo loaded from column 0 / row 0
        const bool wrapx = PER && (gx + V == g.nx) && lane != 31;
        int wrap_r = -1;
        if (PER && y0 + TY > g.ny) {
            const int rr = g.ny - 1 - (y0 + r0);
            if (rr >= 0 && rr < RW) wrap_r = rr;
        }
        float2 bel[RW][NP], ctr[RW][NP], abv[RW][NP];
        int boff[RW];  // source offsets of the warp's rows within a plane
#pragma unroll
        for (int r = 0; r < RW; ++r)
            boff[r] = min(y0 + r0 + r, g.ny - 1) * g.nx + min(gx, g.nx - V);
        SrcRows<RW, V> bnext;
        if constexpr (SRC) bnext.load(b, int64_t(zlo) * P, boff);

        // plane zlo-1: only the own values are needed
        {
            int s;
            uint32_t ph;
            take(s, ph);
            if (!mbar_wait(&full[s], ph, err)) { ok = false; break; }
#pragma unroll
            for (int r = 0; r < RW; ++r) PK::unpack(*stage_row(s, r0 + r + 1), bel[r]);
            release(s);
        }
        int sc;  // stage of the centre plane
        uint32_t phc;
        take(sc, phc);
        if (!mbar_wait(&full[sc], phc, err)) { ok = false; break; }
#pragma unroll
        for (int r = 0; r < RW; ++r) PK::unpack(*stage_row(sc, r0 + r + 1), ctr[r]);

        // One plane z with the below / centre / above planes in the given register sets; the
        // above set is loaded here. ROT rotates the three sets by name (three planes per loop
        // pass, no register copies); otherwise the sets are copied down after every plane.
        auto plane = [&](int z, float2 (&bel)[RW][NP], float2 (&ctr)[RW][NP],
                         float2 (&abv)[RW][NP]) {
            int sa;
            uint32_t pha;
            take(sa, pha);
            if (!mbar_wait(&full[sa], pha, err)) { ok = false; return; }
#pragma unroll
            for (int r = 0; r < RW; ++r) PK::unpack(*stage_row(sa, r0 + r + 1), abv[r]);
            SrcRows<RW, V> bcur;
            if constexpr (SRC) {
                bcur = bnext;
                if (z + 1 < zhi) bnext.load(b, int64_t(z + 1) * P, boff);
            }
            // y-neighbours of the warp's first and last rows come from the staged centre plane
            float2 up[NP], dn[NP], wdn[NP];
            PK::unpack(*stage_row(sc, r0), up);
            PK::unpack(*stage_row(sc, wrap_r == RW - 1 ? TY + 1 : r0 + RW + 1), dn);
            if (wrap_r >= 0 && wrap_r < RW - 1) PK::unpack(*stage_row(sc, TY + 1), wdn);
            const T* sl = side(sc, 0);
            const T* sr = side(sc, 1);
#pragma unroll
            for (int r = 0; r < RW; ++r) {
                const int gy = y0 + r0 + r;
                const float left = __shfl_up_sync(kFullMask, ctr[r][NP - 1].y, 1);
                const float right = __shfl_down_sync(kFullMask, ctr[r][0].x, 1);
                const float xlv = lane == 0 ? to_f(sl[(r0 + r) * HX + HX - 1]) : left;
                const float xrv = (lane == 31 || wrapx) ? to_f(sr[(r0 + r) * HX]) : right;
                float2 bv[NP];
                if constexpr (SRC) {
#pragma unroll
                    for (int q = 0; q < NP / 2; ++q) {
                        const float4 t4 = bcur.v[r][q];
                        bv[2 * q] = make_float2(t4.x, t4.y);
                        bv[2 * q + 1] = make_float2(t4.z, t4.w);
                    }
                }
                // x-neighbour sums, site by site, landing directly in register pairs
                float2 sx[NP];
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    const float l0 = p > 0 ? ctr[r][p - 1].y : xlv;
                    const float r1 = p < NP - 1 ? ctr[r][p + 1].x : xrv;
                    sx[p] = make_float2(__fadd_rn(l0, ctr[r][p].y), __fadd_rn(ctr[r][p].x, r1));
                }
                float2 out[NP];
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    const float2 ym = r > 0 ? ctr[r - 1][p] : up[p];
                    float2 yp = dn[p];
                    if (r < RW - 1) yp = r == wrap_r ? wdn[p] : ctr[r + 1][p];
                    float2 v;
                    if constexpr (PACKED) {
                        v = upd3_sx2(c0v, c1v, ctr[r][p], sx[p], ym, yp, bel[r][p], abv[r][p]);
                        if constexpr (SRC) v = add2(v, bv[p]);
                    } else {  // scalar chain, same rounding
                        const float sx0 = __fadd_rn(__fadd_rn(sx[p].x, __fadd_rn(ym.x, yp.x)),
                                                    __fadd_rn(bel[r][p].x, abv[r][p].x));
                        const float sx1 = __fadd_rn(__fadd_rn(sx[p].y, __fadd_rn(ym.y, yp.y)),
                                                    __fadd_rn(bel[r][p].y, abv[r][p].y));
                        v.x = __fadd_rn(__fmul_rn(c0, ctr[r][p].x), __fmul_rn(c1, sx0));
                        v.y = __fadd_rn(__fmul_rn(c0, ctr[r][p].y), __fmul_rn(c1, sx1));
                        if constexpr (SRC) {
                            v.x = __fadd_rn(v.x, bv[p].x);
                            v.y = __fadd_rn(v.y, bv[p].y);
                        }
                    }
                    out[p] = v;
                }
                if (!((skipy >> r) & 1u)) {
                    T* dst = o + int64_t(z) * P + int64_t(gy) * g.nx + gx;
                    if (skipx == 0) {
                        *reinterpret_cast<LW*>(dst) = PK::pack(out);
                    } else {
#pragma unroll
                        for (int p = 0; p < NP; ++p) {
                            if (!((skipx >> (2 * p)) & 1u)) dst[2 * p] = from_f<T>(out[p].x);
                            if (!((skipx >> (2 * p + 1)) & 1u)) dst[2 * p + 1] = from_f<T>(out[p].y);
                        }
                    }
                }
            }
            release(sc);
            sc = sa;
        };
        if constexpr (ROT) {
            for (int z = zlo; z < zhi; z += 3) {
                plane(z, bel, ctr, abv);
                if (!ok || z + 1 >= zhi) break;
                plane(z + 1, ctr, abv, bel);
                if (!ok || z + 2 >= zhi) break;
                plane(z + 2, abv, bel, ctr);
                if (!ok) break;
            }
        } else {
            for (int z = zlo; z < zhi; ++z) {
                plane(z, bel, ctr, abv);
                if (!ok) break;
#pragma unroll
                for (int r = 0; r < RW; ++r)
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
                        bel[r][p] = ctr[r][p];
                        ctr[r][p] = abv[r][p];
                    }
            }
        }
        if (!ok) break;
        release(sc);  // plane zhi
    }

    if (!ok) {
        // a wait expired: drain the loads this block issued so no copy lands after exit
        if (warp == 0 && lane == 0) {
            const int n_issued = *issued;
            for (int k = int(it) - 1; k < n_issued; ++k) {
                if (k < 0) continue;
                const int s = k % STAGES;
                if (!mbar_wait(&full[s], (uint32_t(k) / STAGES) & 1u, err)) break;
            }
        }
    }
}

// First form of the consumer (scalar float registers, no register cap): kept as a selectable
// configuration because it is measured beside the packed form. The ring stage and parity of
// the next plane advance incrementally (no division by the stage count per plane).
template <typename T, bool PER, int TY, int NWC, int STAGES>
__global__ void __launch_bounds__(32 * (NWC + 1))
zmarch_v1_kernel(const __grid_constant__ CUtensorMap tm_body,
                  const __grid_constant__ CUtensorMap tm_row,
                  const __grid_constant__ CUtensorMap tm_side, T* __restrict__ o,
                  const float* __restrict__ b, ZmGeom g, float c0, float c1, int* err) {
    using C = ZmCfg<T, TY, NWC, STAGES>;
    constexpr int V = C::V, TX = C::TX, HX = C::HX, RW = C::RW;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * C::STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    volatile int* issued = reinterpret_cast<volatile int*>(empty + STAGES);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NWC);
        }
        *issued = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const int64_t P = int64_t(g.nx) * g.ny;

    if (warp == NWC) {
        if (lane == 0)
            zm_produce<T, PER, TY, NWC, STAGES>(&tm_body, &tm_row, &tm_side, g, smem, full,
                                                empty, issued, err);
        return;
    }

    // --------------------------------------------------------------------- consumer warps
    const int r0 = warp * RW;  // first tile row of this warp
    uint32_t it = 0;           // planes taken
    int st = 0;                // ring stage of plane `it` (it % STAGES, kept incrementally)
    uint32_t ph = 0;           // its full-barrier parity ((it / STAGES) & 1)
    auto advance = [&]() {
        ++it;
        if (++st == STAGES) { st = 0; ph ^= 1u; }
    };
    bool ok = true;
    auto body_row = [&](int s, int row) -> const T* {
        return reinterpret_cast<const T*>(smem + s * C::STAGE_BYTES) + row * TX;
    };
    auto side = [&](int s, int right) -> const T* {
        return reinterpret_cast<const T*>(smem + s * C::STAGE_BYTES + C::BODY_BYTES +
                                          right * C::SIDE_BYTES);
    };
    auto release = [&](int s) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    };
    auto lds_vec = [&](const T* p, float (&v)[V]) {
        union { uint4 w; T e[V]; } un;
        un.w = *reinterpret_cast<const uint4*>(p);
#pragma unroll
        for (int j = 0; j < V; ++j) v[j] = to_f(un.e[j]);
    };

    for (int item = blockIdx.x; item < g.nitems && ok; item += gridDim.x) {
        const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty;
        const int ch = item / (g.ntx * g.nty);
        const int x0 = tx * TX, y0 = ty * TY;
        const int zlo = g.zbase + ch * g.zch;
        const int zhi = min(zlo + g.zch, g.zbase + g.nzi);
        const int gx = x0 + lane * V;
        // masks of sites this thread must not write
        uint32_t skipx = 0, skipy = 0;
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gx + j >= g.nx || (!PER && (gx + j == 0 || gx + j == g.nx - 1))) skipx |= 1u << j;
#pragma unroll
        for (int r = 0; r < RW; ++r) {
            const int gy = y0 + r0 + r;
            if (gy >= g.ny || (!PER && (gy == 0 || gy == g.ny - 1))) skipy |= 1u << r;
        }
        // periodic wrap inside a partial tile: the site after column nx-1 / row ny-1 is the
        // halo loaded from column 0 / row 0
        const bool wrapx = PER && (gx + V == g.nx) && lane != 31;
        float bel[RW][V], ctr[RW][V], abv[RW][V];
        int boff[RW];  // source offsets of the warp's rows within a plane
#pragma unroll
        for (int r = 0; r < RW; ++r)
            boff[r] = min(y0 + r0 + r, g.ny - 1) * g.nx + min(gx, g.nx - V);
        SrcRows<RW, V> bnext;
        if (b != nullptr) bnext.load(b, int64_t(zlo) * P, boff);

        // plane zlo-1: only the own values are needed
        {
            const int s = st;
            if (!mbar_wait(&full[s], ph, err)) { ok = false; break; }
#pragma unroll
            for (int r = 0; r < RW; ++r) lds_vec(body_row(s, r0 + r + 1) + lane * V, bel[r]);
            release(s);
            advance();
        }
        int sc = st;  // stage of the centre plane
        if (!mbar_wait(&full[sc], ph, err)) { ok = false; break; }
#pragma unroll
        for (int r = 0; r < RW; ++r) lds_vec(body_row(sc, r0 + r + 1) + lane * V, ctr[r]);
        advance();
        // periodic partial tile: the row after ny-1 is the halo row loaded from row 0
        int wrap_r = -1;
        if (PER && y0 + TY > g.ny) {
            const int rr = g.ny - 1 - (y0 + r0);
            if (rr >= 0 && rr < RW) wrap_r = rr;
        }

        for (int z = zlo; z < zhi; ++z) {
            const int sa = st;
            if (!mbar_wait(&full[sa], ph, err)) { ok = false; break; }
#pragma unroll
            for (int r = 0; r < RW; ++r) lds_vec(body_row(sa, r0 + r + 1) + lane * V, abv[r]);
            SrcRows<RW, V> bcur;
            if (b != nullptr) {
                bcur = bnext;
                if (z + 1 < zhi) bnext.load(b, int64_t(z + 1) * P, boff);
            }
            // y-neighbours of the first and last rows come from the staged centre plane
            float up[V], dn[V], wdn[V];
            lds_vec(body_row(sc, r0) + lane * V, up);
            lds_vec(body_row(sc, wrap_r == RW - 1 ? TY + 1 : r0 + RW + 1) + lane * V, dn);
            if (wrap_r >= 0 && wrap_r < RW - 1) lds_vec(body_row(sc, TY + 1) + lane * V, wdn);
            const T* sl = side(sc, 0);
            const T* sr = side(sc, 1);
#pragma unroll
            for (int r = 0; r < RW; ++r) {
                const int gy = y0 + r0 + r;
                const float left = __shfl_up_sync(kFullMask, ctr[r][V - 1], 1);
                const float right = __shfl_down_sync(kFullMask, ctr[r][0], 1);
                float hl = 0.f, hr = 0.f;
                if (lane == 0) hl = to_f(sl[(r0 + r) * HX + HX - 1]);
                if (lane == 31 || wrapx) hr = to_f(sr[(r0 + r) * HX]);
                float bv[V];
                if (b != nullptr) {
#pragma unroll
                    for (int q = 0; q < V / 4; ++q) {
                        const float4 t = bcur.v[r][q];
                        bv[4 * q] = t.x; bv[4 * q + 1] = t.y; bv[4 * q + 2] = t.z; bv[4 * q + 3] = t.w;
                    }
                }
                float out[V];
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    const float xm = j > 0 ? ctr[r][j - 1] : (lane == 0 ? hl : left);
                    const float xp = j < V - 1 ? ctr[r][j + 1]
                                               : ((lane == 31 || wrapx) ? hr : right);
                    const float ym = r > 0 ? ctr[r - 1][j] : up[j];
                    float yp = dn[j];
                    if (r < RW - 1) yp = r == wrap_r ? wdn[j] : ctr[r + 1][j];
                    float v = upd3(c0, c1, ctr[r][j], xm, xp, ym, yp, bel[r][j], abv[r][j]);
                    if (b != nullptr) v = __fadd_rn(v, bv[j]);
                    out[j] = v;
                }
                if (!((skipy >> r) & 1u)) {
                    T* dst = o + int64_t(z) * P + int64_t(gy) * g.nx + gx;
                    if (skipx == 0) {
                        st_vec<T, V>(dst, out);
                    } else {
#pragma unroll
                        for (int j = 0; j < V; ++j)
                            if (!((skipx >> j) & 1u)) dst[j] = from_f<T>(out[j]);
                    }
                }
            }
            release(sc);
#pragma unroll
            for (int r = 0; r < RW; ++r)
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    bel[r][j] = ctr[r][j];
                    ctr[r][j] = abv[r][j];
                }
            sc = sa;
            advance();
        }
        if (!ok) break;
        release(sc);  // plane zhi
    }

    if (!ok) {
        // a wait expired: drain the loads this block issued so no copy lands after exit
        if (warp == 0 && lane == 0) {
            const int n_issued = *issued;
            for (int k = int(it); k < n_issued; ++k) {
                const int s = k % STAGES;
                if (!mbar_wait(&full[s], (uint32_t(k) / STAGES) & 1u, err)) break;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// 3D single step for rows without 16-byte vectors (any nx), fed by 1D tensor copies.
//
// The field is addressed as one flat array. A warp owns R rows of a 128-column strip (lane l:
// columns x0 + 4l .. +3) and a z-chunk, with its own STAGES-deep shared-memory ring: per plane
// one lane copies R + 2 rows (the warp's rows and the rows above and below) as 1D boxes of SPAN
// elements that start at the 16-byte boundary at or before column x0 - 1, so every box starts
// aligned whatever nx is; out-of-range parts of a box (before the first or after the last
// element of the array) arrive as zeros. Lanes read their four columns at the row's offset in
// the box with the widest shared-memory access the offset allows. Periodic strips at a row end
// take the wrapped neighbour column from a 16-byte box around it. The own rows of planes z-1,
// z, z+1 stay in registers; the ring keeps STAGES - 2 planes in flight. Every warp runs its own
// pipeline (no block barrier) and every wait is bounded.
// ---------------------------------------------------------------------------------------------
template <typename T, bool PER, int R, int STAGES>
struct RgCfg {
    static constexpr int E = 16 / int(sizeof(T));          // elements per 16 bytes
    static constexpr int NCH = (130 + 2 * (E - 1)) / E;     // 16-byte chunks per row box
    static constexpr int SPAN = NCH * E;                    // elements per row box
    static_assert(SPAN >= 130 + E - 1, "a row box covers x0-1 .. x0+128 at any offset");
    static constexpr int ROWB = (SPAN * int(sizeof(T)) + 127) / 128 * 128;  // 128-byte slots
    static constexpr int HALB = 128;                        // slot of one 16-byte halo box
    static constexpr int NHAL = PER ? 2 * R : 0;            // left / right halo of each own row
    static constexpr int STAGEB = (R + 2) * ROWB + NHAL * HALB;
    static constexpr int WARPB = STAGES * STAGEB + 128;     // + the warp's mbarriers
};

template <typename T>
__device__ __forceinline__ void lds4a(const T* p, int a, float (&v)[4]) {
    if (a == 0) {
        ld_vec_shared<T, 4>(p, v);
    } else if (a == 2) {
        float t[2], w[2];
        ld_vec_shared<T, 2>(p, t);
        ld_vec_shared<T, 2>(p + 2, w);
        v[0] = t[0]; v[1] = t[1]; v[2] = w[0]; v[3] = w[1];
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = to_f(p[j]);
    }
}

template <typename T>
__device__ __forceinline__ void ldg4a(const T* p, int a, float (&v)[4]) {
    if (a == 0) {
        ld_vec<T, 4>(p, v);
    } else if (a == 2) {
        float t[2], w[2];
        ld_vec<T, 2>(p, t);
        ld_vec<T, 2>(p + 2, w);
        v[0] = t[0]; v[1] = t[1]; v[2] = w[0]; v[3] = w[1];
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = to_f(__ldg(p + j));
    }
}

template <typename T>
__device__ __forceinline__ void stg4a(T* p, int a, const float (&v)[4]) {
    if (a == 0) {
        st_vec<T, 4>(p, v);
    } else if (a == 2) {
        const float t[2] = {v[0], v[1]}, w[2] = {v[2], v[3]};
        st_vec<T, 2>(p, t);
        st_vec<T, 2>(p + 2, w);
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) p[j] = from_f<T>(v[j]);
    }
}

template <typename T, bool PER, int R, int W, int STAGES>
__global__ void __launch_bounds__(32 * W)
ring3d_kernel(const __grid_constant__ CUtensorMap tm_row, const __grid_constant__ CUtensorMap tm_hal,
              T* __restrict__ o, const float* __restrict__ b, int nz, int ny, int nx, float c0,
              float c1, int zch, int zb, int ze, int* err) {
    using C = RgCfg<T, PER, R, STAGES>;
    constexpr int E = C::E, V = 4;
    static_assert(STAGES >= 3, "planes z and z+1 are held while z+2 is copied");
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wbase = smem + warp * C::WARPB;
    uint64_t* full = reinterpret_cast<uint64_t*>(wbase + STAGES * C::STAGEB);
    const int x0 = blockIdx.x * 128, gx = x0 + lane * V;
    const int row0 = (blockIdx.y * W + warp) * R;
    int zlo = zb + blockIdx.z * zch, zhi = min(zlo + zch, ze);
    if constexpr (!PER) { zlo = max(zlo, 1); zhi = min(zhi, nz - 1); }
    if (x0 >= nx || row0 >= ny || zlo >= zhi) return;  // warp-uniform; no block barrier below
    if (lane == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncwarp();

    const int64_t P = int64_t(nx) * ny;
    const uint32_t P32 = uint32_t(P);  // low bits of plane offsets (element offsets modulo E)
    int yoff[R + 2];                    // element offsets of rows row0-1 .. row0+R in a plane
#pragma unroll
    for (int rr = 0; rr < R + 2; ++rr) yoff[rr] = fix_idx<PER>(row0 - 1 + rr, ny) * nx;
    const bool hleft = PER && x0 == 0, hright = PER && x0 + 128 >= nx;
    const int nhal = (hleft ? R : 0) + (hright ? R : 0);
    const uint32_t tx_bytes = uint32_t((R + 2) * C::SPAN * int(sizeof(T)) + nhal * 16);
    uint32_t skipx = 0, yskip = 0;  // columns / rows this lane must not write
#pragma unroll
    for (int j = 0; j < V; ++j)
        if (gx + j >= nx || (!PER && (gx + j == 0 || gx + j == nx - 1))) skipx |= 1u << j;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (row0 + r >= ny || (!PER && (row0 + r == 0 || row0 + r == ny - 1))) yskip |= 1u << r;
    // the column nx-1 in the last strip of a periodic row: its right neighbour is column 0
    const int cl = nx - 1 - x0;  // its position in the strip (valid when hright)

    const int npl = zhi - zlo + 2;  // planes zlo-1 .. zhi, numbered 0 .. npl-1
    int issued = 0;                  // planes whose copies were started (lane 0)
    auto stage = [&](int i) { return wbase + (i % STAGES) * C::STAGEB; };
    auto issue = [&](int i) {  // lane 0: plane number i into its stage
        const int zz = fix_near<PER>(zlo - 1 + i, nz);
        const int64_t zo = int64_t(zz) * P;
        unsigned char* st = stage(i);
        uint64_t* bar = &full[i % STAGES];
        mbar_arrive_expect_tx(bar, tx_bytes);
#pragma unroll
        for (int rr = 0; rr < R + 2; ++rr) {
            const int64_t e0 = zo + yoff[rr] + x0 - 1;
            tma_load_1d(st + rr * C::ROWB, &tm_row, int(e0 & ~int64_t(E - 1)), bar);
        }
        if constexpr (PER) {
            unsigned char* hs = st + (R + 2) * C::ROWB;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int64_t rs = zo + yoff[r + 1];
                if (hleft)
                    tma_load_1d(hs + (2 * r) * C::HALB, &tm_hal,
                                int((rs + nx - 1) & ~int64_t(E - 1)), bar);
                if (hright)
                    tma_load_1d(hs + (2 * r + 1) * C::HALB, &tm_hal, int(rs & ~int64_t(E - 1)),
                                bar);
            }
        }
        issued = i + 1;
    };
    // offset of column x0 - 1 in the box of row rr of plane zz
    auto off = [&](int zz, int rr) {
        return int((uint32_t(zz) * P32 + uint32_t(yoff[rr] + x0 - 1)) & uint32_t(E - 1));
    };
    auto rowp = [&](const unsigned char* st, int rr) {
        return reinterpret_cast<const T*>(st + rr * C::ROWB);
    };
    auto own_rows = [&](int i, float (&v)[R][V]) {  // the own rows' columns of plane number i
        const int zz = fix_near<PER>(zlo - 1 + i, nz);
        const unsigned char* st = stage(i);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int d = off(zz, r + 1);
            lds4a<T>(rowp(st, r + 1) + d + 1 + 4 * lane, (d + 1) & 3, v[r]);
        }
    };
    int waited = 0;  // planes seen to land by the whole warp
    auto wait = [&](int i) {  // warp-uniform result, so the warp never splits at a shuffle
        const bool r = mbar_wait(&full[i % STAGES], (uint32_t(i) / STAGES) & 1u, err);
        const bool all = __all_sync(kFullMask, r);
        if (all) waited = i + 1;
        return all;
    };

    if (lane == 0)  // fill every stage; afterwards step z refills the stage of plane z-1
        for (int i = 0; i < min(STAGES, npl); ++i) issue(i);
    float bel[R][V], ctr[R][V], abv[R][V];
    bool ok = wait(0);
    if (ok) own_rows(0, bel);
    ok = ok && wait(1);
    if (ok) own_rows(1, ctr);
    for (int z = zlo; ok && z < zhi; ++z) {
        const int ic = z - zlo + 1;  // plane number of z
        // refill the stage of plane z-1 (number ic-1), whose last reads were in the previous
        // step, with plane number ic-1+STAGES
        __syncwarp();
        if (lane == 0 && ic - 1 + STAGES < npl) {
            fence_proxy_async_smem();
            issue(ic - 1 + STAGES);
        }
        if (!wait(ic + 1)) { ok = false; break; }
        own_rows(ic + 1, abv);
        const unsigned char* st = stage(ic);
        float up[V], dn[V];
        {
            const int du = off(z, 0), dd = off(z, R + 1);
            lds4a<T>(rowp(st, 0) + du + 1 + 4 * lane, (du + 1) & 3, up);
            lds4a<T>(rowp(st, R + 1) + dd + 1 + 4 * lane, (dd + 1) & 3, dn);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int d = off(z, r + 1);
            const int a = (d + 1) & 3;  // residue of the row's columns (global and shared)
            const T* rp = rowp(st, r + 1) + d;
            const float left = __shfl_up_sync(kFullMask, ctr[r][V - 1], 1);
            const float right = __shfl_down_sync(kFullMask, ctr[r][0], 1);
            float xm[V], xp[V];
#pragma unroll
            for (int j = 0; j < V; ++j) {
                xm[j] = j > 0 ? ctr[r][j - 1] : (lane == 0 ? to_f(rp[0]) : left);
                xp[j] = j < V - 1 ? ctr[r][j + 1] : (lane == 31 ? to_f(rp[129]) : right);
            }
            if constexpr (PER) {
                const T* hs = reinterpret_cast<const T*>(st + (R + 2) * C::ROWB +
                                                         (2 * r) * C::HALB);
                const uint32_t rs = uint32_t(z) * P32 + uint32_t(yoff[r + 1]);
                if (hleft && lane == 0) xm[0] = to_f(hs[(rs + uint32_t(nx - 1)) & uint32_t(E - 1)]);
                if (hright && lane == (cl >> 2)) {
                    const float w = to_f(hs[C::HALB / int(sizeof(T)) + (rs & uint32_t(E - 1))]);
#pragma unroll
                    for (int j = 0; j < V; ++j)
                        if (j == (cl & 3)) xp[j] = w;
                }
            }
            float out[V];
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const float ym = r > 0 ? ctr[r - 1][j] : up[j];
                const float yp = r < R - 1 ? ctr[r + 1][j] : dn[j];
                out[j] = upd3(c0, c1, ctr[r][j], xm[j], xp[j], ym, yp, bel[r][j], abv[r][j]);
            }
            if (!((yskip >> r) & 1u)) {
                const int64_t ro = int64_t(z) * P + int64_t(row0 + r) * nx + gx;
                if (b != nullptr) {
                    float bv[V];
                    if (gx + V <= nx) {
                        ldg4a<float>(b + ro, a, bv);
                    } else {
#pragma unroll
                        for (int j = 0; j < V; ++j) bv[j] = gx + j < nx ? __ldg(b + ro + j) : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < V; ++j) out[j] = __fadd_rn(out[j], bv[j]);
                }
                if (skipx == 0) {
                    stg4a<T>(o + ro, a, out);
                } else {
#pragma unroll
                    for (int j = 0; j < V; ++j)
                        if (!((skipx >> j) & 1u)) o[ro + j] = from_f<T>(out[j]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int j = 0; j < V; ++j) {
                bel[r][j] = ctr[r][j];
                ctr[r][j] = abv[r][j];
            }
    }
    if (!ok && lane == 0) {
        // a wait expired: let the copies this warp started land before its shared memory goes
        for (int i = waited; i < issued; ++i)
            if (!mbar_wait(&full[i % STAGES], (uint32_t(i) / STAGES) & 1u, err)) break;
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

template <typename T>
CUtensorMapDataType tm_dtype() {
    if constexpr (sizeof(T) == 4) return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    else if constexpr (std::is_same_v<T, __half>) return CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    else return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
}

template <typename T>
bool make_map(CUtensorMap* m, const void* base, int nz, int ny, int nx, int bx, int by) {
    auto enc = get_encode();
    if (enc == nullptr) return false;
    cuuint64_t dims[3] = {cuuint64_t(nx), cuuint64_t(ny), cuuint64_t(nz)};
    cuuint64_t strides[2] = {cuuint64_t(nx) * sizeof(T), cuuint64_t(nx) * ny * sizeof(T)};
    cuuint32_t box[3] = {cuuint32_t(bx), cuuint32_t(by), 1};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, tm_dtype<T>(), 3, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T>
bool make_map_1d(CUtensorMap* m, const void* base, uint64_t n, uint32_t box) {
    auto enc = get_encode();
    if (enc == nullptr) return false;
    cuuint64_t dims[1] = {cuuint64_t(n)};
    cuuint64_t strides[1] = {0};  // unused for rank 1
    cuuint32_t bx[1] = {box};
    cuuint32_t es[1] = {1};
    return enc(m, tm_dtype<T>(), 1, const_cast<void*>(base), dims, strides, bx, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T, bool PER, int R, int W, int STAGES>
cudaError_t ring3d_t(const Launch& L) {
    using C = RgCfg<T, PER, R, STAGES>;
    constexpr int SMEM = W * C::WARPB;
    auto kern = ring3d_kernel<T, PER, R, W, STAGES>;
    static std::atomic<bool> attr_set[64];  // per device; first calls may race harmlessly
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_set[dev].load(std::memory_order_acquire)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
        if (e != cudaSuccess) return e;
        attr_set[dev].store(true, std::memory_order_release);
    }
    const uint64_t n = uint64_t(L.nz) * L.ny * L.nx;
    CUtensorMap tr, th;
    if (!make_map_1d<T>(&tr, L.u, n, C::SPAN) || !make_map_1d<T>(&th, L.u, n, C::E))
        return cudaErrorInvalidValue;
    const int zb = L.ze > 0 ? L.zb : 0, ze = L.ze > 0 ? L.ze : L.nz;
    auto cd = [](long long a, long long b) { return int((a + b - 1) / b); };
    const long long tiles = 1LL * cd(L.nx, 128) * cd(L.ny, W * R);
    const int zch = L.chunk > 0 ? L.chunk : default_chunk(ze - zb, tiles, 16, 16LL * sm_count());
    dim3 grd(cd(L.nx, 128), cd(L.ny, W * R), cd(ze - zb, zch));
    if (grd.y > 65535 || grd.z > 65535) return cudaErrorInvalidConfiguration;
    kern<<<grd, 32 * W, SMEM, L.stream>>>(tr, th, static_cast<T*>(L.out), L.src, L.nz, L.ny, L.nx,
                                          L.c0, L.c1, zch, zb, ze, L.err);
    return cudaGetLastError();
}

template <typename T, bool PER>
cudaError_t ring3d_cfg(const Launch& L, int variant) {
    switch (variant) {
        case 0: return ring3d_t<T, PER, 2, 4, 3>(L);
        case 1: return ring3d_t<T, PER, 2, 4, 4>(L);
        default: return ring3d_t<T, PER, 4, 4, 3>(L);
    }
}

// FORM: 0 the register-capped packed/scalar consumer, 1 the first scalar consumer, 2 form 0
// with the plane register sets rotated by name.
template <typename T, bool PER, int TY, int NWC, int STAGES, bool PACKED = true, int FORM = 0,
          int LB = 16, bool SRC = true>
cudaError_t zmarch_t_src(const Launch& L) {
    static_assert(FORM != 1 || LB == 16, "the first consumer form takes 16-byte lanes");
    using C = ZmCfg<T, TY, NWC, STAGES, LB>;
    auto pick = [] {
        if constexpr (FORM == 1) return zmarch_v1_kernel<T, PER, TY, NWC, STAGES>;
        else return zmarch_tma_kernel<T, PER, TY, NWC, STAGES, PACKED, LB, SRC, FORM == 2>;
    };
    auto kern = pick();
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
        nbl = std::max(1, nb);
        blocks_per_sm[dev].store(nbl, std::memory_order_release);
    }
    CUtensorMap tb, tr, ts;
    if (!make_map<T>(&tb, L.u, L.nz, L.ny, L.nx, C::TX, TY) ||
        !make_map<T>(&tr, L.u, L.nz, L.ny, L.nx, C::TX, 1) ||
        !make_map<T>(&ts, L.u, L.nz, L.ny, L.nx, C::HX, TY))
        return cudaErrorInvalidValue;
    ZmGeom g;
    g.nz = L.nz; g.ny = L.ny; g.nx = L.nx;
    g.ntx = (L.nx + C::TX - 1) / C::TX;
    g.nty = (L.ny + TY - 1) / TY;
    g.zbase = L.periodic ? 0 : 1;
    g.nzi = L.periodic ? L.nz : L.nz - 2;
    if (L.ze > 0) {  // a z range: planes zb-1 .. ze are inside the array, nothing wraps in z
        g.zbase = L.zb;
        g.nzi = L.ze - L.zb;
    }
    if (g.nzi <= 0) return cudaSuccess;
    const long long tiles = 1LL * g.ntx * g.nty;
    const long long resident = 1LL * sm_count() * nbl;
    int zch = L.chunk;
    if (zch <= 0) {
        // chunk-major items; one chunk of the field (read + write) kept around half of L2 so the
        // chunk-edge planes are still there when the next chunk's blocks read them, and at most
        // 32 planes so many more items than resident blocks exist (measured best at 512^3; a
        // one-wave z-slab schedule reads 2.5% less but leaves blocks idle and is slower)
        const long long plane_bytes = 1LL * L.nx * L.ny * sizeof(T);
        const long long cap = std::max(8LL, (64LL << 20) / std::max(1LL, 2 * plane_bytes));
        // small grids: shorter chunks so that there are about three items per resident block;
        // down to two planes for grids of a few tiles (128^3: 3 planes, 64^3: 2), where the
        // step time is one item's march through its chunk
        const long long fill = (1LL * g.nzi * tiles + 3 * resident - 1) / (3 * resident);
        zch = int(std::max(2LL, std::min({cap, 32LL, fill})));
        zch = std::max(1, std::min(zch, g.nzi));
    }
    g.zch = zch;
    g.nchunks = (g.nzi + zch - 1) / zch;
    const long long nitems = tiles * g.nchunks;
    if (nitems > (1LL << 30)) return cudaErrorInvalidValue;
    g.nitems = int(nitems);
    const int grid = int(std::min<long long>(nitems, 1LL * sm_count() * nbl));
    kern<<<grid, C::THREADS, C::SMEM, L.stream>>>(tb, tr, ts, static_cast<T*>(L.out), L.src, g,
                                                  L.c0, L.c1, L.err);
    return cudaGetLastError();
}

// The Jacobi source term is a compile-time choice for the register-capped consumer: without it
// the consumers carry no source prefetch registers.
template <typename T, bool PER, int TY, int NWC, int STAGES, bool PACKED = true, int FORM = 0,
          int LB = 16>
cudaError_t zmarch_t(const Launch& L) {
    if (FORM == 1 || L.src != nullptr)
        return zmarch_t_src<T, PER, TY, NWC, STAGES, PACKED, FORM, LB, true>(L);
    return zmarch_t_src<T, PER, TY, NWC, STAGES, PACKED, FORM, LB, false>(L);
}

}  // namespace

bool zmarch_tma_supported(const Launch& L) {
    const size_t es = L.storage == kF32 ? 4 : 2;
    auto al = [](const void* p) { return p == nullptr || reinterpret_cast<uintptr_t>(p) % 16 == 0; };
    return L.dims == 3 && (size_t(L.nx) * es) % 16 == 0 && al(L.u) && al(L.out) && al(L.src) &&
           L.nx >= int(16 / es) && get_encode() != nullptr;
}

// Compiled z-march configurations: rows per tile (TY), consumer warps (NWC), ring stages; L8:
// 8-byte lanes for 16-bit storage (4 values per lane: tiles half as wide, twice the rows per
// warp for the same registers; fp32 grids run the default configuration instead).
static const char* kZmNames[] = {"TY16_W8_S6", "TY8_W8_S8", "TY32_W8_S4", "TY16_W16_S6",
                                 "TY8_W4_S8", "TY16_W8_S6_scalar", "TY16_W16_S6_scalar",
                                 "TY16_W8_S6_v1", "TY16_W16_S6_v1", "TY32_W8_S6_L8",
                                 "TY16_W8_S6_L8", "TY32_W16_S6_L8", "TY16_W16_S6_rot",
                                 "TY8_W8_S8_rot", "TY16_W8_S6_rot", "TY16_W8_S6_L8_rot",
                                 "TY8_W8_S8_L8_rot"};
constexpr int kZmCount = 17;

int zmarch_configs(const char** names, int max) {
    for (int i = 0; i < kZmCount && names != nullptr && i < max; ++i) names[i] = kZmNames[i];
    return kZmCount;
}

template <typename T, bool PER>
static cudaError_t zmarch_cfg(const Launch& L) {
    int cfg = L.cfg;
    // defaults measured on a B200 at 512^3 (1000-step solves, median of 3): fp32 the scalar
    // consumer with 16 rows x 16 warps (720 GLUPS vs 686 packed), 16-bit the packed 16 x 16
    // with the plane register sets rotated by name (bf16 1238 vs 1185, fp16 1236 vs 1089)
    if (cfg < 0 || cfg >= kZmCount) cfg = sizeof(T) == 4 ? 8 : 12;
    switch (cfg) {
        case 0: return zmarch_t<T, PER, 16, 8, 6>(L);
        case 1: return zmarch_t<T, PER, 8, 8, 8>(L);
        case 2: return zmarch_t<T, PER, 32, 8, 4>(L);
        case 3: return zmarch_t<T, PER, 16, 16, 6>(L);
        case 4: return zmarch_t<T, PER, 8, 4, 8>(L);
        case 5: return zmarch_t<T, PER, 16, 8, 6, false>(L);
        case 6: return zmarch_t<T, PER, 16, 16, 6, false>(L);
        case 7: return zmarch_t<T, PER, 16, 8, 6, true, 1>(L);
        // 8-byte lanes for 16-bit storage only (an fp32 lane would hold a single pair)
        case 9:
            if constexpr (sizeof(T) == 2) return zmarch_t<T, PER, 32, 8, 6, true, 0, 8>(L);
            else return zmarch_t<T, PER, 16, 16, 6, true, 1>(L);
        case 10:
            if constexpr (sizeof(T) == 2) return zmarch_t<T, PER, 16, 8, 6, true, 0, 8>(L);
            else return zmarch_t<T, PER, 16, 16, 6, true, 1>(L);
        case 11:
            if constexpr (sizeof(T) == 2) return zmarch_t<T, PER, 32, 16, 6, true, 0, 8>(L);
            else return zmarch_t<T, PER, 16, 16, 6, true, 1>(L);
        case 12: return zmarch_t<T, PER, 16, 16, 6, true, 2>(L);
        case 13: return zmarch_t<T, PER, 8, 8, 8, true, 2>(L);
        case 14: return zmarch_t<T, PER, 16, 8, 6, true, 2>(L);
        case 15:
            if constexpr (sizeof(T) == 2) return zmarch_t<T, PER, 16, 8, 6, true, 2, 8>(L);
            else return zmarch_t<T, PER, 16, 16, 6, true, 1>(L);
        case 16:
            if constexpr (sizeof(T) == 2) return zmarch_t<T, PER, 8, 8, 8, true, 2, 8>(L);
            else return zmarch_t<T, PER, 16, 16, 6, true, 1>(L);
        default: return zmarch_t<T, PER, 16, 16, 6, true, 1>(L);
    }
}

bool ring3d_supported(const Launch& L) {
    const size_t es = L.storage == kF32 ? 4 : 2;
    auto al = [](const void* p, size_t a) {
        return p == nullptr || reinterpret_cast<uintptr_t>(p) % a == 0;
    };
    const long long n = 1LL * L.nz * L.ny * L.nx;
    return L.dims == 3 && n + 512 < (1LL << 31) && al(L.u, 16) && al(L.out, 4 * es) &&
           al(L.src, 16) && get_encode() != nullptr;
}

cudaError_t launch_ring3d(const Launch& L, int variant) {
    switch (L.storage) {
        case kF32:
            return L.periodic ? ring3d_cfg<float, true>(L, variant)
                              : ring3d_cfg<float, false>(L, variant);
        case kF16:
            return L.periodic ? ring3d_cfg<__half, true>(L, variant)
                              : ring3d_cfg<__half, false>(L, variant);
        case kBF16:
            return L.periodic ? ring3d_cfg<__nv_bfloat16, true>(L, variant)
                              : ring3d_cfg<__nv_bfloat16, false>(L, variant);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_zmarch_tma(const Launch& L) {
    switch (L.storage) {
        case kF32: return L.periodic ? zmarch_cfg<float, true>(L) : zmarch_cfg<float, false>(L);
        case kF16: return L.periodic ? zmarch_cfg<__half, true>(L) : zmarch_cfg<__half, false>(L);
        case kBF16:
            return L.periodic ? zmarch_cfg<__nv_bfloat16, true>(L)
                              : zmarch_cfg<__nv_bfloat16, false>(L);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ph3
