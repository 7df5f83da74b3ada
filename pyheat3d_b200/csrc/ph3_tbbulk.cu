// 3D temporal blocking with a bulk-copy plane ring (sm_100a).
//
// Functional spec: pyheat3d src/pyheat3d/backends/stencil.cu:178-281 (tb3d) — k updates per
// DRAM pass by a (z, t) wavefront over overlapped xy tiles; intermediate levels stay in fp32 and
// are rounded to storage once per pass (src/pyheat3d/validation.py:168-183 emulates this).
//
// Design for B200:
// * Persistent blocks walk a static list of work items (tile_x, tile_y, z-chunk), chunk
//   slowest. The chunk length is chosen on the host to balance the items over the resident
//   blocks against the 2k warm-up planes every chunk costs.
// * The level-0 planes of the block's extended tile (EX x EY sites, EX = 32 lanes x V) stream
//   into a STAGES-deep shared-memory ring with cp.async.bulk row copies (each warp copies its
//   own rows) that complete on an mbarrier. A row is one copy, split in two where
//   it crosses the periodic seam (untiled bulk copies take any 16-byte aligned source address,
//   so the wrap costs nothing); the ring holds the wrapped extended tile exactly. A stage is
//   refilled one iteration after it was read: the named barriers of that iteration already
//   order every read before the refill, so no "empty" barrier is needed.
// * The warps own R rows x V columns each. Per level they keep two planes in registers
//   (c-1 and c; c+1 is the plane the previous level produced in the same iteration), take the
//   x-neighbours from warp shuffles, the y-neighbours from their own rows and, at the warp's
//   first/last row, from a shared-memory edge exchange behind a named barrier. Math is packed
//   fp32x2, bit-identical to the scalar chain.
// * Waits are bounded. If one expires the block records the error, stops waiting (but keeps
//   every barrier so no warp is left behind), skips its stores and drains its copies.
//
// Requirements (else the plain-load tb3d kernel runs): nx * sizeof(T) % 16 == 0, 16-byte aligned
// buffers, nx >= 16 / sizeof(T).
#include <algorithm>
#include <atomic>
#include <type_traits>

#include "ph3_common.cuh"
#include "ph3_internal.h"

namespace ph3 {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// f(integral_constant<int, I>) for I = B .. E-1, unrolled at compile time.
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

struct TbGeom {
    int nz, ny, nx;
    int ntx, nty;
    int zch, nch;
    int nitems;
};

template <typename T, int K, int V, int R, int NWC, int STAGES>
struct TbCfg {
    static constexpr int G = 16 / int(sizeof(T));        // 16-byte granule in elements
    static constexpr int KX = ((K + G - 1) / G) * G;     // x halo, whole granules
    static constexpr int EX = 32 * V, OX = EX - 2 * KX;  // extended / stored tile width
    static constexpr int EY = NWC * R, OY = EY - 2 * K;  // extended / stored tile height
    static_assert(OX > 0 && OY > 0 && EX % G == 0, "tile too small for k");
    static constexpr int ROW_BYTES = EX * int(sizeof(T));
    static constexpr int PLANE_BYTES = EY * ROW_BYTES;
    static constexpr int EDGE_FLOATS = 2 * 2 * NWC * EX;  // [buffer][first/last][warp][column]
    static constexpr int SMEM = STAGES * PLANE_BYTES + EDGE_FLOATS * 4 + STAGES * 8;
    static constexpr int THREADS = 32 * NWC;
};

// V storage values of one lane from shared memory, as V/2 float2 pairs.
template <typename T, int V>
__device__ __forceinline__ void lds_lane(const T* p, float2 (&v)[V / 2]) {
    float f[V];
    ld_vec_shared<T, V>(p, f);
#pragma unroll
    for (int q = 0; q < V / 2; ++q) v[q] = make_float2(f[2 * q], f[2 * q + 1]);
}

// One lane's NP float2 pairs to / from shared memory as a single 8- or 16-byte access
// (consecutive lanes hit consecutive words: no bank conflicts).
template <int NP>
__device__ __forceinline__ void put_lane(float* p, const float2 (&v)[NP]) {
    if constexpr (NP == 2) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
    } else {
#pragma unroll
        for (int q = 0; q < NP; ++q) *reinterpret_cast<float2*>(p + 2 * q) = v[q];
    }
}
template <int NP>
__device__ __forceinline__ void get_lane(const float* p, float2 (&v)[NP]) {
    if constexpr (NP == 2) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = make_float2(t.x, t.y);
        v[1] = make_float2(t.z, t.w);
    } else {
#pragma unroll
        for (int q = 0; q < NP; ++q) v[q] = *reinterpret_cast<const float2*>(p + 2 * q);
    }
}

template <typename T, int V>
__device__ __forceinline__ void stg_lane(T* p, const float2 (&v)[V / 2]) {
    float f[V];
#pragma unroll
    for (int q = 0; q < V / 2; ++q) { f[2 * q] = v[q].x; f[2 * q + 1] = v[q].y; }
    st_vec<T, V>(p, f);
}

template <typename T, bool PER, int K, int V, int R, int NWC, int STAGES, bool SRC,
          bool SCALAR = false>
__global__ void __launch_bounds__(32 * NWC, 1)
tb3d_bulk_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b,
                 TbGeom g, float c0, float c1, int* err) {
    using C = TbCfg<T, K, V, R, NWC, STAGES>;
    constexpr int NP = V / 2, EX = C::EX, EY = C::EY, KX = C::KX, OX = C::OX, OY = C::OY;
    static_assert(V % 2 == 0, "lanes hold whole float2 pairs");
    static_assert(STAGES >= 2, "ring needs two stages");
    extern __shared__ __align__(128) unsigned char smem[];
    T* ring = reinterpret_cast<T*>(smem);
    float* edge = reinterpret_cast<float*>(smem + STAGES * C::PLANE_BYTES);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * C::PLANE_BYTES +
                                                 C::EDGE_FLOATS * 4);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], NWC);  // one arrival per warp
        fence_mbar_init();
    }
    __syncthreads();
    const int64_t P = int64_t(g.nx) * g.ny;

    // ----------------------------------------------------------------------- plane issue
    // Every warp keeps an issue cursor over the same (item, plane) sequence the block consumes
    // and copies its own R rows of each plane (lanes 0..R-1, one row each), announcing their
    // bytes on the stage's mbarrier. A stage is refilled one plane after it was consumed: by
    // then every warp has passed the named barriers of that iteration, so all reads are done.
    int is_item = blockIdx.x, is_iz = 0, is_zend = 0, is_xs = 0, is_ys = 0;
    uint32_t is_it = 0;
    auto cursor_item = [&](int item) {  // the item's tile origin, computed once per item
        if (item >= g.nitems) return;
        const int ch = item / (g.ntx * g.nty);
        const int z0 = ch * g.zch, z1 = min(z0 + g.zch, g.nz);
        is_iz = z0 - K;
        is_zend = z1 + K;
        is_xs = (item % g.ntx) * OX - KX;
        is_ys = ((item / g.ntx) % g.nty) * OY - K;
    };
    auto issue_next = [&]() {
        if (is_item >= g.nitems) return;
        const int xs = is_xs, ys = is_ys;
        const int s = is_it % STAGES;
        const int pz = PER ? wrap_near(is_iz, g.nz) : clamp_idx(is_iz, 0, g.nz - 1);
        if (lane == 0) mbar_arrive_expect_tx(&full[s], R * C::ROW_BYTES);
        __syncwarp();
        T* plane = ring + s * (EY * EX);
        for (int r = warp * R + lane; r < warp * R + R && lane < R; r += 32) {
            const int gy = PER ? wrap_near(ys + r, g.ny) : clamp_idx(ys + r, 0, g.ny - 1);
            const T* row = u + int64_t(pz) * P + int64_t(gy) * g.nx;
            T* dst = plane + r * EX;
            int done = 0;
            while (done < EX) {
                const int x = xs + done;
                int src, len;
                if (PER) {
                    src = wrap_near(x, g.nx);
                    len = min(EX - done, g.nx - src);
                } else if (x < 0) {  // outside the domain: any in-range data will do
                    src = 0;
                    len = min(min(EX - done, -x), g.nx);
                } else if (x >= g.nx) {
                    src = 0;
                    len = min(EX - done, g.nx);
                } else {
                    src = x;
                    len = min(EX - done, g.nx - x);
                }
                bulk_load(dst + done, row + src, uint32_t(len) * sizeof(T), &full[s]);
                done += len;
            }
        }
        ++is_it;
        if (++is_iz >= is_zend) {
            is_item += gridDim.x;
            cursor_item(is_item);
        }
    };
    cursor_item(is_item);
    for (int i = 0; i < STAGES - 1; ++i) issue_next();

    // ------------------------------------------------------------------------ all warps
    const float2 c0v = make_float2(c0, c0), c1v = make_float2(c1, c1);
    const int lx = lane * V;
    uint32_t it = 0, waited = 0;  // planes consumed / planes whose copies were seen to land
    int buf = 0;
    bool ok = true;
    float2 A[K][R][NP], B[K][R][NP];  // level s: plane c (A) and c-1 (B)

    for (int item = blockIdx.x; item < g.nitems; item += gridDim.x) {
        const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty, ch = item / (g.ntx * g.nty);
        const int xs = tx * OX - KX, ys = ty * OY - K;
        const int z0 = ch * g.zch, z1 = min(z0 + g.zch, g.nz);
        const int gx = xs + lx, gy0 = ys + warp * R;
        uint32_t fixx = 0, fixy = 0;  // Dirichlet: boundary / outside sites keep their value
        if constexpr (!PER) {
#pragma unroll
            for (int j = 0; j < V; ++j)
                if (gx + j <= 0 || gx + j >= g.nx - 1) fixx |= 1u << j;
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (gy0 + r <= 0 || gy0 + r >= g.ny - 1) fixy |= 1u << r;
        }
        const bool xwriter = lx >= KX && lx < KX + OX && gx < g.nx;
        const int bcol = PER ? wrap_near(gx, g.nx) : clamp_idx(gx, 0, g.nx - V);
#pragma unroll
        for (int s = 0; s < K; ++s)
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int p = 0; p < NP; ++p) A[s][r][p] = B[s][r][p] = make_float2(0.f, 0.f);

        auto step = [&](int iz, float2 (&Bp)[K][R][NP], float2 (&Ap)[K][R][NP]) {
            if (ok) issue_next();
            const int s = it % STAGES;
            if (ok) {
                if (mbar_wait(&full[s], (it / STAGES) & 1u, err)) ++waited;
                else ok = false;
            }
            float2 N[R][NP];
            const T* plane = ring + s * (EY * EX);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (ok) {
                    lds_lane<T, V>(plane + (warp * R + r) * EX + lx, N[r]);
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p) N[r][p] = make_float2(0.f, 0.f);
                }
            }

#pragma unroll
            for (int lev = 1; lev <= K; ++lev) {
                const int c = iz - lev;
                // y-neighbours of the first / last row: exchange with the adjacent warps
                float* eb = edge + buf * (2 * NWC * EX);
                put_lane<NP>(eb + warp * EX + lx, Ap[lev - 1][0]);
                put_lane<NP>(eb + (NWC + warp) * EX + lx, Ap[lev - 1][R - 1]);
                named_sync(1, NWC * 32);
                float2 up[NP], dn[NP];
                if (warp > 0) {
                    get_lane<NP>(eb + (NWC + warp - 1) * EX + lx, up);
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p) up[p] = Ap[lev - 1][0][p];
                }
                if (warp < NWC - 1) {
                    get_lane<NP>(eb + (warp + 1) * EX + lx, dn);
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p) dn[p] = Ap[lev - 1][R - 1][p];
                }
                buf ^= 1;
                const bool zfix = !PER && (c <= 0 || c >= g.nz - 1);
                const float* bpl = nullptr;
                if constexpr (SRC)
                    bpl = b + int64_t(PER ? wrap_near(c, g.nz) : clamp_idx(c, 0, g.nz - 1)) * P;
                float2 res[R][NP];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const float left = __shfl_up_sync(kFull, Ap[lev - 1][r][NP - 1].y, 1);
                    const float right = __shfl_down_sync(kFull, Ap[lev - 1][r][0].x, 1);
                    float2 bv[NP];
                    if constexpr (SRC) {
                        const int gy = PER ? wrap_near(gy0 + r, g.ny) : clamp_idx(gy0 + r, 0, g.ny - 1);
                        float f[V];
                        ld_vec<float, V>(bpl + int64_t(gy) * g.nx + bcol, f);
#pragma unroll
                        for (int p = 0; p < NP; ++p) bv[p] = make_float2(f[2 * p], f[2 * p + 1]);
                    }
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
                        const float2 ctr = Ap[lev - 1][r][p];
                        // x-neighbour sums by scalar adds straight into a register pair (no
                        // pairs of misaligned neighbours to assemble)
                        const float xl = p > 0 ? Ap[lev - 1][r][p - 1].y : left;
                        const float xr = p < NP - 1 ? Ap[lev - 1][r][p + 1].x : right;
                        const float2 ym = r > 0 ? Ap[lev - 1][r - 1][p] : up[p];
                        const float2 yp = r < R - 1 ? Ap[lev - 1][r + 1][p] : dn[p];
                        float2 v;
                        if constexpr (SCALAR) {  // the same canonical chain site by site
                            const float2 zm = Bp[lev - 1][r][p], zp = N[r][p];
                            v.x = upd3(c0, c1, ctr.x, xl, ctr.y, ym.x, yp.x, zm.x, zp.x);
                            v.y = upd3(c0, c1, ctr.y, ctr.x, xr, ym.y, yp.y, zm.y, zp.y);
                            if constexpr (SRC) {
                                v.x = __fadd_rn(v.x, bv[p].x);
                                v.y = __fadd_rn(v.y, bv[p].y);
                            }
                        } else {
                            const float2 sx =
                                make_float2(__fadd_rn(xl, ctr.y), __fadd_rn(ctr.x, xr));
                            v = upd3_sx2(c0v, c1v, ctr, sx, ym, yp, Bp[lev - 1][r][p], N[r][p]);
                            if constexpr (SRC) v = add2(v, bv[p]);
                        }
                        if constexpr (!PER) {
                            const bool fr = zfix || ((fixy >> r) & 1u);
                            if (fr || ((fixx >> (2 * p)) & 1u)) v.x = ctr.x;
                            if (fr || ((fixx >> (2 * p + 1)) & 1u)) v.y = ctr.y;
                        }
                        res[r][p] = v;
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
                        Bp[lev - 1][r][p] = Ap[lev - 1][r][p];
                        Ap[lev - 1][r][p] = N[r][p];
                        N[r][p] = res[r][p];
                    }
            }
            // N now holds level K of plane iz - K
            const int c = iz - K;
            if (ok && xwriter && c >= z0 && c < z1 && (PER || (c > 0 && c < g.nz - 1))) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int row = warp * R + r, gy = gy0 + r;
                    if (row < K || row >= K + OY || gy >= g.ny || ((fixy >> r) & 1u)) continue;
                    T* dst = o + int64_t(c) * P + int64_t(gy) * g.nx + gx;
                    if (fixx == 0 && gx + V <= g.nx) {
                        stg_lane<T, V>(dst, N[r]);
                    } else {
#pragma unroll
                        for (int p = 0; p < NP; ++p) {
                            const int j = 2 * p;
                            if (gx + j < g.nx && !((fixx >> j) & 1u)) dst[j] = from_f<T>(N[r][p].x);
                            if (gx + j + 1 < g.nx && !((fixx >> (j + 1)) & 1u))
                                dst[j + 1] = from_f<T>(N[r][p].y);
                        }
                    }
                }
            }
            ++it;
        };
        for (int iz = z0 - K; iz < z1 + K; ++iz) step(iz, B, A);
    }

    // every plane this warp issued must land before the block exits (normally all were consumed)
    if (lane == 0) {
        for (uint32_t k = waited; k < is_it; ++k)
            if (!mbar_wait(&full[k % STAGES], (k / STAGES) & 1u, err)) break;
    }
}

// Second form: level 0 is read straight from the ring (no register copies of its planes) and
// the planes of levels 1 .. k-1 live in three register sets per level that rotate by name: plane
// c of level s sits in set c mod 3, the march is unrolled three planes per loop pass so every
// set index is a compile-time constant, and no plane is ever copied. The ring keeps the three
// level-0 planes of a step resident (STAGES >= AHEAD + 3 with AHEAD planes in flight); level 1
// takes the y-neighbours of a warp's first and last rows from the neighbouring warps' rows in the
// ring, so only levels 2 .. k exchange edge rows through shared memory.
template <typename T, bool PER, int K, int V, int R, int NWC, int STAGES, bool SRC>
__global__ void __launch_bounds__(32 * NWC, 1)
tb3d_rot_kernel(const T* __restrict__ u, T* __restrict__ o, const float* __restrict__ b,
                TbGeom g, float c0, float c1, int* err) {
    using C = TbCfg<T, K, V, R, NWC, STAGES>;
    constexpr int NP = V / 2, EX = C::EX, EY = C::EY, KX = C::KX, OX = C::OX, OY = C::OY;
    constexpr int AHEAD = STAGES - 3;  // planes issued ahead of the one being consumed
    constexpr int NL = K > 1 ? K - 1 : 1;  // register-resident levels 1 .. k-1
    static_assert(V % 2 == 0, "lanes hold whole float2 pairs");
    static_assert(AHEAD >= 1, "the ring needs three resident planes and one in flight");
    static_assert(K >= 2, "temporal blocking fuses at least two steps");
    extern __shared__ __align__(128) unsigned char smem[];
    T* ring = reinterpret_cast<T*>(smem);
    float* edge = reinterpret_cast<float*>(smem + STAGES * C::PLANE_BYTES);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * C::PLANE_BYTES +
                                                 C::EDGE_FLOATS * 4);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], NWC);  // one arrival per warp
        fence_mbar_init();
    }
    __syncthreads();
    const int64_t P = int64_t(g.nx) * g.ny;

    // ---- plane issue: every warp copies its own R rows of each plane, as in the first form
    int is_item = blockIdx.x, is_iz = 0, is_zend = 0, is_xs = 0, is_ys = 0;
    uint32_t is_it = 0;
    auto cursor_item = [&](int item) {
        if (item >= g.nitems) return;
        const int ch = item / (g.ntx * g.nty);
        const int z0 = ch * g.zch, z1 = min(z0 + g.zch, g.nz);
        is_iz = z0 - K;
        is_zend = z1 + K;
        is_xs = (item % g.ntx) * OX - KX;
        is_ys = ((item / g.ntx) % g.nty) * OY - K;
    };
    auto issue_next = [&]() {
        if (is_item >= g.nitems) return;
        const int xs = is_xs, ys = is_ys;
        const int s = is_it % STAGES;
        const int pz = PER ? wrap_near(is_iz, g.nz) : clamp_idx(is_iz, 0, g.nz - 1);
        if (lane == 0) mbar_arrive_expect_tx(&full[s], R * C::ROW_BYTES);
        __syncwarp();
        T* plane = ring + s * (EY * EX);
        for (int r = warp * R + lane; r < warp * R + R && lane < R; r += 32) {
            const int gy = PER ? wrap_near(ys + r, g.ny) : clamp_idx(ys + r, 0, g.ny - 1);
            const T* row = u + int64_t(pz) * P + int64_t(gy) * g.nx;
            T* dst = plane + r * EX;
            int done = 0;
            while (done < EX) {
                const int x = xs + done;
                int src, len;
                if (PER) {
                    src = wrap_near(x, g.nx);
                    len = min(EX - done, g.nx - src);
                } else if (x < 0) {
                    src = 0;
                    len = min(min(EX - done, -x), g.nx);
                } else if (x >= g.nx) {
                    src = 0;
                    len = min(EX - done, g.nx);
                } else {
                    src = x;
                    len = min(EX - done, g.nx - x);
                }
                bulk_load(dst + done, row + src, uint32_t(len) * sizeof(T), &full[s]);
                done += len;
            }
        }
        ++is_it;
        if (++is_iz >= is_zend) {
            is_item += gridDim.x;
            cursor_item(is_item);
        }
    };
    cursor_item(is_item);
    for (int i = 0; i < AHEAD; ++i) issue_next();

    const float2 c0v = make_float2(c0, c0), c1v = make_float2(c1, c1);
    const int lx = lane * V;
    const int r0 = warp * R;  // first tile row of this warp
    uint32_t it = 0, waited = 0;
    int buf = 0;
    bool ok = true;
    float2 Lv[NL][3][R][NP];  // level s (1 .. k-1): plane c in set c mod 3

    for (int item = blockIdx.x; item < g.nitems; item += gridDim.x) {
        const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty, ch = item / (g.ntx * g.nty);
        const int xs = tx * OX - KX, ys = ty * OY - K;
        const int z0 = ch * g.zch, z1 = min(z0 + g.zch, g.nz);
        const int gx = xs + lx, gy0 = ys + r0;
        uint32_t fixx = 0, fixy = 0;
        if constexpr (!PER) {
#pragma unroll
            for (int j = 0; j < V; ++j)
                if (gx + j <= 0 || gx + j >= g.nx - 1) fixx |= 1u << j;
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (gy0 + r <= 0 || gy0 + r >= g.ny - 1) fixy |= 1u << r;
        }
        const bool xwriter = lx >= KX && lx < KX + OX && gx < g.nx;
        const int bcol = PER ? wrap_near(gx, g.nx) : clamp_idx(gx, 0, g.nx - V);
#pragma unroll
        for (int s = 0; s < NL; ++s)
#pragma unroll
            for (int q = 0; q < 3; ++q)
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int p = 0; p < NP; ++p) Lv[s][q][r][p] = make_float2(0.f, 0.f);

        // One update of R rows: centre rows `ctr`, y-neighbours of the first / last row `up` /
        // `dn`, z-neighbours `zm` / `zp`, result into `res` (plane c of the new level).
        auto update = [&](const float2 (&ctr)[R][NP], const float2 (&up)[NP],
                          const float2 (&dn)[NP], const float2 (&zm)[R][NP],
                          const float2 (&zp)[R][NP], int c, float2 (&res)[R][NP]) {
            const bool zfix = !PER && (c <= 0 || c >= g.nz - 1);
            const float* bpl = nullptr;
            if constexpr (SRC)
                bpl = b + int64_t(PER ? wrap_near(c, g.nz) : clamp_idx(c, 0, g.nz - 1)) * P;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float left = __shfl_up_sync(kFull, ctr[r][NP - 1].y, 1);
                const float right = __shfl_down_sync(kFull, ctr[r][0].x, 1);
                float2 bv[NP];
                if constexpr (SRC) {
                    const int gy = PER ? wrap_near(gy0 + r, g.ny) : clamp_idx(gy0 + r, 0, g.ny - 1);
                    float f[V];
                    ld_vec<float, V>(bpl + int64_t(gy) * g.nx + bcol, f);
#pragma unroll
                    for (int p = 0; p < NP; ++p) bv[p] = make_float2(f[2 * p], f[2 * p + 1]);
                }
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    const float2 cc = ctr[r][p];
                    const float xl = p > 0 ? ctr[r][p - 1].y : left;
                    const float xr = p < NP - 1 ? ctr[r][p + 1].x : right;
                    const float2 sx = make_float2(__fadd_rn(xl, cc.y), __fadd_rn(cc.x, xr));
                    const float2 ym = r > 0 ? ctr[r - 1][p] : up[p];
                    const float2 yp = r < R - 1 ? ctr[r + 1][p] : dn[p];
                    float2 v = upd3_sx2(c0v, c1v, cc, sx, ym, yp, zm[r][p], zp[r][p]);
                    if constexpr (SRC) v = add2(v, bv[p]);
                    if constexpr (!PER) {
                        const bool fr = zfix || ((fixy >> r) & 1u);
                        if (fr || ((fixx >> (2 * p)) & 1u)) v.x = cc.x;
                        if (fr || ((fixx >> (2 * p + 1)) & 1u)) v.y = cc.y;
                    }
                    res[r][p] = v;
                }
            }
        };
        auto store = [&](int c, const float2 (&v)[R][NP]) {
            if (!ok || !xwriter || c < z0 || c >= z1 || (!PER && (c <= 0 || c >= g.nz - 1))) return;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int row = r0 + r, gy = gy0 + r;
                if (row < K || row >= K + OY || gy >= g.ny || ((fixy >> r) & 1u)) continue;
                T* dst = o + int64_t(c) * P + int64_t(gy) * g.nx + gx;
                if (fixx == 0 && gx + V <= g.nx) {
                    stg_lane<T, V>(dst, v[r]);
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
                        const int j = 2 * p;
                        if (gx + j < g.nx && !((fixx >> j) & 1u)) dst[j] = from_f<T>(v[r][p].x);
                        if (gx + j + 1 < g.nx && !((fixx >> (j + 1)) & 1u))
                            dst[j + 1] = from_f<T>(v[r][p].y);
                    }
                }
            }
        };
        // level-0 rows of this warp (and, for level 1, the neighbouring rows) from ring stage s
        auto ring_row = [&](int s, int row, float2 (&v)[NP]) {
            if (ok) {
                lds_lane<T, V>(ring + s * (EY * EX) + row * EX + lx, v);
            } else {
#pragma unroll
                for (int p = 0; p < NP; ++p) v[p] = make_float2(0.f, 0.f);
            }
        };

        // One step of the march: level-0 plane iz lands; level s = 1 .. k makes plane iz - s.
        // PH = (iz - first plane) mod 3 at compile time: plane iz - s of level s sits in set
        // (PH - s) mod 3.
        auto step = [&](auto ph_tag, int iz) {
            constexpr int PH = decltype(ph_tag)::value;
            if (ok) issue_next();
            const int sa = it % STAGES;  // plane iz
            if (ok) {
                if (mbar_wait(&full[sa], (it / STAGES) & 1u, err)) ++waited;
                else ok = false;
            }
            const int sc = (it + STAGES - 1) % STAGES;  // plane iz - 1
            const int sb = (it + STAGES - 2) % STAGES;  // plane iz - 2
            // ---- level 1: plane iz - 1 straight from the ring
            {
                float2 ctr[R][NP], zm[R][NP], zp[R][NP], up[NP], dn[NP];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    ring_row(sc, r0 + r, ctr[r]);
                    ring_row(sb, r0 + r, zm[r]);
                    ring_row(sa, r0 + r, zp[r]);
                }
                ring_row(sc, warp > 0 ? r0 - 1 : r0, up);
                ring_row(sc, warp < NWC - 1 ? r0 + R : r0 + R - 1, dn);
                constexpr int q = ((PH - 1) % 3 + 3) % 3;
                update(ctr, up, dn, zm, zp, iz - 1, Lv[0][q]);
            }
            // ---- levels 2 .. k: from the previous level's three sets
            auto level = [&](auto s_tag) {
                constexpr int S = decltype(s_tag)::value;
                constexpr int qc = ((PH - S) % 3 + 3) % 3;      // plane iz - S (centre)
                constexpr int qb = ((PH - S - 1) % 3 + 3) % 3;  // plane iz - S - 1 (below)
                constexpr int qa = ((PH - S + 1) % 3 + 3) % 3;  // plane iz - S + 1 (above)
                const float2 (&ctr)[R][NP] = Lv[S - 2][qc];
                float* eb = edge + buf * (2 * NWC * EX);
                put_lane<NP>(eb + warp * EX + lx, ctr[0]);
                put_lane<NP>(eb + (NWC + warp) * EX + lx, ctr[R - 1]);
                named_sync(1, NWC * 32);
                float2 up[NP], dn[NP];
                if (warp > 0) {
                    get_lane<NP>(eb + (NWC + warp - 1) * EX + lx, up);
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p) up[p] = ctr[0][p];
                }
                if (warp < NWC - 1) {
                    get_lane<NP>(eb + (warp + 1) * EX + lx, dn);
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p) dn[p] = ctr[R - 1][p];
                }
                buf ^= 1;
                if constexpr (S < K) {
                    update(ctr, up, dn, Lv[S - 2][qb], Lv[S - 2][qa], iz - S, Lv[S - 1][qc]);
                } else {
                    float2 res[R][NP];
                    update(ctr, up, dn, Lv[S - 2][qb], Lv[S - 2][qa], iz - S, res);
                    store(iz - S, res);
                }
            };
            static_for<2, K + 1>(level);
            ++it;
        };
        // the sets are named by the plane's offset from the item's first plane, mod 3 (the
        // item's first 2k steps fill them, so nothing carries over from the previous item)
        for (int iz = z0 - K; iz < z1 + K;) {
            step(std::integral_constant<int, 0>{}, iz);
            if (++iz >= z1 + K || !ok) break;
            step(std::integral_constant<int, 1>{}, iz);
            if (++iz >= z1 + K || !ok) break;
            step(std::integral_constant<int, 2>{}, iz);
            if (++iz >= z1 + K || !ok) break;
        }
        if (!ok) break;
    }

    // every plane this warp issued must land before the block exits (normally all were consumed)
    if (lane == 0) {
        for (uint32_t k = waited; k < is_it; ++k)
            if (!mbar_wait(&full[k % STAGES], (k / STAGES) & 1u, err)) break;
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

// Chunk length minimising the per-block critical path ceil(items / blocks) * (zch + 2k).
int balanced_chunk(int nz, long long tiles, long long blocks, int k) {
    int best = nz;
    double best_cost = 1e300;
    const int max_ch = std::max(1, nz / std::max(2 * k, 4));
    for (int nch = 1; nch <= max_ch; ++nch) {
        const int zch = (nz + nch - 1) / nch;
        const int real_nch = (nz + zch - 1) / zch;
        const long long items = tiles * real_nch;
        const double waves = double((items + blocks - 1) / blocks);
        const double cost = waves * (zch + 2.0 * k);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = zch;
        }
    }
    return best;
}

template <typename T, bool PER, int K, int V, int R, int NWC, int STAGES, bool SRC, int FORM>
cudaError_t tbbulk_src(const Launch& L) {
    using C = TbCfg<T, K, V, R, NWC, STAGES>;
    auto pick = [] {
        if constexpr (FORM == 1) return tb3d_rot_kernel<T, PER, K, V, R, NWC, STAGES, SRC>;
        else return tb3d_bulk_kernel<T, PER, K, V, R, NWC, STAGES, SRC, FORM == 2>;
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
        if (nb < 1) return cudaErrorInvalidConfiguration;
        nbl = nb;
        blocks_per_sm[dev].store(nbl, std::memory_order_release);
    }
    TbGeom g;
    g.nz = L.nz; g.ny = L.ny; g.nx = L.nx;
    g.ntx = (L.nx + C::OX - 1) / C::OX;
    g.nty = (L.ny + C::OY - 1) / C::OY;
    const long long tiles = 1LL * g.ntx * g.nty;
    const long long blocks = 1LL * sm_count() * nbl;
    g.zch = L.chunk > 0 ? std::min(L.chunk, L.nz) : balanced_chunk(L.nz, tiles, blocks, K);
    g.nch = (L.nz + g.zch - 1) / g.zch;
    const long long items = tiles * g.nch;
    if (items > (1LL << 30)) return cudaErrorInvalidValue;
    if (L.geo != nullptr) {
        L.geo[0] = C::EX; L.geo[1] = C::EY; L.geo[2] = g.zch;
        return cudaSuccess;
    }
    g.nitems = int(items);
    const int grid = int(std::min(items, blocks));
    kern<<<grid, C::THREADS, C::SMEM, L.stream>>>(static_cast<const T*>(L.u),
                                                  static_cast<T*>(L.out), L.src, g, L.c0, L.c1,
                                                  L.err);
    return cudaGetLastError();
}

// The Jacobi source is a compile-time choice: without it the kernel carries neither its loads
// nor the branches around them. FORM: 0 the first form, 1 the second (rotating) form, 2 the
// first form with scalar arithmetic.
template <typename T, bool PER, int K, int V, int R, int NWC, int STAGES, int FORM = 0>
cudaError_t tbbulk_t(const Launch& L) {
    if (L.src != nullptr) return tbbulk_src<T, PER, K, V, R, NWC, STAGES, true, FORM>(L);
    return tbbulk_src<T, PER, K, V, R, NWC, STAGES, false, FORM>(L);
}

// Compiled configurations per k: (V values per lane, R rows per warp, consumer warps, stages).
struct TbEntry {
    int k;
    const char* name;
};
const TbEntry kTbNames[] = {
    {2, "V4_R2_W16_S4"}, {2, "V4_R4_W8_S4"},  {3, "V4_R2_W16_S4"}, {3, "V4_R4_W8_S4"},
    {4, "V4_R2_W16_S4"}, {4, "V2_R2_W16_S6"}, {8, "V2_R2_W16_S6"}, {8, "V2_R4_W8_S6"},
    // 64-row tiles of 8-byte lane vectors: less y overlap, more shuffles (fastest fp32 tb3)
    {3, "V2_R4_W16_S4"}, {4, "V2_R4_W16_S4"},
    // second form: level 0 from the ring, rotating plane sets (no plane copies)
    {2, "rot_V4_R2_W16_S5"}, {3, "rot_V4_R2_W16_S5"}, {3, "rot_V2_R4_W16_S5"},
    {4, "rot_V4_R2_W16_S5"}, {4, "rot_V2_R4_W16_S5"}, {8, "rot_V2_R2_W16_S5"},
    // first form, scalar arithmetic
    {2, "V4_R2_W16_S4_scalar"}, {3, "V2_R4_W16_S4_scalar"}, {4, "V2_R4_W16_S4_scalar"},
    {4, "V4_R2_W16_S4_scalar"}, {8, "V2_R2_W16_S6_scalar"},
};

template <typename T, bool PER>
cudaError_t tbbulk_dispatch(const Launch& L) {
    const int cfg = L.cfg < 0 ? 0 : L.cfg;
    switch (L.k) {
        case 2:
            if (cfg == 2) return tbbulk_t<T, PER, 2, 4, 2, 16, 5, 1>(L);
            if (cfg == 3) return tbbulk_t<T, PER, 2, 4, 2, 16, 4, 2>(L);
            return cfg == 1 ? tbbulk_t<T, PER, 2, 4, 4, 8, 4>(L) : tbbulk_t<T, PER, 2, 4, 2, 16, 4>(L);
        case 3:
            if (cfg == 2) return tbbulk_t<T, PER, 3, 2, 4, 16, 4>(L);
            if (cfg == 3) return tbbulk_t<T, PER, 3, 4, 2, 16, 5, 1>(L);
            if (cfg == 4) return tbbulk_t<T, PER, 3, 2, 4, 16, 5, 1>(L);
            if (cfg == 5) return tbbulk_t<T, PER, 3, 2, 4, 16, 4, 2>(L);
            return cfg == 1 ? tbbulk_t<T, PER, 3, 4, 4, 8, 4>(L) : tbbulk_t<T, PER, 3, 4, 2, 16, 4>(L);
        case 4:
            if (cfg == 2) return tbbulk_t<T, PER, 4, 2, 4, 16, 4>(L);
            if (cfg == 3) return tbbulk_t<T, PER, 4, 4, 2, 16, 5, 1>(L);
            if (cfg == 4) return tbbulk_t<T, PER, 4, 2, 4, 16, 5, 1>(L);
            if (cfg == 5) return tbbulk_t<T, PER, 4, 2, 4, 16, 4, 2>(L);
            if (cfg == 6) return tbbulk_t<T, PER, 4, 4, 2, 16, 4, 2>(L);
            return cfg == 1 ? tbbulk_t<T, PER, 4, 2, 2, 16, 6>(L) : tbbulk_t<T, PER, 4, 4, 2, 16, 4>(L);
        case 8:
            if (cfg == 2) return tbbulk_t<T, PER, 8, 2, 2, 16, 5, 1>(L);
            if (cfg == 3) return tbbulk_t<T, PER, 8, 2, 2, 16, 6, 2>(L);
            return cfg == 1 ? tbbulk_t<T, PER, 8, 2, 4, 8, 6>(L) : tbbulk_t<T, PER, 8, 2, 2, 16, 6>(L);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int tbbulk_configs(int k, const char** names, int max) {
    int n = 0;
    for (const auto& e : kTbNames)
        if (e.k == k) {
            if (names != nullptr && n < max) names[n] = e.name;
            ++n;
        }
    return n;
}

bool tbbulk_supported(const Launch& L) {
    const size_t es = L.storage == kF32 ? 4 : 2;
    auto al = [](const void* p) { return p == nullptr || reinterpret_cast<uintptr_t>(p) % 16 == 0; };
    return L.dims == 3 && (size_t(L.nx) * es) % 16 == 0 && L.nx >= int(16 / es) && al(L.u) &&
           al(L.out) && al(L.src);
}

cudaError_t launch_tbbulk(const Launch& L) {
    switch (L.storage) {
        case kF32: return L.periodic ? tbbulk_dispatch<float, true>(L) : tbbulk_dispatch<float, false>(L);
        case kF16: return L.periodic ? tbbulk_dispatch<__half, true>(L) : tbbulk_dispatch<__half, false>(L);
        case kBF16:
            return L.periodic ? tbbulk_dispatch<__nv_bfloat16, true>(L)
                              : tbbulk_dispatch<__nv_bfloat16, false>(L);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ph3
