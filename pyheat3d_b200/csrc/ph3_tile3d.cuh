// 3D single step for any row alignment with block-wide shared-memory plane tiles (sm_100a).
//
// Functional spec: pyheat3d src/pyheat3d/backends/stencil.cu:101-161 (zmarch3d) — one update
// of the 7-point stencil per launch, u' = c0 u + c1 (sum of the six neighbours) (+ b), periodic
// wrap or fixed Dirichlet boundary (src/pyheat3d/numpy_ref.py:25-45); the summation order is the
// canonical one of upd3.
//
// Design: a block of eight warps owns a 64 x 32 column tile (warp w: rows 4w .. 4w+3; lane:
// columns lane and lane + 32) and marches it through a chunk of planes. Every thread loads its
// own eight sites of a plane with coalesced element loads (a warp row access is 32 consecutive
// elements whatever the row alignment) plus at most one element of the tile's one-site halo
// ring, two planes ahead of the plane it updates. Planes pass through a four-slot ring of fp32
// plane tiles in shared memory: a thread stores plane z+1 into its slot, one block barrier, then
// updates plane z reading its centre values, x- and y-neighbours from slot z and its lower
// neighbours from slot z-1; the upper neighbours are the registers it just stored. With four
// slots one barrier per plane orders every store after the last reads of that slot (plane z-3,
// read while updating plane z-2). Two register planes per thread (the one being stored, the one
// in flight) keep the item within 80 registers. All addressing is per item (row offsets, wrapped
// or clamped halo offsets), so the per-plane work is the loads, shared-memory traffic and packed
// arithmetic of the sites.
#pragma once

#include "ph3_common.cuh"

namespace ph3 {

template <bool B> struct BoolTag { static constexpr bool value = B; };

struct Tile3 {
    static constexpr int R = 4;                      // rows per warp
    static constexpr int W = 8;                      // warps per block
    static constexpr int OX = 64, OY = W * R;        // stored columns / rows of a tile
    static constexpr int SX = OX + 2, SY = OY + 2;   // shared-memory plane tile with halo
    static constexpr int PLANE = SX * SY;            // fp32 words per slot
    static constexpr int HALO = 2 * OX + 2 * SY;     // halo elements per plane
    static constexpr int SLOTS = 4;
    static constexpr int SMEM = SLOTS * PLANE * 4;   // bytes
    static_assert(HALO <= 32 * W, "one halo element per thread at most");
};

// One item: tile (tx, ty) of planes zlo .. zhi-1 from u into o. `sm` is Tile3::SMEM bytes of
// shared memory (16-byte aligned); the caller separates items of one block by a barrier. CG:
// field loads through L2 only (buffers other blocks of the same launch write).
template <typename T, bool PER, bool SRC, bool CG>
__device__ __forceinline__ void tile3d_item(const T* __restrict__ u, T* __restrict__ o,
                                            const float* __restrict__ b, int nz, int ny, int nx,
                                            float c0, float c1, int tx, int ty, int zlo, int zhi,
                                            float* __restrict__ sm) {
    using C = Tile3;
    constexpr int R = C::R, SX = C::SX;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, t = threadIdx.x;
    // the last tile of a row or column of tiles ends at the grid's edge, overlapping its
    // neighbour (the overlap is computed twice and stored twice with the same values), so every
    // tile of a grid at least one tile wide lies inside the grid
    const int x0 = nx >= C::OX ? min(tx * C::OX, nx - C::OX) : tx * C::OX;
    const int y0 = ny >= C::OY ? min(ty * C::OY, ny - C::OY) : ty * C::OY;
    if constexpr (!PER) { zlo = max(zlo, 1); zhi = min(zhi, nz - 1); }
    if (zlo >= zhi) return;  // block-uniform
    const int64_t P = int64_t(nx) * ny;
    auto fx = [&](int i, int n) {
        if constexpr (PER) return wrap_near(i, n);
        else return clamp_idx(i, 0, n - 1);
    };

    // own sites: rows y0 + 4w + r, columns x0 + lane + 32 j
    int roff[R], cx[2];
    uint32_t store = 0;  // bit 2r + j: site is stored (inside the grid, not a fixed boundary)
    uint32_t fixm = 0;   // bit 2r + j: Dirichlet boundary site inside the grid (keeps its value)
#pragma unroll
    for (int j = 0; j < 2; ++j) cx[j] = fx(x0 + lane + 32 * j, nx);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int y = y0 + w * R + r;
        roff[r] = fx(y, ny) * nx;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int x = x0 + lane + 32 * j;
            bool ok = x < nx && y < ny;
            if constexpr (!PER) {
                if (ok && (x == 0 || x == nx - 1 || y == 0 || y == ny - 1))
                    fixm |= 1u << (2 * r + j);
                ok = ok && x > 0 && x < nx - 1 && y > 0 && y < ny - 1;
            }
            if (ok) store |= 1u << (2 * r + j);
        }
    }
    // halo: top row, bottom row (columns x0 .. x0+63), left and right columns (rows y0-1 ..
    // y0+32); thread t < HALO holds one element
    const bool has_h = t < C::HALO;
    int hoff = 0, hs = 0;
    if (has_h) {
        int qy, qx;  // tile coordinates, 0 .. SY-1 / 0 .. SX-1
        if (t < C::OX) { qy = 0; qx = t + 1; }
        else if (t < 2 * C::OX) { qy = C::SY - 1; qx = t - C::OX + 1; }
        else if (t < 2 * C::OX + C::SY) { qy = t - 2 * C::OX; qx = 0; }
        else { qy = t - 2 * C::OX - C::SY; qx = SX - 1; }
        hoff = fx(y0 + qy - 1, ny) * nx + fx(x0 + qx - 1, nx);
        hs = qy * SX + qx;
    }
    const int own0 = (w * R + 1) * SX + lane + 1;  // slot index of (row 0, column j = 0)

    struct Plane {
        float2 v[R];  // (column lane, column lane + 32) of each own row
        float h;
    };
    // A tile inside the grid (FULL: every tile of a grid at least 64 x 32): row r of this warp
    // starts nx elements after row r-1 and column lane + 32 is 32 elements after column lane,
    // so loads and stores walk one pointer with constant offsets, and every own site is stored;
    // a Dirichlet boundary site stores its own unchanged value (the other buffer holds the same
    // boundary values). Other tiles take per-site offsets and store masks.
    const bool full = x0 + C::OX <= nx && y0 + C::OY <= ny;
    const int base0 = roff[0] + cx[0];

    auto run = [&](auto full_tag) {
        constexpr bool FULL = decltype(full_tag)::value;
        auto load = [&](int z, Plane& p) {
            const T* pl = u + int64_t(PER ? wrap_near(z, nz) : z) * P;
            if constexpr (FULL) {
                const T* q = pl + base0;
#pragma unroll
                for (int r = 0; r < R; ++r, q += nx)
                    p.v[r] = make_float2(ldx1<CG>(q), ldx1<CG>(q + 32));
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    p.v[r] = make_float2(ldx1<CG>(pl + roff[r] + cx[0]),
                                         ldx1<CG>(pl + roff[r] + cx[1]));
            }
            p.h = has_h ? ldx1<CG>(pl + hoff) : 0.f;
        };
        auto put = [&](const Plane& p, float* slot, bool halo) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                slot[own0 + r * SX] = p.v[r].x;
                slot[own0 + r * SX + 32] = p.v[r].y;
            }
            if (halo && has_h) slot[hs] = p.h;
        };
        // plane p lives in slot (p - zlo + 1) mod 4
        auto slot = [&](int p) { return sm + ((p - zlo + 1) & (C::SLOTS - 1)) * C::PLANE; };

        const float2 c0v = make_float2(c0, c0), c1v = make_float2(c1, c1);
        Plane A, B;
        load(zlo - 1, A);
        load(zlo, B);
        put(A, slot(zlo - 1), false);  // lower neighbours of the first plane: own sites only
        put(B, slot(zlo), true);
        load(zlo + 1, A);

        // plane z: abv holds plane z+1 (stored now when another plane follows), pre takes z+2
        auto step = [&](int z, const Plane& abv, Plane& pre) -> bool {
            const bool more = z + 1 < zhi;
            if (more) {
                put(abv, slot(z + 1), true);
                load(z + 2, pre);
            }
            __syncthreads();
            const float* cur = slot(z) + own0;
            const float* prv = slot(z - 1) + own0;
            T* opl = o + int64_t(z) * P;
            T* wq = opl + base0;  // FULL: the warp's row r, column lane
            const float* bq = SRC ? b + int64_t(z) * P + base0 : nullptr;
            float2 ym = make_float2(cur[-SX], cur[32 - SX]);  // row y-1 of the warp's first row
            float2 ctr = make_float2(cur[0], cur[32]);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float* row = cur + r * SX;
                const float2 yp = make_float2(row[SX], row[32 + SX]);
                const float2 xm = make_float2(row[-1], row[31]);
                const float2 xp = make_float2(row[1], row[33]);
                const float2 zm = make_float2(prv[r * SX], prv[r * SX + 32]);
                float2 v = upd3_x2(c0v, c1v, ctr, xm, xp, ym, yp, zm, abv.v[r]);
                if constexpr (FULL) {
                    if constexpr (SRC) {
                        v = add2(v, make_float2(__ldg(bq), __ldg(bq + 32)));
                        bq += nx;
                    }
                    if constexpr (!PER) {
                        if (fixm != 0) {
                            if ((fixm >> (2 * r)) & 1u) v.x = ctr.x;
                            if ((fixm >> (2 * r + 1)) & 1u) v.y = ctr.y;
                        }
                    }
                    wq[0] = from_f<T>(v.x);
                    wq[32] = from_f<T>(v.y);
                    wq += nx;
                } else {
                    if constexpr (SRC) {
                        const float* bp = b + int64_t(z) * P + roff[r];
                        v = add2(v, make_float2(__ldg(bp + cx[0]), __ldg(bp + cx[1])));
                    }
                    if ((store >> (2 * r)) & 1u) opl[roff[r] + cx[0]] = from_f<T>(v.x);
                    if ((store >> (2 * r + 1)) & 1u) opl[roff[r] + cx[1]] = from_f<T>(v.y);
                }
                ym = ctr;
                ctr = yp;
            }
            return more;
        };
        for (int z = zlo;;) {
            if (!step(z++, A, B)) break;
            if (!step(z++, B, A)) break;
        }
    };
    if (full) run(BoolTag<true>{});
    else run(BoolTag<false>{});
}

}  // namespace ph3
