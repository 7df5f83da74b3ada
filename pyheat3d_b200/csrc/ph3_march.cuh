// Tile functions of the single-step register marches (2D y-march, 3D z-march), shared by the
// standalone kernels (ph3_stencil.cu) and the persistent batch kernel (ph3_batch.cu).
//
// Functional spec: pyheat3d src/pyheat3d/backends/stencil.cu:101-161 (zmarch3d) and
// :289-385 (tb2d with K = 1, the y-march). Loads go through the read-only path (CG = false) or
// through L2 only (CG = true, for buffers other blocks of the same launch write).
#pragma once

#include "ph3_common.cuh"

namespace ph3 {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------------------------------
// small helpers
// ------------------------------------------------------------------------------------------

// V fp32 source values starting at p (p aligned to V*4 bytes when vec).
template <int V>
__device__ __forceinline__ void ld_src(const float* __restrict__ p, bool vec, float (&v)[V]) {
    // the source is read-only for every launch, so the read-only path is always safe
    if (vec) {
        if constexpr (V % 4 == 0) {
#pragma unroll
            for (int q = 0; q < V / 4; ++q) {
                const float4 t = __ldg(reinterpret_cast<const float4*>(p) + q);
                v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
            }
        } else if constexpr (V == 2) {
            const float2 t = __ldg(reinterpret_cast<const float2*>(p));
            v[0] = t.x; v[1] = t.y;
        } else {
            v[0] = __ldg(p);
        }
    } else {
#pragma unroll
        for (int j = 0; j < V; ++j) v[j] = __ldg(p + j);
    }
}

template <bool PER>
__device__ __forceinline__ int fix_idx(int i, int n) {
    if constexpr (PER) return wrap_idx(i, n);
    else return clamp_idx(i, 0, n - 1);
}
template <bool PER>
__device__ __forceinline__ int fix_near(int i, int n) {  // fix_idx through wrap_near
    if constexpr (PER) return wrap_near(i, n);
    else return clamp_idx(i, 0, n - 1);
}

// Column addressing of one thread's V consecutive x-values starting at gx.
// vec: the V values are one aligned vector (nx % V == 0 and gx % V == 0), addressed by `base`.
// scalar: each value has its own wrapped / clamped column in cx[].
template <bool PER, int V, bool CG = false>
struct Cols {
    int base;
    int cx[V];
    __device__ __forceinline__ void init(int gx, int nx, bool vec) {
        if (vec) {
            base = PER ? wrap_idx(gx, nx) : clamp_idx(gx, 0, nx - V);
#pragma unroll
            for (int j = 0; j < V; ++j) cx[j] = base + j;
        } else {
            base = 0;
#pragma unroll
            for (int j = 0; j < V; ++j) cx[j] = fix_idx<PER>(gx + j, nx);
        }
    }
    template <typename T>
    __device__ __forceinline__ void load(const T* __restrict__ row, bool vec, float (&v)[V]) const {
        if (vec) {
            ld_vec<T, V, CG>(row + base, v);
        } else {
#pragma unroll
            for (int j = 0; j < V; ++j) v[j] = ldx1<CG>(row + cx[j]);
        }
    }
    __device__ __forceinline__ void load_src(const float* __restrict__ row, bool vec,
                                             float (&v)[V]) const {
        if (vec) {
            ld_src<V>(row + base, true, v);
        } else {
#pragma unroll
            for (int j = 0; j < V; ++j) v[j] = __ldg(row + cx[j]);
        }
    }
};

// Store V values at columns gx..gx+V-1 of `row` (unwrapped; only in-domain columns written).
// `skip` has bit j set for columns that must not be written (Dirichlet boundary).
template <typename T, int V>
__device__ __forceinline__ void store_cols(T* __restrict__ row, int gx, int nx, bool vec,
                                           uint32_t skip, const float (&v)[V]) {
    if (vec && skip == 0 && gx + V <= nx) {
        st_vec<T, V>(row + gx, v);
        return;
    }
#pragma unroll
    for (int j = 0; j < V; ++j)
        if (gx + j < nx && !((skip >> j) & 1u)) row[gx + j] = from_f<T>(v[j]);
}

// ------------------------------------------------------------------------------------------
// 2D single step, y-march: warp w of the block owns a strip of 32*V columns (lane l holds
// columns x0 + l*V .. +V-1 as one vector) and walks a chunk of rows, RB rows per iteration, with
// the next RB rows already in flight. x-neighbours come from warp shuffles (lanes 0 and 31 load
// the strip's halo columns), y-neighbours from the row window in registers. No shared memory.
// ------------------------------------------------------------------------------------------
template <typename T, bool PER, int V, int W, int RB, bool CG>
__device__ __forceinline__ void march2d_item(const T* __restrict__ u, T* __restrict__ o,
                                             const float* __restrict__ b, int ny, int nx,
                                             float c0, float c1, int strip0, int cy, int ych,
                                             bool vec) {
    constexpr int EX = 32 * V;
    const int lane = threadIdx.x & 31;
    const int strip = strip0 + (threadIdx.x >> 5);
    const int x0 = strip * EX;
    if (x0 >= nx) return;  // whole warp leaves together; no block-wide sync in this function
    const int gx = x0 + lane * V;
    int ylo = cy * ych, yhi = min(ylo + ych, ny);
    if constexpr (!PER) { ylo = max(ylo, 1); yhi = min(yhi, ny - 1); }
    if (ylo >= yhi) return;

    Cols<PER, V, CG> cols;
    cols.init(gx, nx, vec);
    const int xl = fix_idx<PER>(x0 - 1, nx);
    const int xr = fix_idx<PER>(x0 + EX, nx);
    uint32_t skip = 0;  // Dirichlet boundary / outside columns are never written
    if constexpr (!PER) {
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gx + j <= 0 || gx + j >= nx - 1) skip |= 1u << j;
    }

    // window rows ylo-1 .. ylo+RB (RB + 2 rows), halos per row, prefetch RB rows
    float win[RB + 2][V], hl[RB + 2], hr[RB + 2];
    float pre[RB][V], pl[RB], pr[RB];
    auto load_row = [&](int y, float (&v)[V], float& l, float& r) {
        const T* row = u + int64_t(fix_idx<PER>(y, ny)) * nx;
        cols.load(row, vec, v);
        l = lane == 0 ? ldx1<CG>(row + xl) : 0.f;
        r = lane == 31 ? ldx1<CG>(row + xr) : 0.f;
    };
#pragma unroll
    for (int q = 0; q < RB + 2; ++q) load_row(ylo - 1 + q, win[q], hl[q], hr[q]);

    for (int y = ylo; y < yhi; y += RB) {
        const bool more = y + RB < yhi;
        if (more) {
#pragma unroll
            for (int q = 0; q < RB; ++q) load_row(y + RB + 1 + q, pre[q], pl[q], pr[q]);
        }
#pragma unroll
        for (int q = 0; q < RB; ++q) {
            const int yy = y + q;
            if (yy >= yhi) break;
            float out[V];
            const float left = __shfl_up_sync(kFull, win[q + 1][V - 1], 1);
            const float right = __shfl_down_sync(kFull, win[q + 1][0], 1);
            float bv[V];
            if (b != nullptr) cols.load_src(b + int64_t(yy) * nx, vec, bv);
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const float xm = j > 0 ? win[q + 1][j - 1] : (lane == 0 ? hl[q + 1] : left);
                const float xp = j < V - 1 ? win[q + 1][j + 1] : (lane == 31 ? hr[q + 1] : right);
                float v = upd2(c0, c1, win[q + 1][j], xm, xp, win[q][j], win[q + 2][j]);
                if (b != nullptr) v = __fadd_rn(v, bv[j]);
                out[j] = v;
            }
            store_cols<T, V>(o + int64_t(yy) * nx, gx, nx, vec, skip, out);
        }
        if (more) {
#pragma unroll
            for (int j = 0; j < V; ++j) {
                win[0][j] = win[RB][j];
                win[1][j] = win[RB + 1][j];
            }
            hl[0] = hl[RB]; hl[1] = hl[RB + 1]; hr[0] = hr[RB]; hr[1] = hr[RB + 1];
#pragma unroll
            for (int q = 0; q < RB; ++q) {
#pragma unroll
                for (int j = 0; j < V; ++j) win[q + 2][j] = pre[q][j];
                hl[q + 2] = pl[q];
                hr[q + 2] = pr[q];
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// 2D single step, y-march with raw rows: the same walk as march2d_item, but each row of the
// window and every prefetched row stays one 16-byte storage vector per lane (V = 16 / sizeof(T)
// values) and is widened to fp32 only where it is used. A 16-bit row then costs 4 registers
// instead of 8, so the same register budget keeps twice the rows (bytes) in flight. Requires
// whole 16-byte row vectors (nx % V == 0, 16-byte aligned buffers).
// ------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void widen16(const uint4& w, float (&v)[16 / sizeof(T)]) {
    union { uint4 w; T e[16 / sizeof(T)]; } un;
    un.w = w;
#pragma unroll
    for (int j = 0; j < int(16 / sizeof(T)); ++j) v[j] = to_f(un.e[j]);
}
template <bool CG>
__device__ __forceinline__ uint4 ld16(const void* p) {
    if constexpr (CG) return __ldcg(reinterpret_cast<const uint4*>(p));
    else return __ldg(reinterpret_cast<const uint4*>(p));
}

template <typename T, bool PER, int RB, bool CG>
__device__ __forceinline__ void march2d_raw_item(const T* __restrict__ u, T* __restrict__ o,
                                                 const float* __restrict__ b, int ny, int nx,
                                                 float c0, float c1, int strip, int cy, int ych) {
    constexpr int V = 16 / int(sizeof(T));
    constexpr int EX = 32 * V;
    const int lane = threadIdx.x & 31;
    const int x0 = strip * EX;
    if (x0 >= nx) return;  // whole warp leaves together; no block-wide sync in this function
    const int gx = x0 + lane * V;
    int ylo = cy * ych, yhi = min(ylo + ych, ny);
    if constexpr (!PER) { ylo = max(ylo, 1); yhi = min(yhi, ny - 1); }
    if (ylo >= yhi) return;

    // lanes past the last column read a wrapped (periodic) or clamped vector and store nothing;
    // with periodic wrap the lane after column nx-1 then holds column 0, the right neighbour
    const int base = PER ? wrap_idx(gx, nx) : clamp_idx(gx, 0, nx - V);
    // the strip's halo columns: lane 0 keeps the left one, lane 31 the right one (one register
    // per row serves both, since no lane needs both)
    const T* hcol = lane == 0 ? u + fix_idx<PER>(x0 - 1, nx)
                              : u + fix_idx<PER>(lane == 31 ? x0 + EX : x0, nx);
    const bool edge = lane == 0 || lane == 31;
    const bool writer = gx < nx;
    uint32_t skip = 0;  // Dirichlet boundary columns are never written
    if constexpr (!PER) {
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gx + j <= 0 || gx + j >= nx - 1) skip |= 1u << j;
    }
    auto load_row = [&](int y, uint4& v, float& h) {
        const int64_t off = int64_t(fix_idx<PER>(y, ny)) * nx;
        v = ld16<CG>(u + off + base);
        h = edge ? ldx1<CG>(hcol + off) : 0.f;
    };

    // Two row windows used in turn: a step computes RB rows from window W (rows y-1 .. y+RB)
    // while the next RB rows load straight into window N; only the two overlap rows, already
    // in registers, are copied. Prefetched rows are never moved, so a step never waits for
    // the loads it issued.
    uint4 P[RB + 2], Q[RB + 2];
    float Ph[RB + 2], Qh[RB + 2];
#pragma unroll
    for (int q = 0; q < RB + 2; ++q) load_row(ylo - 1 + q, P[q], Ph[q]);

    auto step = [&](int y, uint4 (&W)[RB + 2], float (&Wh)[RB + 2], uint4 (&N)[RB + 2],
                    float (&Nh)[RB + 2]) -> bool {
        const bool more = y + RB < yhi;
        if (more) {
#pragma unroll
            for (int q = 0; q < RB; ++q) load_row(y + RB + 1 + q, N[q + 2], Nh[q + 2]);
        }
#pragma unroll
        for (int q = 0; q < RB; ++q) {
            const int yy = y + q;
            if (yy >= yhi) break;
            float c[V], m[V], p[V];
            widen16<T>(W[q + 1], c);
            widen16<T>(W[q], m);
            widen16<T>(W[q + 2], p);
            const float left = __shfl_up_sync(kFull, c[V - 1], 1);
            const float right = __shfl_down_sync(kFull, c[0], 1);
            float bv[V];
            if (b != nullptr) ld_src<V>(b + int64_t(yy) * nx + base, true, bv);
            float out[V];
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const float xm = j > 0 ? c[j - 1] : (lane == 0 ? Wh[q + 1] : left);
                const float xp = j < V - 1 ? c[j + 1] : (lane == 31 ? Wh[q + 1] : right);
                float v = upd2(c0, c1, c[j], xm, xp, m[j], p[j]);
                if (b != nullptr) v = __fadd_rn(v, bv[j]);
                out[j] = v;
            }
            if (writer) {
                T* dst = o + int64_t(yy) * nx + gx;
                if (skip == 0) {
                    st_vec<T, V>(dst, out);
                } else {
#pragma unroll
                    for (int j = 0; j < V; ++j)
                        if (!((skip >> j) & 1u)) dst[j] = from_f<T>(out[j]);
                }
            }
        }
        if (more) {
            N[0] = W[RB];
            N[1] = W[RB + 1];
            Nh[0] = Wh[RB];
            Nh[1] = Wh[RB + 1];
        }
        return more;
    };
    for (int y = ylo;;) {
        if (!step(y, P, Ph, Q, Qh)) break;
        y += RB;
        if (!step(y, Q, Qh, P, Ph)) break;
        y += RB;
    }
}

// ------------------------------------------------------------------------------------------
// 3D single step, z-march with plain loads (any shape): the block owns an xy tile of 32*V x
// W*R sites; warp w holds R rows, lane l holds V columns per row as one vector. The z-neighbours
// form a register queue (below / centre / above) and the plane after `above` is in flight while
// a plane is computed. x-neighbours: shuffles (+ halo columns loaded by lanes 0 and 31);
// y-neighbours: own registers, the first/last rows of the neighbouring warps through shared
// memory, and the tile's halo rows loaded by the first and last warp.
// ------------------------------------------------------------------------------------------
template <typename T, bool PER, int V, int R, int W, bool CG>
__device__ __forceinline__ void march3d_item(const T* __restrict__ u, T* __restrict__ o,
                                             const float* __restrict__ b, int nz, int ny, int nx,
                                             float c0, float c1, int bx, int by, int bz, int zch,
                                             bool vec, float* edge_smem) {
    constexpr int EX = 32 * V, EY = W * R;
    float (*edge)[W][EX] = reinterpret_cast<float (*)[W][EX]>(edge_smem);  // [2][W][EX]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x0 = bx * EX, y0 = by * EY;
    const int gx = x0 + lane * V, gy0 = y0 + w * R;
    int zlo = bz * zch, zhi = min(zlo + zch, nz);
    if constexpr (!PER) { zlo = max(zlo, 1); zhi = min(zhi, nz - 1); }
    if (zlo >= zhi) return;  // uniform over the block

    const int64_t P = int64_t(nx) * ny;
    Cols<PER, V, CG> cols;
    cols.init(gx, nx, vec);
    int64_t roff[R];
#pragma unroll
    for (int r = 0; r < R; ++r) roff[r] = int64_t(fix_idx<PER>(gy0 + r, ny)) * nx;
    const int64_t rtop = int64_t(fix_idx<PER>(y0 - 1, ny)) * nx;
    const int64_t rbot = int64_t(fix_idx<PER>(y0 + EY, ny)) * nx;
    const int xl = fix_idx<PER>(x0 - 1, nx), xr = fix_idx<PER>(x0 + EX, nx);
    uint32_t skipx = 0, skipy = 0;
    if constexpr (!PER) {
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gx + j <= 0 || gx + j >= nx - 1) skipx |= 1u << j;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (gy0 + r <= 0 || gy0 + r >= ny - 1) skipy |= 1u << r;
    }

    struct Plane {
        float v[R][V];
        float l[R], r[R];    // halo columns (lanes 0 / 31)
        float t[V], bt[V];   // halo rows (warp 0 / warp W-1)
    };
    auto load_plane = [&](int z, Plane& p) {
        const T* pl = u + int64_t(fix_idx<PER>(z, nz)) * P;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            cols.load(pl + roff[r], vec, p.v[r]);
            p.l[r] = lane == 0 ? ldx1<CG>(pl + roff[r] + xl) : 0.f;
            p.r[r] = lane == 31 ? ldx1<CG>(pl + roff[r] + xr) : 0.f;
        }
        if (w == 0) cols.load(pl + rtop, vec, p.t);
        if (w == W - 1) cols.load(pl + rbot, vec, p.bt);
    };

    float bel[R][V];
    Plane ctr, abv, pre;
    {
        const T* pl = u + int64_t(fix_idx<PER>(zlo - 1, nz)) * P;
#pragma unroll
        for (int r = 0; r < R; ++r) cols.load(pl + roff[r], vec, bel[r]);
    }
    load_plane(zlo, ctr);
    load_plane(zlo + 1, abv);

    for (int z = zlo; z < zhi; ++z) {
        const bool more = z + 1 < zhi;
        if (more) load_plane(z + 2, pre);
        // y-neighbours across warps
        float up[V], dn[V];
        if constexpr (W > 1) {
            __syncthreads();  // previous iteration's reads of edge[] are done
#pragma unroll
            for (int j = 0; j < V; ++j) {
                edge[0][w][lane * V + j] = ctr.v[0][j];
                edge[1][w][lane * V + j] = ctr.v[R - 1][j];
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < V; ++j) {
                up[j] = w > 0 ? edge[1][w - 1][lane * V + j] : ctr.t[j];
                dn[j] = w < W - 1 ? edge[0][w + 1][lane * V + j] : ctr.bt[j];
            }
        } else {
#pragma unroll
            for (int j = 0; j < V; ++j) { up[j] = ctr.t[j]; dn[j] = ctr.bt[j]; }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float left = __shfl_up_sync(kFull, ctr.v[r][V - 1], 1);
            const float right = __shfl_down_sync(kFull, ctr.v[r][0], 1);
            float bv[V];
            if (b != nullptr) cols.load_src(b + int64_t(z) * P + roff[r], vec, bv);
            float out[V];
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const float xm = j > 0 ? ctr.v[r][j - 1] : (lane == 0 ? ctr.l[r] : left);
                const float xp = j < V - 1 ? ctr.v[r][j + 1] : (lane == 31 ? ctr.r[r] : right);
                const float ym = r > 0 ? ctr.v[r - 1][j] : up[j];
                const float yp = r < R - 1 ? ctr.v[r + 1][j] : dn[j];
                float v = upd3(c0, c1, ctr.v[r][j], xm, xp, ym, yp, bel[r][j], abv.v[r][j]);
                if (b != nullptr) v = __fadd_rn(v, bv[j]);
                out[j] = v;
            }
            const int gy = gy0 + r;
            if (gy < ny && !((skipy >> r) & 1u))
                store_cols<T, V>(o + int64_t(z) * P + int64_t(gy) * nx, gx, nx, vec, skipx, out);
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int j = 0; j < V; ++j) bel[r][j] = ctr.v[r][j];
        ctr = abv;
        if (more) abv = pre;
    }
}

// ------------------------------------------------------------------------------------------
// Lean marches for any row alignment: one column per lane, so every row access of a warp is one
// coalesced 128-byte scalar load or store whatever nx is. Warps are fully independent (no shared
// memory, no block barrier): a warp owns R rows of a 32-column strip, keeps the z-queue (3D) or
// a row window (2D) in registers with the next plane / rows already in flight, takes
// x-neighbours by shuffles (lane 0 / 31 hold the strip's halo column in one register per row)
// and, in 3D, loads the rows just above and below its own rows directly.
// ------------------------------------------------------------------------------------------
template <typename T, bool PER, int R, bool CG, bool SRC = true>
__device__ __forceinline__ void lite3d_item(const T* __restrict__ u, T* __restrict__ o,
                                            const float* __restrict__ b, int nz, int ny, int nx,
                                            float c0, float c1, int strip, int row0, int zlo,
                                            int zhi) {
    const int lane = threadIdx.x & 31;
    const int x0 = strip * 32, x = x0 + lane;
    if (x0 >= nx || row0 >= ny) return;  // warp-uniform
    if constexpr (!PER) { zlo = max(zlo, 1); zhi = min(zhi, nz - 1); }
    if (zlo >= zhi) return;
    const int64_t P = int64_t(nx) * ny;
    const int cx = fix_idx<PER>(x, nx);
    const int hcol = lane == 0 ? fix_idx<PER>(x0 - 1, nx) : fix_idx<PER>(x0 + 32, nx);
    const bool hl = lane == 0 || lane == 31;
    int roff[R];
#pragma unroll
    for (int r = 0; r < R; ++r) roff[r] = fix_idx<PER>(row0 + r, ny) * nx;
    const int uoff = fix_idx<PER>(row0 - 1, ny) * nx, doff = fix_idx<PER>(row0 + R, ny) * nx;
    bool xskip = x >= nx;
    uint32_t yskip = 0;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (row0 + r >= ny || (!PER && (row0 + r == 0 || row0 + r == ny - 1))) yskip |= 1u << r;
    if constexpr (!PER) xskip = xskip || x == 0 || x == nx - 1;

    struct Plane {
        float v[R], h[R];  // own rows; halo column (lanes 0 / 31)
        float up, dn;      // rows above / below the warp's rows
        float s[R];        // Jacobi source of the own rows (0 without a source)
    };
    auto load = [&](int z, Plane& p) {
        const int64_t zo = int64_t(fix_near<PER>(z, nz)) * P;
        const T* pl = u + zo;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            p.v[r] = ldx1<CG>(pl + roff[r] + cx);
            p.h[r] = hl ? ldx1<CG>(pl + roff[r] + hcol) : 0.f;
            p.s[r] = (SRC && b != nullptr) ? __ldg(b + zo + roff[r] + cx) : 0.f;
        }
        p.up = ldx1<CG>(pl + uoff + cx);
        p.dn = ldx1<CG>(pl + doff + cx);
    };
    float bel[R];
    {
        const T* pl = u + int64_t(fix_near<PER>(zlo - 1, nz)) * P;
#pragma unroll
        for (int r = 0; r < R; ++r) bel[r] = ldx1<CG>(pl + roff[r] + cx);
    }
    // Three planes in turn (centre, above, in flight): the loop runs three planes per pass
    // and the roles rotate by name, so a loaded plane is never copied and a plane step never
    // waits for the load it issued.
    Plane A, B, C;
    load(zlo, A);
    load(zlo + 1, B);
    auto step = [&](int z, const Plane& ctr, const Plane& abv, Plane& pre) -> bool {
        const bool more = z + 1 < zhi;
        if (more) load(z + 2, pre);
        T* opl = o + int64_t(z) * P;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float c = ctr.v[r];
            float xm = __shfl_up_sync(kFull, c, 1);
            float xp = __shfl_down_sync(kFull, c, 1);
            if (lane == 0) xm = ctr.h[r];
            if (lane == 31) xp = ctr.h[r];
            const float ym = r > 0 ? ctr.v[r - 1] : ctr.up;
            const float yp = r < R - 1 ? ctr.v[r + 1] : ctr.dn;
            float v = upd3(c0, c1, c, xm, xp, ym, yp, bel[r], abv.v[r]);
            if ((SRC && b != nullptr)) v = __fadd_rn(v, ctr.s[r]);
            if (!xskip && !((yskip >> r) & 1u)) opl[roff[r] + x] = from_f<T>(v);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) bel[r] = ctr.v[r];
        return more;
    };
    for (int z = zlo;;) {
        if (!step(z++, A, B, C)) break;
        if (!step(z++, B, C, A)) break;
        if (!step(z++, C, A, B)) break;
    }
}

// ------------------------------------------------------------------------------------------
// 3D single step for any row alignment with four columns per lane. A lane owns the columns
// gx .. gx+3 (gx = x0 + 4 lane), a warp R rows of a 128-column strip. Every row access moves
// the lane's four elements with the widest accesses the row's alignment allows: the element
// index of gx from the array base modulo 4 is the same for every lane of a row, so one warp-
// uniform branch picks one 4-element vector (residue 0), two pairs (2) or four scalars (odd).
// Requires array bases aligned to 4 elements (16 bytes fp32, 8 bytes 16-bit). The last strip
// of a row, when partial, reads per-element columns wrapped (periodic) or clamped (Dirichlet),
// so lanes past the row end hold the neighbours the shuffles need; only in-row columns are
// written. Planes rotate through three register sets by name, one plane in flight.
// ------------------------------------------------------------------------------------------
template <typename T, bool CG>
__device__ __forceinline__ void ld4a(const T* __restrict__ p, int a, float (&v)[4]) {
    if (a == 0) {
        ld_vec<T, 4, CG>(p, v);
    } else if (a == 2) {
        float t[2], w[2];
        ld_vec<T, 2, CG>(p, t);
        ld_vec<T, 2, CG>(p + 2, w);
        v[0] = t[0]; v[1] = t[1]; v[2] = w[0]; v[3] = w[1];
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = ldx1<CG>(p + j);
    }
}

template <typename T>
__device__ __forceinline__ void st4a(T* __restrict__ p, int a, const float (&v)[4]) {
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

template <typename T, bool PER, int R, bool CG>
__device__ __forceinline__ void avec3d_item(const T* __restrict__ u, T* __restrict__ o,
                                            const float* __restrict__ b, int nz, int ny, int nx,
                                            float c0, float c1, int strip, int row0, int zlo,
                                            int zhi) {
    constexpr int V = 4, EX = 32 * V;
    const int lane = threadIdx.x & 31;
    const int x0 = strip * EX, gx = x0 + lane * V;
    if (x0 >= nx || row0 >= ny) return;  // warp-uniform
    if constexpr (!PER) { zlo = max(zlo, 1); zhi = min(zhi, nz - 1); }
    if (zlo >= zhi) return;
    const int64_t P = int64_t(nx) * ny;
    const bool full = x0 + EX <= nx;  // warp-uniform: all 128 columns inside the row
    int cx[V];                        // per-element columns of a partial strip
#pragma unroll
    for (int j = 0; j < V; ++j) cx[j] = fix_idx<PER>(gx + j, nx);
    const int hcol = lane == 0 ? fix_idx<PER>(x0 - 1, nx) : fix_idx<PER>(x0 + EX, nx);
    const bool hl = lane == 0 || lane == 31;
    int roff[R];
#pragma unroll
    for (int r = 0; r < R; ++r) roff[r] = fix_idx<PER>(row0 + r, ny) * nx;
    const int uoff = fix_idx<PER>(row0 - 1, ny) * nx, doff = fix_idx<PER>(row0 + R, ny) * nx;
    uint32_t skipx = 0, yskip = 0;  // columns / rows this lane must not write
#pragma unroll
    for (int j = 0; j < V; ++j)
        if (gx + j >= nx || (!PER && (gx + j == 0 || gx + j == nx - 1))) skipx |= 1u << j;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (row0 + r >= ny || (!PER && (row0 + r == 0 || row0 + r == ny - 1))) yskip |= 1u << r;
    // residue modulo 4 of an element index (the array bases are 4-element aligned)
    const int P4 = int(P & 3), x4 = x0 & 3;
    auto res = [&](int z, int off) { return (z * P4 + off + x4) & 3; };
    auto row4 = [&](const T* rp, int a, float (&v)[V]) {
        if (full) {
            ld4a<T, CG>(rp + gx, a, v);
        } else {
#pragma unroll
            for (int j = 0; j < V; ++j) v[j] = ldx1<CG>(rp + cx[j]);
        }
    };

    struct Plane {
        float v[R][V], h[R];  // own rows; halo column (lanes 0 / 31)
        float up[V], dn[V];   // rows above / below the warp's rows
    };
    auto load = [&](int z, Plane& p) {
        const int zz = fix_near<PER>(z, nz);
        const T* pl = u + int64_t(zz) * P;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            row4(pl + roff[r], res(zz, roff[r]), p.v[r]);
            p.h[r] = hl ? ldx1<CG>(pl + roff[r] + hcol) : 0.f;
        }
        row4(pl + uoff, res(zz, uoff), p.up);
        row4(pl + doff, res(zz, doff), p.dn);
    };
    float bel[R][V];
    {
        const int zz = fix_near<PER>(zlo - 1, nz);
        const T* pl = u + int64_t(zz) * P;
#pragma unroll
        for (int r = 0; r < R; ++r) row4(pl + roff[r], res(zz, roff[r]), bel[r]);
    }
    Plane A, B, C;
    load(zlo, A);
    load(zlo + 1, B);
    auto step = [&](int z, const Plane& ctr, const Plane& abv, Plane& pre) -> bool {
        const bool more = z + 1 < zhi;
        if (more) load(z + 2, pre);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float left = __shfl_up_sync(kFull, ctr.v[r][V - 1], 1);
            const float right = __shfl_down_sync(kFull, ctr.v[r][0], 1);
            const int gy = row0 + r;
            // residue of this row's elements (roff[r] == gy * nx for every written row; the
            // source is read at the same, possibly wrapped, row)
            const int a = res(z, roff[r]);
            float bv[V];
            if (b != nullptr) {
                const float* bp = b + int64_t(z) * P + int64_t(roff[r]);
                if (full) {
                    ld4a<float, false>(bp + gx, a, bv);
                } else {
#pragma unroll
                    for (int j = 0; j < V; ++j) bv[j] = __ldg(bp + cx[j]);
                }
            }
            float out[V];
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const float xm = j > 0 ? ctr.v[r][j - 1] : (lane == 0 ? ctr.h[r] : left);
                const float xp = j < V - 1 ? ctr.v[r][j + 1] : (lane == 31 ? ctr.h[r] : right);
                const float ym = r > 0 ? ctr.v[r - 1][j] : ctr.up[j];
                const float yp = r < R - 1 ? ctr.v[r + 1][j] : ctr.dn[j];
                float v = upd3(c0, c1, ctr.v[r][j], xm, xp, ym, yp, bel[r][j], abv.v[r][j]);
                if (b != nullptr) v = __fadd_rn(v, bv[j]);
                out[j] = v;
            }
            if (!((yskip >> r) & 1u)) {
                T* dst = o + int64_t(z) * P + int64_t(gy) * nx + gx;
                if (skipx == 0) {
                    st4a<T>(dst, a, out);
                } else {
#pragma unroll
                    for (int j = 0; j < V; ++j)
                        if (!((skipx >> j) & 1u)) dst[j] = from_f<T>(out[j]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int j = 0; j < V; ++j) bel[r][j] = ctr.v[r][j];
        return more;
    };
    for (int z = zlo;;) {
        if (!step(z++, A, B, C)) break;
        if (!step(z++, B, C, A)) break;
        if (!step(z++, C, A, B)) break;
    }
}

template <typename T, bool PER, int RB, bool CG, bool SRC = true>
__device__ __forceinline__ void lite2d_item(const T* __restrict__ u, T* __restrict__ o,
                                            const float* __restrict__ b, int ny, int nx,
                                            float c0, float c1, int strip, int ylo, int yhi) {
    const int lane = threadIdx.x & 31;
    const int x0 = strip * 32, x = x0 + lane;
    if (x0 >= nx) return;  // warp-uniform
    if constexpr (!PER) { ylo = max(ylo, 1); yhi = min(yhi, ny - 1); }
    if (ylo >= yhi) return;
    const int cx = fix_idx<PER>(x, nx);
    const int hcol = lane == 0 ? fix_idx<PER>(x0 - 1, nx) : fix_idx<PER>(x0 + 32, nx);
    const bool hl = lane == 0 || lane == 31;
    bool xskip = x >= nx;
    if constexpr (!PER) xskip = xskip || x == 0 || x == nx - 1;
    // two row windows used in turn (rows y-1 .. y+RB and their halo values): the next RB rows
    // load straight into the other window, so only the two overlap rows are ever copied
    float P[RB + 2], Ph[RB + 2], Q[RB + 2], Qh[RB + 2];
    auto row = [&](int y) { return u + int64_t(fix_near<PER>(y, ny)) * nx; };
#pragma unroll
    for (int q = 0; q < RB + 2; ++q) {
        const T* rp = row(ylo - 1 + q);
        P[q] = ldx1<CG>(rp + cx);
        Ph[q] = hl ? ldx1<CG>(rp + hcol) : 0.f;
    }
    auto step = [&](int y, const float (&win)[RB + 2], const float (&wh)[RB + 2],
                    float (&N)[RB + 2], float (&Nh)[RB + 2]) -> bool {
        const bool more = y + RB < yhi;
        if (more) {
#pragma unroll
            for (int q = 0; q < RB; ++q) {
                const T* rp = row(y + RB + 1 + q);
                N[q + 2] = ldx1<CG>(rp + cx);
                Nh[q + 2] = hl ? ldx1<CG>(rp + hcol) : 0.f;
            }
        }
#pragma unroll
        for (int q = 0; q < RB; ++q) {
            const int yy = y + q;
            if (yy >= yhi) break;
            const float c = win[q + 1];
            float xm = __shfl_up_sync(kFull, c, 1);
            float xp = __shfl_down_sync(kFull, c, 1);
            if (lane == 0) xm = wh[q + 1];
            if (lane == 31) xp = wh[q + 1];
            float v = upd2(c0, c1, c, xm, xp, win[q], win[q + 2]);
            if ((SRC && b != nullptr)) v = __fadd_rn(v, __ldg(b + int64_t(yy) * nx + cx));
            if (!xskip) o[int64_t(yy) * nx + x] = from_f<T>(v);
        }
        if (more) {
            N[0] = win[RB]; Nh[0] = wh[RB];
            N[1] = win[RB + 1]; Nh[1] = wh[RB + 1];
        }
        return more;
    };
    for (int y = ylo;;) {
        if (!step(y, P, Ph, Q, Qh)) break;
        y += RB;
        if (!step(y, Q, Qh, P, Ph)) break;
        y += RB;
    }
}

}  // namespace ph3
