// Device function of the 2D temporal-blocking wavefront (one warp per strip and row chunk),
// shared by the standalone kernel (ph3_tb2d.cu) and the persistent batch kernel (ph3_batch.cu).
//
// Functional spec: pyheat3d src/pyheat3d/backends/stencil.cu:289-385 (tb2d) — k updates per
// DRAM pass over overlapped column strips; intermediate levels stay in fp32 and are rounded to
// the storage type once per pass (src/pyheat3d/validation.py:168-183). The design is described
// at the top of ph3_tb2d.cu.
#pragma once

#include "ph3_common.cuh"

namespace ph3 {

constexpr unsigned kT2Lanes = 0xffffffffu;

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
    const float left = __shfl_up_sync(kT2Lanes, r[NP - 1].y, 1);
    const float right = __shfl_down_sync(kT2Lanes, r[0].x, 1);
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

// One warp: strip `strip` (extended columns strip * OX - KX ..) of rows y0 .. y1-1, k = K fused
// updates from u into o. BULK: level 0 through the warp's shared-memory ring `ring` with
// mbarriers `bar` (STAGES of them; 16-byte rows and buffers); otherwise element loads, through L2
// only when CG (buffers other blocks of the same launch write).
template <typename T, bool PER, bool SRC, bool BULK, int K, int V, int STAGES, bool CG = false>
__device__ __forceinline__ void tb2d_pair_item(const T* __restrict__ u, T* __restrict__ o,
                                               const float* __restrict__ b, int ny, int nx,
                                               int strip, int y0, int y1, float c0, float c1,
                                               int* err, T* ring, uint64_t* bar) {
    using C = T2Cfg<T, K, V, STAGES>;
    constexpr int NP = C::NP, EX = C::EX, KX = C::KX, OX = C::OX;
    const int lane = threadIdx.x & 31;
    struct { int ny, nx; } g{ny, nx};
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
            for (int j = 0; j < V; ++j) pre[i][j] = ldx1<CG>(row + col[j]);
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

}  // namespace ph3
