// Shared device helpers of the pyheat3d B200 stencil kernels (sm_100a).
//
// The update every kernel computes (pyheat3d src/pyheat3d/problem.py:3-10,
// src/pyheat3d/backends/numpy_ref.py:30-47):
//
//     u'[c] = c0*u[c] + c1*S[c]  (+ b[c], added last)
//     S     = ((u[x-1]+u[x+1]) + (u[y-1]+u[y+1])) + (u[z-1]+u[z+1])
//
// Arithmetic is fp32 for every storage type. Every add and multiply is an explicitly rounded
// __fadd_rn / __fmul_rn so nvcc cannot contract c0*u + c1*S into an FMA: the result is then
// bit-identical to NumPy, which rounds each ufunc separately.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ph3 {

// ------------------------------------------------------------------------------------------
// storage traits: load converts to fp32 exactly, store rounds to nearest even
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}

template <typename T> __device__ __forceinline__ float ldg1(const T* p) { return to_f(__ldg(p)); }

// Loads that bypass L1 (cache in L2 only): for buffers other blocks of the same launch write,
// where the read-only path could return stale lines.
__device__ __forceinline__ float ldcg1(const float* p) { return __ldcg(p); }
__device__ __forceinline__ float ldcg1(const __half* p) {
    const unsigned short b = __ldcg(reinterpret_cast<const unsigned short*>(p));
    return __half2float(__ushort_as_half(b));
}
__device__ __forceinline__ float ldcg1(const __nv_bfloat16* p) {
    const unsigned short b = __ldcg(reinterpret_cast<const unsigned short*>(p));
    return __uint_as_float(uint32_t(b) << 16);
}
// one element through the chosen path (CG: L2 only)
template <bool CG, typename T> __device__ __forceinline__ float ldx1(const T* p) {
    if constexpr (CG) return ldcg1(p);
    else return ldg1(p);
}

// Vector of V storage elements moved as one 4/8/16-byte access.
template <typename T, int V> struct VecBits;
template <typename T> struct VecBits<T, 1> { using type = T; };
template <int V> struct VecBytes;
template <> struct VecBytes<4> { using type = uint32_t; };
template <> struct VecBytes<8> { using type = uint2; };
template <> struct VecBytes<16> { using type = uint4; };

template <typename T, int V, bool CG = false>
__device__ __forceinline__ void ld_vec(const T* __restrict__ p, float (&v)[V]) {
    constexpr int B = int(sizeof(T)) * V;
    if constexpr (B == 2) {
        v[0] = ldx1<CG>(p);
    } else {
        using W = typename VecBytes<B>::type;
        union { W w; T e[V]; } u;
        if constexpr (CG) u.w = __ldcg(reinterpret_cast<const W*>(p));
        else u.w = __ldg(reinterpret_cast<const W*>(p));
#pragma unroll
        for (int j = 0; j < V; ++j) v[j] = to_f(u.e[j]);
    }
}

// V storage values from shared (or any generic) memory as one 4/8/16-byte access.
template <typename T, int V>
__device__ __forceinline__ void ld_vec_shared(const T* p, float (&v)[V]) {
    constexpr int B = int(sizeof(T)) * V;
    using W = typename VecBytes<B>::type;
    union { W w; T e[V]; } u;
    u.w = *reinterpret_cast<const W*>(p);
#pragma unroll
    for (int j = 0; j < V; ++j) v[j] = to_f(u.e[j]);
}

template <typename T, int V>
__device__ __forceinline__ void st_vec(T* __restrict__ p, const float (&v)[V]) {
    constexpr int B = int(sizeof(T)) * V;
    if constexpr (B == 2) {
        *p = from_f<T>(v[0]);
    } else {
        using W = typename VecBytes<B>::type;
        union { W w; T e[V]; } u;
#pragma unroll
        for (int j = 0; j < V; ++j) u.e[j] = from_f<T>(v[j]);
        *reinterpret_cast<W*>(p) = u.w;
    }
}

// 16 bytes of storage <-> float2 pairs (8 B: 2 fp32; 4 x 16-bit pairs), round to nearest even.
template <typename T> struct Pack16;
template <> struct Pack16<float> {
    static constexpr int NP = 2;
    __device__ __forceinline__ static void unpack(const uint4& w, float2 (&v)[NP]) {
        v[0] = make_float2(__uint_as_float(w.x), __uint_as_float(w.y));
        v[1] = make_float2(__uint_as_float(w.z), __uint_as_float(w.w));
    }
    __device__ __forceinline__ static uint4 pack(const float2 (&v)[NP]) {
        return make_uint4(__float_as_uint(v[0].x), __float_as_uint(v[0].y),
                          __float_as_uint(v[1].x), __float_as_uint(v[1].y));
    }
};
template <> struct Pack16<__nv_bfloat16> {
    static constexpr int NP = 4;
    __device__ __forceinline__ static float2 cvt(uint32_t w) {
        return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
    }
    __device__ __forceinline__ static uint32_t rnd(float2 v) {
        __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        return *reinterpret_cast<uint32_t*>(&h);
    }
    __device__ __forceinline__ static void unpack(const uint4& w, float2 (&v)[NP]) {
        v[0] = cvt(w.x); v[1] = cvt(w.y); v[2] = cvt(w.z); v[3] = cvt(w.w);
    }
    __device__ __forceinline__ static uint4 pack(const float2 (&v)[NP]) {
        return make_uint4(rnd(v[0]), rnd(v[1]), rnd(v[2]), rnd(v[3]));
    }
};
template <> struct Pack16<__half> {
    static constexpr int NP = 4;
    __device__ __forceinline__ static float2 cvt(uint32_t w) {
        return __half22float2(*reinterpret_cast<const __half2*>(&w));
    }
    __device__ __forceinline__ static uint32_t rnd(float2 v) {
        __half2 h = __floats2half2_rn(v.x, v.y);
        return *reinterpret_cast<uint32_t*>(&h);
    }
    __device__ __forceinline__ static void unpack(const uint4& w, float2 (&v)[NP]) {
        v[0] = cvt(w.x); v[1] = cvt(w.y); v[2] = cvt(w.z); v[3] = cvt(w.w);
    }
    __device__ __forceinline__ static uint4 pack(const float2 (&v)[NP]) {
        return make_uint4(rnd(v[0]), rnd(v[1]), rnd(v[2]), rnd(v[3]));
    }
};

// One lane's LB bytes of storage <-> float2 pairs: LB = 16 is Pack16; LB = 8 holds 2 fp32 or
// 4 16-bit values.
template <typename T, int LB> struct PackLane;
template <typename T> struct PackLane<T, 16> : Pack16<T> { using W = uint4; };
template <> struct PackLane<float, 8> {
    using W = uint2;
    static constexpr int NP = 1;
    __device__ __forceinline__ static void unpack(const uint2& w, float2 (&v)[NP]) {
        v[0] = make_float2(__uint_as_float(w.x), __uint_as_float(w.y));
    }
    __device__ __forceinline__ static uint2 pack(const float2 (&v)[NP]) {
        return make_uint2(__float_as_uint(v[0].x), __float_as_uint(v[0].y));
    }
};
template <typename T> struct PackLane16x4 {
    using W = uint2;
    static constexpr int NP = 2;
    __device__ __forceinline__ static void unpack(const uint2& w, float2 (&v)[NP]) {
        v[0] = Pack16<T>::cvt(w.x); v[1] = Pack16<T>::cvt(w.y);
    }
    __device__ __forceinline__ static uint2 pack(const float2 (&v)[NP]) {
        return make_uint2(Pack16<T>::rnd(v[0]), Pack16<T>::rnd(v[1]));
    }
};
template <> struct PackLane<__nv_bfloat16, 8> : PackLane16x4<__nv_bfloat16> {};
template <> struct PackLane<__half, 8> : PackLane16x4<__half> {};

// ------------------------------------------------------------------------------------------
// canonical-order stencil arithmetic
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float upd2(float c0, float c1, float ctr, float xm, float xp,
                                      float ym, float yp) {
    const float s = __fadd_rn(__fadd_rn(xm, xp), __fadd_rn(ym, yp));
    return __fadd_rn(__fmul_rn(c0, ctr), __fmul_rn(c1, s));
}

__device__ __forceinline__ float upd3(float c0, float c1, float ctr, float xm, float xp,
                                      float ym, float yp, float zm, float zp) {
    const float s = __fadd_rn(__fadd_rn(__fadd_rn(xm, xp), __fadd_rn(ym, yp)), __fadd_rn(zm, zp));
    return __fadd_rn(__fmul_rn(c0, ctr), __fmul_rn(c1, s));
}

// Packed fp32x2 add / multiply (sm_100a `add.rn.f32x2`, `mul.rn.f32x2`): each lane rounds
// like __fadd_rn / __fmul_rn. Only additions are chained in packed form: a packed product
// followed by a packed sum may be contracted into a fused multiply-add by the assembler, so the
// final c0*u + c1*S uses the scalar non-contracting intrinsics.
union F2 {
    float2 f;
    unsigned long long u;
};
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    F2 x, y, r;
    x.f = a; y.f = b;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.u) : "l"(x.u), "l"(y.u));
    return r.f;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    F2 x, y, r;
    x.f = a; y.f = b;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.u) : "l"(x.u), "l"(y.u));
    return r.f;
}

// c0*u + c1*S for a pair: packed products, scalar non-contracting sum (checked on the GPU to be
// bit-identical to the scalar chain; a packed sum of packed products is not).
__device__ __forceinline__ float2 lin2(float2 c0, float2 c1, float2 ctr, float2 s) {
    const float2 a = mul2(c0, ctr), b = mul2(c1, s);
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}

// Two neighbouring sites of one row: the same canonical-order update as upd3 / upd2, with the
// neighbour sums packed.
__device__ __forceinline__ float2 upd3_x2(float2 c0, float2 c1, float2 ctr, float2 xm, float2 xp,
                                          float2 ym, float2 yp, float2 zm, float2 zp) {
    const float2 s = add2(add2(add2(xm, xp), add2(ym, yp)), add2(zm, zp));
    return lin2(c0, c1, ctr, s);
}
// Same, with the x-neighbour sum (xm + xp) of both sites already formed.
__device__ __forceinline__ float2 upd3_sx2(float2 c0, float2 c1, float2 ctr, float2 sx, float2 ym,
                                           float2 yp, float2 zm, float2 zp) {
    const float2 s = add2(add2(sx, add2(ym, yp)), add2(zm, zp));
    return lin2(c0, c1, ctr, s);
}
__device__ __forceinline__ float2 upd2_x2(float2 c0, float2 c1, float2 ctr, float2 xm, float2 xp,
                                          float2 ym, float2 yp) {
    const float2 s = add2(add2(xm, xp), add2(ym, yp));
    return lin2(c0, c1, ctr, s);
}

// Periodic index in [0, n).
__device__ __forceinline__ int wrap_idx(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}
// The same result for every i, with compare-and-add paths for indices within one period of the
// domain (halos and tile overhangs) so only far indices pay for a division. Faster where an
// index is wrapped once per plane or row of the temporal-blocking kernels; the division-free
// branches are not used in the register marches, whose unrolled row loads they would separate
// (measured: the 2D raw-row march at half speed with them).
__device__ __forceinline__ int wrap_near(int i, int n) {
    if (i >= 0) {
        if (i < n) return i;
        if (i - n < n) return i - n;
    } else if (i >= -n) {
        return i + n;
    }
    i %= n;
    return i < 0 ? i + n : i;
}
__device__ __forceinline__ int clamp_idx(int i, int lo, int hi) {
    return i < lo ? lo : (i > hi ? hi : i);
}

// ------------------------------------------------------------------------------------------
// error word: kernels whose bounded waits expire record a code here and return early
// ------------------------------------------------------------------------------------------
enum DeviceError : int {
    kDevOk = 0,
    kDevMbarTimeout = 1,     // an mbarrier wait hit its iteration limit
    kDevDependTimeout = 2,   // a persistent work item waited too long for its predecessors
    kDevStopRequested = 3,   // a persistent kernel saw the host stop word
};
// `err` points at the per-device status word owned by the C-ABI layer (may be null).
__device__ __forceinline__ void record_error(int* err, int code) {
    if (err != nullptr) atomicCAS(err, 0, code);
}

// Iteration limit of every spin-wait (each iteration also backs off with __nanosleep), giving
// well over a second of waiting before a wait is declared stuck.
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait until *flag >= target (acquire ordering), backing off with __nanosleep. Gives up
// after `limit` polls, or as soon as *abort (if given) is nonzero; a wait that gives up records
// kDevDependTimeout in the status word and returns false.
__device__ __forceinline__ bool wait_flag_geq(const int* flag, int target, uint32_t limit,
                                              int* err, const int* abort) {
    uint32_t spins = 0;
    while (ld_acquire_gpu(flag) < target) {
        __nanosleep(spins < 64 ? 32 : 256);
        if (++spins > limit ||
            (abort != nullptr && *reinterpret_cast<const volatile int*>(abort) != 0)) {
            record_error(err, kDevDependTimeout);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ unsigned long long ld_acquire_gpu_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// wait_flag_geq for a 64-bit counter.
__device__ __forceinline__ bool wait_u64_geq(const unsigned long long* flag,
                                             unsigned long long target, uint32_t limit, int* err,
                                             const int* abort) {
    uint32_t spins = 0;
    while (ld_acquire_gpu_u64(flag) < target) {
        __nanosleep(spins < 64 ? 32 : 256);
        if (++spins > limit ||
            (abort != nullptr && *reinterpret_cast<const volatile int*>(abort) != 0)) {
            record_error(err, kDevDependTimeout);
            return false;
        }
    }
    return true;
}

// ------------------------------------------------------------------------------------------
// mbarrier + TMA (cp.async.bulk) wrappers, written from the PTX ISA
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase. Returns false (and records the error) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
    if (mbar_try_wait(bar, parity)) return true;
    for (uint32_t it = 0; it < kSpinLimit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(it > 4096 ? 256 : 32);
    }
    record_error(err, kDevMbarTimeout);
    return false;
}

// 3D tiled tensor load global -> shared, completion counted on an mbarrier (bytes).
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// 1D tiled tensor load (x must be a multiple of 16 bytes' worth of elements; out-of-range parts
// of the box, including negative coordinates, arrive as zeros).
__device__ __forceinline__ void tma_load_1d(void* dst, const void* tmap, int x, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2}], [%3];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Untiled bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16),
// completion counted on an mbarrier (bytes).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes),
        "r"(smem_u32(bar))
        : "memory");
}

// Barrier over the first `threads` threads of the block (named barrier `id`, 1..15).
__device__ __forceinline__ void named_sync(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const void* tmap) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

}  // namespace ph3
