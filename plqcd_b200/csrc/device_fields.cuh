// device_fields.cuh -- complex arithmetic and storage accessors for the
// device field layouts documented in include/plqcd_b200.h.
//
// Every accessor converts between a storage format in HBM and compute-type
// complex numbers in registers. Loads go through the read-only path; stores
// use streaming (evict-first) hints because outputs are not re-read by the
// launch that writes them.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "plqcd_b200.h"

namespace plqcd {
namespace dev {

template <typename R>
struct cx {
    R re, im;
};

template <typename R>
__device__ __forceinline__ cx<R> cadd(cx<R> a, cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R>
__device__ __forceinline__ cx<R> csub(cx<R> a, cx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R>
__device__ __forceinline__ cx<R> cmul(cx<R> a, cx<R> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>
__device__ __forceinline__ cx<R> conjmul(cx<R> a, cx<R> b) {  // conj(a) * b
    return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}
template <typename R>
__device__ __forceinline__ cx<R> cconj(cx<R> a) { return {a.re, -a.im}; }

// ---- streaming / read-only memory helpers ----------------------------------
__device__ __forceinline__ double2 ld_ro(const double2 *p) { return __ldg(p); }
__device__ __forceinline__ float4 ld_ro(const float4 *p) { return __ldg(p); }
__device__ __forceinline__ float2 ld_ro(const float2 *p) { return __ldg(p); }
__device__ __forceinline__ uint4 ld_ro(const uint4 *p) { return __ldg(p); }
__device__ __forceinline__ uint2 ld_ro(const uint2 *p) { return __ldg(p); }
__device__ __forceinline__ float ld_ro(const float *p) { return __ldg(p); }

__device__ __forceinline__ void st_cs(double2 *p, double2 v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(float4 *p, float4 v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(float2 *p, float2 v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(uint4 *p, uint4 v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(uint2 *p, uint2 v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(float *p, float v) { __stcs(p, v); }

// ---- asynchronous global->shared copies (cp.async, sm_80+) -------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
// 16 bytes, cached in L2 only
__device__ __forceinline__ void cp_async16_cg(uint32_t s, const void *g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
}
// 16 / 8 / 4 bytes, cached in L1 and L2
__device__ __forceinline__ void cp_async16_ca(uint32_t s, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t s, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t s, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---- 16-bit pair packing ----------------------------------------------------
template <int PREC>
struct Half2;
template <>
struct Half2<PLQCD_F16> {
    __device__ static __forceinline__ uint32_t pack(float a, float b) {
        __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<uint32_t *>(&h);
    }
    __device__ static __forceinline__ float2 unpack(uint32_t w) {
        __half2 h = *reinterpret_cast<__half2 *>(&w);
        return __half22float2(h);
    }
};
template <>
struct Half2<PLQCD_BF16> {
    __device__ static __forceinline__ uint32_t pack(float a, float b) {
        __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<uint32_t *>(&h);
    }
    __device__ static __forceinline__ float2 unpack(uint32_t w) {
        __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162 *>(&w);
        return __bfloat1622float2(h);
    }
};

// =============================================================================
// spinor storage (one parity)
// =============================================================================
template <int PREC>
struct SpinorIO;

template <>
struct SpinorIO<PLQCD_F64> {
    using real = double;
    static constexpr int bytes_per_site = 192;
    // raw loads: values as stored plus the factor that restores them (1 here)
    static constexpr bool kScaled = false;
    __device__ static __forceinline__ void load_raw(const void *b, long Vh, long h, cx<double> s[12], double &n) {
        load(b, Vh, h, s);
        n = 1.0;
    }
    __device__ static __forceinline__ void load_staged_raw(const uint4 *s0, int B, cx<double> s[12], double &n) {
        load_staged(s0, B, s);
        n = 1.0;
    }
    __device__ static __forceinline__ void load(const void *base, long Vh, long h, cx<double> s[12]) {
        const double2 *p = static_cast<const double2 *>(base) + h;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            double2 v = ld_ro(p + c * Vh);
            s[c] = {v.x, v.y};
        }
    }
    __device__ static __forceinline__ void store(void *base, long Vh, long h, const cx<double> s[12]) {
        double2 *p = static_cast<double2 *>(base) + h;
#pragma unroll
        for (int c = 0; c < 12; c++) st_cs(p + c * Vh, make_double2(s[c].re, s[c].im));
    }
    // staged form: NSLOT 16-byte shared-memory slots per site, slot j of
    // this thread at s0 + j*stride bytes
    static constexpr int NSLOT = 12;
    __device__ static __forceinline__ void issue(const void *base, long Vh, long h, uint32_t s0, int stride) {
        const double2 *p = static_cast<const double2 *>(base) + h;
#pragma unroll
        for (int c = 0; c < 12; c++) cp_async16_ca(s0 + c * stride, p + c * Vh);
    }
    __device__ static __forceinline__ void load_staged(const uint4 *s0, int B, cx<double> s[12]) {
#pragma unroll
        for (int c = 0; c < 12; c++) {
            double2 v = *reinterpret_cast<const double2 *>(s0 + c * B);
            s[c] = {v.x, v.y};
        }
    }
};

template <>
struct SpinorIO<PLQCD_F32> {
    using real = float;
    static constexpr int bytes_per_site = 96;
    static constexpr bool kScaled = false;
    __device__ static __forceinline__ void load_raw(const void *b, long Vh, long h, cx<float> s[12], float &n) {
        load(b, Vh, h, s);
        n = 1.0f;
    }
    __device__ static __forceinline__ void load_staged_raw(const uint4 *s0, int B, cx<float> s[12], float &n) {
        load_staged(s0, B, s);
        n = 1.0f;
    }
    __device__ static __forceinline__ void load(const void *base, long Vh, long h, cx<float> s[12]) {
        const float4 *p = static_cast<const float4 *>(base) + h;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            float4 v = ld_ro(p + k * Vh);
            s[2 * k] = {v.x, v.y};
            s[2 * k + 1] = {v.z, v.w};
        }
    }
    __device__ static __forceinline__ void store(void *base, long Vh, long h, const cx<float> s[12]) {
        float4 *p = static_cast<float4 *>(base) + h;
#pragma unroll
        for (int k = 0; k < 6; k++)
            st_cs(p + k * Vh, make_float4(s[2 * k].re, s[2 * k].im, s[2 * k + 1].re, s[2 * k + 1].im));
    }
    static constexpr int NSLOT = 6;
    __device__ static __forceinline__ void issue(const void *base, long Vh, long h, uint32_t s0, int stride) {
        const float4 *p = static_cast<const float4 *>(base) + h;
#pragma unroll
        for (int k = 0; k < 6; k++) cp_async16_ca(s0 + k * stride, p + k * Vh);
    }
    __device__ static __forceinline__ void load_staged(const uint4 *s0, int B, cx<float> s[12]) {
#pragma unroll
        for (int k = 0; k < 6; k++) {
            float4 v = *reinterpret_cast<const float4 *>(s0 + k * B);
            s[2 * k] = {v.x, v.y};
            s[2 * k + 1] = {v.z, v.w};
        }
    }
};

// 16-bit storage with a per-site norm: value = stored * norm,
// norm = max |component| over the 24 reals of the site.
template <int PREC>
struct SpinorIO16 {
    using real = float;
    static constexpr int bytes_per_site = 52;
    // raw loads return the stored values unscaled and the site norm, so
    // the hopping kernels can apply the norm inside their final FMAs
    static constexpr bool kScaled = true;
    __device__ static __forceinline__ void unpack3(const uint4 v[3], cx<float> s[12]) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float2 a = Half2<PREC>::unpack(v[k].x), b = Half2<PREC>::unpack(v[k].y);
            float2 c = Half2<PREC>::unpack(v[k].z), d = Half2<PREC>::unpack(v[k].w);
            s[4 * k + 0] = {a.x, a.y};
            s[4 * k + 1] = {b.x, b.y};
            s[4 * k + 2] = {c.x, c.y};
            s[4 * k + 3] = {d.x, d.y};
        }
    }
    __device__ static __forceinline__ void load_raw(const void *base, long Vh, long h, cx<float> s[12], float &n) {
        const uint4 *p = static_cast<const uint4 *>(base) + h;
        uint4 v[3];
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = ld_ro(p + k * Vh);
        n = ld_ro(norms(base, Vh) + h);
        unpack3(v, s);
    }
    __device__ static __forceinline__ void load_staged_raw(const uint4 *s0, int B, cx<float> s[12], float &n) {
        uint4 v[3];
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = s0[k * B];
        n = *reinterpret_cast<const float *>(s0 + 3 * B);
        unpack3(v, s);
    }
    __device__ static __forceinline__ const float *norms(const void *base, long Vh) {
        return reinterpret_cast<const float *>(static_cast<const uint4 *>(base) + 3 * Vh);
    }
    __device__ static __forceinline__ void load(const void *base, long Vh, long h, cx<float> s[12]) {
        const uint4 *p = static_cast<const uint4 *>(base) + h;
        float n = ld_ro(norms(base, Vh) + h);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            uint4 v = ld_ro(p + k * Vh);
            float2 a = Half2<PREC>::unpack(v.x), b = Half2<PREC>::unpack(v.y);
            float2 c = Half2<PREC>::unpack(v.z), d = Half2<PREC>::unpack(v.w);
            s[4 * k + 0] = {a.x * n, a.y * n};
            s[4 * k + 1] = {b.x * n, b.y * n};
            s[4 * k + 2] = {c.x * n, c.y * n};
            s[4 * k + 3] = {d.x * n, d.y * n};
        }
    }
    __device__ static __forceinline__ void store(void *base, long Vh, long h, const cx<float> s[12]) {
        float m = 0.f;
#pragma unroll
        for (int c = 0; c < 12; c++) m = fmaxf(m, fmaxf(fabsf(s[c].re), fabsf(s[c].im)));
        float inv = m > 0.f ? 1.f / m : 0.f;
        uint4 *p = static_cast<uint4 *>(base) + h;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            uint4 v;
            v.x = Half2<PREC>::pack(s[4 * k + 0].re * inv, s[4 * k + 0].im * inv);
            v.y = Half2<PREC>::pack(s[4 * k + 1].re * inv, s[4 * k + 1].im * inv);
            v.z = Half2<PREC>::pack(s[4 * k + 2].re * inv, s[4 * k + 2].im * inv);
            v.w = Half2<PREC>::pack(s[4 * k + 3].re * inv, s[4 * k + 3].im * inv);
            st_cs(p + k * Vh, v);
        }
        st_cs(const_cast<float *>(norms(base, Vh)) + h, m);
    }
    static constexpr int NSLOT = 4;  // 3 x 16 bytes of values, the norm in slot 3
    __device__ static __forceinline__ void issue(const void *base, long Vh, long h, uint32_t s0, int stride) {
        const uint4 *p = static_cast<const uint4 *>(base) + h;
#pragma unroll
        for (int k = 0; k < 3; k++) cp_async16_ca(s0 + k * stride, p + k * Vh);
        cp_async4(s0 + 3 * stride, norms(base, Vh) + h);
    }
    __device__ static __forceinline__ void load_staged(const uint4 *s0, int B, cx<float> s[12]) {
        const float n = *reinterpret_cast<const float *>(s0 + 3 * B);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            uint4 v = s0[k * B];
            float2 a = Half2<PREC>::unpack(v.x), b = Half2<PREC>::unpack(v.y);
            float2 c = Half2<PREC>::unpack(v.z), d = Half2<PREC>::unpack(v.w);
            s[4 * k + 0] = {a.x * n, a.y * n};
            s[4 * k + 1] = {b.x * n, b.y * n};
            s[4 * k + 2] = {c.x * n, c.y * n};
            s[4 * k + 3] = {d.x * n, d.y * n};
        }
    }
};
template <>
struct SpinorIO<PLQCD_F16> : SpinorIO16<PLQCD_F16> {};
template <>
struct SpinorIO<PLQCD_BF16> : SpinorIO16<PLQCD_BF16> {};

// =============================================================================
// gauge storage: [parity][mu][element][Vh]
// =============================================================================

// row 2 of an SU(3) matrix from rows 0 and 1: conj(row0 x row1)
template <typename R>
__device__ __forceinline__ void reconstruct_row2(cx<R> U[9]) {
    U[6] = cconj(csub(cmul(U[1], U[5]), cmul(U[2], U[4])));
    U[7] = cconj(csub(cmul(U[2], U[3]), cmul(U[0], U[5])));
    U[8] = cconj(csub(cmul(U[0], U[4]), cmul(U[1], U[3])));
}

template <int PREC, int RECON>
struct LinkIO;

template <>
struct LinkIO<PLQCD_F64, 18> {
    using real = double;
    using elem = double2;
    static constexpr int NE = 9;
    static constexpr int NSLOT = 9;
    __device__ static __forceinline__ void issue(const void *base, long Vh, int par, int mu, long h, uint32_t s0,
                                                 int stride) {
        const double2 *p = static_cast<const double2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 9; e++) cp_async16_cg(s0 + e * stride, p + e * Vh);
    }
    __device__ static __forceinline__ void load_staged(const uint4 *s0, int B, cx<double> U[9]) {
#pragma unroll
        for (int e = 0; e < 9; e++) {
            double2 v = *reinterpret_cast<const double2 *>(s0 + e * B);
            U[e] = {v.x, v.y};
        }
    }
    __device__ static __forceinline__ void load(const void *base, long Vh, int par, int mu, long h,
                                                cx<double> U[9]) {
        const double2 *p = static_cast<const double2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            double2 v = ld_ro(p + e * Vh);
            U[e] = {v.x, v.y};
        }
    }
    __device__ static __forceinline__ void store(void *base, long Vh, int par, int mu, long h,
                                                 const cx<double> U[9]) {
        double2 *p = static_cast<double2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 9; e++) p[e * Vh] = make_double2(U[e].re, U[e].im);
    }
};

template <>
struct LinkIO<PLQCD_F64, 12> {
    using real = double;
    using elem = double2;
    static constexpr int NE = 6;
    static constexpr int NSLOT = 6;
    __device__ static __forceinline__ void issue(const void *base, long Vh, int par, int mu, long h, uint32_t s0,
                                                 int stride) {
        const double2 *p = static_cast<const double2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 6; e++) cp_async16_cg(s0 + e * stride, p + e * Vh);
    }
    __device__ static __forceinline__ void load_staged(const uint4 *s0, int B, cx<double> U[9]) {
#pragma unroll
        for (int e = 0; e < 6; e++) {
            double2 v = *reinterpret_cast<const double2 *>(s0 + e * B);
            U[e] = {v.x, v.y};
        }
        reconstruct_row2(U);
    }
    __device__ static __forceinline__ void load(const void *base, long Vh, int par, int mu, long h,
                                                cx<double> U[9]) {
        const double2 *p = static_cast<const double2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 6; e++) {
            double2 v = ld_ro(p + e * Vh);
            U[e] = {v.x, v.y};
        }
        reconstruct_row2(U);
    }
    __device__ static __forceinline__ void store(void *base, long Vh, int par, int mu, long h,
                                                 const cx<double> U[9]) {
        double2 *p = static_cast<double2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 6; e++) p[e * Vh] = make_double2(U[e].re, U[e].im);
    }
};

template <>
struct LinkIO<PLQCD_F32, 18> {
    using real = float;
    using elem = float2;
    static constexpr int NE = 9;
    static constexpr int NSLOT = 9;
    __device__ static __forceinline__ void issue(const void *base, long Vh, int par, int mu, long h, uint32_t s0,
                                                 int stride) {
        const float2 *p = static_cast<const float2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 9; e++) cp_async8(s0 + e * stride, p + e * Vh);
    }
    __device__ static __forceinline__ void load_staged(const uint4 *s0, int B, cx<float> U[9]) {
#pragma unroll
        for (int e = 0; e < 9; e++) {
            float2 v = *reinterpret_cast<const float2 *>(s0 + e * B);
            U[e] = {v.x, v.y};
        }
    }
    __device__ static __forceinline__ void load(const void *base, long Vh, int par, int mu, long h,
                                                cx<float> U[9]) {
        const float2 *p = static_cast<const float2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            float2 v = ld_ro(p + e * Vh);
            U[e] = {v.x, v.y};
        }
    }
    __device__ static __forceinline__ void store(void *base, long Vh, int par, int mu, long h,
                                                 const cx<double> U[9]) {
        float2 *p = static_cast<float2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 9; e++) p[e * Vh] = make_float2((float)U[e].re, (float)U[e].im);
    }
};

template <>
struct LinkIO<PLQCD_F32, 12> {
    using real = float;
    using elem = float4;
    static constexpr int NE = 3;
    static constexpr int NSLOT = 3;
    __device__ static __forceinline__ void issue(const void *base, long Vh, int par, int mu, long h, uint32_t s0,
                                                 int stride) {
        const float4 *p = static_cast<const float4 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 3; e++) cp_async16_cg(s0 + e * stride, p + e * Vh);
    }
    __device__ static __forceinline__ void load_staged(const uint4 *s0, int B, cx<float> U[9]) {
#pragma unroll
        for (int e = 0; e < 3; e++) {
            float4 v = *reinterpret_cast<const float4 *>(s0 + e * B);
            U[2 * e] = {v.x, v.y};
            U[2 * e + 1] = {v.z, v.w};
        }
        reconstruct_row2(U);
    }
    __device__ static __forceinline__ void load(const void *base, long Vh, int par, int mu, long h,
                                                cx<float> U[9]) {
        const float4 *p = static_cast<const float4 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 3; e++) {
            float4 v = ld_ro(p + e * Vh);
            U[2 * e] = {v.x, v.y};
            U[2 * e + 1] = {v.z, v.w};
        }
        reconstruct_row2(U);
    }
    __device__ static __forceinline__ void store(void *base, long Vh, int par, int mu, long h,
                                                 const cx<double> U[9]) {
        float4 *p = static_cast<float4 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 3; e++)
            p[e * Vh] = make_float4((float)U[2 * e].re, (float)U[2 * e].im, (float)U[2 * e + 1].re,
                                    (float)U[2 * e + 1].im);
    }
};

// 16-bit links, rows 0,1 only. SU(3) entries satisfy |U_ij| <= 1, so no
// scale factor is stored.
template <int PREC>
struct LinkIO16 {
    using real = float;
    using elem = uint2;
    static constexpr int NE = 3;
    static constexpr int NSLOT = 3;
    __device__ static __forceinline__ void issue(const void *base, long Vh, int par, int mu, long h, uint32_t s0,
                                                 int stride) {
        const uint2 *p = static_cast<const uint2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 3; e++) cp_async8(s0 + e * stride, p + e * Vh);
    }
    __device__ static __forceinline__ void load_staged(const uint4 *s0, int B, cx<float> U[9]) {
#pragma unroll
        for (int e = 0; e < 3; e++) {
            uint2 v = *reinterpret_cast<const uint2 *>(s0 + e * B);
            float2 a = Half2<PREC>::unpack(v.x), b = Half2<PREC>::unpack(v.y);
            U[2 * e] = {a.x, a.y};
            U[2 * e + 1] = {b.x, b.y};
        }
        reconstruct_row2(U);
    }
    __device__ static __forceinline__ void load(const void *base, long Vh, int par, int mu, long h,
                                                cx<float> U[9]) {
        const uint2 *p = static_cast<const uint2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 3; e++) {
            uint2 v = ld_ro(p + e * Vh);
            float2 a = Half2<PREC>::unpack(v.x), b = Half2<PREC>::unpack(v.y);
            U[2 * e] = {a.x, a.y};
            U[2 * e + 1] = {b.x, b.y};
        }
        reconstruct_row2(U);
    }
    __device__ static __forceinline__ void store(void *base, long Vh, int par, int mu, long h,
                                                 const cx<double> U[9]) {
        uint2 *p = static_cast<uint2 *>(base) + ((long)(par * 4 + mu) * NE) * Vh + h;
#pragma unroll
        for (int e = 0; e < 3; e++) {
            uint2 v;
            v.x = Half2<PREC>::pack((float)U[2 * e].re, (float)U[2 * e].im);
            v.y = Half2<PREC>::pack((float)U[2 * e + 1].re, (float)U[2 * e + 1].im);
            p[e * Vh] = v;
        }
    }
};
template <>
struct LinkIO<PLQCD_F16, 12> : LinkIO16<PLQCD_F16> {};
template <>
struct LinkIO<PLQCD_BF16, 12> : LinkIO16<PLQCD_BF16> {};

// ---- site coordinates of a half-site index ------------------------------------
struct Coords {
    int x, y, z, t;
    long row;  // y + L1*(z + L2*t)
};

__device__ __forceinline__ Coords site_coords(long h, int par, int L0h, int L1, int L2) {
    // 32-bit division (a 64-bit one is a long software sequence per site):
    // plqcd_lattice_create keeps Vh < 2^31
    Coords c;
    const int hi = (int)h;
    const int row = hi / L0h;
    const int xh = hi - row * L0h;
    const int zt = row / L1;
    c.y = row - zt * L1;
    c.t = zt / L2;
    c.z = zt - c.t * L2;
    c.row = row;
    c.x = 2 * xh + ((c.y + c.z + c.t + par) & 1);
    return c;
}

// even/odd indices of the eight neighbours of a site, in the order x+, y+,
// z+, t+, x-, y-, z-, t- (d = 0..3 forward mu, 4..7 backward), periodic;
// 32-bit like site_coords
__device__ __forceinline__ void neighbour_sites(const Coords &c, int xh, int L0, int L0h, int L1, int L2, int L3,
                                                int nb[8]) {
    const int row = (int)c.row;
    const int L012 = L1 * L2;
    const int xp = (c.x + 1 == L0) ? 0 : c.x + 1;
    const int xm = (c.x == 0) ? L0 - 1 : c.x - 1;
    nb[0] = (xp >> 1) + L0h * row;
    nb[1] = xh + L0h * (row + ((c.y + 1 == L1) ? -(L1 - 1) : 1));
    nb[2] = xh + L0h * (row + ((c.z + 1 == L2) ? -(L2 - 1) * L1 : L1));
    nb[3] = xh + L0h * (row + ((c.t + 1 == L3) ? -(L3 - 1) * L012 : L012));
    nb[4] = (xm >> 1) + L0h * row;
    nb[5] = xh + L0h * (row + ((c.y == 0) ? (L1 - 1) : -1));
    nb[6] = xh + L0h * (row + ((c.z == 0) ? (L2 - 1) * L1 : -L1));
    nb[7] = xh + L0h * (row + ((c.t == 0) ? (L3 - 1) * L012 : -L012));
}

}  // namespace dev
}  // namespace plqcd
