// dslash_mrhs_tc.cu -- multi-RHS hopping matrix for 16-bit fields on the
// tensor cores (mma.sync, FP32 accumulation).
//
// The per-link work of the reference's _su3_multiply / _su3_inverse_multiply
// (include/su3.h:298-307) applied to a block of right-hand sides is a small
// GEMM: chi(rhs, spin) = M h(rhs, spin), M = U or U^dag, a 3x3 complex matrix
// times a 3 x (2 spins x nrhs) block. In real form, with complex numbers as
// (re, im) pairs:
//
//   D[m][n] = sum_k A[m][k] B[k][n],   m = rhs + 8 spin   (8 RHS x 2 spins)
//                                      k = 2 c' + re/im   (colour in, 6 of 8)
//                                      n = 2 c  + re/im   (colour out, 6 of 8)
//   A = the projected half-spinors h (16 x 8), B = M in real form (8 x 8):
//   B[2c'][2c] = Re M[c][c'], B[2c'+1][2c] = -Im M[c][c'],
//   B[2c'][2c+1] = Im M[c][c'], B[2c'+1][2c+1] = Re M[c][c'].
//
// One mma.sync.m16n8k8 per site and direction serves a tile of 8 RHS. With
// the m16n8k8 fragment layouts (lane = 4 g + t):
//   A: lane holds h(rhs g, spin 0 / 1) at colour t      (t = 3: padding, 0)
//   B: lane holds the complex M[g/2][t], arranged by g's parity
//   D: lane holds chi(rhs g, spin 0 / 1) at colour t
// so a lane owns the output spinor of (rhs g, colour t) for all four spins:
// the projection, the rebuild of the lower spins (signs and factors of i) and
// the storage norm of the neighbour are applied by the lane to its own
// registers, with no exchange between lanes. One warp computes one output
// site for all right-hand sides of the block (RHS tiles in a loop, the link
// fragment loaded once per direction).
//
// Precision: the fields are 16-bit with a per-site norm (stored value =
// value / norm); the tensor core multiplies the stored values (h rounded to
// the storage type after the projection, M in the storage type, row 2 of a
// link rebuilt in FP32 and rounded) and accumulates in FP32; the norms and
// the sum over directions are applied in FP32. Results agree with the
// scalar kernels (dslash_mrhs.cu) within the 16-bit storage error.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "dslash_core.cuh"
#include "internal.h"

namespace plqcd {
namespace dev {

struct TcArgs {
    const void *gauge;
    const char *in;
    char *out;
    const char *x;
    size_t fbytes;  // bytes of one field of the block
    int nrhs;
    long Vh;
    int L0, L0h, L1, L2, L3;
    int out_parity;
    float a_up, a_low, b, g5_in;
};

// D += A B with A 16x8, B 8x8 (16-bit), D 16x8 FP32
template <int PREC>
__device__ __forceinline__ void mma_16x8x8(float d[4], uint32_t a0, uint32_t a1, uint32_t b0);

template <>
__device__ __forceinline__ void mma_16x8x8<PLQCD_F16>(float d[4], uint32_t a0, uint32_t a1, uint32_t b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(b0));
}

template <>
__device__ __forceinline__ void mma_16x8x8<PLQCD_BF16>(float d[4], uint32_t a0, uint32_t a1, uint32_t b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(b0));
}

// 16-bit complex arithmetic on (re, im) pairs
template <int PREC>
struct H2;
template <>
struct H2<PLQCD_F16> {
    __device__ static __forceinline__ uint32_t fma(uint32_t a, uint32_t b, uint32_t c) {
        __half2 r = __hfma2(*reinterpret_cast<__half2 *>(&a), *reinterpret_cast<__half2 *>(&b),
                            *reinterpret_cast<__half2 *>(&c));
        return *reinterpret_cast<uint32_t *>(&r);
    }
};
template <>
struct H2<PLQCD_BF16> {
    __device__ static __forceinline__ uint32_t fma(uint32_t a, uint32_t b, uint32_t c) {
        __nv_bfloat162 r = __hfma2(*reinterpret_cast<__nv_bfloat162 *>(&a), *reinterpret_cast<__nv_bfloat162 *>(&b),
                                   *reinterpret_cast<__nv_bfloat162 *>(&c));
        return *reinterpret_cast<uint32_t *>(&r);
    }
};

__device__ __forceinline__ uint32_t swap_halves(uint32_t w) { return __byte_perm(w, 0, 0x1032); }

// Per direction MU (0..3) and the projection's lower-spin partners: upper
// spin s pairs with lower spin SIGMA[s] with factor F (1 real, or i times)
// and sign SGN (lib/dirac.c:95-114, 163-195):
//   mu 0: s0 + s2,   s1 + s3        mu 1: s0 + i s3, s1 + i s2
//   mu 2: s0 + s3,   s1 - s2        mu 3: s0 + i s2, s1 - i s3
__host__ __device__ constexpr int tc_sigma(int mu, int s) {
    return (mu == 0 || mu == 3) ? (s == 0 ? 2 : 3) : (s == 0 ? 3 : 2);
}
__host__ __device__ constexpr bool tc_imag(int mu) { return mu == 1 || mu == 3; }
__host__ __device__ constexpr int tc_sign(int mu, int s) { return (s == 1 && (mu == 2 || mu == 3)) ? -1 : 1; }

// multipliers (as 16-bit pairs) of the lower-spin term for sign `sg`:
// real factor f: (f, f) on psi_sigma; imaginary factor i f: (-f, f) on the
// swapped pair (i (x + i y) = -y + i x)
template <int PREC>
__device__ __forceinline__ uint32_t tc_mult(int imag, float f) {
    return imag ? Half2<PREC>::pack(-f, f) : Half2<PREC>::pack(f, f);
}

template <int PREC, int NT, bool XPAY>
__global__ void __launch_bounds__(128) k_dslash_mrhs_tc(const TcArgs a) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const long h = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (h >= a.Vh) return;  // warp-uniform
    const int rhs0 = blockIdx.y * 8 * NT;
    const int par = a.out_parity, opp = par ^ 1;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(h, par, L0h, L1, L2);
    const int xh = (int)(h - c.row * L0h);
    const long L01 = L1, L012 = (long)L1 * L2;
    const int xp = (c.x + 1 == a.L0) ? 0 : c.x + 1;
    const int xm = (c.x == 0) ? a.L0 - 1 : c.x - 1;
    long nb[8];
    nb[0] = (xp >> 1) + L0h * c.row;
    nb[1] = xh + L0h * (c.row + ((c.y + 1 == L1) ? -(long)(L1 - 1) : 1L));
    nb[2] = xh + L0h * (c.row + ((c.z + 1 == L2) ? -(long)(L2 - 1) * L01 : L01));
    nb[3] = xh + L0h * (c.row + ((c.t + 1 == L3) ? -(long)(L3 - 1) * L012 : L012));
    nb[4] = (xm >> 1) + L0h * c.row;
    nb[5] = xh + L0h * (c.row + ((c.y == 0) ? (long)(L1 - 1) : -1L));
    nb[6] = xh + L0h * (c.row + ((c.z == 0) ? (long)(L2 - 1) * L01 : -L01));
    nb[7] = xh + L0h * (c.row + ((c.t == 0) ? (long)(L3 - 1) * L012 : -L012));

    // link of direction d: forward U_mu(x) (this parity, this site),
    // backward U_mu(x - mu) (other parity, neighbour `site`); complex
    // element idx = 3 row + col of rows 0, 1
    const uint32_t *gw = static_cast<const uint32_t *>(a.gauge);
    auto link_word = [&](int d, long site, int idx) -> uint32_t {
        const int blk = d < 4 ? par * 4 + d : opp * 4 + (d - 4);
        return __ldg(gw + (((long)blk * 3 + (idx >> 1)) * Vh + site) * 2 + (idx & 1));
    };
    // row 2 of the eight links, rebuilt once per site: lane (g, t < 3)
    // computes U_g[2][t] = conj(U[0][t1] U[1][t2] - U[0][t2] U[1][t1]) of
    // direction g (its site picked by selects: nb stays in registers)
    float2 r2 = make_float2(0.f, 0.f);
    if (t < 3) {
        long sg_site = h;
#pragma unroll
        for (int d = 4; d < 8; d++) sg_site = g == d ? nb[d] : sg_site;
        const int t1 = t == 2 ? 0 : t + 1, t2 = t == 0 ? 2 : t - 1;
        const float2 a1 = Half2<PREC>::unpack(link_word(g, sg_site, t1));
        const float2 b2 = Half2<PREC>::unpack(link_word(g, sg_site, 3 + t2));
        const float2 a2 = Half2<PREC>::unpack(link_word(g, sg_site, t2));
        const float2 b1 = Half2<PREC>::unpack(link_word(g, sg_site, 3 + t1));
        const float re = (a1.x * b2.x - a1.y * b2.y) - (a2.x * b1.x - a2.y * b1.y);
        const float im = (a1.x * b2.y + a1.y * b2.x) - (a2.x * b1.y + a2.y * b1.x);
        r2 = make_float2(re, -im);
    }

    // byte offsets of psi(spin s, colour t) inside a site of a field: the
    // complex number 3 s + t sits in plane (3 s + t) / 4, slot (3 s + t) % 4
    const int tc = t < 3 ? t : 0;
    long off[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const int idx = 3 * s + tc;
        off[s] = (long)(idx >> 2) * Vh * 16 + (idx & 3) * 4;
    }
    const long norm_off = 3 * Vh * 16;

    // accumulators: lane (g, t < 3) owns spins 0..3 at colour t of RHS
    // rhs0 + 8 j + g, j < NT
    cx<float> acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; j++)
#pragma unroll
        for (int s = 0; s < 4; s++) acc[j][s] = {0.f, 0.f};

    const float sg_in = a.g5_in;
#pragma unroll
    for (int kd = 0; kd < 8; kd++) {
        const int d = dir_at(kd);
        const int mu = d & 3;
        const bool fwd = d < 4;
        // B fragment: M[cr][t] with cr = g / 2, M = U (forward) or U^dag
        // (backward: conj(U[t][cr])); row 2 from the lane that rebuilt it
        const int cr = g >> 1;
        const int row = fwd ? cr : t, col = fwd ? t : cr;
        const float2 sh = make_float2(__shfl_sync(0xffffffffu, r2.x, 4 * d + (col < 3 ? col : 0)),
                                      __shfl_sync(0xffffffffu, r2.y, 4 * d + (col < 3 ? col : 0)));
        uint32_t b0 = 0;
        if (g < 6 && t < 3) {
            float2 m = row < 2 ? Half2<PREC>::unpack(link_word(d, fwd ? h : nb[d], 3 * row + col)) : sh;
            if (!fwd) m.y = -m.y;  // U^dag: conjugate
            b0 = (g & 1) ? Half2<PREC>::pack(m.y, m.x) : Half2<PREC>::pack(m.x, -m.y);
        }
        // projection multipliers; backward and gamma5-on-input flip the
        // lower-spin sign
        const float sg = fwd ? sg_in : -sg_in;
        const uint32_t f0 = tc_mult<PREC>(tc_imag(mu), sg * tc_sign(mu, 0));
        const uint32_t f1 = tc_mult<PREC>(tc_imag(mu), sg * tc_sign(mu, 1));
        const int s0 = tc_sigma(mu, 0), s1 = tc_sigma(mu, 1);
        const long nsite = nb[d] * 16;
#pragma unroll
        for (int j = 0; j < NT; j++) {
            const int r = rhs0 + 8 * j + g;
            uint32_t a0 = 0, a1 = 0;
            float n = 0.f;
            if (t < 3 && r < a.nrhs) {
                const char *f = a.in + (size_t)r * a.fbytes;
                const uint32_t p0 = __ldg(reinterpret_cast<const uint32_t *>(f + nsite + off[0]));
                const uint32_t p1 = __ldg(reinterpret_cast<const uint32_t *>(f + nsite + off[1]));
                uint32_t q0 = __ldg(reinterpret_cast<const uint32_t *>(f + nsite + off[s0]));
                uint32_t q1 = __ldg(reinterpret_cast<const uint32_t *>(f + nsite + off[s1]));
                n = __ldg(reinterpret_cast<const float *>(f + norm_off) + nb[d]);
                if (tc_imag(mu)) {
                    q0 = swap_halves(q0);
                    q1 = swap_halves(q1);
                }
                a0 = H2<PREC>::fma(q0, f0, p0);
                a1 = H2<PREC>::fma(q1, f1, p1);
            }
            float dd[4] = {0.f, 0.f, 0.f, 0.f};
            mma_16x8x8<PREC>(dd, a0, a1, b0);
            // chi0 = (dd[0], dd[1]), chi1 = (dd[2], dd[3]); rebuild as
            // dslash_core.cuh::accumulate (LS = +1 forward, -1 backward)
            const float p = fwd ? n : -n, q = -p;
            cx<float> *o = acc[j];
            o[0] = {fmaf(n, dd[0], o[0].re), fmaf(n, dd[1], o[0].im)};
            o[1] = {fmaf(n, dd[2], o[1].re), fmaf(n, dd[3], o[1].im)};
            if (mu == 0) {
                o[2] = {fmaf(p, dd[0], o[2].re), fmaf(p, dd[1], o[2].im)};
                o[3] = {fmaf(p, dd[2], o[3].re), fmaf(p, dd[3], o[3].im)};
            } else if (mu == 1) {
                o[2] = {fmaf(p, dd[3], o[2].re), fmaf(q, dd[2], o[2].im)};
                o[3] = {fmaf(p, dd[1], o[3].re), fmaf(q, dd[0], o[3].im)};
            } else if (mu == 2) {
                o[2] = {fmaf(q, dd[2], o[2].re), fmaf(q, dd[3], o[2].im)};
                o[3] = {fmaf(p, dd[0], o[3].re), fmaf(p, dd[1], o[3].im)};
            } else {
                o[2] = {fmaf(p, dd[1], o[2].re), fmaf(q, dd[0], o[2].im)};
                o[3] = {fmaf(q, dd[3], o[3].re), fmaf(p, dd[2], o[3].im)};
            }
        }
    }

    // epilogue: a_up / a_low (gamma5 on output) [+ b x], then the 16-bit
    // store with the site norm = max |component| over the quad's lanes
#pragma unroll
    for (int j = 0; j < NT; j++) {
        const int r = rhs0 + 8 * j + g;
        const bool mine = t < 3 && r < a.nrhs;
        cx<float> v[4];
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const float as = s < 2 ? a.a_up : a.a_low;
            v[s] = {as * acc[j][s].re, as * acc[j][s].im};
        }
        if (XPAY && mine) {
            const char *f = a.x + (size_t)r * a.fbytes;
            const float nx = __ldg(reinterpret_cast<const float *>(f + norm_off) + h) * a.b;
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const float2 w = Half2<PREC>::unpack(__ldg(reinterpret_cast<const uint32_t *>(f + h * 16 + off[s])));
                v[s] = {fmaf(nx, w.x, v[s].re), fmaf(nx, w.y, v[s].im)};
            }
        }
        float m = 0.f;
        if (mine)
#pragma unroll
            for (int s = 0; s < 4; s++) m = fmaxf(m, fmaxf(fabsf(v[s].re), fabsf(v[s].im)));
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
        if (!mine) continue;
        const float inv = m > 0.f ? 1.f / m : 0.f;
        char *f = a.out + (size_t)r * a.fbytes;
#pragma unroll
        for (int s = 0; s < 4; s++)
            *reinterpret_cast<uint32_t *>(f + h * 16 + off[s]) = Half2<PREC>::pack(v[s].re * inv, v[s].im * inv);
        if (t == 0) reinterpret_cast<float *>(f + norm_off)[h] = m;
    }
}

template <int PREC, int NT>
int launch_tc_nt(cudaStream_t s, const TcArgs &a, bool xpay) {
    constexpr int kWarps = 4;
    const long nblk = (a.Vh + kWarps - 1) / kWarps;
    const int ngroups = (a.nrhs + 8 * NT - 1) / (8 * NT);
    if (nblk > 0x7fffffffL || ngroups > 65535) return set_error(PLQCD_ERR_ARG, "dslash_mrhs_tc: grid too large");
    dim3 grid((unsigned)nblk, (unsigned)ngroups);
    if (xpay)
        k_dslash_mrhs_tc<PREC, NT, true><<<grid, 32 * kWarps, 0, s>>>(a);
    else
        k_dslash_mrhs_tc<PREC, NT, false><<<grid, 32 * kWarps, 0, s>>>(a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

}  // namespace dev

// The tensor-core multi-RHS hop: 16-bit spinors with 12-real 16-bit links;
// `tiles` RHS tiles of 8 per warp (1, 2 or 4). Same arguments and semantics
// as the scalar multi-RHS kernels (a block of nrhs one-parity fields back to
// back, out = a_up/a_low * H in + b * x).
int launch_dslash_mrhs_tc(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                          const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x, double b,
                          int tiles) {
    if ((prec != PLQCD_F16 && prec != PLQCD_BF16) || recon != 12)
        return set_error(PLQCD_ERR_ARG, "dslash_mrhs_tc: 16-bit fields with 12-real links only");
    dev::TcArgs t{};
    t.gauge = gauge;
    t.in = static_cast<const char *>(in);
    t.out = static_cast<char *>(out);
    t.x = static_cast<const char *>(x);
    t.fbytes = spinor_parity_bytes(g.Vh, prec);
    t.nrhs = nrhs;
    t.Vh = g.Vh;
    t.L0 = g.L[0];
    t.L0h = g.L0h;
    t.L1 = g.L[1];
    t.L2 = g.L[2];
    t.L3 = g.L[3];
    t.out_parity = out_parity;
    t.a_up = (float)a;
    t.a_low = (float)((flags & PLQCD_DSLASH_G5_OUT) ? -a : a);
    t.b = (float)b;
    t.g5_in = (flags & PLQCD_DSLASH_G5_IN) ? -1.f : 1.f;
    const bool xp = x != nullptr;
#define PLQCD_TC_CASE(P)                                                          \
    if (prec == P) {                                                              \
        if (tiles == 1) return dev::launch_tc_nt<P, 1>(s, t, xp);                 \
        if (tiles == 2) return dev::launch_tc_nt<P, 2>(s, t, xp);                 \
        if (tiles == 4) return dev::launch_tc_nt<P, 4>(s, t, xp);                 \
    }
    PLQCD_TC_CASE(PLQCD_F16)
    PLQCD_TC_CASE(PLQCD_BF16)
#undef PLQCD_TC_CASE
    return set_error(PLQCD_ERR_ARG, "dslash_mrhs_tc: %d RHS tiles per warp not available", tiles);
}

}  // namespace plqcd
