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

// asynchronous global -> shared copies that write zeros when `valid` is
// false (source size 0: nothing is read; the address is still a valid one)
__device__ __forceinline__ void cp_async16_zf(uint32_t dst, const void *src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async4_zf(uint32_t dst, const void *src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 4 : 0)
                 : "memory");
}

// the B fragment of M[cr][t] for lane (g, t), from its (re, im) in FP32:
// g even: (Re, -Im), g odd: (Im, Re) (columns 2c and 2c + 1 of the real form)
template <int PREC>
__device__ __forceinline__ uint32_t b_frag(float2 m, int g) {
    return (g & 1) ? Half2<PREC>::pack(m.y, m.x) : Half2<PREC>::pack(m.x, -m.y);
}

// Shared memory of one warp: 2 stages x NT tiles; a tile holds, for the 8
// RHS of the tile, the neighbour spinor (record g: 12 words = the 3 planes
// of 16 bytes, complex number 3 s + c at word 3 s + c) and its norm
// (word 96 + g). Lane (g, t < 3) copies plane t of RHS g, lane (g, 3) the
// norm; the fragment reads (word 12 g + 3 s + t) hit 24 distinct banks.
constexpr int kTcTileWords = 8 * 12 + 8;
constexpr int kTcWarps = 4;

template <int PREC, int NT, bool XPAY>
__global__ void __launch_bounds__(32 * kTcWarps) k_dslash_mrhs_tc(const TcArgs a) {
    // 3 buffers per warp: stages 0 / 1 of the direction pipeline and the
    // epilogue's (xpay operand in, output out)
    constexpr int kStage = NT * kTcTileWords;
    __shared__ __align__(16) uint32_t smem[kTcWarps][3][kStage];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    // the warp's chunk: 32 consecutive sites; lane i works out the neighbour
    // indices of site h0 + i once (32-bit), the loop below takes them by shuffle
    const int Vh = (int)a.Vh;
    const int h0 = (blockIdx.x * kTcWarps + w) * 32;
    if (h0 >= Vh) return;  // warp-uniform
    const int nsite = min(32, Vh - h0);
    const int rhs0 = blockIdx.y * 8 * NT;
    const int par = a.out_parity, opp = par ^ 1;
    int nbl[8];
    {
        const int hl = min(h0 + lane, Vh - 1);
        const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
        const int row = hl / L0h, xh = hl - row * L0h;
        const int y = row % L1, zt = row / L1, z = zt % L2, tt = zt / L2;
        const int x = 2 * xh + ((y + z + tt + par) & 1);
        const int xp = (x + 1 == a.L0) ? 0 : x + 1, xm = (x == 0) ? a.L0 - 1 : x - 1;
        const int L01 = L1, L012 = L1 * L2;
        nbl[0] = (xp >> 1) + L0h * row;
        nbl[1] = xh + L0h * (row + ((y + 1 == L1) ? -(L1 - 1) : 1));
        nbl[2] = xh + L0h * (row + ((z + 1 == L2) ? -(L2 - 1) * L01 : L01));
        nbl[3] = xh + L0h * (row + ((tt + 1 == L3) ? -(L3 - 1) * L012 : L012));
        nbl[4] = (xm >> 1) + L0h * row;
        nbl[5] = xh + L0h * (row + ((y == 0) ? (L1 - 1) : -1));
        nbl[6] = xh + L0h * (row + ((z == 0) ? (L2 - 1) * L01 : -L01));
        nbl[7] = xh + L0h * (row + ((tt == 0) ? (L3 - 1) * L012 : -L012));
    }

    // the lane's source: plane t (t < 3) or the norm plane (t = 3) of RHS
    // rhs0 + 8 j + g; RHS past the block copy zeros from a valid address
    const char *src[NT];
    bool valid[NT];
    const long plane_off = t < 3 ? (long)t * Vh * 16 : 3L * Vh * 16;
    const int esz = t < 3 ? 16 : 4;
#pragma unroll
    for (int j = 0; j < NT; j++) {
        const int r = rhs0 + 8 * j + g;
        valid[j] = r < a.nrhs;
        src[j] = a.in + (size_t)(valid[j] ? r : 0) * a.fbytes + plane_off;
    }
    const uint32_t s_warp = smem_addr(&smem[w][0][0]);
    const uint32_t dst_lane = 4u * (t < 3 ? (uint32_t)(12 * g + 4 * t) : (uint32_t)(96 + g));
    // copies of direction kd's neighbour (site index n) into stage kd & 1
    auto issue = [&](int kd, int n) {
        const uint32_t sb = s_warp + 4u * (uint32_t)((kd & 1) * kStage) + dst_lane;
#pragma unroll
        for (int j = 0; j < NT; j++) {
            const uint32_t dst = sb + 4u * (uint32_t)(j * kTcTileWords);
            const char *p = src[j] + (long)n * esz;
            if (t < 3)
                cp_async16_zf(dst, p, valid[j]);
            else
                cp_async4_zf(dst, p, valid[j]);
        }
        cp_async_commit();
    };
    const uint32_t *gw = static_cast<const uint32_t *>(a.gauge);
    const long Vh2 = 2L * Vh;
    // 32-bit word of complex element idx (= 3 row + col, rows 0, 1) of the
    // link block blk (parity * 4 + mu) at `site`
    auto link_word = [&](int blk, int site, int idx) -> uint32_t {
        return __ldg(gw + ((long)blk * 3 + (idx >> 1)) * Vh2 + 2L * site + (idx & 1));
    };
    const float sgi = a.g5_in;
    const uint32_t m_re[2] = {Half2<PREC>::pack(sgi, sgi), Half2<PREC>::pack(-sgi, -sgi)};
    const uint32_t m_im[2] = {Half2<PREC>::pack(-sgi, sgi), Half2<PREC>::pack(sgi, -sgi)};

    int nb[8];
#pragma unroll
    for (int d = 0; d < 8; d++) nb[d] = __shfl_sync(0xffffffffu, nbl[d], 0);
    issue(0, nb[0]);
    issue(1, nb[4]);

    for (int k = 0; k < nsite; k++) {
        const int h = h0 + k;
        // row 2 of the eight links of site h: lane (g, t < 3) computes
        // U_g[2][t] = conj(U[0][t1] U[1][t2] - U[0][t2] U[1][t1]) of
        // direction g (forward: this site; backward: the neighbour)
        float2 r2 = make_float2(0.f, 0.f);
        if (t < 3) {
            int lsite = h;
#pragma unroll
            for (int d = 4; d < 8; d++) lsite = g == d ? nb[d] : lsite;
            const int blk = g < 4 ? par * 4 + g : opp * 4 + (g - 4);
            const int t1 = t == 2 ? 0 : t + 1, t2 = t == 0 ? 2 : t - 1;
            const float2 a1 = Half2<PREC>::unpack(link_word(blk, lsite, t1));
            const float2 b2 = Half2<PREC>::unpack(link_word(blk, lsite, 3 + t2));
            const float2 a2 = Half2<PREC>::unpack(link_word(blk, lsite, t2));
            const float2 b1 = Half2<PREC>::unpack(link_word(blk, lsite, 3 + t1));
            const float re = (a1.x * b2.x - a1.y * b2.y) - (a2.x * b1.x - a2.y * b1.y);
            const float im = (a1.x * b2.y + a1.y * b2.x) - (a2.x * b1.y + a2.y * b1.x);
            r2 = make_float2(re, -im);
        }

        float2 acc[NT][4];
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int s = 0; s < 4; s++) acc[j][s] = make_float2(0.f, 0.f);

#pragma unroll
        for (int kd = 0; kd < 8; kd++) {
            const int d = dir_at(kd);
            const int mu = d & 3;
            const bool fwd = d < 4;
            const bool imag = mu == 1 || mu == 3;  // the lower spins take a factor i
            // B fragment: M[cr][t] with cr = g / 2, M = U (forward) or U^dag
            // (backward: conj(U[t][cr])); row 2 from the lane that rebuilt it.
            // For mu 1 and 3 a second fragment holds i M, so that the mma
            // also returns i chi for the lower spins.
            const int cr = g >> 1;
            const int row = fwd ? cr : t, col = fwd ? t : cr;
            const int srcl = 4 * d + (col < 3 ? col : 0);
            const float2 sh = make_float2(__shfl_sync(0xffffffffu, r2.x, srcl), __shfl_sync(0xffffffffu, r2.y, srcl));
            float2 m = make_float2(0.f, 0.f);
            if (g < 6 && t < 3) {
                m = row < 2 ? Half2<PREC>::unpack(link_word(fwd ? par * 4 + mu : opp * 4 + mu, fwd ? h : nb[d],
                                                            3 * row + col))
                            : sh;
                if (!fwd) m.y = -m.y;  // U^dag: conjugate
            }
            const uint32_t b0 = b_frag<PREC>(m, g);
            const uint32_t bi = imag ? b_frag<PREC>(make_float2(-m.y, m.x), g) : 0u;
            // projection: spin s (0, 1) pairs with spin sigma(s) of the lower
            // half; the sign carries the direction (forward +, backward -)
            const int sg0 = (fwd ? 1 : -1) * tc_sign(mu, 0), sg1 = (fwd ? 1 : -1) * tc_sign(mu, 1);
            const uint32_t f0 = imag ? m_im[sg0 > 0 ? 0 : 1] : m_re[sg0 > 0 ? 0 : 1];
            const uint32_t f1 = imag ? m_im[sg1 > 0 ? 0 : 1] : m_re[sg1 > 0 ? 0 : 1];
            const int s0 = tc_sigma(mu, 0), s1 = tc_sigma(mu, 1);
            if (kd < 7)
                cp_async_wait<1>();
            else
                cp_async_wait<0>();
            __syncwarp();
            const uint32_t *st = &smem[w][kd & 1][0];
            const float LS = fwd ? 1.f : -1.f;
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const uint32_t *rec = st + j * kTcTileWords + 12 * g;
                uint32_t a0 = 0, a1 = 0;
                if (t < 3) {
                    uint32_t q0 = rec[3 * s0 + t], q1 = rec[3 * s1 + t];
                    if (imag) {
                        q0 = swap_halves(q0);
                        q1 = swap_halves(q1);
                    }
                    a0 = H2<PREC>::fma(q0, f0, rec[t]);
                    a1 = H2<PREC>::fma(q1, f1, rec[3 + t]);
                }
                const float n = *reinterpret_cast<const float *>(st + j * kTcTileWords + 96 + g);
                float dd[4] = {0.f, 0.f, 0.f, 0.f}, di[4] = {0.f, 0.f, 0.f, 0.f};
                mma_16x8x8<PREC>(dd, a0, a1, b0);
                if (imag) mma_16x8x8<PREC>(di, a0, a1, bi);
                // rebuild as dslash_core.cuh::accumulate: spins 0, 1 += n chi;
                // spins 2, 3 from chi (mu 0, 2) or i chi (mu 1, 3) with the
                // direction's signs (p = LS n, q = -p)
                const float2 nn = make_float2(n, n), pp = make_float2(LS * n, LS * n);
                const float2 qq = make_float2(-LS * n, -LS * n);
                const float2 c0 = make_float2(dd[0], dd[1]), c1 = make_float2(dd[2], dd[3]);
                const float2 i0 = make_float2(di[0], di[1]), i1 = make_float2(di[2], di[3]);
                float2 *o = acc[j];
                o[0] = __ffma2_rn(nn, c0, o[0]);
                o[1] = __ffma2_rn(nn, c1, o[1]);
                if (mu == 0) {
                    o[2] = __ffma2_rn(pp, c0, o[2]);
                    o[3] = __ffma2_rn(pp, c1, o[3]);
                } else if (mu == 1) {
                    o[2] = __ffma2_rn(qq, i1, o[2]);
                    o[3] = __ffma2_rn(qq, i0, o[3]);
                } else if (mu == 2) {
                    o[2] = __ffma2_rn(qq, c1, o[2]);
                    o[3] = __ffma2_rn(pp, c0, o[3]);
                } else {
                    o[2] = __ffma2_rn(qq, i0, o[2]);
                    o[3] = __ffma2_rn(pp, i1, o[3]);
                }
            }
            __syncwarp();  // every lane has read this stage before it is refilled
            if (kd + 2 < 8) issue(kd + 2, nb[dir_at(kd + 2)]);
        }

        // the next site's first two directions go in flight during this
        // site's epilogue
        if (k + 1 < nsite) {
#pragma unroll
            for (int d = 0; d < 8; d++) nb[d] = __shfl_sync(0xffffffffu, nbl[d], k + 1);
            issue(0, nb[0]);
            issue(1, nb[4]);
        }

        // epilogue: a_up / a_low (gamma5 on output) [+ b x], then the 16-bit
        // store with the site norm = max |component| over the quad's lanes,
        // through the epilogue buffer (whole 16-byte planes per lane)
        uint32_t *eb = &smem[w][2][0];
        const uint32_t s_eb = s_warp + 4u * (uint32_t)(2 * kStage);
        float2 xv[NT][4];
        float xn[NT];
        if (XPAY) {
            const long xoff = t < 3 ? (long)t * Vh * 16 + (long)h * 16 : 3L * Vh * 16 + (long)h * 4;
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const char *p = a.x + (size_t)(valid[j] ? rhs0 + 8 * j + g : 0) * a.fbytes + xoff;
                const uint32_t dst = s_eb + dst_lane + 4u * (uint32_t)(j * kTcTileWords);
                if (t < 3)
                    cp_async16_zf(dst, p, valid[j]);
                else
                    cp_async4_zf(dst, p, valid[j]);
            }
            cp_async_commit();
            cp_async_wait<0>();  // (also completes the next site's two stages)
            __syncwarp();
#pragma unroll
            for (int j = 0; j < NT; j++) {
                const uint32_t *rec = eb + j * kTcTileWords + 12 * g;
                xn[j] = *reinterpret_cast<const float *>(eb + j * kTcTileWords + 96 + g) * a.b;
#pragma unroll
                for (int s = 0; s < 4; s++) xv[j][s] = t < 3 ? Half2<PREC>::unpack(rec[3 * s + t]) : make_float2(0.f, 0.f);
            }
            __syncwarp();
        }
#pragma unroll
        for (int j = 0; j < NT; j++) {
            const bool mine = t < 3 && valid[j];
            float2 v[4];
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const float as = s < 2 ? a.a_up : a.a_low;
                v[s] = __fmul2_rn(make_float2(as, as), acc[j][s]);
                if (XPAY) v[s] = __ffma2_rn(make_float2(xn[j], xn[j]), xv[j][s], v[s]);
            }
            float mx = 0.f;
            if (mine)
#pragma unroll
                for (int s = 0; s < 4; s++) mx = fmaxf(mx, fmaxf(fabsf(v[s].x), fabsf(v[s].y)));
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
            const float inv = mx > 0.f ? 1.f / mx : 0.f;
            uint32_t *rec = eb + j * kTcTileWords + 12 * g;
            if (t < 3)
#pragma unroll
                for (int s = 0; s < 4; s++) rec[3 * s + t] = Half2<PREC>::pack(v[s].x * inv, v[s].y * inv);
            __syncwarp();
            if (valid[j]) {
                char *f = a.out + (size_t)(rhs0 + 8 * j + g) * a.fbytes;
                if (t < 3)
                    *reinterpret_cast<uint4 *>(f + (long)t * Vh * 16 + (long)h * 16) =
                        *reinterpret_cast<const uint4 *>(rec + 4 * t);
                else
                    reinterpret_cast<float *>(f + 3L * Vh * 16)[h] = mx;
            }
        }
        __syncwarp();  // the epilogue buffer is free for the next site
    }
}

template <int PREC, int NT>
int launch_tc_nt(cudaStream_t s, const TcArgs &a, bool xpay) {
    constexpr int kWarps = kTcWarps;
    if (a.Vh > 0x3fffffffL) return set_error(PLQCD_ERR_ARG, "dslash_mrhs_tc: lattice too large");
    const long nchunk = (a.Vh + 31) / 32;  // 32 consecutive sites per warp
    const long nblk = (nchunk + kWarps - 1) / kWarps;
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
