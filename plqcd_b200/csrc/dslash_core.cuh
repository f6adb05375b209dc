// dslash_core.cuh -- per-direction arithmetic of the Wilson hopping term,
// shared by the single- and multi-RHS kernels.
//
// For output site x and direction mu (reference lib/dirac.c:95-114,
// 163-195 for the projections, 269-311 and 371-398 for the rebuild):
//   forward:  chi  = U_mu(x)        h,  h  = upper((1 - g_mu) psi(x+mu))
//   backward: chi' = U_mu(x-mu)^dag h', h' = upper((1 + g_mu) psi(x-mu))
#pragma once

#include <type_traits>

#include "device_fields.cuh"

namespace plqcd {
namespace dev {

struct DslashArgs {
    const void *gauge;
    const void *in[2];  // input field of parity p (FULL) / in[0] = input (single parity)
    void *out[2];       // output field of parity p (FULL) / out[0] = output
    const void *x;      // xpay operand (single parity only)
    long Vh;
    long h_begin, h_end;  // output half-sites processed: [h_begin, h_end) (single parity)
    int L0, L0h, L1, L2, L3;
    int out_parity;
    double a_up, a_low, b;
    double g5_in;       // +1 or -1: sign applied to input spins 2,3
    // a block of nrhs fields (field r at base + r * fbytes), single parity
    // only: blocks cover the RHS of a site range consecutively (RHS fastest)
    int nrhs;
    long fbytes;
};

// Two FP32 lanes in one register pair, each operation one packed sm_100
// instruction (FFMA2 / FMUL2 / FADD2). Every lane is rounded exactly as the
// scalar operation, so the arithmetic below computes, lane by lane, the
// same bits as with R = float: two sites per thread, one per lane, take half
// the FP32 instructions of two scalar threads.
// (the operations are hidden friends: found for f2 arguments only, so they
// do not hide the scalar fma of the other types)
struct f2 {
    float2 v;
    f2() = default;
    __device__ __forceinline__ explicit f2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ f2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ explicit f2(float2 w) : v(w) {}
    __device__ friend __forceinline__ f2 fma(f2 a, f2 b, f2 c) { return f2(__ffma2_rn(a.v, b.v, c.v)); }
    __device__ friend __forceinline__ f2 operator*(f2 a, f2 b) { return f2(__fmul2_rn(a.v, b.v)); }
    __device__ friend __forceinline__ f2 operator+(f2 a, f2 b) { return f2(__fadd2_rn(a.v, b.v)); }
    __device__ friend __forceinline__ f2 operator-(f2 a) { return f2(-a.v.x, -a.v.y); }
    __device__ friend __forceinline__ f2 operator-(f2 a, f2 b) { return a + (-b); }
    // sign factors (+-1, exact)
    __device__ friend __forceinline__ f2 operator*(int s, f2 a) {
        return s == 1 ? a : (s == -1 ? -a : f2((float)s) * a);
    }
};

// lane pairing of per-site values
__device__ __forceinline__ cx<f2> zip(cx<float> a, cx<float> b) { return {f2(a.re, b.re), f2(a.im, b.im)}; }
__device__ __forceinline__ cx<float> lane(cx<f2> a, int j) {
    return j == 0 ? cx<float>{a.re.v.x, a.im.v.x} : cx<float>{a.re.v.y, a.im.v.y};
}

// projection of the neighbour spinor onto the two upper spin components.
// FWD: (1 - g_mu) psi(x+mu); backward: (1 + g_mu) psi(x-mu). `sg` is the
// sign on the lower spins (backward and gamma5-on-input flip it).
template <int MU, typename R>
__device__ __forceinline__ void project(const cx<R> s[12], R sg, cx<R> h0[3], cx<R> h1[3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const cx<R> s0 = s[c], s1 = s[3 + c], s2 = s[6 + c], s3 = s[9 + c];
        if (MU == 0) {  // s0 + s2, s1 + s3
            h0[c] = {fma(sg, s2.re, s0.re), fma(sg, s2.im, s0.im)};
            h1[c] = {fma(sg, s3.re, s1.re), fma(sg, s3.im, s1.im)};
        } else if (MU == 1) {  // s0 + i s3, s1 + i s2
            h0[c] = {fma(-sg, s3.im, s0.re), fma(sg, s3.re, s0.im)};
            h1[c] = {fma(-sg, s2.im, s1.re), fma(sg, s2.re, s1.im)};
        } else if (MU == 2) {  // s0 + s3, s1 - s2
            h0[c] = {fma(sg, s3.re, s0.re), fma(sg, s3.im, s0.im)};
            h1[c] = {fma(-sg, s2.re, s1.re), fma(-sg, s2.im, s1.im)};
        } else {  // s0 + i s2, s1 - i s3
            h0[c] = {fma(-sg, s2.im, s0.re), fma(sg, s2.re, s0.im)};
            h1[c] = {fma(sg, s3.im, s1.re), fma(-sg, s3.re, s1.im)};
        }
    }
}

template <typename R>
__device__ __forceinline__ void su3_mul(const cx<R> U[9], const cx<R> v[3], cx<R> r[3]) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        R re = U[3 * a].re * v[0].re;
        R im = U[3 * a].re * v[0].im;
        re = fma(-U[3 * a].im, v[0].im, re);
        im = fma(U[3 * a].im, v[0].re, im);
#pragma unroll
        for (int b = 1; b < 3; b++) {
            re = fma(U[3 * a + b].re, v[b].re, re);
            re = fma(-U[3 * a + b].im, v[b].im, re);
            im = fma(U[3 * a + b].re, v[b].im, im);
            im = fma(U[3 * a + b].im, v[b].re, im);
        }
        r[a] = {re, im};
    }
}

template <typename R>
__device__ __forceinline__ void su3_dag_mul(const cx<R> U[9], const cx<R> v[3], cx<R> r[3]) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        R re = U[a].re * v[0].re;
        R im = U[a].re * v[0].im;
        re = fma(U[a].im, v[0].im, re);
        im = fma(-U[a].im, v[0].re, im);
#pragma unroll
        for (int b = 1; b < 3; b++) {
            re = fma(U[3 * b + a].re, v[b].re, re);
            re = fma(U[3 * b + a].im, v[b].im, re);
            im = fma(U[3 * b + a].re, v[b].im, im);
            im = fma(-U[3 * b + a].im, v[b].re, im);
        }
        r[a] = {re, im};
    }
}

// rebuild of the lower spins from chi = (c0, c1); LS = +1 forward, -1 backward.
// SC: chi still carries the neighbour's storage norm n (16-bit spinors are
// loaded unscaled); it is applied here by fused multiply-adds, for free.
template <int MU, int LS, bool LOWER, bool SC, typename R>
__device__ __forceinline__ void accumulate(cx<R> acc[12], const cx<R> c0[3], const cx<R> c1[3], R n) {
    if (SC) {
        const R p = LS * n, q = -LS * n;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            acc[c] = {fma(n, c0[c].re, acc[c].re), fma(n, c0[c].im, acc[c].im)};
            acc[3 + c] = {fma(n, c1[c].re, acc[3 + c].re), fma(n, c1[c].im, acc[3 + c].im)};
            if (!LOWER) continue;
            cx<R> &r2 = acc[6 + c];
            cx<R> &r3 = acc[9 + c];
            if (MU == 0) {
                r2 = {fma(p, c0[c].re, r2.re), fma(p, c0[c].im, r2.im)};
                r3 = {fma(p, c1[c].re, r3.re), fma(p, c1[c].im, r3.im)};
            } else if (MU == 1) {
                r2 = {fma(p, c1[c].im, r2.re), fma(q, c1[c].re, r2.im)};
                r3 = {fma(p, c0[c].im, r3.re), fma(q, c0[c].re, r3.im)};
            } else if (MU == 2) {
                r2 = {fma(q, c1[c].re, r2.re), fma(q, c1[c].im, r2.im)};
                r3 = {fma(p, c0[c].re, r3.re), fma(p, c0[c].im, r3.im)};
            } else {
                r2 = {fma(p, c0[c].im, r2.re), fma(q, c0[c].re, r2.im)};
                r3 = {fma(q, c1[c].im, r3.re), fma(p, c1[c].re, r3.im)};
            }
        }
        return;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        acc[c] = cadd(acc[c], c0[c]);
        acc[3 + c] = cadd(acc[3 + c], c1[c]);
        if (!LOWER) continue;
        cx<R> &r2 = acc[6 + c];
        cx<R> &r3 = acc[9 + c];
        if (MU == 0) {  // r2 += LS c0, r3 += LS c1
            r2 = {r2.re + LS * c0[c].re, r2.im + LS * c0[c].im};
            r3 = {r3.re + LS * c1[c].re, r3.im + LS * c1[c].im};
        } else if (MU == 1) {  // r2 += -LS i c1, r3 += -LS i c0
            r2 = {r2.re + LS * c1[c].im, r2.im - LS * c1[c].re};
            r3 = {r3.re + LS * c0[c].im, r3.im - LS * c0[c].re};
        } else if (MU == 2) {  // r2 += -LS c1, r3 += LS c0
            r2 = {r2.re - LS * c1[c].re, r2.im - LS * c1[c].im};
            r3 = {r3.re + LS * c0[c].re, r3.im + LS * c0[c].im};
        } else {  // r2 += -LS i c0, r3 += LS i c1
            r2 = {r2.re + LS * c0[c].im, r2.im - LS * c0[c].re};
            r3 = {r3.re - LS * c1[c].im, r3.im + LS * c1[c].re};
        }
    }
}

// Projection, SU(3) product and rebuild of one direction on data already in
// registers.
// The reference as shipped drops every forward contribution to spins 2,3
// (its backward mu=0 step overwrites them, include/su3.h:135-138): COMPAT.
// SC / n: see accumulate (n = 1 and unused when SC is false).
template <int MU, bool FWD, bool COMPAT, bool SC, typename R>
__device__ __forceinline__ void compute_dir(cx<R> acc[12], const cx<R> s[12], const cx<R> U[9], R sg_in, R n) {
    cx<R> h0[3], h1[3];
    project<MU, R>(s, FWD ? sg_in : -sg_in, h0, h1);
    cx<R> c0[3], c1[3];
    if (FWD) {
        su3_mul(U, h0, c0);
        su3_mul(U, h1, c1);
    } else {
        su3_dag_mul(U, h0, c0);
        su3_dag_mul(U, h1, c1);
    }
    accumulate<MU, FWD ? 1 : -1, !(COMPAT && FWD), SC, R>(acc, c0, c1, n);
}

// Accumulation order of the eight directions in every kernel: x+, x-, y+,
// y-, z+, z-, t+, t- (d = 0..3 forward mu, 4..7 backward mu). Forward and
// backward terms of one axis read the same rows and links of the other
// parity, so the row-staging kernels consume them back to back; all
// kernels add in this order and give the same bits.
__host__ __device__ constexpr int dir_at(int k) { return (k & 1) ? 4 + (k >> 1) : (k >> 1); }

// FP32 form of compute_dir on packed lanes within one site: lane 0 carries
// spin 0 (upper) / spin 2 (lower), lane 1 spin 1 / spin 3, so one packed
// instruction does the work of the two half-spinor vectors. Every lane runs
// exactly the scalar sequence of project / su3_mul / accumulate (a sign
// +-1 enters through an FMA, which rounds as the scalar add or subtract),
// so the results are the same bits as with R = float.
__device__ __forceinline__ f2 lanes(float a, float b) { return f2(a, b); }

template <int MU, bool FWD, bool COMPAT, bool SC>
__device__ __forceinline__ void compute_dir_pk(cx<float> acc[12], const cx<float> s[12], const cx<float> U[9],
                                               float sg_in, float n) {
    const float sg = FWD ? sg_in : -sg_in;
    // projection: H[c] = (h0[c], h1[c])
    cx<f2> H[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const cx<float> s0 = s[c], s1 = s[3 + c], s2 = s[6 + c], s3 = s[9 + c];
        const f2 lo_re = lanes(s0.re, s1.re), lo_im = lanes(s0.im, s1.im);
        if (MU == 0) {
            H[c] = {fma(f2(sg), lanes(s2.re, s3.re), lo_re), fma(f2(sg), lanes(s2.im, s3.im), lo_im)};
        } else if (MU == 1) {
            H[c] = {fma(f2(-sg), lanes(s3.im, s2.im), lo_re), fma(f2(sg), lanes(s3.re, s2.re), lo_im)};
        } else if (MU == 2) {
            H[c] = {fma(lanes(sg, -sg), lanes(s3.re, s2.re), lo_re), fma(lanes(sg, -sg), lanes(s3.im, s2.im), lo_im)};
        } else {
            H[c] = {fma(lanes(-sg, sg), lanes(s2.im, s3.im), lo_re), fma(lanes(sg, -sg), lanes(s2.re, s3.re), lo_im)};
        }
    }
    // SU(3) product of both vectors: C[a] = (c0[a], c1[a])
    cx<f2> C[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const cx<float> u0 = FWD ? U[3 * a] : U[a];
        const float ui0 = FWD ? u0.im : -u0.im;  // U^dag: conjugate
        f2 re = f2(u0.re) * H[0].re;
        f2 im = f2(u0.re) * H[0].im;
        re = fma(f2(-ui0), H[0].im, re);
        im = fma(f2(ui0), H[0].re, im);
#pragma unroll
        for (int b = 1; b < 3; b++) {
            const cx<float> ub = FWD ? U[3 * a + b] : U[3 * b + a];
            const float uib = FWD ? ub.im : -ub.im;
            re = fma(f2(ub.re), H[b].re, re);
            re = fma(f2(-uib), H[b].im, re);
            im = fma(f2(ub.re), H[b].im, im);
            im = fma(f2(uib), H[b].re, im);
        }
        C[a] = {re, im};
    }
    // rebuild: upper spins (0, 1) += chi; lower spins (2, 3) by the sign / i
    // pattern of the direction (LS = +1 forward, -1 backward)
    constexpr float LS = FWD ? 1.f : -1.f;
    constexpr bool LOWER = !(COMPAT && FWD);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        f2 u_re = lanes(acc[c].re, acc[3 + c].re), u_im = lanes(acc[c].im, acc[3 + c].im);
        f2 l_re = lanes(acc[6 + c].re, acc[9 + c].re), l_im = lanes(acc[6 + c].im, acc[9 + c].im);
        const f2 cre = C[c].re, cim = C[c].im;
        const f2 sre = lanes(cre.v.y, cre.v.x), sim = lanes(cim.v.y, cim.v.x);  // lanes swapped
        if (SC) {
            const float p = LS * n, q = -LS * n;
            u_re = fma(f2(n), cre, u_re);
            u_im = fma(f2(n), cim, u_im);
            if (LOWER) {
                if (MU == 0) {
                    l_re = fma(f2(p), cre, l_re);
                    l_im = fma(f2(p), cim, l_im);
                } else if (MU == 1) {
                    l_re = fma(f2(p), sim, l_re);
                    l_im = fma(f2(q), sre, l_im);
                } else if (MU == 2) {
                    l_re = fma(lanes(q, p), sre, l_re);
                    l_im = fma(lanes(q, p), sim, l_im);
                } else {
                    l_re = fma(lanes(p, q), cim, l_re);
                    l_im = fma(lanes(q, p), cre, l_im);
                }
            }
        } else {
            u_re = u_re + cre;
            u_im = u_im + cim;
            if (LOWER) {
                if (MU == 0) {
                    l_re = fma(f2(LS), cre, l_re);
                    l_im = fma(f2(LS), cim, l_im);
                } else if (MU == 1) {
                    l_re = fma(f2(LS), sim, l_re);
                    l_im = fma(f2(-LS), sre, l_im);
                } else if (MU == 2) {
                    l_re = fma(lanes(-LS, LS), sre, l_re);
                    l_im = fma(lanes(-LS, LS), sim, l_im);
                } else {
                    l_re = fma(lanes(LS, -LS), cim, l_re);
                    l_im = fma(lanes(-LS, LS), cre, l_im);
                }
            }
        }
        acc[c] = {u_re.v.x, u_im.v.x};
        acc[3 + c] = {u_re.v.y, u_im.v.y};
        acc[6 + c] = {l_re.v.x, l_im.v.x};
        acc[9 + c] = {l_re.v.y, l_im.v.y};
    }
}

// PK: FP32 on packed lanes within the site (compute_dir_pk). It pays in
// the single-RHS cp.async pipeline kernel (32^3x64: F16 xpay hop -12%, BF16
// -9%, F32 -1..-4% as tuned) and loses in the direct-load, multi-RHS and TMA
// kernels, which keep the scalar form; both give the same bits.
template <bool COMPAT, bool SC, typename R, bool PK = false>
__device__ __forceinline__ void compute_dir_n(int d, cx<R> acc[12], const cx<R> s[12], const cx<R> U[9], R sg,
                                              R n) {
    // d is a compile-time constant after unrolling, so this switch folds
    if constexpr (PK && std::is_same<R, float>::value) {
        switch (d) {
            case 0: compute_dir_pk<0, true, COMPAT, SC>(acc, s, U, sg, n); break;
            case 1: compute_dir_pk<1, true, COMPAT, SC>(acc, s, U, sg, n); break;
            case 2: compute_dir_pk<2, true, COMPAT, SC>(acc, s, U, sg, n); break;
            case 3: compute_dir_pk<3, true, COMPAT, SC>(acc, s, U, sg, n); break;
            case 4: compute_dir_pk<0, false, COMPAT, SC>(acc, s, U, sg, n); break;
            case 5: compute_dir_pk<1, false, COMPAT, SC>(acc, s, U, sg, n); break;
            case 6: compute_dir_pk<2, false, COMPAT, SC>(acc, s, U, sg, n); break;
            default: compute_dir_pk<3, false, COMPAT, SC>(acc, s, U, sg, n); break;
        }
        return;
    }
    switch (d) {
        case 0: compute_dir<0, true, COMPAT, SC>(acc, s, U, sg, n); break;
        case 1: compute_dir<1, true, COMPAT, SC>(acc, s, U, sg, n); break;
        case 2: compute_dir<2, true, COMPAT, SC>(acc, s, U, sg, n); break;
        case 3: compute_dir<3, true, COMPAT, SC>(acc, s, U, sg, n); break;
        case 4: compute_dir<0, false, COMPAT, SC>(acc, s, U, sg, n); break;
        case 5: compute_dir<1, false, COMPAT, SC>(acc, s, U, sg, n); break;
        case 6: compute_dir<2, false, COMPAT, SC>(acc, s, U, sg, n); break;
        default: compute_dir<3, false, COMPAT, SC>(acc, s, U, sg, n); break;
    }
}

}  // namespace dev
}  // namespace plqcd
