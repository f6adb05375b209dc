// dslash.cu -- the Wilson hopping matrix on device fields (sm_100a).
//
// Gather form of the reference's four-pass hopping pair
// (lib/dirac.c:35-408 eo, 414-791 oe): one thread per output site reads its
// eight neighbours and the eight links directly, so the phip/phim buffers
// of the reference (include/plqcd_global_params.h:170-173) and their write /
// read-back traffic disappear. Per direction:
//   forward, neighbour x+mu:  chi  = U_mu(x)        h,  h  = upper((1 - g_mu) psi(x+mu))
//   backward, neighbour x-mu: chi' = U_mu(x-mu)^dag h', h' = upper((1 + g_mu) psi(x-mu))
// and the lower two spins are rebuilt from chi by the sign / i pattern of
// lib/dirac.c:269-311 (forward) and 371-398 (backward). The periodic wrap
// replaces the reference's MPI face exchange (lib/dirac.c:124-131, 203-228)
// for a lattice held by one GPU.
//
// Memory traffic is the bound (HBM roofline). Compulsory bytes per output
// site for one parity: input spinor once (neighbour re-reads hit L2), the 8
// links, the output spinor: 192 + 8*144 + 192 = 1536 B in FP64/18-real. The
// full-lattice kernel (FULL=true) produces both parities in one launch so
// each link, used by the forward term of x and the backward term of x+mu,
// is read from HBM once: 192 + 4*144 + 192 = 960 B per site.
#include <cuda_runtime.h>

#include <cstdlib>

#include "device_fields.cuh"
#include "internal.h"

namespace plqcd {
namespace dev {

struct DslashArgs {
    const void *gauge;
    const void *in[2];  // input field of parity p (FULL) / in[0] = input (single parity)
    void *out[2];       // output field of parity p (FULL) / out[0] = output
    const void *x;      // xpay operand (single parity only)
    long Vh;
    int L0, L0h, L1, L2, L3;
    int out_parity;
    double a_up, a_low, b;
    double g5_in;       // +1 or -1: sign applied to input spins 2,3
};

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

// rebuild of the lower spins from chi = (c0, c1); LS = +1 forward, -1 backward
template <int MU, int LS, bool LOWER, typename R>
__device__ __forceinline__ void accumulate(cx<R> acc[12], const cx<R> c0[3], const cx<R> c1[3]) {
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

// One direction (MU, FWD) of one output site.
template <class SIO, class LIO, int MU, bool FWD, bool COMPAT>
__device__ __forceinline__ void hop_dir(cx<typename SIO::real> acc[12], const void *in, const void *gauge,
                                        long Vh, long h_nbr, int link_par, long h_link,
                                        typename SIO::real sg_in) {
    using R = typename SIO::real;
    cx<R> s[12];
    SIO::load(in, Vh, h_nbr, s);
    cx<R> h0[3], h1[3];
    project<MU, R>(s, FWD ? sg_in : -sg_in, h0, h1);
    cx<R> U[9];
    LIO::load(gauge, Vh, link_par, MU, h_link, U);
    cx<R> c0[3], c1[3];
    if (FWD) {
        su3_mul(U, h0, c0);
        su3_mul(U, h1, c1);
    } else {
        su3_dag_mul(U, h0, c0);
        su3_dag_mul(U, h1, c1);
    }
    // The reference as shipped drops every forward contribution to spins
    // 2,3 (its backward mu=0 step overwrites them, include/su3.h:135-138).
    accumulate<MU, FWD ? 1 : -1, !(COMPAT && FWD), R>(acc, c0, c1);
}

template <class SIO, class LIO, bool COMPAT, bool XPAY, bool FULL>
__global__ void __launch_bounds__(256) k_dslash(const DslashArgs a) {
    using R = typename SIO::real;
    int par;
    long h;
    if (FULL) {
        par = blockIdx.x & 1;
        h = (long)(blockIdx.x >> 1) * blockDim.x + threadIdx.x;
    } else {
        par = a.out_parity;
        h = (long)blockIdx.x * blockDim.x + threadIdx.x;
    }
    if (h >= a.Vh) return;
    // selects, not a dynamic index into the parameter arrays (which would
    // copy them to local memory)
    const void *in = (FULL && par == 0) ? a.in[1] : a.in[0];
    void *out = (FULL && par == 1) ? a.out[1] : a.out[0];
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(h, par, L0h, L1, L2);
    const int xh = (int)(h - c.row * L0h);
    const long L01 = L1, L012 = (long)L1 * L2;

    // neighbour half-site indices (periodic wrap on the device)
    const int xp = (c.x + 1 == a.L0) ? 0 : c.x + 1;
    const int xm = (c.x == 0) ? a.L0 - 1 : c.x - 1;
    const long h_xp = (xp >> 1) + L0h * c.row;
    const long h_xm = (xm >> 1) + L0h * c.row;
    const long h_yp = xh + L0h * (c.row + ((c.y + 1 == L1) ? -(long)(L1 - 1) : 1L));
    const long h_ym = xh + L0h * (c.row + ((c.y == 0) ? (long)(L1 - 1) : -1L));
    const long h_zp = xh + L0h * (c.row + ((c.z + 1 == L2) ? -(long)(L2 - 1) * L01 : L01));
    const long h_zm = xh + L0h * (c.row + ((c.z == 0) ? (long)(L2 - 1) * L01 : -L01));
    const long h_tp = xh + L0h * (c.row + ((c.t + 1 == L3) ? -(long)(L3 - 1) * L012 : L012));
    const long h_tm = xh + L0h * (c.row + ((c.t == 0) ? (long)(L3 - 1) * L012 : -L012));

    const R sg = (R)a.g5_in;
    const int opp = par ^ 1;
    // as shipped, oe takes forward links of odd site h from the even site
    // with the same half index (lib/dirac.c:643)
    const int fpar = (COMPAT && par == 1) ? 0 : par;

    cx<R> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = {R(0), R(0)};

    hop_dir<SIO, LIO, 0, true, COMPAT>(acc, in, a.gauge, Vh, h_xp, fpar, h, sg);
    hop_dir<SIO, LIO, 1, true, COMPAT>(acc, in, a.gauge, Vh, h_yp, fpar, h, sg);
    hop_dir<SIO, LIO, 2, true, COMPAT>(acc, in, a.gauge, Vh, h_zp, fpar, h, sg);
    hop_dir<SIO, LIO, 3, true, COMPAT>(acc, in, a.gauge, Vh, h_tp, fpar, h, sg);
    hop_dir<SIO, LIO, 0, false, COMPAT>(acc, in, a.gauge, Vh, h_xm, opp, h_xm, sg);
    hop_dir<SIO, LIO, 1, false, COMPAT>(acc, in, a.gauge, Vh, h_ym, opp, h_ym, sg);
    hop_dir<SIO, LIO, 2, false, COMPAT>(acc, in, a.gauge, Vh, h_zm, opp, h_zm, sg);
    hop_dir<SIO, LIO, 3, false, COMPAT>(acc, in, a.gauge, Vh, h_tm, opp, h_tm, sg);

    const R aup = (R)a.a_up, alow = (R)a.a_low;
    if (XPAY) {
        cx<R> xv[12];
        SIO::load(a.x, Vh, h, xv);
        const R b = (R)a.b;
#pragma unroll
        for (int k = 0; k < 12; k++) {
            const R ak = k < 6 ? aup : alow;
            acc[k] = {fma(ak, acc[k].re, b * xv[k].re), fma(ak, acc[k].im, b * xv[k].im)};
        }
    } else {
#pragma unroll
        for (int k = 6; k < 12; k++) acc[k] = {alow * acc[k].re, alow * acc[k].im};
#pragma unroll
        for (int k = 0; k < 6; k++) acc[k] = {aup * acc[k].re, aup * acc[k].im};
    }
    SIO::store(out, Vh, h, acc);
}

template <class SIO, class LIO, bool COMPAT, bool XPAY, bool FULL>
static int launch_t(const Geom &g, cudaStream_t s, const DslashArgs &a, int block) {
    long nblk = (g.Vh + block - 1) / block;
    if (FULL) nblk *= 2;
    k_dslash<SIO, LIO, COMPAT, XPAY, FULL><<<(unsigned)nblk, block, 0, s>>>(a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

template <int PREC, int RECON>
static int launch_pr(const Geom &g, cudaStream_t s, const DslashArgs &a, int block, bool compat, bool xpay,
                     bool full) {
    using S = SpinorIO<PREC>;
    using L = LinkIO<PREC, RECON>;
    if (full) return launch_t<S, L, false, false, true>(g, s, a, block);
    if (compat) {
        if (PREC == PLQCD_F64 && RECON == 18) return launch_t<S, L, true, false, false>(g, s, a, block);
        return set_error(PLQCD_ERR_ARG, "dslash: the bug-compatible mode exists for F64 18-real links only");
    }
    if (xpay) return launch_t<S, L, false, true, false>(g, s, a, block);
    return launch_t<S, L, false, false, false>(g, s, a, block);
}

}  // namespace dev

static int default_block() {
    static int b = -1;
    if (b < 0) {
        const char *e = getenv("PLQCD_DSLASH_BLOCK");
        b = e ? atoi(e) : 128;
    }
    return b;
}

int launch_dslash(const Geom &g, cudaStream_t s, const DslashCall &c) {
    dev::DslashArgs a{};
    a.gauge = c.gauge;
    if (c.full) {
        a.in[0] = c.in;
        a.in[1] = c.in2;
        a.out[0] = c.out;
        a.out[1] = c.out2;
    } else {
        a.in[0] = c.in;
        a.out[0] = c.out;
    }
    a.x = c.x;
    a.Vh = g.Vh;
    a.L0 = g.L[0];
    a.L0h = g.L0h;
    a.L1 = g.L[1];
    a.L2 = g.L[2];
    a.L3 = g.L[3];
    a.out_parity = c.out_parity;
    a.a_up = c.a_up;
    a.a_low = (c.flags & PLQCD_DSLASH_G5_OUT) ? -c.a_low : c.a_low;
    a.b = c.b;
    a.g5_in = (c.flags & PLQCD_DSLASH_G5_IN) ? -1.0 : 1.0;
    const bool compat = (c.flags & PLQCD_DSLASH_COMPAT) != 0;
    const bool xpay = c.x != nullptr;
    if (c.full && (compat || xpay || (c.flags & (PLQCD_DSLASH_G5_IN | PLQCD_DSLASH_G5_OUT))))
        return set_error(PLQCD_ERR_ARG, "dslash_full: flags and xpay are not supported in full-lattice mode");
    int block = c.block > 0 ? c.block : default_block();
    if (block % 32 || block > 256) return set_error(PLQCD_ERR_ARG, "dslash: block size %d invalid", block);
    switch (c.prec * 100 + c.recon) {
        case PLQCD_F64 * 100 + 18: return dev::launch_pr<PLQCD_F64, 18>(g, s, a, block, compat, xpay, c.full);
        case PLQCD_F64 * 100 + 12: return dev::launch_pr<PLQCD_F64, 12>(g, s, a, block, compat, xpay, c.full);
        case PLQCD_F32 * 100 + 18: return dev::launch_pr<PLQCD_F32, 18>(g, s, a, block, compat, xpay, c.full);
        case PLQCD_F32 * 100 + 12: return dev::launch_pr<PLQCD_F32, 12>(g, s, a, block, compat, xpay, c.full);
        case PLQCD_F16 * 100 + 12: return dev::launch_pr<PLQCD_F16, 12>(g, s, a, block, compat, xpay, c.full);
        case PLQCD_BF16 * 100 + 12: return dev::launch_pr<PLQCD_BF16, 12>(g, s, a, block, compat, xpay, c.full);
        default:
            return set_error(PLQCD_ERR_ARG, "dslash: unsupported precision/reconstruction %d/%d", c.prec, c.recon);
    }
}

}  // namespace plqcd
