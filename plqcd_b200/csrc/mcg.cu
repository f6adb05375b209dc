// mcg.cu -- batched multi-RHS even/odd CG: many right-hand sides on several
// lattices of different sizes, mixed precision with FP64 reliable updates,
// run either as an eager loop or as one CUDA-graph launch.
//
// Each lattice in the batch carries a block of nrhs sources. Every RHS runs
// its own CG recursion (own alpha, beta, residuals) on Mhat^dag Mhat,
// Mhat = 1 - kappa^2 H_eo H_oe (the operator of cg.cu), but the hopping
// kernels process the whole block (dslash_mrhs.cu), sharing link traffic.
// Per iteration the vector work is |t|^2, r -= alpha Ap with |r|^2, and
// p = r + beta p with the solution update x_s += alpha p; when the sloppy
// hops are RHS-pair kernels, the first two ride in the hops' epilogues.
// All scalars live in device memory and are finalised by the reductions;
// three small control kernels decide, on the device, whether the iteration
// needs a reliable update (any active RHS whose sloppy residual dropped by
// delta, or that looks converged), which RHS have converged (FP64 Schur
// residual <= tol), and whether the loop goes on.
//
// Graph mode: the loop is a WHILE conditional node whose body holds one
// iteration for every lattice of the batch and an IF conditional node with
// the FP64 reliable update; the control kernels set both conditions with
// cudaGraphSetConditional, so the whole solve is one graph launch with no
// host round trip. Eager mode runs the same kernels and reads the control
// block after each step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "blas.cuh"
#include "device_fields.cuh"
#include "internal.h"

namespace plqcd {

struct McgState {  // device arrays of length nrhs, plus reduction scratch
    double *rr, *rr_old, *pAp, *alpha, *beta, *sr2, *bp2, *maxrr, *target, *aux;
    int *active, *conv_iter;
    int *fresh;  // 1: the sloppy solution x_s was folded into x and counts as zero
    double *partials;  // nrhs * nb
    unsigned *counters;
    int nrhs, nb;
};

struct McgControl {
    int iter, need_reliable, any_active, max_iter;
    int reliable_count, last_reliable;  // iteration of the last reliable update
    double tol2, delta2;
};

enum MOp : int { M_AUX, M_BP2, M_ALPHA, M_RR, M_SR2, M_RR_TRUE, M_RR_INIT };

namespace dev {

__device__ __forceinline__ void mapply(MOp op, int f, double s, const McgState &st, double tol2) {
    switch (op) {
        case M_AUX: st.aux[f] = s; break;
        case M_BP2: st.bp2[f] = s; break;
        case M_ALPHA:
            st.pAp[f] = s;
            st.alpha[f] = s > 0 ? st.rr[f] / s : 0.0;
            break;
        case M_RR:
            st.rr_old[f] = st.rr[f];
            st.rr[f] = s;
            st.beta[f] = st.rr_old[f] > 0 ? s / st.rr_old[f] : 0.0;
            break;
        case M_SR2: st.sr2[f] = s; break;
        case M_RR_TRUE:
            st.rr[f] = s;
            st.beta[f] = st.rr_old[f] > 0 ? s / st.rr_old[f] : 0.0;
            break;
        case M_RR_INIT:
            st.rr[f] = s;
            st.rr_old[f] = s;
            st.maxrr[f] = s;
            st.target[f] = tol2 * s;
            break;
    }
}

// block reduction of v for RHS f = blockIdx.y; last block applies op
__device__ void mreduce(double v, const McgState &st, MOp op, double tol2) {
    __shared__ double ws[kBlasBlock / 32];
    __shared__ bool last;
    const int f = blockIdx.y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) b += ws[k];
        st.partials[(size_t)f * gridDim.x + blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(&st.counters[f], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x)
        t += ((volatile double *)st.partials)[(size_t)f * gridDim.x + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    __syncthreads();
    if (lane == 0) ws[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += ws[k];
        mapply(op, f, tot, st, tol2);
        st.counters[f] = 0;
    }
}

template <typename R>
__device__ __forceinline__ double n2(const cx<R> v[12]) {
    double s = 0;
#pragma unroll
    for (int k = 0; k < 12; k++) s += (double)v[k].re * v[k].re + (double)v[k].im * v[k].im;
    return s;
}

// |x_f|^2 -> op ; `only_active` skips converged RHS (whole grid row)
template <int P>
__global__ void __launch_bounds__(kBlasBlock) k_mnorm2(const char *x, size_t fb, long Vh, McgState st, MOp op,
                                                       bool only_active, double tol2) {
    const int f = blockIdx.y;
    if (only_active && !st.active[f]) return;
    using R = typename SpinorIO<P>::real;
    const void *xf = x + (size_t)f * fb;
    double v = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<R> s[12];
        SpinorIO<P>::load(xf, Vh, h, s);
        v += n2(s);
    }
    mreduce(v, st, op, tol2);
}

// out = a - b (F64) ; |out|^2 -> op
__global__ void __launch_bounds__(kBlasBlock) k_msub_norm2(char *out, const char *a, const char *b, size_t fb,
                                                           long Vh, McgState st, MOp op) {
    const int f = blockIdx.y;
    const size_t o = (size_t)f * fb;
    double v = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<double> av[12], bv[12];
        SpinorIO<PLQCD_F64>::load(a + o, Vh, h, av);
        SpinorIO<PLQCD_F64>::load(b + o, Vh, h, bv);
#pragma unroll
        for (int k = 0; k < 12; k++) av[k] = csub(av[k], bv[k]);
        SpinorIO<PLQCD_F64>::store(out + o, Vh, h, av);
        v += n2(av);
    }
    mreduce(v, st, op, 0.0);
}

// z = a - b (F64) ; |z|^2 -> op ; out = z in the sloppy format SP (the
// FP64 z itself is not stored: the mixed solver only restarts from it)
template <int SP>
__global__ void __launch_bounds__(kBlasBlock) k_msub_norm2_to(char *out, size_t fbo, const char *a, const char *b,
                                                              size_t fb, long Vh, McgState st, MOp op) {
    using RS = typename SpinorIO<SP>::real;
    const int f = blockIdx.y;
    const size_t o = (size_t)f * fb;
    double v = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<double> av[12], bv[12];
        SpinorIO<PLQCD_F64>::load(a + o, Vh, h, av);
        SpinorIO<PLQCD_F64>::load(b + o, Vh, h, bv);
        cx<RS> d[12];
#pragma unroll
        for (int k = 0; k < 12; k++) {
            av[k] = csub(av[k], bv[k]);
            d[k] = {(RS)av[k].re, (RS)av[k].im};
        }
        SpinorIO<SP>::store(out + (size_t)f * fbo, Vh, h, d);
        v += n2(av);
    }
    mreduce(v, st, op, 0.0);
}

// r_s -= alpha_f Ap ; |r_s|^2 -> M_RR (active RHS only). The solution
// update x_s += alpha_f p of the same iteration happens in k_mcg_p, which
// reads p anyway (or, in an iteration with a reliable update, in k_maccum).
template <int P>
__global__ void __launch_bounds__(kBlasBlock) k_mcg_update(char *rs, const char *Ap, size_t fb, long Vh, McgState st) {
    const int f = blockIdx.y;
    if (!st.active[f]) return;
    using R = typename SpinorIO<P>::real;
    const R a = (R)st.alpha[f];
    const size_t o = (size_t)f * fb;
    double v = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<R> av[12], rv[12];
        SpinorIO<P>::load(Ap + o, Vh, h, av);
        SpinorIO<P>::load(rs + o, Vh, h, rv);
#pragma unroll
        for (int k = 0; k < 12; k++) rv[k] = {fma(-a, av[k].re, rv[k].re), fma(-a, av[k].im, rv[k].im)};
        SpinorIO<P>::store(rs + o, Vh, h, rv);
        v += n2(rv);
    }
    mreduce(v, st, M_RR, 0.0);
}

// x_s += alpha_f p (x_s = alpha_f p when fresh), unless this iteration's
// reliable update already folded alpha_f p into x; then p = r + beta_f p
// (active RHS only)
template <int P, int XP>
__global__ void __launch_bounds__(kBlasBlock) k_mcg_p(char *p, const char *rs, char *xs, size_t fb, size_t fbx,
                                                      long Vh, McgState st, const McgControl *ctl) {
    const int f = blockIdx.y;
    if (!st.active[f]) return;
    using R = typename SpinorIO<P>::real;
    using RX = typename SpinorIO<XP>::real;
    const R beta = (R)st.beta[f];
    const RX ax = (RX)st.alpha[f];
    const bool xup = !ctl->need_reliable, fresh = st.fresh[f] != 0;
    const size_t o = (size_t)f * fb, ox = (size_t)f * fbx;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<R> pv[12], rv[12];
        SpinorIO<P>::load(p + o, Vh, h, pv);
        SpinorIO<P>::load(rs + o, Vh, h, rv);
        if (xup) {
            cx<RX> xv[12];
            if (fresh) {
#pragma unroll
                for (int k = 0; k < 12; k++) xv[k] = {RX(0), RX(0)};
            } else {
                SpinorIO<XP>::load(xs + ox, Vh, h, xv);
            }
#pragma unroll
            for (int k = 0; k < 12; k++)
                xv[k] = {fma(ax, (RX)pv[k].re, xv[k].re), fma(ax, (RX)pv[k].im, xv[k].im)};
            SpinorIO<XP>::store(xs + ox, Vh, h, xv);
        }
#pragma unroll
        for (int k = 0; k < 12; k++) pv[k] = {fma(beta, pv[k].re, rv[k].re), fma(beta, pv[k].im, rv[k].im)};
        SpinorIO<P>::store(p + o, Vh, h, pv);
    }
}

// x64 += x_s for every active RHS (WITH_P: x64 += x_s + alpha_f p, the
// update of the current iteration, computed as k_mcg_p would); a fresh x_s
// counts as zero. x_s is not cleared: k_ctl_reliable marks it fresh.
template <int P, int XP, bool WITH_P>
__global__ void __launch_bounds__(kBlasBlock) k_maccum(char *x64, size_t fb64, const char *xs, size_t fbx,
                                                       const char *p, size_t fb, long Vh, McgState st) {
    const int f = blockIdx.y;
    const bool fresh = st.fresh[f] != 0;
    if (!st.active[f] || (fresh && !WITH_P)) return;
    using R = typename SpinorIO<P>::real;
    using RX = typename SpinorIO<XP>::real;
    const RX ax = (RX)st.alpha[f];
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<double> xv[12];
        cx<RX> sv[12];
        SpinorIO<PLQCD_F64>::load(x64 + (size_t)f * fb64, Vh, h, xv);
        if (fresh) {
#pragma unroll
            for (int k = 0; k < 12; k++) sv[k] = {RX(0), RX(0)};
        } else {
            SpinorIO<XP>::load(xs + (size_t)f * fbx, Vh, h, sv);
        }
        if (WITH_P) {
            cx<R> pv[12];
            SpinorIO<P>::load(p + (size_t)f * fb, Vh, h, pv);
#pragma unroll
            for (int k = 0; k < 12; k++)
                sv[k] = {fma(ax, (RX)pv[k].re, sv[k].re), fma(ax, (RX)pv[k].im, sv[k].im)};
        }
#pragma unroll
        for (int k = 0; k < 12; k++) xv[k] = {xv[k].re + (double)sv[k].re, xv[k].im + (double)sv[k].im};
        SpinorIO<PLQCD_F64>::store(x64 + (size_t)f * fb64, Vh, h, xv);
    }
}

// block precision conversion
template <int DP, int SP>
__global__ void __launch_bounds__(kBlasBlock) k_mconvert(char *dst, size_t fbd, const char *src, size_t fbs, long Vh) {
    const int f = blockIdx.y;
    using RS = typename SpinorIO<SP>::real;
    using RD = typename SpinorIO<DP>::real;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<RS> s[12];
        SpinorIO<SP>::load(src + (size_t)f * fbs, Vh, h, s);
        cx<RD> d[12];
#pragma unroll
        for (int k = 0; k < 12; k++) d[k] = {(RD)s[k].re, (RD)s[k].im};
        SpinorIO<DP>::store(dst + (size_t)f * fbd, Vh, h, d);
    }
}

__global__ void k_mfill_int(int *a, int n, int v) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = v;
}

// ---- control kernels (one block) --------------------------------------------
// after the sloppy update: does any active RHS need a reliable update?
__global__ void k_ctl_iter(McgControl *c, const McgState *st, int nst, int mixed, int use_handle,
                           cudaGraphConditionalHandle h_if) {
    __shared__ int need;
    if (threadIdx.x == 0) {
        need = 0;
        c->iter++;
    }
    __syncthreads();
    for (int s = 0; s < nst; s++)
        for (int f = threadIdx.x; f < st[s].nrhs; f += blockDim.x) {
            if (!st[s].active[f]) continue;
            const double rr = st[s].rr[f];
            // (an update is also forced after 100 iterations without one, in
            // case a 16-bit recursion stops reducing its residual)
            if ((mixed && rr < c->delta2 * st[s].maxrr[f]) || rr <= st[s].target[f] || !isfinite(rr) ||
                c->iter - c->last_reliable >= 100)
                atomicOr(&need, 1);
        }
    __syncthreads();
    for (int s = 0; s < nst; s++)
        for (int f = threadIdx.x; f < st[s].nrhs; f += blockDim.x)
            if (!need && st[s].active[f]) st[s].maxrr[f] = fmax(st[s].maxrr[f], st[s].rr[f]);
    if (threadIdx.x == 0) {
        c->need_reliable = need;
        if (use_handle) cudaGraphSetConditional(h_if, need ? 1u : 0u);
    }
}

// within a reliable update, once item s's FP64 Schur residuals are in:
// retire its converged RHS (before its restart, which then skips them)
__global__ void k_ctl_converged(McgControl *c, const McgState *st, int s) {
    for (int f = threadIdx.x; f < st[s].nrhs; f += blockDim.x)
        if (st[s].active[f] && st[s].sr2[f] <= c->tol2 * st[s].bp2[f]) {
            st[s].active[f] = 0;
            st[s].conv_iter[f] = c->iter;
        }
}

// after a reliable update: every x_s was folded into x (fresh); tighten
// the convergence triggers of the RHS still active
__global__ void k_ctl_reliable(McgControl *c, const McgState *st, int nst) {
    for (int s = 0; s < nst; s++)
        for (int f = threadIdx.x; f < st[s].nrhs; f += blockDim.x) {
            st[s].fresh[f] = 1;
            if (!st[s].active[f]) continue;
            st[s].maxrr[f] = st[s].rr[f];
            if (st[s].rr[f] <= st[s].target[f]) st[s].target[f] *= 0.25;
        }
    if (threadIdx.x == 0) {
        c->reliable_count++;
        c->last_reliable = c->iter;
    }
}

// end of an iteration: an x_s that k_mcg_p wrote is no longer fresh;
// continue while any RHS is active and iterations remain
__global__ void k_ctl_loop(McgControl *c, const McgState *st, int nst, int use_handle,
                           cudaGraphConditionalHandle h_while) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int s = 0; s < nst; s++)
        for (int f = threadIdx.x; f < st[s].nrhs; f += blockDim.x)
            if (st[s].active[f]) {
                atomicOr(&any, 1);
                if (!c->need_reliable) st[s].fresh[f] = 0;
            }
    __syncthreads();
    if (threadIdx.x == 0) {
        c->any_active = any;
        const int go = any && c->iter < c->max_iter;
        if (use_handle) cudaGraphSetConditional(h_while, go ? 1u : 0u);
    }
}

}  // namespace dev

namespace {

// blocks per RHS of the batched BLAS kernels: about kMaxRedBlocks (8 per
// SM) in all, at least one per SM per RHS
inline int red_blocks(long Vh, int nrhs) {
    const long b = (Vh + kBlasBlock - 1) / kBlasBlock;
    const long per = std::max<long>(148, kMaxRedBlocks / std::max(nrhs, 1));
    return (int)std::min<long>(b, per);
}

#define MCG_PREC_SWITCH(prec, F)                                                     \
    switch (prec) {                                                                  \
        case PLQCD_F64: F(PLQCD_F64); break;                                         \
        case PLQCD_F32: F(PLQCD_F32); break;                                         \
        case PLQCD_F16: F(PLQCD_F16); break;                                         \
        case PLQCD_BF16: F(PLQCD_BF16); break;                                       \
        default: return set_error(PLQCD_ERR_ARG, "batch cg: unknown precision %d", prec); \
    }

// one lattice of the batch with its workspace
struct Item {
    plqcd_solve_item in;
    const Geom *g = nullptr;
    int ps = PLQCD_F64, xprec = PLQCD_F64;
    size_t fb64 = 0, fbs = 0, fbx = 0;
    char *bprime = nullptr, *r64 = nullptr, *t64 = nullptr, *tmp64 = nullptr;
    char *rs = nullptr, *p = nullptr, *Ap = nullptr, *t = nullptr, *tmps = nullptr, *xs = nullptr;
    McgState st{};
    void *mem = nullptr;
    // the sloppy hops that produce t and Ap carry |t|^2 and r -= alpha Ap,
    // |r|^2 in their epilogues (RHS-pair kernels; see RhsSink)
    bool fused = false;
    double *hop_partials = nullptr;  // nrhs * ceil(Vh / 32)
};

struct Batch {
    std::vector<Item> items;
    double kappa = 0.12, tol = 1e-10, delta = 0.1;
    int mixed = 0;
    McgControl *ctl = nullptr;
    McgState *st_dev = nullptr;
    cudaStream_t s = nullptr;

    int hop(Item &it, const plqcd_gauge *gf, void *out, const void *in, int par, unsigned flags,
            const void *x = nullptr, double a = 1.0, double b = 0.0) {
        return launch_dslash_mrhs(*it.g, s, gf->data, gf->prec, gf->recon, out, in, it.in.nrhs, par, flags, a, x, b);
    }
    // out = Mhat in (dagger: g5 Mhat g5), block of nrhs fields
    int mhat(Item &it, const plqcd_gauge *gf, void *out, const void *in, void *tmp_o, bool dagger) {
        unsigned fi = dagger ? PLQCD_DSLASH_G5_IN : 0u, fo = dagger ? PLQCD_DSLASH_G5_OUT : 0u;
        PLQCD_TRY(hop(it, gf, tmp_o, in, PLQCD_ODD, fi));
        return hop(it, gf, out, tmp_o, PLQCD_EVEN, fo, in, -kappa * kappa, 1.0);
    }
    // rs = Mhat^dag t (the restart of a reliable update) with |rs|^2 -> rr,
    // beta in the second hop's epilogue; RHS pairs that are both retired
    // skip both hops
    int restart_fused(Item &it, const plqcd_gauge *gs) {
        RhsSink k{it.hop_partials, it.st.rr, it.st.rr_old, it.st.pAp, it.st.alpha, it.st.beta, it.st.active, it.rs};
        PLQCD_TRY(launch_dslash_mrhs_sink(*it.g, s, gs->data, gs->prec, gs->recon, it.tmps, it.t, it.in.nrhs,
                                          PLQCD_ODD, PLQCD_DSLASH_G5_IN, 1.0, nullptr, 0.0, 4, k));
        return launch_dslash_mrhs_sink(*it.g, s, gs->data, gs->prec, gs->recon, it.rs, it.tmps, it.in.nrhs,
                                       PLQCD_EVEN, PLQCD_DSLASH_G5_OUT, -kappa * kappa, it.t, 1.0, 3, k);
    }
    // mhat with the CG sums of epi (1: |out|^2 -> pAp, alpha; 2: r -= alpha
    // out, |r|^2 -> rr, beta, out not stored) in the second hop's epilogue
    int mhat_fused(Item &it, const plqcd_gauge *gf, void *out, const void *in, void *tmp_o, bool dagger, int epi) {
        unsigned fi = dagger ? PLQCD_DSLASH_G5_IN : 0u, fo = dagger ? PLQCD_DSLASH_G5_OUT : 0u;
        PLQCD_TRY(hop(it, gf, tmp_o, in, PLQCD_ODD, fi));
        RhsSink k{it.hop_partials, it.st.rr, it.st.rr_old, it.st.pAp, it.st.alpha, it.st.beta, it.st.active, it.rs};
        return launch_dslash_mrhs_sink(*it.g, s, gf->data, gf->prec, gf->recon, out, tmp_o, it.in.nrhs, PLQCD_EVEN,
                                       fo, -kappa * kappa, in, 1.0, epi, k);
    }
    int norm2(Item &it, const void *x, int prec, MOp op, bool only_active) {
        dim3 grid(it.st.nb, it.in.nrhs);
        const size_t fb = spinor_parity_bytes(it.g->Vh, prec);
#define F(P) dev::k_mnorm2<P><<<grid, kBlasBlock, 0, s>>>((const char *)x, fb, it.g->Vh, it.st, op, only_active, tol * tol)
        MCG_PREC_SWITCH(prec, F)
#undef F
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
    // out (sloppy format) = a - b, |a - b|^2 -> op
    int sub_norm2_to(Item &it, void *out, int prec, const void *a, const void *b, MOp op) {
        dim3 grid(it.st.nb, it.in.nrhs);
        const size_t fbo = spinor_parity_bytes(it.g->Vh, prec);
#define F(P) dev::k_msub_norm2_to<P><<<grid, kBlasBlock, 0, s>>>((char *)out, fbo, (const char *)a, (const char *)b, it.fb64, it.g->Vh, it.st, op)
        MCG_PREC_SWITCH(prec, F)
#undef F
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
    // x64 += x_s (with_p: + alpha p, the current iteration's update)
    int accum(Item &it, bool with_p) {
        dim3 grid(it.st.nb, it.in.nrhs);
#define G(P, XP, W) dev::k_maccum<P, XP, W><<<grid, kBlasBlock, 0, s>>>((char *)it.in.x_even, it.fb64, it.xs, it.fbx, it.p, it.fbs, it.g->Vh, it.st)
#define F(P)                                                                 \
    if (it.xprec == PLQCD_F64) {                                             \
        if (with_p) G(P, PLQCD_F64, true); else G(P, PLQCD_F64, false);      \
    } else {                                                                 \
        if (with_p) G(P, PLQCD_F32, true); else G(P, PLQCD_F32, false);      \
    }
        MCG_PREC_SWITCH(it.ps, F)
#undef F
#undef G
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
    int sub_norm2(Item &it, void *out, const void *a, const void *b, MOp op) {
        dim3 grid(it.st.nb, it.in.nrhs);
        dev::k_msub_norm2<<<grid, kBlasBlock, 0, s>>>((char *)out, (const char *)a, (const char *)b, it.fb64,
                                                      it.g->Vh, it.st, op);
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
    int convert(Item &it, void *dst, int dp, const void *src, int sp) {
        dim3 grid(it.st.nb, it.in.nrhs);
        const size_t fd = spinor_parity_bytes(it.g->Vh, dp), fs = spinor_parity_bytes(it.g->Vh, sp);
#define G(DP, SP) dev::k_mconvert<DP, SP><<<grid, kBlasBlock, 0, s>>>((char *)dst, fd, (const char *)src, fs, it.g->Vh)
#define F(SP)                                                                           \
    switch (dp) {                                                                       \
        case PLQCD_F64: G(PLQCD_F64, SP); break;                                        \
        case PLQCD_F32: G(PLQCD_F32, SP); break;                                        \
        case PLQCD_F16: G(PLQCD_F16, SP); break;                                        \
        case PLQCD_BF16: G(PLQCD_BF16, SP); break;                                      \
        default: return set_error(PLQCD_ERR_ARG, "batch cg: unknown precision %d", dp); \
    }
        MCG_PREC_SWITCH(sp, F)
#undef F
#undef G
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }

    // ---- the three parts of one iteration ------------------------------------
    int part_sloppy() {
        for (Item &it : items) {
            const plqcd_gauge *gs = it.in.g_sloppy ? it.in.g_sloppy : it.in.g64;
            if (it.fused) {
                PLQCD_TRY(mhat_fused(it, gs, it.t, it.p, it.tmps, false, 1));   // t, pAp, alpha
                PLQCD_TRY(mhat_fused(it, gs, it.Ap, it.t, it.tmps, true, 2));   // r, rr, beta
                continue;
            }
            PLQCD_TRY(mhat(it, gs, it.t, it.p, it.tmps, false));
            PLQCD_TRY(norm2(it, it.t, it.ps, M_ALPHA, true));
            PLQCD_TRY(mhat(it, gs, it.Ap, it.t, it.tmps, true));
            dim3 grid(it.st.nb, it.in.nrhs);
#define F(P) dev::k_mcg_update<P><<<grid, kBlasBlock, 0, s>>>(it.rs, it.Ap, it.fbs, it.g->Vh, it.st)
            MCG_PREC_SWITCH(it.ps, F)
#undef F
            PLQCD_CUDA_TRY(cudaGetLastError());
        }
        return PLQCD_OK;
    }
    int part_reliable() {
        for (Item &it : items) {
            PLQCD_TRY(accum(it, true));
            // FP64: solution and Schur residual b' - Mhat x (convergence)
            PLQCD_TRY(mhat(it, it.in.g64, it.t64, it.in.x_even, it.tmp64, false));
            // restart direction Mhat^dag r: the sloppy operator's accuracy
            // suffices (FP64 when the solve is FP64), so the mixed solve
            // writes r only in the sloppy format
            if (mixed) {
                const plqcd_gauge *gs = it.in.g_sloppy ? it.in.g_sloppy : it.in.g64;
                PLQCD_TRY(sub_norm2_to(it, it.t, it.ps, it.bprime, it.t64, M_SR2));
                PLQCD_TRY(ctl_converged(it));
                if (it.fused) {
                    // |r|^2 in the second hop; pairs of retired RHS skipped
                    PLQCD_TRY(restart_fused(it, gs));
                } else {
                    PLQCD_TRY(mhat(it, gs, it.rs, it.t, it.tmps, true));
                    PLQCD_TRY(norm2(it, it.rs, it.ps, M_RR_TRUE, false));
                }
            } else {
                PLQCD_TRY(sub_norm2(it, it.r64, it.bprime, it.t64, M_SR2));
                PLQCD_TRY(ctl_converged(it));
                PLQCD_TRY(mhat(it, it.in.g64, it.t64, it.r64, it.tmp64, true));
                PLQCD_TRY(norm2(it, it.t64, PLQCD_F64, M_RR_TRUE, false));
                PLQCD_TRY(convert(it, it.rs, it.ps, it.t64, PLQCD_F64));
            }
        }
        return PLQCD_OK;
    }
    int part_direction() {
        for (Item &it : items) {
            dim3 grid(it.st.nb, it.in.nrhs);
#define F(P)                                                                                                     \
    if (it.xprec == PLQCD_F64)                                                                                   \
        dev::k_mcg_p<P, PLQCD_F64><<<grid, kBlasBlock, 0, s>>>(it.p, it.rs, it.xs, it.fbs, it.fbx, it.g->Vh, it.st, ctl); \
    else                                                                                                         \
        dev::k_mcg_p<P, PLQCD_F32><<<grid, kBlasBlock, 0, s>>>(it.p, it.rs, it.xs, it.fbs, it.fbx, it.g->Vh, it.st, ctl);
            MCG_PREC_SWITCH(it.ps, F)
#undef F
            PLQCD_CUDA_TRY(cudaGetLastError());
        }
        return PLQCD_OK;
    }
    // h: condition to set from the device (graph mode), or none (eager)
    int ctl_iter(const cudaGraphConditionalHandle *h) {
        dev::k_ctl_iter<<<1, 256, 0, s>>>(ctl, st_dev, (int)items.size(), mixed, h != nullptr, h ? *h : 0);
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
    int ctl_converged(const Item &it) {
        dev::k_ctl_converged<<<1, 256, 0, s>>>(ctl, st_dev, (int)(&it - items.data()));
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
    int ctl_reliable() {
        dev::k_ctl_reliable<<<1, 256, 0, s>>>(ctl, st_dev, (int)items.size());
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
    int ctl_loop(const cudaGraphConditionalHandle *h) {
        dev::k_ctl_loop<<<1, 256, 0, s>>>(ctl, st_dev, (int)items.size(), h != nullptr, h ? *h : 0);
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
};

// workspace and state arrays of one item (outside the timed solve). The
// item takes its lattice's solver workspace, kept across solves as
// plqcd_invert_cg keeps it, unless an earlier item of the batch holds it:
// then it allocates its own (`it.mem`, freed after the solve).
int alloc_item(Batch &B, Item &it, bool own_ws) {
    const plqcd_solve_item &in = it.in;
    it.g = &in.lat->geom;
    const long Vh = it.g->Vh;
    const int n = in.nrhs;
    it.fb64 = spinor_parity_bytes(Vh, PLQCD_F64);
    it.fbs = spinor_parity_bytes(Vh, it.ps);
    it.fbx = spinor_parity_bytes(Vh, it.xprec);
    it.st.nrhs = n;
    it.st.nb = red_blocks(Vh, n);
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t nsb = (size_t)(Vh + 31) / 32;  // site blocks of a fused hop, at most
    const size_t need = 4 * al(it.fb64 * n) + 5 * al(it.fbs * n) + al(it.fbx * n) + 10 * al(sizeof(double) * n) +
                        3 * al(sizeof(int) * n) + al(sizeof(double) * n * it.st.nb) + al(sizeof(unsigned) * n) +
                        al(sizeof(double) * n * nsb);
    void *ws = nullptr;
    if (own_ws) {
        if (cudaMalloc(&it.mem, need) != cudaSuccess) {
            cudaGetLastError();
            return set_error(PLQCD_ERR_NOMEM, "batch cg: workspace of %zu bytes", need);
        }
        ws = it.mem;
    } else {
        PLQCD_TRY(lattice_workspace(in.lat, need, &ws));
    }
    char *w = static_cast<char *>(ws);
    auto take = [&](size_t x) {
        char *p = w;
        w += al(x);
        return p;
    };
    it.bprime = take(it.fb64 * n);
    it.r64 = take(it.fb64 * n);
    it.t64 = take(it.fb64 * n);
    it.tmp64 = take(it.fb64 * n);
    it.rs = take(it.fbs * n);
    it.p = take(it.fbs * n);
    it.Ap = take(it.fbs * n);
    it.t = take(it.fbs * n);
    it.tmps = take(it.fbs * n);
    it.xs = take(it.fbx * n);
    double **dd[10] = {&it.st.rr, &it.st.rr_old, &it.st.pAp, &it.st.alpha, &it.st.beta,
                       &it.st.sr2, &it.st.bp2, &it.st.maxrr, &it.st.target, &it.st.aux};
    for (double **d : dd) *d = reinterpret_cast<double *>(take(sizeof(double) * n));
    it.st.active = reinterpret_cast<int *>(take(sizeof(int) * n));
    it.st.conv_iter = reinterpret_cast<int *>(take(sizeof(int) * n));
    it.st.fresh = reinterpret_cast<int *>(take(sizeof(int) * n));
    it.st.partials = reinterpret_cast<double *>(take(sizeof(double) * n * it.st.nb));
    it.st.counters = reinterpret_cast<unsigned *>(take(sizeof(unsigned) * n));
    it.hop_partials = reinterpret_cast<double *>(take(sizeof(double) * n * nsb));
    cudaStream_t s = B.s;
    PLQCD_CUDA_TRY(cudaMemsetAsync(it.st.counters, 0, sizeof(unsigned) * n, s));
    PLQCD_CUDA_TRY(cudaMemsetAsync(it.st.conv_iter, 0xff, sizeof(int) * n, s));
    dev::k_mfill_int<<<1, 256, 0, s>>>(it.st.active, n, 1);
    dev::k_mfill_int<<<1, 256, 0, s>>>(it.st.fresh, n, 1);  // x_s = 0
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

// true the first time a (CUDA context, lattice, format, RHS count, kernel
// configuration) runs the fused hops in this process
bool first_fused_use(const Geom &g, int prec, int recon, int nrhs, int variant, int block) {
    static std::mutex mu;
    static std::set<std::string> seen;
    const unsigned long long ctx = current_context_id();
    if (!ctx) return true;  // no context ID: warm every time
    char key[160];
    snprintf(key, sizeof key, "%llu|%d|%d|%d|%dx%dx%dx%d|%d|%d", ctx, prec, recon, nrhs, g.L[0], g.L[1], g.L[2],
             g.L[3], variant, block);
    std::lock_guard<std::mutex> lk(mu);
    return seen.insert(key).second;
}

// tune the plain and xpay hops of the sloppy and the FP64 operator on this
// item's block (zeroed fields) when the tuner has no entry for them yet: a
// captured launch cannot tune and would take the first candidate
int tune_item(Batch &B, Item &it) {
    const plqcd_solve_item &in = it.in;
    const plqcd_gauge *gs = in.g_sloppy ? in.g_sloppy : in.g64;
    const int n = in.nrhs;
    const bool done = dslash_mrhs_tuned(*it.g, gs->prec, gs->recon, n, false) &&
                      dslash_mrhs_tuned(*it.g, gs->prec, gs->recon, n, true) &&
                      dslash_mrhs_tuned(*it.g, PLQCD_F64, in.g64->recon, n, false) &&
                      dslash_mrhs_tuned(*it.g, PLQCD_F64, in.g64->recon, n, true);
    if (!done) {
        cudaStream_t s = B.s;
        PLQCD_CUDA_TRY(cudaMemsetAsync(it.p, 0, it.fbs * n, s));
        PLQCD_CUDA_TRY(cudaMemsetAsync(it.r64, 0, it.fb64 * n, s));
        PLQCD_TRY(B.mhat(it, gs, it.t, it.p, it.tmps, false));
        PLQCD_TRY(B.mhat(it, in.g64, it.t64, it.r64, it.tmp64, false));
    }
    // fused CG sums when the tuned sloppy xpay hop is an RHS-pair kernel
    // (PLQCD_MCG_FUSED=0: separate passes)
    const char *e = getenv("PLQCD_MCG_FUSED");
    int variant = 0, block = 0;
    it.fused = B.mixed && !(e && e[0] == '0') &&
               dslash_mrhs_sink_ok(*it.g, gs->prec, gs->recon, n, &variant, &block);
    if (it.fused && first_fused_use(*it.g, gs->prec, gs->recon, n, variant, block)) {
        // load the fused kernels and set their shared memory before any
        // capture, once per device and configuration (on zeroed fields; the
        // solve's start overwrites every scalar they set)
        PLQCD_CUDA_TRY(cudaMemsetAsync(it.p, 0, it.fbs * n, B.s));
        PLQCD_CUDA_TRY(cudaMemsetAsync(it.rs, 0, it.fbs * n, B.s));
        PLQCD_TRY(B.mhat_fused(it, gs, it.t, it.p, it.tmps, false, 1));
        PLQCD_TRY(B.mhat_fused(it, gs, it.Ap, it.t, it.tmps, true, 2));
        PLQCD_TRY(B.restart_fused(it, gs));
    }
    return PLQCD_OK;
}

// start of the solve: b' = b_e + kappa H_eo b_o, |b'|^2, x = 0, the start
// residual r = Mhat^dag b' and |r|^2, p = r
int start_item(Batch &B, Item &it) {
    const plqcd_solve_item &in = it.in;
    const int n = in.nrhs;
    cudaStream_t s = B.s;
    PLQCD_TRY(B.hop(it, in.g64, it.bprime, in.b_odd, PLQCD_EVEN, 0, in.b_even, B.kappa, 1.0));
    PLQCD_TRY(B.norm2(it, it.bprime, PLQCD_F64, M_BP2, false));
    PLQCD_CUDA_TRY(cudaMemsetAsync(in.x_even, 0, it.fb64 * n, s));
    const plqcd_gauge *gs = in.g_sloppy ? in.g_sloppy : in.g64;
    if (B.mixed) {
        // the start residual Mhat^dag b' only seeds the sloppy recursion (the
        // FP64 Schur residual of b', which decides convergence, does not use
        // it), so the sloppy operator computes it, as in plqcd_invert_cg
        PLQCD_TRY(B.convert(it, it.t, it.ps, it.bprime, PLQCD_F64));
        PLQCD_TRY(B.mhat(it, gs, it.rs, it.t, it.tmps, true));
        PLQCD_TRY(B.norm2(it, it.rs, it.ps, M_RR_INIT, false));
        PLQCD_CUDA_TRY(cudaMemcpyAsync(it.p, it.rs, it.fbs * n, cudaMemcpyDeviceToDevice, s));
    } else {
        PLQCD_TRY(B.mhat(it, in.g64, it.r64, it.bprime, it.tmp64, true));
        PLQCD_TRY(B.norm2(it, it.r64, PLQCD_F64, M_RR_INIT, false));
        PLQCD_TRY(B.convert(it, it.rs, it.ps, it.r64, PLQCD_F64));
        PLQCD_TRY(B.convert(it, it.p, it.ps, it.r64, PLQCD_F64));
    }
    return PLQCD_OK;
}

// capture the iteration loop (WHILE node: sloppy part, IF node with the
// reliable update, direction part) and instantiate it; nothing runs
int build_graph(Batch &B, cudaGraph_t *gout, cudaGraphExec_t *geout) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    int rc = PLQCD_OK;
    cudaStream_t s = B.s;
    auto cuda = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == PLQCD_OK) rc = set_error(PLQCD_ERR_CUDA, "batch cg graph: %s: %s", what, cudaGetErrorString(e));
        return e == cudaSuccess;
    };
    do {
        if (!cuda(cudaGraphCreate(&g, 0), "create")) break;
        cudaGraphConditionalHandle hw, hif;
        if (!cuda(cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault), "while handle")) break;
        cudaGraphNodeParams wp = {};
        wp.type = cudaGraphNodeTypeConditional;
        wp.conditional.handle = hw;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        cudaGraphNode_t wnode;
        if (!cuda(cudaGraphAddNode(&wnode, g, nullptr, 0, &wp), "while node")) break;
        cudaGraph_t body = wp.conditional.phGraph_out[0];
        if (!cuda(cudaGraphConditionalHandleCreate(&hif, body, 0, cudaGraphCondAssignDefault), "if handle")) break;

        // part 1: sloppy iteration + decision, captured into the body
        if (!cuda(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
                  "capture 1"))
            break;
        int r1 = B.part_sloppy();
        if (r1 == PLQCD_OK) r1 = B.ctl_iter(&hif);
        cudaStreamCaptureStatus cst;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        std::vector<cudaGraphNode_t> leaves;
        if (cuda(cudaStreamGetCaptureInfo(s, &cst, nullptr, nullptr, &deps, &ndeps), "capture info"))
            leaves.assign(deps, deps + ndeps);
        cudaGraph_t tmpg;
        cuda(cudaStreamEndCapture(s, &tmpg), "end capture 1");
        if (r1 != PLQCD_OK) {
            rc = r1;
            break;
        }
        if (rc) break;
        // part 2: IF (reliable update) node after part 1
        cudaGraphNodeParams ip = {};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = hif;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        cudaGraphNode_t inode;
        if (!cuda(cudaGraphAddNode(&inode, body, leaves.data(), leaves.size(), &ip), "if node")) break;
        cudaGraph_t ibody = ip.conditional.phGraph_out[0];
        if (!cuda(cudaStreamBeginCaptureToGraph(s, ibody, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
                  "capture 2"))
            break;
        int r2 = B.part_reliable();
        if (r2 == PLQCD_OK) r2 = B.ctl_reliable();
        cuda(cudaStreamEndCapture(s, &tmpg), "end capture 2");
        if (r2 != PLQCD_OK) {
            rc = r2;
            break;
        }
        if (rc) break;
        // part 3: new search directions + loop condition, after the IF node
        if (!cuda(cudaStreamBeginCaptureToGraph(s, body, &inode, nullptr, 1, cudaStreamCaptureModeRelaxed),
                  "capture 3"))
            break;
        int r3 = B.part_direction();
        if (r3 == PLQCD_OK) r3 = B.ctl_loop(&hw);
        cuda(cudaStreamEndCapture(s, &tmpg), "end capture 3");
        if (r3 != PLQCD_OK) {
            rc = r3;
            break;
        }
        if (rc) break;
        if (!cuda(cudaGraphInstantiate(&ge, g, 0), "instantiate")) break;
    } while (0);
    if (rc) {
        if (ge) cudaGraphExecDestroy(ge);
        if (g) cudaGraphDestroy(g);
        ge = nullptr;
        g = nullptr;
    }
    *gout = g;
    *geout = ge;
    return rc;
}

int run_eager(Batch &B, McgControl *hctl) {
    auto read = [&]() -> int {
        PLQCD_CUDA_TRY(cudaMemcpyAsync(hctl, B.ctl, sizeof(McgControl), cudaMemcpyDeviceToHost, B.s));
        PLQCD_CUDA_TRY(cudaStreamSynchronize(B.s));
        return PLQCD_OK;
    };
    for (;;) {
        PLQCD_TRY(B.part_sloppy());
        PLQCD_TRY(B.ctl_iter(nullptr));
        PLQCD_TRY(read());
        if (hctl->need_reliable) {
            PLQCD_TRY(B.part_reliable());
            PLQCD_TRY(B.ctl_reliable());
        }
        PLQCD_TRY(B.part_direction());
        PLQCD_TRY(B.ctl_loop(nullptr));
        PLQCD_TRY(read());
        if (!hctl->any_active || hctl->iter >= hctl->max_iter) break;
    }
    return PLQCD_OK;
}

}  // namespace
}  // namespace plqcd

using namespace plqcd;

extern "C" int plqcd_invert_cg_batch(plqcd_solve_item *items, int nitems, const plqcd_cg_param *prm, int use_graph,
                                     plqcd_batch_info *info, double *true_residuals) {
    clear_error();
    if (!items || nitems < 1 || !prm) return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg_batch: bad argument");
    if (!(prm->tol > 0) || prm->max_iter <= 0) return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg_batch: bad tol / max_iter");
    const int dev0 = items[0].lat ? items[0].lat->device : -1;
    for (int k = 0; k < nitems; k++) {
        const plqcd_solve_item &in = items[k];
        if (!in.lat || !in.g64 || in.nrhs < 1 || !in.x_even || !in.x_odd || !in.b_even || !in.b_odd)
            return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg_batch: item %d incomplete", k);
        if (in.lat->device != dev0) return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg_batch: items on different devices");
        if (in.g64->prec != PLQCD_F64 || in.g64->lat->geom.Vh != in.lat->geom.Vh)
            return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg_batch: item %d needs an F64 gauge field of its lattice", k);
        const plqcd_gauge *gs = in.g_sloppy ? in.g_sloppy : in.g64;
        if (gs->prec != prm->sloppy_prec || gs->lat->geom.Vh != in.lat->geom.Vh)
            return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg_batch: item %d sloppy gauge does not match", k);
    }
    PLQCD_CUDA_TRY(cudaSetDevice(dev0));

    Batch B;
    B.kappa = prm->kappa;
    B.tol = prm->tol;
    B.delta = prm->delta;
    B.mixed = prm->sloppy_prec != PLQCD_F64;
    // the batch runs on a private stream ordered after the first lattice's
    // stream (graph capture cannot use the legacy default stream)
    cudaStream_t user = items[0].lat->stream;
    PLQCD_CUDA_TRY(cudaStreamCreateWithFlags(&B.s, cudaStreamNonBlocking));
    cudaEvent_t ev0, ev1, evu;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventCreateWithFlags(&evu, cudaEventDisableTiming);
    cudaEventRecord(evu, user);
    cudaStreamWaitEvent(B.s, evu, 0);

    int rc = PLQCD_OK;
    McgControl *hctl = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    plqcd_batch_info inf;
    memset(&inf, 0, sizeof inf);
    do {
        if (cudaMalloc(&B.ctl, sizeof(McgControl)) != cudaSuccess ||
            cudaMalloc(&B.st_dev, sizeof(McgState) * nitems) != cudaSuccess ||
            cudaMallocHost(&hctl, sizeof(McgControl)) != cudaSuccess) {
            cudaGetLastError();
            rc = set_error(PLQCD_ERR_NOMEM, "plqcd_invert_cg_batch: control allocation");
            break;
        }
        McgControl c0{};
        c0.max_iter = prm->max_iter;
        c0.tol2 = prm->tol * prm->tol;
        c0.delta2 = prm->delta * prm->delta;
        if ((rc = cudaMemcpyAsync(B.ctl, &c0, sizeof c0, cudaMemcpyHostToDevice, B.s) == cudaSuccess
                      ? PLQCD_OK
                      : set_error(PLQCD_ERR_CUDA, "plqcd_invert_cg_batch: control upload")))
            break;
        // outside the timed solve: workspaces, tuning of every hop the loop
        // launches, and the graph (capture and instantiation run nothing)
        B.items.resize(nitems);
        for (int k = 0; k < nitems && rc == PLQCD_OK; k++) {
            Item &it = B.items[k];
            it.in = items[k];
            it.ps = prm->sloppy_prec;
            it.xprec = (it.ps == PLQCD_F64) ? PLQCD_F64 : PLQCD_F32;
            bool shared = false;
            for (int j = 0; j < k; j++) shared = shared || items[j].lat == items[k].lat;
            rc = alloc_item(B, it, shared);
        }
        for (int k = 0; k < nitems && rc == PLQCD_OK; k++) rc = tune_item(B, B.items[k]);
        if (rc) break;
        std::vector<McgState> hst(nitems);
        for (int k = 0; k < nitems; k++) hst[k] = B.items[k].st;
        if (cudaMemcpyAsync(B.st_dev, hst.data(), sizeof(McgState) * nitems, cudaMemcpyHostToDevice, B.s) !=
            cudaSuccess) {
            rc = set_error(PLQCD_ERR_CUDA, "plqcd_invert_cg_batch: state upload");
            break;
        }
        cudaStreamSynchronize(B.s);  // hst is a host temporary
        if (use_graph && (rc = build_graph(B, &graph, &gexec))) break;
        // the solve: start residuals, the loop, x_o
        cudaEventRecord(ev0, B.s);
        for (int k = 0; k < nitems && rc == PLQCD_OK; k++) rc = start_item(B, B.items[k]);
        if (rc) break;
        if (use_graph) {
            if (cudaGraphLaunch(gexec, B.s) != cudaSuccess) {
                rc = set_error(PLQCD_ERR_CUDA, "batch cg graph: launch: %s", cudaGetErrorString(cudaGetLastError()));
                break;
            }
            inf.graph_launches = 1;
        } else if ((rc = run_eager(B, hctl))) {
            break;
        }
        // fold in unconverged sloppy solutions, rebuild x_o, full-lattice residuals
        for (Item &it : B.items) {
            if ((rc = B.accum(it, false))) break;
            if ((rc = B.hop(it, it.in.g64, it.in.x_odd, it.in.x_even, PLQCD_ODD, 0, it.in.b_odd, B.kappa, 1.0))) break;
        }
        if (rc) break;
        cudaEventRecord(ev1, B.s);
        PLQCD_CUDA_TRY(cudaMemcpyAsync(hctl, B.ctl, sizeof(McgControl), cudaMemcpyDeviceToHost, B.s));
        // residuals |b - D x| / |b| per RHS (not part of the timed solve)
        int off = 0;
        inf.converged = 1;
        for (Item &it : B.items) {
            const int n = it.in.nrhs;
            std::vector<double> r2(n, 0.0), b2(n, 0.0), tmp(n), sr2(n), bp2(n);
            std::vector<int> act(n), conv(n);
            for (int par = 0; par < 2 && rc == PLQCD_OK; par++) {
                const void *xo = par ? it.in.x_even : it.in.x_odd, *xs_ = par ? it.in.x_odd : it.in.x_even;
                const void *bb = par ? it.in.b_odd : it.in.b_even;
                if ((rc = B.hop(it, it.in.g64, it.t64, xo, par, 0, xs_, -B.kappa, 1.0))) break;
                if ((rc = B.sub_norm2(it, it.r64, bb, it.t64, M_AUX))) break;
                cudaMemcpyAsync(tmp.data(), it.st.aux, sizeof(double) * n, cudaMemcpyDeviceToHost, B.s);
                cudaStreamSynchronize(B.s);
                for (int f = 0; f < n; f++) r2[f] += tmp[f];
                if ((rc = B.norm2(it, bb, PLQCD_F64, M_AUX, false))) break;
                cudaMemcpyAsync(tmp.data(), it.st.aux, sizeof(double) * n, cudaMemcpyDeviceToHost, B.s);
                cudaStreamSynchronize(B.s);
                for (int f = 0; f < n; f++) b2[f] += tmp[f];
            }
            if (rc) break;
            cudaMemcpyAsync(sr2.data(), it.st.sr2, sizeof(double) * n, cudaMemcpyDeviceToHost, B.s);
            cudaMemcpyAsync(bp2.data(), it.st.bp2, sizeof(double) * n, cudaMemcpyDeviceToHost, B.s);
            cudaMemcpyAsync(act.data(), it.st.active, sizeof(int) * n, cudaMemcpyDeviceToHost, B.s);
            cudaStreamSynchronize(B.s);
            for (int f = 0; f < n; f++) {
                const double tr = b2[f] > 0 ? sqrt(r2[f] / b2[f]) : 0.0;
                const double sr = bp2[f] > 0 ? sqrt(sr2[f] / bp2[f]) : 0.0;
                if (true_residuals) true_residuals[off + f] = tr;
                inf.max_true_residual = std::max(inf.max_true_residual, tr);
                inf.max_schur_residual = std::max(inf.max_schur_residual, sr);
                if (act[f]) inf.converged = 0;
            }
            off += n;
        }
        if (rc) break;
        inf.iterations = hctl->iter;
        inf.reliable_updates = hctl->reliable_count;
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        inf.seconds = ms / 1e3;
    } while (0);

    cudaStreamSynchronize(B.s);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    for (Item &it : B.items)
        if (it.mem) cudaFree(it.mem);
    if (B.ctl) cudaFree(B.ctl);
    if (B.st_dev) cudaFree(B.st_dev);
    if (hctl) cudaFreeHost(hctl);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaEventRecord(evu, B.s);
    cudaStreamWaitEvent(user, evu, 0);
    cudaEventDestroy(evu);
    cudaStreamDestroy(B.s);
    if (info) *info = inf;
    if (rc) return rc;
    if (!inf.converged) return set_error(PLQCD_ERR_NOCONV, "plqcd_invert_cg_batch: not converged in %d iterations", inf.iterations);
    return PLQCD_OK;
}
