// cg.cu -- even/odd preconditioned CG for the Wilson operator, FP64 and
// mixed precision with reliable updates.
//
// The reference stops at the hopping matrix (its operator and solver
// parameters are placeholders, include/plqcd_global_params.h:197-201); this
// solver builds on the same operator:
//   D = 1 - kappa H,   D [x_e; x_o] = [b_e; b_o]
//   Mhat = 1 - kappa^2 H_eo H_oe   (Schur complement on even sites)
//   b'   = b_e + kappa H_eo b_o,   Mhat x_e = b',   x_o = b_o + kappa H_oe x_e
// CG runs on the normal equations Mhat^dag Mhat x_e = Mhat^dag b' with
// Mhat^dag = g5 Mhat g5 (gamma5 folded into the hopping kernels).
//
// Mixed precision (Clark et al., "Solving Lattice QCD systems of equations
// using mixed precision solvers on GPUs", 2010): the recursion runs with a
// sloppy operator and sloppy vectors; whenever |r_sloppy| has dropped by
// `delta` since the last update, or looks converged, a reliable update adds
// the sloppy solution into the FP64 solution and recomputes the true
// residual with the FP64 operator (defect correction). Convergence is
// declared on the FP64 Schur residual |b' - Mhat x| / |b'| only; the final
// full-lattice residual |b - D x| / |b| is reported as well. All
// reductions accumulate in FP64 on the device and finalise alpha / beta
// there; the host reads one small state block per iteration to steer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "blas.cuh"
#include "internal.h"

using namespace plqcd;

namespace plqcd {

int lattice_workspace(plqcd_lattice *lat, size_t bytes, void **out) {
    if (lat->ws_bytes < bytes) {
        if (lat->ws) {
            cudaStreamSynchronize(lat->stream);
            cudaFree(lat->ws);
            lat->ws = nullptr;
            lat->ws_bytes = 0;
        }
        if (cudaMalloc(&lat->ws, bytes) != cudaSuccess) {
            cudaGetLastError();
            return set_error(PLQCD_ERR_NOMEM, "solver workspace of %zu bytes", bytes);
        }
        lat->ws_bytes = bytes;
    }
    *out = lat->ws;
    return PLQCD_OK;
}

}  // namespace plqcd

namespace {

struct Op {
    const Geom &g;
    cudaStream_t s;
    double kappa;
    // out_parity-specific hopping with epilogue
    int hop(const plqcd_gauge *gf, void *out, const void *in, int out_parity, unsigned flags, const void *x = nullptr,
            double a = 1.0, double b = 0.0) const {
        DslashCall c;
        c.gauge = gf->data;
        c.prec = gf->prec;
        c.recon = gf->recon;
        c.out = out;
        c.in = in;
        c.out_parity = out_parity;
        c.flags = flags;
        c.x = x;
        c.a_up = c.a_low = a;
        c.b = b;
        return launch_dslash(g, s, c);
    }
    // out = Mhat in (dagger: g5 Mhat g5 in); tmp_o: odd scratch
    int mhat(const plqcd_gauge *gf, void *out, const void *in, void *tmp_o, bool dagger) const {
        unsigned fin = dagger ? PLQCD_DSLASH_G5_IN : 0u, fout = dagger ? PLQCD_DSLASH_G5_OUT : 0u;
        PLQCD_TRY(hop(gf, tmp_o, in, PLQCD_ODD, fin));
        return hop(gf, out, tmp_o, PLQCD_EVEN, fout, in, -kappa * kappa, 1.0);
    }
};

}  // namespace

extern "C" void plqcd_cg_param_default(plqcd_cg_param *p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->kappa = 0.12;
    p->tol = 1e-10;
    p->max_iter = 10000;
    p->sloppy_prec = PLQCD_F64;
    p->delta = 0.01;
    p->verbose = 0;
}

extern "C" int plqcd_invert_cg(plqcd_lattice *lat, const plqcd_gauge *g64, const plqcd_gauge *gs, void *x_even,
                               void *x_odd, const void *b_even, const void *b_odd, const plqcd_cg_param *prm,
                               plqcd_cg_info *info) {
    clear_error();
    if (!lat || !g64 || !x_even || !x_odd || !b_even || !b_odd || !prm)
        return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg: null argument");
    if (!gs) gs = g64;
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    if (g64->prec != PLQCD_F64) return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg: the reliable gauge field must be F64");
    if (gs->prec != prm->sloppy_prec)
        return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg: sloppy gauge precision %d != sloppy_prec %d", gs->prec,
                         prm->sloppy_prec);
    if (g64->lat->geom.Vh != lat->geom.Vh || gs->lat->geom.Vh != lat->geom.Vh)
        return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg: gauge fields belong to another lattice");
    if (!(prm->tol > 0) || prm->max_iter <= 0) return set_error(PLQCD_ERR_ARG, "plqcd_invert_cg: bad tol / max_iter");

    const Geom &g = lat->geom;
    cudaStream_t s = lat->stream;
    const int ps = prm->sloppy_prec;
    const int xprec = (ps == PLQCD_F64) ? PLQCD_F64 : PLQCD_F32;
    const size_t b64 = spinor_parity_bytes(g.Vh, PLQCD_F64);
    const size_t bs = spinor_parity_bytes(g.Vh, ps);
    const size_t bx = spinor_parity_bytes(g.Vh, xprec);
    auto al = [](size_t n) { return (n + 255) & ~(size_t)255; };
    const size_t need = 5 * al(b64) + 5 * al(bs) + al(bx) + al(red_scratch_bytes());
    void *ws = nullptr;
    PLQCD_TRY(lattice_workspace(lat, need, &ws));
    char *w = static_cast<char *>(ws);
    auto take = [&](size_t n) {
        void *p = w;
        w += al(n);
        return p;
    };
    void *bprime = take(b64), *rhs = take(b64), *r64 = take(b64), *t64 = take(b64), *tmp64 = take(b64);
    void *rs = take(bs), *p = take(bs), *Ap = take(bs), *t = take(bs), *tmps = take(bs);
    void *xs = take(bx);
    void *redmem = take(red_scratch_bytes());
    PLQCD_CUDA_TRY(cudaMemsetAsync(redmem, 0, red_scratch_bytes(), s));
    RedScratch red = red_scratch_from(redmem);
    CgState *hst = nullptr;
    PLQCD_CUDA_TRY(cudaMallocHost(&hst, sizeof(CgState)));
    auto read_state = [&]() -> int {
        PLQCD_CUDA_TRY(cudaMemcpyAsync(hst, red.state, sizeof(CgState), cudaMemcpyDeviceToHost, s));
        PLQCD_CUDA_TRY(cudaStreamSynchronize(s));
        return PLQCD_OK;
    };

    Op op{g, s, prm->kappa};
    cudaEvent_t e0 = lat->ev0, e1 = lat->ev1;
    cudaEventRecord(e0, s);
    int rc = PLQCD_OK;
    plqcd_cg_info inf;
    memset(&inf, 0, sizeof inf);
    double bp2 = 0, sr2 = 0;
    bool end_recorded = false;  // device time covers the solve, not the verification

    do {
        const bool mixed = ps != PLQCD_F64;
        // b' = b_e + kappa H_eo b_o ; rhs = Mhat^dag b'
        if ((rc = op.hop(g64, bprime, b_odd, PLQCD_EVEN, 0, b_even, prm->kappa, 1.0))) break;
        if ((rc = blas_norm2(g, s, bprime, PLQCD_F64, red, RED_AUX))) break;
        if (!mixed && (rc = op.mhat(g64, rhs, bprime, tmp64, true))) break;
        if ((rc = read_state())) break;
        bp2 = hst->aux;
        if (!(bp2 > 0)) {  // zero source: zero solution
            cudaMemsetAsync(x_even, 0, b64, s);
            rc = op.hop(g64, x_odd, x_even, PLQCD_ODD, 0, b_odd, prm->kappa, 1.0);
            inf.converged = 1;
            break;
        }
        // x = 0, r = p = rhs. The sloppy solution x_s is not cleared: while
        // `fresh` it counts as zero, and its next update writes it unread
        cudaMemsetAsync(x_even, 0, b64, s);
        bool fresh = true;
        if (mixed) {
            // the sloppy recursion starts from rhs in sloppy precision, so
            // the sloppy operator computes it; convergence is decided on the
            // FP64 Schur residual of b', which does not use rhs
            if ((rc = launch_spinor_convert(g, s, t, ps, bprime, PLQCD_F64))) break;
            if ((rc = op.mhat(gs, rs, t, tmps, true))) break;
            if ((rc = blas_norm2(g, s, rs, ps, red, RED_RR_INIT))) break;
            if (cudaMemcpyAsync(p, rs, bs, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
                rc = set_error(PLQCD_ERR_CUDA, "plqcd_invert_cg: device copy failed");
                break;
            }
            inf.sloppy_hops += 2;
        } else {
            if ((rc = blas_norm2(g, s, rhs, PLQCD_F64, red, RED_RR_INIT))) break;
            if ((rc = launch_spinor_convert(g, s, rs, ps, rhs, PLQCD_F64))) break;
            if ((rc = launch_spinor_convert(g, s, p, ps, rhs, PLQCD_F64))) break;
        }
        if ((rc = read_state())) break;
        const double rhs2 = hst->rr;
        double maxrr = hst->rr;
        double target = prm->tol * prm->tol * rhs2;  // normal-equation trigger for convergence checks
        const double delta2 = prm->delta * prm->delta;
        // a sloppy recursion that stops reducing its residual (16-bit storage
        // with a tiny delta) would never trigger an update: force one after
        // this many iterations without
        const int max_sloppy_run = 100;
        int last_reliable = 0;

        for (int it = 1; it <= prm->max_iter; it++) {
            // Ap = Mhat^dag Mhat p ; pAp = |Mhat p|^2
            if ((rc = op.mhat(gs, t, p, tmps, false))) break;
            if ((rc = blas_norm2(g, s, t, ps, red, RED_ALPHA))) break;
            if ((rc = op.mhat(gs, Ap, t, tmps, true))) break;
            // r -= alpha Ap ; |r|^2. The solution update x_s += alpha p of
            // this iteration runs in the p update below (which reads p
            // anyway), or in the fold of a reliable update
            if ((rc = blas_cg_update_r(g, s, rs, Ap, ps, red))) break;
            inf.sloppy_hops += 4;
            inf.iterations = it;
            if ((rc = read_state())) break;
            const double rr = hst->rr;
            if (!std::isfinite(rr)) {
                rc = set_error(PLQCD_ERR_NOCONV, "plqcd_invert_cg: residual is not finite at iteration %d", it);
                break;
            }
            const bool reliable = (mixed && rr < delta2 * maxrr) || rr <= target || it - last_reliable >= max_sloppy_run;
            if (reliable) {
                // defect correction: x += x_s + alpha p, then the Schur
                // residual b' - Mhat x in FP64 (for the mixed solve written
                // only in the sloppy format: the restart needs nothing more)
                if ((rc = blas_accum(g, s, x_even, xs, xprec, fresh, p, ps, red))) break;
                fresh = true;
                if ((rc = op.mhat(g64, t64, x_even, tmp64, false))) break;
                if (mixed)
                    rc = blas_sub_norm2_to(g, s, t, ps, bprime, t64, red, RED_SR2);
                else
                    rc = blas_sub_norm2(g, s, r64, bprime, t64, red, RED_SR2);
                if (rc) break;
                inf.f64_hops += 2;
                inf.reliable_updates++;
                last_reliable = it;
                if ((rc = read_state())) break;
                sr2 = hst->sr2;
                if (prm->verbose)
                    fprintf(stderr, "plqcd cg: it %d reliable update, |r_schur|/|b'| = %.3e\n", it, sqrt(sr2 / bp2));
                if (sr2 <= prm->tol * prm->tol * bp2) {
                    inf.converged = 1;
                    break;
                }
                // restart the recursion from r = Mhat^dag (b' - Mhat x). The
                // FP64 residual above decides convergence; the restart
                // direction only needs the sloppy operator's accuracy
                if (mixed) {
                    if ((rc = op.mhat(gs, rs, t, tmps, true))) break;
                    if ((rc = blas_norm2(g, s, rs, ps, red, RED_RR_TRUE))) break;
                    inf.sloppy_hops += 2;
                } else {
                    if ((rc = op.mhat(g64, t64, r64, tmp64, true))) break;
                    if ((rc = blas_norm2(g, s, t64, PLQCD_F64, red, RED_RR_TRUE))) break;
                    if ((rc = launch_spinor_convert(g, s, rs, ps, t64, PLQCD_F64))) break;
                    inf.f64_hops += 2;
                }
                if ((rc = read_state())) break;
                maxrr = hst->rr;
                if (hst->rr <= target) target *= 0.25;
            } else {
                maxrr = std::max(maxrr, rr);
            }
            if ((rc = blas_cg_p_x(g, s, p, rs, ps, xs, xprec, reliable ? 0 : (fresh ? 1 : 2), red))) break;
            if (!reliable) fresh = false;
        }
        if (rc) break;
        if (!inf.converged) {
            // fold in what the sloppy recursion has so far
            if ((rc = blas_accum(g, s, x_even, xs, xprec, fresh, nullptr, ps, red))) break;
        }
        // x_o = b_o + kappa H_oe x_e
        if ((rc = op.hop(g64, x_odd, x_even, PLQCD_ODD, 0, b_odd, prm->kappa, 1.0))) break;
        // the solve ends here; what follows is the verification
        cudaEventRecord(e1, s);
        end_recorded = true;
        // full-lattice residual |b - D x| / |b|, D x = x - kappa H x
        double r2 = 0, b2 = 0;
        if ((rc = op.hop(g64, t64, x_odd, PLQCD_EVEN, 0, x_even, -prm->kappa, 1.0))) break;
        if ((rc = blas_sub_norm2(g, s, r64, b_even, t64, red, RED_AUX))) break;
        if ((rc = read_state())) break;
        r2 += hst->aux;
        if ((rc = op.hop(g64, t64, x_even, PLQCD_ODD, 0, x_odd, -prm->kappa, 1.0))) break;
        if ((rc = blas_sub_norm2(g, s, r64, b_odd, t64, red, RED_AUX))) break;
        if ((rc = read_state())) break;
        r2 += hst->aux;
        if ((rc = blas_norm2(g, s, b_even, PLQCD_F64, red, RED_AUX))) break;
        if ((rc = read_state())) break;
        b2 += hst->aux;
        if ((rc = blas_norm2(g, s, b_odd, PLQCD_F64, red, RED_AUX))) break;
        if ((rc = read_state())) break;
        b2 += hst->aux;
        inf.true_residual = sqrt(r2 / b2);
        inf.schur_residual = sqrt(sr2 / bp2);
    } while (0);

    if (!end_recorded) cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    inf.seconds = ms / 1e3;
    cudaFreeHost(hst);
    // a hop whose staged loads never arrived leaves a flag, not a CUDA error
    if (!rc && dslash_tma_status(true))
        rc = set_error(PLQCD_ERR_TIMEOUT, "plqcd_invert_cg: a TMA stage wait of a hop ran out");
    if (info) *info = inf;
    if (rc) return rc;
    if (!inf.converged)
        return set_error(PLQCD_ERR_NOCONV, "plqcd_invert_cg: not converged after %d iterations (|r|/|b'| = %.3e)",
                         inf.iterations, inf.schur_residual);
    return PLQCD_OK;
}
