// blas.cuh -- vector kernels and FP64 reductions for the solvers.
#pragma once

#include <cuda_runtime.h>

#include "internal.h"

namespace plqcd {

// Solver scalars kept in device memory. Reductions finalise them on the
// device (last block of the reducing kernel), so kernels read alpha / beta
// from here and the host only needs them to steer the iteration.
struct CgState {
    double rr;       // |r_sloppy|^2 (iterated), or |r|^2 after a reliable update
    double rr_old;   // previous rr
    double pAp;      // <p, A p> = |Mhat p|^2
    double alpha;    // rr / pAp
    double beta;     // rr / rr_old
    double sr2;      // |b' - Mhat x|^2 at the last reliable update (Schur residual)
    double aux;      // last plain reduction result
    double pad;
};

// Reduction scratch: per-block partials, the arrival counter of the
// last-block pattern, and the CgState block.
struct RedScratch {
    double *partials = nullptr;  // kMaxRedBlocks * 2 doubles
    unsigned *counter = nullptr;
    CgState *state = nullptr;
};
constexpr int kMaxRedBlocks = 1184;  // 8 x 148 SMs
constexpr int kBlasBlock = 256;
size_t red_scratch_bytes();
// carve a RedScratch out of `mem` (red_scratch_bytes(), zero-initialised)
RedScratch red_scratch_from(void *mem);

enum RedOp : int {
    RED_AUX = 0,     // state.aux = sum
    RED_ALPHA = 1,   // state.pAp = sum; state.alpha = state.rr / sum
    RED_RR = 2,      // state.rr_old = state.rr; state.rr = sum; state.beta = sum / state.rr_old
    RED_SR2 = 3,     // state.sr2 = sum
    RED_RR_TRUE = 4, // state.rr = sum; state.beta = sum / state.rr_old (after a reliable update)
    RED_RR_INIT = 5, // state.rr = state.rr_old = sum
};

// sum |x|^2 (FP64 accumulation); finalised by `op`
int blas_norm2(const Geom &g, cudaStream_t s, const void *x, int prec, const RedScratch &r, RedOp op);
// out64 = a64 - b64; sum |out|^2 -> op
int blas_sub_norm2(const Geom &g, cudaStream_t s, void *out, const void *a, const void *b, const RedScratch &r,
                   RedOp op);
// |x_f|^2 of nf fields stored back to back; scratch: nf * norm2_blocks(Vh)
// partials and nf counters (zero on entry, left zero on exit)
int norm2_blocks(long Vh);
int preload_norm2_multi();
int launch_norm2_multi(const Geom &g, cudaStream_t s, const void *fields, int prec, int nf, double *partials,
                       unsigned *counters, double *out);
// y = a x + b y (F64 fields)
int blas_axpby64(const Geom &g, cudaStream_t s, double a, const void *x, double b, void *y);
// r_s -= alpha Ap, |r_s|^2 -> RED_RR (no solution update)
int blas_cg_update_r(const Geom &g, cudaStream_t s, void *rs, const void *Ap, int prec, const RedScratch &r);
// xmode 1: x_s = alpha p, 2: x_s += alpha p, 0: no x update; then p = r + beta p
int blas_cg_p_x(const Geom &g, cudaStream_t s, void *p, const void *rs, int prec, void *xs, int xprec, int xmode,
                const RedScratch &r);
// x64 += x_s (fresh: x_s counts as zero) [+ alpha p when p != null, with p in prec]
int blas_accum(const Geom &g, cudaStream_t s, void *x64, const void *xs, int xprec, bool fresh, const void *p,
               int prec, const RedScratch &r);
// out (prec) = a - b, |a - b|^2 -> op (a, b F64)
int blas_sub_norm2_to(const Geom &g, cudaStream_t s, void *out, int prec, const void *a, const void *b,
                      const RedScratch &r, RedOp op);

}  // namespace plqcd
