// blas.cu -- vector kernels and deterministic FP64 reductions.
//
// Reductions accumulate in FP64 whatever the storage precision. Each block
// writes its partial sum; the last block to arrive (atomic ticket) adds the
// partials in a fixed order, so results do not depend on block scheduling,
// and applies the solver-scalar update selected by RedOp.
#include <cuda_runtime.h>

#include "blas.cuh"
#include "device_fields.cuh"

namespace plqcd {

size_t red_scratch_bytes() { return sizeof(double) * kMaxRedBlocks * 2 + 256 + sizeof(CgState); }

RedScratch red_scratch_from(void *mem) {
    RedScratch r;
    char *p = static_cast<char *>(mem);
    r.partials = reinterpret_cast<double *>(p);
    r.counter = reinterpret_cast<unsigned *>(p + sizeof(double) * kMaxRedBlocks * 2);
    r.state = reinterpret_cast<CgState *>(p + sizeof(double) * kMaxRedBlocks * 2 + 256);
    return r;
}

namespace dev {

inline int blas_grid(long n) {
    long b = (n + kBlasBlock - 1) / kBlasBlock;
    return (int)(b < kMaxRedBlocks ? b : kMaxRedBlocks);
}

__device__ __forceinline__ void apply_op(RedOp op, double sum, CgState *st) {
    switch (op) {
        case RED_AUX: st->aux = sum; break;
        case RED_ALPHA:
            st->pAp = sum;
            st->alpha = sum > 0 ? st->rr / sum : 0.0;
            break;
        case RED_RR:
            st->rr_old = st->rr;
            st->rr = sum;
            st->beta = st->rr_old > 0 ? sum / st->rr_old : 0.0;
            break;
        case RED_SR2: st->sr2 = sum; break;
        case RED_RR_TRUE:
            st->rr = sum;
            st->beta = st->rr_old > 0 ? sum / st->rr_old : 0.0;
            break;
        case RED_RR_INIT:
            st->rr = sum;
            st->rr_old = sum;
            break;
    }
}

// Block-reduce v, publish the partial, and let the last block finish.
__device__ void reduce_finish(double v, RedScratch r, RedOp op) {
    __shared__ double warp_sums[kBlasBlock / 32];
    __shared__ bool last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_sums[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) b += warp_sums[k];
        r.partials[blockIdx.x] = b;
        __threadfence();
        unsigned ticket = atomicAdd(r.counter, 1u);
        last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // fixed-order sum of the partials
    double t = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) t += ((volatile double *)r.partials)[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    __syncthreads();
    if (lane == 0) warp_sums[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += warp_sums[k];
        apply_op(op, tot, r.state);
        *r.counter = 0;  // ready for the next reduction on this scratch
    }
}

template <typename R>
__device__ __forceinline__ double norm2_site(const cx<R> v[12]) {
    double s = 0;
#pragma unroll
    for (int k = 0; k < 12; k++) s += (double)v[k].re * v[k].re + (double)v[k].im * v[k].im;
    return s;
}

template <int P>
__global__ void __launch_bounds__(kBlasBlock) k_norm2(const void *x, long Vh, RedScratch r, RedOp op) {
    using R = typename SpinorIO<P>::real;
    double acc = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<R> v[12];
        SpinorIO<P>::load(x, Vh, h, v);
        acc += norm2_site(v);
    }
    reduce_finish(acc, r, op);
}

__global__ void __launch_bounds__(kBlasBlock) k_sub_norm2(void *out, const void *a, const void *b, long Vh,
                                                          RedScratch r, RedOp op) {
    double acc = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<double> av[12], bv[12];
        SpinorIO<PLQCD_F64>::load(a, Vh, h, av);
        SpinorIO<PLQCD_F64>::load(b, Vh, h, bv);
#pragma unroll
        for (int k = 0; k < 12; k++) av[k] = csub(av[k], bv[k]);
        SpinorIO<PLQCD_F64>::store(out, Vh, h, av);
        acc += norm2_site(av);
    }
    reduce_finish(acc, r, op);
}

// r_s -= alpha Ap ; |r_s|^2 (the solution update of the iteration is in k_cg_p_x)
template <int P>
__global__ void __launch_bounds__(kBlasBlock) k_cg_update_r(void *rs, const void *Ap, long Vh, RedScratch r) {
    using R = typename SpinorIO<P>::real;
    const R a = (R)r.state->alpha;
    double acc = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<R> av[12], rv[12];
        SpinorIO<P>::load(Ap, Vh, h, av);
        SpinorIO<P>::load(rs, Vh, h, rv);
#pragma unroll
        for (int k = 0; k < 12; k++) rv[k] = {fma(-a, av[k].re, rv[k].re), fma(-a, av[k].im, rv[k].im)};
        SpinorIO<P>::store(rs, Vh, h, rv);
        acc += norm2_site(rv);
    }
    reduce_finish(acc, r, RED_RR);
}

// XMODE 1: x_s = alpha p (x_s counts as zero); 2: x_s += alpha p; 0: no x
// update (a reliable update folded alpha p into x). Then p = r + beta p.
template <int P, int XP, int XMODE>
__global__ void __launch_bounds__(kBlasBlock) k_cg_p_x(void *p, const void *rs, void *xs, long Vh, const CgState *st) {
    using R = typename SpinorIO<P>::real;
    using RX = typename SpinorIO<XP>::real;
    const R beta = (R)st->beta;
    const RX ax = (RX)st->alpha;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<R> pv[12], rv[12];
        SpinorIO<P>::load(p, Vh, h, pv);
        SpinorIO<P>::load(rs, Vh, h, rv);
        if (XMODE) {
            cx<RX> xv[12];
            if (XMODE == 1) {
#pragma unroll
                for (int k = 0; k < 12; k++) xv[k] = {RX(0), RX(0)};
            } else {
                SpinorIO<XP>::load(xs, Vh, h, xv);
            }
#pragma unroll
            for (int k = 0; k < 12; k++)
                xv[k] = {fma(ax, (RX)pv[k].re, xv[k].re), fma(ax, (RX)pv[k].im, xv[k].im)};
            SpinorIO<XP>::store(xs, Vh, h, xv);
        }
#pragma unroll
        for (int k = 0; k < 12; k++) pv[k] = {fma(beta, pv[k].re, rv[k].re), fma(beta, pv[k].im, rv[k].im)};
        SpinorIO<P>::store(p, Vh, h, pv);
    }
}

// x64 += x_s (FRESH: x_s counts as zero) [+ alpha p when P >= 0, the
// current iteration's update, computed as k_cg_p_x would]
template <int P, int XP, bool FRESH>
__global__ void __launch_bounds__(kBlasBlock) k_accum(void *x64, const void *xs, const void *p, long Vh,
                                                      const CgState *st) {
    using RX = typename SpinorIO<XP>::real;
    const RX ax = (RX)st->alpha;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<double> xv[12];
        cx<RX> sv[12];
        SpinorIO<PLQCD_F64>::load(x64, Vh, h, xv);
        if (FRESH) {
#pragma unroll
            for (int k = 0; k < 12; k++) sv[k] = {RX(0), RX(0)};
        } else {
            SpinorIO<XP>::load(xs, Vh, h, sv);
        }
        if constexpr (P >= 0) {
            using R = typename SpinorIO<P>::real;
            cx<R> pv[12];
            SpinorIO<P>::load(p, Vh, h, pv);
#pragma unroll
            for (int k = 0; k < 12; k++)
                sv[k] = {fma(ax, (RX)pv[k].re, sv[k].re), fma(ax, (RX)pv[k].im, sv[k].im)};
        }
#pragma unroll
        for (int k = 0; k < 12; k++) xv[k] = {xv[k].re + (double)sv[k].re, xv[k].im + (double)sv[k].im};
        SpinorIO<PLQCD_F64>::store(x64, Vh, h, xv);
    }
}

// z = a - b (F64) ; |z|^2 -> op ; out = z in format SP (z itself is not stored)
template <int SP>
__global__ void __launch_bounds__(kBlasBlock) k_sub_norm2_to(void *out, const void *a, const void *b, long Vh,
                                                             RedScratch r, RedOp op) {
    using RS = typename SpinorIO<SP>::real;
    double acc = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<double> av[12], bv[12];
        SpinorIO<PLQCD_F64>::load(a, Vh, h, av);
        SpinorIO<PLQCD_F64>::load(b, Vh, h, bv);
        cx<RS> d[12];
#pragma unroll
        for (int k = 0; k < 12; k++) {
            av[k] = csub(av[k], bv[k]);
            d[k] = {(RS)av[k].re, (RS)av[k].im};
        }
        SpinorIO<SP>::store(out, Vh, h, d);
        acc += norm2_site(av);
    }
    reduce_finish(acc, r, op);
}

__global__ void __launch_bounds__(kBlasBlock) k_axpby64(double a, const void *x, double b, void *y, long Vh) {
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<double> xv[12], yv[12];
        SpinorIO<PLQCD_F64>::load(x, Vh, h, xv);
        SpinorIO<PLQCD_F64>::load(y, Vh, h, yv);
#pragma unroll
        for (int k = 0; k < 12; k++) yv[k] = {fma(a, xv[k].re, b * yv[k].re), fma(a, xv[k].im, b * yv[k].im)};
        SpinorIO<PLQCD_F64>::store(y, Vh, h, yv);
    }
}

}  // namespace dev

#define BLAS_PREC_SWITCH(prec, F)                                                   \
    switch (prec) {                                                                 \
        case PLQCD_F64: F(PLQCD_F64); break;                                        \
        case PLQCD_F32: F(PLQCD_F32); break;                                        \
        case PLQCD_F16: F(PLQCD_F16); break;                                        \
        case PLQCD_BF16: F(PLQCD_BF16); break;                                      \
        default: return set_error(PLQCD_ERR_ARG, "blas: unknown precision %d", prec); \
    }

int blas_norm2(const Geom &g, cudaStream_t s, const void *x, int prec, const RedScratch &r, RedOp op) {
    const int nb = dev::blas_grid(g.Vh);
#define F(P) dev::k_norm2<P><<<nb, kBlasBlock, 0, s>>>(x, g.Vh, r, op)
    BLAS_PREC_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int blas_sub_norm2(const Geom &g, cudaStream_t s, void *out, const void *a, const void *b, const RedScratch &r,
                   RedOp op) {
    dev::k_sub_norm2<<<dev::blas_grid(g.Vh), kBlasBlock, 0, s>>>(out, a, b, g.Vh, r, op);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int blas_cg_update_r(const Geom &g, cudaStream_t s, void *rs, const void *Ap, int prec, const RedScratch &r) {
    const int nb = dev::blas_grid(g.Vh);
#define F(P) dev::k_cg_update_r<P><<<nb, kBlasBlock, 0, s>>>(rs, Ap, g.Vh, r)
    BLAS_PREC_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int blas_cg_p_x(const Geom &g, cudaStream_t s, void *p, const void *rs, int prec, void *xs, int xprec, int xmode,
                const RedScratch &r) {
    const int nb = dev::blas_grid(g.Vh);
    if (xprec != PLQCD_F64 && xprec != PLQCD_F32)
        return set_error(PLQCD_ERR_ARG, "blas_cg_p_x: solution accumulator must be F64 or F32");
#define G(P, XP)                                                                                        \
    switch (xmode) {                                                                                    \
        case 0: dev::k_cg_p_x<P, XP, 0><<<nb, kBlasBlock, 0, s>>>(p, rs, xs, g.Vh, r.state); break;     \
        case 1: dev::k_cg_p_x<P, XP, 1><<<nb, kBlasBlock, 0, s>>>(p, rs, xs, g.Vh, r.state); break;     \
        default: dev::k_cg_p_x<P, XP, 2><<<nb, kBlasBlock, 0, s>>>(p, rs, xs, g.Vh, r.state); break;   \
    }
#define F(P)                         \
    if (xprec == PLQCD_F64) {        \
        G(P, PLQCD_F64)              \
    } else {                         \
        G(P, PLQCD_F32)              \
    }
    BLAS_PREC_SWITCH(prec, F)
#undef F
#undef G
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int blas_accum(const Geom &g, cudaStream_t s, void *x64, const void *xs, int xprec, bool fresh, const void *p,
               int prec, const RedScratch &r) {
    const int nb = dev::blas_grid(g.Vh);
    if (xprec != PLQCD_F64 && xprec != PLQCD_F32)
        return set_error(PLQCD_ERR_ARG, "blas_accum: accumulator must be F64 or F32");
    if (!p) {
        if (fresh) return PLQCD_OK;  // x_s is zero
        if (xprec == PLQCD_F64)
            dev::k_accum<-1, PLQCD_F64, false><<<nb, kBlasBlock, 0, s>>>(x64, xs, nullptr, g.Vh, r.state);
        else
            dev::k_accum<-1, PLQCD_F32, false><<<nb, kBlasBlock, 0, s>>>(x64, xs, nullptr, g.Vh, r.state);
    } else {
#define G(P, XP)                                                                                   \
    if (fresh)                                                                                     \
        dev::k_accum<P, XP, true><<<nb, kBlasBlock, 0, s>>>(x64, xs, p, g.Vh, r.state);            \
    else                                                                                           \
        dev::k_accum<P, XP, false><<<nb, kBlasBlock, 0, s>>>(x64, xs, p, g.Vh, r.state);
#define F(P)                   \
    if (xprec == PLQCD_F64) {  \
        G(P, PLQCD_F64)        \
    } else {                   \
        G(P, PLQCD_F32)        \
    }
        BLAS_PREC_SWITCH(prec, F)
#undef F
#undef G
    }
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int blas_sub_norm2_to(const Geom &g, cudaStream_t s, void *out, int prec, const void *a, const void *b,
                      const RedScratch &r, RedOp op) {
    const int nb = dev::blas_grid(g.Vh);
#define F(P) dev::k_sub_norm2_to<P><<<nb, kBlasBlock, 0, s>>>(out, a, b, g.Vh, r, op)
    BLAS_PREC_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int blas_axpby64(const Geom &g, cudaStream_t s, double a, const void *x, double b, void *y) {
    dev::k_axpby64<<<dev::blas_grid(g.Vh), kBlasBlock, 0, s>>>(a, x, b, y, g.Vh);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

}  // namespace plqcd

// ---------------------------------------------------------------------------
// |x_f|^2 of nf fields stored back to back (multi-RHS blocks), one grid row
// per field; partials[f * gridDim.x + b], counters[f], results out[f].
// ---------------------------------------------------------------------------
namespace plqcd {
namespace dev {

template <int P>
__global__ void __launch_bounds__(kBlasBlock) k_norm2_multi(const char *fields, size_t field_bytes, long Vh,
                                                            double *partials, unsigned *counters, double *out) {
    using R = typename SpinorIO<P>::real;
    const int f = blockIdx.y;
    const void *x = fields + (size_t)f * field_bytes;
    double v = 0;
    for (long h = (long)blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += (long)gridDim.x * blockDim.x) {
        cx<R> s[12];
        SpinorIO<P>::load(x, Vh, h, s);
        v += norm2_site(s);
    }
    __shared__ double ws[kBlasBlock / 32];
    __shared__ bool last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) b += ws[k];
        partials[(size_t)f * gridDim.x + blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(&counters[f], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x)
        t += ((volatile double *)partials)[(size_t)f * gridDim.x + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    __syncthreads();
    if (lane == 0) ws[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += ws[k];
        out[f] = tot;
        counters[f] = 0;
    }
}

}  // namespace dev

int norm2_blocks(long Vh) { return dev::blas_grid(Vh); }

// Loads k_norm2_multi for every precision on the current device (with lazy
// module loading a kernel is otherwise loaded by its first launch).
int preload_norm2_multi() {
    cudaFuncAttributes a;
    for (const void *k : {(const void *)dev::k_norm2_multi<PLQCD_F64>, (const void *)dev::k_norm2_multi<PLQCD_F32>,
                          (const void *)dev::k_norm2_multi<PLQCD_F16>, (const void *)dev::k_norm2_multi<PLQCD_BF16>})
        PLQCD_CUDA_TRY(cudaFuncGetAttributes(&a, k));
    return PLQCD_OK;
}

int launch_norm2_multi(const Geom &g, cudaStream_t s, const void *fields, int prec, int nf, double *partials,
                       unsigned *counters, double *out) {
    const int nb = dev::blas_grid(g.Vh);
    const size_t fb = spinor_parity_bytes(g.Vh, prec);
    dim3 grid(nb, nf);
#define F(P) dev::k_norm2_multi<P><<<grid, kBlasBlock, 0, s>>>((const char *)fields, fb, g.Vh, partials, counters, out)
    BLAS_PREC_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

}  // namespace plqcd
