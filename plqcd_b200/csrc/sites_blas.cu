// sites_blas.cu -- FP64 vector operations of the even/odd CG on a site range
// of one-parity fields, with the solver scalars read on the device, and a
// one-launch copy of many device segments.
//
// The t-slab decomposition (plqcd_b200/shard.py) runs its CG on the slab
// interior: the reference's solver-free hop has no counterpart
// (include/plqcd_global_params.h:197-201); the operations are those of
// plqcd_invert_cg (cg.cu / blas.cu) restricted to [h_begin, h_begin +
// h_count). Reductions accumulate in FP64 in a fixed order (per-block
// partials summed by the last block to arrive), so results do not depend on
// scheduling. Scalars (alpha = rr / pAp, beta = rr_new / rr) come from device
// arrays, so a caller steers the iteration with one small read when it
// chooses, not one per operation.
//
// plqcd_copy_segments moves the ghost slices of a decomposition (one
// contiguous run per SoA plane, direction and slab) in one launch: the
// segment table travels in the kernel's parameters.
#include <cuda_runtime.h>

#include "blas.cuh"
#include "device_fields.cuh"
#include "internal.h"

namespace plqcd {
namespace dev {

struct SitesArgs {
    long Vh, h0, n;
    double *partials;   // gridDim.x doubles
    unsigned *counter;  // zero on entry, left zero
    double *out;        // the reduction result
};

// block sum of v; the last block to arrive writes the total to a.out
__device__ void sites_reduce(double v, const SitesArgs &a) {
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
        a.partials[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(a.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) t += ((volatile double *)a.partials)[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    __syncthreads();
    if (lane == 0) ws[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += ws[k];
        *a.out = tot;
        *a.counter = 0;
    }
}

using S64 = SpinorIO<PLQCD_F64>;

__device__ __forceinline__ double site_norm2(const cx<double> v[12]) {
    double s = 0;
#pragma unroll
    for (int k = 0; k < 12; k++) s += v[k].re * v[k].re + v[k].im * v[k].im;
    return s;
}

__global__ void __launch_bounds__(kBlasBlock) k_sites_norm2(const void *x, SitesArgs a) {
    double v = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long)gridDim.x * blockDim.x) {
        cx<double> s[12];
        S64::load(x, a.Vh, a.h0 + i, s);
        v += site_norm2(s);
    }
    sites_reduce(v, a);
}

// alpha = coef[0] / coef[1]; x += alpha p; r -= alpha Ap; sum |r|^2
__global__ void __launch_bounds__(kBlasBlock) k_sites_cg_update(void *x, void *r, const void *p, const void *Ap,
                                                                const double *coef, SitesArgs a) {
    const double alpha = coef[1] != 0.0 ? coef[0] / coef[1] : 0.0;
    double v = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long)gridDim.x * blockDim.x) {
        const long h = a.h0 + i;
        cx<double> xv[12], rv[12], pv[12], av[12];
        S64::load(x, a.Vh, h, xv);
        S64::load(r, a.Vh, h, rv);
        S64::load(p, a.Vh, h, pv);
        S64::load(Ap, a.Vh, h, av);
#pragma unroll
        for (int k = 0; k < 12; k++) {
            xv[k] = {fma(alpha, pv[k].re, xv[k].re), fma(alpha, pv[k].im, xv[k].im)};
            rv[k] = {fma(-alpha, av[k].re, rv[k].re), fma(-alpha, av[k].im, rv[k].im)};
        }
        S64::store(x, a.Vh, h, xv);
        S64::store(r, a.Vh, h, rv);
        v += site_norm2(rv);
    }
    sites_reduce(v, a);
}

// beta = coef[0] / coef[1]; p = r + beta p
__global__ void __launch_bounds__(kBlasBlock) k_sites_xpay(void *p, const void *r, const double *coef, long Vh,
                                                           long h0, long n) {
    const double beta = coef[1] != 0.0 ? coef[0] / coef[1] : 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long h = h0 + i;
        cx<double> pv[12], rv[12];
        S64::load(p, Vh, h, pv);
        S64::load(r, Vh, h, rv);
#pragma unroll
        for (int k = 0; k < 12; k++) pv[k] = {fma(beta, pv[k].re, rv[k].re), fma(beta, pv[k].im, rv[k].im)};
        S64::store(p, Vh, h, pv);
    }
}

// z = x - y; sum |z|^2
__global__ void __launch_bounds__(kBlasBlock) k_sites_sub_norm2(void *z, const void *x, const void *y, SitesArgs a) {
    double v = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long)gridDim.x * blockDim.x) {
        const long h = a.h0 + i;
        cx<double> xv[12], yv[12];
        S64::load(x, a.Vh, h, xv);
        S64::load(y, a.Vh, h, yv);
#pragma unroll
        for (int k = 0; k < 12; k++) xv[k] = csub(xv[k], yv[k]);
        S64::store(z, a.Vh, h, xv);
        v += site_norm2(xv);
    }
    sites_reduce(v, a);
}

struct CopyTable {
    uint4 *dst[PLQCD_COPY_MAX_SEGMENTS];
    const uint4 *src[PLQCD_COPY_MAX_SEGMENTS];
    long n16[PLQCD_COPY_MAX_SEGMENTS];  // 16-byte units
};

// blockIdx.y = segment
__global__ void __launch_bounds__(256) k_copy_segments(const __grid_constant__ CopyTable t) {
    const int sg = blockIdx.y;
    uint4 *d = t.dst[sg];
    const uint4 *s = t.src[sg];
    const long n = t.n16[sg];
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) d[i] = s[i];
}

}  // namespace dev

namespace {

int sites_check(plqcd_lattice *lat, long h0, long n, const char *who) {
    if (!lat) return set_error(PLQCD_ERR_ARG, "%s: null lattice", who);
    if (h0 < 0 || n < 1 || h0 + n > lat->geom.Vh)
        return set_error(PLQCD_ERR_ARG, "%s: site range [%ld, %ld) outside [0, %ld)", who, h0, h0 + n,
                         lat->geom.Vh);
    return PLQCD_OK;
}

int sites_grid(long n) {
    const long b = (n + kBlasBlock - 1) / kBlasBlock;
    return (int)(b < kMaxRedBlocks ? b : kMaxRedBlocks);
}

// reduction scratch from the lattice workspace; the counter is cleared here
int sites_args(plqcd_lattice *lat, long h0, long n, double *out, dev::SitesArgs *a) {
    const int nb = sites_grid(n);
    void *ws = nullptr;
    PLQCD_TRY(lattice_workspace(lat, sizeof(double) * kMaxRedBlocks + 256, &ws));
    a->Vh = lat->geom.Vh;
    a->h0 = h0;
    a->n = n;
    a->partials = static_cast<double *>(ws);
    a->counter = reinterpret_cast<unsigned *>(static_cast<char *>(ws) + sizeof(double) * kMaxRedBlocks);
    a->out = out;
    PLQCD_CUDA_TRY(cudaMemsetAsync(a->counter, 0, sizeof(unsigned), lat->stream));
    (void)nb;
    return PLQCD_OK;
}

int aligned8(const void *p, const char *who) {
    if (!p || (reinterpret_cast<uintptr_t>(p) & 7u)) return set_error(PLQCD_ERR_ARG, "%s: bad scalar pointer", who);
    return PLQCD_OK;
}

}  // namespace

}  // namespace plqcd

using namespace plqcd;

extern "C" int plqcd_sites_norm2(plqcd_lattice *lat, const void *x, long h_begin, long h_count, double *out_dev) {
    clear_error();
    PLQCD_TRY(sites_check(lat, h_begin, h_count, "plqcd_sites_norm2"));
    PLQCD_TRY(check_field_ptr(x, "plqcd_sites_norm2"));
    PLQCD_TRY(aligned8(out_dev, "plqcd_sites_norm2"));
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    dev::SitesArgs a;
    PLQCD_TRY(sites_args(lat, h_begin, h_count, out_dev, &a));
    dev::k_sites_norm2<<<sites_grid(h_count), kBlasBlock, 0, lat->stream>>>(x, a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

extern "C" int plqcd_sites_cg_update(plqcd_lattice *lat, void *x, void *r, const void *p, const void *Ap,
                                     long h_begin, long h_count, const double *coef_dev, double *rr_dev) {
    clear_error();
    PLQCD_TRY(sites_check(lat, h_begin, h_count, "plqcd_sites_cg_update"));
    for (const void *f : {(const void *)x, (const void *)r, p, Ap}) PLQCD_TRY(check_field_ptr(f, "plqcd_sites_cg_update"));
    PLQCD_TRY(aligned8(coef_dev, "plqcd_sites_cg_update"));
    PLQCD_TRY(aligned8(rr_dev, "plqcd_sites_cg_update"));
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    dev::SitesArgs a;
    PLQCD_TRY(sites_args(lat, h_begin, h_count, rr_dev, &a));
    dev::k_sites_cg_update<<<sites_grid(h_count), kBlasBlock, 0, lat->stream>>>(x, r, p, Ap, coef_dev, a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

extern "C" int plqcd_sites_xpay(plqcd_lattice *lat, void *p, const void *r, long h_begin, long h_count,
                                const double *coef_dev) {
    clear_error();
    PLQCD_TRY(sites_check(lat, h_begin, h_count, "plqcd_sites_xpay"));
    PLQCD_TRY(check_field_ptr(p, "plqcd_sites_xpay"));
    PLQCD_TRY(check_field_ptr(r, "plqcd_sites_xpay"));
    PLQCD_TRY(aligned8(coef_dev, "plqcd_sites_xpay"));
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    dev::k_sites_xpay<<<sites_grid(h_count), kBlasBlock, 0, lat->stream>>>(p, r, coef_dev, lat->geom.Vh, h_begin,
                                                                            h_count);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

extern "C" int plqcd_sites_sub_norm2(plqcd_lattice *lat, void *z, const void *x, const void *y, long h_begin,
                                     long h_count, double *out_dev) {
    clear_error();
    PLQCD_TRY(sites_check(lat, h_begin, h_count, "plqcd_sites_sub_norm2"));
    for (const void *f : {(const void *)z, x, y}) PLQCD_TRY(check_field_ptr(f, "plqcd_sites_sub_norm2"));
    PLQCD_TRY(aligned8(out_dev, "plqcd_sites_sub_norm2"));
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    dev::SitesArgs a;
    PLQCD_TRY(sites_args(lat, h_begin, h_count, out_dev, &a));
    dev::k_sites_sub_norm2<<<sites_grid(h_count), kBlasBlock, 0, lat->stream>>>(z, x, y, a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

extern "C" int plqcd_copy_segments(plqcd_lattice *lat, int n, void *const *dst, const void *const *src,
                                   const size_t *bytes) {
    clear_error();
    if (!lat || !dst || !src || !bytes || n < 0 || n > PLQCD_COPY_MAX_SEGMENTS)
        return set_error(PLQCD_ERR_ARG, "plqcd_copy_segments: bad argument (n = %d, at most %d segments)", n,
                         PLQCD_COPY_MAX_SEGMENTS);
    if (n == 0) return PLQCD_OK;
    dev::CopyTable t{};
    long most = 0;
    for (int k = 0; k < n; k++) {
        if ((reinterpret_cast<uintptr_t>(dst[k]) | reinterpret_cast<uintptr_t>(src[k]) | bytes[k]) & 15u)
            return set_error(PLQCD_ERR_ARG, "plqcd_copy_segments: segment %d is not 16-byte aligned", k);
        t.dst[k] = static_cast<uint4 *>(dst[k]);
        t.src[k] = static_cast<const uint4 *>(src[k]);
        t.n16[k] = (long)(bytes[k] / 16);
        if (t.n16[k] > most) most = t.n16[k];
    }
    if (most == 0) return PLQCD_OK;
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    const long bx = (most + 255) / 256;
    dim3 grid((unsigned)(bx < 592 ? bx : 592), (unsigned)n);
    dev::k_copy_segments<<<grid, 256, 0, lat->stream>>>(t);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}
