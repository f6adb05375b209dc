// fields.cu -- layout conversion and generation of device fields.
//
// API layout (include/su3.h): a spinor field is V spinors of 12 interleaved
// complex doubles in even/odd site order; a gauge field is 4V su3 links,
// link (i, mu) at u[4*i + mu] (lib/dirac.c:155, 262). The kernels here move
// between that array-of-structures layout and the structure-of-arrays
// layouts the hopping kernels read (include/plqcd_b200.h), in any storage
// precision, and generate random fields from a counter-based generator.
#include <cuda_runtime.h>

#include "device_fields.cuh"
#include "internal.h"
#include "philox.h"

namespace plqcd {
namespace dev {

constexpr int kBlock = 256;

inline unsigned nblocks(long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

template <typename R>
__device__ __forceinline__ void to_real(const cx<double> in[12], cx<R> out[12]) {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = {(R)in[k].re, (R)in[k].im};
}

// ---- spinors ------------------------------------------------------------------
template <int PREC>
__global__ void k_spinor_import(const double2 *__restrict__ aos, long Vh, int parity, void *dst, long first,
                                long count) {
    long h = first + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= first + count) return;
    const double2 *p = aos + (parity * Vh + h) * 12;
    cx<double> s[12];
#pragma unroll
    for (int k = 0; k < 12; k++) {
        double2 v = p[k];
        s[k] = {v.x, v.y};
    }
    using R = typename SpinorIO<PREC>::real;
    cx<R> r[12];
    to_real(s, r);
    SpinorIO<PREC>::store(dst, Vh, h, r);
}

template <int PREC>
__global__ void k_spinor_export(const void *src, long Vh, int parity, double2 *__restrict__ aos, long first,
                                long count) {
    long h = first + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= first + count) return;
    using R = typename SpinorIO<PREC>::real;
    cx<R> r[12];
    SpinorIO<PREC>::load(src, Vh, h, r);
    double2 *p = aos + (parity * Vh + h) * 12;
#pragma unroll
    for (int k = 0; k < 12; k++) p[k] = make_double2((double)r[k].re, (double)r[k].im);
}

// split real / imaginary planes: component k of staged site h at re[12*h+k]
template <int PREC>
__global__ void k_spinor_import_split(const double *__restrict__ re, const double *__restrict__ im, long Vh,
                                      void *dst) {
    long h = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= Vh) return;
    using R = typename SpinorIO<PREC>::real;
    cx<R> r[12];
#pragma unroll
    for (int k = 0; k < 12; k++) r[k] = {(R)re[12 * h + k], (R)im[12 * h + k]};
    SpinorIO<PREC>::store(dst, Vh, h, r);
}

template <int PREC>
__global__ void k_spinor_export_split(const void *src, long Vh, double *__restrict__ re, double *__restrict__ im) {
    long h = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= Vh) return;
    using R = typename SpinorIO<PREC>::real;
    cx<R> r[12];
    SpinorIO<PREC>::load(src, Vh, h, r);
#pragma unroll
    for (int k = 0; k < 12; k++) {
        re[12 * h + k] = (double)r[k].re;
        im[12 * h + k] = (double)r[k].im;
    }
}

template <int DP, int SP>
__global__ void k_spinor_convert(void *dst, const void *src, long Vh) {
    long h = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= Vh) return;
    using RS = typename SpinorIO<SP>::real;
    using RD = typename SpinorIO<DP>::real;
    cx<RS> s[12];
    SpinorIO<SP>::load(src, Vh, h, s);
    cx<RD> d[12];
#pragma unroll
    for (int k = 0; k < 12; k++) d[k] = {(RD)s[k].re, (RD)s[k].im};
    SpinorIO<DP>::store(dst, Vh, h, d);
}

template <int PREC>
__global__ void k_spinor_gaussian(void *dst, long Vh, int parity, uint64_t seed) {
    long h = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= Vh) return;
    const uint64_t site = (uint64_t)parity * Vh + h;
    cx<double> s[12];
#pragma unroll
    for (int k = 0; k < 12; k++) {
        double2 g = philox_gaussian_pair(seed, site, kTagSpinor, (uint32_t)k);
        s[k] = {g.x, g.y};
    }
    using R = typename SpinorIO<PREC>::real;
    cx<R> r[12];
    to_real(s, r);
    SpinorIO<PREC>::store(dst, Vh, h, r);
}

// ---- gauge --------------------------------------------------------------------
template <int PREC, int RECON>
__global__ void k_gauge_import(const double2 *__restrict__ aos, long first, long n, long Vh, void *dst) {
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    long l = first + k;  // global link index 4*i + mu
    long i = l >> 2;
    int mu = (int)(l & 3);
    int par = i >= Vh;
    long h = i - par * Vh;
    const double2 *p = aos + k * 9;
    cx<double> U[9];
#pragma unroll
    for (int e = 0; e < 9; e++) {
        double2 v = p[e];
        U[e] = {v.x, v.y};
    }
    LinkIO<PREC, RECON>::store(dst, Vh, par, mu, h, U);
}

// links from split planes: element e of staged link k at re[9*k+e]
template <int PREC, int RECON>
__global__ void k_gauge_import_split(const double *__restrict__ re, const double *__restrict__ im, long first,
                                     long n, long Vh, void *dst) {
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    long l = first + k;
    long i = l >> 2;
    int mu = (int)(l & 3);
    int par = i >= Vh;
    long h = i - par * Vh;
    cx<double> U[9];
#pragma unroll
    for (int e = 0; e < 9; e++) U[e] = {re[9 * k + e], im[9 * k + e]};
    LinkIO<PREC, RECON>::store(dst, Vh, par, mu, h, U);
}

template <int PREC, int RECON>
__global__ void k_gauge_export(const void *src, long Vh, double2 *__restrict__ aos) {
    long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 8 * Vh) return;
    long i = l >> 2;
    int mu = (int)(l & 3);
    int par = i >= Vh;
    long h = i - par * Vh;
    using R = typename LinkIO<PREC, RECON>::real;
    cx<R> U[9];
    LinkIO<PREC, RECON>::load(src, Vh, par, mu, h, U);
    double2 *p = aos + l * 9;
#pragma unroll
    for (int e = 0; e < 9; e++) p[e] = make_double2((double)U[e].re, (double)U[e].im);
}

// Random SU(3): Gaussian complex 3x3; rows 0,1 Gram-Schmidt orthonormalised;
// row 2 = conj(row0 x row1) (det = 1).
template <int PREC, int RECON>
__global__ void k_gauge_random(void *dst, long Vh, uint64_t seed) {
    long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 8 * Vh) return;
    long i = l >> 2;
    int mu = (int)(l & 3);
    int par = i >= Vh;
    long h = i - par * Vh;
    cx<double> U[9];
#pragma unroll
    for (int e = 0; e < 6; e++) {
        double2 g = philox_gaussian_pair(seed, (uint64_t)i, kTagGauge + mu, (uint32_t)e);
        U[e] = {g.x, g.y};
    }
    double n0 = 0;
#pragma unroll
    for (int b = 0; b < 3; b++) n0 += U[b].re * U[b].re + U[b].im * U[b].im;
    n0 = rsqrt(n0);
#pragma unroll
    for (int b = 0; b < 3; b++) U[b] = {U[b].re * n0, U[b].im * n0};
    cx<double> d = {0, 0};  // <row0, row1>
#pragma unroll
    for (int b = 0; b < 3; b++) d = cadd(d, conjmul(U[b], U[3 + b]));
#pragma unroll
    for (int b = 0; b < 3; b++) U[3 + b] = csub(U[3 + b], cmul(d, U[b]));
    double n1 = 0;
#pragma unroll
    for (int b = 0; b < 3; b++) n1 += U[3 + b].re * U[3 + b].re + U[3 + b].im * U[3 + b].im;
    n1 = rsqrt(n1);
#pragma unroll
    for (int b = 0; b < 3; b++) U[3 + b] = {U[3 + b].re * n1, U[3 + b].im * n1};
    reconstruct_row2(U);
    LinkIO<PREC, RECON>::store(dst, Vh, par, mu, h, U);
}

template <int PREC, int RECON>
__global__ void k_gauge_unit(void *dst, long Vh) {
    long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 8 * Vh) return;
    long i = l >> 2;
    int mu = (int)(l & 3);
    int par = i >= Vh;
    long h = i - par * Vh;
    cx<double> U[9];
#pragma unroll
    for (int e = 0; e < 9; e++) U[e] = {(e % 4 == 0) ? 1.0 : 0.0, 0.0};
    LinkIO<PREC, RECON>::store(dst, Vh, par, mu, h, U);
}

template <int DP, int DR, int SP, int SR>
__global__ void k_gauge_copy(void *dst, const void *src, long Vh) {
    long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 8 * Vh) return;
    long i = l >> 2;
    int mu = (int)(l & 3);
    int par = i >= Vh;
    long h = i - par * Vh;
    using R = typename LinkIO<SP, SR>::real;
    cx<R> U[9];
    LinkIO<SP, SR>::load(src, Vh, par, mu, h, U);
    cx<double> D[9];
#pragma unroll
    for (int e = 0; e < 9; e++) D[e] = {(double)U[e].re, (double)U[e].im};
    LinkIO<DP, DR>::store(dst, Vh, par, mu, h, D);
}

}  // namespace dev

// ---- dispatch helpers ------------------------------------------------------------

#define PLQCD_SPINOR_SWITCH(prec, F)                          \
    switch (prec) {                                           \
        case PLQCD_F64: F(PLQCD_F64); break;                  \
        case PLQCD_F32: F(PLQCD_F32); break;                  \
        case PLQCD_F16: F(PLQCD_F16); break;                  \
        case PLQCD_BF16: F(PLQCD_BF16); break;                \
        default: return set_error(PLQCD_ERR_ARG, "unknown spinor precision %d", prec); \
    }

#define PLQCD_GAUGE_SWITCH(prec, recon, F)                                       \
    switch ((prec) * 100 + (recon)) {                                            \
        case PLQCD_F64 * 100 + 18: F(PLQCD_F64, 18); break;                      \
        case PLQCD_F64 * 100 + 12: F(PLQCD_F64, 12); break;                      \
        case PLQCD_F32 * 100 + 18: F(PLQCD_F32, 18); break;                      \
        case PLQCD_F32 * 100 + 12: F(PLQCD_F32, 12); break;                      \
        case PLQCD_F16 * 100 + 12: F(PLQCD_F16, 12); break;                      \
        case PLQCD_BF16 * 100 + 12: F(PLQCD_BF16, 12); break;                    \
        default: return set_error(PLQCD_ERR_ARG, "unsupported gauge format %d/%d", prec, recon); \
    }

int launch_spinor_import(const Geom &g, cudaStream_t s, const void *aos, int parity, void *dst, int prec, long first,
                         long count) {
    PLQCD_TRY(check_field_ptr(aos, "spinor import (API layout)"));
    PLQCD_TRY(check_field_ptr(dst, "spinor import"));
    if (count < 0) count = g.Vh - first;
#define F(P) dev::k_spinor_import<P><<<dev::nblocks(count), dev::kBlock, 0, s>>>((const double2 *)aos, g.Vh, parity, dst, first, count)
    PLQCD_SPINOR_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_spinor_export(const Geom &g, cudaStream_t s, const void *src, int prec, int parity, void *aos, long first,
                         long count) {
    PLQCD_TRY(check_field_ptr(src, "spinor export"));
    PLQCD_TRY(check_field_ptr(aos, "spinor export (API layout)"));
    if (count < 0) count = g.Vh - first;
#define F(P) dev::k_spinor_export<P><<<dev::nblocks(count), dev::kBlock, 0, s>>>(src, g.Vh, parity, (double2 *)aos, first, count)
    PLQCD_SPINOR_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_spinor_import_split(const Geom &g, cudaStream_t s, const double *re, const double *im, void *dst,
                               int prec) {
#define F(P) dev::k_spinor_import_split<P><<<dev::nblocks(g.Vh), dev::kBlock, 0, s>>>(re, im, g.Vh, dst)
    PLQCD_SPINOR_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_spinor_export_split(const Geom &g, cudaStream_t s, const void *src, int prec, double *re, double *im) {
#define F(P) dev::k_spinor_export_split<P><<<dev::nblocks(g.Vh), dev::kBlock, 0, s>>>(src, g.Vh, re, im)
    PLQCD_SPINOR_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_gauge_import_split(const Geom &g, cudaStream_t s, const double *re, const double *im, long first, long n,
                              void *dst, int prec, int recon) {
#define F(P, R) dev::k_gauge_import_split<P, R><<<dev::nblocks(n), dev::kBlock, 0, s>>>(re, im, first, n, g.Vh, dst)
    PLQCD_GAUGE_SWITCH(prec, recon, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_spinor_convert(const Geom &g, cudaStream_t s, void *dst, int dprec, const void *src, int sprec) {
    PLQCD_TRY(check_field_ptr(dst, "spinor convert"));
    PLQCD_TRY(check_field_ptr(src, "spinor convert"));
#define G(DP, SP) dev::k_spinor_convert<DP, SP><<<dev::nblocks(g.Vh), dev::kBlock, 0, s>>>(dst, src, g.Vh)
#define F(DP)                                                  \
    switch (sprec) {                                           \
        case PLQCD_F64: G(DP, PLQCD_F64); break;               \
        case PLQCD_F32: G(DP, PLQCD_F32); break;               \
        case PLQCD_F16: G(DP, PLQCD_F16); break;               \
        case PLQCD_BF16: G(DP, PLQCD_BF16); break;             \
        default: return set_error(PLQCD_ERR_ARG, "unknown spinor precision %d", sprec); \
    }
    PLQCD_SPINOR_SWITCH(dprec, F)
#undef F
#undef G
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_spinor_gaussian(const Geom &g, cudaStream_t s, void *dst, int prec, int parity, uint64_t seed) {
    PLQCD_TRY(check_field_ptr(dst, "spinor gaussian"));
#define F(P) dev::k_spinor_gaussian<P><<<dev::nblocks(g.Vh), dev::kBlock, 0, s>>>(dst, g.Vh, parity, seed)
    PLQCD_SPINOR_SWITCH(prec, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_gauge_import(const Geom &g, cudaStream_t s, const void *aos, long first, long n, void *dst, int prec,
                        int recon) {
    PLQCD_TRY(check_field_ptr(aos, "gauge import (API layout)"));
#define F(P, R) dev::k_gauge_import<P, R><<<dev::nblocks(n), dev::kBlock, 0, s>>>((const double2 *)aos, first, n, g.Vh, dst)
    PLQCD_GAUGE_SWITCH(prec, recon, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_gauge_export(const Geom &g, cudaStream_t s, const void *src, int prec, int recon, void *aos) {
#define F(P, R) dev::k_gauge_export<P, R><<<dev::nblocks(8 * g.Vh), dev::kBlock, 0, s>>>(src, g.Vh, (double2 *)aos)
    PLQCD_GAUGE_SWITCH(prec, recon, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_gauge_random(const Geom &g, cudaStream_t s, void *dst, int prec, int recon, uint64_t seed) {
#define F(P, R) dev::k_gauge_random<P, R><<<dev::nblocks(8 * g.Vh), dev::kBlock, 0, s>>>(dst, g.Vh, seed)
    PLQCD_GAUGE_SWITCH(prec, recon, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_gauge_unit(const Geom &g, cudaStream_t s, void *dst, int prec, int recon) {
#define F(P, R) dev::k_gauge_unit<P, R><<<dev::nblocks(8 * g.Vh), dev::kBlock, 0, s>>>(dst, g.Vh)
    PLQCD_GAUGE_SWITCH(prec, recon, F)
#undef F
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_gauge_copy(const Geom &g, cudaStream_t s, void *dst, int dprec, int drecon, const void *src, int sprec,
                      int srecon) {
#define G(DP, DR, SP, SR) dev::k_gauge_copy<DP, DR, SP, SR><<<dev::nblocks(8 * g.Vh), dev::kBlock, 0, s>>>(dst, src, g.Vh)
#define F(SP, SR)                                                                    \
    switch (dprec * 100 + drecon) {                                                  \
        case PLQCD_F64 * 100 + 18: G(PLQCD_F64, 18, SP, SR); break;                  \
        case PLQCD_F64 * 100 + 12: G(PLQCD_F64, 12, SP, SR); break;                  \
        case PLQCD_F32 * 100 + 18: G(PLQCD_F32, 18, SP, SR); break;                  \
        case PLQCD_F32 * 100 + 12: G(PLQCD_F32, 12, SP, SR); break;                  \
        case PLQCD_F16 * 100 + 12: G(PLQCD_F16, 12, SP, SR); break;                  \
        case PLQCD_BF16 * 100 + 12: G(PLQCD_BF16, 12, SP, SR); break;                \
        default: return set_error(PLQCD_ERR_ARG, "unsupported gauge format %d/%d", dprec, drecon); \
    }
    PLQCD_GAUGE_SWITCH(sprec, srecon, F)
#undef F
#undef G
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

// ---- sizes -------------------------------------------------------------------------
size_t spinor_parity_bytes(long Vh, int prec) {
    switch (prec) {
        case PLQCD_F64: return (size_t)Vh * 192;
        case PLQCD_F32: return (size_t)Vh * 96;
        case PLQCD_F16:
        case PLQCD_BF16: return (size_t)Vh * 52;
        default: return 0;
    }
}

bool gauge_format_ok(int prec, int recon) {
    if (prec == PLQCD_F64 || prec == PLQCD_F32) return recon == 18 || recon == 12;
    if (prec == PLQCD_F16 || prec == PLQCD_BF16) return recon == 12;
    return false;
}

size_t gauge_elem_bytes(int prec, int recon) {
    if (prec == PLQCD_F64) return 16;
    if (prec == PLQCD_F32) return recon == 18 ? 8 : 16;
    return 8;
}

int gauge_elems(int prec, int recon) {
    if (prec == PLQCD_F64) return recon == 18 ? 9 : 6;
    if (prec == PLQCD_F32) return recon == 18 ? 9 : 3;
    return 3;
}

size_t gauge_total_bytes(long Vh, int prec, int recon) {
    if (!gauge_format_ok(prec, recon)) return 0;
    return (size_t)8 * Vh * gauge_elems(prec, recon) * gauge_elem_bytes(prec, recon);
}

}  // namespace plqcd
