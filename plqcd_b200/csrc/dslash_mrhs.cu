// dslash_mrhs.cu -- hopping matrix on a block of right-hand sides.
//
// Kernel families (the tuner times them per format, lattice and RHS count):
// - RHS tiles: one thread handles one output site for a tile of NR RHS; per
//   direction it loads the link once and applies it to the NR neighbour
//   spinors (direct loads, or a cp.async ring);
// - RHS pairs (FP32, F16, BF16): two RHS on the two lanes of packed FP32
//   instructions, the link loaded, rebuilt and broadcast once per pair;
//   their xpay form can carry the CG's dot products in its epilogue
//   (RhsSink, for the batched solver);
// - FP64 link sharing: a block of RHS warps over 32 sites reads each link
//   from shared memory;
// - the single-RHS kernels with the RHS index folded into the grid
//   (dslash.cu), and the tensor-core kernel (dslash_mrhs_tc.cu).
// Consecutive blocks cover the RHS tiles of the same sites (tile index
// fastest), so the other tiles find the links in L2 and the link traffic per
// launch is paid once for all nrhs right-hand sides: bytes per site and RHS =
// 2 * spinor + 8 * link / nrhs. The per-direction arithmetic is that of the
// single-RHS kernel (dslash_core.cuh), and every family gives the same bits.
//
// A block of fields is nrhs one-parity fields back to back (field r at
// base + r * field_bytes).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "dslash_core.cuh"
#include "internal.h"
#include "tune.h"

namespace plqcd {
namespace dev {

struct MrhsArgs {
    const void *gauge;
    const char *in;
    char *out;
    const char *x;
    size_t fbytes;
    int nrhs, ntiles;
    long Vh;
    int L0, L0h, L1, L2, L3;
    int out_parity;
    double a_up, a_low, b, g5_in;
    RhsSink sink;  // fused CG sums (RHS-pair kernels, epi > 0)
};

template <class SIO, class LIO, int NR, bool XPAY>
__global__ void __launch_bounds__(256) k_dslash_mrhs(const MrhsArgs a) {
    using R = typename SIO::real;
    const int tile = blockIdx.x % a.ntiles;
    const long h = (long)(blockIdx.x / a.ntiles) * blockDim.x + threadIdx.x;
    if (h >= a.Vh) return;
    const int r0 = tile * NR;
    const int nr = min(NR, a.nrhs - r0);
    const int par = a.out_parity, opp = par ^ 1;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(h, par, L0h, L1, L2);
    const int xh = (int)(h - c.row * L0h);
    int nb[8];
    neighbour_sites(c, xh, a.L0, L0h, L1, L2, L3, nb);
    const R sg = (R)a.g5_in;

    cx<R> acc[NR][12];
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int k = 0; k < 12; k++) acc[r][k] = {R(0), R(0)};

#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int d = dir_at(k);
        cx<R> U[9];
        if (d < 4)
            LIO::load(a.gauge, Vh, par, d, h, U);
        else
            LIO::load(a.gauge, Vh, opp, d - 4, nb[d], U);
#pragma unroll
        for (int r = 0; r < NR; r++) {
            if (r < nr) {
                cx<R> s[12];
                R n;
                SIO::load_raw(a.in + (size_t)(r0 + r) * a.fbytes, Vh, nb[d], s, n);
                compute_dir_n<false, SIO::kScaled, R>(d, acc[r], s, U, sg, n);
            }
        }
    }

    const R aup = (R)a.a_up, alow = (R)a.a_low, b = (R)a.b;
#pragma unroll
    for (int r = 0; r < NR; r++) {
        if (r >= nr) continue;
        if (XPAY) {
            cx<R> xv[12];
            SIO::load(a.x + (size_t)(r0 + r) * a.fbytes, Vh, h, xv);
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const R ak = k < 6 ? aup : alow;
                acc[r][k] = {fma(ak, acc[r][k].re, b * xv[k].re), fma(ak, acc[r][k].im, b * xv[k].im)};
            }
        } else {
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const R ak = k < 6 ? aup : alow;
                acc[r][k] = {ak * acc[r][k].re, ak * acc[r][k].im};
            }
        }
        SIO::store(a.out + (size_t)(r0 + r) * a.fbytes, Vh, h, acc[r]);
    }
}

// Pipelined RHS-tile kernel: per direction the link and the NR neighbour
// spinors are copied global->shared with cp.async into slots private to the
// thread, ST directions ahead of the one being computed (no block-level
// synchronisation). The link crosses L2->SM once per tile and the copies
// stay in flight without holding registers.
template <class SIO, class LIO, int NR, int ST, bool XPAY>
__global__ void __launch_bounds__(256) k_dslash_mrhs_pipe(const MrhsArgs a) {
    using R = typename SIO::real;
    extern __shared__ uint4 smem[];
    constexpr int NS = LIO::NSLOT + NR * SIO::NSLOT;
    const int B = blockDim.x;
    const int tile = blockIdx.x % a.ntiles;
    const long h = (long)(blockIdx.x / a.ntiles) * B + threadIdx.x;
    if (h >= a.Vh) return;  // no block-level barrier below
    const int r0 = tile * NR;
    const int nr = min(NR, a.nrhs - r0);
    const int par = a.out_parity, opp = par ^ 1;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(h, par, L0h, L1, L2);
    const int xh = (int)(h - c.row * L0h);
    int nb[8];
    neighbour_sites(c, xh, a.L0, L0h, L1, L2, L3, nb);
    const R sg = (R)a.g5_in;

    const int stride = B * 16;
    const uint32_t s_thread = smem_addr(smem) + threadIdx.x * 16;
    // k-th direction of dir_at into slot k % ST
    auto issue = [&](int k) {
        const int d = dir_at(k);
        const uint32_t s0 = s_thread + (uint32_t)((k % ST) * NS) * stride;
        if (d < 4)
            LIO::issue(a.gauge, Vh, par, d, h, s0, stride);
        else
            LIO::issue(a.gauge, Vh, opp, d - 4, nb[d], s0, stride);
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (r < nr)
                SIO::issue(a.in + (size_t)(r0 + r) * a.fbytes, Vh, nb[d],
                           s0 + (uint32_t)(LIO::NSLOT + r * SIO::NSLOT) * stride, stride);
    };
#pragma unroll
    for (int k = 0; k < ST; k++) {
        issue(k);
        cp_async_commit();
    }
    cx<R> acc[NR][12];
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int k = 0; k < 12; k++) acc[r][k] = {R(0), R(0)};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int d = dir_at(k);
        cp_async_wait<ST - 1>();
        const uint4 *s0 = smem + threadIdx.x + (k % ST) * NS * B;
        cx<R> U[9];
        LIO::load_staged(s0, B, U);
#pragma unroll
        for (int r = 0; r < NR; r++) {
            if (r < nr) {
                cx<R> s[12];
                R n;
                SIO::load_staged_raw(s0 + (LIO::NSLOT + r * SIO::NSLOT) * B, B, s, n);
                compute_dir_n<false, SIO::kScaled, R>(d, acc[r], s, U, sg, n);
            }
        }
        // the slot just consumed is refilled only after its values were used
        if (k + ST < 8) issue(k + ST);
        cp_async_commit();
    }

    const R aup = (R)a.a_up, alow = (R)a.a_low, b = (R)a.b;
#pragma unroll
    for (int r = 0; r < NR; r++) {
        if (r >= nr) continue;
        if (XPAY) {
            cx<R> xv[12];
            SIO::load(a.x + (size_t)(r0 + r) * a.fbytes, Vh, h, xv);
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const R ak = k < 6 ? aup : alow;
                acc[r][k] = {fma(ak, acc[r][k].re, b * xv[k].re), fma(ak, acc[r][k].im, b * xv[k].im)};
            }
        } else {
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const R ak = k < 6 ? aup : alow;
                acc[r][k] = {ak * acc[r][k].re, ak * acc[r][k].im};
            }
        }
        SIO::store(a.out + (size_t)(r0 + r) * a.fbytes, Vh, h, acc[r]);
    }
}

__device__ __forceinline__ double sq_sum(const cx<float> v[12]) {
    double s = 0;
#pragma unroll
    for (int k = 0; k < 12; k++) s += (double)v[k].re * v[k].re + (double)v[k].im * v[k].im;
    return s;
}

// the block's per-RHS sums v0 (RHS r0) and v1 (r0 + 1) into the partials
// [RHS][site block]; k_sink_finish adds them up
__device__ void sink_block(const MrhsArgs &a, int r0, bool two, double v0, double v1) {
    __shared__ double ws[2][8];
    const int nsb = gridDim.x / a.ntiles, sb = blockIdx.x / a.ntiles;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    }
    if (lane == 0) {
        ws[0][w] = v0;
        ws[1][w] = v1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b0 = 0, b1 = 0;
        for (int i = 0; i < nw; i++) {
            b0 += ws[0][i];
            b1 += ws[1][i];
        }
        a.sink.partials[(size_t)r0 * nsb + sb] = b0;
        if (two) a.sink.partials[(size_t)(r0 + 1) * nsb + sb] = b1;
    }
}

// one block per RHS: the sum of its nsb partials in a fixed order (thread
// i takes i, i + blockDim, ..., then a fixed tree), applied to the solver's
// scalars of an active RHS (see RhsSink)
template <int EPI>
__global__ void __launch_bounds__(1024) k_sink_finish(const RhsSink k, int nsb) {
    __shared__ double ws[32];
    const int f = blockIdx.x;
    const double *p = k.partials + (size_t)f * nsb;
    double t = 0;
    for (int i = threadIdx.x; i < nsb; i += blockDim.x) t += p[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x != 0 || !k.active[f]) return;
    double tot = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) tot += ws[i];
    if (EPI == 1) {
        k.pAp[f] = tot;
        k.alpha[f] = tot > 0 ? k.rr[f] / tot : 0.0;
    } else if (EPI == 2) {
        k.rr_old[f] = k.rr[f];
        k.rr[f] = tot;
        k.beta[f] = k.rr_old[f] > 0 ? tot / k.rr_old[f] : 0.0;
    } else {  // 3: the restart residual of a reliable update
        k.rr[f] = tot;
        k.beta[f] = k.rr_old[f] > 0 ? tot / k.rr_old[f] : 0.0;
    }
}

// epilogue of the RHS-pair kernels: scale (and xpay with x from xload(j,
// xv)), then EPI 0 / 1: store (1: |out|^2 to the sink); EPI 2: r -= alpha
// out in place, |r|^2 to the sink (out is not stored). Threads past the last
// site (valid false) only take part in the sums.
template <class SIO, bool XPAY, int EPI, class XLoad>
__device__ __forceinline__ void pair_epilogue(const MrhsArgs &a, int r0, bool two, int h, bool valid,
                                              const cx<f2> acc[12], XLoad xload) {
    const float aup = (float)a.a_up, alow = (float)a.a_low, b = (float)a.b;
    double v[2] = {0.0, 0.0};
#pragma unroll
    for (int j = 0; j < 2; j++) {
        if ((j == 1 && !two) || !valid) break;
        cx<float> o[12];
#pragma unroll
        for (int k = 0; k < 12; k++) o[k] = lane(acc[k], j);
        if (XPAY) {
            cx<float> xv[12];
            xload(j, xv);
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const float ak = k < 6 ? aup : alow;
                o[k] = {fmaf(ak, o[k].re, b * xv[k].re), fmaf(ak, o[k].im, b * xv[k].im)};
            }
        } else {
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const float ak = k < 6 ? aup : alow;
                o[k] = {ak * o[k].re, ak * o[k].im};
            }
        }
        if (EPI == 2) {
            const int f = r0 + j;
            if (a.sink.active[f]) {
                const float al = (float)a.sink.alpha[f];
                char *rf = a.sink.rvec + (size_t)f * a.fbytes;
                cx<float> rv[12];
                SIO::load(rf, a.Vh, h, rv);
#pragma unroll
                for (int k = 0; k < 12; k++) rv[k] = {fmaf(-al, o[k].re, rv[k].re), fmaf(-al, o[k].im, rv[k].im)};
                SIO::store(rf, a.Vh, h, rv);
                v[j] = sq_sum(rv);
            }
        } else {
            SIO::store(a.out + (size_t)(r0 + j) * a.fbytes, a.Vh, h, o);
            if (EPI == 1 || EPI == 3) v[j] = sq_sum(o);
        }
    }
    if (EPI > 0 && EPI < 4) sink_block(a, r0, two, v[0], v[1]);
}

// RHS-pair kernel: one thread, one output site, two right-hand sides on the
// two lanes of Blackwell's packed FP32 instructions (FFMA2 / FMUL2 / FADD2):
// lane 0 carries RHS r0, lane 1 RHS r0 + 1. The link is loaded, converted,
// rebuilt and broadcast to both lanes once per pair, and every arithmetic
// instruction serves both RHS. Each lane runs the scalar sequence of
// compute_dir with the same rounding, so the results are the bits of the
// other kernels. An odd last RHS runs in both lanes and is stored once.
// (FP32-computing formats: F32, F16, BF16.)
template <class SIO, class LIO, bool XPAY, int MINB = 1, int EPI = 0>
__global__ void __launch_bounds__(256, MINB) k_dslash_mrhs_pair(const MrhsArgs a) {
    static_assert(std::is_same<typename SIO::real, float>::value, "packed lanes hold FP32");
    const int tile = blockIdx.x % a.ntiles;
    const int hh = (blockIdx.x / a.ntiles) * blockDim.x + threadIdx.x;
    const bool valid = hh < a.Vh;
    if ((EPI == 0 || EPI == 4) && !valid) return;  // (EPI 1-3: every thread takes part in the sums)
    const int h = valid ? hh : (int)a.Vh - 1;
    const int r0 = 2 * tile;
    // restart hops (EPI 3, 4): a pair of retired RHS has nothing to compute (whole block)
    if (EPI >= 3 && !a.sink.active[r0] && !(r0 + 1 < a.nrhs && a.sink.active[r0 + 1])) return;
    const bool two = r0 + 1 < a.nrhs;
    const char *in0 = a.in + (size_t)r0 * a.fbytes;
    const char *in1 = two ? in0 + a.fbytes : in0;
    const int par = a.out_parity, opp = par ^ 1;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(h, par, L0h, L1, L2);
    const int xh = h - c.row * L0h;
    int nb[8];
    neighbour_sites(c, xh, a.L0, L0h, L1, L2, L3, nb);
    const f2 sg((float)a.g5_in);

    cx<f2> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = {f2(0.f), f2(0.f)};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int d = dir_at(k);
        cx<float> U[9];
        if (d < 4)
            LIO::load(a.gauge, Vh, par, d, h, U);
        else
            LIO::load(a.gauge, Vh, opp, d - 4, nb[d], U);
        cx<f2> Ub[9];
#pragma unroll
        for (int e = 0; e < 9; e++) Ub[e] = {f2(U[e].re), f2(U[e].im)};
        cx<float> sa[12], sb[12];
        float na, nbv;
        SIO::load_raw(in0, Vh, nb[d], sa, na);
        SIO::load_raw(in1, Vh, nb[d], sb, nbv);
        cx<f2> s[12];
#pragma unroll
        for (int e = 0; e < 12; e++) s[e] = zip(sa[e], sb[e]);
        compute_dir_n<false, SIO::kScaled, f2>(d, acc, s, Ub, sg, f2(na, nbv));
    }
    pair_epilogue<SIO, XPAY, EPI>(a, r0, two, h, valid, acc, [&](int j, cx<float> xv[12]) {
        SIO::load(a.x + (size_t)(r0 + j) * a.fbytes, Vh, h, xv);
    });
}

// Pipelined RHS-pair kernel: the link and the two neighbour spinors of a
// direction are copied global->shared with cp.async into slots private to
// the thread, ST directions ahead of the one being computed (as in
// k_dslash_mrhs_pipe), so the loads stay in flight without holding the
// registers the packed arithmetic needs.
template <class SIO, class LIO, int ST, bool XPAY, int MINB = 1, int EPI = 0>
__global__ void __launch_bounds__(256, MINB) k_dslash_mrhs_pair_pipe(const MrhsArgs a) {
    static_assert(std::is_same<typename SIO::real, float>::value, "packed lanes hold FP32");
    extern __shared__ uint4 smem[];
    constexpr int NS = LIO::NSLOT + 2 * SIO::NSLOT;
    const int B = blockDim.x;
    const int tile = blockIdx.x % a.ntiles;
    const int hh = (blockIdx.x / a.ntiles) * B + threadIdx.x;
    const bool valid = hh < a.Vh;
    // no block-level barrier below except the sums of EPI 1-3, in which
    // every thread (a past-the-end one on the last site) takes part
    if ((EPI == 0 || EPI == 4) && !valid) return;
    const int h = valid ? hh : (int)a.Vh - 1;
    // restart hops (EPI 3, 4): a pair of retired RHS has nothing to compute (whole block)
    if (EPI >= 3 && !a.sink.active[2 * tile] && !(2 * tile + 1 < a.nrhs && a.sink.active[2 * tile + 1])) return;
    const int r0 = 2 * tile;
    const bool two = r0 + 1 < a.nrhs;
    const char *in0 = a.in + (size_t)r0 * a.fbytes;
    const char *in1 = two ? in0 + a.fbytes : in0;
    const int par = a.out_parity, opp = par ^ 1;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(h, par, L0h, L1, L2);
    const int xh = h - c.row * L0h;
    int nb[8];
    neighbour_sites(c, xh, a.L0, L0h, L1, L2, L3, nb);
    const f2 sg((float)a.g5_in);

    const int stride = B * 16;
    const uint32_t s_thread = smem_addr(smem) + threadIdx.x * 16;
    // k-th direction of dir_at into slot k % ST: link, then RHS r0, r0 + 1
    auto issue = [&](int k) {
        const int d = dir_at(k);
        const uint32_t s0 = s_thread + (uint32_t)((k % ST) * NS) * stride;
        if (d < 4)
            LIO::issue(a.gauge, Vh, par, d, h, s0, stride);
        else
            LIO::issue(a.gauge, Vh, opp, d - 4, nb[d], s0, stride);
        SIO::issue(in0, Vh, nb[d], s0 + (uint32_t)LIO::NSLOT * stride, stride);
        SIO::issue(in1, Vh, nb[d], s0 + (uint32_t)(LIO::NSLOT + SIO::NSLOT) * stride, stride);
    };
    // xpay: the two x spinors of the output site go in with the first
    // direction, into slots after the ring, so the epilogue does not wait
    const uint32_t s_x = s_thread + (uint32_t)(ST * NS) * stride;
#pragma unroll
    for (int k = 0; k < ST; k++) {
        issue(k);
        if (XPAY && k == 0) {
            SIO::issue(a.x + (size_t)r0 * a.fbytes, Vh, h, s_x, stride);
            SIO::issue(a.x + (size_t)(two ? r0 + 1 : r0) * a.fbytes, Vh, h, s_x + SIO::NSLOT * stride, stride);
        }
        cp_async_commit();
    }
    cx<f2> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = {f2(0.f), f2(0.f)};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int d = dir_at(k);
        cp_async_wait<ST - 1>();
        const uint4 *s0 = smem + threadIdx.x + (k % ST) * NS * B;
        cx<float> U[9];
        LIO::load_staged(s0, B, U);
        cx<f2> Ub[9];
#pragma unroll
        for (int e = 0; e < 9; e++) Ub[e] = {f2(U[e].re), f2(U[e].im)};
        cx<float> sa[12], sb[12];
        float na, nbv;
        SIO::load_staged_raw(s0 + LIO::NSLOT * B, B, sa, na);
        SIO::load_staged_raw(s0 + (LIO::NSLOT + SIO::NSLOT) * B, B, sb, nbv);
        cx<f2> s[12];
#pragma unroll
        for (int e = 0; e < 12; e++) s[e] = zip(sa[e], sb[e]);
        compute_dir_n<false, SIO::kScaled, f2>(d, acc, s, Ub, sg, f2(na, nbv));
        // the slot just consumed is refilled only after its values were used
        if (k + ST < 8) issue(k + ST);
        cp_async_commit();
    }
    pair_epilogue<SIO, XPAY, EPI>(a, r0, two, h, valid, acc, [&](int j, cx<float> xv[12]) {
        SIO::load_staged(smem + threadIdx.x + (ST * NS + j * SIO::NSLOT) * B, B, xv);
    });
}

// ST = 0: direct loads (k_dslash_mrhs_pair), else the cp.async pipeline of
// depth ST; MINB = 2 caps the registers at 128 a thread (more warps per SM)
// epi > 0 (fused CG sums, xpay hops only): see RhsSink
template <class SIO, class LIO, int ST, int MINB = 1>
static int launch_pair(const Geom &g, cudaStream_t s, MrhsArgs a, int block, bool xpay, int epi = 0) {
    if constexpr (!std::is_same<typename SIO::real, float>::value) {
        return set_error(PLQCD_ERR_ARG, "dslash_mrhs: the RHS-pair kernel computes in FP32 only");
    } else {
        if (g.Vh >= (1L << 31)) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: lattice too large for 32-bit sites");
        if (epi && ((epi == 4) == xpay || block > 256 || block % 32))
            return set_error(PLQCD_ERR_ARG, "dslash_mrhs: fused epilogue %d does not fit this hop", epi);
        a.ntiles = (a.nrhs + 1) / 2;
        const long nblk = (g.Vh + block - 1) / block * a.ntiles;
        if (nblk > 0x7fffffffL) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: grid too large");
        if constexpr (ST == 0) {
            auto k = epi == 4 ? k_dslash_mrhs_pair<SIO, LIO, false, MINB, 4>
                   : epi == 3 ? k_dslash_mrhs_pair<SIO, LIO, true, MINB, 3>
                   : epi == 2 ? k_dslash_mrhs_pair<SIO, LIO, true, MINB, 2>
                   : epi == 1 ? k_dslash_mrhs_pair<SIO, LIO, true, MINB, 1>
                   : xpay     ? k_dslash_mrhs_pair<SIO, LIO, true, MINB, 0>
                              : k_dslash_mrhs_pair<SIO, LIO, false, MINB, 0>;
            k<<<(unsigned)nblk, block, 0, s>>>(a);
        } else {
            constexpr int NS = LIO::NSLOT + 2 * SIO::NSLOT;
            const size_t smem = (size_t)(ST * NS + (xpay ? 2 * SIO::NSLOT : 0)) * 16 * block;
            if (smem > 227 * 1024) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: %zu bytes of shared memory", smem);
            auto k = epi == 4 ? k_dslash_mrhs_pair_pipe<SIO, LIO, ST, false, MINB, 4>
                   : epi == 3 ? k_dslash_mrhs_pair_pipe<SIO, LIO, ST, true, MINB, 3>
                   : epi == 2 ? k_dslash_mrhs_pair_pipe<SIO, LIO, ST, true, MINB, 2>
                   : epi == 1 ? k_dslash_mrhs_pair_pipe<SIO, LIO, ST, true, MINB, 1>
                   : xpay     ? k_dslash_mrhs_pair_pipe<SIO, LIO, ST, true, MINB, 0>
                              : k_dslash_mrhs_pair_pipe<SIO, LIO, ST, false, MINB, 0>;
            // (the fused sums hold static shared memory, so opt in to what this launch needs)
            PLQCD_TRY(smem_optin((const void *)k, smem));
            k<<<(unsigned)nblk, block, smem, s>>>(a);
        }
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
}

// FP64 link-sharing kernel: a block of NRB warps covers 32 consecutive
// output sites for NRB right-hand sides (warp w = RHS w of the block's
// group, lane = site). Per direction the block copies the links of its 32
// sites into shared memory once (cp.async, each warp a share of the
// planes) and every warp copies its own neighbour spinors; all NRB warps
// then read the links from shared memory. A link crosses L2->SM once per
// NRB RHS instead of once per RHS, which is what bounds the FP64 multi-RHS
// hop when each RHS is a separate block. The ring holds ST directions with
// one block barrier per direction: stage k + ST - 1 is refilled into the
// slot of stage k - 1 after the barrier that every warp passes once it has
// computed k - 1. Threads past the last site or RHS copy in-bounds data and
// store nothing. Same arithmetic, so the same bits, as the other kernels.
template <class LIO, int NRB, int ST, bool XPAY>
__global__ void __launch_bounds__(32 * NRB) k_dslash_mrhs_f64blk(const MrhsArgs a) {
    using SIO = SpinorIO<PLQCD_F64>;
    constexpr int NT = 32 * NRB;
    constexpr int LP = LIO::NE;            // link planes, 16 bytes a site each
    constexpr int LB = LP * 32;            // link slots of the block's sites
    constexpr int STAGE = LB + SIO::NSLOT * NT;
    extern __shared__ uint4 smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int grp = blockIdx.x % a.ntiles;
    const int h0 = (blockIdx.x / a.ntiles) * 32;
    const int r = grp * NRB + w;
    const bool rhs_ok = r < a.nrhs;
    const int h = h0 + lane;
    const bool site_ok = h < a.Vh;
    const int hc = site_ok ? h : h0;  // h0 < Vh: out-of-range lanes copy a valid site
    const char *in = a.in + (size_t)(rhs_ok ? r : 0) * a.fbytes;
    const int par = a.out_parity, opp = par ^ 1;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(hc, par, L0h, L1, L2);
    const int xh = hc - c.row * L0h;
    int nb[8];
    neighbour_sites(c, xh, a.L0, L0h, L1, L2, L3, nb);
    const double sg = a.g5_in;

    const uint32_t base = smem_addr(smem);
    // direction k of dir_at into ring slot k % ST: link planes e = w, w + NRB,
    // ... of site lane (the link of the lane's own site, or of its backward
    // neighbour), then this thread's neighbour spinor
    auto issue = [&](int k) {
        const int d = dir_at(k);
        const uint32_t st = base + (uint32_t)((k % ST) * STAGE) * 16u;
        const int lsite = d < 4 ? hc : nb[d];
        const int lpar = d < 4 ? par : opp;
        const double2 *lp = static_cast<const double2 *>(a.gauge) + ((long)(lpar * 4 + (d & 3)) * LP) * Vh + lsite;
#pragma unroll
        for (int e = w; e < LP; e += NRB) cp_async16_cg(st + (uint32_t)(e * 32 + lane) * 16u, lp + e * Vh);
        SIO::issue(in, Vh, nb[d], st + (uint32_t)(LB + threadIdx.x) * 16u, NT * 16);
    };
#pragma unroll
    for (int k = 0; k < ST - 1; k++) {
        issue(k);
        cp_async_commit();
    }
    cx<double> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        cp_async_wait<ST - 2>();  // this thread's copies of stage k
        __syncthreads();          // everyone's copies of stage k; everyone done with k - 1
        if (k + ST - 1 < 8) issue(k + ST - 1);
        cp_async_commit();
        const uint4 *stg = smem + (k % ST) * STAGE;
        cx<double> U[9], s[12];
        double n;
        LIO::load_staged(stg + lane, 32, U);
        SIO::load_staged_raw(stg + LB + threadIdx.x, NT, s, n);
        compute_dir_n<false, false, double>(dir_at(k), acc, s, U, sg, n);
    }
    if (!site_ok || !rhs_ok) return;
    const double aup = a.a_up, alow = a.a_low;
    if (XPAY) {
        cx<double> xv[12];
        SIO::load(a.x + (size_t)r * a.fbytes, Vh, h, xv);
        const double b = a.b;
#pragma unroll
        for (int k = 0; k < 12; k++) {
            const double ak = k < 6 ? aup : alow;
            acc[k] = {fma(ak, acc[k].re, b * xv[k].re), fma(ak, acc[k].im, b * xv[k].im)};
        }
    } else {
#pragma unroll
        for (int k = 6; k < 12; k++) acc[k] = {alow * acc[k].re, alow * acc[k].im};
#pragma unroll
        for (int k = 0; k < 6; k++) acc[k] = {aup * acc[k].re, aup * acc[k].im};
    }
    SIO::store(a.out + (size_t)r * a.fbytes, Vh, h, acc);
}

template <class LIO, int NRB, int ST>
static int launch_f64blk(const Geom &g, cudaStream_t s, MrhsArgs a, bool xpay) {
    if (g.Vh >= (1L << 31)) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: lattice too large for 32-bit sites");
    a.ntiles = (a.nrhs + NRB - 1) / NRB;
    const long nblk = (g.Vh + 31) / 32 * a.ntiles;
    if (nblk > 0x7fffffffL) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: grid too large");
    constexpr int STAGE = LIO::NE * 32 + SpinorIO<PLQCD_F64>::NSLOT * 32 * NRB;
    const size_t smem = (size_t)ST * STAGE * 16;
    if (smem > 227 * 1024) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: %zu bytes of shared memory", smem);
    auto k = xpay ? k_dslash_mrhs_f64blk<LIO, NRB, ST, true> : k_dslash_mrhs_f64blk<LIO, NRB, ST, false>;
    PLQCD_TRY(smem_optin((const void *)k, 227 * 1024));
    k<<<(unsigned)nblk, 32 * NRB, smem, s>>>(a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

template <class SIO, class LIO, int NR, int ST>
static int launch_nr_pipe(const Geom &g, cudaStream_t s, MrhsArgs a, int block, bool xpay) {
    a.ntiles = (a.nrhs + NR - 1) / NR;
    const long nblk = (g.Vh + block - 1) / block * a.ntiles;
    if (nblk > 0x7fffffffL) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: grid too large");
    constexpr int NS = LIO::NSLOT + NR * SIO::NSLOT;
    const size_t smem = (size_t)ST * NS * 16 * block;
    if (smem > 227 * 1024) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: %zu bytes of shared memory", smem);
    auto k = xpay ? k_dslash_mrhs_pipe<SIO, LIO, NR, ST, true> : k_dslash_mrhs_pipe<SIO, LIO, NR, ST, false>;
    PLQCD_TRY(smem_optin((const void *)k, 227 * 1024));
    k<<<(unsigned)nblk, block, smem, s>>>(a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

template <class SIO, class LIO, int NR>
static int launch_nr(const Geom &g, cudaStream_t s, MrhsArgs a, int block, bool xpay) {
    a.ntiles = (a.nrhs + NR - 1) / NR;
    const long nsb = (g.Vh + block - 1) / block;
    const long nblk = nsb * a.ntiles;
    if (nblk > 0x7fffffffL) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: grid too large");
    if (xpay)
        k_dslash_mrhs<SIO, LIO, NR, true><<<(unsigned)nblk, block, 0, s>>>(a);
    else
        k_dslash_mrhs<SIO, LIO, NR, false><<<(unsigned)nblk, block, 0, s>>>(a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

template <int P, int RC>
static int launch_pr(const Geom &g, cudaStream_t s, const MrhsArgs &a, int nr, int block, bool xpay, int epi) {
    if (epi && (nr < 2000 || nr >= 3000))
        return set_error(PLQCD_ERR_ARG, "dslash_mrhs: fused sums exist in the RHS-pair kernels only");
    using S = SpinorIO<P>;
    using L = LinkIO<P, RC>;
    switch (nr) {
        // 1000 + 10 * tile + depth: pipelined RHS-tile kernel
        case 1022: return launch_nr_pipe<S, L, 2, 2>(g, s, a, block, xpay);
        case 1042:
            if constexpr (P != PLQCD_F64) return launch_nr_pipe<S, L, 4, 2>(g, s, a, block, xpay);
            break;
        // 2002: RHS-pair kernel on packed FP32 lanes; 2022 / 2032: its
        // cp.async pipeline of depth 2 / 3
        case 2002: return launch_pair<S, L, 0>(g, s, a, block, xpay, epi);
        case 2022: return launch_pair<S, L, 2>(g, s, a, block, xpay, epi);
        case 2032: return launch_pair<S, L, 3>(g, s, a, block, xpay, epi);
        // 4000 + 100 * ring depth + RHS per block: FP64 link-sharing kernel
        case 4208:
        case 4204:
        case 4308:
        case 4304:
            if constexpr (P == PLQCD_F64) {
                switch (nr) {
                    case 4208: return launch_f64blk<L, 8, 2>(g, s, a, xpay);
                    case 4204: return launch_f64blk<L, 4, 2>(g, s, a, xpay);
                    case 4308: return launch_f64blk<L, 8, 3>(g, s, a, xpay);
                    default: return launch_f64blk<L, 4, 3>(g, s, a, xpay);
                }
            }
            break;
        // 2102 / 2122: the same with at most 128 registers a thread
        case 2102: return launch_pair<S, L, 0, 2>(g, s, a, block, xpay, epi);
        case 2122: return launch_pair<S, L, 2, 2>(g, s, a, block, xpay, epi);
        case 1: return launch_nr<S, L, 1>(g, s, a, block, xpay);
        case 2: return launch_nr<S, L, 2>(g, s, a, block, xpay);
        case 4:
            // four FP64 accumulators exceed the register file
            if constexpr (P != PLQCD_F64) return launch_nr<S, L, 4>(g, s, a, block, xpay);
            break;
        default: break;
    }
    return set_error(PLQCD_ERR_ARG, "dslash_mrhs: RHS tile %d not available for this precision", nr);
}

}  // namespace dev

static int mrhs_dispatch(const Geom &g, cudaStream_t s, int prec, int recon, const dev::MrhsArgs &a, int nr,
                         int block, bool xpay, int epi = 0) {
    if (block % 32 || block < 32 || block > 256) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: block %d", block);
    switch (prec * 100 + recon) {
        case PLQCD_F64 * 100 + 18: return dev::launch_pr<PLQCD_F64, 18>(g, s, a, nr, block, xpay, epi);
        case PLQCD_F64 * 100 + 12: return dev::launch_pr<PLQCD_F64, 12>(g, s, a, nr, block, xpay, epi);
        case PLQCD_F32 * 100 + 18: return dev::launch_pr<PLQCD_F32, 18>(g, s, a, nr, block, xpay, epi);
        case PLQCD_F32 * 100 + 12: return dev::launch_pr<PLQCD_F32, 12>(g, s, a, nr, block, xpay, epi);
        case PLQCD_F16 * 100 + 12: return dev::launch_pr<PLQCD_F16, 12>(g, s, a, nr, block, xpay, epi);
        case PLQCD_BF16 * 100 + 12: return dev::launch_pr<PLQCD_BF16, 12>(g, s, a, nr, block, xpay, epi);
        default: return set_error(PLQCD_ERR_ARG, "dslash_mrhs: unsupported format %d/%d", prec, recon);
    }
}

int launch_dslash_mrhs_tc(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                          const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x, double b,
                          int tiles);

// TMA-staged RHS tiles: variant 100000 * nr + 1000 * kind + 100 * nstage + ny
static int launch_mrhs_tma(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                           const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x,
                           double b, int variant) {
    const int nr = variant / 100000, rest = variant % 100000;
    return launch_dslash_tma_mrhs(g, s, gauge, prec, recon, out, in, nrhs, out_parity, flags, a, x, b, rest / 1000,
                                  (rest / 100) % 10, rest % 100, nr);
}

// tuner key of a multi-RHS hop
static void mrhs_key(char *key, size_t n, const Geom &g, int prec, int recon, int nrhs, bool xpay) {
    snprintf(key, n, "%sdslash_mrhs|p%d|r%d|%s|n%d|%dx%dx%dx%d", device_tag().c_str(), prec, recon,
             xpay ? "xpay" : "plain", nrhs, g.L[0], g.L[1], g.L[2], g.L[3]);
}

// true when a launch of this multi-RHS hop would not tune (a tuned entry
// exists, tuning is off, or the environment fixes the configuration)
bool dslash_mrhs_tuned(const Geom &g, int prec, int recon, int nrhs, bool xpay) {
    const char *ev = getenv("PLQCD_MRHS_VARIANT");
    if ((ev && *ev) || !tune_enabled()) return true;
    char key[256];
    mrhs_key(key, sizeof key, g, prec, recon, nrhs, xpay);
    return tune_lookup(key, nullptr);
}

// out (nrhs fields) = a_up/a_low * H in + b * x; tuned over RHS tile and block
static int mrhs_args(const Geom &g, const void *gauge, int prec, void *out, const void *in, int nrhs,
                     int out_parity, unsigned flags, double a, const void *x, double b, dev::MrhsArgs &m) {
    if (nrhs < 1) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: nrhs must be >= 1");
    PLQCD_TRY(check_field_ptr(out, "dslash_mrhs"));
    PLQCD_TRY(check_field_ptr(in, "dslash_mrhs"));
    if (x) PLQCD_TRY(check_field_ptr(x, "dslash_mrhs"));
    m = dev::MrhsArgs{};
    m.gauge = gauge;
    m.in = static_cast<const char *>(in);
    m.out = static_cast<char *>(out);
    m.x = static_cast<const char *>(x);
    m.fbytes = spinor_parity_bytes(g.Vh, prec);
    m.nrhs = nrhs;
    m.Vh = g.Vh;
    m.L0 = g.L[0];
    m.L0h = g.L0h;
    m.L1 = g.L[1];
    m.L2 = g.L[2];
    m.L3 = g.L[3];
    m.out_parity = out_parity;
    m.a_up = a;
    m.a_low = (flags & PLQCD_DSLASH_G5_OUT) ? -a : a;
    m.b = b;
    m.g5_in = (flags & PLQCD_DSLASH_G5_IN) ? -1.0 : 1.0;
    return PLQCD_OK;
}

// the RHS-pair configuration that runs this xpay hop with fused sums: the
// environment's, else the tuned one (false when it is another kernel)
static bool mrhs_sink_config(const Geom &g, int prec, int recon, int nrhs, TuneResult *t, bool xpay = true) {
    const char *ev = getenv("PLQCD_MRHS_VARIANT");
    if (ev && *ev) {
        const char *eb = getenv("PLQCD_MRHS_BLOCK");
        t->variant = atoi(ev);
        t->block = (eb && *eb) ? atoi(eb) : 128;
    } else {
        char key[256];
        mrhs_key(key, sizeof key, g, prec, recon, nrhs, xpay);
        if (!tune_lookup(key, t)) return false;
    }
    const int v = t->variant;
    return v == 2002 || v == 2022 || v == 2032 || v == 2102 || v == 2122;
}

bool dslash_mrhs_sink_ok(const Geom &g, int prec, int recon, int nrhs, int *variant, int *block) {
    TuneResult t, tp;
    if (prec == PLQCD_F64 || nrhs < 2 || !mrhs_sink_config(g, prec, recon, nrhs, &t) ||
        !mrhs_sink_config(g, prec, recon, nrhs, &tp, false))
        return false;
    if (variant) *variant = t.variant;
    if (block) *block = t.block;
    return true;
}

int launch_dslash_mrhs_sink(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                            const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x,
                            double b, int epi, const RhsSink &sink) {
    TuneResult t;
    const bool xpay = epi != 4;
    if (epi < 1 || epi > 4 || (xpay != (x != nullptr)) || prec == PLQCD_F64 ||
        !mrhs_sink_config(g, prec, recon, nrhs, &t, xpay))
        return set_error(PLQCD_ERR_ARG, "dslash_mrhs: no RHS-pair configuration for fused epilogue %d", epi);
    dev::MrhsArgs m;
    PLQCD_TRY(mrhs_args(g, gauge, prec, out, in, nrhs, out_parity, flags, a, x, b, m));
    m.sink = sink;
    PLQCD_TRY(mrhs_dispatch(g, s, prec, recon, m, t.variant, t.block, xpay, epi));
    const int nsb = (int)((g.Vh + t.block - 1) / t.block);
    if (epi == 1)
        dev::k_sink_finish<1><<<nrhs, 1024, 0, s>>>(sink, nsb);
    else if (epi == 2)
        dev::k_sink_finish<2><<<nrhs, 1024, 0, s>>>(sink, nsb);
    else if (epi == 3)
        dev::k_sink_finish<3><<<nrhs, 1024, 0, s>>>(sink, nsb);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

int launch_dslash_mrhs(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                       const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x, double b) {
    dev::MrhsArgs m;
    PLQCD_TRY(mrhs_args(g, gauge, prec, out, in, nrhs, out_parity, flags, a, x, b, m));
    const bool xpay = x != nullptr;
    char key[256];
    mrhs_key(key, sizeof key, g, prec, recon, nrhs, xpay);
    // two families of candidates: the RHS-tile kernel above (variant = tile
    // size 1, 2, 4), and the single-RHS kernels with the RHS index folded
    // into the grid, RHS fastest, so the blocks of one site range run
    // together and share links through L2 (variant = 100 + single-RHS
    // variant: 0 direct loads, 2/3 cp.async pipeline depth)
    std::vector<TuneResult> cands;
    for (int v : {102, 100, 103})
        for (int blk : {64, 128, 256}) {
            TuneResult t;
            t.variant = v;
            t.block = blk;
            cands.push_back(t);
        }

    // FP64: TMA-staged rows with RHS tiles (dslash_tma.cu; variant 100000 *
    // RHS per tile + 1000 * kind + 100 * ring depth + rows per tile): the
    // tile's links are staged once for its RHS, and the spinor rows move
    // without LSU wavefronts
    if (prec == PLQCD_F64 && !(flags & PLQCD_DSLASH_COMPAT) && getenv("PLQCD_NO_TMA") == nullptr)
        for (int nr : {4, 2, 8})
            for (int kind : {2, 4})
                for (int ny : {2, 1, 4})
                    for (int ns : {1, 2, 3}) {
                        if (nrhs % nr || (kind == 2 ? ns == 3 : ns == 1)) continue;
                        int blk = 0;
                        if (dslash_tma_plan(g, prec, recon, kind, ns, ny, &blk, nullptr, nr) != PLQCD_OK) {
                            clear_error();
                            continue;
                        }
                        TuneResult t;
                        t.variant = 100000 * nr + 1000 * kind + 100 * ns + ny;
                        t.block = blk;
                        cands.push_back(t);
                    }
    // FP64: the link-sharing block kernel (4000 + 100 * depth + RHS per block)
    if (prec == PLQCD_F64 && nrhs >= 4)
        for (int v : {4208, 4204, 4308, 4304}) {
            if ((v % 100) > nrhs) continue;
            TuneResult t;
            t.variant = v;
            t.block = 32 * (v % 100);
            cands.push_back(t);
        }
    for (int nr : {2022, 2122, 2032, 2002, 2102, 1022, 1042, 2, 1, 4}) {
        const bool pair = nr >= 2000;
        if (pair && (prec == PLQCD_F64 || nrhs < 2)) continue;
        const int tile = pair ? 2 : nr >= 1000 ? (nr / 10) % 10 : nr;
        if (tile == 4 && prec == PLQCD_F64) continue;
        if (tile > nrhs && tile != 1) continue;
        for (int blk : {64, 128, 256}) {
            TuneResult t;
            t.variant = nr;
            t.block = blk;
            cands.push_back(t);
        }
    }
    // tensor-core kernel (dslash_mrhs_tc.cu), 16-bit fields with 12-real
    // links: variant 3000 + RHS tiles of 8 per warp (block fixed at 128)
    if ((prec == PLQCD_F16 || prec == PLQCD_BF16) && recon == 12 && nrhs >= 8)
        for (int tiles : {1, 2, 4}) {
            if (tiles > 1 && 8 * tiles > nrhs) continue;
            TuneResult t;
            t.variant = 3000 + tiles;
            t.block = 128;
            cands.push_back(t);
        }
    DslashCall dc;
    dc.gauge = gauge;
    dc.prec = prec;
    dc.recon = recon;
    dc.out = out;
    dc.in = in;
    dc.out_parity = out_parity;
    dc.flags = flags;
    dc.x = x;
    dc.a_up = dc.a_low = a;
    dc.b = b;
    dc.nrhs = nrhs;
    void *scratch = nullptr;
    // explicit configuration for experiments and tests: bypasses the tuner
    const char *ev = getenv("PLQCD_MRHS_VARIANT");
    if (ev && *ev) {
        const char *eb = getenv("PLQCD_MRHS_BLOCK");
        TuneResult t;
        t.variant = atoi(ev);
        t.block = (eb && *eb) ? atoi(eb) : 128;
        if (t.variant >= 100 && t.variant < 1000) {
            DslashCall c2 = dc;
            return launch_dslash_config(g, s, c2, t.variant - 100, t.block);
        }
        if (t.variant >= 3000 && t.variant < 4000)
            return launch_dslash_mrhs_tc(g, s, gauge, prec, recon, out, in, nrhs, out_parity, flags, a, x, b,
                                         t.variant - 3000);
        if (t.variant >= 100000)
            return launch_mrhs_tma(g, s, gauge, prec, recon, out, in, nrhs, out_parity, flags, a, x, b, t.variant);
        return mrhs_dispatch(g, s, prec, recon, m, t.variant, t.block, xpay);
    }
    std::vector<int> tma_checked;
    auto launch = [&](const TuneResult &t, char *dst) -> int {
        if (t.variant >= 100000)
            return launch_mrhs_tma(g, s, gauge, prec, recon, dst, in, nrhs, out_parity, flags, a, x, b, t.variant);
        if (t.variant >= 3000 && t.variant < 4000)
            return launch_dslash_mrhs_tc(g, s, gauge, prec, recon, dst, in, nrhs, out_parity, flags, a, x, b,
                                         t.variant - 3000);
        if (t.variant >= 100 && t.variant < 1000) {
            DslashCall c2 = dc;
            c2.out = dst;
            return launch_dslash_config(g, s, c2, t.variant - 100, t.block);
        }
        dev::MrhsArgs tm = m;
        tm.out = dst;
        return mrhs_dispatch(g, s, prec, recon, tm, t.variant, t.block, xpay);
    };
    auto run = [&](const TuneResult &t, bool trial) -> int {
        if (!trial) return launch(t, static_cast<char *>(out));
        if (!scratch && cudaMalloc(&scratch, m.fbytes * nrhs) != cudaSuccess) {
            cudaGetLastError();
            return set_error(PLQCD_ERR_NOMEM, "tune: scratch allocation failed");
        }
        if (t.variant >= 100000 && std::find(tma_checked.begin(), tma_checked.end(), t.variant) == tma_checked.end()) {
            // first trial of a TMA configuration: run it alone and check that
            // no stage wait ran out before it is timed
            tma_checked.push_back(t.variant);
            PLQCD_TRY(launch(t, static_cast<char *>(scratch)));
            PLQCD_CUDA_TRY(cudaStreamSynchronize(s));
            if (dslash_tma_status(true)) return set_error(PLQCD_ERR_CUDA, "dslash_mrhs: TMA stage wait timed out");
        }
        return launch(t, static_cast<char *>(scratch));
    };
    int rc = tune_launch(key, s, cands, run);
    if (scratch) {
        cudaStreamSynchronize(s);
        cudaFree(scratch);
    }
    return rc;
}

}  // namespace plqcd

using namespace plqcd;

static int mrhs_common(plqcd_lattice *lat, const plqcd_gauge *gf, int prec) {
    if (!lat || !gf) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: null lattice or gauge");
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    if (gf->lat->geom.Vh != lat->geom.Vh) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: gauge of another lattice");
    if (gf->prec != prec) return set_error(PLQCD_ERR_ARG, "dslash_mrhs: spinor precision != gauge precision");
    return PLQCD_OK;
}

extern "C" int plqcd_dslash_mrhs(plqcd_lattice *lat, const plqcd_gauge *gf, void *out, const void *in, int nrhs,
                                 int out_parity, int prec, unsigned flags) {
    clear_error();
    PLQCD_TRY(mrhs_common(lat, gf, prec));
    if (!out || !in || (out_parity != 0 && out_parity != 1) || (flags & PLQCD_DSLASH_COMPAT))
        return set_error(PLQCD_ERR_ARG, "dslash_mrhs: bad argument");
    return launch_dslash_mrhs(lat->geom, lat->stream, gf->data, prec, gf->recon, out, in, nrhs, out_parity, flags,
                              1.0, nullptr, 0.0);
}

extern "C" int plqcd_dslash_mrhs_xpay(plqcd_lattice *lat, const plqcd_gauge *gf, void *out, const void *in, int nrhs,
                                      int out_parity, int prec, unsigned flags, double a, const void *x, double b) {
    clear_error();
    PLQCD_TRY(mrhs_common(lat, gf, prec));
    if (!out || !in || !x || (out_parity != 0 && out_parity != 1) || (flags & PLQCD_DSLASH_COMPAT))
        return set_error(PLQCD_ERR_ARG, "dslash_mrhs_xpay: bad argument");
    return launch_dslash_mrhs(lat->geom, lat->stream, gf->data, prec, gf->recon, out, in, nrhs, out_parity, flags, a,
                              x, b);
}
