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

#include <algorithm>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "dslash_core.cuh"
#include "internal.h"
#include "tune.h"

namespace plqcd {
namespace dev {

// One direction (MU, FWD) of one output site.
template <class SIO, class LIO, int MU, bool FWD, bool COMPAT>
__device__ __forceinline__ void hop_dir(cx<typename SIO::real> acc[12], const void *in, const void *gauge,
                                        long Vh, long h_nbr, int link_par, long h_link,
                                        typename SIO::real sg_in) {
    using R = typename SIO::real;
    cx<R> s[12];
    R n;
    SIO::load_raw(in, Vh, h_nbr, s, n);
    cx<R> U[9];
    LIO::load(gauge, Vh, link_par, MU, h_link, U);
    // projection, SU(3) product and rebuild (with COMPAT, the reference's
    // as-shipped loss of the forward terms of spins 2, 3)
    compute_dir_n<COMPAT, SIO::kScaled, R>(FWD ? MU : MU + 4, acc, s, U, sg_in, n);
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
        h = a.h_begin + (long)(blockIdx.x / a.nrhs) * blockDim.x + threadIdx.x;
    }
    if (h >= a.h_end) return;
    // selects, not a dynamic index into the parameter arrays (which would
    // copy them to local memory)
    const long roff = FULL ? 0 : (long)(blockIdx.x % a.nrhs) * a.fbytes;  // RHS of this block
    const void *in = (FULL && par == 0) ? a.in[1] : static_cast<const char *>(a.in[0]) + roff;
    void *out = (FULL && par == 1) ? a.out[1] : static_cast<char *>(a.out[0]) + roff;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(h, par, L0h, L1, L2);
    const int xh = (int)(h - c.row * L0h);

    // neighbour half-site indices (periodic wrap on the device)
    int nbs[8];
    neighbour_sites(c, xh, a.L0, L0h, L1, L2, L3, nbs);
    const int h_xp = nbs[0], h_yp = nbs[1], h_zp = nbs[2], h_tp = nbs[3];
    const int h_xm = nbs[4], h_ym = nbs[5], h_zm = nbs[6], h_tm = nbs[7];

    const R sg = (R)a.g5_in;
    const int opp = par ^ 1;
    // as shipped, oe takes forward links of odd site h from the even site
    // with the same half index (lib/dirac.c:643)
    const int fpar = (COMPAT && par == 1) ? 0 : par;

    cx<R> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = {R(0), R(0)};

    // the order of dir_at: x+, x-, y+, y-, z+, z-, t+, t-
    hop_dir<SIO, LIO, 0, true, COMPAT>(acc, in, a.gauge, Vh, h_xp, fpar, h, sg);
    hop_dir<SIO, LIO, 0, false, COMPAT>(acc, in, a.gauge, Vh, h_xm, opp, h_xm, sg);
    hop_dir<SIO, LIO, 1, true, COMPAT>(acc, in, a.gauge, Vh, h_yp, fpar, h, sg);
    hop_dir<SIO, LIO, 1, false, COMPAT>(acc, in, a.gauge, Vh, h_ym, opp, h_ym, sg);
    hop_dir<SIO, LIO, 2, true, COMPAT>(acc, in, a.gauge, Vh, h_zp, fpar, h, sg);
    hop_dir<SIO, LIO, 2, false, COMPAT>(acc, in, a.gauge, Vh, h_zm, opp, h_zm, sg);
    hop_dir<SIO, LIO, 3, true, COMPAT>(acc, in, a.gauge, Vh, h_tp, fpar, h, sg);
    hop_dir<SIO, LIO, 3, false, COMPAT>(acc, in, a.gauge, Vh, h_tm, opp, h_tm, sg);

    const R aup = (R)a.a_up, alow = (R)a.a_low;
    if (XPAY) {
        cx<R> xv[12];
        SIO::load(static_cast<const char *>(a.x) + roff, Vh, h, xv);
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

// Pipelined variant: the neighbour spinor and link of each of the 8
// directions are copied global->shared with cp.async, ST directions ahead of
// the one being computed, into slots private to the thread (no block-level
// synchronisation). The register file then only holds the direction being
// computed, while ST directions' loads are in flight per thread.
// Shared memory per block: ST * (spinor + link slots) * 16 bytes * blockDim.
template <class SIO, class LIO, int ST, bool COMPAT, bool XPAY, bool FULL>
__global__ void __launch_bounds__(256) k_dslash_pipe(const DslashArgs a) {
    using R = typename SIO::real;
    extern __shared__ uint4 smem[];
    constexpr int NS = SIO::NSLOT + LIO::NSLOT;
    const int B = blockDim.x;
    int par;
    long h;
    if (FULL) {
        par = blockIdx.x & 1;
        h = (long)(blockIdx.x >> 1) * B + threadIdx.x;
    } else {
        par = a.out_parity;
        h = a.h_begin + (long)(blockIdx.x / a.nrhs) * B + threadIdx.x;
    }
    if (h >= a.h_end) return;  // no block-level barrier below
    const long roff = FULL ? 0 : (long)(blockIdx.x % a.nrhs) * a.fbytes;  // RHS of this block
    const void *in = (FULL && par == 0) ? a.in[1] : static_cast<const char *>(a.in[0]) + roff;
    void *out = (FULL && par == 1) ? a.out[1] : static_cast<char *>(a.out[0]) + roff;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    const Coords c = site_coords(h, par, L0h, L1, L2);
    const int xh = (int)(h - c.row * L0h);
    int nb[8];
    neighbour_sites(c, xh, a.L0, L0h, L1, L2, L3, nb);
    const int opp = par ^ 1;
    const int fpar = (COMPAT && par == 1) ? 0 : par;

    const int stride = B * 16;  // bytes between consecutive slots of one thread
    const uint32_t s_thread = smem_addr(smem) + threadIdx.x * 16;
    // k-th direction of dir_at into slot k % ST
    auto issue = [&](int k) {
        const int d = dir_at(k);
        const uint32_t s0 = s_thread + (uint32_t)((k % ST) * NS) * stride;
        SIO::issue(in, Vh, nb[d], s0, stride);
        if (d < 4)
            LIO::issue(a.gauge, Vh, fpar, d, h, s0 + SIO::NSLOT * stride, stride);
        else
            LIO::issue(a.gauge, Vh, opp, d - 4, nb[d], s0 + SIO::NSLOT * stride, stride);
    };
#pragma unroll
    for (int k = 0; k < ST; k++) {
        issue(k);
        cp_async_commit();
    }
    cx<R> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = {R(0), R(0)};
    const R sg = (R)a.g5_in;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        cp_async_wait<ST - 1>();
        const uint4 *s0 = smem + threadIdx.x + (k % ST) * NS * B;
        cx<R> s[12], U[9];
        R n;
        SIO::load_staged_raw(s0, B, s, n);
        LIO::load_staged(s0 + SIO::NSLOT * B, B, U);
        compute_dir_n<COMPAT, SIO::kScaled, R, true>(dir_at(k), acc, s, U, sg, n);
        // the slot just consumed is refilled only after its values were used
        if (k + ST < 8) issue(k + ST);
        cp_async_commit();
    }

    const R aup = (R)a.a_up, alow = (R)a.a_low;
    if (XPAY) {
        cx<R> xv[12];
        SIO::load(static_cast<const char *>(a.x) + roff, Vh, h, xv);
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

template <class SIO, class LIO, int ST, bool COMPAT, bool XPAY, bool FULL>
static int launch_pipe(const Geom &g, cudaStream_t s, const DslashArgs &a, int block) {
    long nblk = (a.h_end - a.h_begin + block - 1) / block * a.nrhs;
    if (FULL) nblk *= 2;
    constexpr int NS = SIO::NSLOT + LIO::NSLOT;
    const size_t smem = (size_t)ST * NS * 16 * block;
    auto k = k_dslash_pipe<SIO, LIO, ST, COMPAT, XPAY, FULL>;
    PLQCD_TRY(smem_optin((const void *)k, 227 * 1024));
    if (smem > 227 * 1024) return set_error(PLQCD_ERR_ARG, "dslash: %zu bytes of shared memory requested", smem);
    k<<<(unsigned)nblk, block, smem, s>>>(a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

// Two sites per thread (sites h and h + blockDim of a 2*blockDim tile),
// direct loads, the direction loops of both sites interleaved: twice the
// independent loads in flight per thread and shared index arithmetic, for
// the 32- and 16-bit formats whose kernels are latency / issue bound.
// PACK: the two sites are the two lanes of packed FP32 instructions (f2),
// which halves the arithmetic instructions and gives the same bits.
// Single parity only (RHS blocks allowed), no bug-compatible mode.
template <class SIO, class LIO, bool XPAY, bool PACK>
__global__ void __launch_bounds__(256) k_dslash_spt2(const DslashArgs a) {
    using R = typename SIO::real;
    constexpr int S = 2;
    const int par = a.out_parity, opp = par ^ 1;
    const long tile = blockIdx.x / a.nrhs;
    const long roff = (long)(blockIdx.x % a.nrhs) * a.fbytes;
    const void *in = static_cast<const char *>(a.in[0]) + roff;
    void *out = static_cast<char *>(a.out[0]) + roff;
    const long Vh = a.Vh;
    const int L0h = a.L0h, L1 = a.L1, L2 = a.L2, L3 = a.L3;
    long hs[S];
    int nb[S][8];
    bool ok[S];
#pragma unroll
    for (int j = 0; j < S; j++) {
        long h = a.h_begin + tile * (S * blockDim.x) + j * blockDim.x + threadIdx.x;
        ok[j] = h < a.h_end;
        if (!ok[j]) h = a.h_begin;  // compute on a valid site, store nothing
        hs[j] = h;
        const Coords c = site_coords(h, par, L0h, L1, L2);
        const int xh = (int)(h - c.row * L0h);
        neighbour_sites(c, xh, a.L0, L0h, L1, L2, L3, nb[j]);
    }
    if (!ok[0]) return;
    const R sg = (R)a.g5_in;
    cx<R> acc[S][12];
    if constexpr (PACK) {
        static_assert(S == 2, "one site per lane");
        cx<f2> acc2[12];
#pragma unroll
        for (int k = 0; k < 12; k++) acc2[k] = {f2(0.f), f2(0.f)};
        const f2 sg2(sg);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int d = dir_at(k);
            cx<R> s[S][12], U[S][9];
            R n[S];
#pragma unroll
            for (int j = 0; j < S; j++) {
                SIO::load_raw(in, Vh, nb[j][d], s[j], n[j]);
                if (d < 4)
                    LIO::load(a.gauge, Vh, par, d, hs[j], U[j]);
                else
                    LIO::load(a.gauge, Vh, opp, d - 4, nb[j][d], U[j]);
            }
            cx<f2> s2[12], U2[9];
#pragma unroll
            for (int k = 0; k < 12; k++) s2[k] = zip(s[0][k], s[1][k]);
#pragma unroll
            for (int k = 0; k < 9; k++) U2[k] = zip(U[0][k], U[1][k]);
            compute_dir_n<false, SIO::kScaled, f2>(d, acc2, s2, U2, sg2, f2(n[0], n[1]));
        }
#pragma unroll
        for (int j = 0; j < S; j++)
#pragma unroll
            for (int k = 0; k < 12; k++) acc[j][k] = lane(acc2[k], j);
    } else {
#pragma unroll
        for (int j = 0; j < S; j++)
#pragma unroll
            for (int k = 0; k < 12; k++) acc[j][k] = {R(0), R(0)};
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int d = dir_at(k);
            cx<R> s[S][12], U[S][9];
            R n[S];
#pragma unroll
            for (int j = 0; j < S; j++) {
                SIO::load_raw(in, Vh, nb[j][d], s[j], n[j]);
                if (d < 4)
                    LIO::load(a.gauge, Vh, par, d, hs[j], U[j]);
                else
                    LIO::load(a.gauge, Vh, opp, d - 4, nb[j][d], U[j]);
            }
#pragma unroll
            for (int j = 0; j < S; j++) compute_dir_n<false, SIO::kScaled, R>(d, acc[j], s[j], U[j], sg, n[j]);
        }
    }
    const R aup = (R)a.a_up, alow = (R)a.a_low;
#pragma unroll
    for (int j = 0; j < S; j++) {
        if (!ok[j]) continue;
        if (XPAY) {
            cx<R> xv[12];
            SIO::load(static_cast<const char *>(a.x) + roff, Vh, hs[j], xv);
            const R b = (R)a.b;
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const R ak = k < 6 ? aup : alow;
                acc[j][k] = {fma(ak, acc[j][k].re, b * xv[k].re), fma(ak, acc[j][k].im, b * xv[k].im)};
            }
        } else {
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const R ak = k < 6 ? aup : alow;
                acc[j][k] = {ak * acc[j][k].re, ak * acc[j][k].im};
            }
        }
        SIO::store(out, Vh, hs[j], acc[j]);
    }
}

template <class SIO, class LIO, bool COMPAT, bool XPAY, bool FULL>
static int launch_direct(const Geom &g, cudaStream_t s, const DslashArgs &a, int block);

template <class SIO, class LIO, bool COMPAT, bool XPAY, bool FULL>
static int launch_spt2(const Geom &g, cudaStream_t s, const DslashArgs &a, int block, bool pack) {
    if constexpr (COMPAT || FULL || std::is_same<typename SIO::real, double>::value) {
        return set_error(PLQCD_ERR_ARG, "dslash: two sites per thread exists for 32/16-bit single-parity calls");
    } else {
        const long nblk = (a.h_end - a.h_begin + 2L * block - 1) / (2L * block) * a.nrhs;
        if (pack)
            k_dslash_spt2<SIO, LIO, XPAY, true><<<(unsigned)nblk, block, 0, s>>>(a);
        else
            k_dslash_spt2<SIO, LIO, XPAY, false><<<(unsigned)nblk, block, 0, s>>>(a);
        PLQCD_CUDA_TRY(cudaGetLastError());
        return PLQCD_OK;
    }
}

// variant 0: direct loads; 2, 3: cp.async pipeline of that depth; 12: two
// sites per thread; 13: the same on packed FP32 lanes
template <class SIO, class LIO, bool COMPAT, bool XPAY, bool FULL>
static int launch_t(const Geom &g, cudaStream_t s, const DslashArgs &a, int variant, int block) {
    if (variant == 2) return launch_pipe<SIO, LIO, 2, COMPAT, XPAY, FULL>(g, s, a, block);
    if (variant == 3) return launch_pipe<SIO, LIO, 3, COMPAT, XPAY, FULL>(g, s, a, block);
    if (variant == 12 || variant == 13) return launch_spt2<SIO, LIO, COMPAT, XPAY, FULL>(g, s, a, block, variant == 13);
    return launch_direct<SIO, LIO, COMPAT, XPAY, FULL>(g, s, a, block);
}

template <class SIO, class LIO, bool COMPAT, bool XPAY, bool FULL>
static int launch_direct(const Geom &g, cudaStream_t s, const DslashArgs &a, int block) {
    long nblk = (a.h_end - a.h_begin + block - 1) / block * a.nrhs;
    if (FULL) nblk *= 2;
    k_dslash<SIO, LIO, COMPAT, XPAY, FULL><<<(unsigned)nblk, block, 0, s>>>(a);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

template <int PREC, int RECON>
static int launch_pr(const Geom &g, cudaStream_t s, const DslashArgs &a, int variant, int block, bool compat,
                     bool xpay, bool full) {
    using S = SpinorIO<PREC>;
    using L = LinkIO<PREC, RECON>;
    if (full) return launch_t<S, L, false, false, true>(g, s, a, variant, block);
    if (compat) {
        if (PREC == PLQCD_F64 && RECON == 18) return launch_t<S, L, true, false, false>(g, s, a, variant, block);
        return set_error(PLQCD_ERR_ARG, "dslash: the bug-compatible mode exists for F64 18-real links only");
    }
    if (xpay) return launch_t<S, L, false, true, false>(g, s, a, variant, block);
    return launch_t<S, L, false, false, false>(g, s, a, variant, block);
}

}  // namespace dev

int launch_dslash_tma(const Geom &g, cudaStream_t s, const dev::DslashArgs &a, int prec, int recon, bool full,
                      bool xpay, int kind, int nstage, int ny);

static int env_int(const char *name, int dflt) {
    const char *e = getenv(name);
    return (e && *e) ? atoi(e) : dflt;  // unset or empty: the default
}

static int dispatch(const Geom &g, cudaStream_t s, const DslashCall &c, const dev::DslashArgs &a, int variant,
                    int block);

static int build_args(const Geom &g, const DslashCall &c, dev::DslashArgs &a);
static int tune_dslash(const Geom &g, cudaStream_t s, const DslashCall &c, const dev::DslashArgs &a,
                       const char *key);

// one launch with an explicit configuration (no tuning)
int launch_dslash_config(const Geom &g, cudaStream_t s, const DslashCall &c, int variant, int block) {
    dev::DslashArgs a{};
    PLQCD_TRY(build_args(g, c, a));
    return dispatch(g, s, c, a, variant, block);
}

int launch_dslash(const Geom &g, cudaStream_t s, const DslashCall &c) {
    dev::DslashArgs a{};
    PLQCD_TRY(build_args(g, c, a));
    const bool compat = (c.flags & PLQCD_DSLASH_COMPAT) != 0;

    // explicit configuration (block from the call, or the environment for
    // experiments) bypasses the tuner
    int env_block = env_int("PLQCD_DSLASH_BLOCK", 0), env_var = env_int("PLQCD_DSLASH_STAGES", -1);
    // PLQCD_DSLASH_FULL_STAGES: the variant of full-lattice F64 calls only
    if (c.full && c.prec == PLQCD_F64 && env_int("PLQCD_DSLASH_FULL_STAGES", -1) >= 0) {
        env_var = env_int("PLQCD_DSLASH_FULL_STAGES", -1);
        if (env_block <= 0) env_block = 64;
    }
    if (c.block > 0 || env_block > 0 || env_var >= 0) {
        int block = c.block > 0 ? c.block : (env_block > 0 ? env_block : 128);
        return dispatch(g, s, c, a, env_var >= 0 ? env_var : 2, block);
    }
    char key[256];
    // a partial site range (the drop-in path's t-slab chunks) is a separate
    // entry: the TMA kernel takes whole fields only
    const bool part = a.h_begin != 0 || a.h_end != g.Vh;
    snprintf(key, sizeof key, "%sdslash|p%d|r%d|%s%s%s%s|%dx%dx%dx%d|n%d", device_tag().c_str(), c.prec, c.recon,
             c.full ? "full" : "half", c.x ? "+xpay" : "", compat ? "+compat" : "", part ? "+range" : "", g.L[0],
             g.L[1], g.L[2], g.L[3], c.nrhs);
    return tune_dslash(g, s, c, a, key);
}

static int build_args(const Geom &g, const DslashCall &c, dev::DslashArgs &a) {
    PLQCD_TRY(check_field_ptr(c.out, "dslash"));
    PLQCD_TRY(check_field_ptr(c.in, "dslash"));
    if (c.full) {
        PLQCD_TRY(check_field_ptr(c.out2, "dslash_full"));
        PLQCD_TRY(check_field_ptr(c.in2, "dslash_full"));
    }
    if (c.x) PLQCD_TRY(check_field_ptr(c.x, "dslash_xpay"));
    a.gauge = c.gauge;
    if (c.nrhs < 1 || (c.full && c.nrhs != 1)) return set_error(PLQCD_ERR_ARG, "dslash: nrhs = %d invalid", c.nrhs);
    a.nrhs = c.nrhs;
    a.fbytes = (long)spinor_parity_bytes(g.Vh, c.prec);
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
    a.h_begin = c.h_begin;
    a.h_end = c.h_count < 0 ? g.Vh : c.h_begin + c.h_count;
    if (a.h_begin < 0 || a.h_end > g.Vh || a.h_end <= a.h_begin || (c.full && (a.h_begin != 0 || a.h_end != g.Vh)))
        return set_error(PLQCD_ERR_ARG, "dslash: site range [%ld, %ld) invalid", a.h_begin, a.h_end);
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
    if (c.full && (compat || c.x || (c.flags & (PLQCD_DSLASH_G5_IN | PLQCD_DSLASH_G5_OUT))))
        return set_error(PLQCD_ERR_ARG, "dslash_full: flags and xpay are not supported in full-lattice mode");
    return PLQCD_OK;
}

static int tune_dslash(const Geom &g, cudaStream_t s, const DslashCall &c, const dev::DslashArgs &a,
                       const char *key) {
    // load strategy (0 direct, 2/3 cp.async pipeline depth, 12 two sites per
    // thread) x block size
    std::vector<TuneResult> cands;
    const bool spt_ok = c.prec != PLQCD_F64 && !c.full && !(c.flags & PLQCD_DSLASH_COMPAT);
    for (int v : {2, 0, 3, 12, 13}) {
        if (v >= 12 && !spt_ok) continue;
        for (int b : {64, 128, 256}) {
            TuneResult r;
            r.variant = v;
            r.block = b;
            cands.push_back(r);
        }
    }
    // TMA-staged rows: ring depth x rows per tile, where the tile fits
    const long slab = (long)g.L0h * g.L[1] * g.L[2];  // TMA tiles cover whole t-slices
    const bool tma_ok = !(c.flags & PLQCD_DSLASH_COMPAT) && c.nrhs == 1 && a.h_begin % slab == 0 &&
                        (a.h_end - a.h_begin) % slab == 0 && getenv("PLQCD_NO_TMA") == nullptr;
    if (tma_ok)
        // (kinds 3 and 5, two own-line buffers, lost to 2 and 4 at every
        // measured point and are not tried). The own-line kernels (4, 2)
        // come first, so they keep a near-tie: they stage fewer bytes per
        // site and hold a higher rate once the power cap settles the clock
        // (FP64 full lattice at 32^3x64, 4 s back to back: 4304 0.666 of
        // HBM against 0.651 for 1204, at 1515 / 1470 MHz)
        for (int kind : {4, 2, 1})
            for (int ny : {4, 8, 16, 2})
                for (int ns : {1, 2, 3, 4, 6}) {
                    if (kind == 2 ? ns == 6 : ns == 1) continue;
                    int blk = 0;
                    if (dslash_tma_plan(g, c.prec, c.recon, kind, ns, ny, &blk, nullptr) != PLQCD_OK) {
                        clear_error();
                        continue;
                    }
                    TuneResult r;
                    r.variant = 1000 * kind + 100 * ns + ny;
                    r.block = blk;
                    cands.push_back(r);
                }
    // trial launches write into scratch outputs: an xpay whose output aliases
    // its x operand must not be applied more than once
    void *scratch[2] = {nullptr, nullptr};
    std::vector<int> tma_checked;
    auto run = [&](const TuneResult &r, bool trial) -> int {
        if (!trial) return dispatch(g, s, c, a, r.variant, r.block);
        if (r.variant >= 1000 && std::find(tma_checked.begin(), tma_checked.end(), r.variant) == tma_checked.end()) {
            // first trial of a TMA configuration: run it alone and check that
            // no stage wait ran out before it is timed
            tma_checked.push_back(r.variant);
            dev::DslashArgs t = a;
            size_t bytes = spinor_parity_bytes(g.Vh, c.prec);
            for (int k = 0; k < (c.full ? 2 : 1); k++)
                if (!scratch[k] && cudaMalloc(&scratch[k], bytes) != cudaSuccess) {
                    cudaGetLastError();
                    return set_error(PLQCD_ERR_NOMEM, "tune: scratch allocation failed");
                }
            t.out[0] = scratch[0];
            if (c.full) t.out[1] = scratch[1];
            PLQCD_TRY(dispatch(g, s, c, t, r.variant, r.block));
            PLQCD_CUDA_TRY(cudaStreamSynchronize(s));
            if (dslash_tma_status(true)) return set_error(PLQCD_ERR_CUDA, "dslash: TMA stage wait timed out");
        }
        size_t bytes = spinor_parity_bytes(g.Vh, c.prec) * c.nrhs;
        for (int k = 0; k < (c.full ? 2 : 1); k++)
            if (!scratch[k] && cudaMalloc(&scratch[k], bytes) != cudaSuccess) {
                cudaGetLastError();
                return set_error(PLQCD_ERR_NOMEM, "tune: scratch allocation failed");
            }
        dev::DslashArgs t = a;
        t.out[0] = scratch[0];
        if (c.full) t.out[1] = scratch[1];
        return dispatch(g, s, c, t, r.variant, r.block);
    };
    int rc = tune_launch(key, s, cands, run);
    for (void *p : scratch)
        if (p) {
            cudaStreamSynchronize(s);
            cudaFree(p);
        }
    return rc;
}

static int dispatch(const Geom &g, cudaStream_t s, const DslashCall &c, const dev::DslashArgs &a, int variant,
                    int block) {
    const bool compat = (c.flags & PLQCD_DSLASH_COMPAT) != 0;
    const bool xpay = c.x != nullptr;
    if (variant >= 1000) {  // TMA-staged rows; the block follows from the tile
        if (compat) return set_error(PLQCD_ERR_ARG, "dslash: no bug-compatible TMA kernel");
        return launch_dslash_tma(g, s, a, c.prec, c.recon, c.full, xpay, variant / 1000, (variant / 100) % 10,
                                 variant % 100);
    }
    if (block % 32 || block < 32 || block > 256) return set_error(PLQCD_ERR_ARG, "dslash: block size %d invalid", block);
    switch (c.prec * 100 + c.recon) {
        case PLQCD_F64 * 100 + 18: return dev::launch_pr<PLQCD_F64, 18>(g, s, a, variant, block, compat, xpay, c.full);
        case PLQCD_F64 * 100 + 12: return dev::launch_pr<PLQCD_F64, 12>(g, s, a, variant, block, compat, xpay, c.full);
        case PLQCD_F32 * 100 + 18: return dev::launch_pr<PLQCD_F32, 18>(g, s, a, variant, block, compat, xpay, c.full);
        case PLQCD_F32 * 100 + 12: return dev::launch_pr<PLQCD_F32, 12>(g, s, a, variant, block, compat, xpay, c.full);
        case PLQCD_F16 * 100 + 12: return dev::launch_pr<PLQCD_F16, 12>(g, s, a, variant, block, compat, xpay, c.full);
        case PLQCD_BF16 * 100 + 12: return dev::launch_pr<PLQCD_BF16, 12>(g, s, a, variant, block, compat, xpay, c.full);
        default:
            return set_error(PLQCD_ERR_ARG, "dslash: unsupported precision/reconstruction %d/%d", c.prec, c.recon);
    }
}

}  // namespace plqcd
