// dslash_tma.cu -- hopping matrix with TMA-staged neighbour rows (sm_100a).
//
// Same operator and arithmetic order as the gather kernels of dslash.cu
// (lib/dirac.c:35-408 eo, 414-791 oe; results are bit-identical), with a
// different way of feeding the SMs. The cp.async kernels copy every
// neighbour spinor and link global->shared with per-thread LDGSTS and read
// it back with LDS: both passes go through the LSU data pipe, which ncu
// shows as the limit of the full-lattice kernel (l1tex data-pipe wavefronts
// ~78% of peak, ~74% of them shared-memory wavefronts). Here one producer
// warp moves whole rows with tensor-memory-access tile loads, which write
// shared memory without LSU wavefronts, and the consumer warps only read.
//
// Work unit ("tile"): NY consecutive rows (a row is the L0/2 half-sites of
// one (y, z, t) line) of one output parity; a CTA has NY*L0/2 consumer
// threads, one output site each, plus one producer warp. CTAs are
// persistent and take tiles round-robin; with both parities (full lattice)
// the tile index runs parity-fastest, so the two parities of the same rows
// are processed at the same time and a link read from HBM for one parity's
// forward term serves the other's backward term from L2.
//
// Per tile the producer fills 8 stages, one per direction in the order of
// dir_at (x+, x-, y+, ...), in a ring of `nstage` shared-memory buffers
// (full / empty mbarrier pairs):
//   x+, x-:  the tile's own rows of the input (the x neighbours sit in the
//            same rows) and the mu=0 links (own parity / opposite parity);
//   y+, y-:  own rows plus one extra row across the tile edge (y0+NY or
//            y0-1, periodic); for y- also the extra link row;
//   z+-, t+-: the NY rows of the neighbouring (z, t) line, links likewise.
// Every coordinate passed to a tile load is a wrapped, in-range coordinate
// and the innermost one is always 0, so no load reads out of bounds.
//
// Consumers read a stage with plain loads, then lane 0 of each warp
// arrives on the stage's empty barrier. The producer refills a buffer only
// after that barrier completes, and fences the async proxy first: the
// refill's tile loads must not land before the consumers' reads of the old
// contents.
//
// The own-line kernel also runs RHS tiles (MR): one parity of a block of
// FP64 fields, a tile of NY rows of nr RHS, the spinor boxes with an RHS
// dimension and the tile's link boxes shared by its nr RHS.
//
// Every mbarrier wait is bounded (2 s by %globaltimer). A wait that runs
// out sets a device status flag (read by dslash_tma_status()), the CTA's
// threads stop, and the producer waits (bounded again) for the copies it
// issued before it returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "dslash_core.cuh"
#include "internal.h"
#include "tile_order.cuh"
#include "tma.cuh"

namespace plqcd {
namespace dev {

struct TmaGeom {
    long Vh;
    int L0, L0h, L1, L2, L3;
    int NY;       // rows per tile (divides L1)
    int nty;      // L1 / NY
    int bz, bt;   // tile order: blocks of bz z-lines x bt t-slices (divide L2 and tc)
    int t0, tc;   // the t-slices computed: [t0, t0 + tc) (all of them for whole fields)
    int nitems;   // tiles (x 2 parities in full mode)
    int nstage;   // shared-memory buffers in the ring
    int ncw;      // consumer warps = NY * L0h / 32
    int full, out_parity;
    // byte offsets inside one stage buffer and the bytes each load brings;
    // a spinor format has 1 or 2 plane groups (16-bit formats: values and
    // the per-site norms), each with its own tensor maps
    int sp_ng;
    uint32_t off_sp_main[2], off_sp_row[2], off_lk_main, off_lk_row, stage_bytes;
    uint32_t sp_main_bytes[2], sp_row_bytes[2], lk_main_bytes, lk_row_bytes;
    // shared own-line kernel (k_dslash_tma_xy): a second ring of nstage_a
    // buffers of a_bytes for the own-line rows (NY rows plus the rows on
    // either side of the tile), and a second link box in a stage buffer;
    // split: one tile-load box per stage
    int nstage_a, split;
    uint32_t a_bytes, off_a_main[2], off_a_lo[2], off_a_hi[2], off_lk2;
    double a_up, a_low, b, g5_in;
    // limit of a consumer's wait for a staged tile; with `stall` (the
    // failure-detection test hook) each consumer warp first waits, with that
    // limit, on a barrier that nothing completes, so the wait runs out
    uint64_t cwait_ns;
    uint32_t wait_hint_ns;  // suspend hint of the mbarrier retries (0: plain polls)
    int stall;
    void *out0, *out1;  // output of parity 0 / 1 (full); out0 otherwise
    const void *x;      // xpay operand (single parity)
    // RHS tiles (k_dslash_tma_xy with MR): nr RHS of a block of fields per
    // tile, ngr = nrhs / nr groups, fields fbytes apart; sp_main_rb /
    // sp_row_rb are the bytes one RHS takes in an NY-row / one-row box
    int nr, ngr;
    size_t fbytes;
    uint32_t sp_main_rb[2], sp_row_rb[2];
};

// tensor maps: input spinor field f (full mode: field 0 = even input, read
// by the odd output; field 1 = odd input) and plane group, NY-row and
// one-row boxes
struct __align__(64) TmaMaps {
    CUtensorMap sp_main[2][2], sp_row[2][2], lk_main, lk_row;
};

// ---- per-format staged loads ---------------------------------------------------
// A stage holds each plane group as [plane][row][x] with the format's own
// element size; element i of plane k is at group base + (i + k * ps) elements.
// The loaders return exactly what the gather kernels' loads return (16-bit
// spinors unscaled plus the site norm), so the arithmetic is identical.
template <class SIO>
struct TmaSpinor;

template <>
struct TmaSpinor<SpinorIO<PLQCD_F64>> {
    __device__ static __forceinline__ void load(const uint8_t *g0, const uint8_t *, int i, int ps, cx<double> s[12],
                                                double &n) {
        const double2 *p = reinterpret_cast<const double2 *>(g0) + i;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            const double2 v = p[c * ps];
            s[c] = {v.x, v.y};
        }
        n = 1.0;
    }
};

template <>
struct TmaSpinor<SpinorIO<PLQCD_F32>> {
    __device__ static __forceinline__ void load(const uint8_t *g0, const uint8_t *, int i, int ps, cx<float> s[12],
                                                float &n) {
        const float4 *p = reinterpret_cast<const float4 *>(g0) + i;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const float4 v = p[k * ps];
            s[2 * k] = {v.x, v.y};
            s[2 * k + 1] = {v.z, v.w};
        }
        n = 1.f;
    }
};

template <int PREC>
struct TmaSpinor16 {
    __device__ static __forceinline__ void load(const uint8_t *g0, const uint8_t *g1, int i, int ps, cx<float> s[12],
                                                float &n) {
        const uint4 *p = reinterpret_cast<const uint4 *>(g0) + i;
        uint4 v[3];
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = p[k * ps];
        n = reinterpret_cast<const float *>(g1)[i];
        SpinorIO16<PREC>::unpack3(v, s);
    }
};
template <>
struct TmaSpinor<SpinorIO<PLQCD_F16>> : TmaSpinor16<PLQCD_F16> {};
template <>
struct TmaSpinor<SpinorIO<PLQCD_BF16>> : TmaSpinor16<PLQCD_BF16> {};

template <class LIO>
struct TmaLink;

template <>
struct TmaLink<LinkIO<PLQCD_F64, 18>> {
    __device__ static __forceinline__ void load(const uint8_t *g, int i, int ps, cx<double> U[9]) {
        const double2 *p = reinterpret_cast<const double2 *>(g) + i;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            const double2 v = p[e * ps];
            U[e] = {v.x, v.y};
        }
    }
};

template <>
struct TmaLink<LinkIO<PLQCD_F64, 12>> {
    __device__ static __forceinline__ void load(const uint8_t *g, int i, int ps, cx<double> U[9]) {
        const double2 *p = reinterpret_cast<const double2 *>(g) + i;
#pragma unroll
        for (int e = 0; e < 6; e++) {
            const double2 v = p[e * ps];
            U[e] = {v.x, v.y};
        }
        reconstruct_row2(U);
    }
};

template <>
struct TmaLink<LinkIO<PLQCD_F32, 18>> {
    __device__ static __forceinline__ void load(const uint8_t *g, int i, int ps, cx<float> U[9]) {
        const float2 *p = reinterpret_cast<const float2 *>(g) + i;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            const float2 v = p[e * ps];
            U[e] = {v.x, v.y};
        }
    }
};

template <>
struct TmaLink<LinkIO<PLQCD_F32, 12>> {
    __device__ static __forceinline__ void load(const uint8_t *g, int i, int ps, cx<float> U[9]) {
        const float4 *p = reinterpret_cast<const float4 *>(g) + i;
#pragma unroll
        for (int e = 0; e < 3; e++) {
            const float4 v = p[e * ps];
            U[2 * e] = {v.x, v.y};
            U[2 * e + 1] = {v.z, v.w};
        }
        reconstruct_row2(U);
    }
};

template <int PREC>
struct TmaLink16 {
    __device__ static __forceinline__ void load(const uint8_t *g, int i, int ps, cx<float> U[9]) {
        const uint2 *p = reinterpret_cast<const uint2 *>(g) + i;
#pragma unroll
        for (int e = 0; e < 3; e++) {
            const uint2 v = p[e * ps];
            const float2 a = Half2<PREC>::unpack(v.x), b = Half2<PREC>::unpack(v.y);
            U[2 * e] = {a.x, a.y};
            U[2 * e + 1] = {b.x, b.y};
        }
        reconstruct_row2(U);
    }
};
template <>
struct TmaLink<LinkIO<PLQCD_F16, 12>> : TmaLink16<PLQCD_F16> {};
template <>
struct TmaLink<LinkIO<PLQCD_BF16, 12>> : TmaLink16<PLQCD_BF16> {};

__device__ int g_tma_status;  // set to 1 when a stage wait ran out

// loads of direction d (0..3 forward mu, 4..7 backward mu) into the stage
// buffer at shared address dst, completing on `bar`
__device__ __forceinline__ void tma_issue_dir(const TmaMaps &m, const TmaGeom &g, const TileCoord &c, int d,
                                              uint32_t dst, uint32_t bar) {
    const int f = g.full ? (c.p == 0 ? 1 : 0) : 0;
    const int q = c.p ^ 1;
    const int mu = d & 3;
    const bool fwd = d < 4;
    int szt = c.zt;  // (z, t) line of the neighbour rows
    if (mu == 2) {
        const int z2 = fwd ? (c.z + 1 == g.L2 ? 0 : c.z + 1) : (c.z == 0 ? g.L2 - 1 : c.z - 1);
        szt = z2 + g.L2 * c.t;
    } else if (mu == 3) {
        const int t2 = fwd ? (c.t + 1 == g.L3 ? 0 : c.t + 1) : (c.t == 0 ? g.L3 - 1 : c.t - 1);
        szt = c.z + g.L2 * t2;
    }
    // forward links sit at the output site, backward ones at the neighbour
    const int lzt = fwd ? c.zt : szt;
    const int lplane = (fwd ? c.p : q) * 4 + mu;
    const bool extra = d == 1 || d == 5;  // y stages: one spinor row across the tile edge
    uint32_t bytes = g.lk_main_bytes + (d == 5 ? g.lk_row_bytes : 0u);
    for (int gr = 0; gr < g.sp_ng; gr++) bytes += g.sp_main_bytes[gr] + (extra ? g.sp_row_bytes[gr] : 0u);
    mbar_arrive_expect_tx(bar, bytes);
    const int yr = d == 1 ? ((c.y0 + g.NY == g.L1) ? 0 : c.y0 + g.NY) : ((c.y0 == 0) ? g.L1 - 1 : c.y0 - 1);
    for (int gr = 0; gr < g.sp_ng; gr++) {
        const void *spm = f ? (const void *)&m.sp_main[1][gr] : (const void *)&m.sp_main[0][gr];
        tma_load_4d(dst + g.off_sp_main[gr], spm, bar, 0, c.y0, szt, 0);
        if (extra) {
            const void *spr = f ? (const void *)&m.sp_row[1][gr] : (const void *)&m.sp_row[0][gr];
            tma_load_4d(dst + g.off_sp_row[gr], spr, bar, 0, yr, c.zt, 0);
        }
    }
    tma_load_5d(dst + g.off_lk_main, &m.lk_main, bar, 0, c.y0, lzt, 0, lplane);
    if (d == 5) tma_load_5d(dst + g.off_lk_row, &m.lk_row, bar, 0, yr, c.zt, 0, q * 4 + 1);
}

constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s
constexpr uint64_t kDrainLimitNs = 200000000ull;  // 0.2 s

// A consumer warp's wait for a stage. The outcome is made warp-uniform, so
// a warp whose wait ran out (or saw another warp's abort) stops as a whole:
// no lane leaves while the others go on to __syncwarp. Lane 0 records the
// abort for the CTA's producer and the timeout for the host.
__device__ __forceinline__ bool consumer_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns,
                                              volatile int *abort, uint32_t hint_ns = 0) {
    const bool ok = __all_sync(0xffffffffu, mbar_wait(bar, parity, limit_ns, abort, hint_ns));
    if (!ok && (threadIdx.x & 31) == 0) {
        *abort = 1;
        atomicExch(&g_tma_status, 1);
    }
    return ok;
}

// Failure-detection test: with g.stall the consumer warp waits on `never`,
// an mbarrier with one expected arrival that nothing performs; the bounded
// wait runs out after g.cwait_ns and the warp stops (consumer_wait).
__device__ __forceinline__ bool stall_test_wait(const TmaGeom &g, uint32_t never, volatile int *abort) {
    return !g.stall || consumer_wait(never, 0, g.cwait_ns, abort);
}

// ---- shared own-line variant ----------------------------------------------------
// The x+-, y+- neighbours of a tile all sit in the own (z, t) line: rows
// y0-1 .. y0+NY of the input. k_dslash_tma_xy stages them once per tile, in
// a ring of their own, and keeps them while the four x / y directions (the
// first four of the dir_at order) are computed; the link ring carries six
// stages per tile:
//   0: U_0 forward (own parity) + U_0 backward (opposite parity), own rows
//                                                  -> x+, x-
//   1: U_1 forward + U_1 backward (and its row y0-1) -> y+, y-
//   2: spinor line z+1 + U_2 forward               -> z+
//   3: spinor line z-1 + U_2 at line z-1           -> z-
//   4: spinor line t+1 + U_3 forward               -> t+
//   5: spinor line t-1 + U_3 at line t-1           -> t-
// The split form carries one box per stage (12 stages per tile, buffers
// about half the size, so more tiles fit on an SM):
//   0: U_0 fwd  1: U_0 bwd  2: U_1 fwd  3: U_1 bwd (+ row y0-1)
//   4: spinor z+1  5: U_2 fwd  6: spinor z-1  7: U_2 at z-1
//   8: spinor t+1  9: U_3 fwd  10: spinor t-1  11: U_3 at t-1
// and a spinor stage is kept until the link stage after it has arrived.
// Directions are accumulated in the order of the other kernels, so the
// results are the same bits. Per tile it stages NY+2 own-line rows instead
// of 4 NY + 2.

// a spinor box: NY rows (or one) of the (z, t) line zt; MR: of the RHS
// c.r0 .. c.r0 + nr - 1 of the block (5-D map, RHS outermost)
template <bool MR>
__device__ __forceinline__ void tma_load_sp(uint32_t dst, const void *map, uint32_t bar, int y, int zt, int r0) {
    if constexpr (MR)
        tma_load_5d(dst, map, bar, 0, y, zt, 0, r0);
    else
        tma_load_4d(dst, map, bar, 0, y, zt, 0);
}

// own-line rows of the input (y0-1 and y0+NY wrapped) into an A buffer
template <bool MR = false>
__device__ __forceinline__ void tma_issue_xy_a(const TmaMaps &m, const TmaGeom &g, const TileCoord &c, uint32_t dst,
                                               uint32_t bar) {
    const int f = g.full ? (c.p == 0 ? 1 : 0) : 0;
    uint32_t bytes = 0;
    for (int gr = 0; gr < g.sp_ng; gr++) bytes += g.sp_main_bytes[gr] + 2u * g.sp_row_bytes[gr];
    mbar_arrive_expect_tx(bar, bytes);
    const int ylo = c.y0 == 0 ? g.L1 - 1 : c.y0 - 1;
    const int yhi = c.y0 + g.NY == g.L1 ? 0 : c.y0 + g.NY;
    for (int gr = 0; gr < g.sp_ng; gr++) {
        const void *spm = f ? (const void *)&m.sp_main[1][gr] : (const void *)&m.sp_main[0][gr];
        const void *spr = f ? (const void *)&m.sp_row[1][gr] : (const void *)&m.sp_row[0][gr];
        tma_load_sp<MR>(dst + g.off_a_main[gr], spm, bar, c.y0, c.zt, c.r0);
        tma_load_sp<MR>(dst + g.off_a_lo[gr], spr, bar, ylo, c.zt, c.r0);
        tma_load_sp<MR>(dst + g.off_a_hi[gr], spr, bar, yhi, c.zt, c.r0);
    }
}

// (z, t) line of the neighbour rows of direction d (0..3 forward mu, 4..7 backward)
__device__ __forceinline__ int neighbour_line(const TmaGeom &g, const TileCoord &c, int d) {
    const int mu = d & 3;
    const bool fwd = d < 4;
    if (mu == 2) {
        const int z2 = fwd ? (c.z + 1 == g.L2 ? 0 : c.z + 1) : (c.z == 0 ? g.L2 - 1 : c.z - 1);
        return z2 + g.L2 * c.t;
    }
    if (mu == 3) {
        const int t2 = fwd ? (c.t + 1 == g.L3 ? 0 : c.t + 1) : (c.t == 0 ? g.L3 - 1 : c.t - 1);
        return c.z + g.L2 * t2;
    }
    return c.zt;
}

// the NY spinor rows of the neighbour line of direction d (2, 3, 6, 7)
template <bool MR = false>
__device__ __forceinline__ uint32_t tma_issue_line_spinor(const TmaMaps &m, const TmaGeom &g, const TileCoord &c,
                                                          int d, uint32_t dst, uint32_t bar) {
    const int f = g.full ? (c.p == 0 ? 1 : 0) : 0;
    const int szt = neighbour_line(g, c, d);
    uint32_t bytes = 0;
    for (int gr = 0; gr < g.sp_ng; gr++) {
        const void *spm = f ? (const void *)&m.sp_main[1][gr] : (const void *)&m.sp_main[0][gr];
        tma_load_sp<MR>(dst + g.off_sp_main[gr], spm, bar, c.y0, szt, c.r0);
        bytes += g.sp_main_bytes[gr];
    }
    return bytes;
}

// the NY link rows of direction d: forward links at the tile's own rows and
// parity, backward ones at the neighbour's rows and the opposite parity
__device__ __forceinline__ void tma_issue_link(const TmaMaps &m, const TmaGeom &g, const TileCoord &c, int d,
                                               uint32_t dst, uint32_t bar) {
    const int mu = d & 3;
    const bool fwd = d < 4;
    const int lzt = fwd ? c.zt : neighbour_line(g, c, d);
    tma_load_5d(dst, &m.lk_main, bar, 0, c.y0, lzt, 0, (fwd ? c.p : (c.p ^ 1)) * 4 + mu);
}

// the link row y0-1 of U_1 at the opposite parity (the y- term of the tile's row 0)
__device__ __forceinline__ void tma_issue_link_row(const TmaMaps &m, const TmaGeom &g, const TileCoord &c,
                                                   uint32_t dst, uint32_t bar) {
    const int ylo = c.y0 == 0 ? g.L1 - 1 : c.y0 - 1;
    tma_load_5d(dst, &m.lk_row, bar, 0, ylo, c.zt, 0, (c.p ^ 1) * 4 + 1);
}

// link-ring stage s (0..5 of the six-stage table) into a B buffer. The
// expected byte count is set before the loads are issued.
template <bool MR = false>
__device__ __forceinline__ void tma_issue_xy_b(const TmaMaps &m, const TmaGeom &g, const TileCoord &c, int s,
                                               uint32_t dst, uint32_t bar) {
    if (s < 2) {  // forward and backward links of mu = s
        mbar_arrive_expect_tx(bar, 2u * g.lk_main_bytes + (s == 1 ? g.lk_row_bytes : 0u));
        tma_issue_link(m, g, c, s, dst + g.off_lk_main, bar);
        tma_issue_link(m, g, c, s + 4, dst + g.off_lk2, bar);
        if (s == 1) tma_issue_link_row(m, g, c, dst + g.off_lk_row, bar);
        return;
    }
    const int d = dir_at(s + 2);  // z+, z-, t+, t-
    uint32_t bytes = g.lk_main_bytes;
    for (int gr = 0; gr < g.sp_ng; gr++) bytes += g.sp_main_bytes[gr];
    mbar_arrive_expect_tx(bar, bytes);
    tma_issue_line_spinor<MR>(m, g, c, d, dst, bar);
    tma_issue_link(m, g, c, d, dst + g.off_lk_main, bar);
}

// direction served by split stage s (a spinor stage: that of the link stage after it)
__host__ __device__ constexpr int split_dir(int s) { return s < 4 ? dir_at(s) : dir_at(4 + (s - 4) / 2); }
__host__ __device__ constexpr bool split_is_spinor(int s) { return s >= 4 && !(s & 1); }
static_assert(split_dir(0) == 0 && split_dir(1) == 4 && split_dir(2) == 1 && split_dir(3) == 5 &&
                  split_dir(4) == 2 && split_dir(5) == 2 && split_dir(6) == 6 && split_dir(7) == 6 &&
                  split_dir(8) == 3 && split_dir(9) == 3 && split_dir(10) == 7 && split_dir(11) == 7,
              "split stage table");
static_assert(dir_at(0) == 0 && dir_at(1) == 4 && dir_at(2) == 1 && dir_at(3) == 5 && dir_at(4) == 2 &&
                  dir_at(5) == 6 && dir_at(6) == 3 && dir_at(7) == 7,
              "accumulation order x+, x-, y+, y-, z+, z-, t+, t-");

// split stage s (0..11) into a B buffer
template <bool MR = false>
__device__ __forceinline__ void tma_issue_xy_split(const TmaMaps &m, const TmaGeom &g, const TileCoord &c, int s,
                                                   uint32_t dst, uint32_t bar) {
    const int d = split_dir(s);
    if (split_is_spinor(s)) {
        uint32_t bytes = 0;
        for (int gr = 0; gr < g.sp_ng; gr++) bytes += g.sp_main_bytes[gr];
        mbar_arrive_expect_tx(bar, bytes);
        tma_issue_line_spinor<MR>(m, g, c, d, dst, bar);
        return;
    }
    mbar_arrive_expect_tx(bar, g.lk_main_bytes + (d == 5 ? g.lk_row_bytes : 0u));
    tma_issue_link(m, g, c, d, dst + g.off_lk_main, bar);
    if (d == 5) tma_issue_link_row(m, g, c, dst + g.off_lk_row, bar);
}

// waits for the full barriers of the last min(issued, n) stages of a ring
__device__ __forceinline__ void tma_drain(uint32_t full_bar, long issued, int n) {
    const long first = issued > n ? issued - n : 0;
    for (long s = first; s < issued; s++) {
        const int bb = (int)(s % n);
        const uint32_t par = (uint32_t)(s / n) & 1;
        if (!mbar_wait(full_bar + 8u * bb, par, kDrainLimitNs, nullptr)) atomicExch(&g_tma_status, 1);
    }
}

// the xpay / scale epilogue and the store of one output site (MR: of RHS
// c.r0 + r of the block)
template <class SIO, bool XPAY, class R, bool MR = false>
__device__ __forceinline__ void tma_epilogue(const TmaGeom &g, const TileCoord &c, int xh, int y, cx<R> acc[12],
                                             int r = 0) {
    const R aup = (R)g.a_up, alow = (R)g.a_low;
    const long h = xh + (long)g.L0h * (y + (long)g.L1 * c.zt);
    void *out = (g.full && c.p == 1) ? g.out1 : g.out0;
    const void *xin = g.x;
    if constexpr (MR) {
        const size_t off = (size_t)(c.r0 + r) * g.fbytes;
        out = static_cast<char *>(g.out0) + off;
        if (XPAY) xin = static_cast<const char *>(g.x) + off;
    }
    if (XPAY) {
        cx<R> xv[12];
        SIO::load(xin, g.Vh, h, xv);
        const R bb = (R)g.b;
#pragma unroll
        for (int e = 0; e < 12; e++) {
            const R ak = e < 6 ? aup : alow;
            acc[e] = {fma(ak, acc[e].re, bb * xv[e].re), fma(ak, acc[e].im, bb * xv[e].im)};
        }
    } else {
#pragma unroll
        for (int e = 6; e < 12; e++) acc[e] = {alow * acc[e].re, alow * acc[e].im};
#pragma unroll
        for (int e = 0; e < 6; e++) acc[e] = {aup * acc[e].re, aup * acc[e].im};
    }
    SIO::store(out, g.Vh, h, acc);
}

template <class SIO, class LIO, bool XPAY>
__global__ void __launch_bounds__(288, 1) k_dslash_tma(const __grid_constant__ TmaMaps m,
                                                        const __grid_constant__ TmaGeom g) {
    using R = typename SIO::real;
    extern __shared__ uint8_t smem_raw[];
    __shared__ int s_abort;
    __shared__ __align__(8) uint64_t s_never;  // the stall test's barrier
    const uint32_t raw = smem_addr(smem_raw);
    const uint32_t pad = ((raw + 127u) & ~127u) - raw;
    const uint8_t *sbase = smem_raw + pad;
    const uint32_t base = raw + pad;
    const uint32_t never = smem_addr(&s_never);
    const uint32_t full_bar = base + (uint32_t)g.nstage * g.stage_bytes;
    const uint32_t empty_bar = full_bar + 8u * g.nstage;
    const int bid = blockIdx.x;
    const int nmine = bid < g.nitems ? (g.nitems - 1 - bid) / (int)gridDim.x + 1 : 0;
    const int nthr_c = g.ncw * 32;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_abort = 0;
        for (int b = 0; b < g.nstage; b++) {
            mbar_init(full_bar + 8u * b, 1);
            mbar_init(empty_bar + 8u * b, (uint32_t)g.ncw);
        }
        mbar_init(never, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (nmine == 0) return;
    volatile int *abort = &s_abort;

    if (tid >= nthr_c) {
        // producer warp: lane 0 issues every stage of every tile of this CTA
        if (tid != nthr_c) return;
        tma_prefetch_map(&m.lk_main);
        // each refill of a buffer: wait until every consumer warp released
        // it, fence the async proxy behind their reads, then load
        int b = 0;
        uint32_t k = 0;  // completed passes over the ring
        long issued = 0;
        bool ok = true;
        for (int it = 0; it < nmine && ok; it++) {
            const TileCoord c = tile_coord(g, bid + it * (int)gridDim.x);
#pragma unroll 1
            for (int kd = 0; kd < 8; kd++) {
                // the consumers released this buffer's previous use
                if (!mbar_wait(empty_bar + 8u * b, (k + 1) & 1, kWaitLimitNs, abort, g.wait_hint_ns)) {
                    ok = false;
                    break;
                }
                fence_async_proxy_shared();  // their reads before the refill
                tma_issue_dir(m, g, c, dir_at(kd), base + (uint32_t)b * g.stage_bytes, full_bar + 8u * b);
                issued++;
                if (++b == g.nstage) {
                    b = 0;
                    k++;
                }
            }
        }
        if (!ok) {
            *abort = 1;
            atomicExch(&g_tma_status, 1);
        }
        // never leave with copies in flight: wait for the last stages issued
        const long first = issued > g.nstage ? issued - g.nstage : 0;
        for (long s = first; s < issued; s++) {
            const int bb = (int)(s % g.nstage);
            const uint32_t par = (uint32_t)(s / g.nstage) & 1;
            if (!mbar_wait(full_bar + 8u * bb, par, kDrainLimitNs, nullptr)) atomicExch(&g_tma_status, 1);
        }
        return;
    }

    // consumers: thread (row j, half-x xh) of the tile
    const int L0h = g.L0h;
    const int j = tid / L0h, xh = tid - j * L0h;
    const int own = j * L0h + xh;
    const int SM = g.NY * L0h;  // plane stride of an NY-row box, in elements
    const R sg = (R)g.g5_in;
    if (!stall_test_wait(g, never, abort)) return;
    int b = 0;
    uint32_t k = 0;
    for (int it = 0; it < nmine; it++) {
        const TileCoord c = tile_coord(g, bid + it * (int)gridDim.x);
        const int y = c.y0 + j;
        const int x = 2 * xh + ((y + c.z + c.t + c.p) & 1);
        const int xph = ((x + 1 == g.L0) ? 0 : x + 1) >> 1;
        const int xmh = ((x == 0) ? g.L0 - 1 : x - 1) >> 1;
        cx<R> acc[12];
#pragma unroll
        for (int e = 0; e < 12; e++) acc[e] = {R(0), R(0)};
#pragma unroll
        for (int kd = 0; kd < 8; kd++) {
            const int d = dir_at(kd);
            if (!consumer_wait(full_bar + 8u * b, k & 1, g.cwait_ns, abort, g.wait_hint_ns)) return;
            const uint8_t *st = sbase + (size_t)b * g.stage_bytes;
            // element index and plane stride of the neighbour spinor and the
            // link, in the NY-row box or in the one-row box of a y stage
            bool sp_row = false, lk_row = false;
            int si, li;
            if (d == 0) {
                si = own - xh + xph;
                li = own;
            } else if (d == 4) {
                si = own - xh + xmh;
                li = si;
            } else if (d == 1) {
                li = own;
                sp_row = j + 1 == g.NY;
                si = sp_row ? xh : own + L0h;
            } else if (d == 5) {
                sp_row = lk_row = j == 0;
                si = li = sp_row ? xh : own - L0h;
            } else {
                si = li = own;
            }
            cx<R> s[12], U[9];
            R n;
            TmaSpinor<SIO>::load(st + (sp_row ? g.off_sp_row[0] : g.off_sp_main[0]),
                                 st + (sp_row ? g.off_sp_row[1] : g.off_sp_main[1]), si, sp_row ? L0h : SM, s, n);
            TmaLink<LIO>::load(st + (lk_row ? g.off_lk_row : g.off_lk_main), li, lk_row ? L0h : SM, U);
            // the values are in registers: release the buffer to the producer
            __syncwarp();
            if ((tid & 31) == 0) mbar_arrive(empty_bar + 8u * b);
            compute_dir_n<false, SIO::kScaled, R>(d, acc, s, U, sg, n);
            if (++b == g.nstage) {
                b = 0;
                k++;
            }
        }
        tma_epilogue<SIO, XPAY, R>(g, c, xh, y, acc);
    }
}


// Shared own-line kernel (stage tables above tma_issue_xy_a; SPLIT: one box
// per stage). Shared memory: [nstage_a A buffers][nstage B buffers][A full |
// A empty | B full | B empty barriers]. Bounded waits and the drain as in
// k_dslash_tma. A consumer warp releases the A buffer after its last read
// of the own-line rows (direction 5), a B buffer after its last read of it.
// MR (RHS tiles, one parity of a block of fields): a tile is NY rows of nr
// RHS; the spinor boxes carry the nr RHS (RHS outermost in shared memory),
// the link boxes are staged once and serve all of them. Consumer thread
// (RHS r, row j, half-x xh); each computes what the single-field kernel
// computes for its RHS, in the same order (the same bits).
template <class SIO, class LIO, bool XPAY, bool SPLIT, bool MR = false>
__global__ void __launch_bounds__(288, 1) k_dslash_tma_xy(const __grid_constant__ TmaMaps m,
                                                           const __grid_constant__ TmaGeom g) {
    using R = typename SIO::real;
    constexpr int kStages = SPLIT ? 12 : 6;  // B stages per tile
    extern __shared__ uint8_t smem_raw[];
    __shared__ int s_abort;
    __shared__ __align__(8) uint64_t s_never;  // the stall test's barrier
    const uint32_t never = smem_addr(&s_never);
    const uint32_t raw = smem_addr(smem_raw);
    const uint32_t pad = ((raw + 127u) & ~127u) - raw;
    const uint8_t *sbase = smem_raw + pad;
    const uint32_t base = raw + pad;
    const int nA = g.nstage_a, nB = g.nstage;
    const uint32_t b_base = base + (uint32_t)nA * g.a_bytes;
    const uint32_t fullA = b_base + (uint32_t)nB * g.stage_bytes;
    const uint32_t emptyA = fullA + 8u * nA;
    const uint32_t fullB = emptyA + 8u * nA;
    const uint32_t emptyB = fullB + 8u * nB;
    const int bid = blockIdx.x;
    const int nmine = bid < g.nitems ? (g.nitems - 1 - bid) / (int)gridDim.x + 1 : 0;
    const int nthr_c = g.ncw * 32;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_abort = 0;
        for (int b = 0; b < nA; b++) {
            mbar_init(fullA + 8u * b, 1);
            mbar_init(emptyA + 8u * b, (uint32_t)g.ncw);
        }
        for (int b = 0; b < nB; b++) {
            mbar_init(fullB + 8u * b, 1);
            mbar_init(emptyB + 8u * b, (uint32_t)g.ncw);
        }
        mbar_init(never, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (nmine == 0) return;
    volatile int *abort = &s_abort;

    if (tid >= nthr_c) {
        // producer warp, lane 0: per tile the A stage, then the B stages
        if (tid != nthr_c) return;
        tma_prefetch_map(&m.lk_main);
        int a = 0, b = 0;
        uint32_t ka = 0, kb = 0;
        long na = 0, nb = 0;
        bool ok = true;
        for (int it = 0; it < nmine && ok; it++) {
            const TileCoord c = tile_coord<MR>(g, bid + it * (int)gridDim.x);
            if (!mbar_wait(emptyA + 8u * a, (ka + 1) & 1, kWaitLimitNs, abort, g.wait_hint_ns)) {
                ok = false;
                break;
            }
            fence_async_proxy_shared();  // the consumers' reads before the refill
            tma_issue_xy_a<MR>(m, g, c, base + (uint32_t)a * g.a_bytes, fullA + 8u * a);
            na++;
            if (++a == nA) {
                a = 0;
                ka++;
            }
#pragma unroll 1
            for (int s = 0; s < kStages; s++) {
                if (!mbar_wait(emptyB + 8u * b, (kb + 1) & 1, kWaitLimitNs, abort, g.wait_hint_ns)) {
                    ok = false;
                    break;
                }
                fence_async_proxy_shared();
                const uint32_t dst = b_base + (uint32_t)b * g.stage_bytes;
                if (SPLIT)
                    tma_issue_xy_split<MR>(m, g, c, s, dst, fullB + 8u * b);
                else
                    tma_issue_xy_b<MR>(m, g, c, s, dst, fullB + 8u * b);
                nb++;
                if (++b == nB) {
                    b = 0;
                    kb++;
                }
            }
        }
        if (!ok) {
            *abort = 1;
            atomicExch(&g_tma_status, 1);
        }
        // never leave with copies in flight
        tma_drain(fullA, na, nA);
        tma_drain(fullB, nb, nB);
        return;
    }

    // consumers: thread (row j, half-x xh) of the tile; MR: of RHS r
    const int L0h = g.L0h;
    const int SM = g.NY * L0h;  // plane stride of an NY-row box, in elements
    const int r = MR ? tid / SM : 0;
    const int ts = tid - r * SM;
    const int j = ts / L0h, xh = ts - j * L0h;
    const int own = j * L0h + xh;
    // byte offset of this thread's RHS in an NY-row / one-row spinor box
    // (plane groups 0 and 1)
    const uint32_t rm0 = MR ? (uint32_t)r * g.sp_main_rb[0] : 0u, rm1 = MR ? (uint32_t)r * g.sp_main_rb[1] : 0u;
    const uint32_t rr0 = MR ? (uint32_t)r * g.sp_row_rb[0] : 0u, rr1 = MR ? (uint32_t)r * g.sp_row_rb[1] : 0u;
    const R sg = (R)g.g5_in;
    const bool top = j + 1 == g.NY, bottom = j == 0;
    if (!stall_test_wait(g, never, abort)) return;
    int a = 0, b = 0;
    uint32_t ka = 0, kb = 0;
    for (int it = 0; it < nmine; it++) {
        const TileCoord c = tile_coord<MR>(g, bid + it * (int)gridDim.x);
        const int y = c.y0 + j;
        const int x = 2 * xh + ((y + c.z + c.t + c.p) & 1);
        const int xph = ((x + 1 == g.L0) ? 0 : x + 1) >> 1;
        const int xmh = ((x == 0) ? g.L0 - 1 : x - 1) >> 1;
        cx<R> acc[12];
#pragma unroll
        for (int e = 0; e < 12; e++) acc[e] = {R(0), R(0)};
        if (!consumer_wait(fullA + 8u * a, ka & 1, g.cwait_ns, abort, g.wait_hint_ns)) return;
        const uint8_t *sa = sbase + (size_t)a * g.a_bytes;
        const uint8_t *sps = nullptr;  // split: the spinor stage waiting for its link stage
        int bsp = 0;
#pragma unroll
        for (int s = 0; s < kStages; s++) {
            if (!consumer_wait(fullB + 8u * b, kb & 1, g.cwait_ns, abort, g.wait_hint_ns)) return;
            const uint8_t *st = sbase + (size_t)nA * g.a_bytes + (size_t)b * g.stage_bytes;
            // directions of this stage: one, or the forward and backward
            // terms of x or y for a two-link stage
            const bool pair = !SPLIT && s < 2;
            if (SPLIT && split_is_spinor(s)) {
                sps = st;
                bsp = b;
            } else {
#pragma unroll
                for (int k = 0; k < (pair ? 2 : 1); k++) {
                    const int d = SPLIT ? split_dir(s) : (pair ? s + 4 * k : dir_at(s + 2));
                    cx<R> sv[12], U[9];
                    R n;
                    // the link of a pair's second direction is the second box
                    const uint8_t *lk = st + (pair && k == 1 ? g.off_lk2 : g.off_lk_main);
                    int rel2 = -1;  // split: the spinor stage's buffer, released with this one
                    if (d == 0 || d == 4) {
                        // x: neighbour in the same row; the backward link sits there too
                        const int si = own - xh + (d == 0 ? xph : xmh);
                        TmaSpinor<SIO>::load(sa + g.off_a_main[0] + rm0, sa + g.off_a_main[1] + rm1, si, SM, sv, n);
                        TmaLink<LIO>::load(lk, d == 0 ? own : si, SM, U);
                    } else if (d == 1 || d == 5) {
                        // y: the row above / below, across the tile edge from the
                        // extra rows; the backward link of row 0 is the link row
                        const bool fwd = d == 1;
                        const bool edge = fwd ? top : bottom;
                        const uint32_t so0 = edge ? (fwd ? g.off_a_hi[0] : g.off_a_lo[0]) + rr0 : g.off_a_main[0] + rm0;
                        const uint32_t so1 = edge ? (fwd ? g.off_a_hi[1] : g.off_a_lo[1]) + rr1 : g.off_a_main[1] + rm1;
                        const int syi = edge ? xh : (fwd ? own + L0h : own - L0h);
                        TmaSpinor<SIO>::load(sa + so0, sa + so1, syi, edge ? L0h : SM, sv, n);
                        if (fwd)
                            TmaLink<LIO>::load(lk, own, SM, U);
                        else if (edge)
                            TmaLink<LIO>::load(st + g.off_lk_row, xh, L0h, U);
                        else
                            TmaLink<LIO>::load(lk, own - L0h, SM, U);
                    } else {
                        // z / t: the neighbour line's rows
                        const uint8_t *sp = SPLIT ? sps : st;
                        TmaSpinor<SIO>::load(sp + g.off_sp_main[0] + rm0, sp + g.off_sp_main[1] + rm1, own, SM, sv, n);
                        TmaLink<LIO>::load(lk, own, SM, U);
                        if (SPLIT) rel2 = bsp;
                    }
                    if (!pair || k == 1) {
                        // the values are in registers: release the buffers
                        __syncwarp();
                        if ((tid & 31) == 0) {
                            mbar_arrive(emptyB + 8u * b);
                            if (rel2 >= 0) mbar_arrive(emptyB + 8u * rel2);
                            if (d == 5) mbar_arrive(emptyA + 8u * a);  // last use of the own-line rows
                        }
                    }
                    compute_dir_n<false, SIO::kScaled, R>(d, acc, sv, U, sg, n);
                }
            }
            if (++b == nB) {
                b = 0;
                kb++;
            }
        }
        if (++a == nA) {
            a = 0;
            ka++;
        }
        tma_epilogue<SIO, XPAY, R, MR>(g, c, xh, y, acc, r);
    }
}


}  // namespace dev

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// Plane groups of a format: element bytes and planes per group (spinor:
// one or two groups; links: one group per (parity, mu) block).
struct TmaFormat {
    int sp_ng, sp_eb[2], sp_np[2];
    int lk_eb, lk_np;
};

bool tma_format(int prec, int recon, TmaFormat *f) {
    *f = TmaFormat{1, {16, 0}, {12, 0}, 16, 9};
    if (prec == PLQCD_F64 && recon == 18) return true;
    if (prec == PLQCD_F64 && recon == 12) {
        f->lk_np = 6;
        return true;
    }
    if (prec == PLQCD_F32) {
        f->sp_np[0] = 6;
        if (recon == 18) {
            f->lk_eb = 8;
            f->lk_np = 9;
        } else {
            f->lk_np = 3;
        }
        return recon == 18 || recon == 12;
    }
    if ((prec == PLQCD_F16 || prec == PLQCD_BF16) && recon == 12) {
        *f = TmaFormat{2, {16, 4}, {3, 1}, 8, 3};
        return true;
    }
    return false;
}

// `planes` planes of `eb`-byte elements over the half lattice, viewed as
// (row elements, L1, L2*L3, planes[, 8 parity-mu blocks]); rows of 16- and
// 8-byte elements are moved as 8-byte words, rows of 4-byte elements as such.
// nfields > 0: a spinor plane group of a block of nfields fields, fstride
// bytes apart, as a fifth dimension whose box takes nbox fields
int encode_map(CUtensorMap *m, const void *base, const Geom &g, int eb, int planes, bool links, int rows,
               int nfields = 0, size_t fstride = 0, int nbox = 1) {
    auto fn = encode_fn();
    if (!fn) return set_error(PLQCD_ERR_CUDA, "dslash: cuTensorMapEncodeTiled is not available");
    const cuuint64_t row_b = (cuuint64_t)g.L0h * eb;
    const int word = eb >= 8 ? 8 : 4;
    const cuuint64_t inner = row_b / word;
    const bool blockf = !links && nfields > 0;
    cuuint64_t dims[5] = {inner, (cuuint64_t)g.L[1], (cuuint64_t)g.L[2] * g.L[3], (cuuint64_t)planes,
                          blockf ? (cuuint64_t)nfields : 8};
    cuuint64_t strides[4] = {row_b, row_b * g.L[1], (cuuint64_t)g.Vh * eb,
                             blockf ? (cuuint64_t)fstride : (cuuint64_t)g.Vh * eb * planes};
    cuuint32_t box[5] = {(cuuint32_t)inner, (cuuint32_t)rows, 1, (cuuint32_t)planes, blockf ? (cuuint32_t)nbox : 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = fn(m, word == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32,
                    (links || blockf) ? 5 : 4,
                    const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(PLQCD_ERR_CUDA, "dslash: tensor map encoding failed (%d)", (int)r);
    return PLQCD_OK;
}

std::atomic<bool> g_tma_launched{false};
// failure-detection test hook (plqcd_tma_timeout_test): the consumer wait
// limit of the stall test, 0 when off
std::atomic<unsigned long long> g_stall_test_ns{0};

int sm_count() {
    static int n[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!n[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        n[dev] = v > 0 ? v : 1;
    }
    return n[dev];
}

inline uint32_t round128(uint32_t v) { return (v + 127u) & ~127u; }

template <class SIO, class LIO, bool XPAY, bool MR = false>
int launch_tma_t(cudaStream_t s, const dev::TmaMaps &m, const dev::TmaGeom &tg, int block, size_t smem) {
    auto k = MR ? (tg.split ? dev::k_dslash_tma_xy<SIO, LIO, XPAY, true, MR>
                            : dev::k_dslash_tma_xy<SIO, LIO, XPAY, false, MR>)
             : !tg.nstage_a ? dev::k_dslash_tma<SIO, LIO, XPAY>
             : tg.split     ? dev::k_dslash_tma_xy<SIO, LIO, XPAY, true>
                            : dev::k_dslash_tma_xy<SIO, LIO, XPAY, false>;
    PLQCD_TRY(smem_optin((const void *)k, smem));
    int occ = 0;
    PLQCD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, block, smem));
    if (occ < 1) return set_error(PLQCD_ERR_ARG, "dslash: TMA tile does not fit on an SM (%zu B)", smem);
    long grid = (long)sm_count() * occ;
    if (grid > tg.nitems) grid = tg.nitems;
    g_tma_launched.store(true, std::memory_order_relaxed);
    k<<<(unsigned)grid, block, smem, s>>>(m, tg);
    PLQCD_CUDA_TRY(cudaGetLastError());
    return PLQCD_OK;
}

}  // namespace

namespace {

// stage layout of a format and tile: offsets (128-byte aligned) and the bytes
// of each box
struct StageLayout {
    uint32_t off_sp_main[2] = {0, 0}, off_sp_row[2] = {0, 0}, off_lk_main = 0, off_lk_row = 0, bytes = 0;
    uint32_t sp_main_bytes[2] = {0, 0}, sp_row_bytes[2] = {0, 0}, lk_main_bytes = 0, lk_row_bytes = 0;
};

// nr > 1: spinor boxes of nr RHS (RHS tiles); the link boxes are per tile
StageLayout stage_layout(const TmaFormat &f, int L0h, int ny, int nr = 1) {
    StageLayout l;
    uint32_t off = 0;
    auto take = [&](uint32_t n) {
        const uint32_t o = off;
        off += round128(n);
        return o;
    };
    for (int gr = 0; gr < f.sp_ng; gr++) {
        l.sp_main_bytes[gr] = (uint32_t)(f.sp_np[gr] * f.sp_eb[gr] * L0h * ny * nr);
        l.off_sp_main[gr] = take(l.sp_main_bytes[gr]);
        l.sp_row_bytes[gr] = (uint32_t)(f.sp_np[gr] * f.sp_eb[gr] * L0h * nr);
        l.off_sp_row[gr] = take(l.sp_row_bytes[gr]);
    }
    l.lk_main_bytes = (uint32_t)(f.lk_np * f.lk_eb * L0h * ny);
    l.off_lk_main = take(l.lk_main_bytes);
    l.lk_row_bytes = (uint32_t)(f.lk_np * f.lk_eb * L0h);
    l.off_lk_row = take(l.lk_row_bytes);
    l.bytes = off;
    return l;
}

// layout of the shared own-line kernel: the A buffer holds the NY own-line
// rows and the rows below and above the tile. A B buffer holds a link box
// and either the neighbour spinor rows (z, t stages) or a second link box
// and the link row (x / y stages) in the same place; split: the spinor rows,
// or one link box and the link row.
struct XyLayout {
    uint32_t off_a_main[2] = {0, 0}, off_a_lo[2] = {0, 0}, off_a_hi[2] = {0, 0}, a_bytes = 0;
    uint32_t off_sp_main[2] = {0, 0}, off_lk_main = 0, off_lk2 = 0, off_lk_row = 0, b_bytes = 0;
};

XyLayout xy_layout(const TmaFormat &f, const StageLayout &l, bool split) {
    XyLayout x;
    uint32_t off = 0;
    auto take = [&](uint32_t n) {
        const uint32_t o = off;
        off += round128(n);
        return o;
    };
    for (int gr = 0; gr < f.sp_ng; gr++) {
        x.off_a_main[gr] = take(l.sp_main_bytes[gr]);
        x.off_a_lo[gr] = take(l.sp_row_bytes[gr]);
        x.off_a_hi[gr] = take(l.sp_row_bytes[gr]);
    }
    x.a_bytes = off;
    off = 0;
    if (!split) x.off_lk_main = take(l.lk_main_bytes);
    const uint32_t second = off;
    for (int gr = 0; gr < f.sp_ng; gr++) x.off_sp_main[gr] = take(l.sp_main_bytes[gr]);
    const uint32_t end_sp = off;
    off = second;
    if (split)
        x.off_lk_main = take(l.lk_main_bytes);
    else
        x.off_lk2 = take(l.lk_main_bytes);
    x.off_lk_row = take(l.lk_row_bytes);
    x.b_bytes = end_sp > off ? end_sp : off;
    return x;
}

// kind of a TMA variant -> A buffers (0: the per-direction kernel) and form
inline int kind_a_buffers(int kind) { return kind <= 1 ? 0 : (kind <= 3 ? kind - 1 : kind - 3); }
inline bool kind_split(int kind) { return kind == 4 || kind == 5; }

// a row of eb-byte elements must be a whole number of 16-byte units (tile
// loads) and at most 256 words
bool row_ok(int L0h, int eb) {
    const int word = eb >= 8 ? 8 : 4;
    return (L0h * eb) % 16 == 0 && L0h * eb / word <= 256;
}

}  // namespace

int dslash_tma_plan(const Geom &g, int prec, int recon, int kind, int nstage, int ny, int *block, size_t *smem,
                    int nr) {
    TmaFormat f;
    if (!tma_format(prec, recon, &f))
        return set_error(PLQCD_ERR_ARG, "dslash: no TMA kernel for precision/reconstruction %d/%d", prec, recon);
    // RHS tiles: FP64 fields, own-line kinds with one own-line buffer
    if (nr < 1 || (nr > 1 && (prec != PLQCD_F64 || (kind != 2 && kind != 4))))
        return set_error(PLQCD_ERR_ARG, "dslash: no TMA RHS tile of %d for kind %d, precision %d", nr, kind, prec);
    bool rows = row_ok(g.L0h, f.lk_eb);
    for (int gr = 0; gr < f.sp_ng; gr++) rows = rows && row_ok(g.L0h, f.sp_eb[gr]);
    // kind 1: one stage per direction (a ring of at least 2); 2, 3: own-line
    // rows in 1 or 2 buffers of their own; 4, 5: the same with one box per
    // stage (a spinor stage waits for the link stage after it: 2 at least)
    const int min_stage = kind == 2 || kind == 3 ? 1 : 2;
    const int nsites = nr * ny * g.L0h;  // consumer threads
    if (kind < 1 || kind > 5 || nstage < min_stage || nstage > 8 || ny < 1 || !rows || g.L[1] % ny ||
        nsites % 32 || nsites > 256)
        return set_error(PLQCD_ERR_ARG, "dslash: TMA tile %d rows x %d stages (kind %d) does not fit %dx%dx%dx%d", ny,
                         nstage, kind, g.L[0], g.L[1], g.L[2], g.L[3]);
    const StageLayout l = stage_layout(f, g.L0h, ny, nr);
    size_t bytes = (size_t)nstage * l.bytes + 16u * nstage + 128;
    if (kind > 1) {
        const XyLayout x = xy_layout(f, l, kind_split(kind));
        const int na = kind_a_buffers(kind);
        bytes = (size_t)na * x.a_bytes + (size_t)nstage * x.b_bytes + 16u * (na + nstage) + 128;
    }
    if (bytes > 227u * 1024 - 64) return set_error(PLQCD_ERR_ARG, "dslash: TMA ring of %zu bytes too large", bytes);
    if (block) *block = nsites + 32;
    if (smem) *smem = bytes;
    return PLQCD_OK;
}

namespace {

// tile geometry, stage layout and wait limits shared by the single-field and
// the RHS-tile launches: tiles of ny rows over the t-slices [h_begin, h_end)
// (half-site range of whole t-slices); `launch` (dev::TileLaunch) picks the
// default tile order
void fill_tile_geom(dev::TmaGeom &tg, const Geom &g, const TmaFormat &fmt, const StageLayout &lay, int kind,
                    int nstage, int ny, long h_begin, long h_end, int launch) {
    const long S = (long)g.L0h * g.L[1] * g.L[2];
    memset(&tg, 0, sizeof tg);
    tg.Vh = g.Vh;
    tg.L0 = g.L[0];
    tg.L0h = g.L0h;
    tg.L1 = g.L[1];
    tg.L2 = g.L[2];
    tg.L3 = g.L[3];
    tg.NY = ny;
    tg.nty = g.L[1] / ny;
    // tile-order block: the launch's default (tile_order.cuh), or
    // PLQCD_TMA_ORDER="bz,bt" (each must divide its extent, else 1; 1,1 = the
    // plain z-fastest order)
    {
        const int tc = (int)((h_end - h_begin) / S);
        tg.t0 = (int)(h_begin / S);
        tg.tc = tc;
        int bz = 1, bt = 1;
        dev::tile_order_default(launch, g.L[2], tc, &bz, &bt);
        if (const char *e = getenv("PLQCD_TMA_ORDER"))
            if (sscanf(e, "%d,%d", &bz, &bt) != 2) bz = bt = 1;
        tg.bz = (bz > 0 && g.L[2] % bz == 0) ? bz : 1;
        tg.bt = (bt > 0 && tc % bt == 0) ? bt : 1;
    }
    tg.nstage = nstage;
    tg.ncw = ny * g.L0h / 32;
    tg.sp_ng = fmt.sp_ng;
    for (int gr = 0; gr < 2; gr++) {
        tg.sp_main_bytes[gr] = lay.sp_main_bytes[gr];
        tg.sp_row_bytes[gr] = lay.sp_row_bytes[gr];
        tg.off_sp_main[gr] = lay.off_sp_main[gr];
        tg.off_sp_row[gr] = lay.off_sp_row[gr];
    }
    tg.lk_main_bytes = lay.lk_main_bytes;
    tg.lk_row_bytes = lay.lk_row_bytes;
    tg.off_lk_main = lay.off_lk_main;
    tg.off_lk_row = lay.off_lk_row;
    tg.stage_bytes = lay.bytes;
    if (kind > 1) {
        const XyLayout xl = xy_layout(fmt, lay, kind_split(kind));
        tg.nstage_a = kind_a_buffers(kind);
        tg.split = kind_split(kind) ? 1 : 0;
        tg.a_bytes = xl.a_bytes;
        for (int gr = 0; gr < 2; gr++) {
            tg.off_a_main[gr] = xl.off_a_main[gr];
            tg.off_a_lo[gr] = xl.off_a_lo[gr];
            tg.off_a_hi[gr] = xl.off_a_hi[gr];
            tg.off_sp_main[gr] = xl.off_sp_main[gr];
        }
        tg.off_lk_main = xl.off_lk_main;
        tg.off_lk2 = xl.off_lk2;
        tg.off_lk_row = xl.off_lk_row;
        tg.stage_bytes = xl.b_bytes;
    }
    tg.cwait_ns = dev::kWaitLimitNs;
    // PLQCD_TMA_WAIT_HINT: suspend hint (ns) of the mbarrier retries
    {
        const char *e = getenv("PLQCD_TMA_WAIT_HINT");
        const long v = (e && *e) ? atol(e) : 0;
        tg.wait_hint_ns = v > 0 && v < 1000000 ? (uint32_t)v : 0u;
    }
    tg.stall = 0;
    if (const unsigned long long ns = g_stall_test_ns.load(std::memory_order_relaxed)) {
        tg.stall = 1;
        tg.cwait_ns = ns;
    }
}

}  // namespace

int launch_dslash_tma(const Geom &g, cudaStream_t s, const dev::DslashArgs &a, int prec, int recon, bool full,
                      bool xpay, int kind, int nstage, int ny) {
    int block = 0;
    size_t smem = 0;
    PLQCD_TRY(dslash_tma_plan(g, prec, recon, kind, nstage, ny, &block, &smem));
    // whole t-slices of one field (all of them for the full lattice)
    const long S = (long)g.L0h * g.L[1] * g.L[2];
    if (a.nrhs != 1 || (full && xpay) || a.h_begin % S || (a.h_end - a.h_begin) % S ||
        (full && (a.h_begin != 0 || a.h_end != g.Vh)))
        return set_error(PLQCD_ERR_ARG, "dslash: the TMA kernel takes whole t-slices of single fields");
    TmaFormat fmt;
    tma_format(prec, recon, &fmt);
    const StageLayout lay = stage_layout(fmt, g.L0h, ny);

    dev::TmaGeom tg;
    fill_tile_geom(tg, g, fmt, lay, kind, nstage, ny, a.h_begin, a.h_end,
                   full ? dev::kTileFull : dev::kTileParity);
    const long ntiles = (long)tg.nty * g.L[2] * tg.tc;
    if (ntiles * (full ? 2 : 1) > 0x7fffffffL) return set_error(PLQCD_ERR_ARG, "dslash: lattice too large");
    tg.nitems = (int)(ntiles * (full ? 2 : 1));
    tg.full = full ? 1 : 0;
    tg.out_parity = a.out_parity;
    tg.a_up = a.a_up;
    tg.a_low = a.a_low;
    tg.b = a.b;
    tg.g5_in = a.g5_in;
    tg.out0 = a.out[0];
    tg.out1 = full ? a.out[1] : a.out[0];
    tg.x = a.x;

    dev::TmaMaps m;
    memset(&m, 0, sizeof m);
    const int nf = full ? 2 : 1;
    for (int f = 0; f < nf; f++) {
        size_t goff = 0;  // byte offset of the plane group in the field
        for (int gr = 0; gr < fmt.sp_ng; gr++) {
            const void *base = static_cast<const char *>(a.in[f]) + goff;
            PLQCD_TRY(encode_map(&m.sp_main[f][gr], base, g, fmt.sp_eb[gr], fmt.sp_np[gr], false, ny));
            PLQCD_TRY(encode_map(&m.sp_row[f][gr], base, g, fmt.sp_eb[gr], fmt.sp_np[gr], false, 1));
            goff += (size_t)fmt.sp_np[gr] * fmt.sp_eb[gr] * g.Vh;
        }
    }
    if (!full)
        for (int gr = 0; gr < 2; gr++) {
            m.sp_main[1][gr] = m.sp_main[0][gr];
            m.sp_row[1][gr] = m.sp_row[0][gr];
        }
    PLQCD_TRY(encode_map(&m.lk_main, a.gauge, g, fmt.lk_eb, fmt.lk_np, true, ny));
    PLQCD_TRY(encode_map(&m.lk_row, a.gauge, g, fmt.lk_eb, fmt.lk_np, true, 1));

    using namespace dev;
#define PLQCD_TMA_CASE(P, RC)                                                                              \
    if (prec == P && recon == RC)                                                                          \
        return xpay ? launch_tma_t<SpinorIO<P>, LinkIO<P, RC>, true>(s, m, tg, block, smem)                \
                    : launch_tma_t<SpinorIO<P>, LinkIO<P, RC>, false>(s, m, tg, block, smem);
    PLQCD_TMA_CASE(PLQCD_F64, 18)
    PLQCD_TMA_CASE(PLQCD_F64, 12)
    PLQCD_TMA_CASE(PLQCD_F32, 18)
    PLQCD_TMA_CASE(PLQCD_F32, 12)
    PLQCD_TMA_CASE(PLQCD_F16, 12)
    PLQCD_TMA_CASE(PLQCD_BF16, 12)
#undef PLQCD_TMA_CASE
    return set_error(PLQCD_ERR_ARG, "dslash: no TMA kernel for precision/reconstruction %d/%d", prec, recon);
}

// RHS tiles: nr RHS of the block per tile, the links staged once per tile.
// Per output site and RHS the staged bytes fall from 6 spinor rows + 8.5
// link rows per row (one field at a time) to 6 spinor rows + 8.5 / nr link
// rows (2 rows per tile).
int launch_dslash_tma_mrhs(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                           const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x,
                           double b, int kind, int nstage, int ny, int nr) {
    int block = 0;
    size_t smem = 0;
    PLQCD_TRY(dslash_tma_plan(g, prec, recon, kind, nstage, ny, &block, &smem, nr));
    if (nr < 2 || nrhs < nr || nrhs % nr || (flags & PLQCD_DSLASH_COMPAT) || (out_parity != 0 && out_parity != 1))
        return set_error(PLQCD_ERR_ARG, "dslash: TMA RHS tile of %d does not divide %d RHS", nr, nrhs);
    TmaFormat fmt;
    tma_format(prec, recon, &fmt);
    const StageLayout lay = stage_layout(fmt, g.L0h, ny, nr);
    const size_t fbytes = spinor_parity_bytes(g.Vh, prec);
    if (fbytes % 16) return set_error(PLQCD_ERR_ARG, "dslash: field stride %zu is not a multiple of 16", fbytes);

    dev::TmaGeom tg;
    fill_tile_geom(tg, g, fmt, lay, kind, nstage, ny, 0, g.Vh, dev::kTileRhs);
    const long ntiles = (long)tg.nty * g.L[2] * tg.tc;
    if (ntiles * (nrhs / nr) > 0x7fffffffL) return set_error(PLQCD_ERR_ARG, "dslash: lattice too large");
    tg.nr = nr;
    tg.ngr = nrhs / nr;
    tg.nitems = (int)(ntiles * tg.ngr);
    tg.ncw = nr * ny * g.L0h / 32;
    tg.fbytes = fbytes;
    for (int gr = 0; gr < fmt.sp_ng; gr++) {
        tg.sp_main_rb[gr] = lay.sp_main_bytes[gr] / (uint32_t)nr;
        tg.sp_row_rb[gr] = lay.sp_row_bytes[gr] / (uint32_t)nr;
    }
    tg.full = 0;
    tg.out_parity = out_parity;
    tg.a_up = a;
    tg.a_low = (flags & PLQCD_DSLASH_G5_OUT) ? -a : a;
    tg.b = b;
    tg.g5_in = (flags & PLQCD_DSLASH_G5_IN) ? -1.0 : 1.0;
    tg.out0 = tg.out1 = out;
    tg.x = x;

    dev::TmaMaps m;
    memset(&m, 0, sizeof m);
    size_t goff = 0;
    for (int gr = 0; gr < fmt.sp_ng; gr++) {
        const void *base = static_cast<const char *>(in) + goff;
        PLQCD_TRY(encode_map(&m.sp_main[0][gr], base, g, fmt.sp_eb[gr], fmt.sp_np[gr], false, ny, nrhs, fbytes, nr));
        PLQCD_TRY(encode_map(&m.sp_row[0][gr], base, g, fmt.sp_eb[gr], fmt.sp_np[gr], false, 1, nrhs, fbytes, nr));
        m.sp_main[1][gr] = m.sp_main[0][gr];
        m.sp_row[1][gr] = m.sp_row[0][gr];
        goff += (size_t)fmt.sp_np[gr] * fmt.sp_eb[gr] * g.Vh;
    }
    PLQCD_TRY(encode_map(&m.lk_main, gauge, g, fmt.lk_eb, fmt.lk_np, true, ny));
    PLQCD_TRY(encode_map(&m.lk_row, gauge, g, fmt.lk_eb, fmt.lk_np, true, 1));

    using namespace dev;
    const bool xpay = x != nullptr;
#define PLQCD_TMA_CASE(P, RC)                                                                              \
    if (prec == P && recon == RC)                                                                          \
        return xpay ? launch_tma_t<SpinorIO<P>, LinkIO<P, RC>, true, true>(s, m, tg, block, smem)          \
                    : launch_tma_t<SpinorIO<P>, LinkIO<P, RC>, false, true>(s, m, tg, block, smem);
    PLQCD_TMA_CASE(PLQCD_F64, 18)
    PLQCD_TMA_CASE(PLQCD_F64, 12)
#undef PLQCD_TMA_CASE
    return set_error(PLQCD_ERR_ARG, "dslash: no TMA RHS-tile kernel for precision/reconstruction %d/%d", prec, recon);
}

// Reads (and with `reset`, clears) the timeout flag of the TMA kernel on the
// current device. Only touches the device when a TMA kernel was launched
// since the last reset.
int dslash_tma_status(bool reset) {
    if (!g_tma_launched.load(std::memory_order_relaxed)) return 0;
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, dev::g_tma_status, sizeof v) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (reset) {
        if (v) {
            const int z = 0;
            cudaMemcpyToSymbol(dev::g_tma_status, &z, sizeof z);
        }
        g_tma_launched.store(false, std::memory_order_relaxed);
    }
    return v;
}

}  // namespace plqcd

// Failure-detection test of the bounded stage waits (the reference's
// counterpart is the exit(1) of lib/dirac.c:128-130): see plqcd_b200.h.
extern "C" int plqcd_tma_timeout_test(int enable, unsigned long long limit_ns) {
    using namespace plqcd;
    clear_error();
    if (!enable) {
        g_stall_test_ns.store(0, std::memory_order_relaxed);
        return PLQCD_OK;
    }
    if (limit_ns < 1000ull || limit_ns > dev::kWaitLimitNs)
        return set_error(PLQCD_ERR_ARG, "plqcd_tma_timeout_test: limit %llu ns outside 1 us .. 2 s", limit_ns);
    g_stall_test_ns.store(limit_ns, std::memory_order_relaxed);
    return PLQCD_OK;
}
