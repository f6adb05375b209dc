/*
 * plqcd_b200.h -- device-resident API of plqcd-b200 (sm_100a).
 *
 * The drop-in entry points of dirac.h take host arrays in the API layout
 * and pay host<->device copies on every call. This header exposes the same
 * operator on fields that stay in HBM, in the layouts the kernels read,
 * plus reduced-precision storage, the even/odd preconditioned Wilson
 * solver, multi-RHS and multi-lattice batches. The reference has no
 * counterpart for anything here except the hopping matrix itself
 * (lib/dirac.c:35-791); its operator and solver parameters are
 * placeholders (include/plqcd_global_params.h:197-201).
 *
 * Conventions
 *  - Every function returns PLQCD_OK (0) or a negative status; the message
 *    is in plqcd_last_error() (thread-local). Nothing aborts the caller.
 *  - Device pointers are plain CUDA device addresses on the lattice's
 *    device; the caller owns them. Work is queued on the lattice's stream.
 *  - Site order is the reference's even/odd order (lib/start.c:406-433):
 *    within one parity, half-site index h = x/2 + L0/2*(y + L1*(z + L2*t)).
 *
 * Device field layouts (one parity, Vh = V/2 half-sites; "plane" = Vh
 * consecutive elements):
 *   spinor PLQCD_F64  : double2 [12][Vh]   plane k = complex 3*spin+colour
 *   spinor PLQCD_F32  : float4  [6][Vh]    plane k = complexes 2k, 2k+1
 *   spinor PLQCD_F16,
 *          PLQCD_BF16 : 16-bit  [3][Vh][8] (uint4 planes, complexes 4k..4k+3)
 *                       followed by float norm[Vh]; value = stored * norm,
 *                       norm = max |real or imaginary part| of the site
 *   gauge (both parities, 4 directions): [parity][mu][element][Vh]
 *          F64 recon 18 : double2, 9 elements (row-major c00..c22)
 *          F64 recon 12 : double2, 6 elements (rows 0,1)
 *          F32 recon 18 : float2,  9 elements
 *          F32 recon 12 : float4,  3 elements (complex pairs of rows 0,1)
 *          F16/BF16 12  : 16-bit x4 (uint2), 3 elements
 *   With 12-real storage row 2 is rebuilt as conj(row0 x row1), exact for
 *   SU(3) links only.
 * A multi-RHS spinor block is n fields back to back: [rhs][...one field...].
 */
#ifndef PLQCD_B200_H
#define PLQCD_B200_H

#include <stddef.h>
#include <stdint.h>
#include "su3.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ----------------------------------------------------------- */
#define PLQCD_OK 0
#define PLQCD_ERR_ARG -1      /* invalid argument */
#define PLQCD_ERR_CUDA -2     /* CUDA runtime error */
#define PLQCD_ERR_NOMEM -3    /* allocation failed */
#define PLQCD_ERR_STATE -4    /* not initialised / wrong object state */
#define PLQCD_ERR_TIMEOUT -5  /* a bounded device wait ran out */
#define PLQCD_ERR_NOCONV -6   /* solver did not converge */
#define PLQCD_ERR_NODEV -7    /* no CUDA device */

const char *plqcd_last_error(void);
int plqcd_last_status(void);
void plqcd_clear_error(void);
/* Library version string. */
const char *plqcd_version(void);

/* ---- precisions and flags --------------------------------------------- */
#define PLQCD_F64 0
#define PLQCD_F32 1
#define PLQCD_F16 2
#define PLQCD_BF16 3

#define PLQCD_EVEN 0
#define PLQCD_ODD 1

/* dslash flags */
#define PLQCD_DSLASH_COMPAT 1u  /* reproduce the reference as shipped (F64/18 only) */
#define PLQCD_DSLASH_G5_IN 2u   /* apply gamma5 to the input spinor */
#define PLQCD_DSLASH_G5_OUT 4u  /* apply gamma5 to H psi before the epilogue */

/* ---- lattice context ---------------------------------------------------- */
typedef struct plqcd_lattice plqcd_lattice;

/* dims: L0..L3, each even and >= 2. device: CUDA ordinal. stream: the
 * cudaStream_t all work of this lattice is queued on (NULL = the device's
 * default stream); the caller keeps ownership of the stream. */
int plqcd_lattice_create(const int dims[4], int device, void *stream, plqcd_lattice **out);
int plqcd_lattice_destroy(plqcd_lattice *lat);
int plqcd_lattice_set_stream(plqcd_lattice *lat, void *stream);
void *plqcd_lattice_stream(const plqcd_lattice *lat);
int plqcd_lattice_synchronize(plqcd_lattice *lat);
long plqcd_lattice_half_volume(const plqcd_lattice *lat);
/* Device time of the last kernel launched through the *_timed calls, ms. */
double plqcd_lattice_last_kernel_ms(const plqcd_lattice *lat);

size_t plqcd_spinor_bytes(const plqcd_lattice *lat, int prec);
size_t plqcd_gauge_bytes(const plqcd_lattice *lat, int prec, int recon);

/* ---- gauge fields (owned by the library) -------------------------------- */
typedef struct plqcd_gauge plqcd_gauge;

int plqcd_gauge_create(plqcd_lattice *lat, int prec, int recon, plqcd_gauge **out);
int plqcd_gauge_destroy(plqcd_gauge *g);
/* Device address of the gauge storage (layout above). */
void *plqcd_gauge_data(plqcd_gauge *g);
/* Load from links in the API layout (4V su3, u[4*i+mu]) on the host or on
 * the device. */
int plqcd_gauge_load_host(plqcd_gauge *g, const su3 *u_host);
int plqcd_gauge_load_device(plqcd_gauge *g, const su3 *u_dev);
/* Store to the API layout (row 2 rebuilt for 12-real storage). */
int plqcd_gauge_store_host(const plqcd_gauge *g, su3 *u_host);
/* Random SU(3) links from a counter-based generator keyed by (seed, site,
 * mu): Gaussian complex 3x3, Gram-Schmidt rows 0,1, row 2 = conj(row0 x
 * row1). */
int plqcd_gauge_random(plqcd_gauge *g, uint64_t seed);
/* Unit links (free field). */
int plqcd_gauge_unit(plqcd_gauge *g);
/* Convert between precisions / storage (dst and src on the same lattice). */
int plqcd_gauge_copy(plqcd_gauge *dst, const plqcd_gauge *src);

/* ---- spinor fields (caller-owned device buffers) ------------------------ */
/* Import / export one parity between the API layout (full-lattice array of
 * V spinors on the device, even/odd order) and a device field. */
int plqcd_spinor_import(plqcd_lattice *lat, const spinor *aos_dev, int parity, void *dst, int prec);
int plqcd_spinor_export(plqcd_lattice *lat, const void *src, int prec, int parity, spinor *aos_dev);
/* Convert one parity between precisions. */
int plqcd_spinor_convert(plqcd_lattice *lat, void *dst, int dst_prec, const void *src, int src_prec);
/* Gaussian N(0,1) complex components, keyed by (seed, parity, site). */
int plqcd_spinor_gaussian(plqcd_lattice *lat, void *dst, int prec, int parity, uint64_t seed);

/* |x_f|^2 (FP64 accumulation, fixed summation order) of `nfields` one-parity
 * fields stored back to back in `fields`; results go to the device array
 * norms_dev[nfields], asynchronously on the lattice stream. Scratch for the
 * per-block partial sums comes from the lattice's device workspace
 * (allocated with cudaMalloc on first use or growth). */
int plqcd_spinor_norm2(plqcd_lattice *lat, const void *fields, int prec, int nfields, double *norms_dev);

/* Same result as plqcd_spinor_norm2, for callers that must not allocate
 * device memory: applications whose device memory all comes from their own
 * pool (a framework that has reserved the GPU's memory, a service held to a
 * fixed budget), where an allocation outside the pool fails or breaks the
 * budget, and latency-bound loops that cannot take the device-wide
 * synchronisation of cudaFree. It calls no cudaMalloc, cudaFree or other
 * allocating routine; its scratch is a static device array of about 303 KB
 * that every GPU loading the library keeps until the process exits.
 *  - nfields must be 1..PLQCD_NORM2_NOALLOC_MAX_FIELDS; larger batches are
 *    rejected with PLQCD_ERR_ARG.
 *  - The first call on each device (and again after cudaDeviceReset gives
 *    the device a new context) does the set-up: it looks up the scratch
 *    address with cudaGetSymbolAddress and loads the reduction kernel of
 *    every precision. Make that first call before any stream capture.
 *  - All calls on a device share the one scratch array, which keeps the
 *    last call's contents (each call clears the arrival counters it uses):
 *    calls that overlap on the GPU (e.g. from two streams at once) race and
 *    give wrong sums.
 * Counterpart in the reference: none (the reference has no device code). */
#define PLQCD_NORM2_NOALLOC_MAX_FIELDS 32
int plqcd_spinor_norm2_noalloc(plqcd_lattice *lat, const void *fields, int prec, int nfields, double *norms_dev);

/* ---- hopping matrix on device fields ------------------------------------ */
/* out (parity out_parity) = a * H in (in on the other parity) [+ b * x]
 * where a applies to spins 0,1 and a_low to spins 2,3 (gamma5 folding),
 * x may be NULL (then b is ignored). Spinor and gauge precisions must
 * match. */
int plqcd_dslash(plqcd_lattice *lat, const plqcd_gauge *g, void *out, const void *in, int out_parity,
                 int prec, unsigned flags);
int plqcd_dslash_xpay(plqcd_lattice *lat, const plqcd_gauge *g, void *out, const void *in,
                      int out_parity, int prec, unsigned flags, double a, const void *x, double b);
/* The same on the output half-sites [h_begin, h_begin + h_count) only (a
 * t-slab range when it is whole slabs); other sites of out are not written.
 * For a lattice held in t-slabs by several devices: the local lattice
 * carries one ghost t-slice on each side, filled from the neighbouring
 * slabs, and the interior slices are computed with this call. x may be
 * NULL. No reference counterpart (the reference computes its MPI faces
 * inside the hop, lib/dirac.c:124-131, 203-228). */
int plqcd_dslash_sites(plqcd_lattice *lat, const plqcd_gauge *g, void *out, const void *in, int out_parity,
                       int prec, unsigned flags, double a, const void *x, double b, long h_begin, long h_count);
/* Full-lattice H in one launch: out_e = H_eo in_o and out_o = H_oe in_e.
 * Each link is used by two sites of the same launch and read from HBM
 * once. */
int plqcd_dslash_full(plqcd_lattice *lat, const plqcd_gauge *g, void *out_even, void *out_odd,
                      const void *in_even, const void *in_odd, int prec);

/* ---- even/odd preconditioned Wilson solver ------------------------------ */
/* D = 1 - kappa H. CG on Mhat^dag Mhat with Mhat = 1 - kappa^2 H_eo H_oe on
 * even sites, x_o = b_o + kappa H_oe x_e. With a sloppy precision other
 * than F64 the recursion runs in that precision and reliable updates (FP64
 * defect correction of the solution and true residual) keep the result
 * exact to `tol`. */
typedef struct {
    double kappa;     /* hopping parameter */
    double tol;       /* target |b' - Mhat x_e| / |b'| (FP64 true residual) */
    int max_iter;
    int sloppy_prec;  /* PLQCD_F64, F32, F16 or BF16: precision of the inner operator */
    double delta;     /* reliable update when |r| drops below delta * max|r| (mixed only) */
    int verbose;
} plqcd_cg_param;

typedef struct {
    int iterations;
    int reliable_updates;
    int converged;
    double schur_residual;  /* |b' - Mhat x_e| / |b'| in FP64 */
    double true_residual;   /* |b - D x| / |b| on the full lattice, FP64 */
    double seconds;         /* device time of the whole solve */
    double sloppy_hops;     /* half-lattice hopping applications in the sloppy precision */
    double f64_hops;        /* ... and in FP64 */
} plqcd_cg_info;

void plqcd_cg_param_default(plqcd_cg_param *p);
/* x and b are F64 device fields of each parity (x is overwritten). g_sloppy
 * must have precision param->sloppy_prec (NULL: use g64). */
int plqcd_invert_cg(plqcd_lattice *lat, const plqcd_gauge *g64, const plqcd_gauge *g_sloppy, void *x_even,
                    void *x_odd, const void *b_even, const void *b_odd, const plqcd_cg_param *param,
                    plqcd_cg_info *info);

/* ---- autotuner ---------------------------------------------------------- */
/* Kernel launch configurations (load strategy, block size) are chosen by
 * timing the candidates on first use per (kernel, format, lattice, GPU) and
 * persisted as JSON lines in PLQCD_TUNE_FILE (default
 * $HOME/.cache/plqcd_b200/tunecache.json). */
int plqcd_tune_enable(int on);
int plqcd_tune_clear(void);
int plqcd_tune_save(const char *path);   /* NULL = default file */
int plqcd_tune_load(const char *path);   /* NULL = default file */
int plqcd_tune_count(void);
int plqcd_tune_get(const char *key, int *variant, int *block, double *ms);

/* ---- multiple right-hand sides ------------------------------------------ */
/* H applied to nrhs one-parity fields stored back to back (field r at
 * in + r * plqcd_spinor_bytes(lat, prec)). Each link is loaded once per
 * tile of right-hand sides and the tiles of a site range run together, so
 * link traffic is shared by all nrhs fields. The RHS tile and block size are
 * autotuned. */
int plqcd_dslash_mrhs(plqcd_lattice *lat, const plqcd_gauge *g, void *out, const void *in, int nrhs,
                      int out_parity, int prec, unsigned flags);
int plqcd_dslash_mrhs_xpay(plqcd_lattice *lat, const plqcd_gauge *g, void *out, const void *in, int nrhs,
                           int out_parity, int prec, unsigned flags, double a, const void *x, double b);

/* ---- batched multi-RHS solver ------------------------------------------- */
/* One lattice of a batch: nrhs sources b (F64 blocks of each parity, field r
 * at b + r * plqcd_spinor_bytes(lat, PLQCD_F64)) and the solution blocks x. */
typedef struct {
    plqcd_lattice *lat;
    const plqcd_gauge *g64;       /* F64 links (reliable updates, setup) */
    const plqcd_gauge *g_sloppy;  /* links in param->sloppy_prec (NULL: g64) */
    int nrhs;
    void *x_even, *x_odd;
    const void *b_even, *b_odd;
} plqcd_solve_item;

typedef struct {
    int iterations;            /* iterations of the batch loop */
    int reliable_updates;      /* FP64 reliable updates (batch-wide) */
    int converged;             /* every RHS reached tol */
    double max_schur_residual; /* max over RHS of |b' - Mhat x_e| / |b'| */
    double max_true_residual;  /* max over RHS of |b - D x| / |b| (FP64, after the solve) */
    double seconds;            /* device time of the solve */
    int graph_launches;        /* 1 when the loop ran as one CUDA-graph launch */
} plqcd_batch_info;

/* Solve D x = b for every RHS of every lattice in `items` (same device):
 * one CG recursion per RHS on Mhat^dag Mhat, hopping kernels on whole RHS
 * blocks, FP64 reliable updates when param->sloppy_prec is not F64. With
 * use_graph the iteration loop is captured once into a CUDA graph whose
 * WHILE and IF conditional nodes are set by device code, and runs as a
 * single graph launch. true_residuals (optional) receives |b - D x|/|b| per
 * RHS in item order. */
int plqcd_invert_cg_batch(plqcd_solve_item *items, int nitems, const plqcd_cg_param *param, int use_graph,
                          plqcd_batch_info *info, double *true_residuals);

/* ---- self-test ------------------------------------------------------------ */
/* Known-answer test on `device`: with unit links, H applied to a point
 * source is non-zero at exactly the 8 neighbours, carrying columns of
 * (1 -/+ g_mu) (the neighbour pattern of the reference's
 * tests/test_comms.c:167-497, here with the gamma structure); then
 * gamma5-hermiticity on random fields. Returns PLQCD_OK or an error. */
int plqcd_selftest(int device, int verbose);

/* ---- drop-in path controls ---------------------------------------------- */
/* Register the host link array `u` of the drop-in hopping calls as
 * current: the next call that passes `u` uploads it, and later calls with
 * `u` reuse the device copy until the next plqcd_gauge_update (or
 * finalize_plqcd). Call it again after changing the links in place. For the
 * lane-packed names pass the su3_256 / su3_512 array, for the split family
 * the u_re plane. NULL clears the registration, and every device copy is
 * reloaded on its next use. Without a registration every call uploads its
 * links, as the reference reads them on every call. Environment:
 * PLQCD_GAUGE_CACHE=0 uploads on every call even when registered;
 * PLQCD_GAUGE_CACHE=1 keeps any link array by address plus a fingerprint
 * of sampled words, for callers that never change links in place. */
int plqcd_gauge_update(const su3 *u);
/* Device time (ms) of the kernels of the last drop-in hopping call and its
 * host<->device byte counts. */
int plqcd_dropin_last_stats(double *kernel_ms, double *h2d_bytes, double *d2h_bytes);

/* ---- site-range vector operations (t-slab solver) ------------------------- */
/* FP64 operations of the even/odd CG on the half-sites [h_begin, h_begin +
 * h_count) of one-parity F64 fields (plqcd_b200/shard.py runs its slab CG on
 * the slab interior with them; no reference counterpart, the reference has
 * no solver: include/plqcd_global_params.h:197-201). Asynchronous on the
 * lattice stream; reductions accumulate in FP64 in a fixed order and write
 * one double to device memory; scalars are read from device memory, so no
 * host round trip is needed. Reduction scratch comes from the lattice's
 * device workspace.
 *   sites_norm2:     *out_dev = sum |x|^2
 *   sites_cg_update: alpha = coef_dev[0] / coef_dev[1] (rr / pAp);
 *                    x += alpha p; r -= alpha Ap; *rr_dev = sum |r|^2
 *   sites_xpay:      beta = coef_dev[0] / coef_dev[1]; p = r + beta p
 *   sites_sub_norm2: z = x - y; *out_dev = sum |z|^2
 * out_dev, rr_dev and coef_dev must be 8-byte aligned device pointers. */
int plqcd_sites_norm2(plqcd_lattice *lat, const void *x, long h_begin, long h_count, double *out_dev);
int plqcd_sites_cg_update(plqcd_lattice *lat, void *x, void *r, const void *p, const void *Ap, long h_begin,
                          long h_count, const double *coef_dev, double *rr_dev);
int plqcd_sites_xpay(plqcd_lattice *lat, void *p, const void *r, long h_begin, long h_count,
                     const double *coef_dev);
int plqcd_sites_sub_norm2(plqcd_lattice *lat, void *z, const void *x, const void *y, long h_begin, long h_count,
                          double *out_dev);

/* Copy n device segments (dst[k] <- src[k], bytes[k] bytes each) in one
 * launch on the lattice stream: the ghost-slice exchange of a t-slab
 * decomposition held on one device (one run per SoA plane, direction and
 * slab). Every pointer and size must be a multiple of 16 bytes; segments
 * must not overlap; n <= PLQCD_COPY_MAX_SEGMENTS. */
#define PLQCD_COPY_MAX_SEGMENTS 128
int plqcd_copy_segments(plqcd_lattice *lat, int n, void *const *dst, const void *const *src, const size_t *bytes);

/* ---- failure detection ----------------------------------------------------- */
/* Test hook of the bounded waits in the TMA-staged hopping kernels (no
 * reference counterpart: the reference calls exit(1) when a face exchange
 * fails, lib/dirac.c:128-130). With `enable` non-zero, every later launch
 * of a TMA kernel in this process makes each consumer warp first wait, with
 * a limit of `limit_ns` (1 us .. 2 s), on a shared-memory barrier that
 * nothing completes. The wait runs out, the warps stop, the producer waits
 * (bounded) for the tile loads it has in flight, the kernel returns, and
 * the next plqcd_lattice_synchronize (or solver) reports PLQCD_ERR_TIMEOUT
 * and clears the flag; that launch's output is incomplete. enable = 0
 * restores normal operation. Nothing faults, traps or hangs. */
int plqcd_tma_timeout_test(int enable, unsigned long long limit_ns);

/* ---- host layout converters for the split entry points ------------------- */
/* No reference counterpart: the reference leaves packing to its callers.
 * API-layout arrays (interleaved complex doubles: spinors 12 per site,
 * links 9 per link, in even/odd site order) <-> the split real / imaginary
 * planes that the split family of include/dirac.h takes (re[k], im[k] =
 * parts of complex number k). n = number of complex numbers. Host memory,
 * multi-threaded for large n. Returns PLQCD_OK, or PLQCD_ERR_ARG for a null
 * pointer or a negative n. */
int plqcd_aos_to_split(const double *aos, double *re, double *im, long n);
int plqcd_split_to_aos(const double *re, const double *im, double *aos, long n);

#ifdef __cplusplus
}
#endif
#endif
