// internal.h -- shared declarations of the plqcd-b200 library (not installed).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>

#include "plqcd_b200.h"

namespace plqcd {

// ---- error state (thread-local; read through plqcd_last_error) ----------
int set_error(int code, const char *fmt, ...);
void clear_error();

#define PLQCD_CUDA_TRY(expr)                                                              \
    do {                                                                                  \
        cudaError_t _e = (expr);                                                          \
        if (_e != cudaSuccess)                                                            \
            return ::plqcd::set_error(PLQCD_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, \
                                      #expr, cudaGetErrorString(_e));                     \
    } while (0)

#define PLQCD_TRY(expr)               \
    do {                              \
        int _s = (expr);              \
        if (_s != PLQCD_OK) return _s; \
    } while (0)

// Device fields are read and written with 16-byte vector and tile loads: a
// pointer that is not 16-byte aligned is refused before any launch.
inline int check_field_ptr(const void *p, const char *what) {
    if (!p) return set_error(PLQCD_ERR_ARG, "%s: null field pointer", what);
    if (reinterpret_cast<uintptr_t>(p) & 15u)
        return set_error(PLQCD_ERR_ARG, "%s: field pointer %p is not 16-byte aligned", what, p);
    return PLQCD_OK;
}

// ---- geometry --------------------------------------------------------------
struct Geom {
    int L[4];
    int L0h;     // L0 / 2
    long Vh;     // V / 2
};

inline bool dims_ok(const int d[4]) {
    for (int k = 0; k < 4; k++)
        if (d[k] < 2 || (d[k] & 1)) return false;
    return true;
}

// ---- element sizes / counts ------------------------------------------------
// bytes of one parity of a spinor field
size_t spinor_parity_bytes(long Vh, int prec);
// number of stored "elements" (planes) per link and bytes per element
int gauge_elems(int prec, int recon);
size_t gauge_elem_bytes(int prec, int recon);
size_t gauge_total_bytes(long Vh, int prec, int recon);
bool gauge_format_ok(int prec, int recon);

}  // namespace plqcd

// ---- opaque objects ----------------------------------------------------------
struct plqcd_lattice {
    plqcd::Geom geom;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_kernel_ms = 0.0;
    // solver workspace (grown on demand, released with the lattice)
    void *ws = nullptr;
    size_t ws_bytes = 0;
};

struct plqcd_gauge {
    plqcd_lattice *lat = nullptr;
    int prec = PLQCD_F64;
    int recon = 18;
    void *data = nullptr;
    size_t bytes = 0;
};

namespace plqcd {

// ---- kernels (fields.cu) ------------------------------------------------------
// half-sites [first, first + count) of one parity (count < 0: to the end)
int launch_spinor_import(const Geom &g, cudaStream_t s, const void *aos, int parity, void *dst, int prec,
                         long first = 0, long count = -1);
int launch_spinor_export(const Geom &g, cudaStream_t s, const void *src, int prec, int parity, void *aos,
                         long first = 0, long count = -1);
int launch_spinor_convert(const Geom &g, cudaStream_t s, void *dst, int dprec, const void *src, int sprec);
// split real / imaginary planes of one parity (12 doubles per site each)
int launch_spinor_import_split(const Geom &g, cudaStream_t s, const double *re, const double *im, void *dst,
                               int prec);
int launch_spinor_export_split(const Geom &g, cudaStream_t s, const void *src, int prec, double *re, double *im);
// links [first, first + n) from split planes (9 doubles per link each)
int launch_gauge_import_split(const Geom &g, cudaStream_t s, const double *re, const double *im, long first, long n,
                              void *dst, int prec, int recon);
int launch_spinor_gaussian(const Geom &g, cudaStream_t s, void *dst, int prec, int parity, uint64_t seed);
int launch_gauge_import(const Geom &g, cudaStream_t s, const void *aos, long first_link, long nlinks,
                        void *dst, int prec, int recon);
int launch_gauge_export(const Geom &g, cudaStream_t s, const void *src, int prec, int recon, void *aos);
int launch_gauge_random(const Geom &g, cudaStream_t s, void *dst, int prec, int recon, uint64_t seed);
int launch_gauge_unit(const Geom &g, cudaStream_t s, void *dst, int prec, int recon);
int launch_gauge_copy(const Geom &g, cudaStream_t s, void *dst, int dprec, int drecon, const void *src,
                      int sprec, int srecon);

// ---- hopping kernels (dslash.cu) ---------------------------------------------
struct DslashCall {
    const void *gauge = nullptr;
    int prec = PLQCD_F64;
    int recon = 18;
    void *out = nullptr;
    const void *in = nullptr;
    int out_parity = 0;
    unsigned flags = 0;
    // epilogue: out = a_up/a_low * H in + b * x   (x may be null)
    double a_up = 1.0, a_low = 1.0, b = 0.0;
    const void *x = nullptr;
    // full-lattice mode
    bool full = false;
    void *out2 = nullptr;      // odd output in full mode (out = even output)
    const void *in2 = nullptr; // odd input in full mode (in = even input)
    int block = 0;             // 0 = library default
    // output half-sites [h_begin, h_begin + h_count) (single parity; -1 = all)
    long h_begin = 0, h_count = -1;
    // single parity: in/out/x are blocks of nrhs fields back to back
    int nrhs = 1;
};
int launch_dslash(const Geom &g, cudaStream_t s, const DslashCall &c);
// TMA-staged hop (dslash_tma.cu): variant 1000 * kind + 100 * nstage + ny
// selects the kernel (kind 1: one stage per direction; 2, 3: own-line rows
// staged once per tile, in 1 or 2 buffers of their own; 4, 5: the same with
// one tile-load box per ring stage), nstage ring buffers and ny rows per
// tile. `plan` checks that the configuration exists for this lattice and
// format and gives block / bytes.
int dslash_tma_plan(const Geom &g, int prec, int recon, int kind, int nstage, int ny, int *block, size_t *smem,
                    int nr = 1);
// TMA-staged hop on a block of nrhs one-parity FP64 fields with RHS tiles
// (own-line kinds 2 and 4 with nr RHS per tile; nrhs % nr == 0): the
// variant 100000 * nr + 1000 * kind + 100 * nstage + ny of the multi-RHS
// tuner. out = a * H in (+ b * x if x != null), flags as launch_dslash_mrhs
int launch_dslash_tma_mrhs(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                           const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x,
                           double b, int kind, int nstage, int ny, int nr);
// the device flag a TMA stage wait sets when it runs out (reset: clear it)
int dslash_tma_status(bool reset);
// variant 0: direct loads, 2/3: cp.async pipeline depth; no tuning
int launch_dslash_config(const Geom &g, cudaStream_t s, const DslashCall &c, int variant, int block);
// nrhs one-parity fields back to back: out = a * H in (+ b * x if x != null)
int launch_dslash_mrhs(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                       const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x, double b);
// true when launch_dslash_mrhs of this configuration would not tune
bool dslash_mrhs_tuned(const Geom &g, int prec, int recon, int nrhs, bool xpay);

// CG dot products fused into the epilogue of a multi-RHS xpay hop (the
// RHS-pair kernels): per-RHS FP64 sums, per-block partials summed in a fixed
// order by a one-block-per-RHS kernel after the hop, applied to the solver's
// scalars of every active RHS.
//   epi 1: out = t as usual; pAp = |t|^2, alpha = rr / pAp
//   epi 2: out = Ap is not stored; r -= alpha Ap in place (rvec);
//          rr_old = rr, rr = |r|^2, beta = rr / rr_old
//   epi 3: out as usual; rr = |out|^2, beta = rr / rr_old (the restart of
//          a reliable update); RHS pairs that are both retired are skipped
//   epi 4: a plain hop (x null), no sums; retired RHS pairs are skipped
struct RhsSink {
    double *partials;    // nrhs * ceil(Vh / 32) doubles
    double *rr, *rr_old, *pAp, *alpha, *beta;
    const int *active;
    char *rvec;
};
// the tuned xpay configuration of this multi-RHS hop is an RHS-pair kernel,
// so launch_dslash_mrhs_sink can run it
bool dslash_mrhs_sink_ok(const Geom &g, int prec, int recon, int nrhs, int *variant = nullptr, int *block = nullptr);
int launch_dslash_mrhs_sink(const Geom &g, cudaStream_t s, const void *gauge, int prec, int recon, void *out,
                            const void *in, int nrhs, int out_parity, unsigned flags, double a, const void *x,
                            double b, int epi, const RhsSink &sink);

// dynamic shared-memory opt-in of kernel `func` on the current device, set
// once per (kernel, device) to at least `bytes` (utils.cpp)
int smem_optin(const void *func, size_t bytes);

// ID of the current CUDA context (unique within the process, never reused;
// a cudaDeviceReset gives the device a new one), 0 when the driver does not
// provide it (utils.cpp)
unsigned long long current_context_id();

// device workspace of at least `bytes`, owned by the lattice (cg.cu)
int lattice_workspace(plqcd_lattice *lat, size_t bytes, void **out);

}  // namespace plqcd
