// dropin.cu -- the reference's hopping entry points on host arrays
// (include/dirac.h; reference lib/dirac.c:35-791).
//
// Each call copies the input parity of `qin` (API layout, host) to the
// device, converts it to the kernel layout, runs the sm_100a hopping kernel
// and copies the output parity back into `qout`; the other half of `qout` is
// not touched, as in the reference. The gauge field is uploaded on first use
// and kept on the device keyed by its host address plus a fingerprint of
// 1024 sampled doubles; plqcd_gauge_update() or PLQCD_GAUGE_CACHE=0 force a
// fresh upload. The return value is the call's wall-clock seconds
// (lib/dirac.c:405-407), or -1 on failure with the reason in
// plqcd_last_error(). Calls are serialised (the reference is not
// re-entrant either: lib/dirac.c:12-13 and the global phip/phim buffers).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "dirac.h"
#include "internal.h"

using namespace plqcd;

namespace {

constexpr int kMaxChunks = 8;

struct DropIn {
    int dims[4] = {0, 0, 0, 0};
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr;  // copy streams
    cudaEvent_t ev_in[kMaxChunks] = {}, ev_out[kMaxChunks] = {}, ev_k0[kMaxChunks] = {}, ev_k1[kMaxChunks] = {};
    plqcd_lattice *lat = nullptr;
    plqcd_gauge *gauge = nullptr;
    void *aos_in = nullptr, *aos_out = nullptr;  // API layout staging, one parity
    void *f_in = nullptr, *f_out = nullptr;      // kernel layout (F64), one parity
    const su3 *cached_u = nullptr;
    uint64_t fingerprint = 0;
    bool dirty = true;
    cudaStream_t stream = nullptr;  // owned by the drop-in path
    double kernel_ms = 0, h2d = 0, d2h = 0;
};

std::mutex g_mu;
DropIn g_d;

void release_locked() {
    if (g_d.lat) cudaSetDevice(g_d.lat->device);
    if (g_d.gauge) plqcd_gauge_destroy(g_d.gauge);
    void *bufs[4] = {g_d.aos_in, g_d.aos_out, g_d.f_in, g_d.f_out};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (int c = 0; c < kMaxChunks; c++)
        for (cudaEvent_t ev : {g_d.ev_in[c], g_d.ev_out[c], g_d.ev_k0[c], g_d.ev_k1[c]})
            if (ev) cudaEventDestroy(ev);
    if (g_d.s_h2d) cudaStreamDestroy(g_d.s_h2d);
    if (g_d.s_d2h) cudaStreamDestroy(g_d.s_d2h);
    if (g_d.lat) plqcd_lattice_destroy(g_d.lat);
    if (g_d.stream) cudaStreamDestroy(g_d.stream);
    g_d = DropIn();
}

bool env_flag(const char *name, bool dflt) {
    const char *v = getenv(name);
    if (!v || !*v) return dflt;
    return !(v[0] == '0' || v[0] == 'n' || v[0] == 'N' || v[0] == 'f' || v[0] == 'F');
}

uint64_t fingerprint(const su3 *u, long nlinks) {
    const uint64_t *w = reinterpret_cast<const uint64_t *>(u);
    long nwords = nlinks * 18;
    uint64_t h = 1469598103934665603ULL;
    const int samples = 1024;
    for (int k = 0; k < samples; k++) {
        long idx = (long)((double)k / samples * nwords);
        h = (h ^ w[idx]) * 1099511628211ULL;
    }
    h = (h ^ w[nwords - 1]) * 1099511628211ULL;
    return h;
}

int ensure_locked() {
    if (!plqcd_g.init) return set_error(PLQCD_ERR_STATE, "hopping matrix called before init_plqcd");
    const int *L = plqcd_g.latdims;
    if (g_d.lat && memcmp(g_d.dims, L, sizeof g_d.dims) == 0) return PLQCD_OK;
    release_locked();
    int dev = 0;
    if (const char *e = getenv("PLQCD_DEVICE")) dev = atoi(e);
    cudaStream_t stream = nullptr;
    if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return set_error(PLQCD_ERR_CUDA, "drop-in: cannot create a stream on device %d", dev);
    }
    if (plqcd_lattice_create(L, dev, stream, &g_d.lat) != PLQCD_OK) {
        cudaStreamDestroy(stream);
        return plqcd_last_status();
    }
    g_d.stream = stream;
    memcpy(g_d.dims, L, sizeof g_d.dims);
    int rc = plqcd_gauge_create(g_d.lat, PLQCD_F64, 18, &g_d.gauge);
    if (rc != PLQCD_OK) {
        release_locked();
        return rc;
    }
    size_t bytes = spinor_parity_bytes(g_d.lat->geom.Vh, PLQCD_F64);
    void **bufs[4] = {&g_d.aos_in, &g_d.aos_out, &g_d.f_in, &g_d.f_out};
    for (void **b : bufs)
        if (cudaMalloc(b, bytes) != cudaSuccess) {
            cudaGetLastError();
            release_locked();
            return set_error(PLQCD_ERR_NOMEM, "drop-in: device allocation of %zu bytes failed", bytes);
        }
    bool ok = cudaStreamCreateWithFlags(&g_d.s_h2d, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&g_d.s_d2h, cudaStreamNonBlocking) == cudaSuccess;
    for (int c = 0; c < kMaxChunks && ok; c++)
        ok = cudaEventCreateWithFlags(&g_d.ev_in[c], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&g_d.ev_out[c], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreate(&g_d.ev_k0[c]) == cudaSuccess && cudaEventCreate(&g_d.ev_k1[c]) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        release_locked();
        return set_error(PLQCD_ERR_CUDA, "drop-in: stream/event creation failed");
    }
    g_d.dirty = true;
    return PLQCD_OK;
}

// out_parity 0: eo (qout even half from qin odd half); 1: oe.
double hop_call(spinor *qin, spinor *qout, su3 *u, int out_parity) {
    double t0 = stop_watch(0.0);
    clear_error();
    if (!qin || !qout || !u) {
        set_error(PLQCD_ERR_ARG, "hopping matrix: null argument");
        return -1.0;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (ensure_locked() != PLQCD_OK) return -1.0;
    plqcd_lattice *lat = g_d.lat;
    const long Vh = lat->geom.Vh;
    cudaStream_t s = lat->stream;
    if (cudaSetDevice(lat->device) != cudaSuccess) {
        set_error(PLQCD_ERR_CUDA, "hopping matrix: cudaSetDevice failed");
        return -1.0;
    }
    g_d.h2d = g_d.d2h = 0;

    // gauge field: upload when new, changed or caching is disabled
    uint64_t fp = fingerprint(u, 8 * Vh);
    if (!env_flag("PLQCD_GAUGE_CACHE", true) || g_d.dirty || g_d.cached_u != u || g_d.fingerprint != fp) {
        if (plqcd_gauge_load_host(g_d.gauge, u) != PLQCD_OK) return -1.0;
        g_d.cached_u = u;
        g_d.fingerprint = fp;
        g_d.dirty = false;
        g_d.h2d += 8.0 * Vh * sizeof(su3);
    }

    // Pipeline over chunks of t-slabs (contiguous half-site ranges): input
    // chunks go up on the copy stream in the order last, 0, 1, ..., and
    // output chunk c is computed once input chunks c-1, c, c+1 (periodic)
    // have arrived, then copied back on a second copy stream while later
    // chunks are still in flight; host->device and device->host transfers
    // overlap each other and the kernels.
    const int in_parity = out_parity ^ 1;
    const unsigned flags = env_flag("PLQCD_REF_COMPAT", false) ? PLQCD_DSLASH_COMPAT : 0u;
    const Geom &geo = lat->geom;
    const int L3 = geo.L[3];
    const long slab = geo.Vh / L3;
    const int nch = L3 < kMaxChunks ? L3 : kMaxChunks;
    auto first = [&](int c) { return slab * (long)((long)c * L3 / nch); };
    auto count = [&](int c) { return first(c + 1) - first(c); };
    const spinor *src = qin + in_parity * Vh;
    spinor *dst = qout + out_parity * Vh;
    spinor *ain = static_cast<spinor *>(g_d.aos_in), *aout = static_cast<spinor *>(g_d.aos_out);
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < nch && e == cudaSuccess; k++) {
        const int c = (k == 0) ? nch - 1 : k - 1;
        e = cudaMemcpyAsync(ain + first(c), src + first(c), count(c) * sizeof(spinor), cudaMemcpyHostToDevice,
                            g_d.s_h2d);
        // staging holds one parity, so it is addressed as parity 0
        if (e == cudaSuccess &&
            launch_spinor_import(geo, g_d.s_h2d, ain, 0, g_d.f_in, PLQCD_F64, first(c), count(c)) != PLQCD_OK)
            return -1.0;
        if (e == cudaSuccess) e = cudaEventRecord(g_d.ev_in[c], g_d.s_h2d);
    }
    for (int c = 0; c < nch && e == cudaSuccess; c++) {
        for (int d : {c - 1, c, c + 1}) cudaStreamWaitEvent(s, g_d.ev_in[(d + nch) % nch], 0);
        cudaEventRecord(g_d.ev_k0[c], s);
        DslashCall dc;
        dc.gauge = g_d.gauge->data;
        dc.prec = PLQCD_F64;
        dc.recon = 18;
        dc.out = g_d.f_out;
        dc.in = g_d.f_in;
        dc.out_parity = out_parity;
        dc.flags = flags;
        dc.h_begin = first(c);
        dc.h_count = count(c);
        if (launch_dslash(geo, s, dc) != PLQCD_OK) return -1.0;
        cudaEventRecord(g_d.ev_k1[c], s);
        if (launch_spinor_export(geo, s, g_d.f_out, PLQCD_F64, 0, aout, first(c), count(c)) != PLQCD_OK) return -1.0;
        cudaEventRecord(g_d.ev_out[c], s);
        cudaStreamWaitEvent(g_d.s_d2h, g_d.ev_out[c], 0);
        e = cudaMemcpyAsync(dst + first(c), aout + first(c), count(c) * sizeof(spinor), cudaMemcpyDeviceToHost,
                            g_d.s_d2h);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(g_d.s_d2h);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(PLQCD_ERR_CUDA, "hopping matrix: %s", cudaGetErrorString(e));
        return -1.0;
    }
    g_d.h2d += (double)Vh * sizeof(spinor);
    g_d.d2h += (double)Vh * sizeof(spinor);
    double kms = 0;
    for (int c = 0; c < nch; c++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, g_d.ev_k0[c], g_d.ev_k1[c]);
        kms += ms;
    }
    g_d.kernel_ms = kms;
    lat->last_kernel_ms = kms;
    return stop_watch(t0);
}

}  // namespace

namespace plqcd {
void dropin_release() {
    std::lock_guard<std::mutex> lk(g_mu);
    release_locked();
}
}  // namespace plqcd

extern "C" int plqcd_gauge_update(const su3 *u) {
    std::lock_guard<std::mutex> lk(g_mu);
    (void)u;
    g_d.dirty = true;
    return PLQCD_OK;
}

extern "C" int plqcd_dropin_last_stats(double *kernel_ms, double *h2d, double *d2h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (kernel_ms) *kernel_ms = g_d.kernel_ms;
    if (h2d) *h2d = g_d.h2d;
    if (d2h) *d2h = g_d.d2h;
    return PLQCD_OK;
}

// lib/dirac.c:35 and :414, plus the same-signature SSE3 names of
// lib/dirac.c:801, 1272, 1748, 2124.
extern "C" double plqcd_hopping_matrix_eo_sse3_assymbly(spinor *qin, spinor *qout, su3 *u) {
    return hop_call(qin, qout, u, 0);
}
extern "C" double plqcd_hopping_matrix_oe_sse3_assymbly(spinor *qin, spinor *qout, su3 *u) {
    return hop_call(qin, qout, u, 1);
}
extern "C" double plqcd_hopping_matrix_eo_sse3_intrin(spinor *qin, spinor *qout, su3 *u) {
    return hop_call(qin, qout, u, 0);
}
extern "C" double plqcd_hopping_matrix_oe_sse3_intrin(spinor *qin, spinor *qout, su3 *u) {
    return hop_call(qin, qout, u, 1);
}
extern "C" double plqcd_hopping_matrix_eo_sse3_intrin_blocking(spinor *qin, spinor *qout, su3 *u) {
    return hop_call(qin, qout, u, 0);
}
extern "C" double plqcd_hopping_matrix_oe_sse3_intrin_blocking(spinor *qin, spinor *qout, su3 *u) {
    return hop_call(qin, qout, u, 1);
}
