// api.cu -- C-ABI of the device-resident API (include/plqcd_b200.h).
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <new>

#include "internal.h"

using namespace plqcd;

namespace {

int check_lat(const plqcd_lattice *lat) {
    if (!lat) return set_error(PLQCD_ERR_ARG, "null lattice");
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    return PLQCD_OK;
}

int check_prec(int prec) {
    if (prec < PLQCD_F64 || prec > PLQCD_BF16) return set_error(PLQCD_ERR_ARG, "unknown precision %d", prec);
    return PLQCD_OK;
}

}  // namespace

extern "C" int plqcd_lattice_create(const int dims[4], int device, void *stream, plqcd_lattice **out) {
    clear_error();
    if (!dims || !out) return set_error(PLQCD_ERR_ARG, "plqcd_lattice_create: null argument");
    *out = nullptr;
    if (!dims_ok(dims))
        return set_error(PLQCD_ERR_ARG, "plqcd_lattice_create: extents must be even and >= 2 (got %d %d %d %d)",
                         dims[0], dims[1], dims[2], dims[3]);
    long V = (long)dims[0] * dims[1] * dims[2] * dims[3];
    if (V / 2 >= (1L << 31)) return set_error(PLQCD_ERR_ARG, "plqcd_lattice_create: volume too large");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(PLQCD_ERR_NODEV, "plqcd_lattice_create: no CUDA device");
    }
    if (device < 0 || device >= n) return set_error(PLQCD_ERR_ARG, "plqcd_lattice_create: bad device %d", device);
    PLQCD_CUDA_TRY(cudaSetDevice(device));
    plqcd_lattice *lat = new (std::nothrow) plqcd_lattice();
    if (!lat) return set_error(PLQCD_ERR_NOMEM, "plqcd_lattice_create: out of host memory");
    for (int k = 0; k < 4; k++) lat->geom.L[k] = dims[k];
    lat->geom.L0h = dims[0] / 2;
    lat->geom.Vh = V / 2;
    lat->device = device;
    // NULL selects the device's default stream, as everywhere in CUDA
    lat->stream = (cudaStream_t)stream;
    cudaError_t e = cudaEventCreate(&lat->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&lat->ev1);
    if (e != cudaSuccess) {
        plqcd_lattice_destroy(lat);
        return set_error(PLQCD_ERR_CUDA, "plqcd_lattice_create: %s", cudaGetErrorString(e));
    }
    *out = lat;
    return PLQCD_OK;
}

extern "C" int plqcd_lattice_destroy(plqcd_lattice *lat) {
    if (!lat) return PLQCD_OK;
    cudaSetDevice(lat->device);
    if (lat->stream) cudaStreamSynchronize(lat->stream);
    if (lat->ws) cudaFree(lat->ws);
    if (lat->ev0) cudaEventDestroy(lat->ev0);
    if (lat->ev1) cudaEventDestroy(lat->ev1);
    delete lat;
    return PLQCD_OK;
}

extern "C" int plqcd_lattice_set_stream(plqcd_lattice *lat, void *stream) {
    PLQCD_TRY(check_lat(lat));
    PLQCD_CUDA_TRY(cudaStreamSynchronize(lat->stream));
    lat->stream = (cudaStream_t)stream;
    return PLQCD_OK;
}

extern "C" int plqcd_lattice_synchronize(plqcd_lattice *lat) {
    PLQCD_TRY(check_lat(lat));
    PLQCD_CUDA_TRY(cudaStreamSynchronize(lat->stream));
    if (dslash_tma_status(true))
        return set_error(PLQCD_ERR_TIMEOUT, "dslash: a TMA stage wait ran out; that launch's output is incomplete");
    return PLQCD_OK;
}

extern "C" void *plqcd_lattice_stream(const plqcd_lattice *lat) { return lat ? (void *)lat->stream : nullptr; }
extern "C" long plqcd_lattice_half_volume(const plqcd_lattice *lat) { return lat ? lat->geom.Vh : 0; }
extern "C" double plqcd_lattice_last_kernel_ms(const plqcd_lattice *lat) { return lat ? lat->last_kernel_ms : 0; }

extern "C" size_t plqcd_spinor_bytes(const plqcd_lattice *lat, int prec) {
    return lat ? spinor_parity_bytes(lat->geom.Vh, prec) : 0;
}

extern "C" size_t plqcd_gauge_bytes(const plqcd_lattice *lat, int prec, int recon) {
    return lat ? gauge_total_bytes(lat->geom.Vh, prec, recon) : 0;
}

// ---- gauge ---------------------------------------------------------------------

extern "C" int plqcd_gauge_create(plqcd_lattice *lat, int prec, int recon, plqcd_gauge **out) {
    clear_error();
    if (!out) return set_error(PLQCD_ERR_ARG, "plqcd_gauge_create: null output");
    *out = nullptr;
    PLQCD_TRY(check_lat(lat));
    if (!gauge_format_ok(prec, recon))
        return set_error(PLQCD_ERR_ARG, "plqcd_gauge_create: unsupported format prec=%d recon=%d", prec, recon);
    plqcd_gauge *g = new (std::nothrow) plqcd_gauge();
    if (!g) return set_error(PLQCD_ERR_NOMEM, "plqcd_gauge_create: out of host memory");
    g->lat = lat;
    g->prec = prec;
    g->recon = recon;
    g->bytes = gauge_total_bytes(lat->geom.Vh, prec, recon);
    cudaError_t e = cudaMalloc(&g->data, g->bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete g;
        return set_error(PLQCD_ERR_NOMEM, "plqcd_gauge_create: cudaMalloc(%zu): %s", (size_t)g->bytes,
                         cudaGetErrorString(e));
    }
    *out = g;
    return PLQCD_OK;
}

extern "C" int plqcd_gauge_destroy(plqcd_gauge *g) {
    if (!g) return PLQCD_OK;
    cudaSetDevice(g->lat->device);
    cudaStreamSynchronize(g->lat->stream);
    cudaFree(g->data);
    delete g;
    return PLQCD_OK;
}

extern "C" void *plqcd_gauge_data(plqcd_gauge *g) { return g ? g->data : nullptr; }

// Upload in chunks through a bounded device staging buffer so a 48^3x96
// field (5.7 GB in the API layout) needs no second full-size copy.
static int gauge_load(plqcd_gauge *g, const su3 *u, bool host) {
    clear_error();
    if (!g || !u) return set_error(PLQCD_ERR_ARG, "plqcd_gauge_load: null argument");
    PLQCD_TRY(check_lat(g->lat));
    const Geom &geo = g->lat->geom;
    cudaStream_t s = g->lat->stream;
    long nlinks = 8 * geo.Vh;
    if (!host) return launch_gauge_import(geo, s, u, 0, nlinks, g->data, g->prec, g->recon);
    const long chunk = 1L << 20;  // links per chunk (144 MiB)
    void *stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    long per = nlinks < chunk ? nlinks : chunk;
    int rc = PLQCD_OK;
    for (int k = 0; k < 2 && rc == PLQCD_OK; k++) {
        if (cudaMalloc(&stage[k], per * sizeof(su3)) != cudaSuccess ||
            cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            rc = set_error(PLQCD_ERR_NOMEM, "plqcd_gauge_load_host: staging allocation failed");
        }
    }
    for (long first = 0, it = 0; rc == PLQCD_OK && first < nlinks; first += per, it++) {
        long n = nlinks - first < per ? nlinks - first : per;
        int k = (int)(it & 1);
        cudaError_t e = cudaEventSynchronize(done[k]);  // staging slot free again
        if (e == cudaSuccess) e = cudaMemcpyAsync(stage[k], u + first, n * sizeof(su3), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            rc = set_error(PLQCD_ERR_CUDA, "plqcd_gauge_load_host: %s", cudaGetErrorString(e));
            break;
        }
        rc = launch_gauge_import(geo, s, stage[k], first, n, g->data, g->prec, g->recon);
        if (rc == PLQCD_OK && cudaEventRecord(done[k], s) != cudaSuccess)
            rc = set_error(PLQCD_ERR_CUDA, "plqcd_gauge_load_host: event record failed");
    }
    cudaStreamSynchronize(s);
    for (int k = 0; k < 2; k++) {
        if (stage[k]) cudaFree(stage[k]);
        if (done[k]) cudaEventDestroy(done[k]);
    }
    return rc;
}

extern "C" int plqcd_gauge_load_host(plqcd_gauge *g, const su3 *u) { return gauge_load(g, u, true); }
extern "C" int plqcd_gauge_load_device(plqcd_gauge *g, const su3 *u) { return gauge_load(g, u, false); }

extern "C" int plqcd_gauge_store_host(const plqcd_gauge *g, su3 *u) {
    clear_error();
    if (!g || !u) return set_error(PLQCD_ERR_ARG, "plqcd_gauge_store_host: null argument");
    PLQCD_TRY(check_lat(g->lat));
    const Geom &geo = g->lat->geom;
    void *tmp = nullptr;
    size_t bytes = (size_t)8 * geo.Vh * sizeof(su3);
    if (cudaMalloc(&tmp, bytes) != cudaSuccess) {
        cudaGetLastError();
        return set_error(PLQCD_ERR_NOMEM, "plqcd_gauge_store_host: staging allocation failed");
    }
    int rc = launch_gauge_export(geo, g->lat->stream, g->data, g->prec, g->recon, tmp);
    if (rc == PLQCD_OK) {
        cudaError_t e = cudaMemcpyAsync(u, tmp, bytes, cudaMemcpyDeviceToHost, g->lat->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->lat->stream);
        if (e != cudaSuccess) rc = set_error(PLQCD_ERR_CUDA, "plqcd_gauge_store_host: %s", cudaGetErrorString(e));
    }
    cudaFree(tmp);
    return rc;
}

extern "C" int plqcd_gauge_random(plqcd_gauge *g, uint64_t seed) {
    clear_error();
    if (!g) return set_error(PLQCD_ERR_ARG, "plqcd_gauge_random: null gauge");
    PLQCD_TRY(check_lat(g->lat));
    return launch_gauge_random(g->lat->geom, g->lat->stream, g->data, g->prec, g->recon, seed);
}

extern "C" int plqcd_gauge_unit(plqcd_gauge *g) {
    clear_error();
    if (!g) return set_error(PLQCD_ERR_ARG, "plqcd_gauge_unit: null gauge");
    PLQCD_TRY(check_lat(g->lat));
    return launch_gauge_unit(g->lat->geom, g->lat->stream, g->data, g->prec, g->recon);
}

extern "C" int plqcd_gauge_copy(plqcd_gauge *dst, const plqcd_gauge *src) {
    clear_error();
    if (!dst || !src) return set_error(PLQCD_ERR_ARG, "plqcd_gauge_copy: null argument");
    if (dst->lat->geom.Vh != src->lat->geom.Vh || memcmp(dst->lat->geom.L, src->lat->geom.L, sizeof(int) * 4))
        return set_error(PLQCD_ERR_ARG, "plqcd_gauge_copy: lattices differ");
    PLQCD_TRY(check_lat(dst->lat));
    return launch_gauge_copy(dst->lat->geom, dst->lat->stream, dst->data, dst->prec, dst->recon, src->data,
                             src->prec, src->recon);
}

// ---- spinors -------------------------------------------------------------------

extern "C" int plqcd_spinor_import(plqcd_lattice *lat, const spinor *aos, int parity, void *dst, int prec) {
    clear_error();
    PLQCD_TRY(check_lat(lat));
    PLQCD_TRY(check_prec(prec));
    if (!aos || !dst || (parity != 0 && parity != 1)) return set_error(PLQCD_ERR_ARG, "plqcd_spinor_import: bad argument");
    return launch_spinor_import(lat->geom, lat->stream, aos, parity, dst, prec);
}

extern "C" int plqcd_spinor_export(plqcd_lattice *lat, const void *src, int prec, int parity, spinor *aos) {
    clear_error();
    PLQCD_TRY(check_lat(lat));
    PLQCD_TRY(check_prec(prec));
    if (!aos || !src || (parity != 0 && parity != 1)) return set_error(PLQCD_ERR_ARG, "plqcd_spinor_export: bad argument");
    return launch_spinor_export(lat->geom, lat->stream, src, prec, parity, aos);
}

extern "C" int plqcd_spinor_convert(plqcd_lattice *lat, void *dst, int dprec, const void *src, int sprec) {
    clear_error();
    PLQCD_TRY(check_lat(lat));
    PLQCD_TRY(check_prec(dprec));
    PLQCD_TRY(check_prec(sprec));
    if (!dst || !src) return set_error(PLQCD_ERR_ARG, "plqcd_spinor_convert: null field");
    return launch_spinor_convert(lat->geom, lat->stream, dst, dprec, src, sprec);
}

extern "C" int plqcd_spinor_gaussian(plqcd_lattice *lat, void *dst, int prec, int parity, uint64_t seed) {
    clear_error();
    PLQCD_TRY(check_lat(lat));
    PLQCD_TRY(check_prec(prec));
    if (!dst || (parity != 0 && parity != 1)) return set_error(PLQCD_ERR_ARG, "plqcd_spinor_gaussian: bad argument");
    return launch_spinor_gaussian(lat->geom, lat->stream, dst, prec, parity, seed);
}

// ---- hopping matrix --------------------------------------------------------------

static int dslash_common(plqcd_lattice *lat, const plqcd_gauge *g, int prec, DslashCall &c) {
    PLQCD_TRY(check_lat(lat));
    if (!g) return set_error(PLQCD_ERR_ARG, "dslash: null gauge");
    if (g->lat->geom.Vh != lat->geom.Vh || memcmp(g->lat->geom.L, lat->geom.L, sizeof(int) * 4))
        return set_error(PLQCD_ERR_ARG, "dslash: gauge field belongs to another lattice");
    if (g->prec != prec) return set_error(PLQCD_ERR_ARG, "dslash: spinor precision %d != gauge precision %d", prec, g->prec);
    c.gauge = g->data;
    c.prec = prec;
    c.recon = g->recon;
    return PLQCD_OK;
}

extern "C" int plqcd_dslash(plqcd_lattice *lat, const plqcd_gauge *g, void *out, const void *in, int out_parity,
                            int prec, unsigned flags) {
    clear_error();
    DslashCall c;
    PLQCD_TRY(dslash_common(lat, g, prec, c));
    if (!out || !in || (out_parity != 0 && out_parity != 1)) return set_error(PLQCD_ERR_ARG, "dslash: bad argument");
    c.out = out;
    c.in = in;
    c.out_parity = out_parity;
    c.flags = flags;
    return launch_dslash(lat->geom, lat->stream, c);
}

extern "C" int plqcd_dslash_xpay(plqcd_lattice *lat, const plqcd_gauge *g, void *out, const void *in, int out_parity,
                                 int prec, unsigned flags, double a, const void *x, double b) {
    clear_error();
    DslashCall c;
    PLQCD_TRY(dslash_common(lat, g, prec, c));
    if (!out || !in || (out_parity != 0 && out_parity != 1)) return set_error(PLQCD_ERR_ARG, "dslash: bad argument");
    if (flags & PLQCD_DSLASH_COMPAT) return set_error(PLQCD_ERR_ARG, "dslash_xpay: compat mode not supported");
    c.out = out;
    c.in = in;
    c.out_parity = out_parity;
    c.flags = flags;
    c.a_up = a;
    c.a_low = a;
    c.x = x;
    c.b = b;
    return launch_dslash(lat->geom, lat->stream, c);
}

extern "C" int plqcd_dslash_sites(plqcd_lattice *lat, const plqcd_gauge *g, void *out, const void *in,
                                  int out_parity, int prec, unsigned flags, double a, const void *x, double b,
                                  long h_begin, long h_count) {
    clear_error();
    DslashCall c;
    PLQCD_TRY(dslash_common(lat, g, prec, c));
    if (!out || !in || (out_parity != 0 && out_parity != 1) || h_count < 0)
        return set_error(PLQCD_ERR_ARG, "dslash_sites: bad argument");
    if ((flags & PLQCD_DSLASH_COMPAT) && x) return set_error(PLQCD_ERR_ARG, "dslash_sites: compat mode without xpay");
    if (h_count == 0) return PLQCD_OK;
    c.out = out;
    c.in = in;
    c.out_parity = out_parity;
    c.flags = flags;
    c.a_up = a;
    c.a_low = a;
    c.x = x;
    c.b = b;
    c.h_begin = h_begin;
    c.h_count = h_count;
    return launch_dslash(lat->geom, lat->stream, c);
}

extern "C" int plqcd_dslash_full(plqcd_lattice *lat, const plqcd_gauge *g, void *out_even, void *out_odd,
                                 const void *in_even, const void *in_odd, int prec) {
    clear_error();
    DslashCall c;
    PLQCD_TRY(dslash_common(lat, g, prec, c));
    if (!out_even || !out_odd || !in_even || !in_odd) return set_error(PLQCD_ERR_ARG, "dslash_full: null field");
    c.full = true;
    c.out = out_even;
    c.out2 = out_odd;
    c.in = in_even;
    c.in2 = in_odd;
    return launch_dslash(lat->geom, lat->stream, c);
}

// ---- norms ----------------------------------------------------------------------

#include "blas.cuh"

extern "C" int plqcd_spinor_norm2(plqcd_lattice *lat, const void *fields, int prec, int nfields, double *norms_dev) {
    clear_error();
    PLQCD_TRY(check_lat(lat));
    PLQCD_TRY(check_prec(prec));
    if (!fields || !norms_dev || nfields < 1 || nfields > 65535)
        return set_error(PLQCD_ERR_ARG, "plqcd_spinor_norm2: bad argument");
    PLQCD_TRY(check_field_ptr(fields, "plqcd_spinor_norm2"));
    if (reinterpret_cast<uintptr_t>(norms_dev) & 7u)
        return set_error(PLQCD_ERR_ARG, "plqcd_spinor_norm2: norms_dev is not 8-byte aligned");
    const int nb = norm2_blocks(lat->geom.Vh);
    const size_t pbytes = sizeof(double) * (size_t)nb * nfields;
    const size_t cbytes = sizeof(unsigned) * (size_t)nfields;
    void *ws = nullptr;
    PLQCD_TRY(lattice_workspace(lat, pbytes + cbytes, &ws));
    double *partials = static_cast<double *>(ws);
    unsigned *counters = reinterpret_cast<unsigned *>(static_cast<char *>(ws) + pbytes);
    PLQCD_CUDA_TRY(cudaMemsetAsync(counters, 0, cbytes, lat->stream));
    return launch_norm2_multi(lat->geom, lat->stream, fields, prec, nfields, partials, counters, norms_dev);
}
