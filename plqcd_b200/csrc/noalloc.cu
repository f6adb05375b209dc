// noalloc.cu -- allocation-free variant of the batched spinor norm.
//
// plqcd_spinor_norm2 takes its reduction scratch (per-block partial sums and
// arrival counters) from the lattice workspace, which is grown with
// cudaMalloc. Some callers cannot allow that: applications whose device
// memory must all come from their own pool allocator (a framework that has
// reserved the GPU's memory, or a service held to a fixed memory budget,
// where an allocation outside the pool fails or breaks the budget), and
// latency-bound loops that cannot take the device-wide synchronisation
// cudaFree implies. For them, plqcd_spinor_norm2_noalloc runs the same
// reduction kernel with its scratch in the file-scope device array below,
// which every GPU that loads the library holds until the process exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "blas.cuh"
#include "internal.h"

namespace {

constexpr int kNoallocMaxFields = PLQCD_NORM2_NOALLOC_MAX_FIELDS;
// counters (one unsigned per field, padded to 256 bytes) then the partials
constexpr size_t kCounterBytes = 256;
constexpr size_t kScratchBytes = kCounterBytes + sizeof(double) * (size_t)plqcd::kMaxRedBlocks * kNoallocMaxFields;
static_assert(sizeof(unsigned) * kNoallocMaxFields <= kCounterBytes, "counter area too small");

// In host code this name is only a host-side stand-in for the device array,
// not a device address: the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_norm2_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // context ID the address belongs to

// Device address of the scratch on the current device. The set-up (the
// first call on a device, with that device current) looks it up with
// cudaGetSymbolAddress and loads the reduction kernel of every precision.
// The address belongs to the device's CUDA context: after cudaDeviceReset
// the context is a new one, with a new ID, and the set-up runs again.
int scratch_address(int device, void **out) {
    if (device < 0 || device >= kMaxDevices)
        return plqcd::set_error(PLQCD_ERR_ARG, "plqcd_spinor_norm2_noalloc: device %d out of range", device);
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long ctx = plqcd::current_context_id();
    if (!g_scratch_ptr[device] || g_scratch_ctx[device] != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_norm2_scratch);
        if (e != cudaSuccess || !p)
            return plqcd::set_error(PLQCD_ERR_CUDA, "plqcd_spinor_norm2_noalloc: cudaGetSymbolAddress: %s",
                                    cudaGetErrorString(e));
        PLQCD_TRY(plqcd::preload_norm2_multi());
        g_scratch_ptr[device] = p;
        g_scratch_ctx[device] = ctx;
    }
    *out = g_scratch_ptr[device];
    return PLQCD_OK;
}

}  // namespace

extern "C" int plqcd_spinor_norm2_noalloc(plqcd_lattice *lat, const void *fields, int prec, int nfields,
                                          double *norms_dev) {
    using namespace plqcd;
    clear_error();
    if (!lat || !fields || !norms_dev) return set_error(PLQCD_ERR_ARG, "plqcd_spinor_norm2_noalloc: null argument");
    if (prec < PLQCD_F64 || prec > PLQCD_BF16)
        return set_error(PLQCD_ERR_ARG, "plqcd_spinor_norm2_noalloc: unknown precision %d", prec);
    if (nfields < 1 || nfields > kNoallocMaxFields)
        return set_error(PLQCD_ERR_ARG,
                         "plqcd_spinor_norm2_noalloc: nfields = %d outside 1..%d (the size of its static scratch)",
                         nfields, kNoallocMaxFields);
    PLQCD_TRY(check_field_ptr(fields, "plqcd_spinor_norm2_noalloc"));
    if (reinterpret_cast<uintptr_t>(norms_dev) & 7u)
        return set_error(PLQCD_ERR_ARG, "plqcd_spinor_norm2_noalloc: norms_dev is not 8-byte aligned");
    PLQCD_CUDA_TRY(cudaSetDevice(lat->device));
    void *base = nullptr;
    PLQCD_TRY(scratch_address(lat->device, &base));
    unsigned *counters = static_cast<unsigned *>(base);
    double *partials = reinterpret_cast<double *>(static_cast<char *>(base) + kCounterBytes);
    // the arrival counters must start at zero; the partials are written
    // before they are read
    PLQCD_CUDA_TRY(cudaMemsetAsync(counters, 0, sizeof(unsigned) * nfields, lat->stream));
    return launch_norm2_multi(lat->geom, lat->stream, fields, prec, nfields, partials, counters, norms_dev);
}
