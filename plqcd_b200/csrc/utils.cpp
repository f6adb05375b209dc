// utils.cpp -- aligned host allocation, timer and tags (include/utils.h).
//
// Same entry points as the reference's lib/utils.c:23-125. amalloc hands out
// page-locked host memory when a CUDA device is usable, so fields that a
// caller allocates with it (as tests/test_hopping.c:96-115 does) cross PCIe
// at full speed in the drop-in hopping calls; otherwise it falls back to
// ordinary aligned heap memory. A registry maps each aligned address back to
// its allocation so afree can release it (and ignores unknown addresses, as
// lib/utils.c:68-90 does).
#include <cuda.h>
#include <cuda_runtime.h>
#include <sys/time.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.h"
#include "utils.h"

namespace {

struct Block {
    void *base;
    bool pinned;
};

std::mutex g_mu;
std::unordered_map<uintptr_t, Block> &registry() {
    static std::unordered_map<uintptr_t, Block> r;
    return r;
}

bool pinned_allowed() {
    static int allowed = -1;
    if (allowed < 0) {
        const char *env = getenv("PLQCD_PINNED_AMALLOC");
        int n = 0;
        allowed = (env && env[0] == '0') ? 0 : (cudaGetDeviceCount(&n) == cudaSuccess && n > 0);
        if (!allowed) cudaGetLastError();
    }
    return allowed == 1;
}

}  // namespace

extern "C" void *alloc(size_t size, size_t alignment) {
    void *p = nullptr;
    if (posix_memalign(&p, alignment, size) != 0 || !p) {
        plqcd::set_error(PLQCD_ERR_NOMEM, "alloc() returned NULL. Out of memory?");
        return nullptr;
    }
    return p;
}

extern "C" void *amalloc(size_t size, int p) {
    if (size == 0 || p < 0 || p > 30) return nullptr;
    size_t shift = (size_t)1 << p;
    void *base = nullptr;
    bool pinned = false;
    if (pinned_allowed() && cudaHostAlloc(&base, size + shift, cudaHostAllocPortable) == cudaSuccess) {
        pinned = true;
    } else {
        cudaGetLastError();
        base = malloc(size + shift);
        if (!base) return nullptr;
    }
    uintptr_t a = ((uintptr_t)base + shift) & ~(uintptr_t)(shift - 1);
    std::lock_guard<std::mutex> lk(g_mu);
    registry()[a] = Block{base, pinned};
    return (void *)a;
}

extern "C" void afree(void *addr) {
    Block b;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = registry().find((uintptr_t)addr);
        if (it == registry().end()) return;
        b = it->second;
        registry().erase(it);
    }
    if (b.pinned)
        cudaFreeHost(b.base);
    else
        free(b.base);
}

// Tag counters (lib/utils.c:6-9, 94-114).
static const int kMaxTag = 32767;
static const int kMaxPermanentTag = kMaxTag / 2;
static int g_pcmn = -1, g_cmn = kMaxTag;

extern "C" int mpi_permanent_tag(void) {
    if (g_pcmn < kMaxPermanentTag) return ++g_pcmn;
    plqcd::set_error(PLQCD_ERR_STATE, "mpi_permanent_tag: requested more than 16384 tags");
    return -1;
}

extern "C" int mpi_tag(void) {
    if (g_cmn == kMaxTag) g_cmn = kMaxPermanentTag;
    return ++g_cmn;
}

extern "C" double stop_watch(double t) {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (tv.tv_sec + tv.tv_usec * 1e-6) - t;
}

// ---- API layout <-> split real / imaginary planes ------------------------------
// A memory-bound copy: n complex numbers, split across host threads in
// contiguous ranges when n is large.
namespace {

template <class F>
void parallel_ranges(long n, F f) {
    const long per_thread = 1L << 20;
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt < 1 ? 1 : (nt > 16 ? 16 : nt);
    if (n < 2 * per_thread || nt == 1) {
        f(0L, n);
        return;
    }
    long parts = n / per_thread;
    if (parts > (long)nt) parts = nt;
    std::vector<std::thread> pool;
    for (long p = 1; p < parts; p++) pool.emplace_back(f, n * p / parts, n * (p + 1) / parts);
    f(0L, n / parts);
    for (auto &t : pool) t.join();
}

}  // namespace

extern "C" int plqcd_aos_to_split(const double *aos, double *re, double *im, long n) {
    if (!aos || !re || !im || n < 0) return plqcd::set_error(PLQCD_ERR_ARG, "plqcd_aos_to_split: bad argument");
    parallel_ranges(n, [=](long a, long b) {
        for (long k = a; k < b; k++) {
            re[k] = aos[2 * k];
            im[k] = aos[2 * k + 1];
        }
    });
    return PLQCD_OK;
}

extern "C" int plqcd_split_to_aos(const double *re, const double *im, double *aos, long n) {
    if (!aos || !re || !im || n < 0) return plqcd::set_error(PLQCD_ERR_ARG, "plqcd_split_to_aos: bad argument");
    parallel_ranges(n, [=](long a, long b) {
        for (long k = a; k < b; k++) {
            aos[2 * k] = re[k];
            aos[2 * k + 1] = im[k];
        }
    });
    return PLQCD_OK;
}

namespace plqcd {

int smem_optin(const void *func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> granted;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return set_error(PLQCD_ERR_CUDA, "smem_optin: no current device");
    }
    std::lock_guard<std::mutex> lk(mu);
    size_t &have = granted[{func, dev}];
    if (bytes <= have) return PLQCD_OK;
    cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(PLQCD_ERR_CUDA, "shared-memory opt-in of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    have = bytes;
    return PLQCD_OK;
}

// ID of the current CUDA context (unique within the process, never reused),
// 0 when the driver does not provide it
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr, *q = nullptr;
        cudaDriverEntryPointQueryResult r1 = cudaDriverEntryPointSymbolNotFound, r2 = r1;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &q, cudaEnableDefault, &r2) == cudaSuccess &&
            r1 == cudaDriverEntryPointSuccess && r2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrent>(p);
            get_id = reinterpret_cast<GetId>(q);
        } else {
            cudaGetLastError();
        }
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_current || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}


}  // namespace plqcd
