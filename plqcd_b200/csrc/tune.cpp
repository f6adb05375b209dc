// tune.cpp -- launch-configuration autotuner with a persistent JSON cache.
//
// A kernel family registers a key (kernel name, storage format, flags,
// lattice extents) and a list of candidate configurations (load strategy and
// block size). The first launch with an unknown key times every candidate
// with CUDA events on the caller's stream, writing into scratch outputs, and
// keeps the fastest; later launches look it up. Results persist across
// processes in a JSON file (PLQCD_TUNE_FILE, default
// $HOME/.cache/plqcd_b200/tunecache.json), one object per line:
//   {"key": "...", "variant": V, "block": B, "ms": T}
// Tuning is skipped (the first candidate is used) while the stream is being
// captured into a CUDA graph, or when PLQCD_TUNE=0.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "internal.h"
#include "tune.h"

namespace plqcd {

namespace {

std::mutex g_mu;
std::map<std::string, TuneResult> &cache() {
    static std::map<std::string, TuneResult> c;
    return c;
}
bool g_loaded = false;
int g_enabled = -1;

std::string default_path() {
    if (const char *p = getenv("PLQCD_TUNE_FILE")) return p;
    const char *home = getenv("HOME");
    std::string dir = std::string(home ? home : "/tmp") + "/.cache/plqcd_b200";
    return dir + "/tunecache.json";
}

void mkdirs(const std::string &path) {
    for (size_t i = 1; i < path.size(); i++)
        if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
}

void load_locked(const std::string &path) {
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return;
    char line[1024];
    while (fgets(line, sizeof line, f)) {
        char key[512];
        TuneResult r;
        if (sscanf(line, " {\"key\": \"%511[^\"]\", \"variant\": %d, \"block\": %d, \"ms\": %lf}", key, &r.variant,
                   &r.block, &r.ms) == 4)
            cache()[key] = r;
    }
    fclose(f);
}

void save_locked(const std::string &path) {
    mkdirs(path);
    std::string tmp = path + ".tmp." + std::to_string((long)getpid());
    FILE *f = fopen(tmp.c_str(), "w");
    if (!f) return;
    for (auto &kv : cache())
        fprintf(f, "{\"key\": \"%s\", \"variant\": %d, \"block\": %d, \"ms\": %.6f}\n", kv.first.c_str(),
                kv.second.variant, kv.second.block, kv.second.ms);
    fclose(f);
    rename(tmp.c_str(), path.c_str());
}

void ensure_loaded_locked() {
    if (!g_loaded) {
        load_locked(default_path());
        g_loaded = true;
    }
}

}  // namespace

bool tune_enabled() {
    if (g_enabled < 0) {
        const char *e = getenv("PLQCD_TUNE");
        g_enabled = !(e && e[0] == '0');
    }
    return g_enabled == 1;
}

const std::string &device_tag() {
    static thread_local std::string tag;
    static thread_local int dev = -1;
    int d = 0;
    cudaGetDevice(&d);
    if (d != dev) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess)
            tag = std::string(p.name) + "/" + std::to_string(p.multiProcessorCount) + "|";
        else
            tag = "unknown|";
        dev = d;
    }
    return tag;
}

// Look up or tune. `run(config, trial)` launches one candidate on `s` and
// returns a status; the first candidate is the fallback.
int tune_launch(const std::string &key, cudaStream_t s, const std::vector<TuneResult> &cands,
                const std::function<int(const TuneResult &, bool)> &run) {
    if (cands.empty()) return set_error(PLQCD_ERR_ARG, "tune: no candidates for %s", key.c_str());
    TuneResult chosen = cands[0];
    bool found = false;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        ensure_loaded_locked();
        auto it = cache().find(key);
        if (it != cache().end()) {
            chosen = it->second;
            found = true;
        }
    }
    if (found || !tune_enabled()) return run(chosen, false);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return run(chosen, false);

    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        return run(chosen, false);
    }
    // each candidate: one warm-up launch, a short probe to size the timed
    // batch (at least ~2 ms of work), then the best of three batches
    auto time_batch = [&](const TuneResult &c, int reps, float *ms) -> bool {
        cudaEventRecord(e0, s);
        int rc = PLQCD_OK;
        for (int r = 0; r < reps && rc == PLQCD_OK; r++) rc = run(c, true);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess || rc != PLQCD_OK) {
            clear_error();
            cudaGetLastError();
            return false;
        }
        cudaEventElapsedTime(ms, e0, e1);
        *ms /= reps;
        return true;
    };
    // pass 1: every candidate (best of three batches), scored against the
    // first feasible candidate timed right before it, so that the clock
    // drift of a long tuning run (the power cap settles in) does not favour
    // the candidates timed first
    struct Timed {
        size_t idx;
        int reps;
        float t;    // pass 1 score: time / reference time
        float raw;  // pass 1 time (ms)
        std::vector<float> rounds;
    };
    std::vector<Timed> timed;
    long ref = -1;
    int ref_reps = 2;
    for (size_t i = 0; i < cands.size(); i++) {
        const TuneResult &c = cands[i];
        if (run(c, true) != PLQCD_OK) {  // infeasible candidate (e.g. shared memory)
            clear_error();
            cudaGetLastError();
            continue;
        }
        float probe = 0;
        if (!time_batch(c, 2, &probe)) continue;
        int reps = probe > 0 ? (int)(2.0f / probe) : 50;
        reps = reps < 2 ? 2 : (reps > 200 ? 200 : reps);
        float tref = 1.f;
        if (ref >= 0 && !time_batch(cands[ref], ref_reps, &tref)) continue;
        float t = 1e30f, ms = 0;
        bool ok = true;
        for (int k = 0; k < 3 && ok; k++) {
            ok = time_batch(c, reps, &ms);
            if (ok && ms < t) t = ms;
        }
        if (!ok) continue;
        if (ref < 0) {
            ref = (long)i;
            ref_reps = reps;
            tref = t;
        }
        timed.push_back({i, reps, t / (tref > 0 ? tref : 1.f), t, {}});
    }
    // pass 2: the fastest four again. Short launches: round-robin, so that
    // all of them see the same clock (median of five rounds). Launches of
    // 100 us or more (large lattices, run back to back for long stretches):
    // each finalist alone for ~0.2 s until the power cap has settled the
    // clock at that kernel's own draw, then timed for ~0.1 s; a kernel that
    // draws less power holds a higher clock there.
    std::vector<Timed> fin = timed;
    std::sort(fin.begin(), fin.end(), [](const Timed &a, const Timed &b) { return a.t < b.t; });
    if (fin.size() > 4) fin.resize(4);
    std::sort(fin.begin(), fin.end(), [](const Timed &a, const Timed &b) { return a.idx < b.idx; });
    bool long_launch = false;
    for (const Timed &f : fin) long_launch = long_launch || f.raw >= 0.1f;
    if (fin.size() > 1 && long_launch) {
        for (Timed &f : fin) {
            const int settle = (int)(200.f / f.raw) + 1, timed_reps = (int)(100.f / f.raw) + 1;
            float ms = 0;
            if (time_batch(cands[f.idx], settle, &ms) && time_batch(cands[f.idx], timed_reps, &ms))
                f.rounds.push_back(ms);
        }
    } else if (fin.size() > 1) {
        for (int round = 0; round < 5; round++)
            for (Timed &f : fin) {
                float ms = 0;
                if (time_batch(cands[f.idx], 2 * f.reps, &ms)) f.rounds.push_back(ms);
            }
    }
    double best = 1e30;
    TuneResult bestc = cands[0];
    for (Timed &f : fin) {
        float score = f.raw;
        if (!f.rounds.empty()) {
            std::sort(f.rounds.begin(), f.rounds.end());
            score = f.rounds[f.rounds.size() / 2];
        }
        // a later candidate must win by more than 1%: near-ties (timing
        // noise) keep the earlier configuration on every GPU
        if (score < best * 0.99) {
            best = score;
            bestc = cands[f.idx];
            bestc.ms = score;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        cache()[key] = bestc;
        save_locked(default_path());
    }
    return run(bestc, false);
}

bool tune_lookup(const std::string &key, TuneResult *out) {
    std::lock_guard<std::mutex> lk(g_mu);
    ensure_loaded_locked();
    auto it = cache().find(key);
    if (it == cache().end()) return false;
    if (out) *out = it->second;
    return true;
}

}  // namespace plqcd

extern "C" int plqcd_tune_enable(int on) {
    plqcd::g_enabled = on ? 1 : 0;
    return PLQCD_OK;
}

extern "C" int plqcd_tune_clear(void) {
    std::lock_guard<std::mutex> lk(plqcd::g_mu);
    plqcd::cache().clear();
    plqcd::g_loaded = true;  // do not reload the file
    return PLQCD_OK;
}

extern "C" int plqcd_tune_save(const char *path) {
    std::lock_guard<std::mutex> lk(plqcd::g_mu);
    plqcd::save_locked(path ? path : plqcd::default_path());
    return PLQCD_OK;
}

extern "C" int plqcd_tune_load(const char *path) {
    std::lock_guard<std::mutex> lk(plqcd::g_mu);
    plqcd::load_locked(path ? path : plqcd::default_path());
    plqcd::g_loaded = true;
    return PLQCD_OK;
}

extern "C" int plqcd_tune_count(void) {
    std::lock_guard<std::mutex> lk(plqcd::g_mu);
    plqcd::ensure_loaded_locked();
    return (int)plqcd::cache().size();
}

extern "C" int plqcd_tune_get(const char *key, int *variant, int *block, double *ms) {
    plqcd::TuneResult r;
    if (!key || !plqcd::tune_lookup(key, &r)) return plqcd::set_error(PLQCD_ERR_ARG, "tune: no entry for key");
    if (variant) *variant = r.variant;
    if (block) *block = r.block;
    if (ms) *ms = r.ms;
    return PLQCD_OK;
}
