// tune.h -- launch-configuration autotuner (tune.cpp).
#pragma once

#include <cuda_runtime.h>
#include <unistd.h>

#include <functional>
#include <string>
#include <vector>

namespace plqcd {

struct TuneResult {
    int variant = 0;  // kernel-family specific (e.g. load strategy)
    int block = 128;
    double ms = 0.0;
};

bool tune_enabled();
// run(config, trial): launch one configuration; trial launches must write
// only to scratch outputs (they are repeated while timing).
int tune_launch(const std::string &key, cudaStream_t s, const std::vector<TuneResult> &cands,
                const std::function<int(const TuneResult &, bool)> &run);
// "<device name>|" prefix for keys, so cache files do not mix GPU models
const std::string &device_tag();
bool tune_lookup(const std::string &key, TuneResult *out);

}  // namespace plqcd
