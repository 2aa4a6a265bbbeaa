// Project autotuner: launch shapes of the hot kernels are picked by timing
// every candidate on the caller's own data, and the choice is cached per
// (stage shape, device) for the process and, when SKB_TUNE_CACHE names a
// file, across processes.
//
// Keys name the stage, its shape and the device, e.g.
//   "tc_gemm.unit_tiles R=129 S=85 groups=7486 columns=686475 members=8 | NVIDIA B200/148"
// so a cached choice is only reused for the same work on the same kind of GPU.
// The cache file holds one entry per line: "<value> <milliseconds> <key>".

#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

namespace skb {

struct TuneEntry {
    std::string key;
    int value = 0;
    double ms = 0.0;
};

// Process-wide cache (thread-safe).  The first access loads SKB_TUNE_CACHE
// if it is set; every new choice is appended to that file.
bool tune_lookup(const std::string& key, int& value);
void tune_store(const std::string& key, int value, double ms);
std::vector<TuneEntry> tune_entries();
void tune_clear();
// Merge a cache file into the process cache (missing file: nothing loaded;
// malformed lines are skipped) / write the whole process cache to a file.
// Return the number of entries read / written.
int tune_load(const std::string& path);
int tune_save(const std::string& path);

// The cached value for `key`, else the fastest of `candidates`: run(c)
// enqueues one execution with candidate c on `s`; each candidate gets
// `warmups` untimed runs and `reps` runs timed with CUDA events on `s`, and
// its best timed run counts.  The winner is stored under `key`.  `bestMs`
// (optional) receives the winner's time (the cached time on a hit).
int tune_pick(const std::string& key, const std::vector<int>& candidates, const std::function<void(int)>& run,
              cudaStream_t s, int warmups = 1, int reps = 3, double* bestMs = nullptr);

// "<device name>/<SM count>" of the current device.
std::string device_tag();

}  // namespace skb
