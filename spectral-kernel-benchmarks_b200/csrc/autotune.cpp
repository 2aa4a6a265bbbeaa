// Project autotuner (see autotune.hpp).

#include "autotune.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <map>
#include <mutex>
#include <sstream>

#include "runtime.hpp"

namespace skb {
namespace {

struct Cache {
    std::mutex mu;
    std::map<std::string, std::pair<int, double>> entries;
    bool envLoaded = false;
};

Cache& cache() {
    static Cache c;
    return c;
}

const char* env_path() {
    const char* p = std::getenv("SKB_TUNE_CACHE");
    return (p != nullptr && *p != '\0') ? p : nullptr;
}

// Parse "<value> <ms> <key...>" lines into `into`; returns entries read.
int parse_file(const std::string& path, std::map<std::string, std::pair<int, double>>& into) {
    std::ifstream in(path);
    if (!in) return 0;
    int n = 0;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        int value = 0;
        double ms = 0.0;
        if (!(ls >> value >> ms)) continue;
        std::string key;
        std::getline(ls, key);
        const auto first = key.find_first_not_of(' ');
        if (first == std::string::npos) continue;
        into[key.substr(first)] = {value, ms};
        ++n;
    }
    return n;
}

// Caller holds the mutex.
void load_env_locked(Cache& c) {
    if (c.envLoaded) return;
    c.envLoaded = true;
    if (const char* p = env_path()) parse_file(p, c.entries);
}

void append_env(const std::string& key, int value, double ms) {
    const char* p = env_path();
    if (p == nullptr) return;
    std::ofstream out(p, std::ios::app);
    if (out) out << value << ' ' << ms << ' ' << key << '\n';
}

}  // namespace

bool tune_lookup(const std::string& key, int& value) {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    load_env_locked(c);
    const auto it = c.entries.find(key);
    if (it == c.entries.end()) return false;
    value = it->second.first;
    return true;
}

void tune_store(const std::string& key, int value, double ms) {
    Cache& c = cache();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        load_env_locked(c);
        c.entries[key] = {value, ms};
    }
    append_env(key, value, ms);
}

std::vector<TuneEntry> tune_entries() {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    load_env_locked(c);
    std::vector<TuneEntry> out;
    for (const auto& [k, v] : c.entries) out.push_back({k, v.first, v.second});
    return out;
}

void tune_clear() {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    c.entries.clear();
    c.envLoaded = true;  // an explicit clear also drops what the file would add
}

int tune_load(const std::string& path) {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    load_env_locked(c);
    return parse_file(path, c.entries);
}

int tune_save(const std::string& path) {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    std::ofstream out(path, std::ios::trunc);
    if (!out) throw Error(-1, "cannot write the tuning cache file " + path);
    for (const auto& [k, v] : c.entries) out << v.first << ' ' << v.second << ' ' << k << '\n';
    return static_cast<int>(c.entries.size());
}

int tune_pick(const std::string& key, const std::vector<int>& candidates, const std::function<void(int)>& run,
              cudaStream_t s, int warmups, int reps, double* bestMs) {
    if (candidates.empty()) throw Error(-1, "autotune: no candidates for " + key);
    int cached = 0;
    if (tune_lookup(key, cached)) {
        if (bestMs != nullptr) {
            Cache& c = cache();
            std::lock_guard<std::mutex> lock(c.mu);
            *bestMs = c.entries[key].second;
        }
        return cached;
    }
    cudaEvent_t a = nullptr, b = nullptr;
    check_cuda(cudaEventCreate(&a), "cudaEventCreate");
    check_cuda(cudaEventCreate(&b), "cudaEventCreate");
    int best = candidates.front();
    double bestTime = std::numeric_limits<double>::infinity();
    try {
        for (const int c : candidates) {
            for (int i = 0; i < warmups; ++i) run(c);
            double t = std::numeric_limits<double>::infinity();
            for (int i = 0; i < std::max(1, reps); ++i) {
                check_cuda(cudaEventRecord(a, s), "cudaEventRecord");
                run(c);
                check_cuda(cudaEventRecord(b, s), "cudaEventRecord");
                check_cuda(cudaEventSynchronize(b), "cudaEventSynchronize");
                float ms = 0.0f;
                check_cuda(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
                t = std::min(t, static_cast<double>(ms));
            }
            if (t < bestTime) {
                bestTime = t;
                best = c;
            }
        }
    } catch (...) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        throw;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    tune_store(key, best, bestTime);
    if (bestMs != nullptr) *bestMs = bestTime;
    return best;
}

std::string device_tag() {
    int device = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return "unknown-device";
    return std::string(prop.name) + "/" + std::to_string(prop.multiProcessorCount);
}

}  // namespace skb
