// The autotuner of the batched small-system solve (fh_batchsolve.cu): for
// each order bucket (orders 128 (b - 1) < m <= 128 b) it times every tile
// configuration (panel width NB x trailing tile TILE) on one item of the
// first system that falls in the bucket -- one CTA, CUDA events, best of
// two runs after a warm-up -- and keeps the fastest.  The table is kept in
// a small JSON file per device name, so later processes skip the
// measurement:
//
//   {"format": 1, "device": "<name>", "buckets": {"<b>": <config>, ...}}
//
// Path: $FH_AUTOTUNE_CACHE, else $XDG_CACHE_HOME/fasterhenry_b200/
// batch_tiles.json, else $HOME/.cache/fasterhenry_b200/batch_tiles.json.
// A file that cannot be read or written only costs the measurement.
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>

#include "fh_batchsolve.h"
#include "fh_device.cuh"

namespace fhb {
namespace {

std::mutex g_mu;
bool g_loaded = false;
std::string g_device;
std::map<int, int> g_table;

std::string device_name() {
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
    return std::string(prop.name) + " sm_" + std::to_string(prop.major) + std::to_string(prop.minor);
}

// Parses this file's own format; anything else leaves the table empty.
void parse(const std::string &text, const std::string &device, std::map<int, int> &out) {
    const size_t d = text.find("\"device\"");
    if (d == std::string::npos) return;
    const size_t q0 = text.find('"', text.find(':', d) + 1);
    const size_t q1 = q0 == std::string::npos ? q0 : text.find('"', q0 + 1);
    if (q1 == std::string::npos || text.substr(q0 + 1, q1 - q0 - 1) != device) return;
    size_t b = text.find("\"buckets\"");
    if (b == std::string::npos) return;
    b = text.find('{', b);
    const size_t e = text.find('}', b);
    if (b == std::string::npos || e == std::string::npos) return;
    size_t pos = b + 1;
    while (pos < e) {
        const size_t k0 = text.find('"', pos);
        if (k0 == std::string::npos || k0 >= e) break;
        const size_t k1 = text.find('"', k0 + 1);
        const size_t colon = text.find(':', k1);
        if (k1 == std::string::npos || colon == std::string::npos || colon >= e) break;
        const int key = std::atoi(text.substr(k0 + 1, k1 - k0 - 1).c_str());
        const int val = std::atoi(text.c_str() + colon + 1);
        if (key > 0 && val >= 0 && val < kBatchConfigs) out[key] = val;
        pos = text.find(',', colon);
        if (pos == std::string::npos) break;
        ++pos;
    }
}

void make_dirs(const std::string &path) {
    for (size_t i = 1; i < path.size(); ++i)
        if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
}

void save(const std::string &path) {
    make_dirs(path);
    std::ostringstream o;
    o << "{\"format\": 1, \"device\": \"" << g_device << "\", \"buckets\": {";
    bool first = true;
    for (const auto &kv : g_table) {
        o << (first ? "" : ", ") << "\"" << kv.first << "\": " << kv.second;
        first = false;
    }
    o << "}}\n";
    const std::string tmp = path + ".tmp" + std::to_string((long long)getpid());
    std::ofstream f(tmp);
    if (!f) return;
    f << o.str();
    f.close();
    std::rename(tmp.c_str(), path.c_str());
}

}  // namespace

std::string BatchTuner::cache_path() const {
    if (const char *p = std::getenv("FH_AUTOTUNE_CACHE")) return p;
    if (const char *x = std::getenv("XDG_CACHE_HOME")) return std::string(x) + "/fasterhenry_b200/batch_tiles.json";
    if (const char *h = std::getenv("HOME")) return std::string(h) + "/.cache/fasterhenry_b200/batch_tiles.json";
    return "batch_tiles.json";
}

fh_status BatchTuner::config_for(const BatchSys &sys, const BatchSys *d_sys_one, cudaStream_t s, int *cfg,
                                 fh_error_info *err) {
    std::lock_guard<std::mutex> lk(g_mu);
    const std::string path = cache_path();
    if (!g_loaded) {
        g_device = device_name();
        std::ifstream f(path);
        if (f) {
            std::stringstream ss;
            ss << f.rdbuf();
            parse(ss.str(), g_device, g_table);
        }
        g_loaded = true;
    }
    const int bucket = bucket_of(sys.m);
    auto it = g_table.find(bucket);
    if (it != g_table.end()) {
        *cfg = it->second;
        return FH_OK;
    }
    // Measure: one item (the system at 100 MHz), one CTA, each configuration.
    const int pmax = (int)std::max<int64_t>(1, sys.p);
    const int64_t mmax = std::max<int64_t>(1, sys.m);
    const size_t slot = batch_slot_bytes(mmax, pmax);
    void *work = nullptr, *items = nullptr, *z = nullptr, *status = nullptr, *counter = nullptr;
    struct Release {
        void **p[5];
        cudaStream_t s;
        ~Release() {
            for (void **q : p)
                if (*q) cache_free(*q, s);
        }
    } release{{&work, &items, &z, &status, &counter}, s};
    FHB_CUDA(cache_alloc(&work, slot, s));
    FHB_CUDA(cache_alloc(&items, sizeof(BatchItem), s));
    FHB_CUDA(cache_alloc(&z, sizeof(double2) * (size_t)pmax * pmax, s));
    FHB_CUDA(cache_alloc(&status, sizeof(int32_t), s));
    FHB_CUDA(cache_alloc(&counter, sizeof(unsigned), s));
    cudaEvent_t e0, e1;
    FHB_CUDA(cudaEventCreate(&e0));
    FHB_CUDA(cudaEventCreate(&e1));
    struct Ev {
        cudaEvent_t a, b;
        ~Ev() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } ev{e0, e1};
    int best = kBatchConfigs - 1;
    float best_ms = 1e30f;
    for (int c = 0; c < kBatchConfigs; ++c) {
        BatchItem item;
        item.sys = 0;
        item.cfg = c;
        item.omega = 6.283185307179586 * 1e8;
        FHB_CUDA(cudaMemcpyAsync(items, &item, sizeof item, cudaMemcpyHostToDevice, s));
        float ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            FHB_CUDA(cudaEventRecord(e0, s));
            fh_status st = batch_launch(d_sys_one, static_cast<BatchItem *>(items), 1, static_cast<unsigned *>(counter),
                                        work, slot, mmax, pmax, static_cast<double2 *>(z),
                                        static_cast<int32_t *>(status), 1, s, err);
            if (st) return st;
            FHB_CUDA(cudaEventRecord(e1, s));
            FHB_CUDA(cudaEventSynchronize(e1));
            float t = 0.f;
            FHB_CUDA(cudaEventElapsedTime(&t, e0, e1));
            if (rep > 0) ms = std::min(ms, t);
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    g_table[bucket] = best;
    ++tuned_now;
    save(path);
    *cfg = best;
    return FH_OK;
}

BatchTuner &batch_tuner() {
    static BatchTuner t;
    return t;
}

}  // namespace fhb
