// Device-event profiler: when enabled, every bracketed launch records a pair
// of CUDA events on its own stream; totals are folded in on read.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "fh_device.cuh"

namespace fhb {
namespace {

struct Pending {
    int cls;
    cudaEvent_t a, b;
    double work;
};

struct Totals {
    long long launches = 0;
    double ms = 0.0, work = 0.0;
};

std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
Totals g_totals[FH_PROF_CLASSES];
thread_local cudaEvent_t t_open[FH_PROF_CLASSES];

cudaEvent_t take() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void fold() {
    for (Pending &p : g_pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            g_totals[p.cls].launches += 1;
            g_totals[p.cls].ms += ms;
            g_totals[p.cls].work += p.work;
        }
        g_pool.push_back(p.a);
        g_pool.push_back(p.b);
    }
    g_pending.clear();
}

}  // namespace

thread_local int t_suppress = 0;

ProfSuppress::ProfSuppress() { ++t_suppress; }
ProfSuppress::~ProfSuppress() { --t_suppress; }

bool prof_on() { return g_on && !t_suppress; }

void prof_begin(cudaStream_t s, int cls) {
    if (!g_on || t_suppress || cls < 0 || cls >= FH_PROF_CLASSES) return;
    std::lock_guard<std::mutex> lk(g_mu);
    t_open[cls] = take();
    cudaEventRecord(t_open[cls], s);
}

void prof_end(cudaStream_t s, int cls, double work) {
    if (!g_on || t_suppress || cls < 0 || cls >= FH_PROF_CLASSES) return;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEvent_t b = take();
    cudaEventRecord(b, s);
    g_pending.push_back(Pending{cls, t_open[cls], b, work});
    if (g_pending.size() > 4096) fold();
}

}  // namespace fhb

extern "C" {

void fh_profile_enable(int32_t on) {
    std::lock_guard<std::mutex> lk(fhb::g_mu);
    fhb::g_on = on != 0;
}

void fh_profile_reset(void) {
    std::lock_guard<std::mutex> lk(fhb::g_mu);
    fhb::fold();
    for (auto &t : fhb::g_totals) t = fhb::Totals();
}

fh_status fh_profile_read(int32_t cls, int64_t *launches, double *ms, double *work) {
    if (cls < 0 || cls >= FH_PROF_CLASSES) return fhb::fail(nullptr, FH_ERR_INVALID_ARGUMENT, "bad profile class");
    std::lock_guard<std::mutex> lk(fhb::g_mu);
    fhb::fold();
    if (launches) *launches = fhb::g_totals[cls].launches;
    if (ms) *ms = fhb::g_totals[cls].ms;
    if (work) *work = fhb::g_totals[cls].work;
    return FH_OK;
}

}  // extern "C"
