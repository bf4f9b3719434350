// Device-event profiler: when enabled, every bracketed launch records a pair
// of CUDA events on its own stream; totals are folded in on read.  Each
// launch's interval is also kept, timed from an origin event recorded at
// enable, so that the time two groups of classes ran at once (launches on
// different streams) can be read back.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <utility>
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

struct Interval {
    int cls;
    double t0, t1;  // ms after the origin
};

std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
Totals g_totals[FH_PROF_CLASSES];
std::vector<Interval> g_intervals;
cudaEvent_t g_origin = nullptr;
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
            float t0 = 0.f;
            if (g_origin && cudaEventElapsedTime(&t0, g_origin, p.a) == cudaSuccess)
                g_intervals.push_back(Interval{p.cls, (double)t0, (double)t0 + ms});
        }
        g_pool.push_back(p.a);
        g_pool.push_back(p.b);
    }
    g_pending.clear();
    cudaGetLastError();
}

// The union of the intervals of the classes in `mask` (bit per class), as
// sorted disjoint intervals.
std::vector<std::pair<double, double>> merged(uint32_t mask) {
    std::vector<std::pair<double, double>> v;
    for (const Interval &iv : g_intervals)
        if (mask >> iv.cls & 1u) v.emplace_back(iv.t0, iv.t1);
    std::sort(v.begin(), v.end());
    std::vector<std::pair<double, double>> out;
    for (const auto &x : v) {
        if (!out.empty() && x.first <= out.back().second)
            out.back().second = std::max(out.back().second, x.second);
        else
            out.push_back(x);
    }
    return out;
}

double measure(const std::vector<std::pair<double, double>> &v) {
    double t = 0.0;
    for (const auto &x : v) t += x.second - x.first;
    return t;
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
    if (on && !fhb::g_on) {
        // a fresh origin: the device's other work on the legacy stream is
        // not waited for, the record only marks a point on the device clock
        if (!fhb::g_origin) cudaEventCreate(&fhb::g_origin);
        fhb::fold();
        fhb::g_intervals.clear();
        if (fhb::g_origin) cudaEventRecord(fhb::g_origin, cudaStreamPerThread);
    }
    fhb::g_on = on != 0;
}

void fh_profile_reset(void) {
    std::lock_guard<std::mutex> lk(fhb::g_mu);
    fhb::fold();
    for (auto &t : fhb::g_totals) t = fhb::Totals();
    fhb::g_intervals.clear();
}

fh_status fh_profile_overlap(uint32_t mask_a, uint32_t mask_b, double *ms_a, double *ms_b, double *ms_both) {
    std::lock_guard<std::mutex> lk(fhb::g_mu);
    fhb::fold();
    const auto a = fhb::merged(mask_a), b = fhb::merged(mask_b);
    double both = 0.0;
    size_t j = 0;
    for (const auto &x : a) {
        while (j < b.size() && b[j].second <= x.first) ++j;
        for (size_t k = j; k < b.size() && b[k].first < x.second; ++k)
            both += std::max(0.0, std::min(x.second, b[k].second) - std::max(x.first, b[k].first));
    }
    if (ms_a) *ms_a = fhb::measure(a);
    if (ms_b) *ms_b = fhb::measure(b);
    if (ms_both) *ms_both = both;
    return FH_OK;
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
