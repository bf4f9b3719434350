// Host part of the precorrected-FFT set-up: parameters, the grid, and the
// near-pair search.  The method is the reference's (pfft/mod.rs:332-460,
// grid.rs:44-95, near.rs:41-106):
//
//   * grid of spacing h over the filaments' bounding box, padded by half a
//     stencil, h from GridSpacing::Auto (about cells_per_filament cells per
//     filament) or fixed;
//   * near pairs: uniform bins about the radius in size; a pair is near when
//     the separating-axis gap of the two bars is below radius = k h; the
//     non-orthogonal ones (i <= j) are the pairs whose grid approximation the
//     device replaces by the exact value.
//
// The projections and the grid approximations of the near pairs are built on
// the device (fh_pfft_setup.cu).  Rows of the search are independent and run
// on the host's cores; each row's result is in a fixed order, so it does not
// depend on the thread count.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>

#include "fh_pfft.h"

namespace fhb {

namespace {

// Runs body(i) for i in [0, n) on the host's cores, `chunk` indices at a
// time, handed out dynamically.  Each index's work is independent and
// deterministic, so the result does not depend on the schedule.
template <class F>
void parallel_for(int64_t n, int64_t chunk, F body) {
    if (n <= 0) return;
    unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    threads = (unsigned)std::min<int64_t>(threads, (n + chunk - 1) / chunk);
    std::atomic<int64_t> next(0);
    auto worker = [&]() {
        for (;;) {
            const int64_t begin = next.fetch_add(chunk);
            if (begin >= n) return;
            const int64_t end = std::min(n, begin + chunk);
            for (int64_t i = begin; i < end; ++i) body(i);
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
}

constexpr double kOrthogonalCos = 1e-14;        // near.rs:25

struct Bar {  // neumann.rs Bar: centre, unit axes, half extents
    double c[3];
    double ax[3][3];
    double half[3];
};

inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

Bar bar_of(const fh_filament &f) {
    Bar b;
    for (int k = 0; k < 3; ++k) {
        b.c[k] = (f.start[k] + f.end[k]) * 0.5;
        b.ax[0][k] = f.dir_length[k];
        b.ax[1][k] = f.dir_width[k];
        b.ax[2][k] = f.dir_height[k];
    }
    b.half[0] = 0.5 * f.length;
    b.half[1] = 0.5 * f.width;
    b.half[2] = 0.5 * f.height;
    return b;
}

double projected_half(const Bar &b, const double *n) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s += b.half[k] * std::fabs(dot3(n, b.ax[k]));
    return s;
}

// Separating-axis lower bound on the distance between two bars
// (neumann.rs:97-122): 15 axes, or centre distance minus the circumradii
// when the bars are far apart.
double separation(const Bar &a, const Bar &b) {
    const double d[3] = {b.c[0] - a.c[0], b.c[1] - a.c[1], b.c[2] - a.c[2]};
    const double dist = std::sqrt(dot3(d, d));
    auto circ = [](const Bar &x) {
        return std::sqrt(x.half[0] * x.half[0] + x.half[1] * x.half[1] + x.half[2] * x.half[2]);
    };
    const double reach = circ(a) + circ(b);
    if (dist > 8.0 * reach) return dist - reach;
    double best = -std::numeric_limits<double>::infinity();
    auto consider = [&](const double *n) {
        const double gap = std::fabs(dot3(n, d)) - projected_half(a, n) - projected_half(b, n);
        best = std::max(best, gap);
    };
    for (int k = 0; k < 3; ++k) {
        consider(a.ax[k]);
        consider(b.ax[k]);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const double *u = a.ax[i], *v = b.ax[j];
            double c[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
            const double nn = std::sqrt(dot3(c, c));
            if (nn > 1e-9) {
                const double e[3] = {c[0] / nn, c[1] / nn, c[2] / nn};
                consider(e);
            }
        }
    return best;
}

// near.rs:41-106: for each i, the j >= i within `radius` (i included), ascending.
void near_pairs(const std::vector<Bar> &bars, double radius, std::vector<std::vector<uint32_t>> &out) {
    const int64_t n = (int64_t)bars.size();
    out.assign(n, {});
    if (n == 0) return;
    std::vector<std::array<double, 6>> boxes(n);
    for (int64_t i = 0; i < n; ++i) {
        double reach[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k)
            for (int a = 0; a < 3; ++a) reach[a] += std::fabs(bars[i].ax[k][a]) * bars[i].half[k];
        for (int a = 0; a < 3; ++a) {
            boxes[i][a] = bars[i].c[a] - reach[a];
            boxes[i][3 + a] = bars[i].c[a] + reach[a];
        }
    }
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = boxes[0][a];
        hi[a] = boxes[0][3 + a];
    }
    for (const auto &b : boxes)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b[a]);
            hi[a] = std::max(hi[a], b[3 + a]);
        }
    double extent[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    const double emax = std::max(extent[0], std::max(extent[1], extent[2]));
    double size = std::max(std::max(radius, emax * 1e-9), std::numeric_limits<double>::min());
    auto bin_dims = [&](double s, int64_t d[3]) {
        for (int a = 0; a < 3; ++a) d[a] = (int64_t)std::floor(extent[a] / s) + 1;
    };
    int64_t dims[3];
    bin_dims(size, dims);
    while (dims[0] * dims[1] * dims[2] > 8 * n + 64) {
        size *= 1.5;
        bin_dims(size, dims);
    }
    auto cell = [&](double x, int a) {
        double c = std::floor((x - lo[a]) / size);
        int64_t v = c > 0.0 ? (int64_t)c : 0;
        return std::min<int64_t>(v, dims[a] - 1);
    };
    std::vector<std::vector<uint32_t>> bins((size_t)(dims[0] * dims[1] * dims[2]));
    for (int64_t idx = 0; idx < n; ++idx) {
        int64_t f[3], l[3];
        for (int a = 0; a < 3; ++a) {
            f[a] = cell(boxes[idx][a], a);
            l[a] = cell(boxes[idx][3 + a], a);
        }
        for (int64_t i = f[0]; i <= l[0]; ++i)
            for (int64_t j = f[1]; j <= l[1]; ++j)
                for (int64_t k = f[2]; k <= l[2]; ++k) bins[(i * dims[1] + j) * dims[2] + k].push_back((uint32_t)idx);
    }
    parallel_for(n, 64, [&](int64_t idx) {
        int64_t f[3], l[3];
        for (int a = 0; a < 3; ++a) {
            f[a] = cell(boxes[idx][a] - radius, a);
            l[a] = cell(boxes[idx][3 + a] + radius, a);
        }
        std::vector<uint32_t> found;
        for (int64_t i = f[0]; i <= l[0]; ++i)
            for (int64_t j = f[1]; j <= l[1]; ++j)
                for (int64_t k = f[2]; k <= l[2]; ++k)
                    for (uint32_t other : bins[(i * dims[1] + j) * dims[2] + k])
                        if ((int64_t)other >= idx) found.push_back(other);
        std::sort(found.begin(), found.end());
        found.erase(std::unique(found.begin(), found.end()), found.end());
        std::vector<uint32_t> keep;
        for (uint32_t other : found)
            if ((int64_t)other == idx || separation(bars[idx], bars[other]) < radius) keep.push_back(other);
        out[idx].swap(keep);
    });
}

}  // namespace

int64_t smooth_size(int64_t n) {
    int64_t m = std::max<int64_t>(n, 1);
    for (;; ++m) {
        int64_t r = m;
        for (int p : {2, 3, 5})
            while (r % p == 0) r /= p;
        if (r == 1) return m;
    }
}

double auto_spacing(const double extent[3], double cells) {
    const double largest = std::max(extent[0], std::max(extent[1], extent[2]));
    auto count = [&](double h) {
        double c = 1.0;
        for (int a = 0; a < 3; ++a) c *= std::max(extent[a] / h, 1.0);
        return c;
    };
    if (cells <= 1.0 || largest <= 0.0) return std::max(largest, std::numeric_limits<double>::min());
    double small = largest / cells, large = largest;
    for (int it = 0; it < 200; ++it) {
        const double mid = std::sqrt(small * large);
        if (count(mid) > cells)
            small = mid;
        else
            large = mid;
    }
    return large;
}

fh_status pfft_setup(const fh_filament *fil, int64_t n, const PfftConfig &cfg, PfftSetup &out, fh_error_info *err) {
    if (cfg.order < 1) return fail(err, FH_ERR_PFFT, "invalid pFFT parameter: interpolation_order must be at least 1");
    if (!(std::isfinite(cfg.near_field_radius) && cfg.near_field_radius >= (double)(cfg.order + 1)))
        return fail(err, FH_ERR_PFFT,
                    "invalid pFFT parameter: near_field_radius must be finite and at least interpolation_order + 1");
    if (cfg.order > 15) return fail(err, FH_ERR_PFFT, "invalid pFFT parameter: interpolation_order above 15");
    if (!cfg.fixed_spacing && !(cfg.cells_per_filament > 0.0 && std::isfinite(cfg.cells_per_filament)))
        return fail(err, FH_ERR_PFFT, "invalid pFFT parameter: cells_per_filament must be positive and finite");
    if (cfg.fixed_spacing && !(cfg.spacing > 0.0 && std::isfinite(cfg.spacing)))
        return fail(err, FH_ERR_PFFT, "invalid pFFT parameter: grid spacing must be positive and finite");
    out = PfftSetup();
    out.n = n;
    if (n == 0) return FH_OK;

    // Bounding box of the filaments' volumes (pfft/mod.rs:600-611).
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = std::numeric_limits<double>::infinity();
        hi[a] = -std::numeric_limits<double>::infinity();
    }
    for (int64_t i = 0; i < n; ++i) {
        const fh_filament &f = fil[i];
        for (int a = 0; a < 3; ++a) {
            const double reach = 0.5 * (f.width * std::fabs(f.dir_width[a]) + f.height * std::fabs(f.dir_height[a]));
            lo[a] = std::min(lo[a], std::min(f.start[a] - reach, f.end[a] - reach));
            hi[a] = std::max(hi[a], std::max(f.start[a] + reach, f.end[a] + reach));
        }
    }
    double extent[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    const double h = cfg.fixed_spacing ? cfg.spacing : auto_spacing(extent, cfg.cells_per_filament * (double)n);
    PfftGrid &g = out.grid;
    g.spacing = h;
    g.stencil = cfg.order + 1;
    const double pad = (double)((g.stencil + 1) / 2);
    for (int a = 0; a < 3; ++a) {
        g.origin[a] = lo[a] - pad * h;
        const double span = (hi[a] - g.origin[a]) / h;
        g.dims[a] = (int64_t)std::floor(span + 0.5 * g.stencil) + 2;
        out.padded[a] = padded_size(g.dims[a]);
    }
    const double padded_pts = (double)out.padded[0] * (double)out.padded[1] * (double)out.padded[2];
    if (padded_pts > (double)kMaxFftPoints || (double)g.len() > 4294967295.0)
        return fail(err, FH_ERR_PFFT,
                    "pFFT grid of " + std::to_string((long long)padded_pts) + " padded points exceeds the limit of " +
                        std::to_string((long long)kMaxFftPoints));
    const double radius = cfg.near_field_radius * h;

    out.radius = radius;

    // Near pairs and the non-orthogonal partners of each row, row-major.
    std::vector<Bar> bars((size_t)n);
    for (int64_t i = 0; i < n; ++i) bars[i] = bar_of(fil[i]);
    std::vector<std::vector<uint32_t>> near;
    near_pairs(bars, radius, near);
    out.pair_off.assign((size_t)n + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
        for (uint32_t j : near[i]) {
            const double c = dot3(fil[i].dir_length, fil[j].dir_length);
            if (std::fabs(c) < kOrthogonalCos) continue;
            out.pair_i.push_back((int32_t)i);
            out.pair_j.push_back((int32_t)j);
            out.pair_cos.push_back(c);
        }
        out.pair_off[(size_t)i + 1] = (int64_t)out.pair_i.size();
    }
    out.directions.resize((size_t)n * 3);
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) out.directions[3 * i + a] = fil[i].dir_length[a];
    for (int a = 0; a < 3; ++a) {
        bool any = false;
        for (int64_t i = 0; i < n && !any; ++i) any = fil[i].dir_length[a] != 0.0;
        if (any) out.components.push_back(a);
    }
    return FH_OK;
}

}  // namespace fhb
