// Host set-up of the precorrected-FFT operator: grid, projection of every
// filament onto it, near-pair search and the grid's approximation of every
// near pair (to be replaced by the exact value).  The method is the
// reference's (pfft/mod.rs:332-460, grid.rs:44-216, near.rs:41-401):
//
//   * grid of spacing h over the filaments' bounding box, padded by half a
//     stencil, h from GridSpacing::Auto (about cells_per_filament cells per
//     filament) or fixed;
//   * projection: a composite Gauss-Legendre rule over each filament's
//     length, width and height (pieces no longer than h, order from the
//     1e-10 / 12 order table at the near-field distance), every node
//     interpolated onto its (order+1)^3 Lagrange stencil, weights summed per
//     grid point;
//   * near pairs: uniform bins about the radius in size; a pair is near when
//     the separating-axis gap of the two bars is below radius = k h;
//   * grid approximation of a near pair, sum_g sum_h W_ig W_jh K(g - h), by
//     the cheaper of the direct double sum and the potential of i's
//     projection over the box spanned by its partners' projections.
//
// Rows are independent and run in parallel (host threads); every row's arithmetic
// is in a fixed order, so the result does not depend on the thread count.
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

constexpr double kQuadratureTolerance = 1e-10;  // grid.rs:38
constexpr int kQuadratureMaxOrder = 12;         // grid.rs:40
constexpr double kOrthogonalCos = 1e-14;        // near.rs:25

struct Rule {
    std::vector<double> x, w;
};

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

// OrderTable(1e-10, 12).order_for (gauss.rs:123-136); 0 when none suffices.
struct OrderTable {
    double threshold[kQuadratureMaxOrder];
    OrderTable() {
        const double lg = std::log(1.0 / kQuadratureTolerance);
        for (int k = 1; k <= kQuadratureMaxOrder; ++k) threshold[k - 1] = std::sinh(lg / (2.0 * k));
    }
    int order_for(double half, double distance) const {
        if (half <= 0.0) return 1;
        if (std::isnan(distance) || distance <= 0.0) return 0;
        const double delta = distance / half;
        for (int k = 0; k < kQuadratureMaxOrder; ++k)
            if (delta >= threshold[k]) return k + 1;
        return 0;
    }
};

// First stencil plane along `axis` for coordinate x and the Lagrange weights
// of the m planes from there (grid.rs:100-120).
int64_t axis_stencil(const PfftGrid &g, int axis, double x, double *w) {
    const int m = g.stencil;
    const double u = (x - g.origin[axis]) / g.spacing;
    double f = std::floor(u - 0.5 * m) + 1.0;
    int64_t first = f > 0.0 ? (int64_t)f : 0;
    first = std::min<int64_t>(first, g.dims[axis] - m);
    const double t = u - (double)first;
    for (int k = 0; k < m; ++k) {
        double v = 1.0;
        for (int l = 0; l < m; ++l)
            if (l != k) v *= (t - (double)l) / ((double)k - (double)l);
        w[k] = v;
    }
    return first;
}

struct Projection {
    std::vector<std::pair<uint32_t, double>> entries;  // ascending grid index
    int64_t lo[3], hi[3];                               // inclusive box, grid coordinates
};

void point_of(const PfftGrid &g, int64_t index, int64_t p[3]) {
    p[2] = index % g.dims[2];
    const int64_t rest = index / g.dims[2];
    p[0] = rest / g.dims[1];
    p[1] = rest % g.dims[1];
}

// grid.rs:145-216.
void project(const PfftGrid &g, const fh_filament &f, double far_distance, const OrderTable &table,
             const std::vector<Rule> &rules, Projection &out) {
    const double *axes[3] = {f.dir_length, f.dir_width, f.dir_height};
    const double extents[3] = {f.length, f.width, f.height};
    double corner[3];
    for (int k = 0; k < 3; ++k) corner[k] = f.start[k] - 0.5 * f.width * f.dir_width[k] - 0.5 * f.height * f.dir_height[k];
    std::vector<std::pair<double, double>> nodes[3];
    for (int d = 0; d < 3; ++d) {
        const double extent = extents[d];
        const int64_t pieces = std::max<int64_t>(1, (int64_t)std::ceil(extent / g.spacing));
        const double piece = extent / (double)pieces;
        int order = table.order_for(0.5 * piece, far_distance);
        if (order == 0) order = kQuadratureMaxOrder;
        const Rule &r = rules[order];
        for (int64_t p = 0; p < pieces; ++p) {
            const double a = (double)p * piece, b = (double)(p + 1) * piece;
            const double mid = 0.5 * (a + b), half = 0.5 * (b - a);
            for (int q = 0; q < order; ++q) nodes[d].push_back({mid + half * r.x[q], half * r.w[q]});
        }
    }
    const double inverse_area = 1.0 / (f.width * f.height);
    const int m = g.stencil;
    std::vector<std::pair<int64_t, double>> raw;
    raw.reserve(nodes[0].size() * nodes[1].size() * nodes[2].size() * m * m * m);
    double wx[16], wy[16], wz[16];
    for (const auto &sn : nodes[0])
        for (const auto &an : nodes[1])
            for (const auto &bn : nodes[2]) {
                double r[3];
                for (int k = 0; k < 3; ++k) r[k] = corner[k] + sn.first * axes[0][k] + an.first * axes[1][k] + bn.first * axes[2][k];
                const double weight = sn.second * an.second * bn.second * inverse_area;
                const int64_t fx = axis_stencil(g, 0, r[0], wx);
                const int64_t fy = axis_stencil(g, 1, r[1], wy);
                const int64_t fz = axis_stencil(g, 2, r[2], wz);
                for (int i = 0; i < m; ++i)
                    for (int j = 0; j < m; ++j) {
                        const int64_t row = ((fx + i) * g.dims[1] + (fy + j)) * g.dims[2] + fz;
                        const double lxy = weight * wx[i] * wy[j];
                        for (int k = 0; k < m; ++k) raw.push_back({row + k, lxy * wz[k]});
                    }
            }
    std::stable_sort(raw.begin(), raw.end(),
                     [](const std::pair<int64_t, double> &a, const std::pair<int64_t, double> &b) { return a.first < b.first; });
    out.entries.clear();
    for (const auto &e : raw) {
        if (!out.entries.empty() && (int64_t)out.entries.back().first == e.first)
            out.entries.back().second += e.second;
        else
            out.entries.push_back({(uint32_t)e.first, e.second});
    }
    for (int a = 0; a < 3; ++a) {
        out.lo[a] = std::numeric_limits<int64_t>::max();
        out.hi[a] = 0;
    }
    for (const auto &e : out.entries) {
        int64_t p[3];
        point_of(g, e.first, p);
        for (int a = 0; a < 3; ++a) {
            out.lo[a] = std::min(out.lo[a], p[a]);
            out.hi[a] = std::max(out.hi[a], p[a]);
        }
    }
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

// grid_kernel tabulated over |d_a| <= reach_a, z fastest (near.rs:134-170).
struct KernelTable {
    int64_t reach[3], dims[3];
    std::vector<double> values;
    KernelTable(const int64_t r[3], double spacing) {
        for (int a = 0; a < 3; ++a) {
            reach[a] = r[a];
            dims[a] = 2 * r[a] + 1;
        }
        values.assign((size_t)(dims[0] * dims[1] * dims[2]), 0.0);
        parallel_for(dims[0], 1, [&](int64_t x) {
            for (int64_t y = 0; y < dims[1]; ++y)
                for (int64_t z = 0; z < dims[2]; ++z)
                    values[(x * dims[1] + y) * dims[2] + z] =
                        grid_kernel(x - reach[0], y - reach[1], z - reach[2], spacing);
        });
    }
    size_t index(int64_t dx, int64_t dy, int64_t dz) const {
        return (size_t)(((dx + reach[0]) * dims[1] + (dy + reach[1])) * dims[2] + (dz + reach[2]));
    }
};

// sum_g sum_h W_ig W_jh K(g - h) for every partner j of row i (near.rs:323-401).
void grid_interactions(const PfftGrid &g, const std::vector<Projection> &proj, int64_t i,
                       const std::vector<uint32_t> &partners, const KernelTable &table, std::vector<double> &out) {
    const Projection &own = proj[i];
    std::vector<std::array<int64_t, 3>> src_pt(own.entries.size());
    for (size_t s = 0; s < own.entries.size(); ++s) {
        int64_t p[3];
        point_of(g, own.entries[s].first, p);
        src_pt[s] = {p[0], p[1], p[2]};
    }
    int64_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = std::numeric_limits<int64_t>::max();
        hi[a] = 0;
    }
    int64_t partner_entries = 0;
    for (uint32_t j : partners) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], proj[j].lo[a]);
            hi[a] = std::max(hi[a], proj[j].hi[a]);
        }
        partner_entries += (int64_t)proj[j].entries.size();
    }
    const int64_t bx = hi[0] - lo[0] + 1, by = hi[1] - lo[1] + 1, bz = hi[2] - lo[2] + 1;
    const int64_t box_len = bx * by * bz;
    const int64_t ns = (int64_t)src_pt.size();
    const int64_t direct_cost = ns * partner_entries;
    const int64_t box_cost = ns * box_len + partner_entries;
    out.assign(partners.size(), 0.0);
    if (direct_cost <= box_cost) {
        for (size_t q = 0; q < partners.size(); ++q) {
            double total = 0.0;
            for (const auto &e : proj[partners[q]].entries) {
                int64_t h[3];
                point_of(g, e.first, h);
                double potential = 0.0;
                for (int64_t s = 0; s < ns; ++s)
                    potential += own.entries[s].second *
                                 table.values[table.index(h[0] - src_pt[s][0], h[1] - src_pt[s][1], h[2] - src_pt[s][2])];
                total += e.second * potential;
            }
            out[q] = total;
        }
        return;
    }
    std::vector<double> psi((size_t)box_len, 0.0);
    for (int64_t s = 0; s < ns; ++s) {
        const double wg = own.entries[s].second;
        const int64_t *gp = src_pt[s].data();
        for (int64_t x = 0; x < bx; ++x) {
            const int64_t at0 = lo[0] + x - gp[0] + table.reach[0];
            size_t start = (size_t)((at0 * table.dims[1] + (lo[1] - gp[1] + table.reach[1])) * table.dims[2] +
                                    (lo[2] - gp[2] + table.reach[2]));
            for (int64_t y = 0; y < by; ++y) {
                const double *k = &table.values[start];
                double *row = &psi[(size_t)((x * by + y) * bz)];
                for (int64_t z = 0; z < bz; ++z) row[z] += wg * k[z];
                start += (size_t)table.dims[2];
            }
        }
    }
    for (size_t q = 0; q < partners.size(); ++q) {
        double total = 0.0;
        for (const auto &e : proj[partners[q]].entries) {
            int64_t p[3];
            point_of(g, e.first, p);
            total += e.second * psi[(size_t)(((p[0] - lo[0]) * by + (p[1] - lo[1])) * bz + (p[2] - lo[2]))];
        }
        out[q] = total;
    }
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

    // Projections.
    std::vector<Rule> rules(kQuadratureMaxOrder + 1);
    for (int k = 1; k <= kQuadratureMaxOrder; ++k) {
        rules[k].x.resize(k);
        rules[k].w.resize(k);
        gauss_rule(k, rules[k].x.data(), rules[k].w.data());
    }
    const OrderTable table;
    std::vector<Projection> proj((size_t)n);
    parallel_for(n, 16, [&](int64_t i) { project(g, fil[i], radius, table, rules, proj[i]); });

    // Near pairs and the non-orthogonal partners of each row.
    std::vector<Bar> bars((size_t)n);
    for (int64_t i = 0; i < n; ++i) bars[i] = bar_of(fil[i]);
    std::vector<std::vector<uint32_t>> near;
    near_pairs(bars, radius, near);
    std::vector<std::vector<uint32_t>> partners((size_t)n);
    parallel_for(n, 256, [&](int64_t i) {
        for (uint32_t j : near[i])
            if (std::fabs(dot3(fil[i].dir_length, fil[j].dir_length)) >= kOrthogonalCos) partners[i].push_back(j);
    });

    // Offsets the precorrection evaluates (near.rs:244-253).
    int64_t reach[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i) {
        if (partners[i].empty()) continue;
        int64_t plo[3], phi[3];
        for (int a = 0; a < 3; ++a) {
            plo[a] = std::numeric_limits<int64_t>::max();
            phi[a] = 0;
        }
        for (uint32_t j : partners[i])
            for (int a = 0; a < 3; ++a) {
                plo[a] = std::min(plo[a], proj[j].lo[a]);
                phi[a] = std::max(phi[a], proj[j].hi[a]);
            }
        const Projection &own = proj[i];
        for (int a = 0; a < 3; ++a) {
            const int64_t r = std::max(phi[a] - std::min(own.lo[a], phi[a]), own.hi[a] - std::min(plo[a], own.hi[a]));
            reach[a] = std::max(reach[a], r);
        }
    }
    const KernelTable ktable(reach, h);

    std::vector<std::vector<double>> approx((size_t)n);
    parallel_for(n, 4, [&](int64_t i) {
        if (!partners[i].empty()) grid_interactions(g, proj, i, partners[i], ktable, approx[i]);
    });

    for (int64_t i = 0; i < n; ++i)
        for (size_t q = 0; q < partners[i].size(); ++q) {
            const uint32_t j = partners[i][q];
            out.pair_i.push_back((int32_t)i);
            out.pair_j.push_back((int32_t)j);
            out.pair_grid.push_back(approx[i][q]);
            out.pair_cos.push_back(dot3(fil[i].dir_length, fil[j].dir_length));
        }

    // Projection CSR and its transpose (pfft/mod.rs:405-431).
    out.proj_offsets.assign((size_t)n + 1, 0);
    std::vector<int64_t> counts((size_t)g.len(), 0);
    for (int64_t i = 0; i < n; ++i) {
        for (const auto &e : proj[i].entries) {
            out.proj_index.push_back(e.first);
            out.proj_weight.push_back(e.second);
            counts[e.first] += 1;
        }
        out.proj_offsets[i + 1] = (int64_t)out.proj_index.size();
    }
    out.spread_offsets.assign((size_t)g.len() + 1, 0);
    for (int64_t p = 0; p < g.len(); ++p) out.spread_offsets[p + 1] = out.spread_offsets[p] + counts[p];
    std::vector<int64_t> fill(out.spread_offsets.begin(), out.spread_offsets.end() - 1);
    out.spread_filament.assign(out.proj_index.size(), 0);
    out.spread_weight.assign(out.proj_index.size(), 0.0);
    for (int64_t i = 0; i < n; ++i)
        for (const auto &e : proj[i].entries) {
            const int64_t slot = fill[e.first]++;
            out.spread_filament[slot] = (uint32_t)i;
            out.spread_weight[slot] = e.second;
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
