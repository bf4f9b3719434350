// CPU oracle for the fasterhenry PEEC dense path — TEST INFRASTRUCTURE ONLY.
//
// A restatement, in plain C++17 with OpenMP, of the reference algorithm
// (2AMLogic/fasterhenry, Rust).  Every routine cites the reference file:line
// it follows; paths are relative to the reference project root.  Floating
// point expressions keep the reference's evaluation order and the library is
// compiled with -ffp-contract=off, so that the method-dispatch decisions
// (orthogonality, parallelism, alignment, separation, Gauss orders) are the
// reference's bit for bit.  Only tests/, __graft_entry__.smoke() and bench.py
// use it.
#include "fh_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <limits>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTau = 6.28318530717958647692;
constexpr double kMu0 = 4.0e-7 * kPi;            // inductance/mod.rs:76
constexpr double kMu0Over4Pi = 1.0e-7;           // inductance/mod.rs:79
constexpr double kClosedFormMaxError = 1e-10;    // inductance/mod.rs:82
constexpr double kOrthogonalCos = 1e-14;         // inductance/mod.rs:84
constexpr size_t kCheapPointPairs = 4096;        // inductance/mod.rs:88
constexpr double kParallelSin = 1e-6;            // inductance/neumann.rs:53
constexpr double kPointTolerance = 1e-8;         // neumann.rs:32
constexpr int kPointMaxOrder = 16;               // neumann.rs:34
constexpr int kCloudCapacity = 256;              // neumann.rs:36
constexpr double kSampleTolerance = 1e-6;        // neumann.rs:38
constexpr int kSampleMaxOrder = 8;               // neumann.rs:40
constexpr int kFarOrder = 10;                    // aligned.rs:239
constexpr int kCornerOrder = 16;                 // aligned.rs:241
constexpr double kSnap = 1e-12;                  // aligned.rs:244
constexpr double kEps = std::numeric_limits<double>::epsilon();

// ---------------------------------------------------------------------------
// 3-vectors with nalgebra's evaluation order: dot = (x*x' + y*y') + z*z'.
// ---------------------------------------------------------------------------
struct V3 {
    double x, y, z;
};
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 dvd(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 vabs(V3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline double rmax(double a, double b) {  // Rust f64::max: NaN loses
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return a > b ? a : b;
}
inline double rmin(double a, double b) {
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return a < b ? a : b;
}
inline double signum(double x) {  // Rust f64::signum
    if (std::isnan(x)) return x;
    return std::signbit(x) ? -1.0 : 1.0;
}

// ---------------------------------------------------------------------------
// Gauss-Legendre rules, inductance/gauss.rs:13-79
// ---------------------------------------------------------------------------
struct Rule {
    std::vector<double> nodes, weights;
};

Rule make_rule(int n) {
    Rule r;
    r.nodes.assign(n, 0.0);
    r.weights.assign(n, 0.0);
    const double nf = (double)n;
    for (int k = 0; k < (n + 1) / 2; ++k) {
        double x = std::cos(kPi * ((double)k + 0.75) / (nf + 0.5));
        double derivative = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p_prev = 1.0, p = x;
            for (int j = 1; j < n; ++j) {
                double jf = (double)j;
                double p_next = ((2.0 * jf + 1.0) * x * p - jf * p_prev) / (jf + 1.0);
                p_prev = p;
                p = p_next;
            }
            derivative = nf * (x * p - p_prev) / (x * x - 1.0);
            double step = p / derivative;
            x -= step;
            if (std::fabs(step) <= 4.0 * kEps * rmax(std::fabs(x), 1e-3)) break;
        }
        if (n % 2 == 1 && k == n / 2) {
            x = 0.0;
            double p_prev = 1.0, p = x;
            for (int j = 1; j < n; ++j) {
                double jf = (double)j;
                double p_next = ((2.0 * jf + 1.0) * x * p - jf * p_prev) / (jf + 1.0);
                p_prev = p;
                p = p_next;
            }
            derivative = nf * (x * p - p_prev) / (x * x - 1.0);
        }
        double weight = 2.0 / ((1.0 - x * x) * derivative * derivative);
        r.nodes[n - 1 - k] = x;
        r.nodes[k] = -x;
        r.weights[n - 1 - k] = weight;
        r.weights[k] = weight;
    }
    return r;
}

const Rule &rule(int n) {
    static std::vector<Rule> rules;
    static std::once_flag once;
    std::call_once(once, [] {
        for (int k = 1; k <= 64; ++k) rules.push_back(make_rule(k));
    });
    n = std::min(std::max(n, 1), 64);
    return rules[n - 1];
}

// Rule::on, gauss.rs:73-79: (mid + half*x, half*w).
inline void rule_on(const Rule &r, double a, double b, int k, double *x, double *w) {
    double mid = 0.5 * (a + b), half = 0.5 * (b - a);
    *x = mid + half * r.nodes[k];
    *w = half * r.weights[k];
}

// OrderTable, gauss.rs:100-137.
struct OrderTable {
    std::vector<double> thresholds;
    OrderTable(double tolerance, int max_order) {
        double log = std::log(1.0 / tolerance);
        for (int n = 1; n <= max_order; ++n) thresholds.push_back(std::sinh(log / (2.0 * (double)n)));
    }
    int max_order() const { return (int)thresholds.size(); }
    // 0 stands for None.
    int order_for(double half_extent, double distance) const {
        if (half_extent <= 0.0) return 1;
        if (std::isnan(distance) || distance <= 0.0) return 0;
        double delta = distance / half_extent;
        for (size_t i = 0; i < thresholds.size(); ++i)
            if (delta >= thresholds[i]) return (int)i + 1;
        return 0;
    }
};
const OrderTable &point_table() {
    static OrderTable t(kPointTolerance, kPointMaxOrder);
    return t;
}
const OrderTable &sample_table() {
    static OrderTable t(kSampleTolerance, kSampleMaxOrder);
    return t;
}

// ---------------------------------------------------------------------------
// Filaments (filament.rs) and bars (neumann.rs:57-87)
// ---------------------------------------------------------------------------
struct Fil {
    V3 start, end;
    double length;
    V3 l, w, h;
    double width, height, sigma;
};
Fil load_fil(const double *p) {
    Fil f;
    f.start = {p[0], p[1], p[2]};
    f.end = {p[3], p[4], p[5]};
    f.length = p[6];
    f.l = {p[7], p[8], p[9]};
    f.w = {p[10], p[11], p[12]};
    f.h = {p[13], p[14], p[15]};
    f.width = p[16];
    f.height = p[17];
    f.sigma = p[18];
    return f;
}
void store_fil(const Fil &f, double *p) {
    double v[19] = {f.start.x, f.start.y, f.start.z, f.end.x, f.end.y, f.end.z, f.length,
                    f.l.x,     f.l.y,     f.l.z,     f.w.x,   f.w.y,   f.w.z,   f.h.x,
                    f.h.y,     f.h.z,     f.width,   f.height, f.sigma};
    std::memcpy(p, v, sizeof v);
}
inline V3 centre_of(const Fil &f) { return mul(add(f.start, f.end), 0.5); }
inline double area_of(const Fil &f) { return f.width * f.height; }

struct Bar {
    V3 centre;
    V3 axes[3];
    double half[3];
};
Bar make_bar(const Fil &f) {
    Bar b;
    b.centre = centre_of(f);
    b.axes[0] = f.l;
    b.axes[1] = f.w;
    b.axes[2] = f.h;
    b.half[0] = 0.5 * f.length;
    b.half[1] = 0.5 * f.width;
    b.half[2] = 0.5 * f.height;
    return b;
}
inline double circumradius(const Bar &b) {
    return std::sqrt((b.half[0] * b.half[0] + b.half[1] * b.half[1]) + b.half[2] * b.half[2]);
}
inline double projected_half_extent(const Bar &b, V3 n) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s = s + b.half[k] * std::fabs(dot(n, b.axes[k]));
    return s;
}

// neumann.rs:97-122
double separation(const Bar &a, const Bar &b) {
    V3 delta = sub(b.centre, a.centre);
    double distance = norm(delta), reach = circumradius(a) + circumradius(b);
    if (distance > 8.0 * reach) return distance - reach;
    double best = -std::numeric_limits<double>::infinity();
    auto consider = [&](V3 n) {
        double gap = std::fabs(dot(n, delta)) - projected_half_extent(a, n) - projected_half_extent(b, n);
        best = rmax(best, gap);
    };
    for (int k = 0; k < 3; ++k) {
        consider(a.axes[k]);
        consider(b.axes[k]);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            V3 n = cross(a.axes[i], b.axes[j]);
            double nn = norm(n);
            if (nn > 1e-9) consider(dvd(n, nn));
        }
    return best;
}

// neumann.rs:127-134; false = None.
bool point_orders(const Bar &bar, double gap, int o[3]) {
    const OrderTable &t = point_table();
    for (int k = 0; k < 3; ++k) {
        o[k] = t.order_for(bar.half[k], gap);
        if (o[k] == 0) return false;
    }
    return o[0] * o[1] * o[2] <= kCloudCapacity;
}

// Cloud::fill, neumann.rs:160-184 (padding is only for SIMD lanes).
struct Cloud {
    double x[kCloudCapacity], y[kCloudCapacity], z[kCloudCapacity], w[kCloudCapacity];
    int len;
};
void fill_cloud(Cloud &c, const Bar &bar, const int o[3]) {
    const Rule &rl = rule(o[0]), &rw = rule(o[1]), &rh = rule(o[2]);
    int i = 0;
    for (int a = 0; a < o[0]; ++a) {
        double xl, wl;
        rule_on(rl, -bar.half[0], bar.half[0], a, &xl, &wl);
        for (int b = 0; b < o[1]; ++b) {
            double xw, ww;
            rule_on(rw, -0.5, 0.5, b, &xw, &ww);
            for (int d = 0; d < o[2]; ++d) {
                double xh, wh;
                rule_on(rh, -0.5, 0.5, d, &xh, &wh);
                V3 p = add(add(add(bar.centre, mul(bar.axes[0], xl)), mul(bar.axes[1], 2.0 * bar.half[1] * xw)),
                           mul(bar.axes[2], 2.0 * bar.half[2] * xh));
                c.x[i] = p.x;
                c.y[i] = p.y;
                c.z[i] = p.z;
                c.w[i] = wl * ww * wh;
                ++i;
            }
        }
    }
    c.len = i;
}

// point_sum_simd, neumann.rs:237-266: four accumulation lanes per inner sum.
double point_sum(const Bar &a, const int oa[3], const Bar &b, const int ob[3]) {
    static thread_local Cloud ca, cb;
    fill_cloud(ca, a, oa);
    fill_cloud(cb, b, ob);
    double total = 0.0;
    for (int i = 0; i < ca.len; ++i) {
        double lane[4] = {0.0, 0.0, 0.0, 0.0};
        for (int j = 0; j < cb.len; ++j) {
            double dx = ca.x[i] - cb.x[j], dy = ca.y[i] - cb.y[j], dz = ca.z[i] - cb.z[j];
            lane[j & 3] += cb.w[j] / std::sqrt(dx * dx + dy * dy + dz * dz);
        }
        total += ca.w[i] * ((lane[0] + lane[1]) + (lane[2] + lane[3]));
    }
    return total;
}

// ---------------------------------------------------------------------------
// Line-line closed forms, inductance/lines.rs:31-170
// ---------------------------------------------------------------------------
inline double parallel_primitive(double q, double rho_sq) {
    q = std::fabs(q);
    double root = std::sqrt(q * q + rho_sq);
    if (q == 0.0) return -root;
    return q * std::log(q + root) - root;
}
inline double axial_overlap(double l1, double l2, double offset) {
    return rmax(rmin(l1, offset + l2) - rmax(offset, 0.0), 0.0);
}
// Returns false for the divergent coaxial overlapping case.
inline bool lines_parallel(double l1, double l2, double offset, double rho, double *out) {
    double rho_sq = rho * rho;
    double smooth = parallel_primitive(offset + l2, rho_sq) - parallel_primitive(offset, rho_sq) -
                    parallel_primitive(offset + l2 - l1, rho_sq) + parallel_primitive(offset - l1, rho_sq);
    double overlap = axial_overlap(l1, l2, offset);
    if (overlap == 0.0) {
        *out = smooth;
        return true;
    }
    if (rho > 0.0) {
        *out = smooth - 2.0 * overlap * std::log(rho);
        return true;
    }
    return false;
}
inline double skew_log_term(double x, double big_r, double a, double residual_sq) {
    if (x == 0.0) return 0.0;
    double argument = a >= 0.0 ? big_r + a : residual_sq / (big_r - a);
    if (argument > 0.0) return x * std::log(argument);
    return 0.0;
}
double skew_primitive(double s, double t, double d, double cosv, double sinv) {
    double sin_sq = sinv * sinv;
    double versine = sin_sq / (1.0 + std::fabs(cosv));
    double planar_sq, a_s, a_t;
    if (cosv >= 0.0) {
        double diff = s - t;
        planar_sq = diff * diff + 2.0 * s * t * versine;
        a_s = s * versine - diff;
        a_t = t * versine + diff;
    } else {
        double sum = s + t;
        planar_sq = sum * sum - 2.0 * s * t * versine;
        a_s = sum - s * versine;
        a_t = sum - t * versine;
    }
    double big_r = std::sqrt(rmax(planar_sq + d * d, 0.0));
    double logs = skew_log_term(s, big_r, a_s, s * s * sin_sq + d * d) +
                  skew_log_term(t, big_r, a_t, t * t * sin_sq + d * d);
    if (d == 0.0 || big_r == 0.0) return logs;
    return logs - (d / sinv) * std::atan((d * d * cosv + s * t * sin_sq) / (d * big_r * sinv));
}
bool lines_skew(V3 a0, V3 a1, V3 b0, V3 b1, double sin_min, double *out) {
    double la = norm(sub(a1, a0)), lb = norm(sub(b1, b0));
    V3 u = dvd(sub(a1, a0), la), v = dvd(sub(b1, b0), lb);
    double cosv = dot(u, v);
    double sinv = norm(cross(u, v));
    if (std::isnan(sinv) || sinv < sin_min) return false;
    V3 w0 = sub(a0, b0);
    double du = dot(u, w0), dv = dot(v, w0);
    double sin_sq = sinv * sinv;
    double s0 = (cosv * dv - du) / sin_sq;
    double t0 = (dv - cosv * du) / sin_sq;
    double d = norm(sub(add(w0, mul(u, s0)), mul(v, t0)));
    if (d <= 1e-14 * (la + lb + norm(w0))) d = 0.0;
    double s_lo = -s0, s_hi = la - s0, t_lo = -t0, t_hi = lb - t0;
    *out = skew_primitive(s_hi, t_hi, d, cosv, sinv) - skew_primitive(s_hi, t_lo, d, cosv, sinv) -
           skew_primitive(s_lo, t_hi, d, cosv, sinv) + skew_primitive(s_lo, t_lo, d, cosv, sinv);
    return true;
}

// ---------------------------------------------------------------------------
// Hoer-Love 64-term closed form, inductance/bar.rs:30-106
// ---------------------------------------------------------------------------
inline void corner_differences(double e1, double e2, double offset, double q[4]) {
    double sum = 0.5 * (e1 + e2), diff = 0.5 * (e1 - e2);
    q[0] = offset + sum;
    q[1] = offset + diff;
    q[2] = offset - diff;
    q[3] = offset - sum;
}
constexpr double kSigns[4] = {1.0, -1.0, -1.0, 1.0};
inline double log_term(double coefficient, double x, double r, double rest_sq) {
    if (coefficient == 0.0 || x == 0.0) return 0.0;
    double argument = x >= 0.0 ? x + r : rest_sq / (r - x);
    return coefficient * x * std::log(argument);
}
inline double atan_term(double x, double y, double z, double r) {
    double product = x * y * z;
    if (product == 0.0) return 0.0;
    return -(product * z * z / 6.0) * std::atan(x * y / (z * r));
}
double primitive(double x, double y, double z) {
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double x4 = x2 * x2, y4 = y2 * y2, z4 = z2 * z2;
    double r = std::sqrt(x2 + y2 + z2);
    return log_term(y2 * z2 / 4.0 - y4 / 24.0 - z4 / 24.0, x, r, y2 + z2) +
           log_term(x2 * z2 / 4.0 - x4 / 24.0 - z4 / 24.0, y, r, x2 + z2) +
           log_term(x2 * y2 / 4.0 - x4 / 24.0 - y4 / 24.0, z, r, x2 + y2) +
           (x4 + y4 + z4 - 3.0 * (x2 * y2 + y2 * z2 + z2 * x2)) * r / 60.0 + atan_term(x, y, z, r) +
           atan_term(x, z, y, r) + atan_term(y, z, x, r);
}
void bar_integral(const double qx[4], const double qy[4], const double qz[4], double *value,
                  double *relative_error) {
    double v = 0.0, magnitude = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) {
                double term = kSigns[i] * kSigns[j] * kSigns[k] * primitive(qx[i], qy[j], qz[k]);
                v += term;
                magnitude += std::fabs(term);
            }
    *value = v;
    *relative_error = v > 0.0 ? 8.0 * kEps * magnitude / v : std::numeric_limits<double>::infinity();
}

// ---------------------------------------------------------------------------
// Aligned-bar quadrature, inductance/aligned.rs:206-402
// ---------------------------------------------------------------------------
struct AlignedBars {
    double length[2], width[2], height[2], offset[3];
};
inline double overlap_weight(double e1, double e2, double offset, double u) {
    double hi = rmin(0.5 * e1, offset + 0.5 * e2 - u);
    double lo = rmax(-0.5 * e1, offset - 0.5 * e2 - u);
    return rmax(hi - lo, 0.0);
}
std::vector<double> break_points(double e1, double e2, double offset) {
    double sum = 0.5 * (e1 + e2), diff = 0.5 * std::fabs(e1 - e2);
    auto snap = [&](double x) { return std::fabs(x) <= kSnap * sum ? 0.0 : x; };
    std::vector<double> p = {snap(offset - sum), snap(offset - diff), snap(offset + diff), snap(offset + sum)};
    if (p[0] < 0.0 && p[3] > 0.0) p.push_back(0.0);
    // total_cmp ordering; no NaN reaches here for valid bars.
    std::stable_sort(p.begin(), p.end(), [](double a, double b) {
        if (a == b) return std::signbit(a) && !std::signbit(b);
        return a < b;
    });
    std::vector<double> out;
    for (double x : p)
        if (out.empty() || !(out.back() == x)) out.push_back(x);
    return out;
}

struct Integrator {
    const AlignedBars *bars;
    double axial_start, axial_scale;

    double integrand(double u, double v) const {
        const AlignedBars &b = *bars;
        double weight = overlap_weight(b.width[0], b.width[1], b.offset[1], u) *
                        overlap_weight(b.height[0], b.height[1], b.offset[2], v);
        if (weight == 0.0) return 0.0;
        double kernel;
        if (!lines_parallel(b.length[0], b.length[1], axial_start, std::hypot(u, v), &kernel)) kernel = 0.0;
        return weight * kernel;
    }
    double direct(double u0, double u1, double v0, double v1) const {
        const Rule &r = rule(kFarOrder);
        double sum = 0.0;
        for (int a = 0; a < kFarOrder; ++a) {
            double uu, wu;
            rule_on(r, u0, u1, a, &uu, &wu);
            for (int b = 0; b < kFarOrder; ++b) {
                double vv, wv;
                rule_on(r, v0, v1, b, &vv, &wv);
                sum += wu * wv * integrand(uu, vv);
            }
        }
        return sum;
    }
    double corner(double a, double b) const {
        const Rule &r = rule(kCornerOrder);
        double sum = 0.0;
        for (int i = 0; i < kCornerOrder; ++i) {
            double tau, w_tau;
            rule_on(r, 0.0, 1.0, i, &tau, &w_tau);
            double s = tau * tau * tau;
            double radial = w_tau * 3.0 * tau * tau * s;
            for (int k = 0; k < kCornerOrder; ++k) {
                double t, w_t;
                rule_on(r, 0.0, 1.0, k, &t, &w_t);
                double value = integrand(a * s, b * s * t) + integrand(a * s * t, b * s);
                sum += radial * w_t * value;
            }
        }
        return sum * std::fabs(a * b);
    }
    double panel(double u0, double u1, double v0, double v1, unsigned depth) const {
        double su = u1 - u0, sv = v1 - v0;
        if (su <= 0.0 || sv <= 0.0) return 0.0;
        auto gap = [](double r0, double r1) { return r0 > 0.0 ? r0 : (r1 < 0.0 ? -r1 : 0.0); };
        double distance = std::hypot(gap(u0, u1), gap(v0, v1));
        double size = rmax(su, sv);
        if (depth >= 200) return direct(u0, u1, v0, v1);
        auto split_u = [&](double at) {
            return panel(u0, at, v0, v1, depth + 1) + panel(at, u1, v0, v1, depth + 1);
        };
        auto split_v = [&](double at) {
            return panel(u0, u1, v0, at, depth + 1) + panel(u0, u1, at, v1, depth + 1);
        };
        if (distance > 0.0) {
            if (size <= distance) return direct(u0, u1, v0, v1);
            if (su >= sv) return split_u(0.5 * (u0 + u1));
            return split_v(0.5 * (v0 + v1));
        }
        double target = rmin(rmin(su, sv), axial_scale);
        auto toward = [](double r0, double len) { return r0 == 0.0 ? len : -len; };
        if (su > 2.0 * target) return split_u(toward(u0, target));
        if (sv > 2.0 * target) return split_v(toward(v0, target));
        auto far = [](double r0, double r1) { return r0 == 0.0 ? r1 : r0; };
        return corner(far(u0, u1), far(v0, v1));
    }
};

double aligned_integral_quadrature(const AlignedBars &bars) {
    double axial_start = bars.offset[0] + 0.5 * (bars.length[0] - bars.length[1]);
    double l1 = bars.length[0], l2 = bars.length[1];
    double separations[4] = {axial_start + l2, axial_start, axial_start + l2 - l1, axial_start - l1};
    double largest = 0.0;
    for (double q : separations) largest = rmax(largest, std::fabs(q));
    double axial_scale = std::numeric_limits<double>::infinity();
    for (double q : separations)
        if (std::fabs(q) > 1e-9 * largest) axial_scale = rmin(axial_scale, std::fabs(q));
    Integrator integ{&bars, axial_start, axial_scale};
    std::vector<double> us = break_points(bars.width[0], bars.width[1], bars.offset[1]);
    std::vector<double> vs = break_points(bars.height[0], bars.height[1], bars.offset[2]);
    double sum = 0.0;
    for (size_t a = 0; a + 1 < us.size(); ++a)
        for (size_t b = 0; b + 1 < vs.size(); ++b) sum += integ.panel(us[a], us[a + 1], vs[b], vs[b + 1], 0);
    return sum;
}

// evaluate_aligned_integral, inductance/mod.rs:265-276
double aligned_integral_eval(const AlignedBars &bars, int *method) {
    double qx[4], qy[4], qz[4], value, rel;
    corner_differences(bars.length[0], bars.length[1], bars.offset[0], qx);
    corner_differences(bars.width[0], bars.width[1], bars.offset[1], qy);
    corner_differences(bars.height[0], bars.height[1], bars.offset[2], qz);
    bar_integral(qx, qy, qz, &value, &rel);
    if (rel <= kClosedFormMaxError) {
        *method = ORC_BAR_CLOSED_FORM;
        return value;
    }
    *method = ORC_ALIGNED_QUADRATURE;
    return aligned_integral_quadrature(bars);
}

// Per-thread direct-mapped memo keyed on the nine numbers' bits, as
// inductance/memo.rs:1-130: a hit returns the bits a miss produced, so it
// never moves a value.
struct MemoEntry {
    bool occupied;
    uint64_t key[9];
    double value;
    int method;
};
double aligned_integral(const AlignedBars &bars, int *method) {
    static thread_local std::vector<MemoEntry> table(1024, MemoEntry{false, {0}, 0.0, 0});
    uint64_t key[9];
    std::memcpy(key + 0, bars.length, 16);
    std::memcpy(key + 2, bars.width, 16);
    std::memcpy(key + 4, bars.height, 16);
    std::memcpy(key + 6, bars.offset, 24);
    uint64_t h = 0x9e3779b97f4a7c15ull;
    for (int i = 0; i < 9; ++i) {
        h = (h ^ key[i]) * 0x9e3779b97f4a7c15ull;
        h = (h << 29) | (h >> 35);
    }
    h ^= h >> 30;
    h *= 0xbf58476d1ce4e5b9ull;
    h ^= h >> 27;
    h *= 0x94d049bb133111ebull;
    h ^= h >> 31;
    MemoEntry &e = table[h & 1023];
    if (e.occupied && std::memcmp(e.key, key, sizeof key) == 0) {
        *method = e.method;
        return e.value;
    }
    double v = aligned_integral_eval(bars, method);
    e.occupied = true;
    std::memcpy(e.key, key, sizeof key);
    e.value = v;
    e.method = *method;
    return v;
}

// aligned_bars, inductance/mod.rs:280-300
bool aligned_bars(const Bar &a, const Bar &b, AlignedBars *out) {
    const double kAligned = 1.0 - 1e-12;
    double wb, hb;
    if (std::fabs(dot(a.axes[1], b.axes[1])) > kAligned) {
        wb = b.half[1];
        hb = b.half[2];
    } else if (std::fabs(dot(a.axes[1], b.axes[2])) > kAligned) {
        wb = b.half[2];
        hb = b.half[1];
    } else {
        return false;
    }
    V3 delta = sub(b.centre, a.centre);
    out->length[0] = 2.0 * a.half[0];
    out->length[1] = 2.0 * b.half[0];
    out->width[0] = 2.0 * a.half[1];
    out->width[1] = 2.0 * wb;
    out->height[0] = 2.0 * a.half[2];
    out->height[1] = 2.0 * hb;
    out->offset[0] = dot(delta, a.axes[0]);
    out->offset[1] = dot(delta, a.axes[1]);
    out->offset[2] = dot(delta, a.axes[2]);
    return true;
}

// sampled_filaments, neumann.rs:280-325; false = a divergent sample.
bool sampled_filaments(const Bar &a, const Bar &b, double gap, bool parallel, double *value, bool *resolved) {
    const OrderTable &t = sample_table();
    *resolved = true;
    auto order = [&](double half, int bump) {
        int n = t.order_for(half, gap);
        if (n) return n;
        *resolved = false;
        return t.max_order() + bump;
    };
    int oa[2] = {order(a.half[1], 0), order(a.half[2], 0)};
    int ob[2] = {order(b.half[1], 1), order(b.half[2], 1)};
    auto samples = [](const Bar &bar, const int o[2], std::vector<V3> &pts, std::vector<double> &ws) {
        const Rule &r0 = rule(o[0]), &r1 = rule(o[1]);
        for (int i = 0; i < o[0]; ++i) {
            double xw, ww;
            rule_on(r0, -0.5, 0.5, i, &xw, &ww);
            for (int k = 0; k < o[1]; ++k) {
                double xh, wh;
                rule_on(r1, -0.5, 0.5, k, &xh, &wh);
                V3 offset = add(mul(bar.axes[1], 2.0 * bar.half[1] * xw), mul(bar.axes[2], 2.0 * bar.half[2] * xh));
                pts.push_back(add(bar.centre, offset));
                ws.push_back(ww * wh);
            }
        }
    };
    std::vector<V3> pa, pb;
    std::vector<double> wa, wb;
    samples(a, oa, pa, wa);
    samples(b, ob, pb, wb);
    double la = 2.0 * a.half[0], lb = 2.0 * b.half[0];
    V3 axis = a.axes[0];
    double v = 0.0;
    for (size_t i = 0; i < pa.size(); ++i)
        for (size_t j = 0; j < pb.size(); ++j) {
            double kernel;
            if (parallel) {
                V3 delta = sub(pb[j], pa[i]);
                double along = dot(delta, axis);
                double rho = norm(sub(delta, mul(axis, along)));
                if (!lines_parallel(la, lb, along + 0.5 * (la - lb), rho, &kernel)) return false;
            } else {
                V3 ha = mul(a.axes[0], a.half[0]), hb = mul(b.axes[0], b.half[0]);
                if (!lines_skew(sub(pa[i], ha), add(pa[i], ha), sub(pb[j], hb), add(pb[j], hb), 0.0, &kernel))
                    return false;
            }
            v += wa[i] * wb[j] * kernel;
        }
    *value = v;
    return true;
}

// canonical, inductance/mod.rs:231-254 (f64::total_cmp on 11 keys)
int total_cmp(double x, double y) {
    int64_t a, b;
    std::memcpy(&a, &x, 8);
    std::memcpy(&b, &y, 8);
    a ^= (int64_t)(((uint64_t)(a >> 63)) >> 1);
    b ^= (int64_t)(((uint64_t)(b >> 63)) >> 1);
    return a < b ? -1 : (a > b ? 1 : 0);
}
int canonical(const Fil &a, const Fil &b) {
    double ka[11] = {a.start.x, a.start.y, a.start.z, a.end.x, a.end.y, a.end.z, a.width, a.height, a.w.x, a.w.y, a.w.z};
    double kb[11] = {b.start.x, b.start.y, b.start.z, b.end.x, b.end.y, b.end.z, b.width, b.height, b.w.x, b.w.y, b.w.z};
    for (int i = 0; i < 11; ++i) {
        int c = total_cmp(ka[i], kb[i]);
        if (c) return c;
    }
    return 0;
}

// evaluate, inductance/mod.rs:303-369.  Returns an ORC status.
int evaluate(const Fil &a0, const Fil &b0, double *out, int *method_out, bool *resolved_out) {
    const Fil *pa = &a0, *pb = &b0;
    if (canonical(a0, b0) > 0) std::swap(pa, pb);
    const Fil &a = *pa, &b = *pb;
    double cosv = dot(a.l, b.l);
    if (std::fabs(cosv) < kOrthogonalCos) {
        *out = 0.0;
        *method_out = ORC_ORTHOGONAL;
        *resolved_out = true;
        return ORC_OK;
    }
    Bar ba = make_bar(a), bb = make_bar(b);
    bool parallel = norm(cross(a.l, b.l)) < kParallelSin;
    AlignedBars ab;
    bool aligned = parallel && aligned_bars(ba, bb, &ab);
    double gap = separation(ba, bb);
    int oa[3], ob[3];
    bool have = point_orders(ba, gap, oa) && point_orders(bb, gap, ob);
    if (have && aligned) {
        size_t pairs = (size_t)(oa[0] * oa[1] * oa[2]) * (size_t)(ob[0] * ob[1] * ob[2]);
        if (pairs > kCheapPointPairs) have = false;
    }
    double integral;
    int method;
    bool resolved = true;
    if (have) {
        integral = point_sum(ba, oa, bb, ob) * cosv;
        method = ORC_POINT_QUADRATURE;
    } else if (aligned) {
        double v = aligned_integral(ab, &method);
        double scale = signum(cosv) / (area_of(a) * area_of(b));
        integral = v * scale;
    } else {
        double v;
        if (!sampled_filaments(ba, bb, gap, parallel, &v, &resolved)) return ORC_ERR_COINCIDENT;
        double direction = parallel ? signum(cosv) : cosv;
        integral = v * direction;
        method = ORC_SAMPLED_FILAMENTS;
    }
    double value = kMu0Over4Pi * integral;
    if (!std::isfinite(value)) return ORC_ERR_NOT_FINITE;
    *out = value;
    *method_out = method;
    *resolved_out = resolved;
    return ORC_OK;
}

// ---------------------------------------------------------------------------
// Frozen-dispatch evaluation, for finite-difference checks of the impedance
// gradient (no reference counterpart).  Every decision the reference's
// evaluate() takes (inductance/mod.rs:303-369: orthogonality, alignment,
// Gauss orders, point quadrature vs aligned path, closed-form acceptance,
// and the aligned quadrature's break points and panel tree, aligned.rs:
// 86-232) is taken on the nominal pair and replayed on the perturbed pair,
// so that a central difference sees the evaluation as one smooth function.
// ---------------------------------------------------------------------------
// Break points with the formula that produced each (aligned.rs:86-120):
// 0 offset-sum, 1 offset-diff, 2 offset+diff, 3 offset+sum, 4 zero.
std::vector<int> break_tags(double e1, double e2, double offset) {
    double sum = 0.5 * (e1 + e2), diff = 0.5 * std::fabs(e1 - e2);
    auto snap = [&](double x) { return std::fabs(x) <= kSnap * sum ? 0.0 : x; };
    double raw[4] = {offset - sum, offset - diff, offset + diff, offset + sum};
    std::vector<std::pair<double, int>> p;
    for (int k = 0; k < 4; ++k) {
        double v = snap(raw[k]);
        p.push_back({v, v == 0.0 ? 4 : k});
    }
    if (p[0].first < 0.0 && p[3].first > 0.0) p.push_back({0.0, 4});
    std::stable_sort(p.begin(), p.end(), [](const std::pair<double, int> &a, const std::pair<double, int> &b) {
        if (a.first == b.first) return std::signbit(a.first) && !std::signbit(b.first);
        return a.first < b.first;
    });
    std::vector<int> out;
    double last = 0.0;
    for (size_t k = 0; k < p.size(); ++k)
        if (out.empty() || !(last == p[k].first)) {
            out.push_back(p[k].second);
            last = p[k].first;
        }
    return out;
}
double break_value(int tag, double e1, double e2, double offset) {
    double sum = 0.5 * (e1 + e2), diff = 0.5 * std::fabs(e1 - e2);
    switch (tag) {
        case 0: return offset - sum;
        case 1: return offset - diff;
        case 2: return offset + diff;
        case 3: return offset + sum;
        default: return 0.0;
    }
}

// Panel decisions (aligned.rs:153-200) as codes: 0 empty, 1 direct, 2/3
// split u/v at the midpoint, 16 + 8 axis + 4 negative + source for a split
// toward zero at +-target (source 0 su, 1 sv, 2 axial scale), 32 + 2 fu + fv
// for a corner (fu: the far u is u1, else u0).
struct FrozenIntegrator {
    Integrator in;
    std::vector<unsigned char> *log;
    size_t cursor = 0;

    double panel(double u0, double u1, double v0, double v1, unsigned depth, bool record) {
        double su = u1 - u0, sv = v1 - v0;
        unsigned char code;
        if (record) {
            if (su <= 0.0 || sv <= 0.0) {
                code = 0;
            } else {
                auto gap = [](double r0, double r1) { return r0 > 0.0 ? r0 : (r1 < 0.0 ? -r1 : 0.0); };
                double distance = std::hypot(gap(u0, u1), gap(v0, v1));
                double size = rmax(su, sv);
                if (depth >= 200) {
                    code = 1;
                } else if (distance > 0.0) {
                    code = size <= distance ? 1 : (su >= sv ? 2 : 3);
                } else {
                    int src = 0;
                    double target = su;
                    if (sv < target) target = sv, src = 1;
                    if (in.axial_scale < target) target = in.axial_scale, src = 2;
                    if (su > 2.0 * target)
                        code = (unsigned char)(16 + (u0 == 0.0 ? 0 : 4) + src);
                    else if (sv > 2.0 * target)
                        code = (unsigned char)(24 + (v0 == 0.0 ? 0 : 4) + src);
                    else
                        code = (unsigned char)(32 + (u0 == 0.0 ? 2 : 0) + (v0 == 0.0 ? 1 : 0));
                }
            }
            log->push_back(code);
        } else {
            code = (*log)[cursor++];
        }
        if (code == 0) return 0.0;
        if (code == 1) return in.direct(u0, u1, v0, v1);
        if (code == 2) {
            double at = 0.5 * (u0 + u1);
            double a = panel(u0, at, v0, v1, depth + 1, record);
            return a + panel(at, u1, v0, v1, depth + 1, record);
        }
        if (code == 3) {
            double at = 0.5 * (v0 + v1);
            double a = panel(u0, u1, v0, at, depth + 1, record);
            return a + panel(u0, u1, at, v1, depth + 1, record);
        }
        if (code >= 32) {
            double fu = (code & 2) ? u1 : u0, fv = (code & 1) ? v1 : v0;
            return in.corner(fu, fv);
        }
        const int src = code & 3;
        const double target = src == 0 ? su : (src == 1 ? sv : in.axial_scale);
        const double at_len = (code & 4) ? -target : target;
        if (code < 24) {
            double a = panel(u0, at_len, v0, v1, depth + 1, record);
            return a + panel(at_len, u1, v0, v1, depth + 1, record);
        }
        double a = panel(u0, u1, v0, at_len, depth + 1, record);
        return a + panel(u0, u1, at_len, v1, depth + 1, record);
    }
};

double frozen_quadrature(const AlignedBars &nom, const AlignedBars &per) {
    auto setup = [](const AlignedBars &b, Integrator &in) {
        double axial_start = b.offset[0] + 0.5 * (b.length[0] - b.length[1]);
        double l1 = b.length[0], l2 = b.length[1];
        double separations[4] = {axial_start + l2, axial_start, axial_start + l2 - l1, axial_start - l1};
        double largest = 0.0;
        for (double q : separations) largest = rmax(largest, std::fabs(q));
        double axial_scale = std::numeric_limits<double>::infinity();
        for (double q : separations)
            if (std::fabs(q) > 1e-9 * largest) axial_scale = rmin(axial_scale, std::fabs(q));
        in = Integrator{&b, axial_start, axial_scale};
    };
    std::vector<unsigned char> log;
    FrozenIntegrator rec, rep;
    setup(nom, rec.in);
    setup(per, rep.in);
    rec.log = rep.log = &log;
    std::vector<int> tu = break_tags(nom.width[0], nom.width[1], nom.offset[1]);
    std::vector<int> tv = break_tags(nom.height[0], nom.height[1], nom.offset[2]);
    double sum = 0.0;
    for (size_t a = 0; a + 1 < tu.size(); ++a)
        for (size_t b = 0; b + 1 < tv.size(); ++b) {
            rec.panel(break_value(tu[a], nom.width[0], nom.width[1], nom.offset[1]),
                      break_value(tu[a + 1], nom.width[0], nom.width[1], nom.offset[1]),
                      break_value(tv[b], nom.height[0], nom.height[1], nom.offset[2]),
                      break_value(tv[b + 1], nom.height[0], nom.height[1], nom.offset[2]), 0, true);
            sum += rep.panel(break_value(tu[a], per.width[0], per.width[1], per.offset[1]),
                             break_value(tu[a + 1], per.width[0], per.width[1], per.offset[1]),
                             break_value(tv[b], per.height[0], per.height[1], per.offset[2]),
                             break_value(tv[b + 1], per.height[0], per.height[1], per.offset[2]), 0, false);
        }
    return sum;
}

// evaluate() with its decisions taken on (na, nb) and its arithmetic on
// (pa, pb).  Sampled-filament pairs are not covered (ORC_ERR_ARGUMENT).
int evaluate_frozen(const Fil &na0, const Fil &nb0, const Fil &pa0, const Fil &pb0, double *out) {
    const bool swap = canonical(na0, nb0) > 0;
    const Fil &na = swap ? nb0 : na0, &nb = swap ? na0 : nb0;
    const Fil &pa = swap ? pb0 : pa0, &pb = swap ? pa0 : pb0;
    double cosv = dot(na.l, nb.l);
    if (std::fabs(cosv) < kOrthogonalCos) {
        *out = 0.0;
        return ORC_OK;
    }
    Bar ba = make_bar(na), bb = make_bar(nb);
    bool parallel = norm(cross(na.l, nb.l)) < kParallelSin;
    AlignedBars ab;
    bool aligned = parallel && aligned_bars(ba, bb, &ab);
    double gap = separation(ba, bb);
    int oa[3], ob[3];
    bool have = point_orders(ba, gap, oa) && point_orders(bb, gap, ob);
    if (have && aligned) {
        size_t pairs = (size_t)(oa[0] * oa[1] * oa[2]) * (size_t)(ob[0] * ob[1] * ob[2]);
        if (pairs > kCheapPointPairs) have = false;
    }
    Bar qa = make_bar(pa), qb = make_bar(pb);
    double integral;
    if (have) {
        integral = point_sum(qa, oa, qb, ob) * dot(pa.l, pb.l);
    } else if (aligned) {
        AlignedBars pab;
        if (!aligned_bars(qa, qb, &pab)) return ORC_ERR_ARGUMENT;
        double qx[4], qy[4], qz[4], value, rel;
        corner_differences(ab.length[0], ab.length[1], ab.offset[0], qx);
        corner_differences(ab.width[0], ab.width[1], ab.offset[1], qy);
        corner_differences(ab.height[0], ab.height[1], ab.offset[2], qz);
        bar_integral(qx, qy, qz, &value, &rel);
        double v;
        if (rel <= kClosedFormMaxError) {
            corner_differences(pab.length[0], pab.length[1], pab.offset[0], qx);
            corner_differences(pab.width[0], pab.width[1], pab.offset[1], qy);
            corner_differences(pab.height[0], pab.height[1], pab.offset[2], qz);
            bar_integral(qx, qy, qz, &v, &rel);
        } else {
            v = frozen_quadrature(ab, pab);
        }
        double scale = signum(dot(pa.l, pb.l)) / (area_of(pa) * area_of(pb));
        integral = v * scale;
    } else {
        return ORC_ERR_ARGUMENT;
    }
    double value = kMu0Over4Pi * integral;
    if (!std::isfinite(value)) return ORC_ERR_NOT_FINITE;
    *out = value;
    return ORC_OK;
}

// ---------------------------------------------------------------------------
// Geometry, discretization, grading (geometry.rs:223-275, filament.rs:227-553,
// filament/grading.rs, solve.rs:388-510)
// ---------------------------------------------------------------------------
double scale_invariant_norm(V3 v) {
    if (!(std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z))) return NAN;
    double scale = rmax(rmax(std::fabs(v.x), std::fabs(v.y)), std::fabs(v.z));
    if (scale == 0.0) return 0.0;
    return norm(dvd(v, scale)) * scale;
}

struct Seg {
    V3 a, b;
    double width, height, sigma;
    bool has_wdir;
    V3 wdir;
};

bool segment_basis(const Seg &s, V3 *L, V3 *W, V3 *H) {
    auto fin = [](V3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
    if (!(fin(s.a) && fin(s.b))) return false;
    if (!(std::isfinite(s.width) && s.width > 0.0)) return false;
    if (!(std::isfinite(s.height) && s.height > 0.0)) return false;
    if (!(std::isfinite(s.sigma) && s.sigma > 0.0)) return false;
    V3 span = sub(s.b, s.a);
    double n = scale_invariant_norm(span);
    if (!(std::isfinite(n) && n > 0.0)) return false;
    V3 length = dvd(span, n);
    V3 hint;
    if (s.has_wdir) {
        double dn = scale_invariant_norm(s.wdir);
        if (!(std::isfinite(dn) && dn > 0.0)) return false;
        V3 dir = dvd(s.wdir, dn);
        V3 perp = sub(dir, mul(length, dot(dir, length)));
        if (norm(perp) <= 1.0e-9) return false;
        hint = perp;
    } else {
        V3 in_plane = cross(V3{0.0, 0.0, 1.0}, length);
        hint = norm(in_plane) < 1.0e-6 ? V3{1.0, 0.0, 0.0} : in_plane;
    }
    V3 w = sub(hint, mul(length, dot(hint, length)));
    w = dvd(w, norm(w));
    *L = length;
    *W = w;
    *H = cross(length, w);
    return true;
}

// __powidf2 (binary exponentiation), the lowering of Rust's f64::powi.
double powi(double a, int b) {
    bool recip = b < 0;
    double r = 1.0;
    while (true) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

bool graded_weights(long long count, double ratio, std::vector<double> &w) {
    if (!(std::isfinite(ratio) && ratio >= 1.0) || count == 0) return false;
    w.resize(count);
    for (long long i = 0; i < count; ++i) w[i] = powi(ratio, (int)std::min(i, count - 1 - i));
    for (double x : w)
        if (!std::isfinite(x)) return false;
    return true;
}

bool graded_cells(double total, long long count, double ratio, std::vector<std::pair<double, double>> &cells) {
    std::vector<double> w;
    if (!graded_weights(count, ratio, w)) return false;
    double sum = 0.0;
    for (double x : w) sum += x;
    double lower = 0.0;
    cells.clear();
    for (double weight : w) {
        double centre = total * ((lower + 0.5 * weight) / sum - 0.5);
        lower += weight;
        cells.push_back({centre, total * (weight / sum)});
    }
    return true;
}

bool grading_validate(const Seg &s, V3 W, V3 H, const std::vector<std::pair<double, double>> &widths,
                      const std::vector<std::pair<double, double>> &heights) {
    double shape_scale = rmax(rmax(norm(sub(s.b, s.a)), s.width), s.height);
    V3 aa = vabs(s.a), bb = vabs(s.b);
    V3 sup = {rmax(aa.x, bb.x), rmax(aa.y, bb.y), rmax(aa.z, bb.z)};
    V3 envelope = add(add(sup, mul(vabs(W), 0.5 * s.width)), mul(vabs(H), 0.5 * s.height));
    const std::vector<std::pair<double, double>> *cells[2] = {&widths, &heights};
    V3 dirs[2] = {W, H};
    for (int axis = 0; axis < 2; ++axis) {
        double coordinate_scale = dot(vabs(dirs[axis]), envelope);
        double minimum = rmax(1e-7 * shape_scale, 32.0 * kEps * coordinate_scale);
        const auto &c = *cells[axis];
        for (const auto &cell : c) {
            double centre = cell.first, size = cell.second;
            if (!(std::isfinite(size) && size > 0.0 && size >= minimum && std::isfinite(centre) &&
                  centre - 0.5 * size < centre && centre + 0.5 * size > centre))
                return false;
        }
        for (size_t i = 0; i + 1 < c.size(); ++i)
            if (!(c[i].first < c[i + 1].first)) return false;
    }
    return true;
}

bool discretize_uniform(const Seg &s, long long nw, long long nh, std::vector<Fil> &out) {
    if (nw == 0 || nh == 0) return false;
    V3 L, W, H;
    if (!segment_basis(s, &L, &W, &H)) return false;
    double length = norm(sub(s.b, s.a));
    double fw = s.width / (double)nw, fh = s.height / (double)nh;
    auto fraction = [](long long index, long long count) { return ((double)index + 0.5) / (double)count - 0.5; };
    for (long long j = 0; j < nh; ++j) {
        V3 along_height = mul(H, fraction(j, nh) * s.height);
        for (long long i = 0; i < nw; ++i) {
            V3 offset = add(mul(W, fraction(i, nw) * s.width), along_height);
            out.push_back(Fil{add(s.a, offset), add(s.b, offset), length, L, W, H, fw, fh, s.sigma});
        }
    }
    return true;
}

int discretize_graded(const Seg &s, long long nw, long long nh, double wr, double hr, std::vector<Fil> &out) {
    for (double r : {wr, hr})
        if (!(std::isfinite(r) && r >= 1.0)) return ORC_ERR_DISCRETIZE;
    if (nw == 0 || nh == 0) return ORC_ERR_DISCRETIZE;
    V3 L, W, H;
    if (!segment_basis(s, &L, &W, &H)) return ORC_ERR_DISCRETIZE;
    double length = norm(sub(s.b, s.a));
    std::vector<std::pair<double, double>> across_w, across_h;
    if (!graded_cells(s.width, nw, wr, across_w) || !graded_cells(s.height, nh, hr, across_h))
        return ORC_ERR_DISCRETIZE;
    if (!grading_validate(s, W, H, across_w, across_h)) return ORC_ERR_DISCRETIZE;
    if (wr == 1.0 && hr == 1.0) return discretize_uniform(s, nw, nh, out) ? ORC_OK : ORC_ERR_DISCRETIZE;
    for (const auto &hc : across_h) {
        V3 along_height = mul(H, hc.first);
        for (const auto &wc : across_w) {
            V3 offset = add(mul(W, wc.first), along_height);
            out.push_back(Fil{add(s.a, offset), add(s.b, offset), length, L, W, H, wc.second, hc.second, s.sigma});
        }
    }
    return ORC_OK;
}

double skin_depth(double f, double sigma) { return 1.0 / std::sqrt(kPi * f * kMu0 * sigma); }

long long skin_count(const orc_discretization &d, double extent, double sigma) {
    double target = d.target_skin_depths * skin_depth(d.frequency_hz, sigma);
    if (std::isinf(target) || extent <= target) return 1;
    for (long long count = 2; count <= d.max_per_axis; ++count) {
        std::vector<double> w;
        if (!graded_weights(count, d.ratio, w)) return count - 1;
        double sum = 0.0;
        for (double x : w) sum += x;
        if (extent / sum <= target) return count;
    }
    return d.max_per_axis;
}

struct Grid {
    long long nw, nh;
    double wr, hr;
};

int resolve_grids(const orc_discretization &d, const std::vector<Seg> &segs, std::vector<Grid> &grids) {
    size_t n = segs.size();
    grids.clear();
    switch (d.kind) {
        case 0:
            grids.assign(n, Grid{d.nw, d.nh, 1.0, 1.0});
            return ORC_OK;
        case 1:
        case 4:
            if ((size_t)d.per_segment_len != n) return ORC_ERR_MESH;
            for (size_t i = 0; i < n; ++i) {
                const orc_axis_grading &g = d.per_segment[i];
                if (d.kind == 4)
                    for (double r : {g.width_ratio, g.height_ratio})
                        if (!(std::isfinite(r) && r >= 1.0)) return ORC_ERR_GRADING;
                grids.push_back(Grid{g.nw, g.nh, d.kind == 4 ? g.width_ratio : 1.0, d.kind == 4 ? g.height_ratio : 1.0});
            }
            return ORC_OK;
        case 2:
            if (!(std::isfinite(d.ratio) && d.ratio >= 1.0)) return ORC_ERR_GRADING;
            grids.assign(n, Grid{d.nw, d.nh, d.ratio, d.ratio});
            return ORC_OK;
        case 3:
            if (!(std::isfinite(d.ratio) && d.ratio >= 1.0)) return ORC_ERR_GRADING;
            if (!(std::isfinite(d.target_skin_depths) && d.target_skin_depths > 0.0)) return ORC_ERR_GRADING;
            if (!(std::isfinite(d.frequency_hz) && d.frequency_hz >= 0.0)) return ORC_ERR_GRADING;
            if (d.max_per_axis == 0) return ORC_ERR_GRADING;
            for (const Seg &s : segs)
                grids.push_back(Grid{skin_count(d, s.width, s.sigma), skin_count(d, s.height, s.sigma), d.ratio, d.ratio});
            return ORC_OK;
    }
    return ORC_ERR_ARGUMENT;
}

int discretize_all(const double *nodes, long long nnode, const orc_segment *segs, long long nseg,
                   const orc_discretization &d, std::vector<Fil> &fils, std::vector<long long> &per_segment) {
    std::vector<Seg> ss;
    for (long long i = 0; i < nseg; ++i) {
        const orc_segment &o = segs[i];
        if (o.a < 0 || o.b < 0 || o.a >= nnode || o.b >= nnode) return ORC_ERR_ARGUMENT;
        Seg s;
        s.a = {nodes[3 * o.a], nodes[3 * o.a + 1], nodes[3 * o.a + 2]};
        s.b = {nodes[3 * o.b], nodes[3 * o.b + 1], nodes[3 * o.b + 2]};
        s.width = o.width;
        s.height = o.height;
        s.sigma = o.sigma;
        s.has_wdir = o.has_width_dir != 0;
        s.wdir = {o.width_dir[0], o.width_dir[1], o.width_dir[2]};
        V3 L, W, H;
        if (!segment_basis(s, &L, &W, &H)) return ORC_ERR_ARGUMENT;
        ss.push_back(s);
    }
    std::vector<Grid> grids;
    int st = resolve_grids(d, ss, grids);
    if (st) return st;
    fils.clear();
    per_segment.clear();
    for (size_t i = 0; i < ss.size(); ++i) {
        size_t before = fils.size();
        if (d.kind == 0 || d.kind == 1) {
            if (!discretize_uniform(ss[i], grids[i].nw, grids[i].nh, fils)) return ORC_ERR_DISCRETIZE;
        } else {
            st = discretize_graded(ss[i], grids[i].nw, grids[i].nh, grids[i].wr, grids[i].hr, fils);
            if (st) return st;
        }
        per_segment.push_back((long long)(fils.size() - before));
    }
    return ORC_OK;
}

// ---------------------------------------------------------------------------
// Loop basis, mesh.rs:170-361
// ---------------------------------------------------------------------------
struct Mesh {
    std::vector<std::vector<std::pair<long long, double>>> rows;
    long long branch_count = 0, internal_count = 0;
};

int build_mesh(const orc_segment *segs, long long nseg, long long nnode, const long long *per_segment,
               const long long *ports, long long nport, Mesh &mesh) {
    for (long long s = 0; s < nseg; ++s)
        if (per_segment[s] == 0) return ORC_ERR_MESH;
    if (nport == 0) return ORC_ERR_MESH;
    std::vector<long long> first(nseg);
    long long next = 0;
    for (long long s = 0; s < nseg; ++s) {
        first[s] = next;
        next += per_segment[s];
    }
    mesh.branch_count = next;
    mesh.rows.clear();
    for (long long s = 0; s < nseg; ++s)
        for (long long k = 1; k < per_segment[s]; ++k) mesh.rows.push_back({{first[s] + k, 1.0}, {first[s], -1.0}});
    // Forest::grow, mesh.rs:301-338
    struct Adj {
        long long next, seg;
        bool fwd;
    };
    std::vector<std::vector<Adj>> adj(nnode);
    for (long long s = 0; s < nseg; ++s) {
        adj[segs[s].a].push_back({segs[s].b, s, true});
        adj[segs[s].b].push_back({segs[s].a, s, false});
    }
    struct Parent {
        bool has;
        long long node, seg;
        bool fwd;
    };
    std::vector<Parent> parent(nnode, Parent{false, 0, 0, false});
    std::vector<long long> depth(nnode, 0), component(nnode, -1);
    std::vector<bool> in_tree(nseg, false);
    long long components = 0;
    for (long long root = 0; root < nnode; ++root) {
        if (component[root] >= 0 || adj[root].empty()) continue;
        component[root] = components;
        std::deque<long long> queue{root};
        while (!queue.empty()) {
            long long node = queue.front();
            queue.pop_front();
            for (const Adj &e : adj[node]) {
                if (component[e.next] < 0) {
                    component[e.next] = components;
                    parent[e.next] = Parent{true, node, e.seg, e.fwd};
                    depth[e.next] = depth[node] + 1;
                    in_tree[e.seg] = true;
                    queue.push_back(e.next);
                }
            }
        }
        ++components;
    }
    auto path = [&](long long from, long long to) {
        std::vector<std::pair<long long, double>> up, down;
        long long x = from, y = to;
        while (x != y) {
            if (depth[x] >= depth[y]) {
                const Parent &p = parent[x];
                up.push_back({p.seg, p.fwd ? -1.0 : 1.0});
                x = p.node;
            } else {
                const Parent &p = parent[y];
                down.push_back({p.seg, p.fwd ? 1.0 : -1.0});
                y = p.node;
            }
        }
        for (auto it = down.rbegin(); it != down.rend(); ++it) up.push_back(*it);
        return up;
    };
    long long links = 0;
    for (long long s = 0; s < nseg; ++s) {
        if (!in_tree[s]) {
            std::vector<std::pair<long long, double>> row{{s, 1.0}};
            auto p = path(segs[s].b, segs[s].a);
            row.insert(row.end(), p.begin(), p.end());
            mesh.rows.push_back(row);
            ++links;
        }
    }
    mesh.internal_count = (long long)mesh.rows.size();
    for (long long q = 0; q < nport; ++q) {
        long long pos = ports[2 * q], neg = ports[2 * q + 1];
        if (pos < 0 || neg < 0 || pos >= nnode || neg >= nnode) return ORC_ERR_MESH;
        if (pos == neg) return ORC_ERR_MESH;
        if (component[pos] < 0 || component[neg] < 0 || component[pos] != component[neg]) return ORC_ERR_MESH;
        mesh.rows.push_back(path(pos, neg));
    }
    for (size_t r = (size_t)(mesh.internal_count - links); r < mesh.rows.size(); ++r)
        for (auto &e : mesh.rows[r]) e.first = first[e.first];
    return ORC_OK;
}

// ---------------------------------------------------------------------------
// Fill (batch.rs:246-372) and congruence (solve.rs:1172-1200)
// ---------------------------------------------------------------------------
int fill_matrix(const std::vector<Fil> &f, double *L, signed char *methods, int threads, long long *ei,
                long long *ej) {
    long long n = (long long)f.size();
    int status = ORC_OK;
    long long bad_i = -1, bad_j = -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (long long i = 0; i < n; ++i) {
        for (long long j = i; j < n; ++j) {
            double v;
            int method;
            bool resolved;
            int st = evaluate(f[i], f[j], &v, &method, &resolved);
            if (st) {
#pragma omp critical
                {
                    if (status == ORC_OK || i < bad_i || (i == bad_i && j < bad_j)) {
                        status = st;
                        bad_i = i;
                        bad_j = j;
                    }
                }
                v = NAN;
                method = -1;
            }
            L[i + j * n] = v;
            L[j + i * n] = v;
            if (methods) {
                methods[i + j * n] = (signed char)method;
                methods[j + i * n] = (signed char)method;
            }
        }
    }
    if (ei) *ei = bad_i;
    if (ej) *ej = bad_j;
    return status;
}

// M * B * M^T, upper triangle mirrored; B given by an accumulate callback.
template <class Acc>
std::vector<double> congruence(const Mesh &mesh, long long branches, Acc accumulate, int threads) {
    long long loops = (long long)mesh.rows.size();
    std::vector<double> upper((size_t)(loops * loops), 0.0);
#pragma omp parallel num_threads(threads)
    {
        std::vector<double> product((size_t)branches);
#pragma omp for schedule(dynamic, 4)
        for (long long i = 0; i < loops; ++i) {
            std::fill(product.begin(), product.end(), 0.0);
            for (const auto &e : mesh.rows[i]) accumulate(e.first, e.second, product.data());
            for (long long j = i; j < loops; ++j) {
                double s = 0.0;
                for (const auto &e : mesh.rows[j]) s += e.second * product[e.first];
                upper[i * loops + j] = s;
            }
        }
    }
    std::vector<double> full((size_t)(loops * loops));
    for (long long i = 0; i < loops; ++i)
        for (long long j = 0; j < loops; ++j) {
            long long lo = std::min(i, j), hi = std::max(i, j);
            full[i + j * loops] = upper[lo * loops + hi];  // column-major
        }
    return full;
}

// ---------------------------------------------------------------------------
// Blocked LU with partial pivoting, dense.rs:43-190 (complex, PANEL = 32)
// ---------------------------------------------------------------------------
struct C {
    double re, im;
};
inline C cmul(C a, C b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C csub(C a, C b) { return {a.re - b.re, a.im - b.im}; }
inline C cdiv(C a, C b) {
    double ns = b.re * b.re + b.im * b.im;
    double re = a.re * b.re + a.im * b.im;
    double im = a.im * b.re - a.re * b.im;
    return {re / ns, im / ns};
}
inline double norm1(C a) { return std::fabs(a.re) + std::fabs(a.im); }
inline void subtract_scaled(C *y, C factor, const C *x, long long len) {
    for (long long k = 0; k < len; ++k) y[k] = csub(y[k], cmul(factor, x[k]));
}

constexpr long long kPanel = 32;

// The loops below visit the entries of a column in another order than
// dense.rs's column-at-a-time `subtract_scaled` sweeps, but every entry still
// receives exactly the reference's operations in the reference's order:
//   y -= h_c * l_c  for c = 0, 1, ... (each product rounded as in cmul, then
//   the subtraction), with h_c = the column's entry in row start + c,
// which is final before any row below it uses it.  So the factors are the
// reference's bit for bit (checked against the plain column sweeps in
// tests/test_oracle_known_answers.py), only the memory traffic changes: the
// trailing update goes row block by row block, four columns at a time, so a
// block of the panel is loaded once for many columns instead of once per
// column and panel column.

// Rows [r0, r1) of `ncols` columns (y_j = col[j]): y_j[r] -= sum over c in
// [0, width) of h[j][c] * l_c[r], in increasing c, where l_c = panel + c*order.
static void rows_update_scalar(C *const *col, int ncols, const C *const *h, const C *panel, long long order,
                               long long width, long long r0, long long r1) {
    for (int j = 0; j < ncols; ++j)
        for (long long r = r0; r < r1; ++r) {
            C y = col[j][r];
            for (long long c = 0; c < width; ++c) y = csub(y, cmul(h[j][c], panel[c * order + r]));
            col[j][r] = y;
        }
}

#if defined(__x86_64__)
#include <immintrin.h>
// The same per-entry sequence with AVX2 lanes: (hr * [lr, li]) addsub
// (hi * [li, lr]) = [hr lr - hi li, hr li + hi lr] is cmul's rounding of both
// parts, then one subtraction; no fused multiply-add is used.
__attribute__((target("avx2"))) static void rows_update_avx2(C *const *col, int ncols, const C *const *h,
                                                             const C *panel, long long order, long long width,
                                                             long long r0, long long r1) {
    long long r = r0;
    if (ncols == 4) {
        for (; r + 4 <= r1; r += 4) {
            __m256d y[4][2];
            for (int j = 0; j < 4; ++j) {
                y[j][0] = _mm256_loadu_pd(&col[j][r].re);
                y[j][1] = _mm256_loadu_pd(&col[j][r + 2].re);
            }
            for (long long c = 0; c < width; ++c) {
                const C *l = panel + c * order + r;
                __m256d l0 = _mm256_loadu_pd(&l[0].re), l1 = _mm256_loadu_pd(&l[2].re);
                __m256d s0 = _mm256_permute_pd(l0, 0x5), s1 = _mm256_permute_pd(l1, 0x5);
                for (int j = 0; j < 4; ++j) {
                    __m256d hr = _mm256_broadcast_sd(&h[j][c].re), hi = _mm256_broadcast_sd(&h[j][c].im);
                    y[j][0] = _mm256_sub_pd(y[j][0], _mm256_addsub_pd(_mm256_mul_pd(hr, l0), _mm256_mul_pd(hi, s0)));
                    y[j][1] = _mm256_sub_pd(y[j][1], _mm256_addsub_pd(_mm256_mul_pd(hr, l1), _mm256_mul_pd(hi, s1)));
                }
            }
            for (int j = 0; j < 4; ++j) {
                _mm256_storeu_pd(&col[j][r].re, y[j][0]);
                _mm256_storeu_pd(&col[j][r + 2].re, y[j][1]);
            }
        }
    } else {
        for (int j = 0; j < ncols; ++j) {
            long long rr = r;
            for (; rr + 2 <= r1; rr += 2) {
                __m256d y = _mm256_loadu_pd(&col[j][rr].re);
                for (long long c = 0; c < width; ++c) {
                    __m256d l = _mm256_loadu_pd(&panel[c * order + rr].re);
                    __m256d s = _mm256_permute_pd(l, 0x5);
                    __m256d hr = _mm256_broadcast_sd(&h[j][c].re), hi = _mm256_broadcast_sd(&h[j][c].im);
                    y = _mm256_sub_pd(y, _mm256_addsub_pd(_mm256_mul_pd(hr, l), _mm256_mul_pd(hi, s)));
                }
                _mm256_storeu_pd(&col[j][rr].re, y);
            }
            rows_update_scalar(&col[j], 1, &h[j], panel, order, width, rr, r1);
        }
        return;
    }
    rows_update_scalar(col, ncols, h, panel, order, width, r, r1);
}
static const bool kHaveAvx2 = __builtin_cpu_supports("avx2");
#else
static const bool kHaveAvx2 = false;
#endif

static inline void rows_update(C *const *col, int ncols, const C *const *h, const C *panel, long long order,
                               long long width, long long r0, long long r1) {
#if defined(__x86_64__)
    if (kHaveAvx2) return rows_update_avx2(col, ncols, h, panel, order, width, r0, r1);
#endif
    rows_update_scalar(col, ncols, h, panel, order, width, r0, r1);
}

// Trailing columns [c0, c1) after the panel [start, start + width): the
// interchanges, the panel's unit-lower forward substitution on rows
// [start, start + width), then the rows below (dense.rs:117-136).
static void update_trailing(C *a, long long order, long long start, long long width, const long long *piv,
                            long long c0, long long c1) {
    const C *panel = a + start * order;
    const long long below = start + width;
    std::vector<C> heads((size_t)((c1 - c0) * width));
    for (long long col = c0; col < c1; ++col) {
        C *y = a + col * order;
        for (long long off = 0; off < width; ++off) std::swap(y[start + off], y[piv[off]]);
        for (long long k = 1; k < width; ++k) {
            C v = y[start + k];
            for (long long c = 0; c < k; ++c) v = csub(v, cmul(y[start + c], panel[c * order + start + k]));
            y[start + k] = v;
        }
        for (long long c = 0; c < width; ++c) heads[(col - c0) * width + c] = y[start + c];
    }
    constexpr long long kRowBlock = 256;
    for (long long r0 = below; r0 < order; r0 += kRowBlock) {
        long long r1 = std::min(order, r0 + kRowBlock);
        for (long long g = c0; g < c1; g += 4) {
            int nc = (int)std::min<long long>(4, c1 - g);
            C *cols[4];
            const C *hs[4];
            for (int j = 0; j < nc; ++j) {
                cols[j] = a + (g + j) * order;
                hs[j] = heads.data() + (g + j - c0) * width;
            }
            rows_update(cols, nc, hs, panel, order, width, r0, r1);
        }
    }
}

// factorize_panel, dense.rs:144-189, column by column (left-looking): column
// o first takes the interchanges and the eliminations of panel columns
// 0..o-1 in order, which hands every entry the same operations in the same
// order as the reference's right-looking sweep (a later interchange only
// swaps rows below every earlier pivot row, in all columns alike).
static bool factorize_panel(C *panel, long long order, long long start, long long width, long long *piv) {
    const C *heads[1];
    for (long long o = 0; o < width; ++o) {
        C *y = panel + o * order;
        for (long long c = 0; c < o; ++c) std::swap(y[start + c], y[piv[c]]);
        // Rows start+1 .. start+o-1: the triangular part, then everything below
        // takes the o eliminations at once.
        for (long long k = 1; k < o; ++k) {
            C v = y[start + k];
            for (long long c = 0; c < k; ++c) v = csub(v, cmul(y[start + c], panel[c * order + start + k]));
            y[start + k] = v;
        }
        if (o > 0) {
            std::vector<C> h(y + start, y + start + o);
            heads[0] = h.data();
            C *cols[1] = {y};
            rows_update(cols, 1, heads, panel, order, o, start + o, order);
        }
        const long long diagonal = start + o;
        long long pivot = diagonal;
        double largest = norm1(y[diagonal]);
        for (long long row = diagonal + 1; row < order; ++row) {
            double m = norm1(y[row]);
            if (m > largest) {
                pivot = row;
                largest = m;
            }
        }
        if (largest == 0.0) return false;
        piv[o] = pivot;
        if (pivot != diagonal)
            for (long long k = 0; k <= o; ++k) std::swap(panel[k * order + diagonal], panel[k * order + pivot]);
        C inverse = cdiv(C{1.0, 0.0}, y[diagonal]);
        for (long long r = diagonal + 1; r < order; ++r) y[r] = cmul(y[r], inverse);
    }
    return true;
}

bool factorize(C *a, long long order, std::vector<long long> &pivots, int threads) {
    pivots.assign(order, 0);
    for (long long start = 0; start < order; start += kPanel) {
        long long width = std::min(kPanel, order - start);
        C *panel = a + start * order;
        if (!factorize_panel(panel, order, start, width, pivots.data() + start)) return false;
        const long long *piv = pivots.data() + start;
        for (long long col = 0; col < start; ++col)
            for (long long off = 0; off < width; ++off) std::swap(a[col * order + start + off], a[col * order + piv[off]]);
        const long long right_begin = start + width;
        const long long chunk = 32;
        const long long tasks = (order - right_begin + chunk - 1) / chunk;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) if (tasks > 1)
        for (long long t = 0; t < tasks; ++t) {
            long long c0 = right_begin + t * chunk;
            update_trailing(a, order, start, width, piv, c0, std::min(order, c0 + chunk));
        }
    }
    return true;
}

// The reference's column-at-a-time form (dense.rs:98-190), kept to check
// that the blocked loops above give the same bits.
bool factorize_plain(C *a, long long order, std::vector<long long> &pivots) {
    pivots.assign(order, 0);
    for (long long start = 0; start < order; start += kPanel) {
        long long width = std::min(kPanel, order - start);
        C *panel = a + start * order;
        for (long long c = 0; c < width; ++c) {
            long long diagonal = start + c;
            C *column = panel + c * order;
            long long pivot = diagonal;
            double largest = norm1(column[diagonal]);
            for (long long row = diagonal + 1; row < order; ++row) {
                double m = norm1(column[row]);
                if (m > largest) {
                    pivot = row;
                    largest = m;
                }
            }
            if (largest == 0.0) return false;
            pivots[start + c] = pivot;
            if (pivot != diagonal)
                for (long long k = 0; k < width; ++k) std::swap(panel[k * order + diagonal], panel[k * order + pivot]);
            C inverse = cdiv(C{1.0, 0.0}, column[diagonal]);
            for (long long r = diagonal + 1; r < order; ++r) column[r] = cmul(column[r], inverse);
            for (long long o = c + 1; o < width; ++o) {
                C *other = panel + o * order;
                subtract_scaled(other + diagonal + 1, other[diagonal], column + diagonal + 1, order - diagonal - 1);
            }
        }
        const long long *piv = pivots.data() + start;
        auto interchange = [&](C *column) {
            for (long long off = 0; off < width; ++off) std::swap(column[start + off], column[piv[off]]);
        };
        for (long long col = 0; col < start; ++col) interchange(a + col * order);
        for (long long col = start + width; col < order; ++col) {
            C *column = a + col * order;
            interchange(column);
            for (long long c = 0; c < width; ++c) {
                const C *l = panel + c * order + start + c + 1;
                subtract_scaled(column + start + c + 1, column[start + c], l, order - (start + c + 1));
            }
        }
    }
    return true;
}

int lu_solve(C *a, long long order, C *x, long long nrhs, int threads, bool plain = false) {
    if (order == 0) return ORC_OK;
    std::vector<long long> pivots;
    if (!(plain ? factorize_plain(a, order, pivots) : factorize(a, order, pivots, threads))) return ORC_ERR_SINGULAR;
#pragma omp parallel for schedule(static) num_threads(threads) if (nrhs > 1)
    for (long long r = 0; r < nrhs; ++r) {
        C *rhs = x + r * order;
        for (long long row = 0; row < order; ++row) std::swap(rhs[row], rhs[pivots[row]]);
        for (long long c = 0; c < order; ++c)
            subtract_scaled(rhs + c + 1, rhs[c], a + c * order + c + 1, order - c - 1);
        for (long long c = order - 1; c >= 0; --c) {
            rhs[c] = cdiv(rhs[c], a[c * order + c]);
            subtract_scaled(rhs, rhs[c], a + c * order, c);
        }
    }
    return ORC_OK;
}

// Real-valued variant for the DC path (solve.rs:812-815).
struct Rw {
    double re;
};

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
struct orc_system {
    std::vector<Fil> fils;
    std::vector<double> resist;
    std::vector<double> L;  // n x n column-major
    Mesh mesh;
    std::vector<double> r_mesh, l_mesh;  // loops x loops column-major
    long long nnode = 0, nseg = 0;
};

extern "C" {

void orc_gauss_rule(int n, double *nodes, double *weights) {
    const Rule &r = rule(n);
    for (size_t k = 0; k < r.nodes.size(); ++k) {
        nodes[k] = r.nodes[k];
        weights[k] = r.weights[k];
    }
}

int orc_order_for(double tolerance, int max_order, double half_extent, double distance) {
    OrderTable t(tolerance, max_order);
    return t.order_for(half_extent, distance);
}

int orc_discretize(const double *nodes, long long nnode, const orc_segment *segs, long long nseg,
                   const orc_discretization *disc, double *filaments, long long cap, long long *nfil,
                   long long *per_segment) {
    std::vector<Fil> fils;
    std::vector<long long> per;
    int st = discretize_all(nodes, nnode, segs, nseg, *disc, fils, per);
    if (st) return st;
    *nfil = (long long)fils.size();
    if ((long long)fils.size() > cap) return ORC_ERR_ARGUMENT;
    for (size_t i = 0; i < fils.size(); ++i) store_fil(fils[i], filaments + 19 * i);
    for (size_t i = 0; i < per.size(); ++i) per_segment[i] = per[i];
    return ORC_OK;
}

int orc_mesh(const orc_segment *segs, long long nseg, long long nnode, const long long *per_segment,
             const long long *ports, long long nport, long long *row_ptr, long long *cols, double *signs,
             long long cap_rows, long long cap_nnz, long long *nrows, long long *nnz, long long *internal) {
    Mesh m;
    int st = build_mesh(segs, nseg, nnode, per_segment, ports, nport, m);
    if (st) return st;
    long long total = 0;
    for (auto &r : m.rows) total += (long long)r.size();
    *nrows = (long long)m.rows.size();
    *nnz = total;
    *internal = m.internal_count;
    if (*nrows + 1 > cap_rows || total > cap_nnz) return ORC_ERR_ARGUMENT;
    long long k = 0;
    for (size_t r = 0; r < m.rows.size(); ++r) {
        row_ptr[r] = k;
        for (auto &e : m.rows[r]) {
            cols[k] = e.first;
            signs[k] = e.second;
            ++k;
        }
    }
    row_ptr[m.rows.size()] = k;
    return ORC_OK;
}

int orc_mutual(const double *fa, const double *fb, double *value, int *method, int *resolved) {
    bool res;
    int st = evaluate(load_fil(fa), load_fil(fb), value, method, &res);
    *resolved = res ? 1 : 0;
    return st;
}

double orc_self_inductance(const double *fp) {
    Fil f = load_fil(fp);
    AlignedBars b{{f.length, f.length}, {f.width, f.width}, {f.height, f.height}, {0.0, 0.0, 0.0}};
    int method;
    double integral = aligned_integral(b, &method);
    return kMu0Over4Pi * (integral * (1.0 / (area_of(f) * area_of(f))));
}

void orc_bar_integral(const double *qx, const double *qy, const double *qz, double *value, double *rel) {
    bar_integral(qx, qy, qz, value, rel);
}

double orc_aligned_quadrature(const double *length2, const double *width2, const double *height2,
                              const double *offset3) {
    AlignedBars b{{length2[0], length2[1]}, {width2[0], width2[1]}, {height2[0], height2[1]},
                  {offset3[0], offset3[1], offset3[2]}};
    return aligned_integral_quadrature(b);
}

double orc_lines_parallel(double l1, double l2, double offset, double rho, int *ok) {
    double v = 0.0;
    *ok = lines_parallel(l1, l2, offset, rho, &v) ? 1 : 0;
    return v;
}

double orc_lines_skew(const double *a0, const double *a1, const double *b0, const double *b1, double sin_min,
                      int *ok) {
    double v = 0.0;
    *ok = lines_skew(V3{a0[0], a0[1], a0[2]}, V3{a1[0], a1[1], a1[2]}, V3{b0[0], b0[1], b0[2]},
                     V3{b1[0], b1[1], b1[2]}, sin_min, &v)
              ? 1
              : 0;
    return v;
}

double orc_separation(const double *fa, const double *fb) {
    return separation(make_bar(load_fil(fa)), make_bar(load_fil(fb)));
}

int orc_fill(const double *filaments, long long n, double *L, signed char *methods, int threads, long long *ei,
             long long *ej) {
    std::vector<Fil> f((size_t)n);
    for (long long i = 0; i < n; ++i) f[i] = load_fil(filaments + 19 * i);
    return fill_matrix(f, L, methods, threads, ei, ej);
}

// near_pairs, pfft/near.rs:41-106: for each filament i the filaments j >= i
// (i itself included) whose separating-axis gap is below `radius`, found
// through uniform bins over the filaments' bounding boxes, ascending in j.
// Output in CSR form: off[n + 1], cols (capacity `cap`; the total count is
// returned through *total even when it exceeds cap).
int orc_near_pairs(const double *filaments, long long n, double radius, long long *off, long long *cols,
                   long long cap, long long *total) {
    *total = 0;
    off[0] = 0;
    if (n == 0) return ORC_OK;
    std::vector<Bar> bars((size_t)n);
    std::vector<V3> blo((size_t)n), bhi((size_t)n);
    for (long long i = 0; i < n; ++i) {
        bars[i] = make_bar(load_fil(filaments + 19 * i));
        V3 reach{0.0, 0.0, 0.0};
        for (int k = 0; k < 3; ++k) {
            V3 a = bars[i].axes[k];
            reach = add(reach, V3{std::fabs(a.x) * bars[i].half[k], std::fabs(a.y) * bars[i].half[k],
                                  std::fabs(a.z) * bars[i].half[k]});
        }
        blo[i] = sub(bars[i].centre, reach);
        bhi[i] = add(bars[i].centre, reach);
    }
    double lo[3] = {blo[0].x, blo[0].y, blo[0].z}, hi[3] = {bhi[0].x, bhi[0].y, bhi[0].z};
    for (long long i = 0; i < n; ++i) {
        const double a[3] = {blo[i].x, blo[i].y, blo[i].z}, b[3] = {bhi[i].x, bhi[i].y, bhi[i].z};
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], a[k]);
            hi[k] = std::max(hi[k], b[k]);
        }
    }
    const double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    double size = std::max(std::max(radius, std::max(ext[0], std::max(ext[1], ext[2])) * 1e-9),
                           std::numeric_limits<double>::min());
    long long dims[3];
    auto set_dims = [&]() {
        for (int k = 0; k < 3; ++k) dims[k] = (long long)std::floor(ext[k] / size) + 1;
    };
    set_dims();
    while (dims[0] * dims[1] * dims[2] > 8 * n + 64) {
        size *= 1.5;
        set_dims();
    }
    auto cell = [&](double x, int k) {
        double c = std::floor((x - lo[k]) / size);
        long long v = c > 0.0 ? (long long)c : 0;
        return std::min(v, dims[k] - 1);
    };
    std::vector<std::vector<long long>> bins((size_t)(dims[0] * dims[1] * dims[2]));
    for (long long i = 0; i < n; ++i) {
        const double a[3] = {blo[i].x, blo[i].y, blo[i].z}, b[3] = {bhi[i].x, bhi[i].y, bhi[i].z};
        for (long long x = cell(a[0], 0); x <= cell(b[0], 0); ++x)
            for (long long y = cell(a[1], 1); y <= cell(b[1], 1); ++y)
                for (long long z = cell(a[2], 2); z <= cell(b[2], 2); ++z)
                    bins[(size_t)((x * dims[1] + y) * dims[2] + z)].push_back(i);
    }
    long long count = 0;
    for (long long i = 0; i < n; ++i) {
        const double a[3] = {blo[i].x - radius, blo[i].y - radius, blo[i].z - radius};
        const double b[3] = {bhi[i].x + radius, bhi[i].y + radius, bhi[i].z + radius};
        std::vector<long long> found;
        for (long long x = cell(a[0], 0); x <= cell(b[0], 0); ++x)
            for (long long y = cell(a[1], 1); y <= cell(b[1], 1); ++y)
                for (long long z = cell(a[2], 2); z <= cell(b[2], 2); ++z)
                    for (long long j : bins[(size_t)((x * dims[1] + y) * dims[2] + z)])
                        if (j >= i) found.push_back(j);
        std::sort(found.begin(), found.end());
        found.erase(std::unique(found.begin(), found.end()), found.end());
        for (long long j : found)
            if (j == i || separation(bars[i], bars[j]) < radius) {
                if (count < cap) cols[count] = j;
                ++count;
            }
        off[i + 1] = count;
    }
    *total = count;
    return ORC_OK;
}

int orc_fill_frozen(const double *nominal, const double *perturbed, long long n, double *L, int threads) {
    std::vector<Fil> fn((size_t)n), fp((size_t)n);
    for (long long i = 0; i < n; ++i) {
        fn[i] = load_fil(nominal + 19 * i);
        fp[i] = load_fil(perturbed + 19 * i);
    }
    int status = ORC_OK;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (long long i = 0; i < n; ++i) {
        for (long long j = i; j < n; ++j) {
            double v = NAN;
            int st = evaluate_frozen(fn[i], fn[j], fp[i], fp[j], &v);
            if (st) {
#pragma omp critical
                status = st;
            }
            L[i + j * n] = v;
            L[j + i * n] = v;
        }
    }
    return status;
}

int orc_fill_frozen_rows(const double *nominal, const double *perturbed, long long n, const long long *rows,
                         long long nrows, double *out, int threads) {
    std::vector<Fil> fn((size_t)n), fp((size_t)n);
    for (long long i = 0; i < n; ++i) {
        fn[i] = load_fil(nominal + 19 * i);
        fp[i] = load_fil(perturbed + 19 * i);
    }
    int status = ORC_OK;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (long long t = 0; t < nrows * n; ++t) {
        const long long r = rows[t / n], j = t % n;
        double v = NAN;
        int st = evaluate_frozen(fn[r], fn[j], fp[r], fp[j], &v);
        if (st) {
#pragma omp critical
            status = st;
        }
        out[t] = v;
    }
    return status;
}

int orc_lu_solve(double *a, long long n, double *b, long long nrhs, int threads) {
    return lu_solve(reinterpret_cast<C *>(a), n, reinterpret_cast<C *>(b), nrhs, threads);
}

int orc_lu_solve_plain(double *a, long long n, double *b, long long nrhs) {
    return lu_solve(reinterpret_cast<C *>(a), n, reinterpret_cast<C *>(b), nrhs, 1, true);
}

int orc_system_assemble(const double *nodes, long long nnode, const orc_segment *segs, long long nseg,
                        const long long *ports, long long nport, const orc_discretization *disc, int threads,
                        orc_system **out, double *timing3) {
    auto t0 = omp_get_wtime();
    orc_system *s = new orc_system;
    std::vector<long long> per;
    int st = discretize_all(nodes, nnode, segs, nseg, *disc, s->fils, per);
    if (!st) st = build_mesh(segs, nseg, nnode, per.data(), ports, nport, s->mesh);
    if (st) {
        delete s;
        return st;
    }
    s->nnode = nnode;
    s->nseg = nseg;
    for (const Fil &f : s->fils) s->resist.push_back(f.length / (f.sigma * area_of(f)));  // solve.rs:941
    long long n = (long long)s->fils.size();
    s->L.assign((size_t)(n * n), 0.0);
    auto t1 = omp_get_wtime();
    st = fill_matrix(s->fils, s->L.data(), nullptr, threads, nullptr, nullptr);
    auto t2 = omp_get_wtime();
    if (st) {
        delete s;
        return st;
    }
    const std::vector<double> &R = s->resist;
    s->r_mesh = congruence(
        s->mesh, n, [&](long long b, double sign, double *row) { row[b] += sign * R[b]; }, threads);
    const double *Lp = s->L.data();
    s->l_mesh = congruence(
        s->mesh, n,
        [&](long long b, double sign, double *row) {
            const double *col = Lp + b * n;
            for (long long k = 0; k < n; ++k) row[k] += sign * col[k];
        },
        threads);
    auto t3 = omp_get_wtime();
    if (timing3) {
        timing3[0] = t2 - t1;
        timing3[1] = t3 - t0;
        timing3[2] = (double)n * (double)(n + 1) / 2.0;
    }
    *out = s;
    return ORC_OK;
}

void orc_system_counts(const orc_system *s, long long *c) {
    c[0] = s->nnode;
    c[1] = s->nseg;
    c[2] = (long long)s->fils.size();
    c[3] = (long long)s->mesh.rows.size();
    c[4] = s->mesh.internal_count;
    c[5] = (long long)s->mesh.rows.size() - s->mesh.internal_count;
}

void orc_system_blocks(const orc_system *s, double *r_mesh, double *l_mesh) {
    std::memcpy(r_mesh, s->r_mesh.data(), s->r_mesh.size() * 8);
    std::memcpy(l_mesh, s->l_mesh.data(), s->l_mesh.size() * 8);
}

void orc_system_filaments(const orc_system *s, double *f) {
    for (size_t i = 0; i < s->fils.size(); ++i) store_fil(s->fils[i], f + 19 * i);
}

void orc_system_inductance(const orc_system *s, double *L) { std::memcpy(L, s->L.data(), s->L.size() * 8); }

// MeshSystem::impedance, solve.rs:806-830, with schur_complement :1154-1164.
int orc_system_impedance(const orc_system *s, double frequency, double *z, int threads) {
    if (!(std::isfinite(frequency) && frequency >= 0.0)) return ORC_ERR_FREQUENCY;
    long long loops = (long long)s->mesh.rows.size();
    long long m = s->mesh.internal_count, p = loops - m;
    double omega = kTau * frequency;
    bool dc = frequency == 0.0;
    auto entry = [&](long long i, long long j) {
        double r = s->r_mesh[i + j * loops];
        if (dc) return C{r, 0.0};
        double l = s->l_mesh[i + j * loops];
        return C{r, omega * l};
    };
    std::vector<C> ee((size_t)(m * m)), ep((size_t)(m * p)), solved;
    for (long long j = 0; j < m; ++j)
        for (long long i = 0; i < m; ++i) ee[i + j * m] = entry(i, j);
    for (long long j = 0; j < p; ++j)
        for (long long i = 0; i < m; ++i) ep[i + j * m] = entry(i, m + j);
    solved = ep;
    if (m > 0) {
        int st = lu_solve(ee.data(), m, solved.data(), p, threads);
        if (st) return st;
    }
    for (long long i = 0; i < p; ++i)
        for (long long j = 0; j < p; ++j) {
            C acc{0.0, 0.0};
            for (long long k = 0; k < m; ++k) {
                C t = cmul(ep[k + i * m], solved[k + j * m]);
                acc.re += t.re;
                acc.im += t.im;
            }
            C pp = entry(m + i, m + j);
            C zz = csub(pp, acc);
            if (!(std::isfinite(zz.re) && std::isfinite(zz.im))) return ORC_ERR_SINGULAR;
            z[2 * (i * p + j)] = zz.re;
            z[2 * (i * p + j) + 1] = dc ? 0.0 : zz.im;
        }
    return ORC_OK;
}

void orc_system_free(orc_system *s) { delete s; }

}  // extern "C"
