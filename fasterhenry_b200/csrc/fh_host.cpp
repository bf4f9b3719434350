// Host side of the extraction path: geometry validation, discretization into
// filament bundles, the loop basis, and the JSON / MAT v4 / SPICE writers.
// Nothing here touches the device.  Compiled with -ffp-contract=off so that
// the filaments are the reference's bit for bit (same operations, same order).
#include <algorithm>
#include <array>
#include <functional>
#include <charconv>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <limits>
#include <string>

#include "fh_internal.h"

namespace fhb {

static thread_local std::string g_last_error;

fh_status fail(fh_error_info *err, fh_status status, const std::string &msg, int64_t a, int64_t b,
               double frequency, int32_t detail) {
    g_last_error = msg;
    if (err) {
        err->status = status;
        err->detail = detail;
        err->index_a = a;
        err->index_b = b;
        err->frequency = frequency;
        err->iterations = -1;
        err->residual = 0.0;
    }
    return status;
}

void clear_error(fh_error_info *err) {
    if (err) {
        err->status = FH_OK;
        err->detail = 0;
        err->index_a = err->index_b = -1;
        err->frequency = 0.0;
        err->iterations = -1;
        err->residual = 0.0;
    }
}

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kMu0 = 4.0e-7 * kPi;
constexpr double kEps = std::numeric_limits<double>::epsilon();

// nalgebra-ordered vector helpers: dot = (x*x' + y*y') + z*z'.
inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator*(Vec3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline Vec3 operator/(Vec3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(Vec3 a, Vec3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double norm(Vec3 a) { return std::sqrt(dot(a, a)); }
inline Vec3 cross(Vec3 a, Vec3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline Vec3 vabs(Vec3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline bool finite3(Vec3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline double fmax_nan(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }

Vec3 node_pos(const fh_node &n) { return {n.x, n.y, n.z}; }

// A segment resolved to coordinates (geometry.rs:140-160).
struct Resolved {
    Vec3 a, b;
    double width, height, sigma;
    bool has_dir;
    Vec3 dir;
};

// The scale-invariant Euclidean norm of geometry.rs (divide by the largest
// component first so that tiny or huge coordinates neither under- nor overflow).
double robust_norm(Vec3 v) {
    if (!finite3(v)) return std::nan("");
    double s = fmax_nan(fmax_nan(std::fabs(v.x), std::fabs(v.y)), std::fabs(v.z));
    if (s == 0.0) return 0.0;
    return norm(v / s) * s;
}

// Segment::basis, geometry.rs:223-275.  Returns an empty string on success or
// the SegmentError description.
std::string frame_of(const Resolved &s, Vec3 &L, Vec3 &W, Vec3 &H) {
    if (!(finite3(s.a) && finite3(s.b))) return "segment end point has a non-finite coordinate";
    if (!(std::isfinite(s.width) && s.width > 0.0)) return "segment width must be positive and finite";
    if (!(std::isfinite(s.height) && s.height > 0.0)) return "segment height must be positive and finite";
    if (!(std::isfinite(s.sigma) && s.sigma > 0.0)) return "segment conductivity must be positive and finite";
    Vec3 span = s.b - s.a;
    double n = robust_norm(span);
    if (!(std::isfinite(n) && n > 0.0)) return "segment has zero length (its end points coincide)";
    L = span / n;
    Vec3 hint;
    if (s.has_dir) {
        double dn = robust_norm(s.dir);
        if (!(std::isfinite(dn) && dn > 0.0))
            return "segment width direction is zero, non-finite, or parallel to the segment";
        Vec3 d = s.dir / dn;
        Vec3 perp = d - L * dot(d, L);
        if (norm(perp) <= 1.0e-9) return "segment width direction is zero, non-finite, or parallel to the segment";
        hint = perp;
    } else {
        Vec3 in_plane = cross(Vec3{0.0, 0.0, 1.0}, L);
        hint = norm(in_plane) < 1.0e-6 ? Vec3{1.0, 0.0, 0.0} : in_plane;
    }
    Vec3 w = hint - L * dot(hint, L);
    W = w / norm(w);
    H = cross(L, W);
    return "";
}

Resolved resolve(const fh_node *nodes, const fh_segment_def &d) {
    Resolved r;
    r.a = node_pos(nodes[d.a]);
    r.b = node_pos(nodes[d.b]);
    r.width = d.width;
    r.height = d.height;
    r.sigma = d.sigma;
    r.has_dir = d.has_width_dir != 0;
    r.dir = {d.width_dir[0], d.width_dir[1], d.width_dir[2]};
    return r;
}

// Rust's f64::powi lowers to binary exponentiation (compiler-rt __powidf2).
double powi(double a, int b) {
    bool recip = b < 0;
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

// Cell weights ratio^min(i, n-1-i) (filament.rs:262-279); false on overflow.
bool cell_weights(int64_t count, double ratio, std::vector<double> &w) {
    w.resize((size_t)count);
    for (int64_t i = 0; i < count; ++i) w[i] = powi(ratio, (int)std::min(i, count - 1 - i));
    for (double x : w)
        if (!std::isfinite(x)) return false;
    return true;
}

struct Cell {
    double centre, size;
};

// graded_cells, filament.rs:534-553.
bool graded(double total, int64_t count, double ratio, std::vector<Cell> &cells) {
    std::vector<double> w;
    if (!cell_weights(count, ratio, w)) return false;
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

fh_filament make_filament(Vec3 a, Vec3 b, double length, Vec3 L, Vec3 W, Vec3 H, double w, double h,
                          double sigma) {
    fh_filament f;
    f.start[0] = a.x, f.start[1] = a.y, f.start[2] = a.z;
    f.end[0] = b.x, f.end[1] = b.y, f.end[2] = b.z;
    f.length = length;
    f.dir_length[0] = L.x, f.dir_length[1] = L.y, f.dir_length[2] = L.z;
    f.dir_width[0] = W.x, f.dir_width[1] = W.y, f.dir_width[2] = W.z;
    f.dir_height[0] = H.x, f.dir_height[1] = H.y, f.dir_height[2] = H.z;
    f.width = w;
    f.height = h;
    f.sigma = sigma;
    return f;
}

// discretize, filament.rs:320-372: cell centres of a uniform grid, width index fastest.
void uniform_bundle(const Resolved &s, Vec3 L, Vec3 W, Vec3 H, int64_t nw, int64_t nh,
                    std::vector<fh_filament> &out) {
    double length = norm(s.b - s.a);
    double fw = s.width / (double)nw, fh = s.height / (double)nh;
    for (int64_t j = 0; j < nh; ++j) {
        Vec3 along_h = H * ((((double)j + 0.5) / (double)nh - 0.5) * s.height);
        for (int64_t i = 0; i < nw; ++i) {
            Vec3 off = W * ((((double)i + 0.5) / (double)nw - 0.5) * s.width) + along_h;
            out.push_back(make_filament(s.a + off, s.b + off, length, L, W, H, fw, fh, s.sigma));
        }
    }
}

// filament/grading.rs:11-55: every graded cell must stay above the kernel's
// conditioning floor and remain resolvable at the segment's coordinates.
bool cells_usable(const Resolved &s, Vec3 W, Vec3 H, const std::vector<Cell> &cw, const std::vector<Cell> &ch,
                  const char **axis, double *extent, double *minimum) {
    double shape = fmax_nan(fmax_nan(norm(s.b - s.a), s.width), s.height);
    Vec3 aa = vabs(s.a), bb = vabs(s.b);
    Vec3 env = Vec3{fmax_nan(aa.x, bb.x), fmax_nan(aa.y, bb.y), fmax_nan(aa.z, bb.z)} + vabs(W) * (0.5 * s.width) +
               vabs(H) * (0.5 * s.height);
    const std::vector<Cell> *sets[2] = {&cw, &ch};
    Vec3 dirs[2] = {W, H};
    const char *names[2] = {"width", "height"};
    for (int k = 0; k < 2; ++k) {
        double scale = dot(vabs(dirs[k]), env);
        double lo = fmax_nan(1e-7 * shape, 32.0 * kEps * scale);
        double ext = std::numeric_limits<double>::infinity();
        for (const Cell &c : *sets[k]) ext = std::min(ext, c.size);
        bool ok = true;
        for (const Cell &c : *sets[k])
            ok = ok && std::isfinite(c.size) && c.size > 0.0 && c.size >= lo && std::isfinite(c.centre) &&
                 c.centre - 0.5 * c.size < c.centre && c.centre + 0.5 * c.size > c.centre;
        for (size_t i = 0; ok && i + 1 < sets[k]->size(); ++i) ok = (*sets[k])[i].centre < (*sets[k])[i + 1].centre;
        if (!ok) {
            *axis = names[k];
            *extent = ext;
            *minimum = lo;
            return false;
        }
    }
    return true;
}

double skin_depth(double f, double sigma) { return 1.0 / std::sqrt(kPi * f * kMu0 * sigma); }

// SkinDepthGrading::count_for, solve.rs:371-386.
int64_t skin_count(const fh_discretization &d, double extent, double sigma) {
    double target = d.target_skin_depths * skin_depth(d.frequency_hz, sigma);
    if (std::isinf(target) || extent <= target) return 1;
    for (int64_t count = 2; count <= d.max_per_axis; ++count) {
        std::vector<double> w;
        if (!cell_weights(count, d.ratio, w)) return count - 1;
        double sum = 0.0;
        for (double x : w) sum += x;
        if (extent / sum <= target) return count;
    }
    return d.max_per_axis;
}

bool ratio_ok(double r) { return std::isfinite(r) && r >= 1.0; }

std::string fmt(const char *f, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

}  // namespace

fh_status validate_geometry(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segs, size_t n_segs,
                            fh_error_info *err) {
    if ((n_nodes && !nodes) || (n_segs && !segs)) return fail(err, FH_ERR_INVALID_ARGUMENT, "null geometry array");
    for (size_t i = 0; i < n_nodes; ++i)
        if (!finite3(node_pos(nodes[i])))
            return fail(err, FH_ERR_GEOMETRY, fmt("node %zu has a non-finite coordinate", i), (int64_t)i, -1, 0.0, 1);
    for (size_t s = 0; s < n_segs; ++s) {
        for (int64_t node : {segs[s].a, segs[s].b})
            if (node < 0 || (size_t)node >= n_nodes)
                return fail(err, FH_ERR_GEOMETRY,
                            fmt("segment %zu refers to node %lld, but the geometry has only %zu nodes", s,
                                (long long)node, n_nodes),
                            (int64_t)s, node, 0.0, 2);
        Vec3 L, W, H;
        std::string why = frame_of(resolve(nodes, segs[s]), L, W, H);
        if (!why.empty())
            return fail(err, FH_ERR_GEOMETRY, fmt("segment %zu is invalid: %s", s, why.c_str()), (int64_t)s, -1, 0.0, 3);
    }
    return FH_OK;
}

// discretize_geometry + Discretization::resolve, solve.rs:468-510 and 947-978.
fh_status discretize_geometry(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segs, size_t n_segs,
                              const fh_discretization *disc, Discretized &out, fh_error_info *err) {
    if (!disc) return fail(err, FH_ERR_INVALID_ARGUMENT, "null discretization");
    fh_status st = validate_geometry(nodes, n_nodes, segs, n_segs, err);
    if (st) return st;
    struct GridSpec {
        int64_t nw, nh;
        double wr, hr;
    };
    std::vector<GridSpec> grids;
    const fh_discretization &d = *disc;
    switch (d.kind) {
        case FH_DISC_UNIFORM:
            grids.assign(n_segs, GridSpec{d.nw, d.nh, 1.0, 1.0});
            break;
        case FH_DISC_PER_SEGMENT:
        case FH_DISC_PER_SEGMENT_GRADED:
            if ((size_t)d.per_segment_len != n_segs || (n_segs && !d.per_segment))
                return fail(err, FH_ERR_MESH,
                            fmt("got filament counts for %lld segments, but the geometry has %zu",
                                (long long)d.per_segment_len, n_segs),
                            (int64_t)n_segs, d.per_segment_len, 0.0, FH_MESH_SEGMENT_COUNT_MISMATCH);
            for (size_t s = 0; s < n_segs; ++s) {
                const fh_axis_grading &g = d.per_segment[s];
                if (d.kind == FH_DISC_PER_SEGMENT_GRADED) {
                    if (!ratio_ok(g.width_ratio))
                        return fail(err, FH_ERR_INVALID_GRADING,
                                    fmt("invalid grading: the width grading ratio must be finite and at least 1, got %g",
                                        g.width_ratio));
                    if (!ratio_ok(g.height_ratio))
                        return fail(err, FH_ERR_INVALID_GRADING,
                                    fmt("invalid grading: the height grading ratio must be finite and at least 1, got %g",
                                        g.height_ratio));
                    grids.push_back({g.nw, g.nh, g.width_ratio, g.height_ratio});
                } else {
                    grids.push_back({g.nw, g.nh, 1.0, 1.0});
                }
            }
            break;
        case FH_DISC_GRADED:
            if (!ratio_ok(d.ratio))
                return fail(err, FH_ERR_INVALID_GRADING,
                            fmt("invalid grading: the grading ratio must be finite and at least 1, got %g", d.ratio));
            grids.assign(n_segs, GridSpec{d.nw, d.nh, d.ratio, d.ratio});
            break;
        case FH_DISC_SKIN_DEPTH: {
            if (!ratio_ok(d.ratio))
                return fail(err, FH_ERR_INVALID_GRADING,
                            fmt("invalid grading: the grading ratio must be finite and at least 1, got %g", d.ratio));
            if (!(std::isfinite(d.target_skin_depths) && d.target_skin_depths > 0.0))
                return fail(err, FH_ERR_INVALID_GRADING,
                            fmt("invalid grading: target_skin_depths must be finite and positive, got %g",
                                d.target_skin_depths));
            if (!(std::isfinite(d.frequency_hz) && d.frequency_hz >= 0.0))
                return fail(err, FH_ERR_INVALID_GRADING,
                            fmt("invalid grading: frequency_hz must be finite and non-negative, got %g", d.frequency_hz));
            if (d.max_per_axis <= 0) return fail(err, FH_ERR_INVALID_GRADING, "invalid grading: max_per_axis must be at least 1");
            for (size_t s = 0; s < n_segs; ++s)
                grids.push_back({skin_count(d, segs[s].width, segs[s].sigma), skin_count(d, segs[s].height, segs[s].sigma),
                                 d.ratio, d.ratio});
            break;
        }
        default:
            return fail(err, FH_ERR_INVALID_ARGUMENT, "unknown discretization kind");
    }
    out.filaments.clear();
    out.per_segment.clear();
    const bool uniform = d.kind == FH_DISC_UNIFORM || d.kind == FH_DISC_PER_SEGMENT;
    for (size_t s = 0; s < n_segs; ++s) {
        const GridSpec &g = grids[s];
        Resolved r = resolve(nodes, segs[s]);
        auto derr = [&](const std::string &why) {
            return fail(err, FH_ERR_DISCRETIZE, fmt("segment %zu: %s", s, why.c_str()), (int64_t)s);
        };
        if (!uniform)
            for (double ratio : {g.wr, g.hr})
                if (!ratio_ok(ratio)) return derr(fmt("the grading ratio must be finite and at least 1, got %g", ratio));
        if (g.nw <= 0 || g.nh <= 0)
            return derr(fmt("filament counts must be at least 1, got nw = %lld, nh = %lld", (long long)g.nw, (long long)g.nh));
        if (g.nw > (int64_t)1 << 31 || g.nh > (int64_t)1 << 31 || g.nw * g.nh > ((int64_t)1 << 31))
            return derr(fmt("filament grid nw * nh overflows, got nw = %lld, nh = %lld", (long long)g.nw, (long long)g.nh));
        Vec3 L, W, H;
        std::string why = frame_of(r, L, W, H);
        if (!why.empty()) return derr(why);
        size_t before = out.filaments.size();
        if (uniform) {
            uniform_bundle(r, L, W, H, g.nw, g.nh, out.filaments);
        } else {
            // discretize_graded_per_axis, filament.rs:478-531
            std::vector<Cell> cw, ch;
            if (!graded(r.width, g.nw, g.wr, cw))
                return derr(fmt("grading ratio %g over %lld filaments overflows to infinity", g.wr, (long long)g.nw));
            if (!graded(r.height, g.nh, g.hr, ch))
                return derr(fmt("grading ratio %g over %lld filaments overflows to infinity", g.hr, (long long)g.nh));
            const char *axis = "";
            double extent = 0, minimum = 0;
            if (!cells_usable(r, W, H, cw, ch, &axis, &extent, &minimum))
                return derr(fmt("unusable graded grid %lld x %lld: %s cell extent %e m requires at least %e m", (long long)g.nw,
                                (long long)g.nh, axis, extent, minimum));
            if (g.wr == 1.0 && g.hr == 1.0) {
                uniform_bundle(r, L, W, H, g.nw, g.nh, out.filaments);
            } else {
                double length = norm(r.b - r.a);
                for (const Cell &hc : ch) {
                    Vec3 along_h = H * hc.centre;
                    for (const Cell &wc : cw) {
                        Vec3 off = W * wc.centre + along_h;
                        out.filaments.push_back(
                            make_filament(r.a + off, r.b + off, length, L, W, H, wc.size, hc.size, r.sigma));
                    }
                }
            }
        }
        out.per_segment.push_back((int64_t)(out.filaments.size() - before));
    }
    return FH_OK;
}

// MeshMatrix::build, mesh.rs:170-263, with the BFS forest of mesh.rs:290-361:
// bundle loops first, then conductor (link) loops, then port loops.
fh_status build_loops(const fh_segment_def *segs, size_t n_segs, size_t n_nodes, const int64_t *per_segment,
                      const fh_port *ports, size_t n_ports, LoopBasis &out, fh_error_info *err) {
    for (size_t s = 0; s < n_segs; ++s)
        if (per_segment[s] <= 0)
            return fail(err, FH_ERR_MESH, fmt("segment %zu has no filaments", s), (int64_t)s, -1, 0.0, FH_MESH_EMPTY_SEGMENT);
    if (n_ports == 0) return fail(err, FH_ERR_MESH, "at least one port is required", -1, -1, 0.0, FH_MESH_NO_PORTS);
    std::vector<int64_t> first(n_segs);
    int64_t total = 0;
    for (size_t s = 0; s < n_segs; ++s) {
        first[s] = total;
        total += per_segment[s];
    }
    if (total >= ((int64_t)1 << 31)) return fail(err, FH_ERR_INVALID_ARGUMENT, "too many filaments");
    out.row_ptr.assign(1, 0);
    out.branch.clear();
    out.sign.clear();
    auto push = [&](int64_t b, double s) {
        out.branch.push_back((int32_t)b);
        out.sign.push_back(s);
    };
    auto close_row = [&] { out.row_ptr.push_back((int64_t)out.branch.size()); };
    for (size_t s = 0; s < n_segs; ++s)
        for (int64_t k = 1; k < per_segment[s]; ++k) {
            push(first[s] + k, 1.0);
            push(first[s], -1.0);
            close_row();
        }
    // Spanning forest by breadth-first search from every unvisited node.
    struct Edge {
        int64_t to, seg;
        bool fwd;
    };
    std::vector<std::vector<Edge>> adj(n_nodes);
    for (size_t s = 0; s < n_segs; ++s) {
        adj[segs[s].a].push_back({segs[s].b, (int64_t)s, true});
        adj[segs[s].b].push_back({segs[s].a, (int64_t)s, false});
    }
    std::vector<int64_t> comp(n_nodes, -1), depth(n_nodes, 0), up_node(n_nodes, -1), up_seg(n_nodes, -1);
    std::vector<char> up_fwd(n_nodes, 0), tree(n_segs, 0);
    int64_t ncomp = 0;
    for (size_t root = 0; root < n_nodes; ++root) {
        if (comp[root] >= 0 || adj[root].empty()) continue;
        comp[root] = ncomp;
        std::deque<int64_t> q{(int64_t)root};
        while (!q.empty()) {
            int64_t v = q.front();
            q.pop_front();
            for (const Edge &e : adj[v])
                if (comp[e.to] < 0) {
                    comp[e.to] = ncomp;
                    up_node[e.to] = v;
                    up_seg[e.to] = e.seg;
                    up_fwd[e.to] = e.fwd;
                    depth[e.to] = depth[v] + 1;
                    tree[e.seg] = 1;
                    q.push_back(e.to);
                }
        }
        ++ncomp;
    }
    // Forest path from `from` to `to` on filament 0 of each segment.
    auto path = [&](int64_t from, int64_t to) {
        std::vector<std::pair<int64_t, double>> up, down;
        int64_t x = from, y = to;
        while (x != y) {
            if (depth[x] >= depth[y]) {
                up.push_back({up_seg[x], up_fwd[x] ? -1.0 : 1.0});
                x = up_node[x];
            } else {
                down.push_back({up_seg[y], up_fwd[y] ? 1.0 : -1.0});
                y = up_node[y];
            }
        }
        up.insert(up.end(), down.rbegin(), down.rend());
        return up;
    };
    for (size_t s = 0; s < n_segs; ++s)
        if (!tree[s]) {
            push(first[s], 1.0);
            for (auto &e : path(segs[s].b, segs[s].a)) push(first[e.first], e.second);
            close_row();
        }
    out.internal = out.rows();
    for (size_t p = 0; p < n_ports; ++p) {
        int64_t pos = ports[p].positive, neg = ports[p].negative;
        for (int64_t node : {pos, neg})
            if (node < 0 || (size_t)node >= n_nodes)
                return fail(err, FH_ERR_MESH,
                            fmt("port %zu refers to node %lld, but the geometry has %zu nodes", p, (long long)node, n_nodes),
                            (int64_t)p, node, 0.0, FH_MESH_UNKNOWN_PORT_NODE);
        if (pos == neg)
            return fail(err, FH_ERR_MESH, fmt("port %zu has the same node (%lld) as both terminals", p, (long long)pos),
                        (int64_t)p, pos, 0.0, FH_MESH_DEGENERATE_PORT);
        if (comp[pos] < 0 || comp[neg] < 0 || comp[pos] != comp[neg])
            return fail(err, FH_ERR_MESH,
                        fmt("port %zu: nodes %lld and %lld are not connected by any chain of segments", p, (long long)pos,
                            (long long)neg),
                        (int64_t)p, pos, 0.0, FH_MESH_PORT_NOT_CONNECTED);
        for (auto &e : path(pos, neg)) push(first[e.first], e.second);
        close_row();
    }
    return FH_OK;
}

// ---------------------------------------------------------------------------
// Output formats
// ---------------------------------------------------------------------------
namespace {

// serde_json / ryu "pretty" formatting of a finite f64: shortest round-trip
// digits, decimal notation for decimal exponents in (-5, 16], otherwise
// scientific with a bare exponent ("1e-7", "1.5e21").
std::string json_number(double v) {
    if (v == 0.0) return std::signbit(v) ? "-0.0" : "0.0";
    char sci[64];
    auto r = std::to_chars(sci, sci + sizeof sci, v, std::chars_format::scientific);
    *r.ptr = 0;
    std::string s(sci);
    bool neg = s[0] == '-';
    if (neg) s = s.substr(1);
    size_t e = s.find('e');
    int exp10 = std::atoi(s.c_str() + e + 1);
    std::string digits;
    for (size_t i = 0; i < e; ++i)
        if (s[i] != '.') digits.push_back(s[i]);
    int length = (int)digits.size();
    int k = exp10 - (length - 1);  // value = digits * 10^k
    int kk = length + k;
    std::string out;
    if (k >= 0 && kk <= 16) {
        out = digits + std::string((size_t)k, '0') + ".0";
    } else if (kk > 0 && kk <= 16) {
        out = digits.substr(0, (size_t)kk) + "." + digits.substr((size_t)kk);
    } else if (kk > -5 && kk <= 0) {
        out = "0." + std::string((size_t)(-kk), '0') + digits;
    } else if (length == 1) {
        out = digits + "e" + std::to_string(kk - 1);
    } else {
        out = digits.substr(0, 1) + "." + digits.substr(1) + "e" + std::to_string(kk - 1);
    }
    return neg ? "-" + out : out;
}

std::string json_string(const char *s) {
    std::string o = "\"";
    for (const char *p = s; *p; ++p) {
        unsigned char c = (unsigned char)*p;
        if (c == '"') o += "\\\"";
        else if (c == '\\') o += "\\\\";
        else if (c == '\n') o += "\\n";
        else if (c == '\r') o += "\\r";
        else if (c == '\t') o += "\\t";
        else if (c < 0x20) {
            char b[8];
            snprintf(b, sizeof b, "\\u%04x", c);
            o += b;
        } else o += (char)c;
    }
    return o + "\"";
}

// Rust's `{:.17e}`: 17 fraction digits, exponent without sign padding.
std::string rust_sci17(double v) {
    char b[64];
    snprintf(b, sizeof b, "%.17e", v);
    std::string s(b);
    size_t e = s.find('e');
    if (e == std::string::npos) return s;
    int ex = std::atoi(s.c_str() + e + 1);
    return s.substr(0, e) + "e" + std::to_string(ex);
}

fh_status emit(const std::string &s, char *buf, size_t capacity, size_t *length) {
    if (length) *length = s.size();
    if (!buf) return FH_OK;
    if (capacity == 0) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "zero-capacity buffer");
    size_t n = std::min(capacity - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
    return s.size() + 1 > capacity ? fail(nullptr, FH_ERR_INVALID_ARGUMENT, "buffer too small") : FH_OK;
}

}  // namespace

// Coupling::resolve (coupling.rs:323-380) with check_transitive (:382-430).
fh_status resolve_coupling(const fh_coupling *c, size_t n_segs, CouplingResolved &out, fh_error_info *err) {
    out = CouplingResolved();
    const bool truncate = c && c->truncate;
    const size_t tags = c ? c->n_segment_groups : 0;
    if (tags && !c->segment_groups) return fail(err, FH_ERR_INVALID_ARGUMENT, "null coupling group list");
    if (c && c->n_couples && !c->couples) return fail(err, FH_ERR_INVALID_ARGUMENT, "null coupling pair list");
    if (tags > n_segs)
        return fail(err, FH_ERR_COUPLING,
                    fmt("coupling names %zu segment groups, but the geometry has %zu segments", tags, n_segs),
                    (int64_t)n_segs, (int64_t)tags, 0.0, FH_COUPLING_SEGMENT_COUNT_MISMATCH);
    auto group_of = [&](size_t s) -> std::string {
        if (s >= tags || !c->segment_groups[s]) return std::string();
        return std::string(c->segment_groups[s]);
    };
    for (size_t s = 0; s < n_segs; ++s) {
        const std::string name = group_of(s);
        auto it = std::find(out.names.begin(), out.names.end(), name);
        if (it == out.names.end()) {
            out.names.push_back(name);
            out.of_segment.push_back((int32_t)out.names.size() - 1);
        } else {
            out.of_segment.push_back((int32_t)(it - out.names.begin()));
        }
    }
    const size_t g = out.names.size();
    out.couples.assign(g * g, 0);
    for (size_t k = 0; k < g; ++k) out.couples[k * g + k] = 1;
    out.all_pairs = !truncate;
    if (truncate) {
        for (size_t k = 0; k < c->n_couples; ++k) {
            int64_t ab[2];
            for (int e = 0; e < 2; ++e) {
                const char *nm = c->couples[2 * k + e];
                const std::string name = nm ? nm : "";
                auto it = std::find(out.names.begin(), out.names.end(), name);
                if (it == out.names.end())
                    return fail(err, FH_ERR_COUPLING,
                                "coupling declares group '" + name + "', which no segment belongs to", (int64_t)k,
                                -1, 0.0, FH_COUPLING_UNKNOWN_GROUP);
                ab[e] = it - out.names.begin();
            }
            out.couples[(size_t)(ab[0] * (int64_t)g + ab[1])] = 1;
            out.couples[(size_t)(ab[1] * (int64_t)g + ab[0])] = 1;
        }
    } else {
        std::fill(out.couples.begin(), out.couples.end(), 1);
    }
    if (g >= 3) {
        std::vector<size_t> parent(g);
        for (size_t k = 0; k < g; ++k) parent[k] = k;
        std::function<size_t(size_t)> find = [&](size_t x) {
            if (parent[x] != x) parent[x] = find(parent[x]);
            return parent[x];
        };
        for (size_t a = 0; a < g; ++a)
            for (size_t b = a + 1; b < g; ++b)
                if (out.couples[a * g + b]) {
                    const size_t ra = find(a), rb = find(b);
                    if (ra != rb) parent[ra] = rb;
                }
        for (size_t a = 0; a < g; ++a)
            for (size_t b = a + 1; b < g; ++b) {
                if (out.couples[a * g + b]) continue;
                if (find(a) == find(b))
                    return fail(err, FH_ERR_COUPLING,
                                "coupling is not transitive: groups '" + out.names[a] + "' and '" + out.names[b] +
                                    "' are only reachable through a third group, but are not declared coupled "
                                    "directly — declare the whole clique",
                                (int64_t)a, (int64_t)b, 0.0, FH_COUPLING_NON_TRANSITIVE);
            }
    }
    return FH_OK;
}

std::vector<fh_truncation_warning> coupling_warnings(const CouplingResolved &r, const fh_node *nodes,
                                                     const fh_segment_def *segs, size_t n_segs) {
    std::vector<fh_truncation_warning> out;
    if (r.all_pairs) return out;
    const size_t g = r.names.size();
    const double inf = std::numeric_limits<double>::infinity();
    std::vector<std::array<double, 6>> box(g, {inf, inf, inf, -inf, -inf, -inf});
    for (size_t s = 0; s < n_segs; ++s)
        for (int64_t node : {segs[s].a, segs[s].b}) {
            const double pt[3] = {nodes[node].x, nodes[node].y, nodes[node].z};
            auto &b = box[(size_t)r.of_segment[s]];
            for (int k = 0; k < 3; ++k) {
                b[k] = std::fmin(b[k], pt[k]);
                b[3 + k] = std::fmax(b[3 + k], pt[k]);
            }
        }
    auto empty = [](const std::array<double, 6> &b) { return b[0] > b[3] || b[1] > b[4] || b[2] > b[5]; };
    auto diagonal = [&](const std::array<double, 6> &b) {
        if (empty(b)) return 0.0;
        double sum = 0.0;
        for (int k = 0; k < 3; ++k) sum += (b[3 + k] - b[k]) * (b[3 + k] - b[k]);
        return std::sqrt(sum);
    };
    auto gap = [&](const std::array<double, 6> &a, const std::array<double, 6> &b) {
        if (empty(a) || empty(b)) return inf;
        double sum = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double apart = std::fmax(std::fmax(a[k] - b[3 + k], b[k] - a[3 + k]), 0.0);
            sum += apart * apart;
        }
        return std::sqrt(sum);
    };
    for (size_t a = 0; a < g; ++a)
        for (size_t b = a + 1; b < g; ++b) {
            if (r.couples[a * g + b]) continue;
            const double extent = std::fmax(diagonal(box[a]), diagonal(box[b]));
            const double separation = gap(box[a], box[b]);
            if (separation < extent) out.push_back(fh_truncation_warning{(int64_t)a, (int64_t)b, separation, extent});
        }
    return out;
}

void conductor_layout(const fh_segment_def *segs, size_t n_segs, size_t n_nodes, const int64_t *per_segment,
                      ConductorLayout &out) {
    std::vector<int64_t> parent(n_nodes);
    for (size_t v = 0; v < n_nodes; ++v) parent[v] = (int64_t)v;
    auto find = [&](int64_t x) {
        while (parent[(size_t)x] != x) {
            parent[(size_t)x] = parent[(size_t)parent[(size_t)x]];
            x = parent[(size_t)x];
        }
        return x;
    };
    for (size_t g = 0; g < n_segs; ++g) {
        const int64_t a = find(segs[g].a), b = find(segs[g].b);
        if (a != b) parent[(size_t)a] = b;
    }
    out = ConductorLayout();
    std::vector<int64_t> roots;
    for (size_t g = 0; g < n_segs; ++g) {
        const int64_t root = find(segs[g].a);
        auto it = std::find(roots.begin(), roots.end(), root);
        if (it == roots.end()) {
            roots.push_back(root);
            out.conductor_of_segment.push_back((int64_t)roots.size() - 1);
        } else {
            out.conductor_of_segment.push_back((int64_t)(it - roots.begin()));
        }
    }
    out.conductors = (int64_t)roots.size();
    out.segment_first.assign(1, 0);
    for (size_t g = 0; g < n_segs; ++g) {
        for (int64_t k = 0; k < per_segment[g]; ++k) out.segment_of_filament.push_back((int64_t)g);
        out.segment_first.push_back(out.segment_first.back() + per_segment[g]);
    }
}

void transpose_loops(const LoopBasis &basis, int64_t n, int64_t rows, TransposedLoops &out) {
    out.offset.assign((size_t)n + 1, 0);
    for (int64_t i = 0; i < rows; ++i)
        for (int64_t k = basis.row_ptr[(size_t)i]; k < basis.row_ptr[(size_t)i + 1]; ++k)
            ++out.offset[(size_t)basis.branch[(size_t)k] + 1];
    for (int64_t b = 0; b < n; ++b) out.offset[(size_t)b + 1] += out.offset[(size_t)b];
    out.loop.assign((size_t)out.offset[(size_t)n], 0);
    out.sign.assign((size_t)out.offset[(size_t)n], 0.0);
    std::vector<int64_t> cursor(out.offset.begin(), out.offset.end() - 1);
    for (int64_t i = 0; i < rows; ++i)
        for (int64_t k = basis.row_ptr[(size_t)i]; k < basis.row_ptr[(size_t)i + 1]; ++k) {
            const int64_t slot = cursor[(size_t)basis.branch[(size_t)k]]++;
            out.loop[(size_t)slot] = (int32_t)i;
            out.sign[(size_t)slot] = basis.sign[(size_t)k];
        }
}

int64_t coupling_kept_pairs(const CouplingResolved &r, const int64_t *per_segment, size_t n_segs) {
    int64_t n = 0;
    const size_t g = r.names.size();
    std::vector<int64_t> sizes(g, 0);
    for (size_t s = 0; s < n_segs; ++s) {
        n += per_segment[s];
        if (!r.of_segment.empty()) sizes[(size_t)r.of_segment[s]] += per_segment[s];
    }
    int64_t dropped = 0;
    for (size_t a = 0; a < g; ++a)
        for (size_t b = a + 1; b < g; ++b)
            if (!r.couples[a * g + b]) dropped += sizes[a] * sizes[b];
    return n * (n + 1) / 2 - dropped;
}

}  // namespace fhb

using namespace fhb;

extern "C" {

int32_t fh_abi_version(void) { return FH_ABI_VERSION; }

const char *fh_last_error(void) { return g_last_error.c_str(); }

int32_t fh_solver_resolve(fh_solver_choice choice, size_t filaments) {
    switch (choice) {
        case FH_SOLVER_DENSE:
            return 0;
        case FH_SOLVER_ITERATIVE:
            return 1;
        default:
            return filaments <= FH_DENSE_PATH_MAX_FILAMENTS ? 0 : 1;
    }
}

fh_status fh_discretize(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segments, size_t n_segments,
                        const fh_discretization *disc, fh_filament *filaments, size_t capacity, size_t *n_filaments,
                        int64_t *per_segment, fh_error_info *err) {
    clear_error(err);
    Discretized d;
    fh_status st = discretize_geometry(nodes, n_nodes, segments, n_segments, disc, d, err);
    if (st) return st;
    if (n_filaments) *n_filaments = d.filaments.size();
    if (per_segment) std::copy(d.per_segment.begin(), d.per_segment.end(), per_segment);
    if (!filaments) return FH_OK;
    if (capacity < d.filaments.size()) return fail(err, FH_ERR_INVALID_ARGUMENT, "filament buffer too small");
    std::copy(d.filaments.begin(), d.filaments.end(), filaments);
    return FH_OK;
}

fh_status fh_mesh_build(const fh_segment_def *segments, size_t n_segments, size_t n_nodes, const int64_t *per_segment,
                        const fh_port *ports, size_t n_ports, int64_t *row_ptr, int64_t *branch, double *sign,
                        size_t cap_rows, size_t cap_nnz, size_t *n_rows, size_t *nnz, size_t *n_internal,
                        fh_error_info *err) {
    clear_error(err);
    if ((n_segments && (!segments || !per_segment)) || (n_ports && !ports))
        return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    for (size_t s = 0; s < n_segments; ++s)
        if (segments[s].a < 0 || segments[s].b < 0 || (size_t)segments[s].a >= n_nodes || (size_t)segments[s].b >= n_nodes)
            return fail(err, FH_ERR_GEOMETRY, "segment refers to a missing node", (int64_t)s);
    LoopBasis lb;
    fh_status st = build_loops(segments, n_segments, n_nodes, per_segment, ports, n_ports, lb, err);
    if (st) return st;
    if (n_rows) *n_rows = (size_t)lb.rows();
    if (nnz) *nnz = lb.branch.size();
    if (n_internal) *n_internal = (size_t)lb.internal;
    if (!row_ptr) return FH_OK;
    if (cap_rows < lb.row_ptr.size() || cap_nnz < lb.branch.size() || !branch || !sign)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "mesh buffers too small");
    std::copy(lb.row_ptr.begin(), lb.row_ptr.end(), row_ptr);
    for (size_t k = 0; k < lb.branch.size(); ++k) {
        branch[k] = lb.branch[k];
        sign[k] = lb.sign[k];
    }
    return FH_OK;
}

fh_status fh_sweep_json(const fh_port *ports, const char *const *port_names, size_t n_ports,
                        const double *frequencies_hz, size_t nf, const double *z, const fh_counts *counts,
                        const fh_timing *timing, char *buf, size_t capacity, size_t *length) {
    if ((n_ports && !ports) || (nf && (!frequencies_hz || !z)))
        return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    std::string o = "{\"schema_version\":1,\"ports\":[";
    for (size_t p = 0; p < n_ports; ++p) {
        if (p) o += ",";
        o += "{\"positive\":" + std::to_string(ports[p].positive) + ",\"negative\":" + std::to_string(ports[p].negative);
        if (port_names && port_names[p]) o += ",\"name\":" + json_string(port_names[p]);
        o += "}";
    }
    o += "],\"frequencies_hz\":[";
    for (size_t k = 0; k < nf; ++k) o += (k ? "," : "") + json_number(frequencies_hz[k]);
    o += "],\"impedance_ohm\":[";
    for (size_t k = 0; k < nf; ++k) {
        o += k ? ",[" : "[";
        for (size_t i = 0; i < n_ports; ++i) {
            o += i ? ",[" : "[";
            for (size_t j = 0; j < n_ports; ++j) {
                const double *e = z + 2 * ((k * n_ports + i) * n_ports + j);
                o += (j ? ",{\"re\":" : "{\"re\":") + json_number(e[0]) + ",\"im\":" + json_number(e[1]) + "}";
            }
            o += "]";
        }
        o += "]";
    }
    o += "],\"provenance\":{\"fasterhenry_version\":\"fasterhenry_b200 0.1.0\",\"counts\":{";
    fh_counts c = counts ? *counts : fh_counts{0, 0, 0, 0, 0, 0};
    o += "\"nodes\":" + std::to_string(c.nodes) + ",\"segments\":" + std::to_string(c.segments) +
         ",\"filaments\":" + std::to_string(c.filaments) + ",\"meshes\":" + std::to_string(c.meshes) +
         ",\"internal_meshes\":" + std::to_string(c.internal_meshes) + ",\"ports\":" + std::to_string(c.ports) + "}";
    if (timing)
        o += ",\"timing\":{\"threads\":1,\"inductance_s\":" + json_number(timing->inductance_s) +
             ",\"assembly_s\":" + json_number(timing->assembly_s) + ",\"solve_s\":" + json_number(timing->solve_s) +
             ",\"total_s\":" + json_number(timing->total_s) + "}";
    o += "}}";
    return emit(o, buf, capacity, length);
}

fh_status fh_write_zc_mat(const char *path, size_t n, const double *freqs, size_t nf, const double *z) {
    if (!path || (nf && (!freqs || !z))) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
    auto header = [&](const std::string &name, int32_t m, int32_t cols, int32_t imag) {
        int32_t h[5] = {0, m, cols, imag, (int32_t)name.size()};
        std::fwrite(h, 4, 5, f);
        std::fwrite(name.data(), 1, name.size(), f);
    };
    header("freqs", 1, (int32_t)nf, 0);
    std::fwrite(freqs, 8, nf, f);
    for (size_t k = 0; k < nf; ++k) {
        header("Zc_" + std::to_string(k + 1), (int32_t)n, (int32_t)n, 1);
        for (int part = 0; part < 2; ++part)
            for (size_t col = 0; col < n; ++col)
                for (size_t row = 0; row < n; ++row) {
                    double v = z[2 * ((k * n + row) * n + col) + part];
                    std::fwrite(&v, 8, 1, f);
                }
    }
    bool ok = std::fclose(f) == 0;
    return ok ? FH_OK : fail(nullptr, FH_ERR_INVALID_ARGUMENT, "write failed");
}

fh_status fh_spice_subckt(size_t n, const double *freqs, size_t nf, const double *z, size_t k, const char *name,
                          char *buf, size_t capacity, size_t *length) {
    if (!freqs || !z || !name || k >= nf) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "bad argument");
    double f = freqs[k];
    double omega = 6.283185307179586 * f;
    auto zr = [&](size_t i, size_t j) { return z[2 * ((k * n + i) * n + j)]; };
    auto zl = [&](size_t i, size_t j) { return z[2 * ((k * n + i) * n + j) + 1] / omega; };
    std::string o = "* fasterhenry SPICE export: " + std::string(name) + " at " + rust_sci17(f) + " Hz\n";
    o += "* port current is positive into p<i>; Z from the R (H sources) and L (coupled inductors) stamps\n";
    o += ".subckt " + std::string(name);
    for (size_t i = 0; i < n; ++i) o += " p" + std::to_string(i + 1) + " n" + std::to_string(i + 1);
    o += "\n";
    for (size_t i = 0; i < n; ++i) {
        double l = f > 0.0 ? zl(i, i) : 0.0;
        o += "L" + std::to_string(i + 1) + " p" + std::to_string(i + 1) + " a" + std::to_string(i) + "_0 " + rust_sci17(l) + "\n";
        std::string node = "a" + std::to_string(i) + "_0";
        for (size_t j = 0; j < n; ++j) {
            double r = zr(i, j);
            if (r != 0.0) {
                std::string next = "a" + std::to_string(i) + "_" + std::to_string(j + 1);
                o += "H" + std::to_string(i + 1) + "_" + std::to_string(j + 1) + " " + node + " " + next + " vsense" +
                     std::to_string(j + 1) + " " + rust_sci17(r) + "\n";
                node = next;
            }
        }
        o += "vsense" + std::to_string(i + 1) + " " + node + " n" + std::to_string(i + 1) + " 0\n";
    }
    if (f > 0.0)
        for (size_t i = 0; i < n; ++i)
            for (size_t j = i + 1; j < n; ++j) {
                double den = std::sqrt(zl(i, i) * zl(j, j));
                double c = std::min(std::max(zl(i, j) / den, -(1.0 - 1e-12)), 1.0 - 1e-12);
                o += "K" + std::to_string(i + 1) + "_" + std::to_string(j + 1) + " L" + std::to_string(i + 1) + " L" +
                     std::to_string(j + 1) + " " + rust_sci17(c) + "\n";
            }
    o += ".ends " + std::string(name) + "\n";
    return emit(o, buf, capacity, length);
}

}  // extern "C"
