// Partial-inductance fill on the device (FP64 throughout).
//
// Replaces the reference's rayon row loop over `evaluate`
// (fasterhenry/src/inductance/batch.rs:355-372, inductance/mod.rs:303-369).
// The upper triangle is classified first — orthogonal pairs stay zero, every
// other pair is appended to a work list for its method — and each method
// then runs as its own kernel so that warps never diverge across methods:
//
//   point quadrature   thread per pair, lists bucketed by log2(#point pairs)
//   bar closed form    thread per pair, 64 Hoer-Love terms summed in order
//   aligned quadrature one CTA per distinct aligned-bar key: the panel tree
//                      is walked by one thread, its Gauss points evaluated
//                      by the whole CTA (the GPU analogue of memo.rs: equal
//                      keys give bit-equal values, so one evaluation serves
//                      every pair that shares the key)
//   sampled filaments  warp per pair, lanes over cross-section samples
//
// Dispatch-critical arithmetic (direction cosines, alignment, the separating-
// axis gap, Gauss orders) uses non-contracted __d*_rn operations in the
// reference's order, so method choices match the reference's bit for bit on
// identical inputs.  The value arithmetic is free to use FMA.
#include <cub/cub.cuh>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "fh_device.cuh"
#include "fh_geom.cuh"

namespace fhb {

__constant__ QuadTables c_quad;

namespace {

// Method ids (inductance/mod.rs:130-152).
enum : int8_t { kOrthogonal = 0, kClosedForm = 1, kAlignedQuadrature = 2, kPoint = 3, kSampled = 4 };

constexpr int kPointBuckets = 17;                     // log2(cost) in 0..16
constexpr int kCatAligned = kPointBuckets;            // aligned-bar pairs
constexpr int kCatSampled = kPointBuckets + 1;        // sampled filaments
constexpr int kCats = kPointBuckets + 2;
constexpr double kMu0Over4Pi = 1.0e-7;
constexpr double kClosedFormMaxError = 1e-10;
constexpr double kEps = 2.220446049250313e-16;

__device__ __forceinline__ int total_cmp(double x, double y) {
    long long a = __double_as_longlong(x), b = __double_as_longlong(y);
    a ^= (long long)(((unsigned long long)(a >> 63)) >> 1);
    b ^= (long long)(((unsigned long long)(b >> 63)) >> 1);
    return a < b ? -1 : (a > b ? 1 : 0);
}

// canonical, inductance/mod.rs:231-254.
__device__ bool canonical_greater(const DevFil &a, const DevFil &b) {
    const double ka[11] = {a.start[0], a.start[1], a.start[2], a.end[0], a.end[1], a.end[2],
                           a.width,    a.height,   a.axes[3],  a.axes[4], a.axes[5]};
    const double kb[11] = {b.start[0], b.start[1], b.start[2], b.end[0], b.end[1], b.end[2],
                           b.width,    b.height,   b.axes[3],  b.axes[4], b.axes[5]};
    for (int i = 0; i < 11; ++i) {
        int c = total_cmp(ka[i], kb[i]);
        if (c) return c > 0;
    }
    return false;
}

// OrderTable::order_for, gauss.rs:123-136; 0 = None.
__device__ __forceinline__ int order_for(const double *thresholds, int count, double half, double distance) {
    if (half <= 0.0) return 1;
    if (isnan(distance) || distance <= 0.0) return 0;
    double delta = __ddiv_rn(distance, half);
    for (int i = 0; i < count; ++i)
        if (delta >= thresholds[i]) return i + 1;
    return 0;
}

__device__ __forceinline__ bool point_orders(const DevFil &f, double gap, int o[3]) {
    for (int k = 0; k < 3; ++k) {
        o[k] = order_for(c_quad.point_thresholds, 16, f.half[k], gap);
        if (!o[k]) return false;
    }
    return o[0] * o[1] * o[2] <= 256;
}

// aligned_bars, inductance/mod.rs:280-300.  Returns false when not aligned.
struct Aligned {
    double length[2], width[2], height[2], offset[3];
};
__device__ bool aligned_bars(const DevFil &a, const DevFil &b, Aligned *o) {
    const double kAligned = 1.0 - 1e-12;
    double wb, hb;
    if (fabs(ndot(a.axes + 3, b.axes + 3)) > kAligned) {
        wb = b.half[1];
        hb = b.half[2];
    } else if (fabs(ndot(a.axes + 3, b.axes + 6)) > kAligned) {
        wb = b.half[2];
        hb = b.half[1];
    } else {
        return false;
    }
    if (o) {
        double delta[3] = {__dsub_rn(b.centre[0], a.centre[0]), __dsub_rn(b.centre[1], a.centre[1]),
                           __dsub_rn(b.centre[2], a.centre[2])};
        o->length[0] = 2.0 * a.half[0];
        o->length[1] = 2.0 * b.half[0];
        o->width[0] = 2.0 * a.half[1];
        o->width[1] = 2.0 * wb;
        o->height[0] = 2.0 * a.half[2];
        o->height[1] = 2.0 * hb;
        o->offset[0] = ndot(delta, a.axes);
        o->offset[1] = ndot(delta, a.axes + 3);
        o->offset[2] = ndot(delta, a.axes + 6);
    }
    return true;
}

// Work-item flags of the coordinate derivative fill (int4.w).
constexpr int kCoordTauMask = 3;   // a's cross-section axis along z x l_a: 1 width, 2 height, 0 none
constexpr int kCoordSigmaNeg = 4;  // z x l_a points along minus that axis
constexpr int kCoordRot = 8;       // rotation derivatives wanted
constexpr int kCoordOrtho = 16;    // orthogonal pair, as two boxes in a's frame (ortho_aligned)
constexpr int kCoordSame = 32;     // both filaments in one segment: stretch derivatives only

// z x l: how a unit vector l changes per unit rotation about the z axis.
__device__ __forceinline__ void zcross(const double *l, double o[3]) {
    o[0] = -l[1];
    o[1] = l[0];
    o[2] = 0.0;
}

// An orthogonal pair as two boxes in a's frame: b's extents along a's axes,
// each of b's axes coinciding with one of a's up to sign (false otherwise).
// Its bar integral is the scalar coupling  int int 1/|r - r'|  of the two
// volumes, whose rate under a rotation gives an orthogonal pair's derivative.
__device__ bool ortho_aligned(const DevFil &a, const DevFil &b, Aligned *o, int *length_axis = nullptr) {
    double ext[3] = {0.0, 0.0, 0.0};
    for (int m = 0; m < 3; ++m) {
        int hit = -1;
        for (int k = 0; k < 3; ++k)
            if (fabs(ndot(b.axes + 3 * m, a.axes + 3 * k)) > 1.0 - 1e-12) hit = k;
        if (hit < 0) return false;
        ext[hit] += 2.0 * b.half[m];
        if (m == 0 && length_axis) *length_axis = hit;
    }
    if (o) {
        const double delta[3] = {b.centre[0] - a.centre[0], b.centre[1] - a.centre[1], b.centre[2] - a.centre[2]};
        o->length[0] = 2.0 * a.half[0];
        o->length[1] = ext[0];
        o->width[0] = 2.0 * a.half[1];
        o->width[1] = ext[1];
        o->height[0] = 2.0 * a.half[2];
        o->height[1] = ext[2];
        o->offset[0] = ndot(delta, a.axes);
        o->offset[1] = ndot(delta, a.axes + 3);
        o->offset[2] = ndot(delta, a.axes + 6);
    }
    return true;
}

struct Classified {
    int cat;          // -1 orthogonal
    int orders;       // packed 5-bit orders (point), 6 fields
    int cost;
    bool swap;        // canonical order is (j, i)
};

// The dispatch of inductance/mod.rs:303-356 up to (not including) the
// evaluation itself.
__device__ Classified classify(const DevFil &fi, const DevFil &fj) {
    Classified c{-1, 0, 0, false};
    c.swap = canonical_greater(fi, fj);
    const DevFil &a = c.swap ? fj : fi;
    const DevFil &b = c.swap ? fi : fj;
    double cosv = ndot(a.axes, b.axes);
    if (fabs(cosv) < 1e-14) return c;
    double cr[3];
    ncross(a.axes, b.axes, cr);
    bool parallel = nnorm(cr) < 1e-6;
    bool aligned = parallel && aligned_bars(a, b, nullptr);
    double gap = separation(a, b);
    int oa[3], ob[3];
    bool point = point_orders(a, gap, oa) && point_orders(b, gap, ob);
    int cost = 0;
    if (point) {
        cost = oa[0] * oa[1] * oa[2] * ob[0] * ob[1] * ob[2];
        if (aligned && cost > 4096) point = false;
    }
    if (point) {
        int bucket = 31 - __clz(cost);
        c.cat = bucket;
        c.cost = cost;
        c.orders = oa[0] | (oa[1] << 5) | (oa[2] << 10) | (ob[0] << 15) | (ob[1] << 20) | (ob[2] << 25);
    } else if (aligned) {
        c.cat = kCatAligned;
    } else {
        c.cat = kCatSampled;
    }
    return c;
}

// Error record: smallest (row, column) of the upper triangle that failed.
struct DevError {
    unsigned long long key;  // (row << 32) | col, ~0 when none
    int code;                // FH_ERR_KERNEL_*
};

__device__ void record_error(DevError *e, int i, int j, int code) {
    int lo = min(i, j), hi = max(i, j);
    unsigned long long key = ((unsigned long long)lo << 32) | (unsigned)hi;
    unsigned long long old = atomicMin(&e->key, key);
    if (key < old) atomicExch(&e->code, code);
}

// Writes L[i][j] = L[j][i] and the method, or records a non-finite value.
// Pair-list mode (n == 0): L and methods are indexed by the item's slot.
__device__ __forceinline__ void store_pair(double *L, int8_t *methods, int64_t n, const int4 &it, double v, int8_t m,
                                           DevError *e) {
    const int i = it.x, j = it.y;
    if (!isfinite(v)) {
        record_error(e, i, j, FH_ERR_KERNEL_NOT_FINITE);
        return;
    }
    if (n == 0) {
        L[it.w] = v;
        if (methods) methods[it.w] = m;
        return;
    }
    L[(int64_t)i + (int64_t)j * n] = v;
    L[(int64_t)j + (int64_t)i * n] = v;
    if (methods) {
        methods[(int64_t)i + (int64_t)j * n] = m;
        methods[(int64_t)j + (int64_t)i * n] = m;
    }
}

// ---------------------------------------------------------------------------
// Classification: pass 0 counts per category, pass 1 writes the work lists.
// Block (32, 8) covers a 32 x 32 tile of the upper triangle.  With `rec`, the
// counting pass also keeps each pair's classification (8 bytes: category + 1,
// canonical swap and cost; packed orders) per upper tile, and the writing
// pass is classify_scatter_kernel, which reads them back instead of
// classifying again.
// ---------------------------------------------------------------------------
// Linear index of upper tile (ti <= tj) of a T x T tile grid.
__device__ __forceinline__ int64_t upper_tile(int ti, int tj, int T) {
    return (int64_t)ti * T - (int64_t)ti * (ti - 1) / 2 + (tj - ti);
}

template <bool kWrite>
__global__ void __launch_bounds__(256) classify_kernel(const DevFil *__restrict__ fil, int n,
                                                       unsigned long long *__restrict__ counts,
                                                       unsigned long long *__restrict__ cursor,
                                                       int4 *__restrict__ items, PairMaskDev mask,
                                                       uint2 *__restrict__ rec) {
    const int ti = blockIdx.y, tj = blockIdx.x;
    if (ti > tj) return;
    __shared__ DevFil s_i[32], s_j[32];
    __shared__ unsigned s_count[kCats];
    __shared__ unsigned long long s_base[kCats];
    const int tid = threadIdx.x + 32 * threadIdx.y;
    {
        const double *gi = reinterpret_cast<const double *>(fil + (int64_t)ti * 32);
        const double *gj = reinterpret_cast<const double *>(fil + (int64_t)tj * 32);
        double *si = reinterpret_cast<double *>(s_i), *sj = reinterpret_cast<double *>(s_j);
        int rows_i = min(32, n - ti * 32), rows_j = min(32, n - tj * 32);
        for (int k = tid; k < 32 * 32; k += 256) {
            if (k < rows_i * 32) si[k] = gi[k];
            if (k < rows_j * 32) sj[k] = gj[k];
        }
    }
    if (tid < kCats) s_count[tid] = 0;
    __syncthreads();
    const int j = tj * 32 + threadIdx.x;
    Classified cls[4];
    unsigned slot[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = ti * 32 + threadIdx.y + 8 * r;
        cls[r].cat = -1;
        if (i < n && j < n && i <= j &&
            (!mask.group || mask.coupled[(int64_t)mask.group[i] * mask.groups + mask.group[j]])) {
            cls[r] = classify(s_i[threadIdx.y + 8 * r], s_j[threadIdx.x]);
            if (cls[r].cat >= 0) slot[r] = atomicAdd(&s_count[cls[r].cat], 1u);
        }
    }
    if (!kWrite && rec) {
        uint2 *out = rec + upper_tile(ti, tj, gridDim.x) * 1024;
#pragma unroll
        for (int r = 0; r < 4; ++r)
            out[(threadIdx.y + 8 * r) * 32 + threadIdx.x] =
                cls[r].cat < 0 ? make_uint2(0u, 0u)
                               : make_uint2((unsigned)(cls[r].cat + 1) | ((cls[r].swap ? 1u : 0u) << 6) |
                                                ((unsigned)cls[r].cost << 7),
                                            (unsigned)cls[r].orders);
    }
    __syncthreads();
    if (!kWrite) {
        if (tid < kCats && s_count[tid]) atomicAdd(&counts[tid], (unsigned long long)s_count[tid]);
        return;
    }
    if (tid < kCats) s_base[tid] = s_count[tid] ? atomicAdd(&cursor[tid], (unsigned long long)s_count[tid]) : 0ull;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        if (cls[r].cat < 0) continue;
        const int i = ti * 32 + threadIdx.y + 8 * r;
        int a = cls[r].swap ? j : i, b = cls[r].swap ? i : j;
        items[s_base[cls[r].cat] + slot[r]] = make_int4(a, b, cls[r].orders, cls[r].cost);
    }
}

// The writing pass from kept classifications (see classify_kernel): the same
// work lists, with the slots taken per tile in the same way.
__global__ void __launch_bounds__(256) classify_scatter_kernel(const uint2 *__restrict__ rec,
                                                               unsigned long long *__restrict__ cursor,
                                                               int4 *__restrict__ items) {
    const int ti = blockIdx.y, tj = blockIdx.x;
    if (ti > tj) return;
    __shared__ unsigned s_count[kCats];
    __shared__ unsigned long long s_base[kCats];
    const int tid = threadIdx.x + 32 * threadIdx.y;
    if (tid < kCats) s_count[tid] = 0;
    __syncthreads();
    const uint2 *in = rec + upper_tile(ti, tj, gridDim.x) * 1024;
    const int j = tj * 32 + threadIdx.x;
    uint2 c[4];
    unsigned slot[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        c[r] = in[(threadIdx.y + 8 * r) * 32 + threadIdx.x];
        const int cat = (int)(c[r].x & 63u) - 1;
        if (cat >= 0) slot[r] = atomicAdd(&s_count[cat], 1u);
    }
    __syncthreads();
    if (tid < kCats) s_base[tid] = s_count[tid] ? atomicAdd(&cursor[tid], (unsigned long long)s_count[tid]) : 0ull;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int cat = (int)(c[r].x & 63u) - 1;
        if (cat < 0) continue;
        const int i = ti * 32 + threadIdx.y + 8 * r;
        const bool swap = (c[r].x >> 6) & 1u;
        const int a = swap ? j : i, b = swap ? i : j;
        items[s_base[cat] + slot[r]] = make_int4(a, b, (int)c[r].y, (int)(c[r].x >> 7));
    }
}

// Classification of an explicit list of pairs (pair-list mode): the same
// passes, one thread per pair; items carry the pair's slot in .w.
template <bool kWrite>
__global__ void __launch_bounds__(256) classify_list_kernel(const DevFil *__restrict__ fil,
                                                            const int2 *__restrict__ pairs, int64_t count,
                                                            unsigned long long *__restrict__ counts,
                                                            unsigned long long *__restrict__ cursor,
                                                            int4 *__restrict__ items) {
    __shared__ unsigned s_count[kCats];
    __shared__ unsigned long long s_base[kCats];
    if (threadIdx.x < kCats) s_count[threadIdx.x] = 0;
    __syncthreads();
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    Classified cls;
    cls.cat = -1;
    unsigned slot = 0;
    int2 pr = make_int2(0, 0);
    if (t < count) {
        pr = pairs[t];
        cls = classify(fil[pr.x], fil[pr.y]);
        if (cls.cat >= 0) slot = atomicAdd(&s_count[cls.cat], 1u);
    }
    __syncthreads();
    if (!kWrite) {
        if (threadIdx.x < kCats && s_count[threadIdx.x])
            atomicAdd(&counts[threadIdx.x], (unsigned long long)s_count[threadIdx.x]);
        return;
    }
    if (threadIdx.x < kCats)
        s_base[threadIdx.x] =
            s_count[threadIdx.x] ? atomicAdd(&cursor[threadIdx.x], (unsigned long long)s_count[threadIdx.x]) : 0ull;
    __syncthreads();
    if (cls.cat >= 0) {
        const int a = cls.swap ? pr.y : pr.x, b = cls.swap ? pr.x : pr.y;
        items[s_base[cls.cat] + slot] = make_int4(a, b, cls.orders, (int)t);
    }
}

// ---------------------------------------------------------------------------
// Point quadrature (neumann.rs:196-266), thread per pair.
// ---------------------------------------------------------------------------
// The offset B.centre - A.centre a point-quadrature pair is evaluated with:
// quantized to a multiple of q = 2^-36 times the smallest cross-section half
// size (exact when it does not fit; `exact` bit d then set), so pairs that
// differ only by the rounding of their absolute coordinates have the same
// offset, quantum `code` and value.
__device__ __forceinline__ void point_offset(const DevFil &A, const DevFil &B, double delta[3], long long code[3],
                                             unsigned &exact) {
    const double mh = fmin(fmin(A.half[1], A.half[2]), fmin(B.half[1], B.half[2]));
    const double inv_q = mh > 0.0 ? ldexp(1.0 / mh, 36) : 0.0;
    exact = 0;
    for (int d = 0; d < 3; ++d) {
        const double dd = __dsub_rn(B.centre[d], A.centre[d]);
        const double sc = dd * inv_q;
        if (inv_q > 0.0 && isfinite(sc) && fabs(sc) < 4.0e18) {
            code[d] = llrint(sc);
            delta[d] = (double)code[d] / inv_q;
        } else {
            code[d] = __double_as_longlong(dd);
            delta[d] = dd;
            exact |= 1u << d;
        }
    }
}

// The point sum of one pair, scaled to L: mu0/4pi cos(a, b) sum w_a w_b / |p_a - p_b|.
// The points are placed relative to the centre of A; `delta` is the offset
// B.centre - A.centre (see point_offset).
// Two bars of the same half sizes whose frames coincide up to the sign of
// each axis.
__device__ __forceinline__ bool same_frame(const DevFil &A, const DevFil &B) {
    for (int d = 0; d < 3; ++d) {
        const double *a = A.axes + 3 * d, *b = B.axes + 3 * d;
        const bool plus = a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
        const bool minus = a[0] == -b[0] && a[1] == -b[1] && a[2] == -b[2];
        if (!(plus || minus) || A.half[d] != B.half[d]) return false;
    }
    return true;
}

// The point sum of two such bars with the same orders.  B's node set along
// each axis is A's (a sign of the axis only relabels a symmetric Gauss set:
// nodes[n - 1 - k] = -nodes[k], equal weights), so a node pair's separation
// depends on the per-axis differences x_i - x_j alone, and the pairs (i, j)
// and (n - 1 - j, n - 1 - i) have the same difference and weight: the sum
// runs over the n (n + 1) / 2 classes i + j <= n - 1 of each axis, weight
// doubled off the anti-diagonal, instead of all n^2 pairs (the same terms
// grouped, in another order).
__device__ double point_value_same(const DevFil &A, int n0, int n1, int n2, const double *aa, const double bc[3]) {
    const double h0 = A.half[0], h1 = A.half[1], h2 = A.half[2];
    double total = 0.0;
    for (int i0 = 0; i0 < n0; ++i0)
        for (int j0 = 0; i0 + j0 < n0; ++j0) {
            const double d0 = h0 * c_quad.nodes[n0][i0] - h0 * c_quad.nodes[n0][j0];
            const double w0 = (h0 * c_quad.weights[n0][i0]) * (h0 * c_quad.weights[n0][j0]) *
                              (i0 + j0 == n0 - 1 ? 1.0 : 2.0);
            double r0[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) r0[d] = aa[d] * d0 - bc[d];
            double s0 = 0.0;
            for (int i1 = 0; i1 < n1; ++i1)
                for (int j1 = 0; i1 + j1 < n1; ++j1) {
                    const double d1 = h1 * c_quad.nodes[n1][i1] - h1 * c_quad.nodes[n1][j1];
                    const double w1 = (0.5 * c_quad.weights[n1][i1]) * (0.5 * c_quad.weights[n1][j1]) *
                                      (i1 + j1 == n1 - 1 ? 1.0 : 2.0);
                    double r1[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) r1[d] = r0[d] + aa[3 + d] * d1;
                    double s1 = 0.0;
                    for (int i2 = 0; i2 < n2; ++i2)
                        for (int j2 = 0; i2 + j2 < n2; ++j2) {
                            const double d2 = h2 * c_quad.nodes[n2][i2] - h2 * c_quad.nodes[n2][j2];
                            const double w2 = (0.5 * c_quad.weights[n2][i2]) * (0.5 * c_quad.weights[n2][j2]) *
                                              (i2 + j2 == n2 - 1 ? 1.0 : 2.0);
                            const double dx = r1[0] + aa[6] * d2, dy = r1[1] + aa[7] * d2, dz = r1[2] + aa[8] * d2;
                            s1 += w2 * rsqrt(dx * dx + dy * dy + dz * dz);
                        }
                    s0 += w1 * s1;
                }
            total += w0 * s0;
        }
    return total;
}

__device__ __forceinline__ double point_value(const DevFil &A, const DevFil &B, int orders, const double delta[3]) {
    const int oa0 = orders & 31, oa1 = (orders >> 5) & 31, oa2 = (orders >> 10) & 31;
    const int ob0 = (orders >> 15) & 31, ob1 = (orders >> 20) & 31, ob2 = (orders >> 25) & 31;
    double bc[3] = {delta[0], delta[1], delta[2]};
    double aa[9], ba[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        aa[k] = A.axes[k];
        ba[k] = B.axes[k];
    }
    if (oa0 == ob0 && oa1 == ob1 && oa2 == ob2 && same_frame(A, B))
        return kMu0Over4Pi * (point_value_same(A, oa0, oa1, oa2, aa, bc) * ndot(A.axes, B.axes));
    const double ah0 = A.half[0], ah1 = 2.0 * A.half[1], ah2 = 2.0 * A.half[2];
    const double bh0 = B.half[0], bh1 = 2.0 * B.half[1], bh2 = 2.0 * B.half[2];
    double total = 0.0;
    for (int la = 0; la < oa0; ++la) {
        const double xl = ah0 * c_quad.nodes[oa0][la], wl = ah0 * c_quad.weights[oa0][la];
        for (int wa = 0; wa < oa1; ++wa) {
            const double xw = ah1 * (0.5 * c_quad.nodes[oa1][wa]), ww = 0.5 * c_quad.weights[oa1][wa];
            for (int ha = 0; ha < oa2; ++ha) {
                const double xh = ah2 * (0.5 * c_quad.nodes[oa2][ha]), wh = 0.5 * c_quad.weights[oa2][ha];
                double p[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) p[d] = aa[d] * xl + aa[3 + d] * xw + aa[6 + d] * xh;
                const double wpa = wl * ww * wh;
                double inner = 0.0;
                for (int lb = 0; lb < ob0; ++lb) {
                    const double yl = bh0 * c_quad.nodes[ob0][lb], vl = bh0 * c_quad.weights[ob0][lb];
                    for (int wb = 0; wb < ob1; ++wb) {
                        const double yw = bh1 * (0.5 * c_quad.nodes[ob1][wb]);
                        const double vlw = vl * (0.5 * c_quad.weights[ob1][wb]);
                        double q[3];
#pragma unroll
                        for (int d = 0; d < 3; ++d) q[d] = p[d] - (bc[d] + ba[d] * yl + ba[3 + d] * yw);
                        for (int hb = 0; hb < ob2; ++hb) {
                            const double yh = bh2 * (0.5 * c_quad.nodes[ob2][hb]);
                            const double vh = 0.5 * c_quad.weights[ob2][hb];
                            const double dx = q[0] - ba[6] * yh, dy = q[1] - ba[7] * yh, dz = q[2] - ba[8] * yh;
                            inner += (vlw * vh) * rsqrt(dx * dx + dy * dy + dz * dz);
                        }
                    }
                }
                total += wpa * inner;
            }
        }
    }
    const double cosv = ndot(A.axes, B.axes);
    return kMu0Over4Pi * (total * cosv);
}

__global__ void __launch_bounds__(128) point_kernel(const DevFil *__restrict__ fil, const int4 *__restrict__ items,
                                                    int64_t count, double *__restrict__ L, int8_t *methods,
                                                    int64_t n, DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        double delta[3];
        long long code[3];
        unsigned exact;
        point_offset(fil[it.x], fil[it.y], delta, code, exact);
        store_pair(L, methods, n, it, point_value(fil[it.x], fil[it.y], it.z, delta), kPoint, err);
    }
}

// Every point pair takes the value of its key's run head.
__global__ void point_scatter_kernel(const int4 *__restrict__ items, const int64_t *__restrict__ item_head,
                                     const double *__restrict__ values, int64_t count, double *__restrict__ L,
                                     int8_t *methods, int64_t n, DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x)
        store_pair(L, methods, n, items[t], values[item_head[t]], kPoint, err);
}

// ---------------------------------------------------------------------------
// Hoer-Love closed form (bar.rs:30-106), thread per pair, terms in order.
// Every operation is an explicit round-to-nearest intrinsic, so nothing is
// contracted into an FMA: the 64 terms cancel down to a value up to ~1e8
// times smaller than their magnitudes, which would amplify any departure
// from the reference's operation-by-operation rounding (its own rounding
// estimate accepts the result up to 1e-10).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double div_(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ double log_term(double coefficient, double x, double r, double rest_sq) {
    if (coefficient == 0.0 || x == 0.0) return 0.0;
    double argument = x >= 0.0 ? add_(x, r) : div_(rest_sq, sub_(r, x));
    return mul_(mul_(coefficient, x), log(argument));
}
__device__ __forceinline__ double atan_term(double x, double y, double z, double r) {
    double product = mul_(mul_(x, y), z);
    if (product == 0.0) return 0.0;
    return -mul_(div_(mul_(mul_(product, z), z), 6.0), atan(div_(mul_(x, y), mul_(z, r))));
}
__device__ double primitive(double x, double y, double z) {
    const double x2 = mul_(x, x), y2 = mul_(y, y), z2 = mul_(z, z);
    const double x4 = mul_(x2, x2), y4 = mul_(y2, y2), z4 = mul_(z2, z2);
    const double r = __dsqrt_rn(add_(add_(x2, y2), z2));
    auto coef = [](double a2, double b2, double a4, double b4) {
        return sub_(sub_(div_(mul_(a2, b2), 4.0), div_(a4, 24.0)), div_(b4, 24.0));
    };
    double s = log_term(coef(y2, z2, y4, z4), x, r, add_(y2, z2));
    s = add_(s, log_term(coef(x2, z2, x4, z4), y, r, add_(x2, z2)));
    s = add_(s, log_term(coef(x2, y2, x4, y4), z, r, add_(x2, y2)));
    const double cross = add_(add_(mul_(x2, y2), mul_(y2, z2)), mul_(z2, x2));
    s = add_(s, div_(mul_(sub_(add_(add_(x4, y4), z4), mul_(3.0, cross)), r), 60.0));
    s = add_(s, atan_term(x, y, z, r));
    s = add_(s, atan_term(x, z, y, r));
    s = add_(s, atan_term(y, z, x, r));
    return s;
}
__device__ __forceinline__ void corner_differences(double e1, double e2, double offset, double q[4]) {
    double sum = mul_(0.5, add_(e1, e2)), diff = mul_(0.5, sub_(e1, e2));
    q[0] = add_(offset, sum);
    q[1] = add_(offset, diff);
    q[2] = sub_(offset, diff);
    q[3] = sub_(offset, sum);
}
__device__ void bar_integral(const Aligned &b, double *value, double *rel) {
    double qx[4], qy[4], qz[4];
    corner_differences(b.length[0], b.length[1], b.offset[0], qx);
    corner_differences(b.width[0], b.width[1], b.offset[1], qy);
    corner_differences(b.height[0], b.height[1], b.offset[2], qz);
    const double signs[4] = {1.0, -1.0, -1.0, 1.0};
    double v = 0.0, mag = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) {
                double term = mul_(mul_(mul_(signs[i], signs[j]), signs[k]), primitive(qx[i], qy[j], qz[k]));
                v = add_(v, term);
                mag = add_(mag, fabs(term));
            }
    *value = v;
    *rel = v > 0.0 ? div_(mul_(mul_(8.0, kEps), mag), v) : INFINITY;
}

// Aligned pairs: closed form when its error estimate allows, else queue the
// pair for the quadrature kernel.
__global__ void __launch_bounds__(128) closed_form_kernel(const DevFil *__restrict__ fil,
                                                          const int4 *__restrict__ items, int64_t count,
                                                          double *__restrict__ L, int8_t *methods, int64_t n,
                                                          int4 *__restrict__ quad_items,
                                                          unsigned long long *__restrict__ quad_count,
                                                          DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        const DevFil &A = fil[it.x];
        const DevFil &B = fil[it.y];
        Aligned ab;
        aligned_bars(A, B, &ab);
        double v, rel;
        bar_integral(ab, &v, &rel);
        if (rel <= kClosedFormMaxError) {
            const double cosv = ndot(A.axes, B.axes);
            const double scale = signum(cosv) / (A.area * B.area);
            store_pair(L, methods, n, it, kMu0Over4Pi * (v * scale), kClosedForm, err);
        } else {
            unsigned long long k = atomicAdd(quad_count, 1ull);
            quad_items[k] = it;
        }
    }
}

// ---------------------------------------------------------------------------
// Aligned quadrature (aligned.rs:206-402): CTA per distinct key.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double overlap_weight(double e1, double e2, double offset, double u) {
    double hi = rmin(0.5 * e1, offset + 0.5 * e2 - u);
    double lo = rmax(-0.5 * e1, offset - 0.5 * e2 - u);
    return rmax(hi - lo, 0.0);
}
__device__ __forceinline__ double parallel_primitive(double q, double rho_sq) {
    q = fabs(q);
    double root = sqrt(q * q + rho_sq);
    if (q == 0.0) return -root;
    return q * log(q + root) - root;
}
// lines::parallel (lines.rs:54-70); false for coaxial overlap.
__device__ __forceinline__ bool lines_parallel(double l1, double l2, double offset, double rho, double *out) {
    double rho_sq = rho * rho;
    double smooth = parallel_primitive(offset + l2, rho_sq) - parallel_primitive(offset, rho_sq) -
                    parallel_primitive(offset + l2 - l1, rho_sq) + parallel_primitive(offset - l1, rho_sq);
    double overlap = rmax(rmin(l1, offset + l2) - rmax(offset, 0.0), 0.0);
    if (overlap == 0.0) {
        *out = smooth;
        return true;
    }
    if (rho > 0.0) {
        *out = smooth - 2.0 * overlap * log(rho);
        return true;
    }
    return false;
}

// An orthogonal pair for the product rule over both cross-sections: A's
// extents along its own axes (length, width, height), b's box in A's frame
// (extents and centre offset) and the axis of A's frame (1 or 2) along which
// b's length lies.
struct OrthoBoxes {
    double ea[3], eb[3], off[3];
    int kb;
};

struct QuadCtx {
    Aligned b;
    OrthoBoxes o;
    double axial_start;
    // coordinate derivatives: a's in-plane transverse axis (1 width, 2
    // height), its sign, and whether the rotation integrals are wanted
    int tau;
    int rot;
    double sigma;
};
__device__ __forceinline__ double integrand(const QuadCtx &c, double u, double v) {
    double weight = overlap_weight(c.b.width[0], c.b.width[1], c.b.offset[1], u) *
                    overlap_weight(c.b.height[0], c.b.height[1], c.b.offset[2], v);
    if (weight == 0.0) return 0.0;
    double k;
    if (!lines_parallel(c.b.length[0], c.b.length[1], c.axial_start, hypot(u, v), &k)) k = 0.0;
    return weight * k;
}

struct Panel {
    double u0, u1, v0, v1;
    int depth;
    int pad;
};
struct Leaf {
    double a0, a1, b0, b1;  // direct: [a0,a1] x [b0,b1]; corner: a0 = a, b0 = b
    int corner;
    int pad;
};

constexpr int kQuadThreads = 128;
constexpr int kStack = 320;
constexpr int kLeaves = 32;
constexpr long long kMaxPanels = 1 << 22;

__device__ int break_points(double e1, double e2, double offset, double *out) {
    double sum = 0.5 * (e1 + e2), diff = 0.5 * fabs(e1 - e2);
    auto snap = [&](double x) { return fabs(x) <= 1e-12 * sum ? 0.0 : x; };
    double p[5] = {snap(offset - sum), snap(offset - diff), snap(offset + diff), snap(offset + sum), 0.0};
    int cnt = 4;
    if (p[0] < 0.0 && p[3] > 0.0) cnt = 5;
    // insertion sort (total order; values are finite, zeros are +0.0)
    for (int i = 1; i < cnt; ++i) {
        double x = p[i];
        int k = i - 1;
        while (k >= 0 && total_cmp(p[k], x) > 0) {
            p[k + 1] = p[k];
            --k;
        }
        p[k + 1] = x;
    }
    int m = 0;
    for (int i = 0; i < cnt; ++i)
        if (m == 0 || !(out[m - 1] == p[i])) out[m++] = p[i];
    return m;
}

// Partials of one overlap weight (overlap_weight) with respect to e1, e2 and
// offset at a fixed abscissa u: piecewise constant, following the branch
// that min/max take.
__device__ __forceinline__ double overlap_weight_grad(double e1, double e2, double offset, double u, double d[3]) {
    const double a = 0.5 * e1, b = offset + 0.5 * e2 - u;
    const double c = -0.5 * e1, e = offset - 0.5 * e2 - u;
    const bool hi_a = a < b, lo_c = c > e;
    const double hi = hi_a ? a : b, lo = lo_c ? c : e;
    if (!(hi - lo > 0.0)) {
        d[0] = d[1] = d[2] = 0.0;
        return 0.0;
    }
    d[0] = (hi_a ? 0.5 : 0.0) - (lo_c ? -0.5 : 0.0);
    d[1] = (hi_a ? 0.0 : 0.5) - (lo_c ? 0.0 : -0.5);
    d[2] = (hi_a ? 0.0 : 1.0) - (lo_c ? 0.0 : 1.0);
    return hi - lo;
}
// The integrand and its partials with respect to the six cross-section
// inputs (width[0], width[1], offset[1], height[0], height[1], offset[2]) at
// fixed (u, v): the axial kernel does not depend on them.  g[0] is the value.
__device__ __forceinline__ void integrand_grad(const QuadCtx &c, double u, double v, double g[7]) {
    double dw[3], dh[3];
    const double ww = overlap_weight_grad(c.b.width[0], c.b.width[1], c.b.offset[1], u, dw);
    const double wh = overlap_weight_grad(c.b.height[0], c.b.height[1], c.b.offset[2], v, dh);
    if (ww == 0.0 || wh == 0.0) {
        for (int k = 0; k < 7; ++k) g[k] = 0.0;
        return;
    }
    double k;
    if (!lines_parallel(c.b.length[0], c.b.length[1], c.axial_start, hypot(u, v), &k)) k = 0.0;
    g[0] = ww * wh * k;
    for (int q = 0; q < 3; ++q) {
        g[1 + q] = dw[q] * wh * k;
        g[4 + q] = ww * dh[q] * k;
    }
}

// Axial terms of two parallel lines A = [0, l1] and B = [as, as + l2] at
// transverse distance rho (the coordinates of lines_parallel): the kernel
// k = int int 1/R, its partials with respect to as, l1 and l2, and with
// `moments` the first moments j1 = int int (x - l1/2) / R^3 and
// j1b = int int (x' - as - l2/2) / R^3 (x on A, x' on B) that a rotation of
// either line about its midpoint weighs.  Every double integral of a
// function of x' - x over the rectangle is F(as + l2) - F(as) - F(as + l2 -
// l1) + F(as - l1) for a second antiderivative F: here R(t) / rho^2 for
// 1/R^3, and t R(t) / (2 rho^2) - asinh(t / rho) / 2 for t / R^3 after one
// integration by parts.  The partials of lines_parallel follow its own
// split: d/dq of |q| log(|q| + R) - R is sign(q) log(|q| + R), and the
// -2 overlap log(rho) term moves with the overlap (a tie of the min / max
// it is made of takes the mean of the two one-sided rates, consistent with
// sign(0) = 0 on the primitive).
struct LineTerms {
    double k, das, dl1, dl2, j1, j1b;
};
// line_terms evaluates the four corner distances q of the rectangle once:
// R = sqrt(q^2 + rho^2) and L = log(|q| + R) serve the kernel (|q| L - R,
// the terms of lines_parallel in its own operation order, so k is the same
// double), its partials (sign(q) L) and the moments (R).
__device__ bool line_terms(double l1, double l2, double as, double rho, bool moments, LineTerms *t) {
    const double r2 = rho * rho;
    const double e = as + l2;
    const double q[4] = {e, as, e - l1, as - l1};
    double R[4], P[4], D[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double aq = fabs(q[i]);
        R[i] = sqrt(aq * aq + r2);
        if (aq == 0.0) {
            P[i] = -R[i];
            D[i] = 0.0;
        } else {
            const double L = log(aq + R[i]);
            P[i] = aq * L - R[i];
            D[i] = q[i] > 0.0 ? L : -L;
        }
    }
    const double smooth = P[0] - P[1] - P[2] + P[3];
    const double overlap = rmax(rmin(l1, e) - rmax(as, 0.0), 0.0);
    double log_rho = 0.0;
    if (overlap == 0.0) {
        t->k = smooth;
    } else if (rho > 0.0) {
        log_rho = log(rho);
        t->k = smooth - 2.0 * overlap * log_rho;
    } else {
        return false;
    }
    t->das = D[0] - D[1] - D[2] + D[3];
    t->dl1 = D[2] - D[3];
    t->dl2 = D[0] - D[2];
    if (overlap > 0.0) {
        const double hi = l1 < e ? 1.0 : (l1 == e ? 0.5 : 0.0);    // d min(l1, e) / d l1
        const double lo = as > 0.0 ? 1.0 : (as == 0.0 ? 0.5 : 0.0);  // d max(as, 0) / d as
        const double lr = 2.0 * log_rho;
        t->dl1 -= lr * hi;
        t->dl2 -= lr * (1.0 - hi);
        t->das -= lr * ((1.0 - hi) - lo);
    }
    t->j1 = t->j1b = 0.0;
    if (moments && r2 > 0.0) {
        // psi(x) = x R(x) / (2 rho^2) - asinh(x / rho) / 2 at the four
        // corners; asinh(|x| / rho) = log(|x| + R) - log(rho), taken from the
        // log already formed where |x| >= rho / 2 (there the difference
        // keeps all but a few ulps of a result of at least 0.48)
        const double lr1 = log_rho != 0.0 ? log_rho : log(rho);
        double psi[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double aq = fabs(q[i]);
            double ash;
            if (aq >= 0.5 * rho) {
                const double L = q[i] > 0.0 ? D[i] : -D[i];  // log(|x| + R)
                ash = q[i] > 0.0 ? L - lr1 : lr1 - L;
            } else {
                ash = asinh(q[i] / rho);
            }
            psi[i] = q[i] * R[i] / (2.0 * r2) - 0.5 * ash;
        }
        const double a = as, b = e;
        const double i00 = (R[0] - R[2] - R[1] + R[3]) / r2;
        const double i10 = (b * (R[0] - R[2]) / r2 + psi[2] - psi[0]) - (a * (R[1] - R[3]) / r2 + psi[3] - psi[1]);
        const double i01 = i10 - t->das;  // int int (x' - x) / R^3 = -dk/das
        t->j1 = i10 - 0.5 * l1 * i00;
        t->j1b = i01 - (as + 0.5 * l2) * i00;
    }
    return true;
}

// The integrand of the coordinate derivatives at relative cross-section
// offset (u, v) (b minus a): g[0] the value, g[1] d/d offset[0], g[2]
// d/d offset[1], g[3] d/d offset[2], g[4] d/d length[0], g[5] d/d length[1]
// (each length stretched about its own centre: as = offset[0] + (length[0] -
// length[1]) / 2), and with c.rot the rates g[6], g[7] of the integral under
// a rotation of a, resp. b, about the z axis through its centre.  For a,
// the rotation moves a point at axial s and transverse t (along
// p = z x l = sigma e_tau) by s p - t l, so the rate is
//   sigma [u_tau W j1 + m_tau w_other dk/das],
// m_tau = int y_tau dy_tau over the overlap at this offset (a's first
// moment); for b, with its own centred coordinates,
//   -sigma [u_tau W j1b + (m_tau + (u_tau - offset_tau) w_tau) w_other dk/das].
__device__ __forceinline__ void integrand_coord(const QuadCtx &c, double u, double v, double g[8]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) g[k] = 0.0;
    double dw[3], dh[3];
    const double ww = overlap_weight_grad(c.b.width[0], c.b.width[1], c.b.offset[1], u, dw);
    const double wh = overlap_weight_grad(c.b.height[0], c.b.height[1], c.b.offset[2], v, dh);
    if (ww == 0.0 || wh == 0.0) return;
    LineTerms t;
    if (!line_terms(c.b.length[0], c.b.length[1], c.axial_start, hypot(u, v), c.rot != 0, &t)) return;
    const double W = ww * wh;
    g[0] = W * t.k;
    g[1] = W * t.das;
    g[2] = dw[2] * wh * t.k;
    g[3] = ww * dh[2] * t.k;
    g[4] = W * (t.dl1 + 0.5 * t.das);
    g[5] = W * (t.dl2 - 0.5 * t.das);
    if (c.rot) {
        const bool ty = c.tau == 1;
        const double ut = ty ? u : v;
        const double e1 = ty ? c.b.width[0] : c.b.height[0], e2 = ty ? c.b.width[1] : c.b.height[1];
        const double ot = ty ? c.b.offset[1] : c.b.offset[2];
        const double hi = rmin(0.5 * e1, ot + 0.5 * e2 - ut), lo = rmax(-0.5 * e1, ot - 0.5 * e2 - ut);
        const double wt = hi - lo;
        const double m = 0.5 * (hi * hi - lo * lo);
        const double wo = ty ? wh : ww;
        g[6] = c.sigma * (ut * W * t.j1 + m * wo * t.das);
        g[7] = -c.sigma * (ut * W * t.j1b + (m + (ut - ot) * wt) * wo * t.das);
    }
}

// The coordinate derivatives of a pair whose cross-sections lie far apart
// against their size, without the panel tree: a p x p Gauss rule on each of
// the overlap weights' break-point panels (the integrand is a product of
// linear weights and a kernel smooth there), p = 4 for gaps g >= 4 s, 5 for
// g >= 2 s, 6 for g >= s (s the largest cross-section side).  The error
// falls like r^(-2p) with r = 1 + 2 g / s, the Bernstein ellipse of the
// nearest singularity (rho = 0); against the restated aligned quadrature
// of the reference the values agreed to 2e-11, 7e-13 and 8e-12 in those
// bands (random pairs of 50-400 um bars with 0.2-3 um sides).
__device__ __forceinline__ int far_rule_order(const Aligned &b) {
    const double gu = rmax(fabs(b.offset[1]) - 0.5 * (b.width[0] + b.width[1]), 0.0);
    const double gv = rmax(fabs(b.offset[2]) - 0.5 * (b.height[0] + b.height[1]), 0.0);
    const double g = hypot(gu, gv);
    const double side = rmax(rmax(b.width[0], b.width[1]), rmax(b.height[0], b.height[1]));
    if (g >= 4.0 * side) return 4;
    if (g >= 2.0 * side) return 5;
    if (g >= side) return 6;
    return 0;
}
// Gauss-Legendre rules of orders 3 to 6 in shared memory (row m - 3): the
// far rules' threads index them at different points, which constant memory
// would serialize.
struct FarRules {
    double n[4][6], w[4][6];
};

// The scalar coupling int int 1/R of two orthogonal boxes far apart against
// their cross-sections, as a product Gauss rule over both cross-sections of
// the double integral over two perpendicular segments, whose antiderivative
// is X log(Y + R) + Y log(X + R) - d atan(X Y / (d R)) (R^2 = X^2 + Y^2 + d^2,
// d the distance between the segments' parallel planes).  log(a + R) is
// taken as log((b^2 + d^2) / (R - a)) for negative a, which has no
// cancellation.  Against the restated aligned quadrature of the reference
// the rule agreed to below 1.2e-11 with m = 3 for gaps of at least eight
// times the largest cross-section side, 6e-13 with m = 4 for at least four
// times, 1.2e-13 with m = 5 for at least twice and 3.5e-13 with m = 6 for at
// least once (random pairs of 50-400 um segments with 0.2-3 um sides).
__device__ __forceinline__ double perp_primitive(double X, double Y, double d) {
    const double d2 = d * d, R = sqrt(X * X + Y * Y + d2);
    auto lg = [&](double a, double b) { return a >= 0.0 ? log(a + R) : log((b * b + d2) / (R - a)); };
    double f = 0.0;
    if (X != 0.0) f += X * lg(Y, X);
    if (Y != 0.0) f += Y * lg(X, Y);
    if (d != 0.0) f -= d * atan(X * Y / (d * R));
    return f;
}
__device__ __forceinline__ int ortho_rule_order(const OrthoBoxes &o) {
    double g2 = 0.0;
    for (int k = 0; k < 3; ++k) {
        const double gk = rmax(fabs(o.off[k]) - 0.5 * (o.ea[k] + o.eb[k]), 0.0);
        g2 += gk * gk;
    }
    const double g = sqrt(g2);
    const int kq = 3 - o.kb;
    const double side = rmax(rmax(o.ea[1], o.ea[2]), rmax(o.eb[0], o.eb[kq]));
    if (g >= 8.0 * side) return 3;
    if (g >= 4.0 * side) return 4;
    if (g >= 2.0 * side) return 5;
    if (g >= side) return 6;
    return 0;
}
__device__ __forceinline__ double ortho_point(const OrthoBoxes &o, const FarRules &fr, int m, int k) {
    const int i = k % m, j = (k / m) % m, kx = (k / (m * m)) % m, l = k / (m * m * m);
    const int kb = o.kb, kq = 3 - kb;
    const double *nd = fr.n[m - 3], *wt = fr.w[m - 3];
    const double ap = 0.5 * o.ea[kb] * nd[i], aq = 0.5 * o.ea[kq] * nd[j];
    const double xb = o.off[0] + 0.5 * o.eb[0] * nd[kx];
    const double bq = o.off[kq] + 0.5 * o.eb[kq] * nd[l];
    const double w = (0.25 * o.ea[kb] * o.ea[kq]) * (0.25 * o.eb[0] * o.eb[kq]) * wt[i] * wt[j] * wt[kx] * wt[l];
    const double x0 = -0.5 * o.ea[0] - xb, x1 = 0.5 * o.ea[0] - xb;
    const double y0 = o.off[kb] - 0.5 * o.eb[kb] - ap, y1 = o.off[kb] + 0.5 * o.eb[kb] - ap;
    const double d = bq - aq;
    return w * (perp_primitive(x1, y1, d) - perp_primitive(x0, y1, d) - perp_primitive(x1, y0, d) +
                perp_primitive(x0, y0, d));
}

// kMode 0: values[h] = the integral.  kMode 1: values[7 h + 0..6] = the
// integral and its partials with respect to (width[0], width[1], offset[1],
// height[0], height[1], offset[2]).  kMode 2: values[8 h + 0..7] = the
// coordinate derivatives of integrand_coord (the work item's flags choose
// the frame and the rotation axis).  The rule (panel tree, leaves, nodes) is
// held at the pair's own geometry, except in kMode 1 and 2 for pairs whose
// cross-sections lie at least one largest side apart (far_rule_order,
// ortho_rule_order), which take fixed rules.  With key_counter the CTAs draw their keys
// from it (keys differ widely in cost), else take every gridDim.x-th; in
// kMode 2 the threads share the points of a batch of leaves evenly (a
// direct leaf has 49 there, fewer than the CTA's threads).
template <int kMode>
__global__ void __launch_bounds__(kQuadThreads) aligned_quadrature_kernel(
    const DevFil *__restrict__ fil, const int4 *__restrict__ items, const int64_t *__restrict__ heads,
    int64_t n_heads, double *__restrict__ values, unsigned long long *__restrict__ key_counter = nullptr) {
    constexpr int kVals = kMode == 0 ? 1 : (kMode == 1 ? 7 : 8);
    __shared__ Panel stack[kStack];
    __shared__ Leaf leaves[kLeaves];
    __shared__ int s_leaf_off[kLeaves + 1];
    __shared__ long long s_key;
    __shared__ int s_nleaves, s_done, s_far, s_npanels;
    __shared__ FarRules far_rules;
    __shared__ QuadCtx ctx;
    __shared__ double s_red[kVals][kQuadThreads / 32];
    __shared__ double r10n[10], r10w[10], r16n[16], r16w[16], r7n[7], r7w[7];
    if (threadIdx.x < 10) {
        r10n[threadIdx.x] = c_quad.nodes[10][threadIdx.x];
        r10w[threadIdx.x] = c_quad.weights[10][threadIdx.x];
        if (threadIdx.x < 7) {
            r7n[threadIdx.x] = c_quad.nodes[7][threadIdx.x];
            r7w[threadIdx.x] = c_quad.weights[7][threadIdx.x];
        }
        if (kMode >= 1 && threadIdx.x < 6)
            for (int m = 3; m <= 6; ++m) {
                far_rules.n[m - 3][threadIdx.x] = threadIdx.x < m ? c_quad.nodes[m][threadIdx.x] : 0.0;
                far_rules.w[m - 3][threadIdx.x] = threadIdx.x < m ? c_quad.weights[m][threadIdx.x] : 0.0;
            }
    }
    if (threadIdx.x < 16) {
        r16n[threadIdx.x] = c_quad.nodes[16][threadIdx.x];
        r16w[threadIdx.x] = c_quad.weights[16][threadIdx.x];
    }
    auto draw = [&](int64_t prev) -> int64_t {
        if (!key_counter) return prev < 0 ? (int64_t)blockIdx.x : prev + gridDim.x;
        if (threadIdx.x == 0) s_key = (long long)atomicAdd(key_counter, 1ull);
        __syncthreads();
        return s_key;
    };
    for (int64_t h = draw(-1); h < n_heads; h = draw(h)) {
        const int4 it = items[heads[h]];
        int sp = 0;
        double axial_scale = 0.0;
        if (threadIdx.x == 0) {
            const DevFil &A = fil[it.x];
            const DevFil &B = fil[it.y];
            bool ortho = false;
            if (kMode == 2 && (it.w & kCoordOrtho)) {
                int kb = 1;
                ortho_aligned(A, B, &ctx.b, &kb);
                ortho = kb == 1 || kb == 2;
                if (ortho) {
                    const Aligned &q = ctx.b;
                    ctx.o = OrthoBoxes{{q.length[0], q.width[0], q.height[0]},
                                       {q.length[1], q.width[1], q.height[1]},
                                       {q.offset[0], q.offset[1], q.offset[2]},
                                       kb};
                }
            } else {
                aligned_bars(A, B, &ctx.b);
            }
            ctx.tau = kMode == 2 ? (it.w & kCoordTauMask) : 0;
            ctx.rot = kMode == 2 && (it.w & kCoordRot) && ctx.tau != 0;
            ctx.sigma = (it.w & kCoordSigmaNeg) ? -1.0 : 1.0;
            const Aligned &b = ctx.b;
            ctx.axial_start = b.offset[0] + 0.5 * (b.length[0] - b.length[1]);
            double l1 = b.length[0], l2 = b.length[1], as = ctx.axial_start;
            double sep[4] = {as + l2, as, as + l2 - l1, as - l1};
            double largest = 0.0;
            for (int k = 0; k < 4; ++k) largest = rmax(largest, fabs(sep[k]));
            axial_scale = INFINITY;
            for (int k = 0; k < 4; ++k)
                if (fabs(sep[k]) > 1e-9 * largest) axial_scale = rmin(axial_scale, fabs(sep[k]));
            double us[5], vs[5];
            int nu = break_points(b.width[0], b.width[1], b.offset[1], us);
            int nv = break_points(b.height[0], b.height[1], b.offset[2], vs);
            // Push panels in reverse so that they pop in the reference's order.
            for (int a = nu - 2; a >= 0; --a)
                for (int c = nv - 2; c >= 0; --c) stack[sp++] = Panel{us[a], us[a + 1], vs[c], vs[c + 1], 0, 0};
            // product rules for pairs far apart: negative order for the
            // orthogonal form
            s_far = kMode == 0 ? 0 : (ortho ? -ortho_rule_order(ctx.o) : far_rule_order(b));
            s_npanels = sp;  // the break-point panels, for the far rule
        }
        double acc = 0.0, gacc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        long long visited = 0;  // panels popped; bounded so that no input can loop without end
        bool overflow = false;
        int far_m = 0;
        if (kMode >= 1) {
            __syncthreads();
            far_m = s_far;
            if (far_m > 0) {
                // p x p points on each break-point panel, the panels as pushed
                const int pp = far_m * far_m, points = s_npanels * pp;
                const double *nd = far_rules.n[far_m - 3], *wt = far_rules.w[far_m - 3];
                for (int k = threadIdx.x; k < points; k += kQuadThreads) {
                    const Panel pn = stack[k / pp];
                    const int a = (k % pp) / far_m, c = k % far_m;
                    const double hu = 0.5 * (pn.u1 - pn.u0), hv = 0.5 * (pn.v1 - pn.v0);
                    if (!(hu > 0.0 && hv > 0.0)) continue;
                    const double uu = 0.5 * (pn.u0 + pn.u1) + hu * nd[a], vv = 0.5 * (pn.v0 + pn.v1) + hv * nd[c];
                    const double wuv = (hu * wt[a]) * (hv * wt[c]);
                    if (kMode == 2) {
                        double g[8];
                        integrand_coord(ctx, uu, vv, g);
                        acc += wuv * g[0];
                        for (int q = 0; q < 7; ++q) gacc[q] += wuv * g[1 + q];
                    } else {
                        double g[7];
                        integrand_grad(ctx, uu, vv, g);
                        acc += wuv * g[0];
                        for (int q = 0; q < 6; ++q) gacc[q] += wuv * g[1 + q];
                    }
                }
            } else if (far_m < 0) {
                const int mo = -far_m, points = mo * mo * mo * mo;
                for (int k = threadIdx.x; k < points; k += kQuadThreads) acc += ortho_point(ctx.o, far_rules, mo, k);
            }
        }
        for (; !far_m;) {
            if (threadIdx.x == 0) {
                // Walk the panel tree until the leaf buffer is full or the tree is done.
                int nl = 0;
                while (sp > 0 && nl < kLeaves) {
                    if (++visited > kMaxPanels) {
                        overflow = true;
                        sp = 0;
                        break;
                    }
                    Panel p = stack[--sp];
                    double su = p.u1 - p.u0, sv = p.v1 - p.v0;
                    if (su <= 0.0 || sv <= 0.0) continue;
                    auto gap = [](double r0, double r1) { return r0 > 0.0 ? r0 : (r1 < 0.0 ? -r1 : 0.0); };
                    double distance = hypot(gap(p.u0, p.u1), gap(p.v0, p.v1));
                    double size = rmax(su, sv);
                    bool split_u = false, split_v = false;
                    double at = 0.0;
                    if (p.depth >= 200 || sp + 2 > kStack) {
                        leaves[nl++] = Leaf{p.u0, p.u1, p.v0, p.v1, 0, 0};
                        continue;
                    }
                    if (distance > 0.0) {
                        if (size <= distance) {
                            leaves[nl++] = Leaf{p.u0, p.u1, p.v0, p.v1, 0, 0};
                            continue;
                        }
                        if (su >= sv) {
                            split_u = true;
                            at = 0.5 * (p.u0 + p.u1);
                        } else {
                            split_v = true;
                            at = 0.5 * (p.v0 + p.v1);
                        }
                    } else {
                        double target = rmin(rmin(su, sv), axial_scale);
                        if (su > 2.0 * target) {
                            split_u = true;
                            at = p.u0 == 0.0 ? target : -target;
                        } else if (sv > 2.0 * target) {
                            split_v = true;
                            at = p.v0 == 0.0 ? target : -target;
                        } else {
                            double fa = p.u0 == 0.0 ? p.u1 : p.u0;
                            double fb = p.v0 == 0.0 ? p.v1 : p.v0;
                            leaves[nl++] = Leaf{fa, 0.0, fb, 0.0, 1, 0};
                            continue;
                        }
                    }
                    // push second half first so the first half is processed next
                    if (split_u) {
                        stack[sp++] = Panel{at, p.u1, p.v0, p.v1, p.depth + 1, 0};
                        stack[sp++] = Panel{p.u0, at, p.v0, p.v1, p.depth + 1, 0};
                    } else if (split_v) {
                        stack[sp++] = Panel{p.u0, p.u1, at, p.v1, p.depth + 1, 0};
                        stack[sp++] = Panel{p.u0, p.u1, p.v0, at, p.depth + 1, 0};
                    }
                }
                s_nleaves = nl;
                s_done = sp == 0;
                s_leaf_off[0] = 0;
                for (int l = 0; l < nl; ++l)
                    s_leaf_off[l + 1] = s_leaf_off[l] + (leaves[l].corner ? 256 : kMode == 2 ? 49 : 100);
            }
            __syncthreads();
            const int nl = s_nleaves;
            if (kMode == 2) {
                // the batch's points in one sequence, every kQuadThreads-th per thread
                const int total = s_leaf_off[nl];
                int l = 0;
                for (int k = threadIdx.x; k < total; k += kQuadThreads) {
                    while (k >= s_leaf_off[l + 1]) ++l;
                    const Leaf lf = leaves[l];
                    const int kk = k - s_leaf_off[l];
                    if (!lf.corner) {
                        const double mu = 0.5 * (lf.a0 + lf.a1), hu = 0.5 * (lf.a1 - lf.a0);
                        const double mv = 0.5 * (lf.b0 + lf.b1), hv = 0.5 * (lf.b1 - lf.b0);
                        // a direct leaf is no larger than its distance from
                        // rho = 0, so the nearest singularity lies outside
                        // the Bernstein ellipse of parameter 3 + 2 sqrt 2 and
                        // 7 x 7 points leave below 1e-10 of it (the
                        // reference's 10 x 10 serve the values)
                        const int a = kk / 7, c = kk % 7;
                        const double uu = mu + hu * r7n[a], wu = hu * r7w[a];
                        const double vv = mv + hv * r7n[c], wv = hv * r7w[c];
                        double g[8];
                        integrand_coord(ctx, uu, vv, g);
                        acc += wu * wv * g[0];
                        for (int q = 0; q < 7; ++q) gacc[q] += wu * wv * g[1 + q];
                    } else {
                        const double A = lf.a0, B = lf.b0, ab = fabs(A * B);
                        const int a = kk / 16, c = kk % 16;
                        const double tau = 0.5 + 0.5 * r16n[a], w_tau = 0.5 * r16w[a];
                        const double s3 = tau * tau * tau;
                        const double radial = w_tau * 3.0 * tau * tau * s3;
                        const double t = 0.5 + 0.5 * r16n[c], w_t = 0.5 * r16w[c];
                        double g1[8], g2[8];
                        integrand_coord(ctx, A * s3, B * s3 * t, g1);
                        integrand_coord(ctx, A * s3 * t, B * s3, g2);
                        const double f = radial * w_t * ab;
                        acc += f * (g1[0] + g2[0]);
                        for (int q = 0; q < 7; ++q) gacc[q] += f * (g1[1 + q] + g2[1 + q]);
                    }
                }
            }
            // Evaluate the leaves: direct leaves have 100 points, corner leaves 256 (each two terms).
            for (int l = 0; l < nl && kMode != 2; ++l) {
                const Leaf lf = leaves[l];
                if (!lf.corner) {
                    double mu = 0.5 * (lf.a0 + lf.a1), hu = 0.5 * (lf.a1 - lf.a0);
                    double mv = 0.5 * (lf.b0 + lf.b1), hv = 0.5 * (lf.b1 - lf.b0);
                    for (int k = threadIdx.x; k < 100; k += kQuadThreads) {
                        int a = k / 10, c = k % 10;
                        double uu = mu + hu * r10n[a], wu = hu * r10w[a];
                        double vv = mv + hv * r10n[c], wv = hv * r10w[c];
                        if (kMode == 1) {
                            double g[7];
                            integrand_grad(ctx, uu, vv, g);
                            acc += wu * wv * g[0];
                            for (int q = 0; q < 6; ++q) gacc[q] += wu * wv * g[1 + q];
                        } else {
                            acc += wu * wv * integrand(ctx, uu, vv);
                        }
                    }
                } else {
                    const double A = lf.a0, B = lf.b0, ab = fabs(A * B);
                    for (int k = threadIdx.x; k < 256; k += kQuadThreads) {
                        int a = k / 16, c = k % 16;
                        double tau = 0.5 + 0.5 * r16n[a], w_tau = 0.5 * r16w[a];
                        double s = tau * tau * tau;
                        double radial = w_tau * 3.0 * tau * tau * s;
                        double t = 0.5 + 0.5 * r16n[c], w_t = 0.5 * r16w[c];
                        if (kMode == 1) {
                            double g1[7], g2[7];
                            integrand_grad(ctx, A * s, B * s * t, g1);
                            integrand_grad(ctx, A * s * t, B * s, g2);
                            const double f = radial * w_t * ab;
                            acc += f * (g1[0] + g2[0]);
                            for (int q = 0; q < 6; ++q) gacc[q] += f * (g1[1 + q] + g2[1 + q]);
                        } else {
                            double value = integrand(ctx, A * s, B * s * t) + integrand(ctx, A * s * t, B * s);
                            acc += radial * w_t * value * ab;
                        }
                    }
                }
            }
            __syncthreads();
            if (s_done) break;
        }
        // block reduction
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) s_red[0][threadIdx.x >> 5] = acc;
        for (int q = 0; q + 1 < kVals; ++q) {
            double x = gacc[q];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31) == 0) s_red[1 + q][threadIdx.x >> 5] = x;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int q = 0; q < kVals; ++q) {
                double s = 0.0;
                for (int w = 0; w < kQuadThreads / 32; ++w) s += s_red[q][w];
                values[kVals * h + q] = overflow ? NAN : s;  // reported as NotFinite by the scatter
            }
        }
        __syncthreads();
    }
}

// Writes every aligned-quadrature pair from its key's value.
__global__ void aligned_scatter_kernel(const DevFil *__restrict__ fil, const int4 *__restrict__ items,
                                       const int64_t *__restrict__ head_of, const double *__restrict__ head_value,
                                       int64_t count, double *__restrict__ L, int8_t *methods, int64_t n,
                                       DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        const DevFil &A = fil[it.x];
        const DevFil &B = fil[it.y];
        const double cosv = ndot(A.axes, B.axes);
        const double scale = signum(cosv) / (A.area * B.area);
        store_pair(L, methods, n, it, kMu0Over4Pi * (head_value[head_of[t]] * scale), kAlignedQuadrature,
                   err);
    }
}

// Key of an aligned pair: the nine numbers of AlignedBars (memo.rs:61-76).
struct AlignedKey {
    static constexpr int kWords = 9;
    __device__ static void get(const DevFil *fil, int4 it, unsigned long long k[kWords]) {
        Aligned b;
        aligned_bars(fil[it.x], fil[it.y], &b);
        const double v[9] = {b.length[0], b.length[1], b.width[0], b.width[1], b.height[0],
                             b.height[1], b.offset[0], b.offset[1], b.offset[2]};
        for (int i = 0; i < 9; ++i) k[i] = (unsigned long long)__double_as_longlong(v[i]);
    }
};

// Key of a coordinate-derivative quadrature pair: the nine numbers of its
// frame (aligned_bars, or ortho_aligned for an orthogonal pair) and the
// flags that choose the frame and the rotation axis.
struct CoordKey {
    static constexpr int kWords = 10;
    __device__ static void get(const DevFil *fil, int4 it, unsigned long long k[kWords]) {
        Aligned b;
        if (it.w & kCoordOrtho)
            ortho_aligned(fil[it.x], fil[it.y], &b);
        else
            aligned_bars(fil[it.x], fil[it.y], &b);
        const double v[9] = {b.length[0], b.length[1], b.width[0], b.width[1], b.height[0],
                             b.height[1], b.offset[0], b.offset[1], b.offset[2]};
        for (int i = 0; i < 9; ++i) k[i] = (unsigned long long)__double_as_longlong(v[i]);
        k[9] = (unsigned long long)(it.w & (kCoordTauMask | kCoordSigmaNeg | kCoordRot | kCoordOrtho));
    }
};

// Key of a point-quadrature pair: its geometry up to a translation -- the
// half sizes and axes of both filaments and the orders exactly, the offset
// of the centres as point_offset quantizes it.  The pair's value is a
// function of the key alone (point_value with that offset), so it does not
// depend on which pair of a run is evaluated; it differs from the sum at the
// unquantized offset by about q / distance, below 1e-11 of it (the point
// method is only chosen for pairs at least a cross-section apart).
struct PointKey {
    static constexpr int kWords = 29;
    __device__ static void get(const DevFil *fil, int4 it, unsigned long long k[kWords]) {
        const DevFil &A = fil[it.x], &B = fil[it.y];
        double delta[3];
        long long code[3];
        unsigned exact;
        point_offset(A, B, delta, code, exact);
        for (int d = 0; d < 3; ++d) k[d] = (unsigned long long)code[d];
        k[3] = exact;
        for (int d = 0; d < 3; ++d) {
            k[4 + d] = (unsigned long long)__double_as_longlong(A.half[d]);
            k[7 + d] = (unsigned long long)__double_as_longlong(B.half[d]);
        }
        for (int d = 0; d < 9; ++d) {
            k[10 + d] = (unsigned long long)__double_as_longlong(A.axes[d]);
            k[19 + d] = (unsigned long long)__double_as_longlong(B.axes[d]);
        }
        k[28] = (unsigned)it.z;
    }
};

template <class Key>
__global__ void key_hash_kernel(const DevFil *__restrict__ fil, const int4 *__restrict__ items, int64_t count,
                                unsigned long long *__restrict__ hash, int64_t *__restrict__ index) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long k[Key::kWords];
        Key::get(fil, items[t], k);
        unsigned long long h = 0x9e3779b97f4a7c15ull;
        for (int i = 0; i < Key::kWords; ++i) {
            h = (h ^ k[i]) * 0x9e3779b97f4a7c15ull;
            h = (h << 29) | (h >> 35);
        }
        h ^= h >> 30;
        h *= 0xbf58476d1ce4e5b9ull;
        h ^= h >> 27;
        h *= 0x94d049bb133111ebull;
        h ^= h >> 31;
        hash[t] = h;
        index[t] = t;
    }
}

// After sorting by hash: head_pos[t] = t when sorted item t starts a new
// key run (hash or full key differs from item t - 1), else 0.  A block takes
// 255 consecutive items and computes each key once into shared memory (256
// keys: its items and the one before them).
constexpr int kHeadsBlock = 256;
template <class Key>
__global__ void __launch_bounds__(kHeadsBlock) key_heads_kernel(const DevFil *__restrict__ fil,
                                                                const int4 *__restrict__ items,
                                                                const unsigned long long *__restrict__ hash_sorted,
                                                                const int64_t *__restrict__ order, int64_t count,
                                                                int64_t *__restrict__ head_pos) {
    extern __shared__ unsigned long long keys[];  // [kHeadsBlock][Key::kWords]
    for (int64_t s0 = (int64_t)blockIdx.x * (kHeadsBlock - 1); s0 < count;
         s0 += (int64_t)gridDim.x * (kHeadsBlock - 1)) {
        const int64_t u = s0 - 1 + threadIdx.x;  // the item whose key this thread forms
        if (u >= 0 && u < count) Key::get(fil, items[order[u]], keys + threadIdx.x * Key::kWords);
        __syncthreads();
        const int64_t t = u;
        if (threadIdx.x > 0 && t < count) {
            bool head = t == 0 || hash_sorted[t] != hash_sorted[t - 1];
            if (!head) {
                const unsigned long long *a = keys + threadIdx.x * Key::kWords, *b = a - Key::kWords;
                for (int i = 0; i < Key::kWords; ++i)
                    if (a[i] != b[i]) head = true;
            }
            head_pos[t] = head ? t : 0;
        }
        __syncthreads();
    }
}

// values[rank[h]] = the value of the pair items[heads[h]] (heads in work-list
// order, which is cost order for the point pairs).
__global__ void __launch_bounds__(128) point_heads_ordered_kernel(const DevFil *__restrict__ fil,
                                                                  const int4 *__restrict__ items,
                                                                  const int64_t *__restrict__ heads,
                                                                  const int64_t *__restrict__ rank, int64_t n_heads,
                                                                  double *__restrict__ values) {
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < n_heads;
         h += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[heads[h]];
        double delta[3];
        long long code[3];
        unsigned exact;
        point_offset(fil[it.x], fil[it.y], delta, code, exact);
        values[rank[h]] = point_value(fil[it.x], fil[it.y], it.z, delta);
    }
}

// rank[h] = h (the identity permutation).
__global__ void iota_kernel(int64_t *__restrict__ v, int64_t count) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x)
        v[t] = t;
}

// flag[t] = 1 where sorted item t heads its key's run.
__global__ void head_flag_kernel(const int64_t *__restrict__ headof, int64_t count, int64_t *__restrict__ flag) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x)
        flag[t] = headof[t] == t ? 1 : 0;
}

// heads[rank] = the item of each run head; item_head[item] = its head's rank.
__global__ void head_compact_kernel(const int64_t *__restrict__ order, const int64_t *__restrict__ headof,
                                    const int64_t *__restrict__ rank, const int64_t *__restrict__ flag, int64_t count,
                                    int64_t *__restrict__ heads, int64_t *__restrict__ item_head) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        if (flag[t]) heads[rank[t]] = order[t];
        item_head[order[t]] = rank[headof[t]];
    }
}

// ---------------------------------------------------------------------------
// Sampled filaments (neumann.rs:280-325 with lines.rs:72-170), warp per pair.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double skew_log_term(double x, double big_r, double a, double residual_sq) {
    if (x == 0.0) return 0.0;
    double argument = a >= 0.0 ? big_r + a : residual_sq / (big_r - a);
    return argument > 0.0 ? x * log(argument) : 0.0;
}
__device__ double skew_primitive(double s, double t, double d, double cosv, double sinv) {
    double sin_sq = sinv * sinv;
    double versine = sin_sq / (1.0 + fabs(cosv));
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
    double big_r = sqrt(rmax(planar_sq + d * d, 0.0));
    double logs = skew_log_term(s, big_r, a_s, s * s * sin_sq + d * d) + skew_log_term(t, big_r, a_t, t * t * sin_sq + d * d);
    if (d == 0.0 || big_r == 0.0) return logs;
    return logs - (d / sinv) * atan((d * d * cosv + s * t * sin_sq) / (d * big_r * sinv));
}
__device__ bool lines_skew(const double *a0, const double *a1, const double *b0, const double *b1, double *out) {
    double da[3] = {a1[0] - a0[0], a1[1] - a0[1], a1[2] - a0[2]};
    double db[3] = {b1[0] - b0[0], b1[1] - b0[1], b1[2] - b0[2]};
    double la = sqrt(da[0] * da[0] + da[1] * da[1] + da[2] * da[2]);
    double lb = sqrt(db[0] * db[0] + db[1] * db[1] + db[2] * db[2]);
    double u[3] = {da[0] / la, da[1] / la, da[2] / la}, v[3] = {db[0] / lb, db[1] / lb, db[2] / lb};
    double cosv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
    double c[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    double sinv = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    if (isnan(sinv) || sinv < 0.0) return false;
    double w0[3] = {a0[0] - b0[0], a0[1] - b0[1], a0[2] - b0[2]};
    double du = u[0] * w0[0] + u[1] * w0[1] + u[2] * w0[2];
    double dv = v[0] * w0[0] + v[1] * w0[1] + v[2] * w0[2];
    double sin_sq = sinv * sinv;
    double s0 = (cosv * dv - du) / sin_sq, t0 = (dv - cosv * du) / sin_sq;
    double r[3] = {w0[0] + u[0] * s0 - v[0] * t0, w0[1] + u[1] * s0 - v[1] * t0, w0[2] + u[2] * s0 - v[2] * t0};
    double d = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    double w0n = sqrt(w0[0] * w0[0] + w0[1] * w0[1] + w0[2] * w0[2]);
    if (d <= 1e-14 * (la + lb + w0n)) d = 0.0;
    double s_lo = -s0, s_hi = la - s0, t_lo = -t0, t_hi = lb - t0;
    *out = skew_primitive(s_hi, t_hi, d, cosv, sinv) - skew_primitive(s_hi, t_lo, d, cosv, sinv) -
           skew_primitive(s_lo, t_hi, d, cosv, sinv) + skew_primitive(s_lo, t_lo, d, cosv, sinv);
    return true;
}

__global__ void __launch_bounds__(128) sampled_kernel(const DevFil *__restrict__ fil, const int4 *__restrict__ items,
                                                      int64_t count, double *__restrict__ L, int8_t *methods,
                                                      int64_t n, DevError *err) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = warp; t < count; t += warps) {
        const int4 it = items[t];
        const DevFil &A = fil[it.x];
        const DevFil &B = fil[it.y];
        const double cosv = ndot(A.axes, B.axes);
        double cr[3];
        ncross(A.axes, B.axes, cr);
        const bool parallel = nnorm(cr) < 1e-6;
        const double gap = separation(A, B);
        auto order = [&](double half, int bump) {
            int o = order_for(c_quad.sample_thresholds, 8, half, gap);
            return o ? o : 8 + bump;
        };
        const int oa0 = order(A.half[1], 0), oa1 = order(A.half[2], 0);
        const int ob0 = order(B.half[1], 1), ob1 = order(B.half[2], 1);
        const int na = oa0 * oa1, nb = ob0 * ob1;
        const double la = 2.0 * A.half[0], lb = 2.0 * B.half[0];
        double acc = 0.0;
        int bad = 0;
        for (int k = lane; k < na * nb; k += 32) {
            const int ia = k / nb, ib = k % nb;
            const int iaw = ia / oa1, iah = ia % oa1, ibw = ib / ob1, ibh = ib % ob1;
            double pa[3], pb[3];
            const double xaw = 0.5 * c_quad.nodes[oa0][iaw], xah = 0.5 * c_quad.nodes[oa1][iah];
            const double xbw = 0.5 * c_quad.nodes[ob0][ibw], xbh = 0.5 * c_quad.nodes[ob1][ibh];
            const double wa = (0.5 * c_quad.weights[oa0][iaw]) * (0.5 * c_quad.weights[oa1][iah]);
            const double wb = (0.5 * c_quad.weights[ob0][ibw]) * (0.5 * c_quad.weights[ob1][ibh]);
            for (int d = 0; d < 3; ++d) {
                pa[d] = A.centre[d] + (A.axes[3 + d] * (2.0 * A.half[1] * xaw) + A.axes[6 + d] * (2.0 * A.half[2] * xah));
                pb[d] = B.centre[d] + (B.axes[3 + d] * (2.0 * B.half[1] * xbw) + B.axes[6 + d] * (2.0 * B.half[2] * xbh));
            }
            double kernel = 0.0;
            bool ok;
            if (parallel) {
                double delta[3] = {pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]};
                double along = delta[0] * A.axes[0] + delta[1] * A.axes[1] + delta[2] * A.axes[2];
                double rr[3] = {delta[0] - A.axes[0] * along, delta[1] - A.axes[1] * along, delta[2] - A.axes[2] * along};
                double rho = sqrt(rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2]);
                ok = lines_parallel(la, lb, along + 0.5 * (la - lb), rho, &kernel);
            } else {
                double a0[3], a1[3], b0[3], b1[3];
                for (int d = 0; d < 3; ++d) {
                    a0[d] = pa[d] - A.axes[d] * A.half[0];
                    a1[d] = pa[d] + A.axes[d] * A.half[0];
                    b0[d] = pb[d] - B.axes[d] * B.half[0];
                    b1[d] = pb[d] + B.axes[d] * B.half[0];
                }
                ok = lines_skew(a0, a1, b0, b1, &kernel);
            }
            if (!ok) bad = 1;
            acc += wa * wb * kernel;
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        bad = __any_sync(0xffffffffu, bad);
        if (lane == 0) {
            if (bad) {
                record_error(err, it.x, it.y, FH_ERR_KERNEL_COINCIDENT);
            } else {
                const double direction = parallel ? signum(cosv) : cosv;
                store_pair(L, methods, n, it, kMu0Over4Pi * (acc * direction), kSampled, err);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Derivative fill: for every pair (a, b) the partial derivatives of L_ab with
// respect to the width and the thickness of the segment of a (b held fixed)
// and of the segment of b (a held fixed), evaluated with the pair's own
// dispatch (method, Gauss orders, closed-form acceptance, panel tree).
// Written to Dw/Dh as D[a + b n] = dL_ab / d(side a), D[b + a n] = dL_ab /
// d(side b); on the diagonal only the first side (the second is equal by the
// symmetry of the integral).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_grad(const GradOut &g, int64_t n, int a, int b, const double d[4],
                                           DevError *e) {
    if (!(isfinite(d[0]) && isfinite(d[1]) && isfinite(d[2]) && isfinite(d[3]))) {
        record_error(e, a, b, FH_ERR_KERNEL_NOT_FINITE);
        return;
    }
    g.Dw[(int64_t)a + (int64_t)b * n] = d[0];
    g.Dh[(int64_t)a + (int64_t)b * n] = d[1];
    if (a != b) {
        g.Dw[(int64_t)b + (int64_t)a * n] = d[2];
        g.Dh[(int64_t)b + (int64_t)a * n] = d[3];
    }
}

// Point quadrature: the Gauss points of a move with its centre (sw, sh along
// its width / height axes) and with its cross-section (gw, gh times the
// point's fraction of the width / height); the weights do not move.  With
// S = sum wp wq / |p - q| and d = p - q, dS = -sum wp wq d . (dp - dq) / |d|^3.
__global__ void __launch_bounds__(128) point_grad_kernel(const DevFil *__restrict__ fil, const FilTan *__restrict__ tan,
                                                         const int4 *__restrict__ items, int64_t count, GradOut g,
                                                         int64_t n, DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        const DevFil &A = fil[it.x];
        const DevFil &B = fil[it.y];
        const int oa0 = it.z & 31, oa1 = (it.z >> 5) & 31, oa2 = (it.z >> 10) & 31;
        const int ob0 = (it.z >> 15) & 31, ob1 = (it.z >> 20) & 31, ob2 = (it.z >> 25) & 31;
        double aa[9], ba[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            aa[k] = A.axes[k];
            ba[k] = B.axes[k];
        }
        const double ah0 = A.half[0], ah1 = 2.0 * A.half[1], ah2 = 2.0 * A.half[2];
        const double bh0 = B.half[0], bh1 = 2.0 * B.half[1], bh2 = 2.0 * B.half[2];
        // Pair totals: G = sum wp wq d / r^3, and the same weighted by a's
        // width / height fraction (Aw, Ah) or by b's (Kw, Kh).
        double G[3] = {0, 0, 0}, Aw[3] = {0, 0, 0}, Ah[3] = {0, 0, 0}, Kw[3] = {0, 0, 0}, Kh[3] = {0, 0, 0};
        for (int la = 0; la < oa0; ++la) {
            const double xl = ah0 * c_quad.nodes[oa0][la], wl = ah0 * c_quad.weights[oa0][la];
            for (int wa = 0; wa < oa1; ++wa) {
                const double fw = 0.5 * c_quad.nodes[oa1][wa];
                const double xw = ah1 * fw, ww = 0.5 * c_quad.weights[oa1][wa];
                for (int ha = 0; ha < oa2; ++ha) {
                    const double fh = 0.5 * c_quad.nodes[oa2][ha];
                    const double xh = ah2 * fh, wh = 0.5 * c_quad.weights[oa2][ha];
                    double p[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) p[d] = A.centre[d] + aa[d] * xl + aa[3 + d] * xw + aa[6 + d] * xh;
                    const double wpa = wl * ww * wh;
                    double gi[3] = {0, 0, 0}, kw[3] = {0, 0, 0}, kh[3] = {0, 0, 0};
                    for (int lb = 0; lb < ob0; ++lb) {
                        const double yl = bh0 * c_quad.nodes[ob0][lb], vl = bh0 * c_quad.weights[ob0][lb];
                        for (int wb = 0; wb < ob1; ++wb) {
                            const double gwb = 0.5 * c_quad.nodes[ob1][wb];
                            const double yw = bh1 * gwb;
                            const double vlw = vl * (0.5 * c_quad.weights[ob1][wb]);
                            double q[3];
#pragma unroll
                            for (int d = 0; d < 3; ++d) q[d] = p[d] - (B.centre[d] + ba[d] * yl + ba[3 + d] * yw);
                            double sw[3] = {0, 0, 0};
                            for (int hb = 0; hb < ob2; ++hb) {
                                const double ghb = 0.5 * c_quad.nodes[ob2][hb];
                                const double yh = bh2 * ghb;
                                const double vh = 0.5 * c_quad.weights[ob2][hb];
                                const double dx = q[0] - ba[6] * yh, dy = q[1] - ba[7] * yh, dz = q[2] - ba[8] * yh;
                                const double ir = rsqrt(dx * dx + dy * dy + dz * dz);
                                const double e = (vlw * vh) * ir * ir * ir;
                                sw[0] += e * dx;
                                sw[1] += e * dy;
                                sw[2] += e * dz;
                                kh[0] += e * ghb * dx;
                                kh[1] += e * ghb * dy;
                                kh[2] += e * ghb * dz;
                            }
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                gi[d] += sw[d];
                                kw[d] += gwb * sw[d];
                            }
                        }
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        G[d] += wpa * gi[d];
                        Aw[d] += wpa * fw * gi[d];
                        Ah[d] += wpa * fh * gi[d];
                        Kw[d] += wpa * kw[d];
                        Kh[d] += wpa * kh[d];
                    }
                }
            }
        }
        const FilTan ta = tan[it.x], tb = tan[it.y];
        const double scale = kMu0Over4Pi * ndot(A.axes, B.axes);
        double out[4];
        out[0] = -scale * (ta.sw * ndot(aa + 3, G) + ta.gw * ndot(aa + 3, Aw));
        out[1] = -scale * (ta.sh * ndot(aa + 6, G) + ta.gh * ndot(aa + 6, Ah));
        out[2] = scale * (tb.sw * ndot(ba + 3, G) + tb.gw * ndot(ba + 3, Kw));
        out[3] = scale * (tb.sh * ndot(ba + 6, G) + tb.gh * ndot(ba + 6, Kh));
        store_grad(g, n, it.x, it.y, out, err);
    }
}

// Forward-mode value of the Hoer-Love primitive with two tangents (along its
// y and z arguments); x is held fixed.
struct D2 {
    double v, y, z;
};
__device__ __forceinline__ D2 operator+(D2 a, D2 b) { return {a.v + b.v, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D2 operator-(D2 a, D2 b) { return {a.v - b.v, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D2 operator-(D2 a) { return {-a.v, -a.y, -a.z}; }
__device__ __forceinline__ D2 operator*(D2 a, D2 b) { return {a.v * b.v, a.y * b.v + a.v * b.y, a.z * b.v + a.v * b.z}; }
__device__ __forceinline__ D2 operator*(double s, D2 a) { return {s * a.v, s * a.y, s * a.z}; }
__device__ __forceinline__ D2 operator/(D2 a, D2 b) {
    const double q = a.v / b.v;
    return {q, (a.y - q * b.y) / b.v, (a.z - q * b.z) / b.v};
}
__device__ __forceinline__ D2 dlog(D2 a) { return {log(a.v), a.y / a.v, a.z / a.v}; }
__device__ __forceinline__ D2 datan(D2 a) {
    const double s = 1.0 / (1.0 + a.v * a.v);
    return {atan(a.v), a.y * s, a.z * s};
}
__device__ __forceinline__ D2 dsqrt(D2 a) {
    const double r = sqrt(a.v);
    return {r, 0.5 * a.y / r, 0.5 * a.z / r};
}
__device__ __forceinline__ bool dzero(D2 a) { return a.v == 0.0 && a.y == 0.0 && a.z == 0.0; }

__device__ __forceinline__ D2 log_term_d(D2 coefficient, D2 x, D2 r, D2 rest_sq) {
    if (dzero(coefficient)) return {0.0, 0.0, 0.0};
    const D2 argument = x.v >= 0.0 ? x + r : rest_sq / (r - x);
    return coefficient * x * dlog(argument);
}
// x y z z^2 atan(x y / (z r)) / 6 vanishes with all its first derivatives
// wherever one of x, y, z is zero.
__device__ __forceinline__ D2 atan_term_d(D2 x, D2 y, D2 z, D2 r) {
    if (x.v == 0.0 || y.v == 0.0 || z.v == 0.0) return {0.0, 0.0, 0.0};
    const D2 product = x * y * z;
    return -((1.0 / 6.0) * (product * z * z)) * datan((x * y) / (z * r));
}
// The primitive is O(rho^5 log rho) at the origin, so its gradient is zero
// there.
__device__ D2 primitive_d(double xv, double yv, double zv) {
    const D2 x{xv, 0.0, 0.0}, y{yv, 1.0, 0.0}, z{zv, 0.0, 1.0};
    const D2 x2 = x * x, y2 = y * y, z2 = z * z;
    const D2 x4 = x2 * x2, y4 = y2 * y2, z4 = z2 * z2;
    const double rr = xv * xv + yv * yv + zv * zv;
    if (rr == 0.0) return {0.0, 0.0, 0.0};
    const D2 r = dsqrt(x2 + y2 + z2);
    auto coef = [](D2 a2, D2 b2, D2 a4, D2 b4) {
        return 0.25 * (a2 * b2) - (1.0 / 24.0) * a4 - (1.0 / 24.0) * b4;
    };
    D2 s = log_term_d(coef(y2, z2, y4, z4), x, r, y2 + z2);
    s = s + log_term_d(coef(x2, z2, x4, z4), y, r, x2 + z2);
    s = s + log_term_d(coef(x2, y2, x4, y4), z, r, x2 + y2);
    const D2 cross = x2 * y2 + y2 * z2 + z2 * x2;
    s = s + (1.0 / 60.0) * ((x4 + y4 + z4 - 3.0 * cross) * r);
    s = s + atan_term_d(x, y, z, r);
    s = s + atan_term_d(x, z, y, r);
    s = s + atan_term_d(y, z, x, r);
    return s;
}

// Chain rule from the partials of the aligned-bar integral V with respect to
// (width[0], width[1], offset[1], height[0], height[1], offset[2]) to the four
// side derivatives of L_ab = mu0/4pi sign(cos) V / (area_a area_b).  The
// cross-section inputs follow aligned_bars: b's width is width[1] when its
// width axis is a's, else height[1].
__device__ __forceinline__ void aligned_chain(const DevFil &A, const DevFil &B, const FilTan &ta, const FilTan &tb,
                                              double V, const double dV[6], double out[4]) {
    const double *wa = A.axes + 3, *ha = A.axes + 6, *wb = B.axes + 3, *hb = B.axes + 6;
    const bool same = fabs(ndot(wa, wb)) > 1.0 - 1e-12;
    const double dVwA = dV[0] * ta.gw - ta.sw * (dV[2] * ndot(wa, wa) + dV[5] * ndot(wa, ha));
    const double dVhA = dV[3] * ta.gh - ta.sh * (dV[2] * ndot(ha, wa) + dV[5] * ndot(ha, ha));
    const double dVwB = (same ? dV[1] : dV[4]) * tb.gw + tb.sw * (dV[2] * ndot(wb, wa) + dV[5] * ndot(wb, ha));
    const double dVhB = (same ? dV[4] : dV[1]) * tb.gh + tb.sh * (dV[2] * ndot(hb, wa) + dV[5] * ndot(hb, ha));
    const double scale = kMu0Over4Pi * signum(ndot(A.axes, B.axes)) / (A.area * B.area);
    out[0] = scale * (dVwA - V * ta.gw / A.width);
    out[1] = scale * (dVhA - V * ta.gh / A.height);
    out[2] = scale * (dVwB - V * tb.gw / B.width);
    out[3] = scale * (dVhB - V * tb.gh / B.height);
}

// Aligned pairs: the closed form where it is accepted (its derivative by
// forward mode through the 64 corner primitives), else queued for the
// quadrature.
__global__ void __launch_bounds__(128) closed_form_grad_kernel(const DevFil *__restrict__ fil,
                                                               const FilTan *__restrict__ tan,
                                                               const int4 *__restrict__ items, int64_t count,
                                                               GradOut g, int64_t n, int4 *__restrict__ quad_items,
                                                               unsigned long long *__restrict__ quad_count,
                                                               DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        const DevFil &A = fil[it.x];
        const DevFil &B = fil[it.y];
        Aligned ab;
        aligned_bars(A, B, &ab);
        double v, rel;
        bar_integral(ab, &v, &rel);
        if (!(rel <= kClosedFormMaxError)) {
            unsigned long long k = atomicAdd(quad_count, 1ull);
            quad_items[k] = it;
            continue;
        }
        double qx[4], qy[4], qz[4];
        corner_differences(ab.length[0], ab.length[1], ab.offset[0], qx);
        corner_differences(ab.width[0], ab.width[1], ab.offset[1], qy);
        corner_differences(ab.height[0], ab.height[1], ab.offset[2], qz);
        const double signs[4] = {1.0, -1.0, -1.0, 1.0};
        double py[4] = {0, 0, 0, 0}, pz[4] = {0, 0, 0, 0};
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                for (int k = 0; k < 4; ++k) {
                    const D2 f = primitive_d(qx[i], qy[j], qz[k]);
                    const double s = signs[i] * signs[j] * signs[k];
                    py[j] += s * f.y;
                    pz[k] += s * f.z;
                }
        // q[0] = o + (e1 + e2)/2, q[1] = o + (e1 - e2)/2, q[2] = o - (e1 - e2)/2, q[3] = o - (e1 + e2)/2
        const double dV[6] = {0.5 * (py[0] + py[1] - py[2] - py[3]), 0.5 * (py[0] - py[1] + py[2] - py[3]),
                              py[0] + py[1] + py[2] + py[3],         0.5 * (pz[0] + pz[1] - pz[2] - pz[3]),
                              0.5 * (pz[0] - pz[1] + pz[2] - pz[3]), pz[0] + pz[1] + pz[2] + pz[3]};
        double out[4];
        aligned_chain(A, B, tan[it.x], tan[it.y], v, dV, out);
        store_grad(g, n, it.x, it.y, out, err);
    }
}

// Quadrature pairs: the key's integral and partials, then the chain rule.
__global__ void aligned_grad_scatter_kernel(const DevFil *__restrict__ fil, const FilTan *__restrict__ tan,
                                            const int4 *__restrict__ items, const int64_t *__restrict__ head_of,
                                            const double *__restrict__ head_value, int64_t count, GradOut g,
                                            int64_t n, DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        const double *hv = head_value + 7 * head_of[t];
        double out[4];
        aligned_chain(fil[it.x], fil[it.y], tan[it.x], tan[it.y], hv[0], hv + 1, out);
        store_grad(g, n, it.x, it.y, out, err);
    }
}

// ---------------------------------------------------------------------------
// Coordinate derivative fill (no reference counterpart).  A node moving in
// the xy plane moves every filament of the segments that meet there by a
// translation of its centre, a stretch of its length about its centre and a
// rotation about the z axis through its centre.  For every pair (a, b) this
// writes the partial derivatives of L_ab with respect to these coordinates
// of a (b held fixed) to D[a + b n] and of b to D[b + a n]:
//   Dl  translation along l_a          Dp  translation along z x l_a
//   Ds  stretch of the length          Dr  rotation about z
// Two filaments of one segment move together rigidly except for the common
// stretch, which leaves their L_ab unchanged but for the stretch, so such
// pairs get Ds only.  An orthogonal pair has L = 0, and only a rotation
// changes it to first order: dL = mu0/4pi d(cos) / (A_a A_b) int int 1/R.
// On the diagonal Ds holds half of dL_aa / d length (the products add both
// sides, as in the width / thickness fill).
// Methods: point quadrature where the fill takes it (one more Gauss node
// per axis: the derivative kernel d/R^3 is one order steeper); otherwise the
// closed form for a segment's own pairs (forward mode through the 64 corner
// primitives along the length) and for orthogonal pairs (the bar integral
// in a's frame), and the aligned quadrature with the integrand_coord terms
// for pairs of different segments and wherever the closed form's error
// estimate rejects it.
// ---------------------------------------------------------------------------
constexpr int kCoordCatPoint = 0, kCoordCatSame = 1, kCoordCatDiff = 2, kCoordCatOrtho = 3, kCoordCats = 4;

struct CoordClass {
    int cat;  // -1 nothing to write
    int orders;
    int flags;
    int fail;  // FH_ERR_UNSUPPORTED for a pair this fill has no derivative for
    bool swap;
};

__device__ __forceinline__ int bump_order(int o) { return o < kMaxRule - 1 ? o + 1 : o; }

__device__ CoordClass coord_classify(const DevFil &fi, const DevFil &fj, bool same) {
    CoordClass c{-1, 0, 0, 0, false};
    c.swap = canonical_greater(fi, fj);
    const DevFil &a = c.swap ? fj : fi;
    const DevFil &b = c.swap ? fi : fj;
    const double cosv = ndot(a.axes, b.axes);
    int oa[3], ob[3];
    auto pack = [&]() {
        return bump_order(oa[0]) | (bump_order(oa[1]) << 5) | (bump_order(oa[2]) << 10) | (bump_order(ob[0]) << 15) |
               (bump_order(ob[1]) << 20) | (bump_order(ob[2]) << 25);
    };
    if (fabs(cosv) < 1e-14) {
        if (same) return c;
        double za[3], zb[3];
        zcross(a.axes, za);
        zcross(b.axes, zb);
        if (ndot(za, b.axes) == 0.0 && ndot(zb, a.axes) == 0.0) return c;  // stays orthogonal
        const double gap = separation(a, b);
        if (point_orders(a, gap, oa) && point_orders(b, gap, ob)) {
            c.cat = kCoordCatPoint;
            c.orders = pack();
        } else if (ortho_aligned(a, b, nullptr)) {
            c.cat = kCoordCatOrtho;
            c.flags = kCoordOrtho;
        } else {
            c.fail = FH_ERR_UNSUPPORTED;
        }
        return c;
    }
    double cr[3];
    ncross(a.axes, b.axes, cr);
    Aligned ab;
    if (!(nnorm(cr) < 1e-6 && aligned_bars(a, b, &ab))) {
        c.fail = FH_ERR_UNSUPPORTED;
        return c;
    }
    const double gap = separation(a, b);
    bool point = point_orders(a, gap, oa) && point_orders(b, gap, ob);
    if (point && oa[0] * oa[1] * oa[2] * ob[0] * ob[1] * ob[2] > 4096) point = false;
    if (point) {
        c.cat = kCoordCatPoint;
        c.orders = pack();
        c.flags = same ? kCoordSame : 0;
        return c;
    }
    if (same) {
        c.cat = kCoordCatSame;
        c.flags = kCoordSame;
        return c;
    }
    c.cat = kCoordCatDiff;
    double za[3];
    zcross(a.axes, za);
    const double zn = nnorm(za);
    if (zn > 1e-12) {  // not vertical: rotations about z apply
        const double dw = ndot(za, a.axes + 3) / zn, dh = ndot(za, a.axes + 6) / zn;
        const bool tw = fabs(dw) >= fabs(dh);
        const double d = tw ? dw : dh;
        // z x l must be a cross-section axis, and the cross-sections must
        // not meet when projected along the length (the moment integrals
        // are singular there).
        if (fabs(d) < 1.0 - 1e-12 || fabs(a.axes[2]) > 1e-12 ||
            (fabs(ab.offset[1]) <= 0.5 * (ab.width[0] + ab.width[1]) &&
             fabs(ab.offset[2]) <= 0.5 * (ab.height[0] + ab.height[1]))) {
            c.cat = -1;
            c.fail = FH_ERR_UNSUPPORTED;
            return c;
        }
        c.flags = (tw ? 1 : 2) | (d < 0.0 ? kCoordSigmaNeg : 0) | kCoordRot;
    }
    return c;
}

// Classification over the upper triangle (tiles as classify_kernel): pairs
// with at least one moving filament, outside the coupling mask's dropped
// pairs.  Pass 0 counts per category and records unsupported pairs; pass 1
// writes the work lists (a, b, packed orders, flags).
template <bool kWrite>
__global__ void __launch_bounds__(256) coord_classify_kernel(const DevFil *__restrict__ fil,
                                                             const int32_t *__restrict__ seg,
                                                             const uint8_t *__restrict__ move, int n,
                                                             unsigned long long *__restrict__ counts,
                                                             unsigned long long *__restrict__ cursor,
                                                             int4 *__restrict__ items, PairMaskDev mask,
                                                             DevError *err) {
    const int ti = blockIdx.y, tj = blockIdx.x;
    if (ti > tj) return;
    __shared__ DevFil s_i[32], s_j[32];
    __shared__ unsigned s_count[kCoordCats];
    __shared__ unsigned long long s_base[kCoordCats];
    const int tid = threadIdx.x + 32 * threadIdx.y;
    {
        const double *gi = reinterpret_cast<const double *>(fil + (int64_t)ti * 32);
        const double *gj = reinterpret_cast<const double *>(fil + (int64_t)tj * 32);
        double *si = reinterpret_cast<double *>(s_i), *sj = reinterpret_cast<double *>(s_j);
        int rows_i = min(32, n - ti * 32), rows_j = min(32, n - tj * 32);
        for (int k = tid; k < 32 * 32; k += 256) {
            if (k < rows_i * 32) si[k] = gi[k];
            if (k < rows_j * 32) sj[k] = gj[k];
        }
    }
    if (tid < kCoordCats) s_count[tid] = 0;
    __syncthreads();
    const int j = tj * 32 + threadIdx.x;
    CoordClass cls[4];
    unsigned slot[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = ti * 32 + threadIdx.y + 8 * r;
        cls[r].cat = -1;
        if (i < n && j < n && i <= j && (move[i] || move[j]) &&
            (!mask.group || mask.coupled[(int64_t)mask.group[i] * mask.groups + mask.group[j]])) {
            cls[r] = coord_classify(s_i[threadIdx.y + 8 * r], s_j[threadIdx.x], seg[i] == seg[j]);
            if (!kWrite && cls[r].fail) record_error(err, i, j, cls[r].fail);
            if (cls[r].cat >= 0) slot[r] = atomicAdd(&s_count[cls[r].cat], 1u);
        }
    }
    __syncthreads();
    if (!kWrite) {
        if (tid < kCoordCats && s_count[tid]) atomicAdd(&counts[tid], (unsigned long long)s_count[tid]);
        return;
    }
    if (tid < kCoordCats)
        s_base[tid] = s_count[tid] ? atomicAdd(&cursor[tid], (unsigned long long)s_count[tid]) : 0ull;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        if (cls[r].cat < 0) continue;
        const int i = ti * 32 + threadIdx.y + 8 * r;
        const int a = cls[r].swap ? j : i, b = cls[r].swap ? i : j;
        items[s_base[cls[r].cat] + slot[r]] = make_int4(a, b, cls[r].orders, cls[r].flags);
    }
}

__device__ __forceinline__ void store_coord(const CoordOut &o, int64_t n, int a, int b, const double da[4],
                                            const double db[4], DevError *e) {
    bool ok = true;
    for (int k = 0; k < 4; ++k) ok = ok && isfinite(da[k]) && isfinite(db[k]);
    if (!ok) {
        record_error(e, a, b, FH_ERR_KERNEL_NOT_FINITE);
        return;
    }
    const int64_t ab = (int64_t)a + (int64_t)b * n, ba = (int64_t)b + (int64_t)a * n;
    o.Dl[ab] = da[0];
    o.Dp[ab] = da[1];
    o.Ds[ab] = da[2];
    o.Dr[ab] = da[3];
    if (a != b) {
        o.Dl[ba] = db[0];
        o.Dp[ba] = db[1];
        o.Ds[ba] = db[2];
        o.Dr[ba] = db[3];
    }
}

// z x l normalized (zero for a vertical l).
__device__ __forceinline__ void plane_normal(const double *l, double p[3]) {
    zcross(l, p);
    const double nrm = nnorm(p);
    for (int k = 0; k < 3; ++k) p[k] = nrm > 0.0 ? p[k] / nrm : 0.0;
}

// Point quadrature: with d = p - q over the Gauss points of a and b,
// V = sum w / |d| (L = mu0/4pi cos V), G = sum w d / |d|^3, and the moments
// SA = sum w x_a (d . l_a) / |d|^3, SB likewise with b's axial coordinate,
// RA = sum w d . (z x (p - c_a)) / |d|^3, RB likewise for b.  A translation
// e of a changes V by -G . e, of b by G . e; a stretch of a moves its
// points by x_a / length along l_a and scales its weights; a rotation moves
// its points by z x (p - c) and turns l by z x l.
__global__ void __launch_bounds__(128) point_coord_kernel(const DevFil *__restrict__ fil,
                                                          const int4 *__restrict__ items, int64_t count, CoordOut out,
                                                          int64_t n, DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        const DevFil &A = fil[it.x];
        const DevFil &B = fil[it.y];
        const int oa0 = it.z & 31, oa1 = (it.z >> 5) & 31, oa2 = (it.z >> 10) & 31;
        const int ob0 = (it.z >> 15) & 31, ob1 = (it.z >> 20) & 31, ob2 = (it.z >> 25) & 31;
        double aa[9], ba[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            aa[k] = A.axes[k];
            ba[k] = B.axes[k];
        }
        const double ah0 = A.half[0], ah1 = 2.0 * A.half[1], ah2 = 2.0 * A.half[2];
        const double bh0 = B.half[0], bh1 = 2.0 * B.half[1], bh2 = 2.0 * B.half[2];
        double V = 0.0, G[3] = {0.0, 0.0, 0.0}, SA = 0.0, SB = 0.0, RA = 0.0, RB = 0.0;
        for (int la = 0; la < oa0; ++la) {
            const double xl = ah0 * c_quad.nodes[oa0][la], wl = ah0 * c_quad.weights[oa0][la];
            for (int wa = 0; wa < oa1; ++wa) {
                const double xw = ah1 * (0.5 * c_quad.nodes[oa1][wa]), ww = 0.5 * c_quad.weights[oa1][wa];
                for (int ha = 0; ha < oa2; ++ha) {
                    const double xh = ah2 * (0.5 * c_quad.nodes[oa2][ha]), wh = 0.5 * c_quad.weights[oa2][ha];
                    double oA[3], p[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        oA[d] = aa[d] * xl + aa[3 + d] * xw + aa[6 + d] * xh;
                        p[d] = A.centre[d] + oA[d];
                    }
                    const double wpa = wl * ww * wh;
                    double vi = 0.0, gi[3] = {0.0, 0.0, 0.0}, sbi = 0.0, rbi = 0.0;
                    for (int lb = 0; lb < ob0; ++lb) {
                        const double yl = bh0 * c_quad.nodes[ob0][lb], vl = bh0 * c_quad.weights[ob0][lb];
                        for (int wb = 0; wb < ob1; ++wb) {
                            const double yw = bh1 * (0.5 * c_quad.nodes[ob1][wb]);
                            const double vlw = vl * (0.5 * c_quad.weights[ob1][wb]);
                            for (int hb = 0; hb < ob2; ++hb) {
                                const double yh = bh2 * (0.5 * c_quad.nodes[ob2][hb]);
                                const double vh = 0.5 * c_quad.weights[ob2][hb];
                                double oB[3], d[3];
#pragma unroll
                                for (int k = 0; k < 3; ++k) {
                                    oB[k] = ba[k] * yl + ba[3 + k] * yw + ba[6 + k] * yh;
                                    d[k] = p[k] - (B.centre[k] + oB[k]);
                                }
                                const double ir = rsqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                                const double w = vlw * vh;
                                const double e = w * ir * ir * ir;
                                vi += w * ir;
                                gi[0] += e * d[0];
                                gi[1] += e * d[1];
                                gi[2] += e * d[2];
                                sbi += e * yl * (d[0] * ba[0] + d[1] * ba[1] + d[2] * ba[2]);
                                rbi += e * (d[1] * oB[0] - d[0] * oB[1]);
                            }
                        }
                    }
                    V += wpa * vi;
#pragma unroll
                    for (int k = 0; k < 3; ++k) G[k] += wpa * gi[k];
                    SA += wpa * xl * (gi[0] * aa[0] + gi[1] * aa[1] + gi[2] * aa[2]);
                    RA += wpa * (gi[1] * oA[0] - gi[0] * oA[1]);
                    SB += wpa * sbi;
                    RB += wpa * rbi;
                }
            }
        }
        const double cosv = ndot(aa, ba);
        double za[3], zb[3], pa[3], pb[3];
        zcross(aa, za);
        zcross(ba, zb);
        plane_normal(aa, pa);
        plane_normal(ba, pb);
        const double k = kMu0Over4Pi;
        double da[4], db[4];
        da[2] = k * cosv * (V - SA) / (2.0 * A.half[0]);
        db[2] = k * cosv * (V + SB) / (2.0 * B.half[0]);
        if (it.w & kCoordSame) {
            da[0] = da[1] = da[3] = db[0] = db[1] = db[3] = 0.0;
        } else {
            da[0] = -k * cosv * ndot(G, aa);
            da[1] = -k * cosv * ndot(G, pa);
            da[3] = k * (ndot(za, ba) * V - cosv * RA);
            db[0] = k * cosv * ndot(G, ba);
            db[1] = k * cosv * ndot(G, pb);
            db[3] = k * (ndot(zb, aa) * V + cosv * RB);
        }
        store_coord(out, n, it.x, it.y, da, db, err);
    }
}

// A segment's own aligned pairs (kOrtho false: the stretch by forward mode
// along the length through the 64 corner primitives, which are symmetric in
// their three arguments) and near orthogonal pairs (kOrtho: the bar integral
// in a's frame), each where the closed form's error estimate accepts it;
// the rest go to the quadrature list.
template <bool kOrtho>
__global__ void __launch_bounds__(128) closed_form_coord_kernel(const DevFil *__restrict__ fil,
                                                                const int4 *__restrict__ items, int64_t count,
                                                                CoordOut out, int64_t n, int4 *__restrict__ quad_items,
                                                                unsigned long long *__restrict__ quad_count,
                                                                DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        const DevFil &A = fil[it.x];
        const DevFil &B = fil[it.y];
        Aligned ab;
        if (kOrtho)
            ortho_aligned(A, B, &ab);
        else
            aligned_bars(A, B, &ab);
        double v, rel;
        bar_integral(ab, &v, &rel);
        if (!(rel <= kClosedFormMaxError)) {
            unsigned long long k = atomicAdd(quad_count, 1ull);
            quad_items[k] = it;
            continue;
        }
        double da[4] = {0.0, 0.0, 0.0, 0.0}, db[4] = {0.0, 0.0, 0.0, 0.0};
        if (kOrtho) {
            double za[3], zb[3];
            zcross(A.axes, za);
            zcross(B.axes, zb);
            const double scale = kMu0Over4Pi / (A.area * B.area);
            da[3] = scale * ndot(za, B.axes) * v;
            db[3] = scale * ndot(zb, A.axes) * v;
        } else {
            double qx[4], qy[4], qz[4];
            corner_differences(ab.length[0], ab.length[1], ab.offset[0], qx);
            corner_differences(ab.width[0], ab.width[1], ab.offset[1], qy);
            corner_differences(ab.height[0], ab.height[1], ab.offset[2], qz);
            const double signs[4] = {1.0, -1.0, -1.0, 1.0};
            double px[4] = {0.0, 0.0, 0.0, 0.0};
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j)
                    for (int k = 0; k < 4; ++k) px[i] += signs[i] * signs[j] * signs[k] *
                                                          primitive_d(qy[j], qx[i], qz[k]).y;
            const double d0 = 0.5 * (px[0] + px[1] - px[2] - px[3]), d1 = 0.5 * (px[0] - px[1] + px[2] - px[3]);
            const double scale = kMu0Over4Pi * signum(ndot(A.axes, B.axes)) / (A.area * B.area);
            if (it.x == it.y) {
                da[2] = 0.5 * scale * (d0 + d1);
            } else {
                da[2] = scale * d0;
                db[2] = scale * d1;
            }
        }
        store_coord(out, n, it.x, it.y, da, db, err);
    }
}

// Quadrature pairs: the key's eight values (integrand_coord), then the chain
// rule to the two filaments' coordinates.
__global__ void coord_quad_scatter_kernel(const DevFil *__restrict__ fil, const int4 *__restrict__ items,
                                          const int64_t *__restrict__ head_of, const double *__restrict__ head_value,
                                          int64_t count, CoordOut out, int64_t n, DevError *err) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int4 it = items[t];
        const double *hv = head_value + 8 * head_of[t];
        const DevFil &A = fil[it.x];
        const DevFil &B = fil[it.y];
        double da[4] = {0.0, 0.0, 0.0, 0.0}, db[4] = {0.0, 0.0, 0.0, 0.0};
        if (it.w & kCoordOrtho) {
            double za[3], zb[3];
            zcross(A.axes, za);
            zcross(B.axes, zb);
            const double scale = kMu0Over4Pi / (A.area * B.area);
            da[3] = scale * ndot(za, B.axes) * hv[0];
            db[3] = scale * ndot(zb, A.axes) * hv[0];
        } else {
            const double c = signum(ndot(A.axes, B.axes));
            const double scale = kMu0Over4Pi * c / (A.area * B.area);
            if (it.x == it.y) {
                da[2] = 0.5 * scale * (hv[4] + hv[5]);
            } else if (it.w & kCoordSame) {
                da[2] = scale * hv[4];
                db[2] = scale * hv[5];
            } else {
                const int tau = it.w & kCoordTauMask;
                const double sigma = (it.w & kCoordSigmaNeg) ? -1.0 : 1.0;
                const double dtau = tau == 1 ? hv[2] : (tau == 2 ? hv[3] : 0.0);
                const bool rot = (it.w & kCoordRot) && tau != 0;
                da[0] = -scale * hv[1];
                da[1] = -scale * sigma * dtau;
                da[2] = scale * hv[4];
                da[3] = rot ? scale * hv[6] : 0.0;
                db[0] = scale * c * hv[1];
                db[1] = scale * c * sigma * dtau;
                db[2] = scale * hv[5];
                db[3] = rot ? scale * hv[7] : 0.0;
            }
        }
        store_coord(out, n, it.x, it.y, da, db, err);
    }
}

// Congruence M B M^T in the reference's two steps (solve.rs:1172-1200):
// for loop row i, product_i = sum over (a, s_a) in row i of s_a B[a, :], then
// entry (i, j), j >= i, = sum over (b, s_b) in row j of s_b product_i[b],
// each sum in row order, mirrored.  Here product_i is materialized as row i
// of U (loops x n, column-major), so that both steps are coalesced column
// combinations and no (long row) x (long row) pair is evaluated term by term.
constexpr int kRowsCols = 32;  // columns of B per block in loop_rows_kernel
constexpr int kShortRow = 8;   // longer rows go to loop_rows_long_kernel

// U[i + c loops] = sum_p s_p B[a_p + c n], p over row i in order.
__global__ void __launch_bounds__(128) loop_rows_kernel(const double *__restrict__ B, int64_t n,
                                                        const int64_t *__restrict__ row_ptr,
                                                        const int32_t *__restrict__ branch,
                                                        const double *__restrict__ sign, int64_t loops,
                                                        double *__restrict__ U) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= loops) return;
    const int64_t c0 = (int64_t)blockIdx.y * kRowsCols, c1 = min(n, c0 + kRowsCols);
    const int64_t p0 = row_ptr[i], p1 = row_ptr[i + 1];
    if (p1 - p0 > kShortRow) return;  // loop_rows_long_kernel
    for (int64_t c = c0; c < c1; ++c) {
        const double *col = B + c * n;
        double inner = 0.0;
        for (int64_t p = p0; p < p1; ++p) inner = __dadd_rn(inner, __dmul_rn(sign[p], col[branch[p]]));
        U[i + c * loops] = inner;
    }
}

// Rows longer than kShortRow (link and port loops along a path): one thread
// per column, the row's entries in order.
__global__ void __launch_bounds__(256) loop_rows_long_kernel(const double *__restrict__ B, int64_t n,
                                                             const int64_t *__restrict__ row_ptr,
                                                             const int32_t *__restrict__ branch,
                                                             const double *__restrict__ sign, int64_t loops,
                                                             const int64_t *__restrict__ long_rows,
                                                             double *__restrict__ U) {
    const int64_t i = long_rows[blockIdx.y];
    const int64_t p0 = row_ptr[i], p1 = row_ptr[i + 1];
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const double *col = B + c * n;
        double inner = 0.0;
        for (int64_t p = p0; p < p1; ++p) inner = __dadd_rn(inner, __dmul_rn(sign[p], col[branch[p]]));
        U[i + c * loops] = inner;
    }
}

// The same for a diagonal B (resistances): row i of U is zero except
// s_p R[a_p] at column a_p (the zero terms of the sum change no bit; loop
// rows hold each branch once).  U must be zero-filled.
__global__ void loop_rows_diag_kernel(const double *__restrict__ Rdiag, const int64_t *__restrict__ row_ptr,
                                      const int32_t *__restrict__ branch, const double *__restrict__ sign,
                                      int64_t loops, double *__restrict__ U) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < loops; i += (int64_t)gridDim.x * blockDim.x)
        for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p)
            U[i + (int64_t)branch[p] * loops] = __dmul_rn(sign[p], Rdiag[branch[p]]);
}

// out[i + j loops] = sum_q s_q U[i + b_q loops], q over row j in order, for
// i <= j, mirrored through a shared-memory tile.  Block (32, 8) covers a
// 32 x 32 tile of the upper triangle.
__global__ void __launch_bounds__(256) loop_cols_kernel(const double *__restrict__ U, const int64_t *__restrict__ row_ptr,
                                                        const int32_t *__restrict__ branch,
                                                        const double *__restrict__ sign, int64_t loops,
                                                        double *__restrict__ out) {
    const int64_t I = blockIdx.y, J = blockIdx.x;
    if (I > J) return;
    __shared__ double tile[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const int64_t i = I * 32 + tx, j = J * 32 + r;
        double v = 0.0;
        if (i < loops && j < loops && i <= j) {
            for (int64_t q = row_ptr[j]; q < row_ptr[j + 1]; ++q)
                v = __dadd_rn(v, __dmul_rn(sign[q], U[i + (int64_t)branch[q] * loops]));
            out[i + j * loops] = v;
        }
        tile[r][tx] = v;
    }
    __syncthreads();
    // Mirror: out[row + col*loops] = value(i = col, j = row) for row > col,
    // with row = 32J + tx (coalesced) and col = 32I + r.
    for (int r = ty; r < 32; r += 8) {
        const int64_t row = J * 32 + tx, col = I * 32 + r;
        if (row < loops && col < loops && row > col) out[row + col * loops] = tile[tx][r];
    }
}

}  // namespace

DevFil make_devfil(const fh_filament &f) {
    DevFil d{};
    for (int k = 0; k < 3; ++k) {
        d.centre[k] = (f.start[k] + f.end[k]) * 0.5;
        d.axes[k] = f.dir_length[k];
        d.axes[3 + k] = f.dir_width[k];
        d.axes[6 + k] = f.dir_height[k];
        d.start[k] = f.start[k];
        d.end[k] = f.end[k];
    }
    d.half[0] = 0.5 * f.length;
    d.half[1] = 0.5 * f.width;
    d.half[2] = 0.5 * f.height;
    d.area = f.width * f.height;
    d.width = f.width;
    d.height = f.height;
    d.length = f.length;
    return d;
}

namespace {
bool g_tables_uploaded[64] = {false};
}

namespace {

// The fill pipeline: classification, then the method kernels.  With
// d_pairs == nullptr it evaluates the upper triangle of the n x n matrix
// into d_L (mirrored); with a pair list it evaluates those pairs into
// d_L[k] (pair-list mode: orthogonal pairs are zero).
// Distinct keys of a list of pairs: hash, sort by hash, flag the heads of
// runs of equal keys (full keys compared), max-scan to map every pair to its
// run head, compact the heads.  heads[r] = the list index of distinct key r;
// item_head[t] = the rank of pair t's key.  `alloc(ptr, bytes)` takes
// stream-ordered scratch that the caller releases.
template <class Key, class Alloc>
fh_status distinct_keys(Key, const DevFil *d_fil, const int4 *d_list, int64_t count, Alloc &alloc,
                        cudaStream_t stream, int64_t &n_heads, int64_t *&d_heads, int64_t *&d_item_head,
                        fh_error_info *err) {
    const int sms = 148;
    unsigned long long *d_hash, *d_hash_sorted;
    int64_t *d_idx, *d_order, *d_headpos, *d_headof;
    FHB_CUDA(alloc((void **)&d_hash, 8 * count));
    FHB_CUDA(alloc((void **)&d_hash_sorted, 8 * count));
    FHB_CUDA(alloc((void **)&d_idx, 8 * count));
    FHB_CUDA(alloc((void **)&d_order, 8 * count));
    FHB_CUDA(alloc((void **)&d_headpos, 8 * count));
    FHB_CUDA(alloc((void **)&d_headof, 8 * count));
    const int blocks = (int)std::min<int64_t>((count + 255) / 256, (int64_t)sms * 16);
    key_hash_kernel<Key><<<blocks, 256, 0, stream>>>(d_fil, d_list, count, d_hash, d_idx);
    FHB_CUDA(cudaGetLastError());
    size_t tmp_bytes = 0, tmp2 = 0;
    // 32 bits of the hash are enough to group the keys: a collision only
    // splits a run, because the full keys are compared after the sort.
    FHB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_hash, d_hash_sorted, d_idx, d_order,
                                             (int)count, 0, 32, stream));
    FHB_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tmp2, d_headpos, d_headof, cub::Max(), (int)count, stream));
    void *d_tmp = nullptr;
    FHB_CUDA(alloc(&d_tmp, std::max(tmp_bytes, tmp2)));
    tmp_bytes = std::max(tmp_bytes, tmp2);
    FHB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_hash, d_hash_sorted, d_idx, d_order, (int)count,
                                             0, 32, stream));
    {
        const size_t key_smem = sizeof(unsigned long long) * kHeadsBlock * Key::kWords;
        FHB_CUDA(cudaFuncSetAttribute(key_heads_kernel<Key>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)key_smem));
        const int hb = (int)std::min<int64_t>((count + kHeadsBlock - 2) / (kHeadsBlock - 1), (int64_t)sms * 8);
        key_heads_kernel<Key><<<hb, kHeadsBlock, key_smem, stream>>>(d_fil, d_list, d_hash_sorted, d_order, count,
                                                                    d_headpos);
    }
    FHB_CUDA(cudaGetLastError());
    FHB_CUDA(cub::DeviceScan::InclusiveScan(d_tmp, tmp_bytes, d_headpos, d_headof, cub::Max(), (int)count, stream));
    // Compact the heads on the device: head positions are where
    // headof[t] == t; their ranks (exclusive sum of the flags) number
    // the distinct keys.
    int64_t *d_flag = d_headpos, *d_rank = reinterpret_cast<int64_t *>(d_hash);
    head_flag_kernel<<<blocks, 256, 0, stream>>>(d_headof, count, d_flag);
    FHB_CUDA(cudaGetLastError());
    size_t tmp3 = 0;
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp3, d_flag, d_rank, (int)count, stream));
    if (tmp3 > tmp_bytes) {
        FHB_CUDA(alloc(&d_tmp, tmp3));
        tmp_bytes = tmp3;
    }
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_flag, d_rank, (int)count, stream));
    int64_t last[2];
    FHB_CUDA(cudaMemcpyAsync(&last[0], d_rank + count - 1, 8, cudaMemcpyDeviceToHost, stream));
    FHB_CUDA(cudaMemcpyAsync(&last[1], d_flag + count - 1, 8, cudaMemcpyDeviceToHost, stream));
    FHB_CUDA(cudaStreamSynchronize(stream));
    n_heads = last[0] + last[1];
    FHB_CUDA(alloc((void **)&d_heads, 8 * n_heads));
    FHB_CUDA(alloc((void **)&d_item_head, 8 * count));
    head_compact_kernel<<<blocks, 256, 0, stream>>>(d_order, d_headof, d_rank, d_flag, count, d_heads,
                                                    d_item_head);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

// The Gauss rules and order thresholds in constant memory, once per device.
fh_status upload_quad_tables(fh_error_info *err) {
    int dev = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    static std::mutex init_mu;  // first use on a device may race between host threads
    std::lock_guard<std::mutex> lk(init_mu);
    if (dev < 64 && !g_tables_uploaded[dev]) {
        QuadTables t;
        host_quad_tables(t);
        FHB_CUDA(cudaMemcpyToSymbol(c_quad, &t, sizeof t));
        g_tables_uploaded[dev] = true;
    }
    return FH_OK;
}

fh_status fill_run(const DevFil *d_fil, int64_t n, const int2 *d_pairs, int64_t n_pairs, double *d_L,
                   int8_t *d_methods, cudaStream_t stream, FillStats *stats, fh_error_info *err,
                   const FilTan *d_tan = nullptr, const GradOut *grad = nullptr,
                   const PairMaskDev *mask = nullptr) {
    const bool list = d_pairs != nullptr;
    if (mask && mask->group && list) return fail(err, FH_ERR_INVALID_ARGUMENT, "the pair-list fill takes no mask");
    const PairMaskDev no_mask;
    const PairMaskDev &pm = mask ? *mask : no_mask;
    if (grad && list) return fail(err, FH_ERR_INVALID_ARGUMENT, "the derivative fill has no pair-list mode");
    if (list ? n_pairs == 0 : n == 0) return FH_OK;
    if (n > 2000000000LL / 32) return fail(err, FH_ERR_INVALID_ARGUMENT, "too many filaments for the fill");
    if (list && n_pairs > INT32_MAX) return fail(err, FH_ERR_INVALID_ARGUMENT, "too many pairs for one list fill");
    const int64_t n_arg = list ? 0 : n;  // the method kernels' store mode
    fh_status ts = upload_quad_tables(err);
    if (ts) return ts;
    FillStats local;
    FillStats &st = stats ? *stats : local;
    st = FillStats();
    st.pairs = list ? n_pairs : n * (n + 1) / 2;
    if (list) FHB_CUDA(cudaMemsetAsync(d_L, 0, sizeof(double) * n_pairs, stream));
    cudaEvent_t ev[6];
    for (auto &e : ev) FHB_CUDA(cudaEventCreate(&e));
    // Scratch comes from the stream-ordered memory cache: no device-wide
    // synchronization per buffer, released after the last kernel that reads
    // it.
    struct Guard {
        std::vector<void *> ptrs;
        cudaEvent_t *ev;
        cudaStream_t s;
        ~Guard() {
            for (void *p : ptrs) cache_free(p, s);
            for (int k = 0; k < 6; ++k) cudaEventDestroy(ev[k]);
        }
    } guard{{}, ev, stream};
    auto alloc = [&](void **p, size_t bytes) -> cudaError_t {
        cudaError_t e = cache_alloc(p, bytes, stream);
        if (e == cudaSuccess) guard.ptrs.push_back(*p);
        return e;
    };
    unsigned long long *d_counts = nullptr, *d_cursor = nullptr;
    DevError *d_err = nullptr;
    FHB_CUDA(alloc((void **)&d_counts, sizeof(unsigned long long) * kCats * 2 + sizeof(DevError) + 64));
    d_cursor = d_counts + kCats;
    d_err = reinterpret_cast<DevError *>(d_counts + 2 * kCats);
    FHB_CUDA(cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * kCats * 2, stream));
    FHB_CUDA(cudaMemsetAsync(d_err, 0xff, sizeof(unsigned long long), stream));
    FHB_CUDA(cudaMemsetAsync(&d_err->code, 0, sizeof(int), stream));
    const int T = (int)((n + 31) / 32);
    dim3 grid(T, T), block(32, 8);
    // The counting pass keeps every pair's classification for the writing
    // pass (8 bytes per pair of the upper tiles) when the memory is there;
    // otherwise the writing pass classifies again.
    uint2 *d_rec = nullptr;
    if (!list) {
        const size_t rec_bytes = sizeof(uint2) * 1024 * ((size_t)T * (T + 1) / 2);
        if (alloc((void **)&d_rec, rec_bytes) != cudaSuccess) {
            cudaGetLastError();
            d_rec = nullptr;
        }
    }
    const unsigned list_blocks = (unsigned)((n_pairs + 255) / 256);
    FHB_CUDA(cudaEventRecord(ev[0], stream));
    if (list)
        classify_list_kernel<false><<<list_blocks, 256, 0, stream>>>(d_fil, d_pairs, n_pairs, d_counts, nullptr,
                                                                      nullptr);
    else
        classify_kernel<false><<<grid, block, 0, stream>>>(d_fil, (int)n, d_counts, nullptr, nullptr, pm, d_rec);
    FHB_CUDA(cudaGetLastError());
    unsigned long long counts[kCats];
    FHB_CUDA(cudaMemcpyAsync(counts, d_counts, sizeof counts, cudaMemcpyDeviceToHost, stream));
    FHB_CUDA(cudaStreamSynchronize(stream));
    unsigned long long offsets[kCats + 1];
    offsets[0] = 0;
    for (int c = 0; c < kCats; ++c) offsets[c + 1] = offsets[c] + counts[c];
    const unsigned long long total_items = offsets[kCats];
    int4 *d_items = nullptr;
    FHB_CUDA(alloc((void **)&d_items, sizeof(int4) * total_items));
    FHB_CUDA(cudaMemcpyAsync(d_cursor, offsets, sizeof(unsigned long long) * kCats, cudaMemcpyHostToDevice, stream));
    if (list)
        classify_list_kernel<true><<<list_blocks, 256, 0, stream>>>(d_fil, d_pairs, n_pairs, nullptr, d_cursor,
                                                                     d_items);
    else if (d_rec)
        classify_scatter_kernel<<<grid, block, 0, stream>>>(d_rec, d_cursor, d_items);
    else
        classify_kernel<true><<<grid, block, 0, stream>>>(d_fil, (int)n, nullptr, d_cursor, d_items, pm, nullptr);
    FHB_CUDA(cudaGetLastError());
    FHB_CUDA(cudaEventRecord(ev[1], stream));
    const int sms = 148;
    auto distinct = [&](auto key, const int4 *d_list, int64_t count, int64_t &n_heads, int64_t *&d_heads,
                        int64_t *&d_item_head) -> fh_status {
        return distinct_keys(key, d_fil, d_list, count, alloc, stream, n_heads, d_heads, d_item_head, err);
    };
    // Point quadrature over all buckets (contiguous, cost ascending).
    const int64_t n_point = (int64_t)offsets[kPointBuckets];
    st.point = n_point;
    for (int c = 0; c < kPointBuckets; ++c) st.point_evaluations += (double)counts[c] * (1.5 * (double)(1ull << c));
    if (n_point) {
        int blocks = (int)std::min<int64_t>((n_point + 127) / 128, (int64_t)sms * 64);
        if (grad) {
            point_grad_kernel<<<blocks, 128, 0, stream>>>(d_fil, d_tan, d_items, n_point, *grad, n, d_err);
        } else if (n_point > INT32_MAX) {  // beyond the sort's 32-bit counts: every pair evaluated
            point_kernel<<<blocks, 128, 0, stream>>>(d_fil, d_items, n_point, d_L, d_methods, n_arg, d_err);
        } else {
            // Pairs that are the same geometry up to a translation share one
            // evaluation (PointKey).
            int64_t n_heads = 0, *d_heads = nullptr, *d_item_head = nullptr;
            fh_status ds = distinct(PointKey{}, d_items, n_point, n_heads, d_heads, d_item_head);
            if (ds) return ds;
            st.unique_point = n_heads;
            double *d_pvalues;
            int64_t *d_rank_in, *d_heads_sorted, *d_rank_sorted;
            FHB_CUDA(alloc((void **)&d_pvalues, 8 * n_heads));
            FHB_CUDA(alloc((void **)&d_rank_in, 8 * n_heads));
            FHB_CUDA(alloc((void **)&d_heads_sorted, 8 * n_heads));
            FHB_CUDA(alloc((void **)&d_rank_sorted, 8 * n_heads));
            // Heads in work-list order (cost ascending), so a warp's pairs
            // have similar loop counts; each value goes to its key's rank.
            const int iblocks = (int)std::min<int64_t>((n_heads + 255) / 256, (int64_t)sms * 16);
            iota_kernel<<<iblocks, 256, 0, stream>>>(d_rank_in, n_heads);
            FHB_CUDA(cudaGetLastError());
            size_t sort_bytes = 0;
            const int bits = 64 - __builtin_clzll((unsigned long long)std::max<int64_t>(1, n_point));
            FHB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, d_heads, d_heads_sorted, d_rank_in,
                                                     d_rank_sorted, (int)n_heads, 0, bits, stream));
            void *d_sort_tmp = nullptr;
            FHB_CUDA(alloc(&d_sort_tmp, std::max<size_t>(sort_bytes, 16)));
            FHB_CUDA(cub::DeviceRadixSort::SortPairs(d_sort_tmp, sort_bytes, d_heads, d_heads_sorted, d_rank_in,
                                                     d_rank_sorted, (int)n_heads, 0, bits, stream));
            const int hblocks = (int)std::min<int64_t>((n_heads + 127) / 128, (int64_t)sms * 64);
            point_heads_ordered_kernel<<<hblocks, 128, 0, stream>>>(d_fil, d_items, d_heads_sorted, d_rank_sorted,
                                                                    n_heads, d_pvalues);
            FHB_CUDA(cudaGetLastError());
            const int sblocks = (int)std::min<int64_t>((n_point + 255) / 256, (int64_t)sms * 16);
            point_scatter_kernel<<<sblocks, 256, 0, stream>>>(d_items, d_item_head, d_pvalues, n_point, d_L, d_methods,
                                                             n_arg, d_err);
        }
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(cudaEventRecord(ev[2], stream));
    // Aligned pairs: closed form, then the quadrature for the rest.
    const int64_t n_aligned = (int64_t)counts[kCatAligned];
    const int4 *d_aligned = d_items + offsets[kCatAligned];
    int4 *d_quad = nullptr;
    unsigned long long *d_qcount = d_cursor + kCatAligned;  // reuse the slot as a counter
    FHB_CUDA(cudaMemsetAsync(d_qcount, 0, sizeof(unsigned long long), stream));
    int64_t n_quad = 0;
    if (n_aligned) {
        FHB_CUDA(alloc((void **)&d_quad, sizeof(int4) * n_aligned));
        int blocks = (int)std::min<int64_t>((n_aligned + 127) / 128, (int64_t)sms * 32);
        if (grad)
            closed_form_grad_kernel<<<blocks, 128, 0, stream>>>(d_fil, d_tan, d_aligned, n_aligned, *grad, n, d_quad,
                                                                d_qcount, d_err);
        else
            closed_form_kernel<<<blocks, 128, 0, stream>>>(d_fil, d_aligned, n_aligned, d_L, d_methods, n_arg, d_quad,
                                                           d_qcount, d_err);
        FHB_CUDA(cudaGetLastError());
        unsigned long long q = 0;
        FHB_CUDA(cudaMemcpyAsync(&q, d_qcount, sizeof q, cudaMemcpyDeviceToHost, stream));
        FHB_CUDA(cudaStreamSynchronize(stream));
        n_quad = (int64_t)q;
    }
    FHB_CUDA(cudaEventRecord(ev[3], stream));
    st.closed_form = n_aligned - n_quad;
    st.aligned_quadrature = n_quad;
    if (n_quad) {
        int64_t n_heads = 0, *d_heads = nullptr, *d_item_head = nullptr;
        fh_status ds = distinct(AlignedKey{}, d_quad, n_quad, n_heads, d_heads, d_item_head);
        if (ds) return ds;
        st.unique_aligned = n_heads;
        double *d_values;
        FHB_CUDA(alloc((void **)&d_values, (grad ? 56 : 8) * n_heads));
        const int blocks = (int)std::min<int64_t>((n_quad + 255) / 256, (int64_t)sms * 16);
        int qblocks = (int)std::min<int64_t>(n_heads, (int64_t)sms * 16);
        if (grad) {
            aligned_quadrature_kernel<1><<<qblocks, kQuadThreads, 0, stream>>>(d_fil, d_quad, d_heads, n_heads,
                                                                                 d_values);
            FHB_CUDA(cudaGetLastError());
            aligned_grad_scatter_kernel<<<blocks, 256, 0, stream>>>(d_fil, d_tan, d_quad, d_item_head, d_values, n_quad,
                                                                    *grad, n, d_err);
        } else {
            aligned_quadrature_kernel<0><<<qblocks, kQuadThreads, 0, stream>>>(d_fil, d_quad, d_heads, n_heads,
                                                                                  d_values);
            FHB_CUDA(cudaGetLastError());
            aligned_scatter_kernel<<<blocks, 256, 0, stream>>>(d_fil, d_quad, d_item_head, d_values, n_quad, d_L,
                                                               d_methods, n_arg, d_err);
        }
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(cudaEventRecord(ev[4], stream));
    const int64_t n_sampled = (int64_t)counts[kCatSampled];
    st.sampled = n_sampled;
    if (n_sampled && grad)
        return fail(err, FH_ERR_UNSUPPORTED,
                    std::to_string(n_sampled) +
                        " filament pairs are evaluated by sampled filaments (parallel bars with rotated "
                        "cross-sections, or skew bars); their derivatives are not provided");
    if (n_sampled) {
        int blocks = (int)std::min<int64_t>((n_sampled * 32 + 127) / 128, (int64_t)sms * 32);
        sampled_kernel<<<blocks, 128, 0, stream>>>(d_fil, d_items + offsets[kCatSampled], n_sampled, d_L, d_methods,
                                                   n_arg, d_err);
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(cudaEventRecord(ev[5], stream));
    DevError h_err;
    FHB_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof h_err, cudaMemcpyDeviceToHost, stream));
    FHB_CUDA(cudaStreamSynchronize(stream));
    st.truncated = pm.group ? pm.dropped : 0;
    st.orthogonal = st.pairs - (int64_t)total_items - st.truncated;
    cudaEventElapsedTime(&st.ms_classify, ev[0], ev[1]);
    cudaEventElapsedTime(&st.ms_point, ev[1], ev[2]);
    cudaEventElapsedTime(&st.ms_aligned, ev[2], ev[3]);
    cudaEventElapsedTime(&st.ms_quadrature, ev[3], ev[4]);
    cudaEventElapsedTime(&st.ms_sampled, ev[4], ev[5]);
    if (h_err.key != ~0ull) {
        int64_t i = (int64_t)(h_err.key >> 32), j = (int64_t)(h_err.key & 0xffffffffull);
        if (h_err.code == FH_ERR_KERNEL_COINCIDENT)
            return fail(err, FH_ERR_KERNEL_COINCIDENT,
                        "overlapping parallel filaments " + std::to_string(i) + " and " + std::to_string(j) +
                            " have misaligned cross-sections and coincident sample lines",
                        i, j);
        return fail(err, FH_ERR_KERNEL_NOT_FINITE,
                    "partial inductance of filaments " + std::to_string(i) + " and " + std::to_string(j) +
                        " is not finite",
                    i, j);
    }
    return FH_OK;
}

}  // namespace

fh_status device_fill(const DevFil *d_fil, int64_t n, double *d_L, int8_t *d_methods, cudaStream_t stream,
                      FillStats *stats, fh_error_info *err, const PairMaskDev *mask) {
    return fill_run(d_fil, n, nullptr, 0, d_L, d_methods, stream, stats, err, nullptr, nullptr, mask);
}

fh_status device_fill_pairs(const DevFil *d_fil, int64_t n, const int2 *d_pairs, int64_t n_pairs, double *d_out,
                            cudaStream_t stream, FillStats *stats, fh_error_info *err) {
    return fill_run(d_fil, n, d_pairs, n_pairs, d_out, nullptr, stream, stats, err);
}

fh_status device_fill_grad(const DevFil *d_fil, const FilTan *d_tan, int64_t n, GradOut out, cudaStream_t stream,
                           FillStats *stats, fh_error_info *err, const PairMaskDev *mask) {
    if (!d_tan || !out.Dw || !out.Dh) return fail(err, FH_ERR_INVALID_ARGUMENT, "null derivative-fill argument");
    return fill_run(d_fil, n, nullptr, 0, nullptr, nullptr, stream, stats, err, d_tan, &out, mask);
}

fh_status device_fill_coord(const DevFil *d_fil, const int32_t *d_seg, const uint8_t *d_move, int64_t n,
                            CoordOut out, cudaStream_t stream, FillStats *stats, fh_error_info *err,
                            const PairMaskDev *mask) {
    if (!d_seg || !d_move || !out.Dl || !out.Dp || !out.Ds || !out.Dr)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "null coordinate-fill argument");
    if (n == 0) return FH_OK;
    if (n > 2000000000LL / 32) return fail(err, FH_ERR_INVALID_ARGUMENT, "too many filaments for the fill");
    const PairMaskDev no_mask;
    const PairMaskDev &pm = mask ? *mask : no_mask;
    fh_status ts = upload_quad_tables(err);
    if (ts) return ts;
    FillStats local;
    FillStats &st = stats ? *stats : local;
    st = FillStats();
    st.pairs = n * (n + 1) / 2;
    struct Guard {
        std::vector<void *> ptrs;
        cudaStream_t s;
        ~Guard() {
            for (void *p : ptrs) cache_free(p, s);
        }
    } guard{{}, stream};
    auto alloc = [&](void **p, size_t bytes) -> cudaError_t {
        cudaError_t e = cache_alloc(p, std::max<size_t>(bytes, 16), stream);
        if (e == cudaSuccess) guard.ptrs.push_back(*p);
        return e;
    };
    unsigned long long *d_counts = nullptr;
    FHB_CUDA(alloc((void **)&d_counts, sizeof(unsigned long long) * (2 * kCoordCats + 2) + sizeof(DevError) + 64));
    unsigned long long *d_cursor = d_counts + kCoordCats, *d_qcount = d_counts + 2 * kCoordCats;
    DevError *d_err = reinterpret_cast<DevError *>(d_counts + 2 * kCoordCats + 2);
    FHB_CUDA(cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * (2 * kCoordCats + 2), stream));
    FHB_CUDA(cudaMemsetAsync(d_err, 0xff, sizeof(unsigned long long), stream));
    FHB_CUDA(cudaMemsetAsync(&d_err->code, 0, sizeof(int), stream));
    const int T = (int)((n + 31) / 32);
    const dim3 grid(T, T), block(32, 8);
    coord_classify_kernel<false><<<grid, block, 0, stream>>>(d_fil, d_seg, d_move, (int)n, d_counts, nullptr, nullptr,
                                                             pm, d_err);
    FHB_CUDA(cudaGetLastError());
    unsigned long long counts[kCoordCats];
    DevError h_err;
    FHB_CUDA(cudaMemcpyAsync(counts, d_counts, sizeof counts, cudaMemcpyDeviceToHost, stream));
    FHB_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof h_err, cudaMemcpyDeviceToHost, stream));
    FHB_CUDA(cudaStreamSynchronize(stream));
    if (h_err.key != ~0ull) {
        const int64_t i = (int64_t)(h_err.key >> 32), j = (int64_t)(h_err.key & 0xffffffffull);
        return fail(err, FH_ERR_UNSUPPORTED,
                    "filaments " + std::to_string(i) + " and " + std::to_string(j) +
                        " have no coordinate derivative here: a pair evaluated by sampled filaments (skew bars "
                        "or rotated cross-sections), a segment off the xy plane, or parallel filaments of two "
                        "segments whose cross-sections meet when projected along their length",
                    i, j);
    }
    unsigned long long offsets[kCoordCats + 1];
    offsets[0] = 0;
    for (int c = 0; c < kCoordCats; ++c) offsets[c + 1] = offsets[c] + counts[c];
    int4 *d_items = nullptr, *d_quad = nullptr;
    FHB_CUDA(alloc((void **)&d_items, sizeof(int4) * offsets[kCoordCats]));
    FHB_CUDA(cudaMemcpyAsync(d_cursor, offsets, sizeof(unsigned long long) * kCoordCats, cudaMemcpyHostToDevice,
                             stream));
    coord_classify_kernel<true><<<grid, block, 0, stream>>>(d_fil, d_seg, d_move, (int)n, nullptr, d_cursor, d_items,
                                                            pm, d_err);
    FHB_CUDA(cudaGetLastError());
    const int sms = 148;
    const int64_t n_point = (int64_t)counts[kCoordCatPoint];
    st.point = n_point;
    if (n_point) {
        const int blocks = (int)std::min<int64_t>((n_point + 127) / 128, (int64_t)sms * 64);
        point_coord_kernel<<<blocks, 128, 0, stream>>>(d_fil, d_items + offsets[kCoordCatPoint], n_point, out, n,
                                                       d_err);
        FHB_CUDA(cudaGetLastError());
    }
    // Quadrature list: the pairs of different segments, then whatever the
    // closed forms reject.
    const int64_t n_same = (int64_t)counts[kCoordCatSame], n_diff = (int64_t)counts[kCoordCatDiff];
    const int64_t n_ortho = (int64_t)counts[kCoordCatOrtho];
    FHB_CUDA(alloc((void **)&d_quad, sizeof(int4) * (size_t)(n_same + n_diff + n_ortho)));
    if (n_diff)
        FHB_CUDA(cudaMemcpyAsync(d_quad, d_items + offsets[kCoordCatDiff], sizeof(int4) * n_diff,
                                 cudaMemcpyDeviceToDevice, stream));
    const unsigned long long start = (unsigned long long)n_diff;
    FHB_CUDA(cudaMemcpyAsync(d_qcount, &start, sizeof start, cudaMemcpyHostToDevice, stream));
    if (n_same) {
        const int blocks = (int)std::min<int64_t>((n_same + 127) / 128, (int64_t)sms * 32);
        closed_form_coord_kernel<false><<<blocks, 128, 0, stream>>>(d_fil, d_items + offsets[kCoordCatSame], n_same,
                                                                    out, n, d_quad, d_qcount, d_err);
        FHB_CUDA(cudaGetLastError());
    }
    if (n_ortho) {
        const int blocks = (int)std::min<int64_t>((n_ortho + 127) / 128, (int64_t)sms * 32);
        closed_form_coord_kernel<true><<<blocks, 128, 0, stream>>>(d_fil, d_items + offsets[kCoordCatOrtho], n_ortho,
                                                                   out, n, d_quad, d_qcount, d_err);
        FHB_CUDA(cudaGetLastError());
    }
    unsigned long long q = 0;
    FHB_CUDA(cudaMemcpyAsync(&q, d_qcount, sizeof q, cudaMemcpyDeviceToHost, stream));
    FHB_CUDA(cudaStreamSynchronize(stream));
    const int64_t n_quad = (int64_t)q;
    st.closed_form = n_same + n_ortho - (n_quad - n_diff);
    st.aligned_quadrature = n_quad;
    if (n_quad) {
        int64_t n_heads = 0, *d_heads = nullptr, *d_item_head = nullptr;
        fh_status ds = distinct_keys(CoordKey{}, d_fil, d_quad, n_quad, alloc, stream, n_heads, d_heads, d_item_head,
                                     err);
        if (ds) return ds;
        st.unique_aligned = n_heads;
        double *d_values = nullptr;
        FHB_CUDA(alloc((void **)&d_values, 64 * (size_t)n_heads));
        unsigned long long *d_keys = nullptr;
        FHB_CUDA(alloc((void **)&d_keys, sizeof(unsigned long long)));
        FHB_CUDA(cudaMemsetAsync(d_keys, 0, sizeof(unsigned long long), stream));
        const int qblocks = (int)std::min<int64_t>(n_heads, (int64_t)sms * 16);
        aligned_quadrature_kernel<2><<<qblocks, kQuadThreads, 0, stream>>>(d_fil, d_quad, d_heads, n_heads, d_values,
                                                                          d_keys);
        FHB_CUDA(cudaGetLastError());
        const int blocks = (int)std::min<int64_t>((n_quad + 255) / 256, (int64_t)sms * 16);
        coord_quad_scatter_kernel<<<blocks, 256, 0, stream>>>(d_fil, d_quad, d_item_head, d_values, n_quad, out, n,
                                                              d_err);
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof h_err, cudaMemcpyDeviceToHost, stream));
    FHB_CUDA(cudaStreamSynchronize(stream));
    if (h_err.key != ~0ull) {
        const int64_t i = (int64_t)(h_err.key >> 32), j = (int64_t)(h_err.key & 0xffffffffull);
        return fail(err, FH_ERR_KERNEL_NOT_FINITE,
                    "coordinate derivative of the partial inductance of filaments " + std::to_string(i) + " and " +
                        std::to_string(j) + " is not finite",
                    i, j);
    }
    return FH_OK;
}

fh_status device_congruence(const double *d_L, const double *d_R, int64_t n, const int64_t *d_row_ptr,
                            const int32_t *d_branch, const double *d_sign, int64_t loops, const int64_t *h_row_ptr,
                            double *d_Lm, double *d_Rm, cudaStream_t stream, fh_error_info *err) {
    if (loops == 0) return FH_OK;
    std::vector<int64_t> long_rows;
    for (int64_t i = 0; i < loops; ++i)
        if (h_row_ptr[i + 1] - h_row_ptr[i] > kShortRow) long_rows.push_back(i);
    double *d_U = nullptr;
    const size_t ubytes = sizeof(double) * (size_t)loops * (size_t)n;
    if (cache_alloc((void **)&d_U, ubytes, stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(err, FH_ERR_OUT_OF_MEMORY,
                    "device allocation of " + std::to_string(ubytes) + " bytes for the congruence failed");
    }
    struct Free {
        double *p;
        cudaStream_t s;
        ~Free() { cache_free(p, s); }
    } free_u{d_U, stream};
    const int T = (int)((loops + 31) / 32);
    const dim3 rows_grid((unsigned)((loops + 127) / 128), (unsigned)((n + kRowsCols - 1) / kRowsCols));
    loop_rows_kernel<<<rows_grid, 128, 0, stream>>>(d_L, n, d_row_ptr, d_branch, d_sign, loops, d_U);
    FHB_CUDA(cudaGetLastError());
    int64_t *d_long = nullptr;
    if (!long_rows.empty()) {
        if (cache_alloc((void **)&d_long, 8 * long_rows.size(), stream) != cudaSuccess) {
            cudaGetLastError();
            return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation for the congruence failed");
        }
        FHB_CUDA(cudaMemcpyAsync(d_long, long_rows.data(), 8 * long_rows.size(), cudaMemcpyHostToDevice, stream));
        const unsigned bx = (unsigned)std::min<int64_t>((n + 255) / 256, 64);
        loop_rows_long_kernel<<<dim3(bx, (unsigned)long_rows.size()), 256, 0, stream>>>(
            d_L, n, d_row_ptr, d_branch, d_sign, loops, d_long, d_U);
        cudaError_t le = cudaGetLastError();
        cache_free(d_long, stream);
        if (le != cudaSuccess) return fail(err, FH_ERR_CUDA, std::string("congruence: ") + cudaGetErrorString(le));
    }
    loop_cols_kernel<<<dim3(T, T), dim3(32, 8), 0, stream>>>(d_U, d_row_ptr, d_branch, d_sign, loops, d_Lm);
    FHB_CUDA(cudaGetLastError());
    FHB_CUDA(cudaMemsetAsync(d_U, 0, ubytes, stream));
    loop_rows_diag_kernel<<<(unsigned)std::min<int64_t>((loops + 255) / 256, 148 * 8), 256, 0, stream>>>(
        d_R, d_row_ptr, d_branch, d_sign, loops, d_U);
    FHB_CUDA(cudaGetLastError());
    loop_cols_kernel<<<dim3(T, T), dim3(32, 8), 0, stream>>>(d_U, d_row_ptr, d_branch, d_sign, loops, d_Rm);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

}  // namespace fhb
