// Dispatch-critical FP64 geometry on the device: dot and cross products,
// norms and the separating-axis gap of two bars, in non-contracted __d*_rn
// operations in the reference's order (neumann.rs:57-122), so that decisions
// taken on them (method dispatch, near pairs) match the reference's bit for
// bit.  Shared by the fill (fh_fill.cu) and the near-pair search (fh_near.cu).
#pragma once

#include "fh_device.cuh"

namespace fhb {

__device__ __forceinline__ double ndot(const double *a, const double *b) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}
__device__ __forceinline__ void ncross(const double *a, const double *b, double *o) {
    o[0] = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
    o[1] = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
    o[2] = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
}
__device__ __forceinline__ double nnorm(const double *a) { return __dsqrt_rn(ndot(a, a)); }
__device__ __forceinline__ double rmax(double a, double b) {
    return isnan(a) ? b : (isnan(b) ? a : (a > b ? a : b));
}
__device__ __forceinline__ double rmin(double a, double b) {
    return isnan(a) ? b : (isnan(b) ? a : (a < b ? a : b));
}
__device__ __forceinline__ double signum(double x) { return isnan(x) ? x : (signbit(x) ? -1.0 : 1.0); }

__device__ __forceinline__ double circumradius(const DevFil &f) {
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(f.half[0], f.half[0]), __dmul_rn(f.half[1], f.half[1])),
                                __dmul_rn(f.half[2], f.half[2])));
}
__device__ __forceinline__ double projected_half_extent(const DevFil &f, const double *n) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s = __dadd_rn(s, __dmul_rn(f.half[k], fabs(ndot(n, f.axes + 3 * k))));
    return s;
}

// neumann::separation, neumann.rs:97-122.
__device__ inline double separation(const DevFil &a, const DevFil &b) {
    double delta[3] = {__dsub_rn(b.centre[0], a.centre[0]), __dsub_rn(b.centre[1], a.centre[1]),
                       __dsub_rn(b.centre[2], a.centre[2])};
    double distance = nnorm(delta);
    double reach = __dadd_rn(circumradius(a), circumradius(b));
    if (distance > __dmul_rn(8.0, reach)) return __dsub_rn(distance, reach);
    double best = -INFINITY;
    auto consider = [&](const double *n) {
        double gap = __dsub_rn(__dsub_rn(fabs(ndot(n, delta)), projected_half_extent(a, n)),
                               projected_half_extent(b, n));
        best = rmax(best, gap);
    };
    for (int k = 0; k < 3; ++k) {
        consider(a.axes + 3 * k);
        consider(b.axes + 3 * k);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double c[3];
            ncross(a.axes + 3 * i, b.axes + 3 * j, c);
            double nn = nnorm(c);
            if (nn > 1e-9) {
                double u[3] = {__ddiv_rn(c[0], nn), __ddiv_rn(c[1], nn), __ddiv_rn(c[2], nn)};
                consider(u);
            }
        }
    return best;
}

}  // namespace fhb
