// Device-side shared definitions: filament records in HBM, CUDA error
// plumbing, non-contracted FP64 helpers for dispatch-critical arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "fh_internal.h"

namespace fhb {

// A filament as the fill kernels read it: 32 doubles (256 B), all derived
// quantities computed once on the host in the reference's operation order.
struct __align__(16) DevFil {
    double centre[3];   // (start + end) * 0.5
    double axes[9];     // length, width, height unit vectors
    double half[3];     // 0.5 * length, 0.5 * width, 0.5 * height
    double area;        // width * height
    double start[3];
    double end[3];
    double width, height;
    double length;
    double pad[7];
};
static_assert(sizeof(DevFil) == 256, "DevFil is 256 bytes");

DevFil make_devfil(const fh_filament &f);

// Gauss-Legendre rules 1..kMaxRule and the order thresholds, uploaded once.
constexpr int kMaxRule = 17;
struct QuadTables {
    double nodes[kMaxRule + 1][kMaxRule];
    double weights[kMaxRule + 1][kMaxRule];
    double point_thresholds[16];   // tolerance 1e-8, orders 1..16
    double sample_thresholds[8];   // tolerance 1e-6, orders 1..8
};
void host_quad_tables(QuadTables &t);

#define FHB_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return ::fhb::fail(err, FH_ERR_CUDA,                                         \
                               std::string(#call " failed: ") + cudaGetErrorString(e_)); \
    } while (0)

fh_status ensure_device(fh_error_info *err);

// Process-wide cache of device memory (fh_mem.cu): stream-ordered
// allocations from a per-device pool that keeps freed memory for reuse.
cudaError_t cache_alloc(void **p, size_t bytes, cudaStream_t s);
void cache_free(void *p, cudaStream_t s);
// Memory held by the cache and not in use (counted as available when sizing
// sweep batches).
size_t cache_idle_bytes();

// Device-event profiler of kernel classes (enabled through fh_profile_enable).
// prof_begin/prof_end bracket one launch on `s`; `work` is its algorithmic
// flop (or byte) count.
bool prof_on();
void prof_begin(cudaStream_t s, int cls);
void prof_end(cudaStream_t s, int cls, double work);
// While alive, the profiler records nothing on this thread (it would create
// CUDA events); used by entry points that promise to acquire no resources.
struct ProfSuppress {
    ProfSuppress();
    ~ProfSuppress();
};

// Fill the n x n column-major L on the device (d_L must be zero-filled by the
// caller).  `d_methods` optional (n*n int8).  `stream` orders the work.
struct FillStats {
    int64_t pairs = 0, orthogonal = 0, point = 0, closed_form = 0, aligned_quadrature = 0, sampled = 0;
    int64_t truncated = 0;
    int64_t unique_aligned = 0;
    int64_t unique_point = 0;  // distinct point-quadrature keys (value fill)
    double point_evaluations = 0.0;
    float ms_classify = 0, ms_point = 0, ms_aligned = 0, ms_quadrature = 0, ms_sampled = 0;
};
// A coupling's pair mask on the device (PairMask, inductance/batch.rs:37-117):
// the group of every filament and the groups x groups table of kept pairs.
// Pairs of uncoupled groups are never evaluated and stay zero.
struct PairMaskDev {
    const int32_t *group = nullptr;
    const uint8_t *coupled = nullptr;
    int32_t groups = 0;
    int64_t dropped = 0;  // pairs the mask drops (for the statistics)
};
fh_status device_fill(const DevFil *d_fil, int64_t n, double *d_L, int8_t *d_methods, cudaStream_t stream,
                      FillStats *stats, fh_error_info *err, const PairMaskDev *mask = nullptr);
// The same evaluation for an explicit list of filament pairs: d_out[k] =
// L(pairs[k].x, pairs[k].y), zero for orthogonal pairs.
fh_status device_fill_pairs(const DevFil *d_fil, int64_t n, const int2 *d_pairs, int64_t n_pairs, double *d_out,
                            cudaStream_t stream, FillStats *stats, fh_error_info *err);

// How a filament moves with the cross-section of its segment: d centre /
// d width = sw * width axis, d (own width) / d width = gw, and likewise sh,
// gh for the segment's thickness (the discretization's counts and grading
// ratios held fixed).
struct FilTan {
    double sw, sh, gw, gh;
};
// Outputs of the derivative fill: n x n column-major, D[a + b n] = the
// derivative of L_ab with respect to the width (Dw) or thickness (Dh) of the
// segment of filament a, filament b held fixed.
struct GradOut {
    double *Dw, *Dh;
};
// Both matrices must be zero-filled by the caller (orthogonal pairs stay 0).
// Pairs evaluated by sampled filaments (non-aligned parallel or skew bars)
// have no derivative here: FH_ERR_UNSUPPORTED.
fh_status device_fill_grad(const DevFil *d_fil, const FilTan *d_tan, int64_t n, GradOut out, cudaStream_t stream,
                           FillStats *stats, fh_error_info *err, const PairMaskDev *mask = nullptr);

// Outputs of the coordinate derivative fill: n x n column-major,
// D[a + b n] = the derivative of L_ab with respect to a coordinate of
// filament a (b held fixed): translation of its centre along its length axis
// (Dl) and along z x l normalized (Dp), stretch of its length about its
// centre (Ds), rotation about the z axis through its centre (Dr).  Pairs of
// one segment (equal d_seg) get Ds only; the diagonal of Ds holds half of
// dL_aa / d length.
struct CoordOut {
    double *Dl, *Dp, *Ds, *Dr;
};
// Pairs with a moving filament (d_move[i] != 0); the four matrices must be
// zero-filled by the caller.  Pairs evaluated by sampled filaments, and
// parallel pairs of different segments whose cross-sections meet when
// projected along their length: FH_ERR_UNSUPPORTED.
fh_status device_fill_coord(const DevFil *d_fil, const int32_t *d_seg, const uint8_t *d_move, int64_t n,
                            CoordOut out, cudaStream_t stream, FillStats *stats, fh_error_info *err,
                            const PairMaskDev *mask = nullptr);

// y = D_w I and D_h I for p complex vectors I (n x p, column q at 2 q n):
// y holds 2 x p columns (D_w's products first).  d_part is scratch of
// gradient_part_elems(n, p) doubles.
fh_status gradient_products(const double *d_Dw, const double *d_Dh, int64_t n, const double *d_I, int p, double *d_y,
                            double *d_part, cudaStream_t stream, fh_error_info *err);
size_t gradient_part_elems(int64_t n, int p);

// Branch currents, |J|, power per filament and per-segment sums / peaks for
// `count` frequencies from X = Z_ee^-1 Z_ep (count x p x m complex) and the
// excitation d_ip (p complex); with `applied`, d_x holds Z_ee^-1 Z_ep I_p
// (count x m complex) instead.  The transposed loop basis lists, per branch,
// (loop, sign) in increasing loop order; d_whr holds (w, h, R) per filament,
// d_first the first filament of each segment (nseg + 1).  Outputs are count x
// n (complex / real) and count x nseg.
fh_status launch_currents(const double *d_x, const double *d_ip, int64_t m, int p, bool applied, int64_t n,
                          int count, const int64_t *d_col_ptr, const int32_t *d_col_loop, const double *d_col_sign,
                          const double *d_whr, const int64_t *d_first, int64_t nseg, double *d_ib, double *d_dens,
                          double *d_pow, double *d_seg_cur, double *d_seg_pow, double *d_seg_peak,
                          int64_t *d_seg_idx, cudaStream_t s, fh_error_info *err);

// R_m = M diag(R) M^T and L_m = M L M^T (loops x loops, column-major), upper
// triangle evaluated in the reference's order and mirrored.
// h_row_ptr: the same row pointers on the host (long rows take their own kernel).
fh_status device_congruence(const double *d_L, const double *d_R, int64_t n, const int64_t *d_row_ptr,
                            const int32_t *d_branch, const double *d_sign, int64_t loops, const int64_t *h_row_ptr,
                            double *d_Lm, double *d_Rm, cudaStream_t stream, fh_error_info *err);

}  // namespace fhb
