// Internal declarations of the precorrected-FFT operator (pfft/mod.rs,
// grid.rs, fft.rs, near.rs of the reference).  The host chooses the grid
// (fh_pfft_setup.cpp); the near-pair search (fh_near.cu), the projections and
// precorrection (fh_pfft_setup.cu), the exact near pairs (the device fill)
// and the products (fh_pfft.cu) run on the device.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "fh_fftconv.h"
#include "fh_internal.h"

namespace fhb {

struct DevFil;

// Uniform grid (grid.rs:44-95): point (i, j, k) at origin + h (i, j, k),
// linear index (i dims[1] + j) dims[2] + k.
struct PfftGrid {
    double origin[3] = {0, 0, 0};
    double spacing = 0;
    int64_t dims[3] = {0, 0, 0};
    int stencil = 0;  // interpolation points per axis, order + 1
    int64_t len() const { return dims[0] * dims[1] * dims[2]; }
};

// The host part of the set-up: the grid, the near-field radius and the
// filament directions.
struct PfftSetup {
    int64_t n = 0;
    PfftGrid grid;
    int64_t padded[3] = {0, 0, 0};
    double radius = 0.0;
    std::vector<double> directions;  // 3 n, unit length vectors
    std::vector<int> components;     // Cartesian components some direction carries
};

// The near pairs on the device (fh_near.cu): for each filament i the
// filaments j >= i (i included) whose separating-axis gap is below the radius
// and whose directions are not orthogonal, as CSR rows ascending in j
// (off[n + 1], pairs (i, j) and their direction cosines).  Memory from the
// device cache; release with near_pairs_free.
struct NearPairs {
    int64_t n = 0, count = 0;
    int64_t *off = nullptr;
    int2 *pairs = nullptr;
    double *cos = nullptr;
};
fh_status near_pairs_device(const DevFil *d_fil, int64_t n, double radius, cudaStream_t s, NearPairs &out,
                            fh_error_info *err);
void near_pairs_free(NearPairs &p, cudaStream_t s);

// Parameters (PfftParams, pfft/mod.rs:183-232), validated.
struct PfftConfig {
    bool fixed_spacing = false;
    double cells_per_filament = 8.0;
    double spacing = 0.0;
    double near_field_radius = 8.0;
    int order = 5;
    bool fft_fp32 = false;  // grid convolution in FP32 (else FP64)
};

// Largest padded FFT grid, in points (MAX_FFT_POINTS, pfft/mod.rs:168).
constexpr int64_t kMaxFftPoints = int64_t(1) << 26;

// Smallest 2^a 3^b 5^c >= n (fft.rs:66-80) and the padded size of an axis.
int64_t smooth_size(int64_t n);
inline int64_t padded_size(int64_t n) { return smooth_size(2 * n - 1); }

// The spacing h for which prod_a max(extent_a / h, 1) = cells (auto_spacing,
// pfft/mod.rs:614-631).
double auto_spacing(const double extent[3], double cells);

// Validates the parameters and builds the grid (the near pairs are found on
// the device, near_pairs_device).
fh_status pfft_setup(const fh_filament *fil, int64_t n, const PfftConfig &cfg, PfftSetup &out, fh_error_info *err);

// Projection quadrature (grid.rs:38-40): tolerance and largest order.
constexpr double kProjectionTolerance = 1e-10;
constexpr int kProjectionMaxOrder = 12;

// Device part of the set-up (fh_pfft_setup.cu), on `stream`:
//   projection of every filament onto its stencil (CSR by filament, ascending
//   grid index) and its transpose (CSR by grid point, ascending filament);
//   the grid approximation sum_g sum_h W_ig W_jh K(g - h) of every near pair.
struct PfftDeviceSetup {
    int64_t *proj_off = nullptr;   // n + 1
    uint32_t *proj_idx = nullptr;  // entries
    double *proj_w = nullptr;
    int64_t *spread_off = nullptr;   // G + 1
    uint32_t *spread_fil = nullptr;  // entries
    double *spread_w = nullptr;
    double *pair_grid = nullptr;  // one per near pair
    int64_t entries = 0;
};
fh_status pfft_device_setup(const PfftSetup &st, const fh_filament *fil, const NearPairs &near, cudaStream_t stream,
                            PfftDeviceSetup &out, fh_error_info *err);
// The near-field matrix: mirrored rows of exact - mu0/4pi cos grid for the
// near pairs (d_exact, d_grid, d_cos per pair; pair lists on the device),
// each row ascending in column (near.rs:263-298).
fh_status pfft_near_csr(int64_t n, int64_t np, const int2 *d_pairs, const double *d_exact, const double *d_grid,
                        const double *d_cos, cudaStream_t stream, int64_t **near_off, uint32_t **near_col,
                        double **near_val, int64_t *near_entries, fh_error_info *err);

// The grid kernel 1 / |r_g - r_h| for an integer offset, zero at the origin
// (near.rs:114-123).
inline double grid_kernel(int64_t dx, int64_t dy, int64_t dz, double spacing);

// The operator on the device (fh_pfft.cu).  Owns its device memory and its
// convolution tables; products run on `stream`.
struct PfftDevice {
    int64_t n = 0, G = 0, P = 0;  // filaments, grid points, padded points
    PfftGrid grid;
    int64_t padded[3] = {0, 0, 0};
    std::vector<int> components;
    double *d_dir = nullptr;
    int64_t *d_proj_off = nullptr;
    uint32_t *d_proj_idx = nullptr;
    double *d_proj_w = nullptr;
    int64_t *d_spread_off = nullptr;
    uint32_t *d_spread_fil = nullptr;
    double *d_spread_w = nullptr;
    int64_t *d_near_off = nullptr;
    uint32_t *d_near_col = nullptr;
    double *d_near_val = nullptr;
    FftConvTables conv;            // twiddles and the kernel's spectrum (fh_fftconv.cu)
    bool fft_fp32 = false;
    FftConvTables conv64;          // with fft_fp32: FP64 tables for full-precision products (residuals)
    void *d_work = nullptr;        // the convolution's grids, reused across products (device cache)
    size_t work_bytes = 0;
    void *stream = nullptr;        // cudaStream_t
    bool own_stream = false;
    int64_t projection_entries = 0, near_entries = 0;
    double setup_host_s = 0, setup_device_s = 0, setup_near_s = 0;  // setup_near_s: the near-pair search (part of the device time)
    PfftDevice() = default;
    PfftDevice(const PfftDevice &) = delete;
    PfftDevice &operator=(const PfftDevice &) = delete;
    ~PfftDevice();
    size_t memory_bytes() const;
};

// Builds the operator for `fil` (host set-up, exact near pairs on the device,
// kernel spectrum).  `stream` may be null: the operator then owns one.
fh_status pfft_build(const fh_filament *fil, int64_t n, const PfftConfig &cfg, void *stream, PfftDevice &op,
                     fh_error_info *err);
// y = L x for `count` vectors of length n (device pointers, vector v at
// x + v n), on op.stream.  With full_precision, an operator built with the
// FP32 convolution convolves in FP64 (for refinement residuals).
fh_status pfft_apply(PfftDevice &op, const double *d_x, double *d_y, int count, fh_error_info *err,
                     bool full_precision = false);

}  // namespace fhb

#include <cmath>

namespace fhb {
inline double grid_kernel(int64_t dx, int64_t dy, int64_t dz, double spacing) {
    const double r2 = (double)(dx * dx + dy * dy + dz * dz);
    return r2 == 0.0 ? 0.0 : 1.0 / (spacing * std::sqrt(r2));
}
}  // namespace fhb
