// The pFFT convolution without a library FFT (fh_fftconv.cu): pruned
// mixed-radix Stockham transforms in shared memory, FP32 or FP64.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fh_internal.h"

namespace fhb {

constexpr int kFftMaxFactors = 24;
constexpr int64_t kFftMaxLength = 4800;  // longest padded axis: two FP64 lines of it and its twiddles fit a CTA

// One axis: its length and its radices (4, then 2, 3, 5), passed by value to
// the kernels.
struct FftAxis {
    int m = 1;
    int nfac = 0;
    int fac[kFftMaxFactors] = {};
};
bool fft_axis_plan(int64_t m, FftAxis &ax);

// Unpadded grid n (axis 2 fastest) and the padded torus m (m_a >= 2 n_a - 1).
struct FftConvShape {
    int64_t n[3] = {1, 1, 1};
    int64_t m[3] = {1, 1, 1};
};

// Per-operator tables: twiddles exp(-2 pi i t / m_a) per axis (in the
// convolution's precision, and FP64 for the set-up) and the kernel's real
// spectrum on the padded grid (times 1 / P), laid out [i][j][k].
struct FftConvTables {
    FftConvShape shape;
    FftAxis axis[3];
    void *tw[3] = {nullptr, nullptr, nullptr};
    void *tw64[3] = {nullptr, nullptr, nullptr};
    void *spectrum = nullptr;
    bool fp32 = false;
};

// Complex elements of the work buffer per complex grid: the sources /
// potentials A (n0 n1 n2), then B (n0 n1 m2), then C (n0 m1 m2); a batch of
// grids keeps each part contiguous per grid (A of every grid first).
size_t fftconv_work_elems(const FftConvShape &sh);

// T = float or double: the precision of the convolution.
template <class T>
fh_status fftconv_setup(const FftConvShape &sh, double spacing, FftConvTables &tab, cudaStream_t s,
                        fh_error_info *err);
// The convolution of `grids` complex grids in place: on entry A[g] holds the
// sources of grid g (two real fields as real and imaginary parts, [i][j][k]),
// on return the potentials.
template <class T>
fh_status fftconv_run(const FftConvTables &tab, void *work, int grids, cudaStream_t s, fh_error_info *err);
void fftconv_free(FftConvTables &tab, cudaStream_t s);

}  // namespace fhb
