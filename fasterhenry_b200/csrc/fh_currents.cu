// Filament currents, densities and powers from solved loop currents
// (currents.rs:172-274): branch currents I_b = M^T [I_e; I_p] through the
// transposed loop basis (per branch, its loops in increasing order, which is
// the order in which the reference's row-by-row scatter adds them), then
// |J| = |I| / (w h) and P = |I|^2 R / 2 per filament, and per segment the
// sums and the first filament of largest |J|.
#include <cuda_runtime.h>

#include <algorithm>

#include "fh_device.cuh"

namespace fhb {
namespace {

// Thread per (frequency, filament).  X holds Z_ee^-1 Z_ep per frequency
// (count x p x m complex) and the internal loop currents are -X I_p; or, with
// `applied`, X holds Z_ee^-1 Z_ep I_p itself (count x m).
__global__ void branch_currents_kernel(const double2 *__restrict__ X, const double2 *__restrict__ ip, int64_t m,
                                       int p, bool applied, int64_t n, int count, const int64_t *__restrict__ col_ptr,
                                       const int32_t *__restrict__ col_loop, const double *__restrict__ col_sign,
                                       const double *__restrict__ whr, double2 *__restrict__ ib,
                                       double *__restrict__ dens, double *__restrict__ pow) {
    const int64_t total = (int64_t)count * n;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int f = (int)(t / n);
        const int64_t k = t % n;
        double re = 0.0, im = 0.0;
        for (int64_t e = col_ptr[k]; e < col_ptr[k + 1]; ++e) {
            const int64_t r = col_loop[e];
            const double s = col_sign[e];
            double xr, xi;
            if (r < m && applied) {
                const double2 x = X[(int64_t)f * m + r];
                xr = -x.x;
                xi = -x.y;
            } else if (r < m) {
                double ar = 0.0, ai = 0.0;
                for (int q = 0; q < p; ++q) {
                    const double2 x = X[((int64_t)f * p + q) * m + r], c = ip[q];
                    ar += x.x * c.x - x.y * c.y;
                    ai += x.x * c.y + x.y * c.x;
                }
                xr = -ar;
                xi = -ai;
            } else {
                xr = ip[r - m].x;
                xi = ip[r - m].y;
            }
            re += xr * s;
            im += xi * s;
        }
        ib[t] = make_double2(re, im);
        const double mag = hypot(re, im);
        dens[t] = mag / (whr[3 * k] * whr[3 * k + 1]);
        pow[t] = 0.5 * (re * re + im * im) * whr[3 * k + 2];
    }
}

// Thread per (frequency, segment): the segment's filaments in order.
__global__ void segment_sums_kernel(const double2 *__restrict__ ib, const double *__restrict__ dens,
                                    const double *__restrict__ pow, const int64_t *__restrict__ first, int64_t nseg,
                                    int64_t n, int count, double2 *__restrict__ seg_cur, double *__restrict__ seg_pow,
                                    double *__restrict__ seg_peak, int64_t *__restrict__ seg_peak_idx) {
    const int64_t total = (int64_t)count * nseg;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = t / nseg, s = t % nseg;
        double re = 0.0, im = 0.0, pw = 0.0, best = -1.0;
        int64_t at = -1;
        for (int64_t k = first[s]; k < first[s + 1]; ++k) {
            const int64_t o = f * n + k;
            re += ib[o].x;
            im += ib[o].y;
            pw += pow[o];
            if (at < 0 || dens[o] > best) {
                best = dens[o];
                at = k;
            }
        }
        seg_cur[t] = make_double2(re, im);
        seg_pow[t] = pw;
        seg_peak[t] = best;
        seg_peak_idx[t] = at;
    }
}

}  // namespace

fh_status launch_currents(const double *d_x, const double *d_ip, int64_t m, int p, bool applied, int64_t n, int count,
                          const int64_t *d_col_ptr, const int32_t *d_col_loop, const double *d_col_sign,
                          const double *d_whr, const int64_t *d_first, int64_t nseg, double *d_ib, double *d_dens,
                          double *d_pow, double *d_seg_cur, double *d_seg_pow, double *d_seg_peak,
                          int64_t *d_seg_idx, cudaStream_t s, fh_error_info *err) {
    const int64_t total = (int64_t)count * n;
    if (total) {
        const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 32);
        branch_currents_kernel<<<blocks, 256, 0, s>>>(
            reinterpret_cast<const double2 *>(d_x), reinterpret_cast<const double2 *>(d_ip), m, p, applied, n, count,
            d_col_ptr, d_col_loop, d_col_sign, d_whr, reinterpret_cast<double2 *>(d_ib), d_dens, d_pow);
        FHB_CUDA(cudaGetLastError());
    }
    const int64_t segs = (int64_t)count * nseg;
    if (segs) {
        const unsigned blocks = (unsigned)std::min<int64_t>((segs + 127) / 128, 148 * 32);
        segment_sums_kernel<<<blocks, 128, 0, s>>>(reinterpret_cast<const double2 *>(d_ib), d_dens, d_pow, d_first,
                                                   nseg, n, count, reinterpret_cast<double2 *>(d_seg_cur), d_seg_pow,
                                                   d_seg_peak, d_seg_idx);
        FHB_CUDA(cudaGetLastError());
    }
    return FH_OK;
}

}  // namespace fhb
