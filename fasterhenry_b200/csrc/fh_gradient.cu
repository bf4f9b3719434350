// Products of the derivative matrices with the branch currents, for the
// adjoint (stationary) form of the impedance gradient:
//
//   dZ_ab / dp = I_a^T (dR/dp + j w dL/dp) I_b,   I = M^T [-Z_ee^-1 Z_ep; 1]
//
// With D[i + j n] = dL_ij / d(side i) (device_fill_grad), the L part for the
// width or thickness of segment s is sum over i in s of I_a,i (D I_b)_i +
// I_b,i (D I_a)_i, so one matrix-vector product per derivative matrix and
// port gives every segment's entry.  HBM-bound: each D entry is read once.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "fh_device.cuh"

namespace fhb {
namespace {

constexpr int kRows = 128;    // rows of D per block (one per thread)
constexpr int kCols = 256;    // columns of D per block
constexpr int kPorts = 8;     // ports per launch

// part[((c * 2 + which) * pq + q) * n + i] = sum over the columns j of chunk c
// of D_which[i + j n] * I[(q0 + q) n + j] (complex I, real D).
__global__ void __launch_bounds__(kRows) deriv_gemv_kernel(const double *__restrict__ Dw,
                                                           const double *__restrict__ Dh, int64_t n,
                                                           const double2 *__restrict__ I, int q0, int pq,
                                                           double2 *__restrict__ part) {
    __shared__ double2 s_i[kPorts][kCols];
    const int which = blockIdx.z;
    const double *D = which ? Dh : Dw;
    const int64_t i = (int64_t)blockIdx.x * kRows + threadIdx.x;
    const int64_t j0 = (int64_t)blockIdx.y * kCols;
    const int cols = (int)std::min<int64_t>(kCols, n - j0);
    for (int k = threadIdx.x; k < pq * kCols; k += kRows) {
        const int q = k / kCols, c = k % kCols;
        s_i[q][c] = c < cols ? I[(int64_t)(q0 + q) * n + j0 + c] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (i >= n) return;
    double re[kPorts], im[kPorts];
#pragma unroll
    for (int q = 0; q < kPorts; ++q) re[q] = im[q] = 0.0;
    const double *col = D + i + j0 * n;
    for (int c = 0; c < cols; ++c) {
        const double d = col[(int64_t)c * n];
#pragma unroll
        for (int q = 0; q < kPorts; ++q)
            if (q < pq) {
                re[q] += d * s_i[q][c].x;
                im[q] += d * s_i[q][c].y;
            }
    }
    for (int q = 0; q < pq; ++q)
        part[(((int64_t)blockIdx.y * 2 + which) * pq + q) * n + i] = make_double2(re[q], im[q]);
}

// y[(which * p + q0 + q) n + i] = sum over chunks, in chunk order.
__global__ void deriv_gemv_reduce_kernel(const double2 *__restrict__ part, int chunks, int64_t n, int p, int q0,
                                         int pq, double2 *__restrict__ y) {
    const int64_t total = 2 * (int64_t)pq * n;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t % n;
        const int64_t wq = t / n;  // which * pq + q
        const int which = (int)(wq / pq), q = (int)(wq % pq);
        double re = 0.0, im = 0.0;
        for (int c = 0; c < chunks; ++c) {
            const double2 v = part[(int64_t)c * 2 * pq * n + wq * n + i];
            re += v.x;
            im += v.y;
        }
        y[((int64_t)which * p + q0 + q) * n + i] = make_double2(re, im);
    }
}

}  // namespace

fh_status gradient_products(const double *d_Dw, const double *d_Dh, int64_t n, const double *d_I, int p, double *d_y,
                            double *d_part, cudaStream_t stream, fh_error_info *err) {
    if (n == 0 || p == 0) return FH_OK;
    const int chunks = (int)((n + kCols - 1) / kCols);
    for (int q0 = 0; q0 < p; q0 += kPorts) {
        const int pq = std::min(kPorts, p - q0);
        dim3 grid((unsigned)((n + kRows - 1) / kRows), (unsigned)chunks, 2);
        deriv_gemv_kernel<<<grid, kRows, 0, stream>>>(d_Dw, d_Dh, n, reinterpret_cast<const double2 *>(d_I), q0, pq,
                                                      reinterpret_cast<double2 *>(d_part));
        FHB_CUDA(cudaGetLastError());
        const int64_t total = 2 * (int64_t)pq * n;
        const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 16);
        deriv_gemv_reduce_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<const double2 *>(d_part), chunks, n, p,
                                                             q0, pq, reinterpret_cast<double2 *>(d_y));
        FHB_CUDA(cudaGetLastError());
    }
    return FH_OK;
}

size_t gradient_part_elems(int64_t n, int p) {
    const int64_t chunks = (n + kCols - 1) / kCols;
    return (size_t)(chunks * 2 * std::min(p, kPorts) * n * 2);  // doubles
}

}  // namespace fhb
