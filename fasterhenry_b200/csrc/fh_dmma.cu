// The FP64 trailing update A22 -= L21 U12 of the complex LU on the FP64 tensor
// cores (mma.sync m8n8k4 f64, the only FP64 tensor-core instruction; the
// 5th-generation tcgen05 MMA has no FP64 kind).  The complex product runs as
// four real products on split real / imaginary planes:
//   C_re -= L_re U_re - L_im U_im,   C_im -= L_re U_im + L_im U_re,
// each an FP64 MMA with exact products and FP64 accumulation, so the result
// is an FP64 GEMM (a different summation order from the SIMT kernel's, same
// precision).
//
// CTA tile 64 x 64 complex entries, K in chunks of 32 through shared memory;
// 8 warps as 2 (rows) x 4 (columns), each warp 32 x 16 of C: 4 x 2 fragments
// of 8 x 8, re and im, held in registers (32 FP64 per thread).  Fragment
// layout of m8n8k4 f64 (PTX ISA): A a0 at (row g, k t), B b0 at (k t, col
// g), C c0, c1 at (row g, cols 2 t, 2 t + 1), with g = lane / 4 and
// t = lane % 4.  The L chunk is kept [k][row] (rows fastest, as read from
// the column-major matrix) with rows padded to 68 doubles, the U chunk
// [column][k] (k fastest, as read) padded to 36: both strides are 8 words
// off a bank period, so a warp's fragment load touches every bank twice,
// the minimum for 32 doubles, and the stores from global memory are
// conflict-free.
#include <cuda_runtime.h>

#include <algorithm>

#include "fh_device.cuh"
#include "fh_lu.cuh"

namespace fhb {
namespace {

constexpr int kDmTile = 64;             // C tile edge (complex entries)
constexpr int kDmChunk = 32;            // K per shared-memory stage
constexpr int kDmLdL = kDmTile + 4;     // L chunk row (one k) length, doubles
constexpr int kDmLdU = kDmChunk + 4;    // U chunk row (one column) length, doubles
constexpr int kDmThreads = 256;
constexpr size_t kDmSmem = sizeof(double) * (2 * (size_t)kDmChunk * kDmLdL + 2 * (size_t)kDmTile * kDmLdU);

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Matrix f at a + f m m (complex, column-major, ld m): rows / columns
// [base, m) of the trailing matrix, base = k0 + nb; L21 = columns
// [k0, k0 + nb) of those rows, U12 = rows [k0, k0 + nb) of those columns.
__global__ void __launch_bounds__(kDmThreads, 2) dmma_update_kernel(double2 *__restrict__ a, int64_t m, int k0,
                                                                    int nb) {
    extern __shared__ __align__(16) double dm_smem[];
    double(*Lre)[kDmLdL] = reinterpret_cast<double(*)[kDmLdL]>(dm_smem);  // [k][row]
    double(*Lim)[kDmLdL] = Lre + kDmChunk;
    double(*Ure)[kDmLdU] = reinterpret_cast<double(*)[kDmLdU]>(dm_smem + 2 * kDmChunk * kDmLdL);  // [column][k]
    double(*Uim)[kDmLdU] = Ure + kDmTile;
    double2 *A = a + (int64_t)blockIdx.z * m * m;
    const int64_t base = (int64_t)k0 + nb;
    const int64_t i0 = base + (int64_t)blockIdx.y * kDmTile, j0 = base + (int64_t)blockIdx.x * kDmTile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wr = warp >> 2, wc = warp & 3;  // warp tile: rows 32 wr .. +32, cols 16 wc .. +16
    // Accumulators start as C: fragment (fm, fn) covers rows 32 wr + 8 fm + g,
    // cols 16 wc + 8 fn + 2 t + {0, 1}.
    double cre[4][2][2], cim[4][2][2];
#pragma unroll
    for (int fm = 0; fm < 4; ++fm)
#pragma unroll
        for (int fn = 0; fn < 2; ++fn)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int64_t row = i0 + 32 * wr + 8 * fm + g, col = j0 + 16 * wc + 8 * fn + 2 * t + e;
                double2 v = make_double2(0.0, 0.0);
                if (row < m && col < m) v = A[row + col * m];
                cre[fm][fn][e] = v.x;
                cim[fm][fn][e] = v.y;
            }
    for (int kc = 0; kc < nb; kc += kDmChunk) {
        const int kw = min(kDmChunk, nb - kc);
        __syncthreads();  // the previous chunk's fragment loads are done
        // L21 chunk: rows i0 .. +64, k kc .. +kw (zero beyond); consecutive
        // threads take consecutive rows (coalesced column reads).
        for (int idx = tid; idx < kDmTile * kDmChunk; idx += kDmThreads) {
            const int r = idx & (kDmTile - 1), k = idx / kDmTile;
            const int64_t row = i0 + r;
            double2 v = make_double2(0.0, 0.0);
            if (k < kw && row < m) v = A[row + (int64_t)(k0 + kc + k) * m];
            Lre[k][r] = v.x;
            Lim[k][r] = v.y;
        }
        // U12 chunk: k kc .. +kw, columns j0 .. +64; consecutive threads take
        // consecutive k of one column (a contiguous run).
        for (int idx = tid; idx < kDmTile * kDmChunk; idx += kDmThreads) {
            const int k = idx % kDmChunk, c = idx / kDmChunk;
            const int64_t col = j0 + c;
            double2 v = make_double2(0.0, 0.0);
            if (k < kw && col < m) v = A[(int64_t)(k0 + kc + k) + col * m];
            Ure[c][k] = v.x;
            Uim[c][k] = v.y;
        }
        __syncthreads();
#pragma unroll 2
        for (int k4 = 0; k4 < kDmChunk; k4 += 4) {
            double lre[4], lim[4], ure[2], uim[2];
#pragma unroll
            for (int fm = 0; fm < 4; ++fm) {
                const int r = 32 * wr + 8 * fm + g;
                lre[fm] = -Lre[k4 + t][r];
                lim[fm] = Lim[k4 + t][r];
            }
#pragma unroll
            for (int fn = 0; fn < 2; ++fn) {
                const int c = 16 * wc + 8 * fn + g;
                ure[fn] = Ure[c][k4 + t];
                uim[fn] = Uim[c][k4 + t];
            }
#pragma unroll
            for (int fm = 0; fm < 4; ++fm)
#pragma unroll
                for (int fn = 0; fn < 2; ++fn) {
                    // re -= L_re U_re - L_im U_im;  im -= L_re U_im + L_im U_re
                    dmma(cre[fm][fn][0], cre[fm][fn][1], lre[fm], ure[fn]);
                    dmma(cre[fm][fn][0], cre[fm][fn][1], lim[fm], uim[fn]);
                    dmma(cim[fm][fn][0], cim[fm][fn][1], lre[fm], uim[fn]);
                    dmma(cim[fm][fn][0], cim[fm][fn][1], -lim[fm], ure[fn]);
                }
        }
    }
#pragma unroll
    for (int fm = 0; fm < 4; ++fm)
#pragma unroll
        for (int fn = 0; fn < 2; ++fn)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int64_t row = i0 + 32 * wr + 8 * fm + g, col = j0 + 16 * wc + 8 * fn + 2 * t + e;
                if (row < m && col < m) A[row + col * m] = make_double2(cre[fm][fn][e], cim[fm][fn][e]);
            }
}

}  // namespace

fh_status dmma_update(double *av, int64_t m, int count, int64_t k0, int nb, cudaStream_t s, fh_error_info *err) {
    const int64_t ncols = m - k0 - nb;
    if (ncols <= 0 || nb <= 0) return FH_OK;
    const unsigned tiles = (unsigned)((ncols + kDmTile - 1) / kDmTile);
    FHB_CUDA(cudaFuncSetAttribute(dmma_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmSmem));
    dmma_update_kernel<<<dim3(tiles, tiles, (unsigned)count), kDmThreads, kDmSmem, s>>>(
        reinterpret_cast<double2 *>(av), m, (int)k0, nb);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

}  // namespace fhb
