// Batched mixed-precision sweeps of many small, unevenly sized systems in ONE
// persistent launch (the batched form of MeshSystem::sweep over many
// geometries, solve.rs:881-893 / 1039-1079; the reference sweeps them one
// after another).
//
// A work item is one (system, frequency).  Items are sorted by cost (m^3,
// largest first) on the host and handed out through an atomic counter to
// persistent CTAs, one per SM slot.  A CTA solves its item alone, in its own
// workspace slot:
//
//   1. A = R_ee + j w L_ee in FP32 (column-major), b = Z_ep in FP64;
//   2. LU without interchanges, blocked right-looking: panel of NB columns
//      (per-column scaling and rank-1 updates), U12 = L11^-1 A12 (a thread
//      per column, the column in registers), trailing update A22 -= L21 U12
//      in TILE x TILE tiles staged in shared memory (thread tiles of
//      TILE/16 x TILE/16).  Without pivoting the factorization is stable for
//      R + j w L with R, L symmetric positive definite (N. J. Higham, Math.
//      Comp. 67, 1998), as in the large-system mixed path; the refinement
//      below decides the result;
//   3. iterative refinement: d = (LU)^-1 r in FP32 (blocked triangular
//      solves: a warp per 32-row diagonal block, the CTA for the rows
//      beyond), x += d in FP64, r = b - (R + j w L) x in FP64 straight from
//      R_m, L_m; the stopping rule of the large-system path;
//   4. Z = Z_pp - Z_ep^T x in FP64.
//
// An item whose pivot vanishes or whose refinement does not converge is
// marked; the host redoes it with the FP64 LU.  NB and TILE come per item
// from the autotuner's table (fh_batchtune.cpp), by order bucket.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "fh_batchsolve.h"
#include "fh_device.cuh"

namespace fhb {
namespace {

constexpr int kBT = 256;        // threads per CTA (16 x 16 thread tile grid)
constexpr int kMaxRefine = 30;  // refinement iterations before an item is marked

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 csub_mul(float2 acc, float2 a, float2 b) {  // acc - a b
    acc.x -= a.x * b.x - a.y * b.y;
    acc.y -= a.x * b.y + a.y * b.x;
    return acc;
}
__device__ __forceinline__ float2 shfl2(float2 v, int lane) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, lane), __shfl_sync(0xffffffffu, v.y, lane));
}

// Block-wide max over the CTA (all threads get the result).
__device__ double block_max(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    for (int w = 0; w < kBT / 32; ++w) r = fmax(r, red[w]);
    return r;
}

// Block-wide complex sum (thread 0's result is the deterministic sum in
// warp order).
__device__ double2 block_sum(double2 v, double2 *red) {
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    for (int w = 0; w < kBT / 32; ++w) {
        r.x += red[w].x;
        r.y += red[w].y;
    }
    return r;
}

struct Slot {
    float2 *A;   // m x m
    float2 *d;   // m x p (correction)
    double2 *x;  // m x p
    double2 *r;  // m x p
    double2 *b;  // m x p
};

// The trailing update A22 -= L21 U12 for the panel [k0, k1).
template <int NB, int TILE>
__device__ void trailing_update(float2 *A, int64_t m, int64_t k0, int64_t k1, float2 *smem) {
    float2 *Ls = smem;              // Ls[k * TILE + r]
    float2 *Us = smem + NB * TILE;  // Us[k * TILE + c]
    constexpr int PT = TILE / 16;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t rem = m - k1;
    const int64_t tiles = (rem + TILE - 1) / TILE;
    for (int64_t t = 0; t < tiles * tiles; ++t) {
        const int64_t r0 = k1 + (t % tiles) * TILE, c0 = k1 + (t / tiles) * TILE;
        __syncthreads();
        for (int idx = threadIdx.x; idx < NB * TILE; idx += kBT) {
            const int r = idx % TILE, k = idx / TILE;
            Ls[k * TILE + r] = r0 + r < m ? A[(r0 + r) + (k0 + k) * m] : make_float2(0.f, 0.f);
        }
        for (int idx = threadIdx.x; idx < NB * TILE; idx += kBT) {
            const int k = idx % NB, c = idx / NB;
            Us[k * TILE + c] = c0 + c < m ? A[(k0 + k) + (c0 + c) * m] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        float2 acc[PT][PT];
#pragma unroll
        for (int i = 0; i < PT; ++i)
#pragma unroll
            for (int j = 0; j < PT; ++j) acc[i][j] = make_float2(0.f, 0.f);
#pragma unroll 4
        for (int k = 0; k < NB; ++k) {
            float2 l[PT], u[PT];
#pragma unroll
            for (int i = 0; i < PT; ++i) l[i] = Ls[k * TILE + tx + 16 * i];
#pragma unroll
            for (int j = 0; j < PT; ++j) u[j] = Us[k * TILE + ty + 16 * j];
#pragma unroll
            for (int i = 0; i < PT; ++i)
#pragma unroll
                for (int j = 0; j < PT; ++j) {
                    acc[i][j].x += l[i].x * u[j].x - l[i].y * u[j].y;
                    acc[i][j].y += l[i].x * u[j].y + l[i].y * u[j].x;
                }
        }
#pragma unroll
        for (int i = 0; i < PT; ++i) {
            const int64_t r = r0 + tx + 16 * i;
#pragma unroll
            for (int j = 0; j < PT; ++j) {
                const int64_t c = c0 + ty + 16 * j;
                if (r < m && c < m) {
                    float2 v = A[r + c * m];
                    v.x -= acc[i][j].x;
                    v.y -= acc[i][j].y;
                    A[r + c * m] = v;
                }
            }
        }
    }
    __syncthreads();
}

// LU without interchanges of the m x m A in place; *bad set on a zero or
// non-finite pivot.
template <int NB, int TILE>
__device__ void lu_nopivot(float2 *A, int64_t m, float2 *smem, int *bad) {
    for (int64_t k0 = 0; k0 < m; k0 += NB) {
        const int w = (int)(m - k0 < NB ? m - k0 : NB);
        for (int j = 0; j < w; ++j) {
            const int64_t jj = k0 + j;
            __syncthreads();
            const float2 piv = A[jj + jj * m];
            const float den = piv.x * piv.x + piv.y * piv.y;
            const bool ok = den > 0.f && isfinite(den);
            if (!ok && threadIdx.x == 0) *bad = 1;
            const float2 inv = ok ? make_float2(piv.x / den, -piv.y / den) : make_float2(0.f, 0.f);
            for (int64_t r = jj + 1 + threadIdx.x; r < m; r += kBT) A[r + jj * m] = cmul(A[r + jj * m], inv);
            __syncthreads();
            for (int64_t r = jj + 1 + threadIdx.x; r < m; r += kBT) {
                const float2 l = A[r + jj * m];
                for (int64_t c = jj + 1; c < k0 + w; ++c) A[r + c * m] = csub_mul(A[r + c * m], l, A[jj + c * m]);
            }
        }
        __syncthreads();
        const int64_t k1 = k0 + w;
        if (k1 >= m) break;
        // U12 = L11^-1 A12 (w == NB here): L11 into shared memory, a column
        // per thread in registers.
        float2 *L11 = smem;
        for (int idx = threadIdx.x; idx < NB * NB; idx += kBT) {
            const int i = idx % NB, j = idx / NB;
            L11[idx] = A[(k0 + i) + (k0 + j) * m];
        }
        __syncthreads();
        for (int64_t c = k1 + threadIdx.x; c < m; c += kBT) {
            float2 v[NB];
#pragma unroll
            for (int i = 0; i < NB; ++i) v[i] = A[(k0 + i) + c * m];
#pragma unroll
            for (int jj = 1; jj < NB; ++jj) {
                float2 acc = v[jj];
#pragma unroll
                for (int i = 0; i < jj; ++i) acc = csub_mul(acc, L11[jj + i * NB], v[i]);
                v[jj] = acc;
            }
#pragma unroll
            for (int i = 1; i < NB; ++i) A[(k0 + i) + c * m] = v[i];
        }
        trailing_update<NB, TILE>(A, m, k0, k1, smem);
    }
    __syncthreads();
}

// d = (LU)^-1 d for p columns (unit L, non-unit U, both in A).
__device__ void lu_solve_blocked(const float2 *A, int64_t m, int p, float2 *d) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // forward, unit lower
    for (int64_t b0 = 0; b0 < m; b0 += 32) {
        const int bw = (int)(m - b0 < 32 ? m - b0 : 32);
        if (warp == 0) {
            for (int q = 0; q < p; ++q) {
                float2 di = lane < bw ? d[b0 + lane + (int64_t)q * m] : make_float2(0.f, 0.f);
                for (int jj = 0; jj < bw; ++jj) {
                    const float2 dj = shfl2(di, jj);
                    if (lane > jj && lane < bw) di = csub_mul(di, A[(b0 + lane) + (b0 + jj) * m], dj);
                }
                if (lane < bw) d[b0 + lane + (int64_t)q * m] = di;
            }
        }
        __syncthreads();
        for (int64_t r = b0 + bw + threadIdx.x; r < m; r += kBT)
            for (int q = 0; q < p; ++q) {
                float2 acc = d[r + (int64_t)q * m];
                for (int jj = 0; jj < bw; ++jj)
                    acc = csub_mul(acc, A[r + (b0 + jj) * m], d[b0 + jj + (int64_t)q * m]);
                d[r + (int64_t)q * m] = acc;
            }
        __syncthreads();
    }
    // backward, upper with its diagonal
    for (int64_t b1 = m; b1 > 0; b1 -= 32) {
        const int64_t b0 = b1 > 32 ? b1 - 32 : 0;
        const int bw = (int)(b1 - b0);
        if (warp == 0) {
            for (int q = 0; q < p; ++q) {
                float2 di = lane < bw ? d[b0 + lane + (int64_t)q * m] : make_float2(0.f, 0.f);
                for (int jj = bw - 1; jj >= 0; --jj) {
                    if (lane == jj) {
                        const float2 u = A[(b0 + jj) + (b0 + jj) * m];
                        const float den = u.x * u.x + u.y * u.y;
                        di = den > 0.f ? make_float2((di.x * u.x + di.y * u.y) / den, (di.y * u.x - di.x * u.y) / den)
                                       : make_float2(0.f, 0.f);
                    }
                    const float2 dj = shfl2(di, jj);
                    if (lane < jj) di = csub_mul(di, A[(b0 + lane) + (b0 + jj) * m], dj);
                }
                if (lane < bw) d[b0 + lane + (int64_t)q * m] = di;
            }
        }
        __syncthreads();
        for (int64_t r = threadIdx.x; r < b0; r += kBT)
            for (int q = 0; q < p; ++q) {
                float2 acc = d[r + (int64_t)q * m];
                for (int jj = 0; jj < bw; ++jj)
                    acc = csub_mul(acc, A[r + (b0 + jj) * m], d[b0 + jj + (int64_t)q * m]);
                d[r + (int64_t)q * m] = acc;
            }
        __syncthreads();
    }
}

template <int NB, int TILE>
__device__ __noinline__ void solve_item(const BatchSys &S, const BatchItem &it, Slot sl, float2 *smem, double *dred,
                           double2 *cred, int *s_bad, double2 *z_all, int32_t *status) {
    const int64_t m = S.m, ld = S.ld;
    const int p = (int)S.p;
    const double w = it.omega;
    const double *R = S.R, *L = S.L;
    if (threadIdx.x == 0) *s_bad = 0;
    // 1. the FP32 system and the FP64 right-hand sides
    for (int64_t idx = threadIdx.x; idx < m * m; idx += kBT) {
        const int64_t i = idx % m, j = idx / m;
        sl.A[idx] = make_float2((float)R[i + j * ld], (float)(w * L[i + j * ld]));
    }
    for (int64_t idx = threadIdx.x; idx < m * p; idx += kBT) {
        const int64_t i = idx % m, q = idx / m;
        const double2 bq = make_double2(R[i + (m + q) * ld], w * L[i + (m + q) * ld]);
        sl.b[idx] = bq;
        sl.r[idx] = bq;
        sl.x[idx] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    // 2. factors
    lu_nopivot<NB, TILE>(sl.A, m, smem, s_bad);
    double bmax = 0.0;
    for (int64_t idx = threadIdx.x; idx < m * p; idx += kBT)
        bmax = fmax(bmax, fmax(fabs(sl.b[idx].x), fabs(sl.b[idx].y)));
    const double hb = block_max(bmax, dred);
    // 3. refinement
    int iters = 0;
    bool done = m == 0, failed = false;
    double prev = INFINITY;
    int grow = 0;
    while (!done && !failed) {
        if (*s_bad) {
            failed = true;
            break;
        }
        for (int64_t idx = threadIdx.x; idx < m * p; idx += kBT)
            sl.d[idx] = make_float2((float)sl.r[idx].x, (float)sl.r[idx].y);
        __syncthreads();
        lu_solve_blocked(sl.A, m, p, sl.d);
        double dmax = 0.0, xmax = 0.0;
        for (int64_t idx = threadIdx.x; idx < m * p; idx += kBT) {
            double2 xv = sl.x[idx];
            const float2 dv = sl.d[idx];
            xv.x += (double)dv.x;
            xv.y += (double)dv.y;
            sl.x[idx] = xv;
            dmax = fmax(dmax, fmax(fabs((double)dv.x), fabs((double)dv.y)));
            xmax = fmax(xmax, fmax(fabs(xv.x), fabs(xv.y)));
        }
        __syncthreads();
        // r = b - (R + j w L) x in FP64
        double rmax = 0.0;
        for (int64_t i = threadIdx.x; i < m; i += kBT)
            for (int q = 0; q < p; ++q) {
                double2 acc = sl.b[i + (int64_t)q * m];
                const double2 *xq = sl.x + (int64_t)q * m;
                for (int64_t k = 0; k < m; ++k) {
                    const double rv = R[i + k * ld], lv = w * L[i + k * ld];
                    const double2 xk = xq[k];
                    acc.x -= rv * xk.x - lv * xk.y;
                    acc.y -= rv * xk.y + lv * xk.x;
                }
                sl.r[i + (int64_t)q * m] = acc;
                rmax = fmax(rmax, fmax(fabs(acc.x), fabs(acc.y)));
            }
        const double hd = block_max(dmax, dred);
        const double hx = block_max(xmax, dred);
        const double hr = block_max(rmax, dred);
        ++iters;
        // stopping rule of the large-system mixed path
        const double rel = hx > 0.0 ? hd / hx : 0.0;
        const bool stalled = hd > 0.5 * prev;
        const double rho = isfinite(prev) && prev > 0.0 ? hd / prev : 1.0;
        const bool contracted = rho < 0.1 && rel * rho / (1.0 - rho) <= 1e-12;
        const bool resid_ok = hr <= 1e-6 * hb;
        if (resid_ok && (rel <= 1e-12 || hd == 0.0 || contracted || (stalled && rel <= 1e-10))) {
            done = true;
            break;
        }
        if (stalled) ++grow;
        if (grow >= 3 || !isfinite(hd) || iters >= kMaxRefine) {
            failed = true;
            break;
        }
        prev = hd;
    }
    // 4. Z = Z_pp - Z_ep^T x
    for (int a = 0; a < p; ++a)
        for (int c = 0; c < p; ++c) {
            double2 part = make_double2(0.0, 0.0);
            for (int64_t i = threadIdx.x; i < m; i += kBT) {
                const double ea = R[i + (m + a) * ld], la = w * L[i + (m + a) * ld];
                const double2 xc = sl.x[i + (int64_t)c * m];
                part.x += ea * xc.x - la * xc.y;
                part.y += ea * xc.y + la * xc.x;
            }
            const double2 sum = block_sum(part, cred);
            if (threadIdx.x == 0) {
                const double zr = R[(m + a) + (m + c) * ld] - sum.x;
                const double zi = w == 0.0 ? 0.0 : w * L[(m + a) + (m + c) * ld] - sum.y;
                z_all[it.z_offset + a * p + c] = make_double2(zr, zi);
            }
            __syncthreads();
        }
    if (threadIdx.x == 0) status[it.index] = failed ? -1 : iters;
    __syncthreads();
}

__global__ void __launch_bounds__(kBT) batch_mixed_kernel(const BatchSys *__restrict__ systems,
                                                          const BatchItem *__restrict__ items, int nitems,
                                                          unsigned *counter, unsigned char *work, size_t slot_bytes,
                                                          int64_t mmax, int pmax, double2 *z_all, int32_t *status) {
    extern __shared__ __align__(16) unsigned char batch_smem[];
    __shared__ int s_item, s_bad;
    __shared__ double dred[kBT / 32];
    __shared__ double2 cred[kBT / 32];
    unsigned char *base = work + (size_t)blockIdx.x * slot_bytes;
    Slot sl;
    sl.A = reinterpret_cast<float2 *>(base);
    const int64_t f32 = mmax * mmax + mmax * pmax;  // FP32 complex entries, padded to an even count
    sl.d = sl.A + mmax * mmax;
    sl.x = reinterpret_cast<double2 *>(sl.A + f32 + (f32 & 1));
    sl.r = sl.x + mmax * pmax;
    sl.b = sl.r + mmax * pmax;
    float2 *smem = reinterpret_cast<float2 *>(batch_smem);
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int k = s_item;
        __syncthreads();
        if (k >= nitems) return;
        const BatchItem it = items[k];
        const BatchSys S = systems[it.sys];
        switch (it.cfg) {
            case 0: solve_item<16, 32>(S, it, sl, smem, dred, cred, &s_bad, z_all, status); break;
            case 1: solve_item<16, 64>(S, it, sl, smem, dred, cred, &s_bad, z_all, status); break;
            case 2: solve_item<32, 32>(S, it, sl, smem, dred, cred, &s_bad, z_all, status); break;
            default: solve_item<32, 64>(S, it, sl, smem, dred, cred, &s_bad, z_all, status); break;
        }
    }
}

}  // namespace

size_t batch_smem_bytes() {
    // the largest staging of the configurations: 2 x 32 x 64 complex FP32
    return 2 * 32 * 64 * sizeof(float2);
}

size_t batch_slot_bytes(int64_t mmax, int pmax) {
    const size_t mp = (size_t)(mmax * pmax), f32 = (size_t)(mmax * mmax) + mp;
    const size_t bytes = sizeof(float2) * (f32 + (f32 & 1)) + 3 * sizeof(double2) * mp;
    return (bytes + 255) / 256 * 256;
}

int batch_resident_ctas() {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(batch_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batch_smem_bytes());
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_mixed_kernel, kBT, batch_smem_bytes());
    return std::max(1, sms) * std::max(1, per);
}

fh_status batch_launch(const BatchSys *d_systems, const BatchItem *d_items, int nitems, unsigned *d_counter,
                       void *d_work, size_t slot_bytes, int64_t mmax, int pmax, double2 *d_z, int32_t *d_status,
                       int ctas, cudaStream_t s, fh_error_info *err) {
    FHB_CUDA(cudaFuncSetAttribute(batch_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)batch_smem_bytes()));
    FHB_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned), s));
    batch_mixed_kernel<<<ctas, kBT, batch_smem_bytes(), s>>>(d_systems, d_items, nitems, d_counter,
                                                            static_cast<unsigned char *>(d_work), slot_bytes, mmax,
                                                            pmax, d_z, d_status);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

}  // namespace fhb
