// Cooperative batched triangular solves with the FP32 factors of the
// two-level factorization:
//
//     x <- U^{-1} L^{-1} P x        for every (matrix, right-hand side)
//
// One launch does the forward and the backward pass.  The CTAs of one
// (matrix, right-hand side) pair form a group that meets at a bounded
// barrier of its own; groups never wait for each other.  Per nb-block k:
//
//   * every CTA of the group reads the block's entries of x and forms
//     x_k = Inv_k x_k with the inverse of the diagonal block kept from the
//     factorization (a 128 x 128 matrix-vector product, so no CTA waits on a
//     sequential substitution);
//   * the rows below (forward) or above (backward) the block are split
//     evenly among the group's CTAs, and each subtracts L[r, k] x_k
//     (U[r, k] x_k) from its rows: one coalesced pass over the factor
//     columns, the bandwidth-bound part;
//   * barrier; CTA 0 then stores x_k (deferred, so that no CTA can read a
//     block entry after it was overwritten).
//
// Row interchanges are applied per interchange group (a super-panel) at its
// start by CTA 0, staged in shared memory as in the one-launch-per-block
// forward solve, followed by a barrier.  Each factor entry is read once per
// solve: 8 m^2 bytes per (matrix, right-hand side), the roofline of the pass.
#include <algorithm>
#include <string>

#include "fh_cx.cuh"
#include "fh_lu.cuh"
#include "fh_sync.cuh"

namespace fhb {
namespace {

constexpr int kThreads = 256;
constexpr int kNb = 128;
constexpr int kMaxGroup = 1024;
constexpr int kMaxPerGroup = 16;

struct SolveArgs {
    const Cx<float> *a;
    int64_t m;
    int count, nrhs, nb, group, per_group;
    const int *pivots;
    const Cx<float> *linv, *uinv;  // slot k: count * nb * nb, matrix f at + f * nb * nb
    Cx<float> *x;                  // (f * nrhs + q) * m
    unsigned *bar;
    int *error;
};

// xs = Inv * xin for the wk x wk column-major block inverse `inv`.  Thread t
// takes row t % 128 and half t / 128 of the columns; the halves meet in
// `part`.  Every thread of the CTA calls it.
__device__ __forceinline__ void diag_apply(const Cx<float> *__restrict__ inv, int wk, const Cx<float> *xin,
                                           Cx<float> *xs, Cx<float> *part) {
    const int r = threadIdx.x % kNb, h = threadIdx.x / kNb;
    Cx<float> acc{0.f, 0.f};
    if (r < wk) {
        const int c0 = h * (kNb / 2), c1 = min(wk, c0 + kNb / 2);
#pragma unroll 8
        for (int c = c0; c < c1; ++c) {
            const float2 l = __ldg(reinterpret_cast<const float2 *>(inv) + r + (int64_t)c * wk);
            const Cx<float> v = xin[c];
            acc.re += l.x * v.re - l.y * v.im;
            acc.im += l.x * v.im + l.y * v.re;
        }
    }
    if (h == 1) part[r] = acc;
    __syncthreads();
    if (h == 0 && r < wk) xs[r] = Cx<float>{acc.re + part[r].re, acc.im + part[r].im};
    __syncthreads();
}

// X[r] -= sum_c F[r + c m] xs[c] for the rows [r0, r1) of this CTA's share.
// F points at column 0 of the block.  Loads of 16 columns are issued together.
__device__ __forceinline__ void block_update(const Cx<float> *__restrict__ F, int64_t m, int wk, const Cx<float> *xs,
                                             Cx<float> *X, int64_t r0, int64_t r1) {
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) {
        Cx<float> acc = ldcg(X + r);
        for (int c0 = 0; c0 < wk; c0 += 16) {
            float2 l[16];
#pragma unroll
            for (int q = 0; q < 16; ++q)
                if (c0 + q < wk) l[q] = __ldcs(reinterpret_cast<const float2 *>(F) + r + (int64_t)(c0 + q) * m);
#pragma unroll
            for (int q = 0; q < 16; ++q)
                if (c0 + q < wk) {
                    const Cx<float> v = xs[c0 + q];
                    acc.re -= l[q].x * v.re - l[q].y * v.im;
                    acc.im -= l[q].x * v.im + l[q].y * v.re;
                }
        }
        X[r] = acc;
    }
}

// This CTA's share of the rows [lo, hi): contiguous chunks, multiples of 32.
__device__ __forceinline__ void share(int64_t lo, int64_t hi, int per_group, int slice, int64_t &r0, int64_t &r1) {
    const int64_t rows = hi - lo;
    int64_t chunk = (rows + per_group - 1) / per_group;
    chunk = (chunk + 31) / 32 * 32;
    r0 = min(hi, lo + (int64_t)slice * chunk);
    r1 = min(hi, r0 + chunk);
}

__global__ void __launch_bounds__(kThreads) trisolve_kernel(SolveArgs g) {
    const int grp = blockIdx.x / g.per_group, slice = blockIdx.x % g.per_group;
    const int f = grp / g.nrhs;
    const int64_t m = g.m;
    const Cx<float> *A = g.a + (int64_t)f * m * m;
    Cx<float> *X = g.x + (int64_t)grp * m;
    unsigned *bar = g.bar + (size_t)grp * kGroupBarrierStride;
    const unsigned expected = (unsigned)g.per_group;
    const int tid = threadIdx.x, nb = g.nb;
    const size_t blk_stride = (size_t)g.count * nb * nb;

    __shared__ Cx<float> xin[kNb], xs[kNb], part[kNb];
    __shared__ Cx<float> sx[kMaxGroup], ext[kMaxGroup];
    __shared__ int piv[kMaxGroup], first[kMaxGroup];

    // ---------------- forward: x <- L^{-1} P x ----------------
    for (int64_t g0 = 0; g0 < m; g0 += g.group) {
        const int wg = (int)min((int64_t)g.group, m - g0);
        if (slice == 0) {
            // the group's interchanges, in order, on rows >= g0 of x
            for (int t = tid; t < wg; t += kThreads) {
                sx[t] = ldcg(X + g0 + t);
                piv[t] = g.pivots[(int64_t)f * m + g0 + t];
            }
            __syncthreads();
            for (int t = tid; t < wg; t += kThreads) {
                const int p = piv[t];
                int fst = t;
                if (p >= g0 + wg) {
                    for (int q = 0; q < t; ++q)
                        if (piv[q] == p) {
                            fst = q;
                            break;
                        }
                    if (fst == t) ext[t] = ldcg(X + p);
                }
                first[t] = fst;
            }
            __syncthreads();
            if (tid == 0) {
                for (int jj = 0; jj < wg; ++jj) {
                    const int p = piv[jj];
                    if (p == g0 + jj) continue;
                    Cx<float> &other = p < g0 + wg ? sx[p - g0] : ext[first[jj]];
                    const Cx<float> tmp = sx[jj];
                    sx[jj] = other;
                    other = tmp;
                }
            }
            __syncthreads();
            for (int t = tid; t < wg; t += kThreads) {
                if (piv[t] >= g0 + wg && first[t] == t) X[piv[t]] = ext[t];
                X[g0 + t] = sx[t];
            }
        }
        if (!group_barrier(bar, expected, g.error)) return;
        for (int64_t k0 = g0; k0 < g0 + wg; k0 += nb) {
            const int wk = (int)min((int64_t)nb, g0 + wg - k0);
            int64_t r0, r1;
            share(k0 + wk, m, g.per_group, slice, r0, r1);
            if (slice == 0 || r0 < r1) {  // a CTA without rows in this step only meets the barrier
                for (int t = tid; t < wk; t += kThreads) xin[t] = ldcg(X + k0 + t);
                __syncthreads();
                diag_apply(g.linv + (size_t)(k0 / nb) * blk_stride + (size_t)f * nb * nb, wk, xin, xs, part);
                block_update(A + k0 * m, m, wk, xs, X, r0, r1);
            }
            if (!group_barrier(bar, expected, g.error)) return;
            if (slice == 0)
                for (int t = tid; t < wk; t += kThreads) X[k0 + t] = xs[t];
        }
    }
    // the last deferred block store is visible before the backward pass reads it
    if (!group_barrier(bar, expected, g.error)) return;

    // ---------------- backward: x <- U^{-1} x ----------------
    const int64_t nblk = (m + nb - 1) / nb;
    for (int64_t blk = nblk - 1; blk >= 0; --blk) {
        const int64_t k0 = blk * nb;
        const int wk = (int)min((int64_t)nb, m - k0);
        int64_t r0, r1;
        share(0, k0, g.per_group, slice, r0, r1);
        if (slice == 0 || r0 < r1) {
            for (int t = tid; t < wk; t += kThreads) xin[t] = ldcg(X + k0 + t);
            __syncthreads();
            diag_apply(g.uinv + (size_t)blk * blk_stride + (size_t)f * nb * nb, wk, xin, xs, part);
            block_update(A + k0 * m, m, wk, xs, X, r0, r1);
        }
        if (!group_barrier(bar, expected, g.error)) return;
        if (slice == 0)
            for (int t = tid; t < wk; t += kThreads) X[k0 + t] = xs[t];
    }
}

}  // namespace

fh_status trisolve_plan(int groups, int64_t m, int *per_group, size_t *bytes, fh_error_info *err, int share) {
    int dev = 0, sms = 0, occ = 0, coop = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    FHB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    FHB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return fail(err, FH_ERR_NO_DEVICE, "the device does not support cooperative launches");
    FHB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, trisolve_kernel, kThreads, 0));
    const int capacity = occ * sms / std::max(1, share);
    if (groups <= 0 || groups > capacity) {
        *per_group = 0;  // the caller falls back to the one-launch-per-block solve
        *bytes = 0;
        return FH_OK;
    }
    int pg = std::min(kMaxPerGroup, capacity / groups);
    pg = (int)std::min<int64_t>(pg, std::max<int64_t>(1, (m + 255) / 256));
    *per_group = std::max(1, pg);
    *bytes = 128 + (size_t)groups * kGroupBarrierStride * 4;
    return FH_OK;
}

void trisolve_bind(void *mem, int groups, int per_group, SolveScratch &ss) {
    unsigned char *p = static_cast<unsigned char *>(mem);
    ss.error = reinterpret_cast<int *>(p);
    ss.barrier = reinterpret_cast<unsigned *>(p + 128);
    ss.groups = groups;
    ss.per_group = per_group;
}

fh_status lu_solve_inv(const LuBatch<float> &b, const void *linv, const void *uinv, float *x, int nrhs, int nb,
                       int group, const SolveScratch &ss, cudaStream_t s, fh_error_info *err) {
    if (b.m == 0 || b.count == 0 || nrhs == 0) return FH_OK;
    if (nb != kNb || group % nb || group > kMaxGroup || !linv || !uinv)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "cooperative solve needs nb = 128, group | 1024 and block inverses");
    if (ss.per_group <= 0 || ss.groups != b.count * nrhs)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "cooperative solve scratch does not match the batch");
    FHB_CUDA(cudaMemsetAsync(ss.barrier, 0, (size_t)ss.groups * kGroupBarrierStride * 4, s));
    SolveArgs g;
    g.a = reinterpret_cast<const Cx<float> *>(b.a);
    g.m = b.m;
    g.count = b.count;
    g.nrhs = nrhs;
    g.nb = nb;
    g.group = group;
    g.per_group = ss.per_group;
    g.pivots = b.pivots;
    g.linv = reinterpret_cast<const Cx<float> *>(linv);
    g.uinv = reinterpret_cast<const Cx<float> *>(uinv);
    g.x = reinterpret_cast<Cx<float> *>(x);
    g.bar = ss.barrier;
    g.error = ss.error;
    void *params[] = {&g};
    prof_begin(s, FH_PROF_SOLVE_BARRIER);
    FHB_CUDA(cudaLaunchCooperativeKernel((const void *)trisolve_kernel, dim3(ss.groups * ss.per_group), dim3(kThreads),
                                         params, 0, s));
    prof_end(s, FH_PROF_SOLVE_BARRIER, 8.0 * (double)b.m * (double)b.m * nrhs * b.count);
    return FH_OK;
}

fh_status trisolve_check(const SolveScratch &ss, cudaStream_t s, fh_error_info *err) {
    int flag = 0;
    FHB_CUDA(cudaMemcpyAsync(&flag, ss.error, sizeof(int), cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    if (flag) {
        cudaMemsetAsync(ss.error, 0, sizeof(int), s);
        return fail(err, FH_ERR_DEVICE_TIMEOUT, "a triangular-solve barrier ran out of its iteration limit");
    }
    return FH_OK;
}

}  // namespace fhb
