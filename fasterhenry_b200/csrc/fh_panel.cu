// Cooperative panel factorization: one launch factors an outer panel of NB
// (<= 128) columns of every matrix of the batch with partial pivoting.
//
// Each CTA owns a contiguous slice of the panel's rows of one matrix
// (per_matrix CTAs per matrix, all CTAs co-resident: cooperative launch).
// The panel is factored in sub-panels of 16 columns:
//
//   per column j:   local arg-max of |re| + |im| over the CTA's rows, published
//                   with the candidate row's NB values (and row j's, by its
//                   owner) into a buffer double-buffered by the parity of j;
//                   one barrier of the matrix's CTAs; every CTA picks the pivot
//                   (largest, then first row, as dense.rs:157-166), the owners
//                   of rows j and p exchange them across all NB panel columns,
//                   and each CTA scales and rank-1-updates its own rows inside
//                   the sub-panel.  The rank-1 pass writes column j+1, so the
//                   arg-max of column j+1 is taken in that pass, not reread.
//   per sub-panel:  barrier; U12 of the sub-panel (L11^-1 A12 over the rest of
//                   the outer panel) by slice 0 of each matrix; barrier; each
//                   CTA updates its own rows of the rest of the outer panel
//                   (a tall GEMM with K = 16, which also yields the arg-max of
//                   the next sub-panel's first column).
//
// The rank-1 traffic therefore stays inside 16 columns, and one launch
// replaces the 2 x NB launches of a column-at-a-time panel.  Row interchanges
// cover every column of the outer panel, so the forward substitution can
// apply one outer panel's interchanges at a time.  Barriers synchronise only
// the CTAs of one matrix (a counter per matrix) and are bounded: a barrier
// that gives up sets the error flag, which stays set for the whole
// factorization, and every CTA returns.
#include <cooperative_groups.h>

#include <climits>
#include <mutex>

#include "fh_cx.cuh"
#include "fh_lu.cuh"
#include "fh_sync.cuh"

namespace fhb {
namespace {

constexpr int kW = 16;         // sub-panel width
constexpr int kNbMax = 128;    // outer panel width limit
constexpr int kThreads = 256;
constexpr int kBarrierStride = kGroupBarrierStride;

struct CoopArgs {
    unsigned *barrier;
    int *error;
    double *cand_val;
    int *cand_row;
    void *cand_data;
    void *rowj;
    int per_matrix;
};

// kCluster: the CTAs of one matrix form a thread-block cluster (one
// cluster per matrix); the pivot candidates and the rows they carry are
// exchanged through distributed shared memory, and the matrix's barriers are
// the cluster's hardware barrier.  Otherwise the CTAs of a cooperative launch
// exchange them through global memory and meet at a bounded counter barrier.
template <class T, bool kCluster>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 2 : 1) panel_coop_kernel(Cx<T> *__restrict__ a, int64_t m, int64_t K0, int NB,
                                                              int *__restrict__ pivots, int *__restrict__ singular,
                                                              CoopArgs args) {
    const int per_matrix = args.per_matrix;
    const int f = blockIdx.x / per_matrix, slice = blockIdx.x % per_matrix;
    Cx<T> *A = a + (int64_t)f * m * m;
    const int64_t rows_total = m - K0;
    const int64_t chunk = (rows_total + per_matrix - 1) / per_matrix;
    const int64_t r_begin = K0 + (int64_t)slice * chunk;
    const int64_t r_end = min(m, r_begin + chunk);
    Cx<T> *cand_data = reinterpret_cast<Cx<T> *>(args.cand_data);
    Cx<T> *rowj_buf = reinterpret_cast<Cx<T> *>(args.rowj);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned *bar = args.barrier + (size_t)f * kBarrierStride;

    __shared__ Cx<T> P[kNbMax];
    __shared__ Cx<T> Rj[kNbMax];
    __shared__ Cx<T> U[kW][kNbMax];
    __shared__ double s_val[kThreads / 32];
    __shared__ int s_idx[kThreads / 32];
    __shared__ int s_best_slot, s_piv;
    // Cluster form: this CTA's candidate (value, row, its panel row) and, on
    // the owner of row j, row j, double-buffered by the parity of j.
    __shared__ double c_val[kCluster ? 2 : 1];
    __shared__ int c_row[kCluster ? 2 : 1];
    __shared__ Cx<T> c_data[kCluster ? 2 : 1][kCluster ? kNbMax : 1];
    __shared__ Cx<T> c_rowj[kCluster ? 2 : 1][kCluster ? kNbMax : 1];
    const int64_t rows_chunk = chunk;

    auto better = [](double v2, int i2, double v1, int i1) { return v2 > v1 || (v2 == v1 && i2 < i1); };

    // This thread's arg-max candidate for the next column, gathered while the
    // previous step wrote that column (rank-1 update or sub-panel GEMM).
    double best = -1.0;
    int bi = INT_MAX;
    bool fused = false;
    for (int s0 = 0; s0 < NB; s0 += kW) {
        const int w = min(kW, NB - s0);
        const int64_t k0 = K0 + s0;
        for (int c = 0; c < w; ++c) {
            const int64_t j = k0 + c;
            const int par = (int)(j & 1);
            // 1. local arg-max over the CTA's rows i >= j
            if (!fused) {
                best = -1.0;
                bi = INT_MAX;
                for (int64_t i = max(r_begin, j) + tid; i < r_end; i += kThreads) {
                    const Cx<T> v = ldcg(A + i + j * m);
                    const double n1 = (double)(fabs(v.re) + fabs(v.im));
                    if (n1 > best || (n1 == best && (int)i < bi)) {
                        best = n1;
                        bi = (int)i;
                    }
                }
            }
            fused = false;
            for (int o = 16; o > 0; o >>= 1) {
                const double v2 = __shfl_down_sync(0xffffffffu, best, o);
                const int i2 = __shfl_down_sync(0xffffffffu, bi, o);
                if (better(v2, i2, best, bi)) {
                    best = v2;
                    bi = i2;
                }
            }
            if (lane == 0) {
                s_val[warp] = best;
                s_idx[warp] = bi;
            }
            __syncthreads();
            if (tid == 0) {
                for (int q = 1; q < kThreads / 32; ++q)
                    if (better(s_val[q], s_idx[q], best, bi)) {
                        best = s_val[q];
                        bi = s_idx[q];
                    }
                if constexpr (kCluster) {
                    c_val[par] = best;
                    c_row[par] = bi == INT_MAX ? -1 : bi;
                } else {
                    const int slot = (f * per_matrix + slice) * 2 + par;
                    args.cand_val[slot] = best;
                    args.cand_row[slot] = bi == INT_MAX ? -1 : bi;
                }
                s_idx[0] = bi;
            }
            __syncthreads();
            {
                const int brow = s_idx[0];
                const int slot = (f * per_matrix + slice) * 2 + par;
                if (brow != INT_MAX)
                    for (int t = tid; t < NB; t += kThreads) {
                        const Cx<T> v = ldcg(A + brow + (K0 + t) * m);
                        if constexpr (kCluster)
                            c_data[par][t] = v;
                        else
                            cand_data[(int64_t)slot * kNbMax + t] = v;
                    }
                if (j >= r_begin && j < r_end)
                    for (int t = tid; t < NB; t += kThreads) {
                        const Cx<T> v = ldcg(A + j + (K0 + t) * m);
                        if constexpr (kCluster)
                            c_rowj[par][t] = v;
                        else
                            rowj_buf[(int64_t)(f * 2 + par) * kNbMax + t] = v;
                    }
            }
            // 2. every CTA's candidate is published
            if constexpr (kCluster) {
                cooperative_groups::this_cluster().sync();
            } else {
                if (!group_barrier(bar, (unsigned)per_matrix, args.error)) return;
            }
            // 3. the pivot (warp 0 reduces the candidates of this matrix), and
            //    the interchange of rows j and p
            double bv = -1.0;
            int brow = INT_MAX, bslot = -1;
            if (warp == 0) {
                for (int q = lane; q < per_matrix; q += 32) {
                    double v2;
                    int r2, slot;
                    if constexpr (kCluster) {
                        auto cl = cooperative_groups::this_cluster();
                        v2 = *cl.map_shared_rank(&c_val[par], (unsigned)q);
                        r2 = *cl.map_shared_rank(&c_row[par], (unsigned)q);
                        slot = q;
                    } else {
                        slot = (f * per_matrix + q) * 2 + par;
                        v2 = __ldcg(args.cand_val + slot);
                        r2 = __ldcg(args.cand_row + slot);
                    }
                    if (r2 >= 0 && better(v2, r2, bv, brow)) {
                        bv = v2;
                        brow = r2;
                        bslot = slot;
                    }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const double v2 = __shfl_down_sync(0xffffffffu, bv, o);
                    const int r2 = __shfl_down_sync(0xffffffffu, brow, o);
                    const int s2 = __shfl_down_sync(0xffffffffu, bslot, o);
                    if (s2 >= 0 && better(v2, r2, bv, brow)) {
                        bv = v2;
                        brow = r2;
                        bslot = s2;
                    }
                }
            }
            if (tid == 0) {  // lane 0 of warp 0 holds the reduced candidate
                int p = (int)j;
                if (bv == 0.0) {
                    if (slice == 0) singular[f] = 1;  // exactly zero pivot (dense.rs:166-168)
                    bslot = -1;
                } else if (bv > 0.0) {
                    p = brow;
                } else {
                    bslot = -1;  // all-NaN column: keep the diagonal
                }
                if (p == (int)j) bslot = -1;
                s_piv = p;
                s_best_slot = bslot;
                if (slice == 0) pivots[(int64_t)f * m + j] = p;
            }
            __syncthreads();
            const int p = s_piv, pslot = s_best_slot;
            if constexpr (kCluster) {
                auto cl = cooperative_groups::this_cluster();
                const unsigned owner_j = (unsigned)((j - K0) / rows_chunk);
                const Cx<T> *rj_src = cl.map_shared_rank(&c_rowj[par][0], owner_j);
                const Cx<T> *p_src = pslot >= 0 ? cl.map_shared_rank(&c_data[par][0], (unsigned)pslot) : rj_src;
                for (int t = tid; t < NB; t += kThreads) {
                    Rj[t] = rj_src[t];
                    P[t] = p_src[t];
                }
            } else {
                for (int t = tid; t < NB; t += kThreads) {
                    const Cx<T> rj = ldcg(rowj_buf + (int64_t)(f * 2 + par) * kNbMax + t);
                    Rj[t] = rj;
                    P[t] = pslot >= 0 ? ldcg(cand_data + (int64_t)pslot * kNbMax + t) : rj;
                }
            }
            __syncthreads();
            if (p != (int)j) {
                if (p >= r_begin && p < r_end)
                    for (int t = tid; t < NB; t += kThreads) A[p + (K0 + t) * m] = Rj[t];
                if (j >= r_begin && j < r_end)
                    for (int t = tid; t < NB; t += kThreads) A[j + (K0 + t) * m] = P[t];
            }
            __syncthreads();
            // 4. scale by the pivot's reciprocal and rank-1 update inside the
            //    sub-panel; column j+1's new values feed its arg-max.
            const Cx<T> one{(T)1, (T)0};
            const Cx<T> inv = cdiv(one, P[s0 + c]);
            best = -1.0;
            bi = INT_MAX;
            // Rows go kG at a time (their column-j entries loaded together),
            // then the sub-panel columns right of j kQ at a time for all kG
            // rows, so a group of rows costs a few memory latencies instead of
            // two per row.  Each row's arithmetic and the arg-max order (rows
            // ascending per thread, ties keep the first) are unchanged.
            constexpr int kG = sizeof(T) == 4 ? 4 : 2;
            constexpr int kQ = sizeof(T) == 4 ? 4 : 2;
            for (int64_t ib = max(r_begin, j + 1) + tid; ib < r_end; ib += (int64_t)kG * kThreads) {
                Cx<T> l[kG];
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                    const int64_t i = ib + (int64_t)g * kThreads;
                    if (i < r_end) l[g] = ldcg(A + i + j * m);
                }
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                    const int64_t i = ib + (int64_t)g * kThreads;
                    if (i < r_end) {
                        l[g] = cmul(l[g], inv);
                        A[i + j * m] = l[g];
                    }
                }
                for (int q0 = c + 1; q0 < w; q0 += kQ) {
                    Cx<T> y[kG][kQ];
#pragma unroll
                    for (int g = 0; g < kG; ++g)
#pragma unroll
                        for (int qq = 0; qq < kQ; ++qq) {
                            const int64_t i = ib + (int64_t)g * kThreads;
                            if (i < r_end && q0 + qq < w) y[g][qq] = ldcg(A + i + (k0 + q0 + qq) * m);
                        }
#pragma unroll
                    for (int g = 0; g < kG; ++g)
#pragma unroll
                        for (int qq = 0; qq < kQ; ++qq) {
                            const int64_t i = ib + (int64_t)g * kThreads;
                            if (i < r_end && q0 + qq < w) {
                                csubmul(y[g][qq], P[s0 + q0 + qq], l[g]);
                                A[i + (k0 + q0 + qq) * m] = y[g][qq];
                                if (q0 + qq == c + 1) {
                                    const double n1 = (double)(fabs(y[g][qq].re) + fabs(y[g][qq].im));
                                    if (n1 > best) {  // rows ascend per thread: ties keep the first
                                        best = n1;
                                        bi = (int)i;
                                    }
                                }
                            }
                        }
                }
            }
            fused = c + 1 < w;
        }
        const int rest = NB - s0 - w;  // outer-panel columns right of the sub-panel
        if (rest <= 0) continue;
        // 5. the sub-panel is final everywhere
        if constexpr (kCluster) {
            cooperative_groups::this_cluster().sync();
        } else {
            if (!group_barrier(bar, (unsigned)per_matrix, args.error)) return;
        }
        // 6. U12 of the sub-panel: rows [k0, k0+w), columns [k0+w, K0+NB)
        if (slice == 0) {
            // the unit lower w x w block, staged once (U doubles as its buffer)
            for (int idx = tid; idx < kW * kW; idx += kThreads) {
                const int r = idx % kW, k = idx / kW;
                U[r][k] = (r < w && k < w) ? ldcg(A + (k0 + r) + (k0 + k) * m) : Cx<T>{0, 0};
            }
            __syncthreads();
            for (int t = tid; t < rest; t += kThreads) {
                const int64_t col = k0 + w + t;
                Cx<T> x[kW];
#pragma unroll
                for (int r = 0; r < kW; ++r)
                    if (r < w) x[r] = ldcg(A + (k0 + r) + col * m);
#pragma unroll
                for (int k = 0; k < kW; ++k) {
                    if (k >= w) break;
#pragma unroll
                    for (int r = k + 1; r < kW; ++r)
                        if (r < w) csubmul(x[r], x[k], U[r][k]);
                }
#pragma unroll
                for (int r = 0; r < kW; ++r)
                    if (r < w) A[(k0 + r) + col * m] = x[r];
            }
        }
        // 7. U12 is visible to every CTA (and slice 0 is done with U)
        if constexpr (kCluster) {
            cooperative_groups::this_cluster().sync();
        } else {
            if (!group_barrier(bar, (unsigned)per_matrix, args.error)) return;
        }
        // 8. own rows i >= k0+w: A[i, k0+w ..] -= A[i, k0 .. k0+w) U12
        for (int idx = tid; idx < w * rest; idx += kThreads) {
            const int r = idx / rest, t = idx % rest;
            U[r][t] = ldcg(A + (k0 + r) + (k0 + w + t) * m);
        }
        __syncthreads();
        // Column k0+w (t = 0) starts the next sub-panel: its arg-max is taken here.
        best = -1.0;
        bi = INT_MAX;
        // Columns go kT at a time, double-buffered: the loads of the next
        // batch are in flight while the current one is updated and stored
        // (the sub-panel width w is 16 here: only the last sub-panel is
        // narrower, and it has no columns to its right).
        constexpr int kT = 4;
        for (int64_t i = max(r_begin, k0 + w) + tid; i < r_end; i += kThreads) {
            const Cx<T> *row = A + i + (k0 + w) * m;  // column k0+w+t at row[t m]
            Cx<T> l[kW], y[kT], yn[kT];
#pragma unroll
            for (int r = 0; r < kW; ++r) l[r] = ldcg(A + i + (k0 + r) * m);
#pragma unroll
            for (int q = 0; q < kT; ++q)
                if (q < rest) y[q] = ldcg(row + (int64_t)q * m);
            for (int t0 = 0; t0 < rest; t0 += kT) {
                const int tn = t0 + kT;
#pragma unroll
                for (int q = 0; q < kT; ++q)
                    if (tn + q < rest) yn[q] = ldcg(row + (int64_t)(tn + q) * m);
#pragma unroll
                for (int q = 0; q < kT; ++q) {
                    if (t0 + q < rest) {
#pragma unroll
                        for (int r = 0; r < kW; ++r) csubmul(y[q], l[r], U[r][t0 + q]);
                        A[i + (k0 + w + t0 + q) * m] = y[q];
                    }
                }
                if (t0 == 0) {
                    const double n1 = (double)(fabs(y[0].re) + fabs(y[0].im));
                    if (n1 > best) {
                        best = n1;
                        bi = (int)i;
                    }
                }
#pragma unroll
                for (int q = 0; q < kT; ++q) y[q] = yn[q];
            }
        }
        fused = true;
        __syncthreads();
    }
    // No CTA leaves while another may still read its shared memory.
    if constexpr (kCluster) cooperative_groups::this_cluster().sync();
}

}  // namespace

// Largest cluster of CTAs of the cluster form that the device can schedule
// (0: none), for sizes up to kMaxCluster.
constexpr int kMaxCluster = 16;

template <class T>
int cluster_fits_query(int size);

// cluster_fits_query, asked once per device and size (the occupancy query
// costs milliseconds; sweeps ask on every batch).
template <class T>
int cluster_fits(int size) {
    if (size < 2 || size > kMaxCluster) return 0;
    static std::mutex mu;
    static int known[64][kMaxCluster + 1];
    static bool asked[64][kMaxCluster + 1] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 0;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (!asked[dev][size]) {
        known[dev][size] = cluster_fits_query<T>(size);
        asked[dev][size] = true;
    }
    return known[dev][size];
}

template <class T>
int cluster_fits_query(int size) {
    auto kernel = panel_coop_kernel<T, true>;
    if (size > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)size);
    cfg.blockDim = dim3(kThreads);
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = (unsigned)size;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, (void *)kernel, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return clusters;
}

template <class T>
fh_status coop_plan(int count, int64_t m, int *per_matrix, size_t *bytes, fh_error_info *err, int share) {
    int dev = 0, sms = 0, occ = 0, coop = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    FHB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    FHB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return fail(err, FH_ERR_NO_DEVICE, "the device does not support cooperative launches");
    FHB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_coop_kernel<T, false>, kThreads, 0));
    const int capacity = occ * sms / std::max(1, share);
    int pm = std::max(1, capacity / std::max(1, count));
    pm = (int)std::min<int64_t>(pm, std::max<int64_t>(1, (m + 63) / 64));
    // A batch whose matrices get at most kMaxCluster CTAs each runs them as
    // one cluster per matrix, of the largest size at which every matrix's
    // cluster (of every sweep sharing the device) is resident at once: a
    // second wave of clusters would double the panel's time.
    if (pm >= 2 && pm <= kMaxCluster) {
        int size = pm;
        while (size >= 2 && cluster_fits<T>(size) < count * std::max(1, share)) --size;
        if (size >= 2) pm = size;
    }
    if ((int64_t)pm * count > capacity)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "batch too large for one cooperative panel launch");
    *per_matrix = pm;
    const size_t slots = (size_t)count * pm * 2;
    *bytes = 128 + (size_t)count * kBarrierStride * 4 + slots * 8 + slots * 4 + slots * kNbMax * sizeof(Cx<T>) +
             (size_t)count * 2 * kNbMax * sizeof(Cx<T>) + 256;
    return FH_OK;
}

template <class T>
bool coop_cluster(int count, int per_matrix, int share) {
    return per_matrix >= 2 && per_matrix <= kMaxCluster &&
           cluster_fits<T>(per_matrix) >= count * std::max(1, share);
}

template <class T>
void coop_bind(void *mem, int count, int per_matrix, CoopScratch &cs, int share) {
    unsigned char *p = static_cast<unsigned char *>(mem);
    const size_t slots = (size_t)count * per_matrix * 2;
    // [error flag, 128 B] [one 128-byte barrier per matrix] [candidates] [rows j]
    cs.error = reinterpret_cast<int *>(p);
    cs.barrier = reinterpret_cast<unsigned *>(p + 128);
    size_t off = 128 + (size_t)count * kBarrierStride * 4;
    cs.cand_val = reinterpret_cast<double *>(p + off);
    off += slots * 8;
    cs.cand_row = reinterpret_cast<int *>(p + off);
    off += slots * 4;
    off = (off + 15) & ~(size_t)15;
    cs.cand_data = p + off;
    off += slots * kNbMax * sizeof(Cx<T>);
    cs.rowj = p + off;
    cs.per_matrix = per_matrix;
    cs.cluster = coop_cluster<T>(count, per_matrix, share);
}

template <class T>
fh_status panel_coop(LuBatch<T> &b, int64_t K0, int nb, const CoopScratch &cs, cudaStream_t s, fh_error_info *err) {
    if (nb > kNbMax) return fail(err, FH_ERR_INVALID_ARGUMENT, "cooperative panel wider than 128 columns");
    // Barrier counters are reset for every launch (a barrier that gave up may
    // leave arrivals behind); the error flag only at the start of a
    // factorization, so that coop_check sees a failure of any panel.
    FHB_CUDA(cudaMemsetAsync(cs.barrier, 0, (size_t)b.count * kBarrierStride * 4, s));
    if (K0 == 0) FHB_CUDA(cudaMemsetAsync(cs.error, 0, sizeof(int), s));
    CoopArgs args{cs.barrier, cs.error, cs.cand_val, cs.cand_row, cs.cand_data, cs.rowj, cs.per_matrix};
    Cx<T> *a = reinterpret_cast<Cx<T> *>(b.a);
    int64_t m = b.m;
    if (cs.cluster) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(cs.per_matrix * b.count));
        cfg.blockDim = dim3(kThreads);
        cfg.stream = s;
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = (unsigned)cs.per_matrix;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        FHB_CUDA(cudaLaunchKernelEx(&cfg, panel_coop_kernel<T, true>, a, m, K0, nb, b.pivots, b.singular, args));
        return FH_OK;
    }
    void *params[] = {&a, &m, &K0, &nb, &b.pivots, &b.singular, &args};
    FHB_CUDA(cudaLaunchCooperativeKernel((const void *)panel_coop_kernel<T, false>, dim3(cs.per_matrix * b.count),
                                         dim3(kThreads), params, 0, s));
    return FH_OK;
}

fh_status coop_check(const CoopScratch &cs, cudaStream_t s, fh_error_info *err) {
    int flag = 0;
    FHB_CUDA(cudaMemcpyAsync(&flag, cs.error, sizeof(int), cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    if (flag) return fail(err, FH_ERR_DEVICE_TIMEOUT, "a panel grid barrier ran out of its iteration limit");
    return FH_OK;
}

template fh_status coop_plan<double>(int, int64_t, int *, size_t *, fh_error_info *, int);
template fh_status coop_plan<float>(int, int64_t, int *, size_t *, fh_error_info *, int);
template void coop_bind<double>(void *, int, int, CoopScratch &, int);
template void coop_bind<float>(void *, int, int, CoopScratch &, int);
template bool coop_cluster<double>(int, int, int);
template bool coop_cluster<float>(int, int, int);
template fh_status panel_coop<double>(LuBatch<double> &, int64_t, int, const CoopScratch &, cudaStream_t, fh_error_info *);
template fh_status panel_coop<float>(LuBatch<float> &, int64_t, int, const CoopScratch &, cudaStream_t, fh_error_info *);

}  // namespace fhb
