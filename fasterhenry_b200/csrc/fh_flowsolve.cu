// Batched triangular solves with the FP32 factors of the two-level
// factorization without interchanges, as a dataflow over 128-row blocks:
//
//     x <- U^{-1} L^{-1} x        for every (matrix, right-hand side)
//
// The CTAs of one (matrix, right-hand side) pair form a group and own its
// row blocks cyclically (block i -> CTA i mod per_group).  Forward: a CTA
// takes its blocks in increasing order; for block i it subtracts L_ij y_j
// for j = 0 .. i-1 as each y_j is published (a flag per block), then forms
// y_i = Linv_i (b_i - sum) with the diagonal block's stored inverse, writes
// it over b_i and publishes it.  Backward: its blocks in decreasing order,
// x_i = Uinv_i (y_i - sum_{j > i} U_ij x_j), the x_j taken from the last
// block down.  There is no barrier over the group: only one source block
// and one inverse per block lie on the chain from block to block, while
// the other CTAs stream their blocks' contributions, so the reads of the
// factors (8 m^2 bytes per solve) overlap the chain.  Every block's
// contributions are subtracted in block order, as a right-looking solve
// does.
//
// The factor tiles and the inverses reach shared memory through a ring of
// TMA loads issued ahead along each CTA's fixed sequence of tiles: the
// factors do not change during the solve, so a CTA waits only for the
// 128-entry vector pieces, never for a tile of the factor.
//
// Publication: the block's entries are written, __threadfence, barrier,
// then thread 0 stores the flag with release semantics; a reader's thread 0
// polls the flag with acquire loads, then a barrier, then all threads read
// the entries through L2.  Flags hold the launch's epoch (the caller zeroes
// them once per batch), so no reset is needed between solves.  Every wait
// (flags and the ring's mbarriers) is bounded: one that runs out, or that
// sees the error flag raised by another CTA, raises the error flag and the
// CTA returns after its loads in flight have landed.  The CTAs of a launch
// are co-resident (cooperative launch), so the earliest unfinished block of
// a group always has all it needs.
#include <algorithm>
#include <string>

#include <cuda.h>

#include "fh_cx.cuh"
#include "fh_lu.cuh"

namespace fhb {
namespace {

constexpr int kFlowThreads = 256;
constexpr int kNb = 128;
constexpr long long kFlowSpin = 1LL << 22;

struct FlowArgs {
    const Cx<float> *a;
    int64_t m;
    int count, nrhs, nblk, per_group;
    const Cx<float> *linv, *uinv;  // slot k: count * nb * nb, matrix f at + f * nb * nb; (r, c) at r + c * wk
    Cx<float> *x;                  // (f * nrhs + q) * m
    unsigned *flags;               // [group][2][nblk]: forward, backward
    unsigned epoch;
    int *error;
};

__device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void store_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0 waits (bounded) for *flag == epoch; the CTA then meets at a
// barrier.  False (for every thread) when the wait ran out or an error was
// raised.
__device__ __forceinline__ bool flow_wait(const unsigned *flag, unsigned epoch, int *error) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 0;
        for (long long i = 0; i < kFlowSpin; ++i) {
            if (load_acquire(flag) == epoch) {
                ok = 1;
                break;
            }
            if (*(volatile int *)error) break;
            __nanosleep(64);
        }
        if (!ok) atomicExch(error, 1);
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Factor tiles and the blocks' inverses stream through a ring of
// kFlowStages shared-memory tiles of 128 rows x 32 columns (32 KB): a factor
// tile by one 2D TMA load (rows past m read as zeros), an inverse tile by a
// bulk copy of its kFlowTileCols contiguous columns.  The loads run ahead along the
// CTA's own sequence of tiles, independent of the flags: the factors do not
// change during the solve, so only the vector pieces wait.
constexpr int kFlowTileCols = 32;
constexpr int kFlowStages = 3;
constexpr int kFlowTileElems = kNb * kFlowTileCols;
constexpr int kFlowTileBytes = kFlowTileElems * 8;
constexpr int kFlowTilesPerBlock = kNb / kFlowTileCols;
constexpr int kFlowWarpCols = kFlowTileCols / (kFlowThreads / 32);  // backward: a warp's columns per tile
static_assert(kFlowTilesPerBlock * kFlowWarpCols * 2 == 32, "backward sums: one value per lane");
constexpr int kFlowSmemBytes = kFlowStages * kFlowTileBytes + kFlowStages * 8;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kFlowSpin; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// Plain (non-multicast) loads into this CTA's shared memory.
__device__ __forceinline__ void tensor_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Position in a CTA's tile sequence: forward blocks i = slice, slice + P, ...
// then backward blocks from the last down; per block its source blocks
// (forward j = 0 .. i-1, backward j = nblk-1 .. i+1), then its inverse, each
// as kFlowTilesPerBlock tiles of kFlowTileCols columns.
struct TileCursor {
    int pass;  // 0 forward, 1 backward, 2 done
    int i;     // output block
    int s;     // source index; s == nsrc() is the block's inverse
    int q;     // tile of kFlowTileCols columns
    __device__ int nsrc(int nblk) const { return pass == 0 ? i : nblk - 1 - i; }
    __device__ void start(int slice) {
        pass = 0;
        i = slice;
        s = 0;
        q = 0;
    }
    __device__ void next(int slice, int per_group, int nblk) {
        if (++q < kFlowTilesPerBlock) return;
        q = 0;
        if (++s <= nsrc(nblk)) return;
        s = 0;
        if (pass == 0) {
            i += per_group;
            if (i >= nblk) {
                pass = 1;
                i = slice + ((nblk - 1 - slice) / per_group) * per_group;
            }
        } else if ((i -= per_group) < 0) {
            pass = 2;
        }
    }
};

// Thread 0: starts the load of tile t into the ring slot at dst, completion
// counted on bar.  An inverse tile past the block's columns loads nothing
// (the barrier still completes).
__device__ __forceinline__ void issue_tile(const FlowArgs &g, const CUtensorMap *map, int f, const TileCursor &t,
                                           uint32_t dst, uint32_t bar) {
    if (t.s < t.nsrc(g.nblk)) {
        // forward: L_ij (rows of block i, columns of block j); backward:
        // L_ji (rows of block j, columns of block i), read transposed
        const int j = t.pass == 0 ? t.s : g.nblk - 1 - t.s;
        const int rb = t.pass == 0 ? t.i : j, cb = t.pass == 0 ? j : t.i;
        mbar_expect_tx(bar, kFlowTileBytes);
        tensor_load_2d(dst, map, rb * kNb, (int)((int64_t)f * g.m + (int64_t)cb * kNb + t.q * kFlowTileCols), bar);
    } else {
        const int wi = (int)min((int64_t)kNb, g.m - (int64_t)t.i * kNb), c0 = t.q * kFlowTileCols;
        const uint32_t bytes = (uint32_t)max(0, min(kFlowTileCols, wi - c0)) * wi * 8;
        mbar_expect_tx(bar, bytes);
        if (bytes) {
            const Cx<float> *inv = (t.pass == 0 ? g.linv : g.uinv) + (size_t)t.i * g.count * kNb * kNb +
                                   (size_t)f * kNb * kNb + (size_t)c0 * wi;
            bulk_load(dst, inv, bytes, bar);
        }
    }
}

__global__ void __launch_bounds__(kFlowThreads) flowsolve_kernel(FlowArgs g, const __grid_constant__ CUtensorMap map) {
    extern __shared__ __align__(128) unsigned char flow_smem[];
    const Cx<float> *ring = reinterpret_cast<const Cx<float> *>(flow_smem);
    uint64_t *full = reinterpret_cast<uint64_t *>(flow_smem + kFlowStages * kFlowTileBytes);
    const int grp = blockIdx.x / g.per_group, slice = blockIdx.x % g.per_group;
    const int f = grp / g.nrhs;
    const int64_t m = g.m;
    Cx<float> *X = g.x + (int64_t)grp * m;
    unsigned *ff = g.flags + (size_t)grp * 2 * g.nblk, *fb = ff + g.nblk;
    const int tid = threadIdx.x, r = tid % kNb, h = tid / kNb, warp = tid >> 5, lane = tid & 31;
    const Cx<float> *Af = g.a + (int64_t)f * m * m;
    __shared__ __align__(16) Cx<float> vs[kNb], part[kNb];

    if (tid == 0) {
        for (int k = 0; k < kFlowStages; ++k) mbar_init(smem_addr(&full[k]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // Tile t goes to slot t % kFlowStages; its barrier phase is t / kFlowStages.
    TileCursor issue;
    issue.start(slice);
    long long t_issue = 0, t_comp = 0;
    auto issue_next = [&]() {
        if (issue.pass == 2) return;
        if (tid == 0) {
            const int slot = (int)(t_issue % kFlowStages);
            issue_tile(g, &map, f, issue, smem_addr(ring + slot * kFlowTileElems), smem_addr(&full[slot]));
        }
        issue.next(slice, g.per_group, g.nblk);
        ++t_issue;
    };
    for (int k = 0; k < kFlowStages; ++k) issue_next();

    // Waits for the next tile, acc += tile(r, c) v[c] over this half's
    // columns c < ncols (column stride ld), then frees the slot and starts
    // the next load into it.  False for every thread when a wait ran out.
    auto step = [&](const Cx<float> *v, int ld, int ncols, Cx<float> &acc) -> bool {
        const int slot = (int)(t_comp % kFlowStages);
        const bool ok = mbar_wait(smem_addr(&full[slot]), (uint32_t)((t_comp / kFlowStages) & 1));
        if (ok) {
            const Cx<float> *tile = ring + slot * kFlowTileElems;
#pragma unroll
            for (int k = 0; k < kFlowTileCols / 2; ++k) {
                const int c = h * (kFlowTileCols / 2) + k;
                if (c < ncols) {
                    const Cx<float> l = tile[c * ld + r], x = v[c];
                    acc.re += l.re * x.re - l.im * x.im;
                    acc.im += l.re * x.im + l.im * x.re;
                }
            }
        } else {
            atomicExch(g.error, 1);
        }
        if (!__syncthreads_and(ok)) return false;
        ++t_comp;
        issue_next();
        return true;
    };

    // Backward source tile q (L_ji, 128 rows of block j x kFlowTileCols
    // columns of block i): t[q][c] += sum_r L_ji(r, q kFlowTileCols +
    // kFlowWarpCols warp + c) x_j(r) over the lane's rows r = 4 lane ..
    // 4 lane + 3, kept per lane until the block's sources are done
    // (U_ij = D_i L_ji^T, so U is never read).
    float bt[kFlowTilesPerBlock][kFlowWarpCols][2];
    auto step_t = [&](int q, const Cx<float> (&xr)[4]) -> bool {
        const int slot = (int)(t_comp % kFlowStages);
        const bool ok = mbar_wait(smem_addr(&full[slot]), (uint32_t)((t_comp / kFlowStages) & 1));
        if (ok) {
            const Cx<float> *tile = ring + slot * kFlowTileElems;
#pragma unroll
            for (int c = 0; c < kFlowWarpCols; ++c) {
                const float4 *col = reinterpret_cast<const float4 *>(tile + (kFlowWarpCols * warp + c) * kNb + 4 * lane);
                const float4 p0 = col[0], p1 = col[1];  // rows 4 lane, +1 | +2, +3
                bt[q][c][0] += p0.x * xr[0].re - p0.y * xr[0].im + p0.z * xr[1].re - p0.w * xr[1].im +
                               p1.x * xr[2].re - p1.y * xr[2].im + p1.z * xr[3].re - p1.w * xr[3].im;
                bt[q][c][1] += p0.x * xr[0].im + p0.y * xr[0].re + p0.z * xr[1].im + p0.w * xr[1].re +
                               p1.x * xr[2].im + p1.y * xr[2].re + p1.z * xr[3].im + p1.w * xr[3].re;
            }
        } else {
            atomicExch(g.error, 1);
        }
        if (!__syncthreads_and(ok)) return false;
        ++t_comp;
        issue_next();
        return true;
    };

    // One output block: its sources as their flags come, then the stored
    // inverse of the diagonal block, then publication.  Forward
    // y_i = Linv_i (b_i - sum_j L_ij y_j); backward
    // x_i = Uinv_i (y_i - D_i sum_j L_ji^T x_j), D_i the diagonal of U.
    auto block = [&](int pass, int i) -> bool {
        const int64_t i0 = (int64_t)i * kNb;
        const int wi = (int)min((int64_t)kNb, m - i0);
        unsigned *flags = pass == 0 ? ff : fb;
        Cx<float> acc{0.f, 0.f}, dii{0.f, 0.f};
        if (h == 0 && r < wi) {
            acc = ldcg(X + i0 + r);
            if (pass == 1) dii = Af[(i0 + r) * (m + 1)];
        }
        const int nsrc = pass == 0 ? i : g.nblk - 1 - i;
        if (pass == 1) {
#pragma unroll
            for (int q = 0; q < kFlowTilesPerBlock; ++q)
#pragma unroll
                for (int c = 0; c < kFlowWarpCols; ++c) bt[q][c][0] = bt[q][c][1] = 0.f;
        }
        for (int s = 0; s < nsrc; ++s) {
            const int j = pass == 0 ? s : g.nblk - 1 - s;
            if (!flow_wait(flags + j, g.epoch, g.error)) return false;
            const int64_t j0 = (int64_t)j * kNb;
            const int wj = (int)min((int64_t)kNb, m - j0);
            if (tid < kNb) {  // forward: negated, the steps accumulate -L_ij y_j
                const Cx<float> x = tid < wj ? ldcg(X + j0 + tid) : Cx<float>{0.f, 0.f};
                vs[tid] = pass == 0 ? Cx<float>{-x.re, -x.im} : x;
            }
            __syncthreads();
            if (pass == 0) {
                for (int q = 0; q < kFlowTilesPerBlock; ++q)
                    if (!step(vs + q * kFlowTileCols, kNb, wj - q * kFlowTileCols, acc)) return false;
            } else {
                Cx<float> xr[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) xr[k] = vs[4 * lane + k];
#pragma unroll
                for (int q = 0; q < kFlowTilesPerBlock; ++q)
                    if (!step_t(q, xr)) return false;
            }
        }
        if (pass == 0) {
            if (h == 1) part[r] = acc;
        } else {
            // Sum bt over the warp's lanes: each halving exchanges half of the
            // remaining values, so lane l ends with the total of value l,
            // which is part of column q kFlowTileCols + kFlowWarpCols warp + c
            // (l = 2 (kFlowWarpCols q + c) + re/im).
            float v[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) v[k] = bt[(k >> 1) / kFlowWarpCols][(k >> 1) % kFlowWarpCols][k & 1];
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) {
                const bool hi = (lane & off) != 0;
#pragma unroll
                for (int k = 0; k < off; ++k) {
                    const float send = hi ? v[k] : v[k + off], keep = hi ? v[k + off] : v[k];
                    v[k] = keep + __shfl_xor_sync(0xffffffffu, send, off);
                }
            }
            const int q = (lane >> 1) / kFlowWarpCols, c = (lane >> 1) % kFlowWarpCols;
            reinterpret_cast<float *>(part)[(q * kFlowTileCols + kFlowWarpCols * warp + c) * 2 + (lane & 1)] = v[0];
        }
        __syncthreads();
        if (h == 0) {
            Cx<float> y{0.f, 0.f};
            if (r < wi) {
                const Cx<float> t = part[r];
                y = pass == 0 ? Cx<float>{acc.re + t.re, acc.im + t.im}
                              : Cx<float>{acc.re - (dii.re * t.re - dii.im * t.im),
                                          acc.im - (dii.re * t.im + dii.im * t.re)};
            }
            vs[r] = y;
        }
        __syncthreads();
        Cx<float> out{0.f, 0.f};
        for (int q = 0; q < kFlowTilesPerBlock; ++q)
            if (!step(vs + q * kFlowTileCols, wi, wi - q * kFlowTileCols, out)) return false;
        if (h == 1) part[r] = out;
        __syncthreads();
        if (h == 0 && r < wi) X[i0 + r] = Cx<float>{out.re + part[r].re, out.im + part[r].im};
        __threadfence();
        __syncthreads();
        if (tid == 0) store_release(flags + i, g.epoch);
        return true;
    };

    bool ok = true;
    // ---------------- forward: y <- L^{-1} b ----------------
    for (int i = slice; ok && i < g.nblk; i += g.per_group) ok = block(0, i);
    // ---------------- backward: x <- U^{-1} y ----------------
    const int last = slice + ((g.nblk - 1 - slice) / g.per_group) * g.per_group;
    for (int i = last; ok && i >= 0; i -= g.per_group) ok = block(1, i);
    // After an error: no load outlives the CTA (each wait bounded).
    if (!ok && tid == 0)
        for (long long t = t_comp; t < t_issue; ++t)
            mbar_wait(smem_addr(&full[t % kFlowStages]), (uint32_t)((t / kFlowStages) & 1));
}

}  // namespace

fh_status flowsolve_plan(int groups, int64_t m, int *per_group, size_t *bytes, fh_error_info *err, int share) {
    int dev = 0, sms = 0, occ = 0, coop = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    FHB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    FHB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return fail(err, FH_ERR_NO_DEVICE, "the device does not support cooperative launches");
    FHB_CUDA(cudaFuncSetAttribute(flowsolve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kFlowSmemBytes));
    FHB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, flowsolve_kernel, kFlowThreads, kFlowSmemBytes));
    const int capacity = occ * sms / std::max(1, share);
    const int nblk = (int)((m + kNb - 1) / kNb);
    // the tensor map needs an even order and 32-bit column coordinates
    if (groups <= 0 || groups > capacity || m <= 0 || m % 2 || (int64_t)groups * m + kNb > INT32_MAX) {
        *per_group = 0;  // the caller uses the barrier-based cooperative solve
        *bytes = 0;
        return FH_OK;
    }
    *per_group = std::max(1, std::min(nblk, capacity / groups));
    *bytes = 128 + (size_t)groups * 2 * nblk * sizeof(unsigned);
    return FH_OK;
}

void flowsolve_bind(void *mem, int groups, int per_group, int64_t m, FlowScratch &fs) {
    unsigned char *p = static_cast<unsigned char *>(mem);
    fs.error = reinterpret_cast<int *>(p);
    fs.flags = reinterpret_cast<unsigned *>(p + 128);
    fs.groups = groups;
    fs.per_group = per_group;
    fs.nblk = (int)((m + kNb - 1) / kNb);
    fs.epoch = 0;
}

fh_status lu_solve_flow(const LuBatch<float> &b, const void *linv, const void *uinv, float *x, int nrhs,
                        FlowScratch &fs, cudaStream_t s, fh_error_info *err) {
    if (b.m == 0 || b.count == 0 || nrhs == 0) return FH_OK;
    if (!linv || !uinv) return fail(err, FH_ERR_INVALID_ARGUMENT, "dataflow solve needs the block inverses");
    if (fs.per_group <= 0 || fs.groups != b.count * nrhs || fs.nblk != (int)((b.m + kNb - 1) / kNb))
        return fail(err, FH_ERR_INVALID_ARGUMENT, "dataflow solve scratch does not match the batch");
    FlowArgs g;
    g.a = reinterpret_cast<const Cx<float> *>(b.a);
    g.m = b.m;
    g.count = b.count;
    g.nrhs = nrhs;
    g.nblk = fs.nblk;
    g.per_group = fs.per_group;
    g.linv = reinterpret_cast<const Cx<float> *>(linv);
    g.uinv = reinterpret_cast<const Cx<float> *>(uinv);
    g.x = reinterpret_cast<Cx<float> *>(x);
    g.flags = fs.flags;
    g.epoch = ++fs.epoch;
    g.error = fs.error;
    alignas(64) CUtensorMap map;
    fh_status st = encode_column_tiles(&map, b.a, b.m, b.count, kNb, kFlowTileCols, err);
    if (st) return st;
    void *params[] = {&g, &map};
    prof_begin(s, FH_PROF_SOLVE_FLOW);
    FHB_CUDA(cudaLaunchCooperativeKernel((const void *)flowsolve_kernel, dim3(fs.groups * fs.per_group),
                                         dim3(kFlowThreads), params, kFlowSmemBytes, s));
    prof_end(s, FH_PROF_SOLVE_FLOW, 8.0 * (double)b.m * (double)b.m * nrhs * b.count);
    return FH_OK;
}

fh_status flowsolve_check(const FlowScratch &fs, cudaStream_t s, fh_error_info *err) {
    int flag = 0;
    FHB_CUDA(cudaMemcpyAsync(&flag, fs.error, sizeof(int), cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    if (flag) {
        cudaMemsetAsync(fs.error, 0, sizeof(int), s);
        return fail(err, FH_ERR_DEVICE_TIMEOUT, "a triangular-solve flag wait ran out of its iteration limit");
    }
    return FH_OK;
}

}  // namespace fhb
