// C ABI of the device path: the dense system (MeshSystem), sweeps, and the
// library-level kernels (fill, LU).  See include/fasterhenry_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <atomic>
#include <mutex>
#include <thread>

#include "fh_batchsolve.h"
#include "fh_device.cuh"
#include "fh_lu.cuh"

using namespace fhb;

// Device workspace of a system's sweeps, kept between calls: one buffer per
// role (slot), grown when a sweep needs more.  Repeated sweeps then allocate
// nothing, and no cudaFree (which synchronizes the device) runs inside a
// sweep after the first.
struct DevPool {
    std::vector<std::pair<void *, size_t>> slot;
    cudaStream_t stream = nullptr;  // the owner's stream: allocations and frees are ordered on it
    ~DevPool() { release(); }
    void release() {
        for (auto &b : slot)
            if (b.first) cache_free(b.first, stream);
        slot.clear();
    }
    size_t held() const {
        size_t t = 0;
        for (const auto &b : slot) t += b.second;
        return t;
    }
    cudaError_t get(int id, size_t bytes, void **out) {
        if ((int)slot.size() <= id) slot.resize((size_t)id + 1, {nullptr, 0});
        auto &b = slot[(size_t)id];
        if (b.second < bytes) {
            if (b.first) cache_free(b.first, stream);
            b = {nullptr, 0};
            const cudaError_t e = cache_alloc(&b.first, std::max<size_t>(bytes, 1), stream);
            if (e != cudaSuccess) {
                b.first = nullptr;
                return e;
            }
            b.second = bytes;
        }
        *out = b.first;
        return cudaSuccess;
    }
};

struct fh_system {
    DevPool pool;
    // Sweeps of this many systems may run at once (fh_batch_sweep): the
    // cooperative kernels and the batch sizing take 1 / share of the device.
    int share = 1;
    std::vector<fh_node> nodes;
    std::vector<fh_segment_def> segments;
    std::vector<fh_port> ports;
    Discretized disc;
    LoopBasis loops;
    std::vector<double> resistances;
    int64_t n = 0, nloops = 0, m = 0, p = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    // The factorization's look-ahead stream, joined to `stream` before each
    // factorization returns.
    cudaStream_t side = nullptr;
    double *d_Lm = nullptr, *d_Rm = nullptr;
    // Layout (currents.rs:128-170) and, once currents are asked for, the
    // transposed loop basis and per-filament (w, h, R) on the device.
    std::vector<int64_t> segment_of_filament, conductor_of_segment, segment_first;
    int64_t conductors = 0;
    // Coupling (coupling.rs): resolved groups, warnings, kept pairs, and the
    // device mask when it truncates.
    CouplingResolved coupling;
    std::vector<fh_truncation_warning> warnings;
    int64_t kept_pairs = 0, total_pairs = 0;
    int32_t *d_group = nullptr;
    uint8_t *d_coupled = nullptr;
    PairMaskDev mask() const {
        PairMaskDev m;
        if (coupling.all_pairs) return m;
        m.group = d_group;
        m.coupled = d_coupled;
        m.groups = (int32_t)coupling.groups();
        m.dropped = total_pairs - kept_pairs;
        return m;
    }
    int64_t *d_col_ptr = nullptr, *d_first = nullptr;
    int32_t *d_col_loop = nullptr;
    double *d_col_sign = nullptr, *d_whr = nullptr;
    // The loop basis, its transpose over the internal loops and the branch
    // resistances on the device: R_ee x of the refinement residuals.
    int64_t *d_rp = nullptr, *d_toff = nullptr;
    int32_t *d_br = nullptr, *d_tloop = nullptr;
    double *d_sign = nullptr, *d_tsign = nullptr, *d_R = nullptr;
    fh_counts counts{};
    fh_timing timing{};
    FillStats fill{};
    float ms_congruence = 0;
    ~fh_system() {
        pool.release();
        cache_free(d_Lm, stream);
        cache_free(d_Rm, stream);
        for (void *q : {(void *)d_rp, (void *)d_toff, (void *)d_br, (void *)d_tloop, (void *)d_sign, (void *)d_tsign,
                        (void *)d_R})
            cache_free(q, stream);
        cache_free(d_col_ptr, stream);
        cache_free(d_first, stream);
        cache_free(d_col_loop, stream);
        cache_free(d_col_sign, stream);
        cache_free(d_whr, stream);
        cache_free(d_group, stream);
        cache_free(d_coupled, stream);
        if (side) {
            cudaStreamSynchronize(side);
            cudaStreamDestroy(side);
        }
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace fhb {

// CUDA events that are destroyed on every return path of the scope that
// holds them (error returns and time-outs included).
template <int N>
struct ScopedEvents {
    cudaEvent_t e[N] = {};
    ScopedEvents() {
        for (auto &x : e) cudaEventCreate(&x);
    }
    ~ScopedEvents() {
        for (auto &x : e)
            if (x) cudaEventDestroy(x);
    }
    ScopedEvents(const ScopedEvents &) = delete;
    ScopedEvents &operator=(const ScopedEvents &) = delete;
};


fh_status ensure_device(fh_error_info *err) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(err, FH_ERR_NO_DEVICE, "no CUDA device is available (this library has no CPU fallback)");
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return fail(err, FH_ERR_NO_DEVICE, "cannot query the CUDA device");
    if (prop.major != 10)
        return fail(err, FH_ERR_NO_DEVICE,
                    std::string("this build targets sm_100a (B200); found ") + prop.name + " sm_" +
                        std::to_string(prop.major) + std::to_string(prop.minor));
    return FH_OK;
}

namespace {

// RAII device buffer.  With a stream, allocated from the memory cache and
// freed in that stream's order; without, plain cudaMalloc / cudaFree.
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    bool cached = false;
    DBuf() = default;
    explicit DBuf(cudaStream_t stream) : s(stream), cached(true) {}
    DBuf(const DBuf &) = delete;
    ~DBuf() {
        if (!p) return;
        if (cached) cache_free(p, s);
        else cudaFree(p);
    }
    cudaError_t alloc(size_t count) {
        n = count;
        const size_t bytes = std::max<size_t>(1, count) * sizeof(T);
        return cached ? cache_alloc((void **)&p, bytes, s) : cudaMalloc((void **)&p, bytes);
    }
};

// A view of a pooled buffer (the pool owns the memory).
template <class T>
struct PBuf {
    T *p = nullptr;
};

// Workspace slots of the sweep paths (FP64 and mixed share the roles they have
// in common, so the larger of the two is kept).
enum PoolSlot {
    kSlotA, kSlotD32, kSlotR, kSlotRnorm, kSlotBnorm, kSlotDnorm, kSlotXnorm, kSlotPiv, kSlotSing, kSlotPv,
    kSlotPi, kSlotTk, kSlotCoop, kSlotLinv, kSlotUinv, kSlotSolve, kSlotPackA, kSlotPackB, kSlotOmega, kSlotX,
    kSlotZ, kSlotXinv, kSlotXpack, kSlotTbuf, kSlotDvec, kSlotFlow, kSlotResPart, kSlotSparseT, kSlotSparseY,
    kSlotTileCounter,
    // the persistent batched solve (fh_batch_sweep, mixed), in the first system's pool
    kSlotBatchSys, kSlotBatchOne, kSlotBatchItems, kSlotBatchZ, kSlotBatchStatus, kSlotBatchCounter, kSlotBatchWork
};

#define FHB_PALLOC(pool, buf, slot_id, count)                                                          \
    do {                                                                                               \
        void *pp_ = nullptr;                                                                           \
        if ((pool).get((slot_id), (size_t)(count) * sizeof(*(buf).p), &pp_) != cudaSuccess) {         \
            cudaGetLastError();                                                                        \
            return fail(err, FH_ERR_OUT_OF_MEMORY,                                                     \
                        "device allocation of " + std::to_string((size_t)(count) * sizeof(*(buf).p)) + \
                            " bytes failed");                                                          \
        }                                                                                              \
        (buf).p = static_cast<decltype((buf).p)>(pp_);                                                 \
    } while (0)

#define FHB_ALLOC(buf, count)                                                                   \
    do {                                                                                        \
        if ((buf).alloc(count) != cudaSuccess) {                                                \
            cudaGetLastError();                                                                 \
            return fail(err, FH_ERR_OUT_OF_MEMORY,                                              \
                        "device allocation of " + std::to_string((size_t)(count) * sizeof(*(buf).p)) + \
                            " bytes failed");                                                   \
        }                                                                                       \
    } while (0)

double wall() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

std::string fstr(double v) {
    char b[64];
    snprintf(b, sizeof b, "%g", v);
    return b;
}

constexpr double kTau = 6.283185307179586;
// Outer panel widths: FP64 stays at 64 (shared-memory budget of its TRSM and
// SIMT update); the FP32 form uses 128, which halves the trailing update's
// C traffic per flop.
constexpr int kNbFp64 = 64;
constexpr int kNbFp32 = 128;
// Super-panel width of the two-level FP32 factorization on the tensor cores:
// the deep trailing update runs with K = 512, four times the arithmetic per
// byte of C of a one-panel update.
constexpr int kOuterFp32 = 512;

// Super-panel width used for an FP32 batch of order m (0: one-level).
int outer_for(int64_t m, TrailingUpdate mode) {
    return mode == TrailingUpdate::TensorBf16x3 && m > kOuterFp32 ? kOuterFp32 : 0;
}

// Factor + solve + Schur for `count` frequencies in FP64.  x_out (count x m x
// p complex) receives the FP64 solutions; z (count x p x p) the impedances.
fh_status sweep_chunk_fp64(fh_system *s, const double *d_omega, int count, double *d_x, double *d_z, int *h_singular,
                           float *ms_factor, fh_error_info *err) {
    const int64_t m = s->m, p = s->p, ld = s->nloops;
    cudaStream_t st = s->stream;
    if (m > 0) {
        PBuf<double> a;
        PBuf<int> piv, sing;
        FHB_PALLOC(s->pool, a, kSlotA, (size_t)count * m * m * 2);
        FHB_PALLOC(s->pool, piv, kSlotPiv, (size_t)count * m);
        FHB_PALLOC(s->pool, sing, kSlotSing, (size_t)count);
        FHB_CUDA(cudaMemsetAsync(sing.p, 0, sizeof(int) * count, st));
        fh_status e = form_system<double>(s->d_Rm, s->d_Lm, ld, m, d_omega, count, a.p, st, err);
        if (e) return e;
        e = form_rhs<double>(s->d_Rm, s->d_Lm, ld, m, p, d_omega, count, d_x, st, err);
        if (e) return e;
        LuWork w;
        PBuf<double> pv;
        PBuf<int> pi;
        PBuf<unsigned> tk;
        w.max_chunks = 16;
        FHB_PALLOC(s->pool, pv, kSlotPv, (size_t)count * w.max_chunks);
        FHB_PALLOC(s->pool, pi, kSlotPi, (size_t)count * w.max_chunks);
        FHB_PALLOC(s->pool, tk, kSlotTk, (size_t)count);
        FHB_CUDA(cudaMemsetAsync(tk.p, 0, sizeof(unsigned) * count, st));
        w.partial_val = pv.p;
        w.partial_idx = pi.p;
        w.tickets = tk.p;
        CoopScratch cs;
        PBuf<unsigned char> coop_mem;
        int per_matrix = 0;
        size_t coop_bytes = 0;
        e = coop_plan<double>(count, m, &per_matrix, &coop_bytes, err, s->share);
        if (e) return e;
        FHB_PALLOC(s->pool, coop_mem, kSlotCoop, coop_bytes);
        coop_bind<double>(coop_mem.p, count, per_matrix, cs, s->share);
        w.coop = &cs;
        PBuf<double> linv_mem;
        FHB_PALLOC(s->pool, linv_mem, kSlotLinv, (size_t)count * kNbFp64 * kNbFp64 * 2);
        w.linv = linv_mem.p;
        LuBatch<double> b;
        b.a = a.p;
        b.pivots = piv.p;
        b.singular = sing.p;
        b.m = m;
        b.count = count;
        ScopedEvents<2> ev;
        cudaEventRecord(ev.e[0], st);
        e = lu_factor<double>(b, w, kNbFp64, TrailingUpdate::Simt, st, err);
        cudaEventRecord(ev.e[1], st);
        if (!e) e = lu_solve<double>(b, d_x, (int)p, kNbFp64, st, err);
        if (e) return e;
        FHB_CUDA(cudaMemcpyAsync(h_singular, sing.p, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]);
        if (ms_factor) *ms_factor += ms;
    } else {
        std::fill(h_singular, h_singular + count, 0);
    }
    return schur(s->d_Rm, s->d_Lm, ld, m, p, d_omega, count, d_x, d_z, st, err);
}

// Mixed form: FP32 factors (trailing updates on the tensor cores when
// available), FP64 residuals, iterative refinement of x.  Frequencies that do
// not converge are flagged in h_failed.
fh_status sweep_chunk_mixed(fh_system *s, const double *d_omega, int count, double *d_x, double *d_z, int *h_singular,
                            int *h_failed, int32_t *iters_out, double *resid_out, float *ms_factor, float *ms_refine,
                            TrailingUpdate mode, fh_error_info *err) {
    const int64_t m = s->m, p = s->p, ld = s->nloops;
    cudaStream_t st = s->stream;
    std::fill(h_failed, h_failed + count, 0);
    if (m == 0) {
        std::fill(h_singular, h_singular + count, 0);
        return schur(s->d_Rm, s->d_Lm, ld, m, p, d_omega, count, d_x, d_z, st, err);
    }
    PBuf<float> a, d32;
    PBuf<double> r, rnorm, bnorm, dnorm, xnorm;
    PBuf<int> piv, sing;
    const int64_t vec = m * p;  // complex entries per frequency
    // The FP32 system is factored at an even order mo: an odd Z_ee is bordered
    // by one row and column of the identity, [Z_ee 0; 0 1], whose factors are
    // Z_ee's plus a unit pivot and whose solve leaves the extra entry at zero.
    // The column stride is then a multiple of 16 bytes, which the tensor
    // copies of the rows-below pass and of the dataflow solve need.
    const int64_t mo = m + (m & 1);
    const int64_t vec32 = mo * p;  // complex entries per frequency, FP32 corrections
    DevPool &pool = s->pool;
    FHB_PALLOC(pool, a, kSlotA, (size_t)count * mo * mo * 2);
    FHB_PALLOC(pool, d32, kSlotD32, (size_t)count * vec32 * 2);
    FHB_PALLOC(pool, r, kSlotR, (size_t)count * vec * 2);
    FHB_PALLOC(pool, rnorm, kSlotRnorm, (size_t)count);
    FHB_PALLOC(pool, bnorm, kSlotBnorm, (size_t)count);
    FHB_PALLOC(pool, dnorm, kSlotDnorm, (size_t)count);
    FHB_PALLOC(pool, xnorm, kSlotXnorm, (size_t)count);
    FHB_PALLOC(pool, piv, kSlotPiv, (size_t)count * mo);
    FHB_PALLOC(pool, sing, kSlotSing, (size_t)count);
    FHB_CUDA(cudaMemsetAsync(sing.p, 0, sizeof(int) * count, st));
    // The two-level form factors without pivoting and forms every U entry it
    // reads from L: the tiles above the diagonal are not needed.
    fh_status e =
        form_system<float>(s->d_Rm, s->d_Lm, ld, m, d_omega, count, a.p, st, err, outer_for(mo, mode) > 0, mo);
    if (e) return e;
    e = form_rhs<double>(s->d_Rm, s->d_Lm, ld, m, p, d_omega, count, r.p, st, err);  // r0 = b
    if (e) return e;
    e = max_abs_per_matrix(r.p, 2 * vec, count, bnorm.p, st, err);
    if (e) return e;
    FHB_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * 2 * count * vec, st));
    LuWork w;
    PBuf<double> pv;
    PBuf<int> pi;
    PBuf<unsigned> tk;
    w.max_chunks = 16;
    FHB_PALLOC(pool, pv, kSlotPv, (size_t)count * w.max_chunks);
    FHB_PALLOC(pool, pi, kSlotPi, (size_t)count * w.max_chunks);
    FHB_PALLOC(pool, tk, kSlotTk, (size_t)count);
    FHB_CUDA(cudaMemsetAsync(tk.p, 0, sizeof(unsigned) * count, st));
    w.partial_val = pv.p;
    w.partial_idx = pi.p;
    w.tickets = tk.p;
    CoopScratch cs;
    PBuf<unsigned char> coop_mem;
    int per_matrix = 0;
    size_t coop_bytes = 0;
    e = coop_plan<float>(count, mo, &per_matrix, &coop_bytes, err, s->share);
    if (e) return e;
    FHB_PALLOC(pool, coop_mem, kSlotCoop, coop_bytes);
    coop_bind<float>(coop_mem.p, count, per_matrix, cs, s->share);
    w.coop = &cs;
    const int outer = outer_for(mo, mode);
    // Two-level form: the inverses of every diagonal block of L and U are
    // kept for the cooperative solve; one-level form: one panel's L inverse.
    const int64_t nblk = (mo + kNbFp32 - 1) / kNbFp32;
    PBuf<float> linv_mem, uinv_mem;
    FHB_PALLOC(pool, linv_mem, kSlotLinv, (size_t)count * kNbFp32 * kNbFp32 * 2 * (outer ? nblk : 1));
    w.linv = linv_mem.p;
    SolveScratch ss;
    FlowScratch fs;
    PBuf<unsigned char> solve_mem, flow_mem;
    if (outer) {
        FHB_PALLOC(pool, uinv_mem, kSlotUinv, (size_t)count * kNbFp32 * kNbFp32 * 2 * nblk);
        w.uinv = uinv_mem.p;
        // The two-level form has no interchanges: the dataflow solve (flags
        // per 128-row block), or the barrier-based one when it does not fit.
        int flow_group = 0;
        size_t flow_bytes = 0;
        e = flowsolve_plan(count * (int)p, mo, &flow_group, &flow_bytes, err, s->share);
        if (e) return e;
        if (flow_group > 0) {
            FHB_PALLOC(pool, flow_mem, kSlotFlow, flow_bytes);
            FHB_CUDA(cudaMemsetAsync(flow_mem.p, 0, flow_bytes, st));
            flowsolve_bind(flow_mem.p, count * (int)p, flow_group, mo, fs);
        }
        // the dataflow solve reads U_ij as D_i L_ji^T: no U12 beyond the
        // diagonal regions is written for it
        w.upper = flow_group == 0;
        int per_group = 0;
        size_t solve_bytes = 0;
        if (flow_group == 0) e = trisolve_plan(count * (int)p, mo, &per_group, &solve_bytes, err, s->share);
        if (e) return e;
        if (per_group > 0) {
            FHB_PALLOC(pool, solve_mem, kSlotSolve, solve_bytes);
            FHB_CUDA(cudaMemsetAsync(solve_mem.p, 0, solve_bytes, st));
            trisolve_bind(solve_mem.p, count * (int)p, per_group, ss);
        }
    }
    PBuf<unsigned char> pack_a, pack_b, xpack;
    PBuf<int> tile_counter;
    PBuf<float> xinv, tbuf, dvec;
    if (outer) {
        const size_t pb = packed_operand_bytes(mo - outer, outer, count);
        FHB_PALLOC(pool, pack_a, kSlotPackA, pb);
        w.outer = outer;
        w.pack_a = pack_a.p;
        // the rows-below pass packs one operand for both sides of the update;
        // the separate B operand is for orders it does not take
        if (!(panel_solve_supported(mo) && (int64_t)count * mo <= INT32_MAX)) {
            FHB_PALLOC(pool, pack_b, kSlotPackB, pb);
            w.pack_b = pack_b.p;
        } else if (s->side) {
            // look-ahead of the fused form: the deep update's shared tile counter
            FHB_PALLOC(pool, tile_counter, kSlotTileCounter, 1);
            w.side = s->side;
            w.tile_counter = tile_counter.p;
        }
        // Z_ee = R_ee + jw L_ee with R_ee, L_ee symmetric positive definite:
        // the FP32 factors go without pivoting (stable for this class; the
        // FP64 residual refinement and its FP64 fallback decide the result).
        w.nopivot = true;
        FHB_PALLOC(pool, xinv, kSlotXinv, (size_t)count * outer * outer * 2);
        FHB_PALLOC(pool, xpack, kSlotXpack, packed_operand_bytes(outer, outer, count));
        FHB_PALLOC(pool, tbuf, kSlotTbuf, (size_t)count * kNbFp32 * (outer - kNbFp32) * 2);
        FHB_PALLOC(pool, dvec, kSlotDvec, (size_t)count * outer * 4);
        w.xinv = xinv.p;
        w.xpack = xpack.p;
        w.tbuf = tbuf.p;
        w.dvec = dvec.p;
    }
    LuBatch<float> b;
    b.a = a.p;
    b.pivots = piv.p;
    b.singular = sing.p;
    b.m = mo;
    b.count = count;
    ScopedEvents<3> ev;
    cudaEvent_t e0 = ev.e[0], e1 = ev.e[1], e2 = ev.e[2];
    cudaEventRecord(e0, st);
    e = lu_factor<float>(b, w, kNbFp32, mode, st, err);
    cudaEventRecord(e1, st);
    if (e) return e;
    if (mode == TrailingUpdate::TensorBf16x3) {
        FHB_CUDA(cudaStreamSynchronize(st));
        e = gemm_tc_check(err);
        if (!e) e = gemm_tc_packed_check(err);
        if (e) return e;
    }
    PBuf<unsigned char> res_part;
    if (const size_t rb = residual_scratch_bytes(m, p, count)) FHB_PALLOC(pool, res_part, kSlotResPart, rb);
    PBuf<double> sp_t, sp_y;
    FHB_PALLOC(pool, sp_t, kSlotSparseT, (size_t)std::max<int64_t>(1, 2 * count * p * s->n));
    FHB_PALLOC(pool, sp_y, kSlotSparseY, (size_t)std::max<int64_t>(1, 2 * count * p * m));
    SparseR sparse_r;
    sparse_r.row_ptr = s->d_rp;
    sparse_r.branch = s->d_br;
    sparse_r.sign = s->d_sign;
    sparse_r.t_off = s->d_toff;
    sparse_r.t_loop = s->d_tloop;
    sparse_r.t_sign = s->d_tsign;
    sparse_r.R = s->d_R;
    sparse_r.n = s->n;
    sparse_r.t = sp_t.p;
    sparse_r.y = sp_y.p;
    std::vector<double> hb(count), hd(count), hx(count), hr(count), prev(count, INFINITY);
    std::vector<int> done(count, 0), grow(count, 0);
    FHB_CUDA(cudaMemcpyAsync(hb.data(), bnorm.p, 8 * count, cudaMemcpyDeviceToHost, st));
    const int kMaxIter = 40;
    // The error a converged frequency may keep, relative to x.
    constexpr double kRefineLeft = 1e-12;
    int it = 0;
    for (; it < kMaxIter; ++it) {
        e = convert_c64_to_c32(r.p, d32.p, count * vec, st, err, m, mo);
        if (!e) {
            if (fs.per_group > 0)
                e = lu_solve_flow(b, w.linv, w.uinv, d32.p, (int)p, fs, st, err);
            else if (ss.per_group > 0)
                e = lu_solve_inv(b, w.linv, w.uinv, d32.p, (int)p, kNbFp32, outer, ss, st, err);
            else
                e = lu_solve<float>(b, d32.p, (int)p, kNbFp32, st, err, outer);
        }
        if (!e) e = add_c32_to_c64(d_x, d32.p, count * vec, st, err, m, mo);
        if (!e)
            e = residual_fp64(s->d_Rm, s->d_Lm, ld, m, p, d_omega, count, d_x, r.p, rnorm.p, st, err, res_part.p,
                              &sparse_r);
        if (e) return e;
        // correction and solution norms (max-abs) for the stopping rule
        e = max_abs_per_matrix_f32(d32.p, 2 * vec32, count, dnorm.p, st, err);
        if (!e) e = max_abs_per_matrix(d_x, 2 * vec, count, xnorm.p, st, err);
        if (e) return e;
        FHB_CUDA(cudaMemcpyAsync(hd.data(), dnorm.p, 8 * count, cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaMemcpyAsync(hx.data(), xnorm.p, 8 * count, cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaMemcpyAsync(hr.data(), rnorm.p, 8 * count, cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaStreamSynchronize(st));
        bool all = true;
        for (int f = 0; f < count; ++f) {
            if (done[f]) continue;
            // Stopping rule: the correction is negligible (1e-12 of x); or the
            // iteration contracts geometrically (rho = |d_k| / |d_k-1| < 0.1)
            // and the error left after this correction, estimated as
            // |d_k| rho / (1 - rho), is below kRefineLeft of x; or the
            // correction has stopped shrinking at a level below 1e-10 of x,
            // which is the attainable accuracy of an FP64 residual (about
            // kappa * u64).
            double rel = hx[f] > 0 ? hd[f] / hx[f] : 0.0;
            const bool stalled = hd[f] > 0.5 * prev[f];
            const double rho = std::isfinite(prev[f]) && prev[f] > 0 ? hd[f] / prev[f] : 1.0;
            const bool contracted = rho < 0.1 && rel * rho / (1.0 - rho) <= kRefineLeft;
            // A small correction is only trusted with a small FP64 residual:
            // |b - A x| <= 1e-6 |b| holds for any accurate x up to kappa ~ 1e10.
            const bool resid_ok = hr[f] <= 1e-6 * hb[f];
            if (resid_ok && (rel <= 1e-12 || hd[f] == 0.0 || contracted || (stalled && rel <= 1e-10))) {
                done[f] = 1;
                if (iters_out) iters_out[f] = it + 1;
                continue;
            }
            if (stalled) ++grow[f];
            if (grow[f] >= 3 || !std::isfinite(hd[f])) {
                done[f] = 1;
                h_failed[f] = 1;
                if (iters_out) iters_out[f] = it + 1;
                continue;
            }
            prev[f] = hd[f];
            all = false;
        }
        if (all) break;
    }
    for (int f = 0; f < count; ++f) {
        if (!done[f]) {
            h_failed[f] = 1;
            if (iters_out) iters_out[f] = it;
        }
        if (resid_out) resid_out[f] = hb[f] > 0 ? hr[f] / hb[f] : 0.0;
    }
    if (ss.per_group > 0) {
        e = trisolve_check(ss, st, err);
        if (e) return e;
    }
    if (fs.per_group > 0) {
        e = flowsolve_check(fs, st, err);
        if (e) return e;
    }
    cudaEventRecord(e2, st);
    FHB_CUDA(cudaMemcpyAsync(h_singular, sing.p, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
    e = schur(s->d_Rm, s->d_Lm, ld, m, p, d_omega, count, d_x, d_z, st, err);
    if (e) return e;
    FHB_CUDA(cudaStreamSynchronize(st));
    float ms1 = 0, ms2 = 0;
    cudaEventElapsedTime(&ms1, e0, e1);
    cudaEventElapsedTime(&ms2, e1, e2);
    if (ms_factor) *ms_factor += ms1;
    if (ms_refine) *ms_refine += ms2;
    return FH_OK;
}

// fh_batch_sweep in a mixed precision: every (system, frequency) of the
// systems with m <= FH_BATCH_MAX_ORDER in one persistent launch
// (fh_batchsolve.cu), largest first; items whose refinement did not converge
// are redone by the FP64 sweep.  Frequencies are checked per system first:
// a system with an invalid frequency is left to the per-system path, which
// reports it.  done[i] is set for the systems finished here.
fh_status batch_sweep_persistent(fh_system *const *systems, size_t k, const double *const *freqs, const size_t *nf,
                                 double *const *z_out, std::vector<char> &done, fh_error_info *err) {
    std::vector<size_t> take;
    int dev0 = systems[0]->device;
    for (size_t i = 0; i < k; ++i) {
        const fh_system *s = systems[i];
        bool ok = s->m <= FH_BATCH_MAX_ORDER && s->device == dev0 && (nf[i] == 0 || freqs[i]);
        for (size_t f = 0; ok && f < nf[i]; ++f) ok = std::isfinite(freqs[i][f]) && freqs[i][f] >= 0.0;
        if (ok) take.push_back(i);
    }
    if (take.empty()) return FH_OK;
    FHB_CUDA(cudaSetDevice(dev0));
    cudaStream_t st = systems[take[0]]->stream;
    for (size_t i : take) FHB_CUDA(cudaStreamSynchronize(systems[i]->stream));
    const double t0 = wall();
    std::vector<BatchSys> sys(take.size());
    int64_t mmax = 1;
    int pmax = 1;
    for (size_t t = 0; t < take.size(); ++t) {
        const fh_system *s = systems[take[t]];
        sys[t].R = s->d_Rm;
        sys[t].L = s->d_Lm;
        sys[t].ld = s->nloops;
        sys[t].m = s->m;
        sys[t].p = s->p;
        mmax = std::max<int64_t>(mmax, s->m);
        pmax = std::max<int>(pmax, (int)s->p);
    }
    PBuf<unsigned char> d_sys, d_one;
    DevPool &pool = systems[take[0]]->pool;
    FHB_PALLOC(pool, d_sys, kSlotBatchSys, sizeof(BatchSys) * sys.size());
    FHB_PALLOC(pool, d_one, kSlotBatchOne, sizeof(BatchSys));
    FHB_CUDA(cudaMemcpyAsync(d_sys.p, sys.data(), sizeof(BatchSys) * sys.size(), cudaMemcpyHostToDevice, st));
    // tile configurations per order bucket (measured on first use)
    std::vector<int> cfg(sys.size(), 0);
    for (size_t t = 0; t < sys.size(); ++t) {
        FHB_CUDA(cudaMemcpyAsync(d_one.p, &sys[t], sizeof(BatchSys), cudaMemcpyHostToDevice, st));
        fh_status e = batch_tuner().config_for(sys[t], reinterpret_cast<const BatchSys *>(d_one.p), st, &cfg[t], err);
        if (e) return e;
    }
    // items, largest first
    std::vector<BatchItem> items;
    std::vector<int64_t> zoff(sys.size() + 1, 0);
    for (size_t t = 0; t < sys.size(); ++t) zoff[t + 1] = zoff[t] + (int64_t)nf[take[t]] * sys[t].p * sys[t].p;
    for (size_t t = 0; t < sys.size(); ++t)
        for (size_t f = 0; f < nf[take[t]]; ++f) {
            BatchItem it;
            it.sys = (int32_t)t;
            it.cfg = cfg[t];
            it.omega = kTau * freqs[take[t]][f];
            it.z_offset = zoff[t] + (int64_t)f * sys[t].p * sys[t].p;
            it.index = (int32_t)items.size();
            items.push_back(it);
        }
    std::stable_sort(items.begin(), items.end(), [&](const BatchItem &a, const BatchItem &b) {
        return sys[a.sys].m > sys[b.sys].m;
    });
    const int nitems = (int)items.size();
    std::vector<double> z((size_t)(2 * std::max<int64_t>(1, zoff.back())));
    std::vector<int32_t> status((size_t)std::max(1, nitems), 0);
    if (nitems > 0) {
        const int ctas = std::min(batch_resident_ctas(), nitems);
        const size_t slot = batch_slot_bytes(mmax, pmax);
        PBuf<unsigned char> d_items, d_z, d_status, d_counter, d_work;
        FHB_PALLOC(pool, d_items, kSlotBatchItems, sizeof(BatchItem) * items.size());
        FHB_PALLOC(pool, d_z, kSlotBatchZ, 8 * z.size());
        FHB_PALLOC(pool, d_status, kSlotBatchStatus, sizeof(int32_t) * status.size());
        FHB_PALLOC(pool, d_counter, kSlotBatchCounter, 16);
        FHB_PALLOC(pool, d_work, kSlotBatchWork, slot * (size_t)ctas);
        FHB_CUDA(cudaMemcpyAsync(d_items.p, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice, st));
        double work = 0.0;
        for (const BatchItem &it : items) work += 8.0 / 3.0 * std::pow((double)sys[it.sys].m, 3.0);
        prof_begin(st, FH_PROF_BATCH);
        fh_status e = batch_launch(reinterpret_cast<const BatchSys *>(d_sys.p),
                                   reinterpret_cast<const BatchItem *>(d_items.p), nitems,
                                   reinterpret_cast<unsigned *>(d_counter.p), d_work.p, slot, mmax, pmax,
                                   reinterpret_cast<double2 *>(d_z.p), reinterpret_cast<int32_t *>(d_status.p), ctas,
                                   st, err);
        prof_end(st, FH_PROF_BATCH, work);
        if (e) return e;
        FHB_CUDA(cudaMemcpyAsync(z.data(), d_z.p, 8 * z.size(), cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaMemcpyAsync(status.data(), d_status.p, sizeof(int32_t) * status.size(), cudaMemcpyDeviceToHost,
                                 st));
        FHB_CUDA(cudaStreamSynchronize(st));
    }
    // outputs; FP64 for the items that did not converge
    std::vector<size_t> item_of(items.size());
    for (size_t q = 0; q < items.size(); ++q) item_of[(size_t)items[q].index] = q;
    size_t idx = 0;
    for (size_t t = 0; t < sys.size(); ++t) {
        const size_t i = take[t];
        const int64_t pp = sys[t].p * sys[t].p;
        for (size_t f = 0; f < nf[i]; ++f, ++idx) {
            double *dst = z_out[i] + 2 * (int64_t)f * pp;
            if (status[idx] < 0) {
                fh_error_info e{};
                const fh_status s2 = fh_sweep(systems[i], freqs[i] + f, 1, FH_PRECISION_FP64, dst, nullptr, &e);
                if (s2) {
                    const char *msg = fh_last_error();
                    fh_status r = fail(err, s2, "system " + std::to_string(i) + ": " + (msg ? msg : ""), e.index_a,
                                       e.index_b, e.frequency, (int32_t)i);
                    return r;
                }
                continue;
            }
            const double *src = z.data() + 2 * (zoff[t] + (int64_t)f * pp);
            bool bad = false;
            for (int64_t q = 0; q < 2 * pp; ++q) bad = bad || !std::isfinite(src[q]);
            if (bad)
                return fail(err, FH_ERR_SINGULAR,
                            "system " + std::to_string(i) + ": the mesh system is singular or ill-conditioned at " +
                                fstr(freqs[i][f]) + " Hz",
                            (int64_t)f, -1, freqs[i][f], (int32_t)i);
            std::memcpy(dst, src, 16 * (size_t)pp);
        }
        fh_system *s = systems[i];
        s->timing.solve_s = wall() - t0;
        s->timing.total_s = s->timing.assembly_s + s->timing.solve_s;
        done[i] = 1;
    }
    return FH_OK;
}

}  // namespace
}  // namespace fhb

extern "C" {

const char *fh_build_info(void) {
    return "fasterhenry_b200 0.1.0 (sm_100a; FP64 fill; batched complex LU FP64 / FP32+bf16x3 tensor trailing "
           "updates with FP64 iterative refinement)";
}

int32_t fh_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int usable = 0;
    for (int d = 0; d < count; ++d) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10) ++usable;
    }
    return usable;
}

fh_status fh_partial_inductance_matrix(const fh_filament *filaments, size_t n, double *L, int8_t *methods,
                                       fh_error_info *err) {
    clear_error(err);
    if ((n && (!filaments || !L))) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    fh_status st = ensure_device(err);
    if (st) return st;
    if (n == 0) return FH_OK;
    std::vector<DevFil> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = make_devfil(filaments[i]);
    DBuf<DevFil> d_fil;
    DBuf<double> d_L;
    DBuf<int8_t> d_m;
    FHB_ALLOC(d_fil, n);
    FHB_ALLOC(d_L, n * n);
    if (methods) FHB_ALLOC(d_m, n * n);
    cudaStream_t s;
    FHB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, decltype(&cudaStreamDestroy)> guard(s, &cudaStreamDestroy);
    FHB_CUDA(cudaMemcpyAsync(d_fil.p, h.data(), n * sizeof(DevFil), cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemsetAsync(d_L.p, 0, n * n * sizeof(double), s));
    if (methods) FHB_CUDA(cudaMemsetAsync(d_m.p, 0, n * n, s));
    st = device_fill(d_fil.p, (int64_t)n, d_L.p, methods ? d_m.p : nullptr, s, nullptr, err);
    if (st) return st;
    FHB_CUDA(cudaMemcpyAsync(L, d_L.p, n * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (methods) FHB_CUDA(cudaMemcpyAsync(methods, d_m.p, n * n, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    return FH_OK;
}

fh_status fh_test_trailing_update(float *a, int64_t m, int32_t count, int64_t k0, int32_t nb, int32_t mode,
                                  fh_error_info *err) {
    clear_error(err);
    if (!a || m <= 0 || count <= 0 || k0 < 0 || nb <= 0 || k0 + nb > m)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "bad trailing-update arguments");
    fh_status st = ensure_device(err);
    if (st) return st;
    const size_t bytes = (size_t)count * m * m * 8;
    DBuf<float> d;
    FHB_ALLOC(d, bytes / 4);
    FHB_CUDA(cudaMemcpy(d.p, a, bytes, cudaMemcpyHostToDevice));
    DBuf<unsigned char> pa, pb;
    if (mode == 2) {
        if (nb % 16) return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update needs nb a multiple of 16");
        const int64_t base = k0 + nb, rem = m - base;
        if (rem > 0) {
            FHB_ALLOC(pa, packed_operand_bytes(rem, nb, count));
            FHB_ALLOC(pb, packed_operand_bytes(rem, nb, count));
            float *A = d.p;
            auto at = [&](int64_t r, int64_t c) { return A + 2 * (r + c * m); };
            st = gemm_tc_packed_update(at(base, k0), m, m * m, at(k0, base), m, m * m, at(base, base), m, m * m, rem,
                                       rem, nb, count, pa.p, pb.p, nullptr, err);
        }
    } else {
        st = mode == 1 ? gemm_tc_update(d.p, m, count, k0, nb, nullptr, err)
                       : gemm_simt_update<float>(d.p, m, count, k0, nb, nullptr, err);
    }
    if (st) return st;
    FHB_CUDA(cudaDeviceSynchronize());
    st = gemm_tc_check(err);
    if (!st) st = gemm_tc_packed_check(err);
    if (st) return st;
    FHB_CUDA(cudaMemcpy(a, d.p, bytes, cudaMemcpyDeviceToHost));
    return FH_OK;
}

fh_status fh_lu_solve_c64(const double *a, size_t n, const double *b, size_t nrhs, double *x, fh_error_info *err) {
    clear_error(err);
    if (n && (!a || !b || !x)) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    fh_status st = ensure_device(err);
    if (st) return st;
    if (n == 0) return FH_OK;
    if (n > (size_t)INT32_MAX / 2) return fail(err, FH_ERR_INVALID_ARGUMENT, "order too large");
    DBuf<double> d_a, d_x, pv;
    DBuf<int> piv, sing, pi;
    DBuf<unsigned> tk;
    FHB_ALLOC(d_a, 2 * n * n);
    FHB_ALLOC(d_x, 2 * n * nrhs);
    FHB_ALLOC(piv, n);
    FHB_ALLOC(sing, 1);
    FHB_ALLOC(pv, 16);
    FHB_ALLOC(pi, 16);
    FHB_ALLOC(tk, 1);
    cudaStream_t s;
    FHB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, decltype(&cudaStreamDestroy)> guard(s, &cudaStreamDestroy);
    FHB_CUDA(cudaMemcpyAsync(d_a.p, a, 16 * n * n, cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemcpyAsync(d_x.p, b, 16 * n * nrhs, cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemsetAsync(sing.p, 0, sizeof(int), s));
    FHB_CUDA(cudaMemsetAsync(tk.p, 0, sizeof(unsigned), s));
    LuWork w;
    w.partial_val = pv.p;
    w.partial_idx = pi.p;
    w.tickets = tk.p;
    w.max_chunks = 16;
    LuBatch<double> lb;
    lb.a = d_a.p;
    lb.pivots = piv.p;
    lb.singular = sing.p;
    lb.m = (int64_t)n;
    lb.count = 1;
    st = lu_factor<double>(lb, w, 64, TrailingUpdate::Simt, s, err);
    if (!st) st = lu_solve<double>(lb, d_x.p, (int)nrhs, 64, s, err);
    if (st) return st;
    int singular = 0;
    FHB_CUDA(cudaMemcpyAsync(&singular, sing.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaMemcpyAsync(x, d_x.p, 16 * n * nrhs, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    if (singular) return fail(err, FH_ERR_SINGULAR, "the matrix is singular (zero pivot)");
    return FH_OK;
}

fh_status fh_system_create(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segments, size_t n_segments,
                           const fh_port *ports, size_t n_ports, const fh_discretization *disc,
                           fh_solver_choice choice, fh_system **out, fh_error_info *err) {
    return fh_system_create_coupled(nodes, n_nodes, segments, n_segments, ports, n_ports, disc, nullptr, choice, out,
                                    err);
}

fh_status fh_system_coupling(const fh_system *sys, int64_t *kept_pairs, int64_t *total_pairs,
                             fh_truncation_warning *warnings, size_t capacity, size_t *count) {
    if (!sys) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null system");
    if (kept_pairs) *kept_pairs = sys->kept_pairs;
    if (total_pairs) *total_pairs = sys->total_pairs;
    if (count) *count = sys->warnings.size();
    if (warnings)
        for (size_t k = 0; k < std::min(capacity, sys->warnings.size()); ++k) warnings[k] = sys->warnings[k];
    return FH_OK;
}

fh_status fh_system_create_coupled(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segments,
                                   size_t n_segments, const fh_port *ports, size_t n_ports,
                                   const fh_discretization *disc, const fh_coupling *coupling,
                                   fh_solver_choice choice, fh_system **out, fh_error_info *err) {
    clear_error(err);
    if (!out) return fail(err, FH_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    const double t0 = wall();
    std::unique_ptr<fh_system> s(new fh_system);
    s->nodes.assign(nodes, nodes + n_nodes);
    s->segments.assign(segments, segments + n_segments);
    if (n_ports && !ports) return fail(err, FH_ERR_INVALID_ARGUMENT, "null ports");
    s->ports.assign(ports, ports + n_ports);
    // The coupling is checked before anything is paid for (solve.rs:710-712).
    fh_status st = validate_geometry(nodes, n_nodes, segments, n_segments, err);
    if (st) return st;
    st = resolve_coupling(coupling, n_segments, s->coupling, err);
    if (st) return st;
    s->warnings = coupling_warnings(s->coupling, nodes, segments, n_segments);
    st = discretize_geometry(nodes, n_nodes, segments, n_segments, disc, s->disc, err);
    if (st) return st;
    st = build_loops(segments, n_segments, n_nodes, s->disc.per_segment.data(), ports, n_ports, s->loops, err);
    if (st) return st;
    s->n = (int64_t)s->disc.filaments.size();
    if (fh_solver_resolve(choice, (size_t)s->n) != 0)
        return fail(err, FH_ERR_UNSUPPORTED,
                    "this choice resolves to the matrix-free path, which is fh_iterative_create (IterativeSystem); "
                    "fh_system_create builds the dense MeshSystem");
    st = ensure_device(err);
    if (st) return st;
    FHB_CUDA(cudaGetDevice(&s->device));
    FHB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    // Default priority: the look-ahead gets its SMs by the update leaving
    // them free, not by scheduling ahead of queued update CTAs.
    FHB_CUDA(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    cudaStream_t cs = s->stream;
    s->pool.stream = cs;
    s->nloops = s->loops.rows();
    s->m = s->loops.internal;
    s->p = s->nloops - s->m;
    for (const fh_filament &f : s->disc.filaments)
        s->resistances.push_back(f.length / (f.sigma * (f.width * f.height)));  // solve.rs:941-943
    const int64_t n = s->n, loops = s->nloops;
    std::vector<DevFil> h(n);
    for (int64_t i = 0; i < n; ++i) h[i] = make_devfil(s->disc.filaments[i]);
    DBuf<DevFil> d_fil(cs);
    DBuf<double> d_L(cs);
    FHB_ALLOC(d_fil, (size_t)n);
    FHB_ALLOC(d_L, (size_t)n * n);
    TransposedLoops internal;
    transpose_loops(s->loops, n, s->m, internal);
    {
        auto keep = [&](void **d, size_t bytes) { return cache_alloc(d, std::max<size_t>(bytes, 16), cs); };
        if (keep((void **)&s->d_R, 8 * (size_t)n) || keep((void **)&s->d_rp, 8 * s->loops.row_ptr.size()) ||
            keep((void **)&s->d_br, 4 * s->loops.branch.size()) || keep((void **)&s->d_sign, 8 * s->loops.sign.size()) ||
            keep((void **)&s->d_toff, 8 * internal.offset.size()) || keep((void **)&s->d_tloop, 4 * internal.loop.size()) ||
            keep((void **)&s->d_tsign, 8 * internal.sign.size())) {
            cudaGetLastError();
            return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation of the loop basis failed");
        }
    }
    if (cache_alloc((void **)&s->d_Lm, std::max<size_t>(1, (size_t)loops * loops) * 8, cs) != cudaSuccess ||
        cache_alloc((void **)&s->d_Rm, std::max<size_t>(1, (size_t)loops * loops) * 8, cs) != cudaSuccess) {
        cudaGetLastError();
        return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation of the mesh matrices failed");
    }
    FHB_CUDA(cudaMemcpyAsync(d_fil.p, h.data(), n * sizeof(DevFil), cudaMemcpyHostToDevice, cs));
    FHB_CUDA(cudaMemcpyAsync(s->d_R, s->resistances.data(), n * 8, cudaMemcpyHostToDevice, cs));
    FHB_CUDA(cudaMemcpyAsync(s->d_rp, s->loops.row_ptr.data(), s->loops.row_ptr.size() * 8, cudaMemcpyHostToDevice, cs));
    FHB_CUDA(cudaMemcpyAsync(s->d_br, s->loops.branch.data(), s->loops.branch.size() * 4, cudaMemcpyHostToDevice, cs));
    FHB_CUDA(cudaMemcpyAsync(s->d_sign, s->loops.sign.data(), s->loops.sign.size() * 8, cudaMemcpyHostToDevice, cs));
    FHB_CUDA(cudaMemcpyAsync(s->d_toff, internal.offset.data(), internal.offset.size() * 8, cudaMemcpyHostToDevice, cs));
    if (!internal.loop.empty()) {
        FHB_CUDA(cudaMemcpyAsync(s->d_tloop, internal.loop.data(), internal.loop.size() * 4, cudaMemcpyHostToDevice, cs));
        FHB_CUDA(cudaMemcpyAsync(s->d_tsign, internal.sign.data(), internal.sign.size() * 8, cudaMemcpyHostToDevice, cs));
    }
    FHB_CUDA(cudaMemsetAsync(d_L.p, 0, (size_t)n * n * 8, cs));
    s->total_pairs = n * (n + 1) / 2;
    s->kept_pairs = coupling_kept_pairs(s->coupling, s->disc.per_segment.data(), n_segments);
    if (!s->coupling.all_pairs) {
        std::vector<int32_t> group;
        group.reserve((size_t)n);
        for (size_t g = 0; g < n_segments; ++g)
            for (int64_t k = 0; k < s->disc.per_segment[g]; ++k) group.push_back(s->coupling.of_segment[g]);
        const size_t tb = s->coupling.couples.size();
        if (cache_alloc((void **)&s->d_group, 4 * group.size(), cs) != cudaSuccess ||
            cache_alloc((void **)&s->d_coupled, std::max<size_t>(tb, 1), cs) != cudaSuccess) {
            cudaGetLastError();
            return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation of the coupling mask failed");
        }
        FHB_CUDA(cudaMemcpyAsync(s->d_group, group.data(), 4 * group.size(), cudaMemcpyHostToDevice, cs));
        FHB_CUDA(cudaMemcpyAsync(s->d_coupled, s->coupling.couples.data(), tb, cudaMemcpyHostToDevice, cs));
    }
    const PairMaskDev pm = s->mask();
    const double t1 = wall();
    st = device_fill(d_fil.p, n, d_L.p, nullptr, cs, &s->fill, err, &pm);
    if (st) return st;
    FHB_CUDA(cudaStreamSynchronize(cs));
    const double t2 = wall();
    ScopedEvents<2> cev;
    cudaEvent_t c0 = cev.e[0], c1 = cev.e[1];
    cudaEventRecord(c0, cs);
    st = device_congruence(d_L.p, s->d_R, n, s->d_rp, s->d_br, s->d_sign, loops, s->loops.row_ptr.data(), s->d_Lm,
                           s->d_Rm, cs, err);
    cudaEventRecord(c1, cs);
    if (st) return st;
    FHB_CUDA(cudaStreamSynchronize(cs));
    cudaEventElapsedTime(&s->ms_congruence, c0, c1);
    const double t3 = wall();
    {
        ConductorLayout layout;
        conductor_layout(segments, n_segments, n_nodes, s->disc.per_segment.data(), layout);
        s->segment_of_filament = std::move(layout.segment_of_filament);
        s->conductor_of_segment = std::move(layout.conductor_of_segment);
        s->segment_first = std::move(layout.segment_first);
        s->conductors = layout.conductors;
    }
    s->counts = fh_counts{(int64_t)n_nodes, (int64_t)n_segments, n, loops, s->m, s->p};
    s->timing.inductance_s = t2 - t1;
    s->timing.assembly_s = t3 - t0;
    s->timing.solve_s = 0.0;
    s->timing.total_s = s->timing.assembly_s;
    *out = s.release();
    return FH_OK;
}

void fh_system_destroy(fh_system *sys) { delete sys; }

fh_status fh_system_counts(const fh_system *sys, fh_counts *counts) {
    if (!sys || !counts) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    *counts = sys->counts;
    return FH_OK;
}

fh_status fh_system_fill_stats(const fh_system *sys, fh_fill_stats *o) {
    if (!sys || !o) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    const FillStats &f = sys->fill;
    o->pairs = f.pairs;
    o->orthogonal = f.orthogonal;
    o->point_quadrature = f.point;
    o->closed_form = f.closed_form;
    o->aligned_quadrature = f.aligned_quadrature;
    o->sampled = f.sampled;
    o->distinct_aligned_keys = f.unique_aligned;
    o->point_evaluations = f.point_evaluations;
    o->ms_classify = f.ms_classify;
    o->ms_point = f.ms_point;
    o->ms_closed_form = f.ms_aligned;
    o->ms_aligned_quadrature = f.ms_quadrature;
    o->ms_sampled = f.ms_sampled;
    o->ms_congruence = sys->ms_congruence;
    o->truncated = f.truncated;
    o->distinct_point_keys = f.unique_point;
    return FH_OK;
}

fh_status fh_system_timing(const fh_system *sys, fh_timing *timing) {
    if (!sys || !timing) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    *timing = sys->timing;
    return FH_OK;
}

fh_status fh_system_filaments(const fh_system *sys, fh_filament *out, size_t capacity) {
    if (!sys || !out) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    if (capacity < sys->disc.filaments.size()) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "buffer too small");
    std::copy(sys->disc.filaments.begin(), sys->disc.filaments.end(), out);
    return FH_OK;
}

fh_status fh_system_resistances(const fh_system *sys, double *out, size_t capacity) {
    if (!sys || !out) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    if (capacity < sys->resistances.size()) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "buffer too small");
    std::copy(sys->resistances.begin(), sys->resistances.end(), out);
    return FH_OK;
}

fh_status fh_system_mesh_matrices(const fh_system *sys, double *r_mesh, double *l_mesh) {
    if (!sys) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    fh_error_info *err = nullptr;
    size_t bytes = (size_t)sys->nloops * sys->nloops * 8;
    if (r_mesh) FHB_CUDA(cudaMemcpy(r_mesh, sys->d_Rm, bytes, cudaMemcpyDeviceToHost));
    if (l_mesh) FHB_CUDA(cudaMemcpy(l_mesh, sys->d_Lm, bytes, cudaMemcpyDeviceToHost));
    return FH_OK;
}

fh_status fh_system_device_l_mesh(const fh_system *sys, const double **l_mesh, const double **r_mesh) {
    if (!sys) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    if (l_mesh) *l_mesh = sys->d_Lm;
    if (r_mesh) *r_mesh = sys->d_Rm;
    return FH_OK;
}

fh_status fh_sweep(fh_system *sys, const double *freqs, size_t nf, fh_precision precision, double *z_out,
                   fh_sweep_report *report, fh_error_info *err) {
    clear_error(err);
    if (!sys || (nf && (!freqs || !z_out))) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    for (size_t k = 0; k < nf; ++k)
        if (!(std::isfinite(freqs[k]) && freqs[k] >= 0.0))
            return fail(err, FH_ERR_INVALID_FREQUENCY,
                        "frequency " + std::to_string(k) + " is " + fstr(freqs[k]) +
                            " Hz; frequencies must be finite and non-negative",
                        (int64_t)k, -1, freqs[k]);
    if (nf == 0) return FH_OK;
    FHB_CUDA(cudaSetDevice(sys->device));
    const double t0 = wall();
    const int64_t m = sys->m, p = sys->p;
    cudaStream_t st = sys->stream;
    // Frequencies per batch from free device memory (the analogue of the
    // reference's 2 GiB sweep budget, solve.rs:91 and 884).
    size_t free_b = 0, total_b = 0;
    FHB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    // Own workspace is reused; memory the cache holds idle is available too.
    free_b = (free_b + cache_idle_bytes()) / (size_t)std::max(1, sys->share) + sys->pool.held();
    if (precision < FH_PRECISION_FP64 || precision > FH_PRECISION_MIXED_FP32)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "unknown precision");
    const bool mixed = precision != FH_PRECISION_FP64;
    const TrailingUpdate update =
        precision == FH_PRECISION_MIXED_BF16X3 ? TrailingUpdate::TensorBf16x3 : TrailingUpdate::Simt;
    // Per frequency: the matrix, the vectors, and for the two-level FP32
    // form its two packed operands (8 bytes per entry of an m x 512 block
    // each), the inverses of the diagonal blocks of L and U, and a
    // super-panel's U^-1 in FP32 and packed.
    const double per = (mixed ? 8.0 : 16.0) * (double)m * (double)m + 64.0 * (double)(m * p + 64) +
                       (outer_for(m, update) ? 16.0 * (double)m * kOuterFp32 + 16.0 * (double)(m + kNbFp32) * kNbFp32 +
                                                   16.0 * kOuterFp32 * kOuterFp32 + 8.0 * kNbFp32 * kOuterFp32
                                             : 0.0);
    int chunk = (int)std::max(1.0, std::min<double>((double)nf, 0.8 * (double)free_b / std::max(per, 1.0)));
    PBuf<double> d_omega, d_x, d_z;
    FHB_PALLOC(sys->pool, d_omega, kSlotOmega, (size_t)chunk);
    FHB_PALLOC(sys->pool, d_x, kSlotX, (size_t)chunk * m * p * 2);
    FHB_PALLOC(sys->pool, d_z, kSlotZ, (size_t)chunk * p * p * 2);
    float ms_factor = 0, ms_refine = 0;
    ScopedEvents<2> ev;
    cudaEvent_t e0 = ev.e[0], e1 = ev.e[1];
    cudaEventRecord(e0, st);
    std::vector<int> singular((size_t)nf, 0), failed((size_t)nf, 0);
    for (size_t c0 = 0; c0 < nf; c0 += (size_t)chunk) {
        const int count = (int)std::min<size_t>((size_t)chunk, nf - c0);
        std::vector<double> omega(count);
        for (int f = 0; f < count; ++f) omega[f] = kTau * freqs[c0 + f];
        FHB_CUDA(cudaMemcpyAsync(d_omega.p, omega.data(), 8 * count, cudaMemcpyHostToDevice, st));
        fh_status e;
        if (mixed) {
            e = sweep_chunk_mixed(sys, d_omega.p, count, d_x.p, d_z.p, singular.data() + c0, failed.data() + c0,
                                  report && report->refinement_iterations ? report->refinement_iterations + c0 : nullptr,
                                  report && report->residual ? report->residual + c0 : nullptr, &ms_factor, &ms_refine,
                                  update, err);
        } else {
            e = sweep_chunk_fp64(sys, d_omega.p, count, d_x.p, d_z.p, singular.data() + c0, &ms_factor, err);
        }
        if (e) return e;
        FHB_CUDA(cudaMemcpyAsync(z_out + 2 * c0 * p * p, d_z.p, 16 * (size_t)count * p * p, cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaStreamSynchronize(st));
        // Refinement that did not converge: redo those frequencies in FP64.
        std::vector<int> redo;
        for (int f = 0; f < count; ++f)
            if (failed[c0 + f]) redo.push_back(f);
        if (!redo.empty()) {
            std::vector<double> om2;
            for (int f : redo) om2.push_back(omega[f]);
            DBuf<double> d_om2, d_x2, d_z2;
            FHB_ALLOC(d_om2, om2.size());
            FHB_ALLOC(d_x2, om2.size() * m * p * 2);
            FHB_ALLOC(d_z2, om2.size() * p * p * 2);
            FHB_CUDA(cudaMemcpyAsync(d_om2.p, om2.data(), 8 * om2.size(), cudaMemcpyHostToDevice, st));
            std::vector<int> sing2(om2.size(), 0);
            e = sweep_chunk_fp64(sys, d_om2.p, (int)om2.size(), d_x2.p, d_z2.p, sing2.data(), &ms_factor, err);
            if (e) return e;
            std::vector<double> z2(om2.size() * p * p * 2);
            FHB_CUDA(cudaMemcpyAsync(z2.data(), d_z2.p, 8 * z2.size(), cudaMemcpyDeviceToHost, st));
            FHB_CUDA(cudaStreamSynchronize(st));
            for (size_t k = 0; k < redo.size(); ++k) {
                int f = redo[k];
                singular[c0 + f] = sing2[k];
                std::memcpy(z_out + 2 * (c0 + f) * p * p, z2.data() + 2 * k * p * p, 16 * (size_t)p * p);
                if (report && report->refinement_iterations) report->refinement_iterations[c0 + f] = -1;
            }
        }
    }
    cudaEventRecord(e1, st);
    FHB_CUDA(cudaStreamSynchronize(st));
    float ms_total = 0;
    cudaEventElapsedTime(&ms_total, e0, e1);
    // First failing frequency in list order (solve.rs:877-879).
    for (size_t k = 0; k < nf; ++k) {
        bool bad = singular[k] != 0;
        for (int64_t q = 0; q < p * p && !bad; ++q)
            bad = !(std::isfinite(z_out[2 * (k * p * p + q)]) && std::isfinite(z_out[2 * (k * p * p + q) + 1]));
        if (bad)
            return fail(err, FH_ERR_SINGULAR,
                        "the mesh system is singular or ill-conditioned at " + fstr(freqs[k]) + " Hz", (int64_t)k, -1,
                        freqs[k]);
    }
    const double t1 = wall();
    sys->timing.solve_s = t1 - t0;
    sys->timing.total_s = sys->timing.assembly_s + sys->timing.solve_s;
    if (report) {
        report->solve_s = ms_total * 1e-3;
        report->factor_s = ms_factor * 1e-3;
        report->refine_s = ms_refine * 1e-3;
    }
    return FH_OK;
}

fh_status fh_batch_sweep(fh_system *const *systems, size_t k, const double *const *freqs, const size_t *nf,
                         fh_precision precision, double *const *z_out, int32_t concurrency, fh_error_info *err) {
    clear_error(err);
    if (k && (!systems || !freqs || !nf || !z_out)) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    for (size_t i = 0; i < k; ++i)
        if (!systems[i]) return fail(err, FH_ERR_INVALID_ARGUMENT, "null system " + std::to_string(i));
    if (k == 0) return FH_OK;
    if (precision < FH_PRECISION_FP64 || precision > FH_PRECISION_MIXED_FP32)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "unknown precision");
    // Mixed precisions: the small systems in one persistent launch; the
    // others (and every system in FP64) through the per-system sweeps below.
    std::vector<char> done(k, 0);
    if (precision != FH_PRECISION_FP64) {
        fh_status st = batch_sweep_persistent(systems, k, freqs, nf, z_out, done, err);
        if (st) return st;
    }
    std::vector<size_t> rest;
    for (size_t i = 0; i < k; ++i)
        if (!done[i]) rest.push_back(i);
    if (rest.empty()) return FH_OK;
    const int workers = (int)std::min<size_t>(rest.size(), (size_t)(concurrency > 0 ? concurrency : 4));
    for (size_t i = 0; i < k; ++i) systems[i]->share = workers;
    std::atomic<size_t> next(0);
    std::mutex mu;
    size_t failed = k;
    fh_status failed_status = FH_OK;
    fh_error_info failed_info{};
    std::string failed_msg;
    auto worker = [&]() {
        for (;;) {
            const size_t ri = next.fetch_add(1);
            if (ri >= rest.size()) return;
            const size_t i = rest[ri];
            fh_error_info e{};
            const fh_status st = fh_sweep(systems[i], freqs[i], nf[i], precision, z_out[i], nullptr, &e);
            if (st) {
                std::lock_guard<std::mutex> lk(mu);
                if (i < failed) {
                    failed = i;
                    failed_status = st;
                    failed_info = e;
                    const char *m = fh_last_error();
                    failed_msg = m ? m : "";
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < workers; ++t) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
    for (size_t i = 0; i < k; ++i) systems[i]->share = 1;
    if (failed < k) {
        fh_status st = fail(err, failed_status, "system " + std::to_string(failed) + ": " + failed_msg,
                            failed_info.index_a, failed_info.index_b, failed_info.frequency, (int32_t)failed);
        if (err) {
            err->iterations = failed_info.iterations;
            err->residual = failed_info.residual;
        }
        return st;
    }
    return FH_OK;
}

fh_status fh_impedance(fh_system *sys, double frequency_hz, fh_precision precision, double *z_out,
                       fh_error_info *err) {
    return fh_sweep(sys, &frequency_hz, 1, precision, z_out, nullptr, err);
}

fh_status fh_system_layout(const fh_system *sys, int64_t *segment_of_filament, int64_t *conductor_of_segment,
                           int64_t *conductor_count) {
    if (!sys) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null system");
    if (segment_of_filament)
        std::copy(sys->segment_of_filament.begin(), sys->segment_of_filament.end(), segment_of_filament);
    if (conductor_of_segment)
        std::copy(sys->conductor_of_segment.begin(), sys->conductor_of_segment.end(), conductor_of_segment);
    if (conductor_count) *conductor_count = sys->conductors;
    return FH_OK;
}

fh_status fh_currents(fh_system *sys, const double *freqs, size_t nf, const double *excitation, size_t n_excitation,
                      fh_precision precision, double *filament_current, double *current_density, double *power_w,
                      double *segment_current, double *segment_power_w, int64_t *conductor_peak_filament,
                      double *conductor_peak_density, fh_power_balance *balance, fh_error_info *err) {
    clear_error(err);
    if (!sys || (nf && !freqs) || (n_excitation && !excitation))
        return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    for (size_t k = 0; k < nf; ++k)
        if (!(std::isfinite(freqs[k]) && freqs[k] >= 0.0))
            return fail(err, FH_ERR_INVALID_FREQUENCY,
                        "frequency " + std::to_string(k) + " is " + fstr(freqs[k]) +
                            " Hz; frequencies must be finite and non-negative",
                        (int64_t)k, -1, freqs[k]);
    const int64_t n = sys->n, m = sys->m, p = sys->p, loops = sys->nloops;
    const int64_t nseg = (int64_t)sys->segments.size(), ncond = sys->conductors;
    bool finite = (int64_t)n_excitation == p;
    for (size_t q = 0; q < 2 * n_excitation && finite; ++q) finite = std::isfinite(excitation[q]);
    if (!finite)
        return fail(err, FH_ERR_INVALID_EXCITATION,
                    "excitation must have one finite entry per port (" + std::to_string(p) + "), got " +
                        std::to_string(n_excitation) + " entries",
                    p, (int64_t)n_excitation);
    if (precision < FH_PRECISION_FP64 || precision > FH_PRECISION_MIXED_FP32)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "unknown precision");
    if (nf == 0) return FH_OK;
    FHB_CUDA(cudaSetDevice(sys->device));
    cudaStream_t st = sys->stream;
    // Device layout, once: per branch its (loop, sign) in increasing loop order.
    if (!sys->d_col_ptr) {
        TransposedLoops cols;
        transpose_loops(sys->loops, n, loops, cols);
        const std::vector<int64_t> &col_ptr = cols.offset;
        const std::vector<int32_t> &col_loop = cols.loop;
        const std::vector<double> &col_sign = cols.sign;
        std::vector<double> whr((size_t)(3 * n));
        for (int64_t k = 0; k < n; ++k) {
            whr[(size_t)(3 * k)] = sys->disc.filaments[(size_t)k].width;
            whr[(size_t)(3 * k + 1)] = sys->disc.filaments[(size_t)k].height;
            whr[(size_t)(3 * k + 2)] = sys->resistances[(size_t)k];
        }
        auto up = [&](void **d, const void *h, size_t bytes) -> cudaError_t {
            cudaError_t e = cache_alloc(d, bytes, st);
            if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(*d, h, bytes, cudaMemcpyHostToDevice, st);
            return e;
        };
        FHB_CUDA(up((void **)&sys->d_col_ptr, col_ptr.data(), 8 * col_ptr.size()));
        FHB_CUDA(up((void **)&sys->d_col_loop, col_loop.data(), 4 * col_loop.size()));
        FHB_CUDA(up((void **)&sys->d_col_sign, col_sign.data(), 8 * col_sign.size()));
        FHB_CUDA(up((void **)&sys->d_whr, whr.data(), 8 * whr.size()));
        FHB_CUDA(up((void **)&sys->d_first, sys->segment_first.data(), 8 * sys->segment_first.size()));
        FHB_CUDA(cudaStreamSynchronize(st));
    }
    const bool mixed = precision != FH_PRECISION_FP64;
    const TrailingUpdate update =
        precision == FH_PRECISION_MIXED_BF16X3 ? TrailingUpdate::TensorBf16x3 : TrailingUpdate::Simt;
    size_t free_b = 0, total_b = 0;
    FHB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    free_b = (free_b + cache_idle_bytes()) / (size_t)std::max(1, sys->share) + sys->pool.held();
    const double per = (mixed ? 8.0 : 16.0) * (double)m * (double)m + 64.0 * (double)(m * p + 64) + 48.0 * (double)n +
                       32.0 * (double)nseg +
                       (outer_for(m, update) ? 16.0 * (double)m * kOuterFp32 + 16.0 * (double)(m + kNbFp32) * kNbFp32 +
                                                   16.0 * kOuterFp32 * kOuterFp32 + 8.0 * kNbFp32 * kOuterFp32
                                             : 0.0);
    const int chunk = (int)std::max(1.0, std::min<double>((double)nf, 0.8 * (double)free_b / std::max(per, 1.0)));
    PBuf<double> d_omega, d_x, d_z;
    FHB_PALLOC(sys->pool, d_omega, kSlotOmega, (size_t)chunk);
    FHB_PALLOC(sys->pool, d_x, kSlotX, (size_t)std::max<int64_t>(1, chunk * m * p * 2));
    FHB_PALLOC(sys->pool, d_z, kSlotZ, (size_t)chunk * p * p * 2);
    DBuf<double> d_ip(st), d_ib(st), d_dens(st), d_pow(st), d_segc(st), d_segp(st), d_segpk(st);
    DBuf<int64_t> d_segi(st);
    FHB_ALLOC(d_ip, (size_t)(2 * p));
    FHB_ALLOC(d_ib, (size_t)(chunk * n * 2));
    FHB_ALLOC(d_dens, (size_t)(chunk * n));
    FHB_ALLOC(d_pow, (size_t)(chunk * n));
    FHB_ALLOC(d_segc, (size_t)(chunk * nseg * 2));
    FHB_ALLOC(d_segp, (size_t)(chunk * nseg));
    FHB_ALLOC(d_segpk, (size_t)(chunk * nseg));
    FHB_ALLOC(d_segi, (size_t)(chunk * nseg));
    FHB_CUDA(cudaMemcpyAsync(d_ip.p, excitation, 16 * (size_t)p, cudaMemcpyHostToDevice, st));
    typedef std::complex<double> C;
    std::vector<double> z((size_t)(chunk * p * p * 2)), segp((size_t)(chunk * nseg)), segpk((size_t)(chunk * nseg));
    std::vector<int64_t> segi((size_t)(chunk * nseg));
    float ms_factor = 0, ms_refine = 0;
    for (size_t c0 = 0; c0 < nf; c0 += (size_t)chunk) {
        const int count = (int)std::min<size_t>((size_t)chunk, nf - c0);
        std::vector<double> omega((size_t)count);
        for (int f = 0; f < count; ++f) omega[(size_t)f] = kTau * freqs[c0 + (size_t)f];
        FHB_CUDA(cudaMemcpyAsync(d_omega.p, omega.data(), 8 * (size_t)count, cudaMemcpyHostToDevice, st));
        std::vector<int> singular((size_t)count, 0), failed((size_t)count, 0);
        fh_status e;
        bool redo = false;
        if (mixed) {
            e = sweep_chunk_mixed(sys, d_omega.p, count, d_x.p, d_z.p, singular.data(), failed.data(), nullptr,
                                  nullptr, &ms_factor, &ms_refine, update, err);
            if (e) return e;
            for (int f = 0; f < count; ++f) redo = redo || failed[(size_t)f];
        }
        if (!mixed || redo) {  // refinement that did not converge: the whole batch in FP64
            e = sweep_chunk_fp64(sys, d_omega.p, count, d_x.p, d_z.p, singular.data(), &ms_factor, err);
            if (e) return e;
        }
        e = launch_currents(d_x.p, d_ip.p, m, (int)p, false, n, count, sys->d_col_ptr, sys->d_col_loop, sys->d_col_sign,
                            sys->d_whr, sys->d_first, nseg, d_ib.p, d_dens.p, d_pow.p, d_segc.p, d_segp.p, d_segpk.p,
                            d_segi.p, st, err);
        if (e) return e;
        FHB_CUDA(cudaMemcpyAsync(z.data(), d_z.p, 16 * (size_t)(count * p * p), cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaMemcpyAsync(segp.data(), d_segp.p, 8 * (size_t)(count * nseg), cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaMemcpyAsync(segpk.data(), d_segpk.p, 8 * (size_t)(count * nseg), cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaMemcpyAsync(segi.data(), d_segi.p, 8 * (size_t)(count * nseg), cudaMemcpyDeviceToHost, st));
        const size_t o = c0;
        if (filament_current)
            FHB_CUDA(cudaMemcpyAsync(filament_current + 2 * o * n, d_ib.p, 16 * (size_t)(count * n),
                                     cudaMemcpyDeviceToHost, st));
        if (current_density)
            FHB_CUDA(cudaMemcpyAsync(current_density + o * n, d_dens.p, 8 * (size_t)(count * n),
                                     cudaMemcpyDeviceToHost, st));
        if (power_w)
            FHB_CUDA(cudaMemcpyAsync(power_w + o * n, d_pow.p, 8 * (size_t)(count * n), cudaMemcpyDeviceToHost, st));
        if (segment_current)
            FHB_CUDA(cudaMemcpyAsync(segment_current + 2 * o * nseg, d_segc.p, 16 * (size_t)(count * nseg),
                                     cudaMemcpyDeviceToHost, st));
        FHB_CUDA(cudaStreamSynchronize(st));
        // Singular or non-finite: the first such frequency in list order.
        for (int f = 0; f < count; ++f) {
            bool bad = singular[(size_t)f] != 0;
            for (int64_t q = 0; q < 2 * p * p && !bad; ++q) bad = !std::isfinite(z[(size_t)(2 * f * p * p + q)]);
            if (bad)
                return fail(err, FH_ERR_SINGULAR,
                            "the mesh system is singular or ill-conditioned at " + fstr(freqs[c0 + (size_t)f]) + " Hz",
                            (int64_t)(c0 + (size_t)f), -1, freqs[c0 + (size_t)f]);
        }
        for (int f = 0; f < count; ++f) {
            const size_t k = c0 + (size_t)f;
            if (segment_power_w)
                std::copy(segp.begin() + (size_t)f * nseg, segp.begin() + (size_t)(f + 1) * nseg,
                          segment_power_w + k * nseg);
            // Conductor peaks: segments are contiguous in filament order, so
            // the first strictly larger segment peak is the reference's
            // first filament of largest |J|.
            std::vector<double> best((size_t)ncond, -1.0);
            std::vector<int64_t> at((size_t)ncond, -1);
            double dissipated = 0.0;
            for (int64_t g = 0; g < nseg; ++g) {
                const size_t t = (size_t)(f * nseg + g);
                dissipated += segp[t];
                const int64_t c = sys->conductor_of_segment[(size_t)g];
                if (segi[t] >= 0 && (at[(size_t)c] < 0 || segpk[t] > best[(size_t)c])) {
                    best[(size_t)c] = segpk[t];
                    at[(size_t)c] = segi[t];
                }
            }
            if (conductor_peak_filament) std::copy(at.begin(), at.end(), conductor_peak_filament + k * ncond);
            if (conductor_peak_density) std::copy(best.begin(), best.end(), conductor_peak_density + k * ncond);
            if (balance) {
                // V_p = Z I_p; input = 1/2 Re(I_p^H V_p).
                double input = 0.0;
                for (int64_t a = 0; a < p; ++a) {
                    C v(0.0, 0.0);
                    for (int64_t b = 0; b < p; ++b) {
                        const size_t zi = (size_t)(2 * (f * p * p + a * p + b));
                        v += C(z[zi], z[zi + 1]) * C(excitation[2 * b], excitation[2 * b + 1]);
                    }
                    input += (std::conj(C(excitation[2 * a], excitation[2 * a + 1])) * v).real();
                }
                input *= 0.5;
                const double scale = std::max(dissipated, input);
                balance[k] = fh_power_balance{dissipated, input, scale > 0.0 ? std::fabs(dissipated - input) / scale : 0.0};
            }
        }
    }
    return FH_OK;
}

// ---------------------------------------------------------------------------
// Impedance gradient by the stationary form (no reference counterpart).
// Z_ab = I_a^T Zm I_b with the loop currents I = [-Z_ee^-1 Z_ep; 1] of unit
// port currents; Zm = M (R + j w L) M^T is complex symmetric and Zm I has no
// internal-loop rows, so the first-order change of I drops out and
// dZ_ab = (M^T I_a)^T (dR + j w dL) (M^T I_b).
// ---------------------------------------------------------------------------
fh_status fh_gradient(fh_system *sys, double frequency_hz, const fh_param_spec *params, size_t np, double *z_out,
                      double *dz_out, fh_gradient_report *report, fh_error_info *err) {
    clear_error(err);
    if (!sys || (np && (!params || !dz_out))) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    if (!(std::isfinite(frequency_hz) && frequency_hz >= 0.0))
        return fail(err, FH_ERR_INVALID_FREQUENCY,
                    "frequency 0 is " + fstr(frequency_hz) + " Hz; frequencies must be finite and non-negative", 0, -1,
                    frequency_hz);
    const int64_t nseg = (int64_t)sys->segments.size(), nnodes = (int64_t)sys->nodes.size();
    // Segments that meet at a node (for node-coordinate parameters).
    std::vector<std::vector<int64_t>> at_node((size_t)nnodes);
    for (int64_t g = 0; g < nseg; ++g) {
        at_node[(size_t)sys->segments[(size_t)g].a].push_back(g);
        at_node[(size_t)sys->segments[(size_t)g].b].push_back(g);
    }
    std::vector<int64_t> first_fil((size_t)nseg + 1, 0);
    for (int64_t g = 0; g < nseg; ++g) first_fil[(size_t)g + 1] = first_fil[(size_t)g] + sys->disc.per_segment[(size_t)g];
    bool want_dims = false, want_coords = false;
    std::vector<uint8_t> seg_moves((size_t)nseg, 0);
    for (size_t k = 0; k < np; ++k) {
        const fh_param_spec &q = params[k];
        if (q.kind == FH_PARAM_NODE_X || q.kind == FH_PARAM_NODE_Y) {
            if (q.index < 0 || q.index >= nnodes)
                return fail(err, FH_ERR_INVALID_ARGUMENT,
                            "parameter " + std::to_string(k) + " names node " + std::to_string(q.index) +
                                ", but the geometry has " + std::to_string(nnodes),
                            (int64_t)k, q.index);
            // A node moving in the xy plane turns its segments about z: every
            // filament of them must lie in the plane with z along one of its
            // cross-section axes, so that its frame turns with it.
            for (int64_t g : at_node[(size_t)q.index]) {
                const fh_filament &f = sys->disc.filaments[(size_t)first_fil[(size_t)g]];
                const bool flat = std::fabs(f.dir_length[2]) <= 1e-12 &&
                                  (std::fabs(std::fabs(f.dir_width[2]) - 1.0) <= 1e-12 ||
                                   std::fabs(std::fabs(f.dir_height[2]) - 1.0) <= 1e-12);
                if (!flat)
                    return fail(err, FH_ERR_UNSUPPORTED,
                                "parameter " + std::to_string(k) + " moves node " + std::to_string(q.index) +
                                    ", which segment " + std::to_string(g) +
                                    " joins; node-coordinate derivatives need segments in a plane z = const "
                                    "with z along their width or height",
                                (int64_t)k, g);
                seg_moves[(size_t)g] = 1;
            }
            want_coords = true;
            continue;
        }
        if (q.kind == FH_PARAM_NODE_Z)
            return fail(err, FH_ERR_UNSUPPORTED,
                        "parameter " + std::to_string(k) +
                            " is a node's z coordinate; node-coordinate derivatives are provided for x and y",
                        (int64_t)k);
        if (q.kind != FH_PARAM_WIDTH && q.kind != FH_PARAM_THICKNESS)
            return fail(err, FH_ERR_INVALID_ARGUMENT, "parameter " + std::to_string(k) + " has an unknown kind",
                        (int64_t)k);
        if (q.index < 0 || q.index >= nseg)
            return fail(err, FH_ERR_INVALID_ARGUMENT,
                        "parameter " + std::to_string(k) + " names segment " + std::to_string(q.index) +
                            ", but the geometry has " + std::to_string(nseg),
                        (int64_t)k, q.index);
        want_dims = true;
    }
    FHB_CUDA(cudaSetDevice(sys->device));
    const double t0 = wall();
    const int64_t n = sys->n, m = sys->m, p = sys->p, loops = sys->nloops;
    cudaStream_t st = sys->stream;
    // 1. Loop currents X = Z_ee^-1 Z_ep and Z, in FP64.
    PBuf<double> d_omega, d_x, d_z;
    FHB_PALLOC(sys->pool, d_omega, kSlotOmega, 1);
    FHB_PALLOC(sys->pool, d_x, kSlotX, (size_t)std::max<int64_t>(1, m * p * 2));
    FHB_PALLOC(sys->pool, d_z, kSlotZ, (size_t)p * p * 2);
    const double omega = kTau * frequency_hz;
    FHB_CUDA(cudaMemcpyAsync(d_omega.p, &omega, 8, cudaMemcpyHostToDevice, st));
    int singular = 0;
    fh_status e = sweep_chunk_fp64(sys, d_omega.p, 1, d_x.p, d_z.p, &singular, nullptr, err);
    if (e) return e;
    std::vector<double> x((size_t)(m * p * 2)), z((size_t)(p * p * 2));
    if (m) FHB_CUDA(cudaMemcpyAsync(x.data(), d_x.p, 8 * x.size(), cudaMemcpyDeviceToHost, st));
    FHB_CUDA(cudaMemcpyAsync(z.data(), d_z.p, 8 * z.size(), cudaMemcpyDeviceToHost, st));
    FHB_CUDA(cudaStreamSynchronize(st));
    bool bad = singular != 0;
    for (double v : z) bad = bad || !std::isfinite(v);
    if (bad)
        return fail(err, FH_ERR_SINGULAR,
                    "the mesh system is singular or ill-conditioned at " + fstr(frequency_hz) + " Hz", 0, -1,
                    frequency_hz);
    const double t1 = wall();
    // 2. Branch currents I_b = M^T [-X; 1], n x p complex (column q at 2 q n).
    std::vector<double> ib((size_t)(2 * n * p), 0.0);
    for (int64_t r = 0; r < loops; ++r)
        for (int64_t q = 0; q < p; ++q) {
            double re, im;
            if (r < m) {
                re = -x[2 * (q * m + r)];
                im = -x[2 * (q * m + r) + 1];
            } else {
                re = r - m == q ? 1.0 : 0.0;
                im = 0.0;
            }
            if (re == 0.0 && im == 0.0) continue;
            for (int64_t k = sys->loops.row_ptr[r]; k < sys->loops.row_ptr[r + 1]; ++k) {
                const int64_t b = sys->loops.branch[k];
                const double sg = sys->loops.sign[k];
                ib[2 * (q * n + b)] += sg * re;
                ib[2 * (q * n + b) + 1] += sg * im;
            }
        }
    // 3. How each filament moves with its segment's width and thickness:
    // the discretization places it at a + W c_w w + H c_h h with its own
    // width f_w w and height f_h h (counts and grading ratios fixed).
    std::vector<FilTan> tan((size_t)n);
    std::vector<int64_t> seg_of((size_t)n);
    {
        int64_t i = 0;
        for (int64_t s = 0; s < nseg; ++s) {
            const fh_segment_def &sd = sys->segments[(size_t)s];
            const fh_node &a = sys->nodes[(size_t)sd.a];
            for (int64_t k = 0; k < sys->disc.per_segment[(size_t)s]; ++k, ++i) {
                const fh_filament &f = sys->disc.filaments[(size_t)i];
                const double d[3] = {f.start[0] - a.x, f.start[1] - a.y, f.start[2] - a.z};
                const double cw = d[0] * f.dir_width[0] + d[1] * f.dir_width[1] + d[2] * f.dir_width[2];
                const double ch = d[0] * f.dir_height[0] + d[1] * f.dir_height[1] + d[2] * f.dir_height[2];
                tan[(size_t)i] = FilTan{cw / sd.width, ch / sd.height, f.width / sd.width, f.height / sd.height};
                seg_of[(size_t)i] = s;
            }
        }
    }
    // 4. Derivative fills and the products with the branch currents.
    size_t free_b = 0, total_b = 0;
    FHB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t part = gradient_part_elems(n, (int)p);
    const double need = (want_dims ? 16.0 : 0.0) * (double)n * (double)n +
                        (want_coords ? 32.0 * (double)n * (double)n + 64.0 * (double)(n * p) : 0.0) +
                        8.0 * (double)(part + 6 * n * p) + 296.0 * (double)n;
    if (need > 0.9 * (double)free_b)
        return fail(err, FH_ERR_OUT_OF_MEMORY,
                    "the derivative fill of " + std::to_string(n) + " filaments needs " + fstr(need) +
                        " bytes of device memory; " + std::to_string(free_b) + " are free");
    std::vector<DevFil> h((size_t)n);
    for (int64_t i = 0; i < n; ++i) h[(size_t)i] = make_devfil(sys->disc.filaments[(size_t)i]);
    DBuf<DevFil> d_fil(st);
    DBuf<FilTan> d_tan(st);
    DBuf<double> d_D(st), d_I(st), d_y(st), d_part(st), d_C(st), d_yc(st);
    DBuf<int32_t> d_seg(st);
    DBuf<uint8_t> d_move(st);
    FHB_ALLOC(d_fil, (size_t)n);
    FHB_ALLOC(d_tan, (size_t)n);
    FHB_ALLOC(d_D, (size_t)(want_dims ? 2 * n * n : 1));
    FHB_ALLOC(d_I, (size_t)(2 * n * p));
    FHB_ALLOC(d_y, (size_t)(4 * n * p));
    FHB_ALLOC(d_part, part);
    FHB_CUDA(cudaMemcpyAsync(d_fil.p, h.data(), sizeof(DevFil) * n, cudaMemcpyHostToDevice, st));
    FHB_CUDA(cudaMemcpyAsync(d_tan.p, tan.data(), sizeof(FilTan) * n, cudaMemcpyHostToDevice, st));
    FHB_CUDA(cudaMemcpyAsync(d_I.p, ib.data(), 8 * ib.size(), cudaMemcpyHostToDevice, st));
    if (want_dims) FHB_CUDA(cudaMemsetAsync(d_D.p, 0, 16 * (size_t)n * n, st));
    std::vector<int32_t> seg32((size_t)n);
    std::vector<uint8_t> move((size_t)n);
    if (want_coords) {
        for (int64_t i = 0; i < n; ++i) {
            seg32[(size_t)i] = (int32_t)seg_of[(size_t)i];
            move[(size_t)i] = seg_moves[(size_t)seg_of[(size_t)i]];
        }
        FHB_ALLOC(d_C, (size_t)(4 * n * n));
        FHB_ALLOC(d_yc, (size_t)(8 * n * p));
        FHB_ALLOC(d_seg, (size_t)n);
        FHB_ALLOC(d_move, (size_t)n);
        FHB_CUDA(cudaMemcpyAsync(d_seg.p, seg32.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, st));
        FHB_CUDA(cudaMemcpyAsync(d_move.p, move.data(), (size_t)n, cudaMemcpyHostToDevice, st));
        FHB_CUDA(cudaMemsetAsync(d_C.p, 0, 32 * (size_t)n * n, st));
    }
    cudaEvent_t ev[3];
    for (auto &v : ev) FHB_CUDA(cudaEventCreate(&v));
    struct EvGuard {
        cudaEvent_t *ev;
        ~EvGuard() {
            for (int k = 0; k < 3; ++k) cudaEventDestroy(ev[k]);
        }
    } evg{ev};
    FillStats fs, fc;
    FHB_CUDA(cudaEventRecord(ev[0], st));
    const PairMaskDev pm = sys->mask();
    if (want_dims) {
        e = device_fill_grad(d_fil.p, d_tan.p, n, GradOut{d_D.p, d_D.p + n * n}, st, &fs, err, &pm);
        if (e) return e;
    }
    if (want_coords) {
        const size_t nn = (size_t)(n * n);
        e = device_fill_coord(d_fil.p, d_seg.p, d_move.p, n,
                              CoordOut{d_C.p, d_C.p + nn, d_C.p + 2 * nn, d_C.p + 3 * nn}, st, &fc, err, &pm);
        if (e) return e;
    }
    FHB_CUDA(cudaEventRecord(ev[1], st));
    if (want_dims) {
        e = gradient_products(d_D.p, d_D.p + n * n, n, d_I.p, (int)p, d_y.p, d_part.p, st, err);
        if (e) return e;
    }
    if (want_coords) {
        const size_t nn = (size_t)(n * n);
        e = gradient_products(d_C.p, d_C.p + nn, n, d_I.p, (int)p, d_yc.p, d_part.p, st, err);
        if (e) return e;
        e = gradient_products(d_C.p + 2 * nn, d_C.p + 3 * nn, n, d_I.p, (int)p, d_yc.p + 4 * n * p, d_part.p, st,
                              err);
        if (e) return e;
    }
    FHB_CUDA(cudaEventRecord(ev[2], st));
    std::vector<double> y((size_t)(4 * n * p)), yc(want_coords ? (size_t)(8 * n * p) : 0);
    if (want_dims) FHB_CUDA(cudaMemcpyAsync(y.data(), d_y.p, 8 * y.size(), cudaMemcpyDeviceToHost, st));
    if (want_coords) FHB_CUDA(cudaMemcpyAsync(yc.data(), d_yc.p, 8 * yc.size(), cudaMemcpyDeviceToHost, st));
    FHB_CUDA(cudaStreamSynchronize(st));
    float ms_fill = 0, ms_prod = 0;
    cudaEventElapsedTime(&ms_fill, ev[0], ev[1]);
    cudaEventElapsedTime(&ms_prod, ev[1], ev[2]);
    // 5. Per segment and kind: sum over its filaments of
    //    I_a I_b dR_i + j w (I_a (D I_b)_i + I_b (D I_a)_i).
    typedef std::complex<double> C;
    const size_t pp = (size_t)(p * p);
    std::vector<C> acc((size_t)(2 * nseg) * pp, C(0.0, 0.0));
    auto I = [&](int64_t q, int64_t i) { return C(ib[2 * (q * n + i)], ib[2 * (q * n + i) + 1]); };
    auto Y = [&](int which, int64_t q, int64_t i) {
        const size_t o = (size_t)(2 * (((int64_t)which * p + q) * n + i));
        return C(y[o], y[o + 1]);
    };
    const C jw(0.0, omega);
    if (want_dims)
        for (int64_t i = 0; i < n; ++i) {
            const fh_filament &f = sys->disc.filaments[(size_t)i];
            const double r = sys->resistances[(size_t)i];
            const double dr[2] = {-r * tan[(size_t)i].gw / f.width, -r * tan[(size_t)i].gh / f.height};
            for (int which = 0; which < 2; ++which) {
                C *out = acc.data() + (size_t)(2 * seg_of[(size_t)i] + which) * pp;
                for (int64_t a = 0; a < p; ++a)
                    for (int64_t b = 0; b < p; ++b)
                        out[a * p + b] += I(a, i) * I(b, i) * dr[which] +
                                          jw * (I(a, i) * Y(which, b, i) + I(b, i) * Y(which, a, i));
            }
        }
    // Node coordinates: a node moving by e (x or y) moves the segment a -> b
    // with da or db = e; every filament of it stretches by dl = l . (db - da),
    // turns about z by dphi = (z x l) . (db - da) / length, and its centre
    // moves by (da + db) / 2 + dphi z x (c - (a + b) / 2).  Its resistance
    // changes by R dl / length.
    auto YC = [&](int which, int64_t q, int64_t i) {
        const size_t o = (size_t)(2 * (((int64_t)which * p + q) * n + i));
        return C(yc[o], yc[o + 1]);
    };
    auto node_grad = [&](int64_t node, int axis, C *out) {
        for (size_t q = 0; q < pp; ++q) out[q] = C(0.0, 0.0);
        for (int64_t g : at_node[(size_t)node]) {
            const fh_segment_def &sd = sys->segments[(size_t)g];
            const fh_node &na = sys->nodes[(size_t)sd.a], &nb = sys->nodes[(size_t)sd.b];
            double da[3] = {0, 0, 0}, db[3] = {0, 0, 0};
            if (sd.a == node) da[axis] = 1.0;
            if (sd.b == node) db[axis] = 1.0;
            const double span[3] = {nb.x - na.x, nb.y - na.y, nb.z - na.z};
            const double len = std::sqrt(span[0] * span[0] + span[1] * span[1] + span[2] * span[2]);
            const double l[3] = {span[0] / len, span[1] / len, span[2] / len};
            const double dd[3] = {db[0] - da[0], db[1] - da[1], db[2] - da[2]};
            const double dl = l[0] * dd[0] + l[1] * dd[1] + l[2] * dd[2];
            const double dphi = (-l[1] * dd[0] + l[0] * dd[1]) / len;
            const double mid[3] = {0.5 * (na.x + nb.x), 0.5 * (na.y + nb.y), 0.5 * (na.z + nb.z)};
            for (int64_t i = first_fil[(size_t)g]; i < first_fil[(size_t)g + 1]; ++i) {
                const fh_filament &f = sys->disc.filaments[(size_t)i];
                const double o[3] = {0.5 * (f.start[0] + f.end[0]) - mid[0], 0.5 * (f.start[1] + f.end[1]) - mid[1],
                                     0.5 * (f.start[2] + f.end[2]) - mid[2]};
                const double dc[3] = {0.5 * (da[0] + db[0]) - dphi * o[1], 0.5 * (da[1] + db[1]) + dphi * o[0],
                                      0.5 * (da[2] + db[2])};
                const double *fl = f.dir_length;
                double pl[3] = {-fl[1], fl[0], 0.0};
                const double pn = std::sqrt(pl[0] * pl[0] + pl[1] * pl[1]);
                for (double &v : pl) v = pn > 0.0 ? v / pn : 0.0;
                const double dq[4] = {dc[0] * fl[0] + dc[1] * fl[1] + dc[2] * fl[2], dc[0] * pl[0] + dc[1] * pl[1], dl,
                                      dphi};
                const double drl = sys->resistances[(size_t)i] * dl / f.length;
                for (int64_t a = 0; a < p; ++a)
                    for (int64_t b = 0; b < p; ++b) {
                        C sum(0.0, 0.0);
                        for (int w = 0; w < 4; ++w)
                            if (dq[w] != 0.0) sum += dq[w] * (I(a, i) * YC(w, b, i) + I(b, i) * YC(w, a, i));
                        out[a * p + b] += I(a, i) * I(b, i) * drl + jw * sum;
                    }
            }
        }
    };
    std::vector<C> node_out(pp);
    for (size_t k = 0; k < np; ++k) {
        const C *src;
        if (params[k].kind == FH_PARAM_NODE_X || params[k].kind == FH_PARAM_NODE_Y) {
            node_grad(params[k].index, params[k].kind == FH_PARAM_NODE_X ? 0 : 1, node_out.data());
            src = node_out.data();
        } else {
            src = acc.data() + (size_t)(2 * params[k].index + (params[k].kind == FH_PARAM_THICKNESS)) * pp;
        }
        for (size_t q = 0; q < pp; ++q) {
            dz_out[2 * (k * pp + q)] = src[q].real();
            dz_out[2 * (k * pp + q) + 1] = src[q].imag();
        }
    }
    if (z_out) std::memcpy(z_out, z.data(), 8 * z.size());
    if (report) {
        report->solve_s = t1 - t0;
        report->derivative_fill_s = ms_fill * 1e-3;
        report->contract_s = ms_prod * 1e-3;
        report->total_s = wall() - t0;
        report->pairs = want_dims ? fs.pairs : fc.pairs;
    }
    return FH_OK;
}

fh_status fh_test_inductance_gradient(const fh_filament *filaments, const double *tangents, size_t n, double *Dw,
                                      double *Dh, fh_error_info *err) {
    clear_error(err);
    if (n && (!filaments || !tangents || !Dw || !Dh)) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    fh_status st = ensure_device(err);
    if (st) return st;
    if (n == 0) return FH_OK;
    std::vector<DevFil> h(n);
    std::vector<FilTan> t(n);
    for (size_t i = 0; i < n; ++i) {
        h[i] = make_devfil(filaments[i]);
        t[i] = FilTan{tangents[4 * i], tangents[4 * i + 1], tangents[4 * i + 2], tangents[4 * i + 3]};
    }
    DBuf<DevFil> d_fil;
    DBuf<FilTan> d_tan;
    DBuf<double> d_D;
    FHB_ALLOC(d_fil, n);
    FHB_ALLOC(d_tan, n);
    FHB_ALLOC(d_D, 2 * n * n);
    cudaStream_t s;
    FHB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, decltype(&cudaStreamDestroy)> guard(s, &cudaStreamDestroy);
    FHB_CUDA(cudaMemcpyAsync(d_fil.p, h.data(), n * sizeof(DevFil), cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemcpyAsync(d_tan.p, t.data(), n * sizeof(FilTan), cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemsetAsync(d_D.p, 0, 16 * n * n, s));
    st = device_fill_grad(d_fil.p, d_tan.p, (int64_t)n, GradOut{d_D.p, d_D.p + n * n}, s, nullptr, err);
    if (st) return st;
    FHB_CUDA(cudaMemcpyAsync(Dw, d_D.p, 8 * n * n, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaMemcpyAsync(Dh, d_D.p + n * n, 8 * n * n, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    return FH_OK;
}

fh_status fh_test_coordinate_gradient(const fh_filament *filaments, const int32_t *segment, size_t n, double *Dl,
                                      double *Dp, double *Ds, double *Dr, fh_error_info *err) {
    clear_error(err);
    if (n && (!filaments || !segment || !Dl || !Dp || !Ds || !Dr))
        return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    fh_status st = ensure_device(err);
    if (st) return st;
    if (n == 0) return FH_OK;
    std::vector<DevFil> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = make_devfil(filaments[i]);
    const std::vector<uint8_t> move(n, 1);
    DBuf<DevFil> d_fil;
    DBuf<int32_t> d_seg;
    DBuf<uint8_t> d_move;
    DBuf<double> d_D;
    FHB_ALLOC(d_fil, n);
    FHB_ALLOC(d_seg, n);
    FHB_ALLOC(d_move, n);
    FHB_ALLOC(d_D, 4 * n * n);
    cudaStream_t s;
    FHB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, decltype(&cudaStreamDestroy)> guard(s, &cudaStreamDestroy);
    FHB_CUDA(cudaMemcpyAsync(d_fil.p, h.data(), n * sizeof(DevFil), cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemcpyAsync(d_seg.p, segment, n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemcpyAsync(d_move.p, move.data(), n, cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemsetAsync(d_D.p, 0, 32 * n * n, s));
    const size_t nn = n * n;
    st = device_fill_coord(d_fil.p, d_seg.p, d_move.p, (int64_t)n,
                           CoordOut{d_D.p, d_D.p + nn, d_D.p + 2 * nn, d_D.p + 3 * nn}, s, nullptr, err);
    if (st) return st;
    double *outs[4] = {Dl, Dp, Ds, Dr};
    for (int k = 0; k < 4; ++k)
        FHB_CUDA(cudaMemcpyAsync(outs[k], d_D.p + k * nn, 8 * nn, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    return FH_OK;
}

}  // extern "C"
