// fh_lu_solve_c64_noalloc: the device FP64 LU solve without any device
// memory allocation.
//
// Who needs it: a caller that cannot allocate device memory while it solves,
// for example a host application that hands every byte of device memory to
// its own pool or caching allocator (a raw cudaMalloc would bypass that
// pool's accounting, or fail because the pool has already reserved the free
// memory), or a latency-critical service loop in which a cudaMalloc or
// cudaFree, with the device synchronisation they can imply, is not allowed.
// Such a caller already owns the matrix and right-hand-side buffers on the
// device; what the solver still needs is a little scratch (the pivot indices,
// the pivot-search partials, a ticket counter and the zero-pivot flag), and
// here that scratch is a file-scope __device__ array of fixed size instead of
// an allocation.
//
// Limits and behaviour:
//   * order n <= FH_NOALLOC_MAX_ORDER (65536); larger orders are rejected with
//     FH_ERR_INVALID_ARGUMENT before anything is launched;
//   * the scratch array (about 257 KB) lives in every device that loads the
//     library, until the process exits;
//   * the first call in each device context (a device's primary context, and
//     again after cudaDeviceReset has replaced it) looks up the array's
//     device address with cudaGetSymbolAddress, with that device current;
//   * the call waits on the host until the solve has finished on its stream
//     (it reads the zero-pivot flag back with a copy and a stream
//     synchronize), so it cannot be recorded into a CUDA graph: no call may
//     be made while its stream, or the legacy stream, is being captured;
//   * all calls share the one array: calls whose work overlaps on the GPU
//     (concurrent streams, or threads on the same device) race on it and must
//     be serialised by the caller.  Each call clears the parts that must
//     start at zero.
#include <cuda_runtime.h>

#include <mutex>

#include "fh_lu.cuh"

namespace fhb {
namespace {

constexpr int64_t kMaxOrder = FH_NOALLOC_MAX_ORDER;
constexpr int kMaxChunks = 16;
// Layout: pivots[kMaxOrder] (int), singular (int), ticket (unsigned), pad,
// partial_val[kMaxChunks] (double), partial_idx[kMaxChunks] (int).
constexpr size_t kPivotBytes = sizeof(int) * kMaxOrder;
constexpr size_t kFlagsOffset = kPivotBytes;
constexpr size_t kValOffset = kFlagsOffset + 16;
constexpr size_t kIdxOffset = kValOffset + sizeof(double) * kMaxChunks;
constexpr size_t kScratchBytes = kIdxOffset + sizeof(int) * kMaxChunks;

// In host code this name is only a stand-in for the symbol, not a device
// address: host code reaches the array through the address looked up below.
static __device__ __align__(256) unsigned char g_lu_scratch[kScratchBytes];

// The address of the array belongs to the module loaded in one context: a
// cudaDeviceReset ends the primary context, the module is loaded again in the
// next one and the array may move.  So the looked-up address is kept per
// device together with the id of the context it was looked up in, and looked
// up again when the current context is another one.
using CtxGetCurrentFn = int (*)(void **);
using CtxGetIdFn = int (*)(void *, unsigned long long *);

struct ScratchSlot {
    unsigned long long ctx_id = 0;
    void *ptr = nullptr;
};

std::mutex g_mu;
ScratchSlot g_scratch[64];

fh_status current_context_id(unsigned long long *id, fh_error_info *err) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void *f0 = nullptr, *f1 = nullptr;
        cudaDriverEntryPointQueryResult q0, q1;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) != cudaSuccess ||
            q0 != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return fail(err, FH_ERR_CUDA, "fh_lu_solve_c64_noalloc: the driver's context queries are unavailable");
        get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
        get_id = reinterpret_cast<CtxGetIdFn>(f1);
    }
    void *ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, id) != 0)
        return fail(err, FH_ERR_CUDA, "fh_lu_solve_c64_noalloc: no current device context");
    return FH_OK;
}

fh_status scratch_for_current_device(unsigned char **out, fh_error_info *err) {
    int dev = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(err, FH_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    unsigned long long ctx_id = 0;
    fh_status st = current_context_id(&ctx_id, err);
    if (st) return st;
    ScratchSlot &slot = g_scratch[dev];
    if (!slot.ptr || slot.ctx_id != ctx_id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_lu_scratch);
        if (e != cudaSuccess || !p)
            return fail(err, FH_ERR_CUDA, std::string("cudaGetSymbolAddress of the LU scratch failed: ") +
                                              cudaGetErrorString(e));
        slot.ptr = p;
        slot.ctx_id = ctx_id;
    }
    *out = static_cast<unsigned char *>(slot.ptr);
    return FH_OK;
}

}  // namespace
}  // namespace fhb

using namespace fhb;

extern "C" fh_status fh_lu_solve_c64_noalloc(double *a, size_t n, double *b, size_t nrhs, void *stream,
                                             fh_error_info *err) {
    clear_error(err);
    if (n > (size_t)kMaxOrder)
        return fail(err, FH_ERR_INVALID_ARGUMENT,
                    "fh_lu_solve_c64_noalloc: order " + std::to_string(n) + " exceeds the maximum of " +
                        std::to_string((long long)kMaxOrder));
    if (n && (!a || !b)) return fail(err, FH_ERR_INVALID_ARGUMENT, "fh_lu_solve_c64_noalloc: null device pointer");
    if (nrhs > (size_t)INT32_MAX) return fail(err, FH_ERR_INVALID_ARGUMENT, "fh_lu_solve_c64_noalloc: too many columns");
    fh_status st = ensure_device(err);
    if (st) return st;
    if (n == 0 || nrhs == 0) return FH_OK;
    unsigned char *scratch = nullptr;
    st = scratch_for_current_device(&scratch, err);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ProfSuppress no_profile;
    int *pivots = reinterpret_cast<int *>(scratch);
    int *singular = reinterpret_cast<int *>(scratch + kFlagsOffset);
    unsigned *ticket = reinterpret_cast<unsigned *>(scratch + kFlagsOffset + 4);
    // The array keeps the previous call's contents: the flag and the ticket
    // must start at zero.
    FHB_CUDA(cudaMemsetAsync(scratch + kFlagsOffset, 0, 16, s));
    LuWork w;
    w.partial_val = reinterpret_cast<double *>(scratch + kValOffset);
    w.partial_idx = reinterpret_cast<int *>(scratch + kIdxOffset);
    w.tickets = ticket;
    w.max_chunks = kMaxChunks;
    LuBatch<double> lb;
    lb.a = a;
    lb.pivots = pivots;
    lb.singular = singular;
    lb.m = (int64_t)n;
    lb.count = 1;
    st = lu_factor<double>(lb, w, 64, TrailingUpdate::Simt, s, err);
    if (!st) st = lu_solve<double>(lb, b, (int)nrhs, 64, s, err);
    if (st) return st;
    int flag = 0;
    FHB_CUDA(cudaMemcpyAsync(&flag, singular, sizeof(int), cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    if (flag) return fail(err, FH_ERR_SINGULAR, "the matrix is singular (zero pivot)");
    return FH_OK;
}
