// Trailing update of the FP32 complex LU on the 5th-generation tensor cores:
//
//     A22 -= L21 * U12        (complex, FP32 storage, FP32 accumulation)
//
// with every FP32 operand split into two BF16 terms, x = x_hi + x_lo
// (x_hi = bf16(x), x_lo = bf16(x - x_hi)), and each real product formed from
// three BF16 products (hi*hi + hi*lo + lo*hi; the lo*lo term is below the
// FP32 rounding of the sum).  The complex product is four real products:
//
//     Re += Ar Br - Ai Bi        Im += Ar Bi + Ai Br
//
// so one 16-wide complex k-chunk is 12 tcgen05.mma (kind::f16, BF16 inputs,
// FP32 accumulators in TMEM); the minus sign of Ai Bi is the instruction
// descriptor's A-negate bit.
//
// CTA tile: 128 rows x 128 columns of complex C; two accumulators of 128 TMEM
// columns (Re at column 0, Im at column 128).  All 256 threads load the
// chunk's FP32 operands from global memory, split them, and store them to
// shared memory in the canonical K-major no-swizzle layout (8 x 16-byte core
// matrices); thread 0 issues the MMAs and commits them to an mbarrier; chunks
// are double-buffered in shared memory, and the global loads of chunk c+2 are
// issued into registers right after chunk c+1 is stored, so they are in
// flight during the MMAs of chunk c+1.
// The epilogue reads the accumulators with tcgen05.ld (warp w owns TMEM lanes
// 32 (w % 4) .. +31 = rows of the tile, and half w / 4 of the columns) and
// applies C -= acc with coalesced loads and stores, 16 independent loads in
// flight per thread.  The update is bound by the read + write of C (16 bytes
// per complex entry per panel); two CTAs per SM keep enough bytes in flight.
// Every mbarrier wait is bounded; a wait that runs out sets the error flag,
// skips the epilogue and still frees the TMEM.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "fh_lu.cuh"

namespace fhb {

namespace {

constexpr int kTileM = 128;
constexpr int kTileN = 128;
constexpr int kChunk = 16;                                  // complex k per chunk = one MMA K-step
constexpr int kTileBytes = kTileM * kChunk * 2;             // one bf16 operand tile: 4 KB
constexpr int kTilesPerChunk = 8;                           // Ar/Ai hi/lo, Br/Bi hi/lo
constexpr int kBufBytes = kTileBytes * kTilesPerChunk;      // 32 KB
// Two 32 KB buffers + alignment + barriers, padded to 100 KB so that at most
// two CTAs (2 x 256 TMEM columns = all 512) are resident per SM.  The padding
// also keeps every address a descriptor could form inside the allocation.
constexpr int kSmemBytes = 100 * 1024;
constexpr int kTmemCols = 256;
constexpr long long kSpinLimit = 1LL << 22;

// Operand tile order inside a buffer.
enum { ArH = 0, ArL, AiH, AiL, BrH, BrL, BiH, BiL };

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// SM100 shared-memory matrix descriptor, K-major, no swizzle.
// start>>4 at [0,14), LBO>>4 at [16,30), SBO>>4 at [32,46), version 1 at [46,48).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: kind::f16, BF16 x BF16 -> F32, K-major A and B,
// M = 128, N = 128, optional A negate.
__host__ __device__ constexpr uint32_t instr_desc(bool negate_a) {
    return (1u << 4)                     // D format F32
           | (1u << 7)                   // A format BF16
           | (1u << 10)                  // B format BF16
           | ((negate_a ? 1u : 0u) << 13)
           | ((uint32_t)(kTileN >> 3) << 17)
           | ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Bounded wait for the given phase parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kSpinLimit; ++i) {
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

__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Two FP32 values split into BF16 hi and lo terms (x = hi + lo to 16 bits),
// each pair converted by one cvt.rn.bf16x2.f32: the 32-bit words of the hi
// and lo terms, first value in the low half.
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const float2 back = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(a - back.x, b - back.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

// Byte offset of (row r, k-group j) inside a tile: [j][r/8][r%8][8 bf16].
__device__ __forceinline__ uint32_t tile_off(int r, int j) {
    return (uint32_t)(j * (kTileM / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16);
}

constexpr int kThreads = 256;

struct GemmArgs {
    const float2 *A;  // A operand: (row r, k) at A[f sA + r + k lda]
    int64_t lda, sA;
    const float2 *B;  // B operand: (k, column n) at B[f sB + k + n ldb]
    int64_t ldb, sB;
    float2 *C;        // C: (r, n) at C[f sC + r + n ldc]
    int64_t ldc, sC;
    int64_t M, N;
    int K;
    int assign;
};

// 16 consecutive TMEM columns of this warp's 32 lanes (one row per thread).
// Asynchronous: the registers may be read only after tcgen05.wait::ld.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Splits 8 complex values into the four 16-byte core-matrix rows (re hi, re
// lo, im hi, im lo) of tiles t_re_hi, t_re_hi+1, t_im_hi, t_im_hi+1.
__device__ __forceinline__ void split_store8(const float2 *v, uint8_t *buf, int t_re_hi, int t_im_hi, uint32_t off) {
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        split2(v[2 * q].x, v[2 * q + 1].x, rh[q], rl[q]);
        split2(v[2 * q].y, v[2 * q + 1].y, ih[q], il[q]);
    }
    *reinterpret_cast<uint4 *>(buf + t_re_hi * kTileBytes + off) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
    *reinterpret_cast<uint4 *>(buf + (t_re_hi + 1) * kTileBytes + off) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
    *reinterpret_cast<uint4 *>(buf + t_im_hi * kTileBytes + off) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
    *reinterpret_cast<uint4 *>(buf + (t_im_hi + 1) * kTileBytes + off) = make_uint4(il[0], il[1], il[2], il[3]);
}

// Chunk `c` of a thread: 8 values of A (row t % 128 of the tile, k-half
// t / 128) and 8 of B (column t % 128, same k-half), held in registers
// between their global loads and their split into shared memory.
struct ChunkRegs {
    float2 a[8], b[8];
};

// Issues the global loads of chunk `c` (16 columns of A for the tile's 128
// rows and 16 rows of B for its 128 columns): the A loads are coalesced
// across rows, each B column half is one 64-byte run read with 16-byte loads.
__device__ __forceinline__ void load_chunk(const GemmArgs &g, int f, int64_t row0, int64_t col0, int c, ChunkRegs &v) {
    const int t = threadIdx.x & 127, j = threadIdx.x >> 7;
    const int64_t kk = (int64_t)c * kChunk + 8 * j;
    const int64_t row = row0 + t;
    const int64_t col = col0 + t;
    const float2 *Aop = g.A + (int64_t)f * g.sA;
    const float2 *Bop = g.B + (int64_t)f * g.sB;
#pragma unroll
    for (int k = 0; k < 8; ++k) v.a[k] = row < g.M ? __ldg(Aop + row + (kk + k) * g.lda) : make_float2(0.f, 0.f);
    if (col < g.N) {
        const float4 *src = reinterpret_cast<const float4 *>(Bop + kk + col * g.ldb);
        if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 w = __ldg(src + q);
                v.b[2 * q] = make_float2(w.x, w.y);
                v.b[2 * q + 1] = make_float2(w.z, w.w);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) v.b[k] = __ldg(Bop + kk + k + col * g.ldb);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) v.b[k] = make_float2(0.f, 0.f);
    }
}

// Splits a thread's chunk values and stores the 8 operand tiles of `buf`.
__device__ __forceinline__ void store_chunk(const ChunkRegs &v, uint8_t *buf) {
    const uint32_t off = tile_off(threadIdx.x & 127, threadIdx.x >> 7);
    split_store8(v.a, buf, ArH, AiH, off);
    split_store8(v.b, buf, BrH, BiH, off);
}

// C (M x N) = C - A B  (assign == 0), C = A B  (assign == 1) or C = -A B
// (assign == 2), batched over
// blockIdx.z; K a multiple of 16.  In the assign form C may be B itself when
// M <= 128 (one tile row), or A itself when N <= 128 (one tile column): a CTA
// reads all of the aliased operand's part it writes before the epilogue
// writes it, and no other CTA reads that part.
__global__ void __launch_bounds__(kThreads, 2) gemm_bf16x3_kernel(GemmArgs g, int *__restrict__ err_flag) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint8_t *bufs[2] = {smem, smem + kBufBytes};
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * kBufBytes);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);

    const int f = blockIdx.z;
    float2 *C = g.C + (int64_t)f * g.sC;
    const int64_t row0 = (int64_t)blockIdx.y * kTileM;
    const int64_t col0 = (int64_t)blockIdx.x * kTileN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nchunks = g.K / kChunk;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bars[0]), 1);
        mbar_init(smem_u32(&bars[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    ChunkRegs regs;
    load_chunk(g, f, row0, col0, 0, regs);
    store_chunk(regs, bufs[0]);
    if (nchunks > 1) load_chunk(g, f, row0, col0, 1, regs);  // in flight during chunk 0's MMAs
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t tmem_re = tmem, tmem_im = tmem + kTileN;

    bool ok = true;
    uint32_t uses[2] = {0u, 0u};  // commits made on each barrier
    for (int c = 0; c < nchunks && ok; ++c) {
        const int b = c & 1;
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t s = smem_u32(bufs[b]);
            auto d = [&](int tile) { return smem_desc(s + tile * kTileBytes, (kTileM / 8) * 128, 128); };
            const uint32_t acc = c > 0 ? 1u : 0u;
            const uint32_t pos = instr_desc(false), neg = instr_desc(true);
            // Re += Ar Br - Ai Bi
            mma_bf16(tmem_re, d(ArH), d(BrH), pos, acc);
            mma_bf16(tmem_re, d(ArH), d(BrL), pos, 1u);
            mma_bf16(tmem_re, d(ArL), d(BrH), pos, 1u);
            mma_bf16(tmem_re, d(AiH), d(BiH), neg, 1u);
            mma_bf16(tmem_re, d(AiH), d(BiL), neg, 1u);
            mma_bf16(tmem_re, d(AiL), d(BiH), neg, 1u);
            // Im += Ar Bi + Ai Br
            mma_bf16(tmem_im, d(ArH), d(BiH), pos, acc);
            mma_bf16(tmem_im, d(ArH), d(BiL), pos, 1u);
            mma_bf16(tmem_im, d(ArL), d(BiH), pos, 1u);
            mma_bf16(tmem_im, d(AiH), d(BrH), pos, 1u);
            mma_bf16(tmem_im, d(AiH), d(BrL), pos, 1u);
            mma_bf16(tmem_im, d(AiL), d(BrH), pos, 1u);
            mma_commit(smem_u32(&bars[b]));
        }
        uses[b] += 1;
        if (c + 1 < nchunks) {
            const int nbuf = (c + 1) & 1;
            if (uses[nbuf] > 0) {
                // The MMAs of chunk c-1 read buffer nbuf; wait for them.
                if (!mbar_wait(smem_u32(&bars[nbuf]), (uses[nbuf] - 1) & 1)) ok = false;
            }
            if (ok) {
                store_chunk(regs, bufs[nbuf]);  // chunk c + 1, loaded one step ahead
                if (c + 2 < nchunks) load_chunk(g, f, row0, col0, c + 2, regs);
                fence_async_shared();
            }
            tc_fence_before();
            ok = __syncthreads_and(ok);
        }
    }
    // Completion of the last commit implies completion of every earlier MMA.
    if (ok && nchunks > 0) {
        const int b = (nchunks - 1) & 1;
        if (!mbar_wait(smem_u32(&bars[b]), (uses[b] - 1) & 1)) ok = false;
    }
    ok = __syncthreads_and(ok);
    tc_fence_after();
    if (ok) {
        // Warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows) and the
        // column half w / 4, 16 columns at a time; the 16 C loads of a step are
        // issued together before any store.
        const int quarter = warp & 3, half = warp >> 2;
        const int64_t row = row0 + quarter * 32 + lane;
        const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
        for (int cc = half * (kTileN / 2); cc < (half + 1) * (kTileN / 2); cc += 16) {
            uint32_t re[16], im[16];
            tmem_ld16(tmem_re + lane_off + cc, re);
            tmem_ld16(tmem_im + lane_off + cc, im);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < g.M) {
                float2 *p = C + row + (col0 + cc) * g.ldc;
                const int ncol = (int)min((int64_t)16, g.N - (col0 + cc));
                if (g.assign) {
                    const float sg = g.assign == 2 ? -1.f : 1.f;
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj)
                        if (jj < ncol)
                            p[jj * g.ldc] = make_float2(sg * __uint_as_float(re[jj]), sg * __uint_as_float(im[jj]));
                } else {
                    float2 v[16];
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) v[jj] = jj < ncol ? p[jj * g.ldc] : make_float2(0.f, 0.f);
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj)
                        if (jj < ncol)
                            p[jj * g.ldc] =
                                make_float2(v[jj].x - __uint_as_float(re[jj]), v[jj].y - __uint_as_float(im[jj]));
                }
            }
        }
    } else if (threadIdx.x == 0) {
        atomicExch(err_flag, 1);
        // Give MMAs still in flight a second bounded chance to drain before
        // the TMEM and shared memory they use are released.
        if (nchunks > 0) {
            const int b = (nchunks - 1) & 1;
            mbar_wait(smem_u32(&bars[b]), (uses[b] - 1) & 1);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

int *g_err_flag[64] = {nullptr};

}  // namespace

fh_status gemm_tc_launch(const GemmArgs &g, int count, cudaStream_t s, fh_error_info *err) {
    if (g.K % kChunk) return fail(err, FH_ERR_INVALID_ARGUMENT, "tensor-core GEMM needs K a multiple of 16");
    if (g.M <= 0 || g.N <= 0 || g.K <= 0) return FH_OK;
    // In place (C aliasing B, or C aliasing A) is safe when each tile reads
    // the part of the aliased operand it writes and nothing else reads it:
    // one tile along M (C = B) or along N (C = A).  The caller aliases the
    // operand that matches.
    if (g.assign && g.M > kTileM && g.N > kTileN)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "in-place assign GEMM needs M <= 128 or N <= 128");
    int dev = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    static std::mutex init_mu;  // first use on a device may race between host threads
    std::lock_guard<std::mutex> lk(init_mu);
    if (!g_err_flag[dev]) {
        FHB_CUDA(cudaMalloc(&g_err_flag[dev], sizeof(int)));
        FHB_CUDA(cudaMemset(g_err_flag[dev], 0, sizeof(int)));
        FHB_CUDA(cudaFuncSetAttribute(gemm_bf16x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
    }
    dim3 grid((unsigned)((g.N + kTileN - 1) / kTileN), (unsigned)((g.M + kTileM - 1) / kTileM), (unsigned)count);
    gemm_bf16x3_kernel<<<grid, kThreads, kSmemBytes, s>>>(g, g_err_flag[dev]);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

fh_status gemm_tc_update(float *a, int64_t m, int count, int64_t k0, int nb, cudaStream_t s, fh_error_info *err) {
    if (nb % kChunk) return fail(err, FH_ERR_INVALID_ARGUMENT, "tensor-core update needs a panel width multiple of 16");
    const int64_t base = k0 + nb;
    const int64_t rem = m - base;
    if (rem <= 0) return FH_OK;
    float2 *A = reinterpret_cast<float2 *>(a);
    GemmArgs g;
    g.A = A + base + k0 * m;  // L21: rows base.., panel columns
    g.lda = m;
    g.sA = m * m;
    g.B = A + k0 + base * m;  // U12: panel rows, columns base..
    g.ldb = m;
    g.sB = m * m;
    g.C = A + base + base * m;
    g.ldc = m;
    g.sC = m * m;
    g.M = rem;
    g.N = rem;
    g.K = nb;
    g.assign = 0;
    return gemm_tc_launch(g, count, s, err);
}

fh_status gemm_tc_tri_apply(const float *linv, int nb, float *a, int64_t m, int count, int64_t k0, cudaStream_t s,
                            fh_error_info *err) {
    const int64_t c0 = k0 + nb;
    if (c0 >= m) return FH_OK;
    float2 *A = reinterpret_cast<float2 *>(a);
    GemmArgs g;
    g.A = reinterpret_cast<const float2 *>(linv);
    g.lda = nb;
    g.sA = (int64_t)nb * nb;
    g.B = A + k0 + c0 * m;
    g.ldb = m;
    g.sB = m * m;
    g.C = A + k0 + c0 * m;
    g.ldc = m;
    g.sC = m * m;
    g.M = nb;
    g.N = m - c0;
    g.K = nb;
    g.assign = 1;
    return gemm_tc_launch(g, count, s, err);
}

fh_status gemm_tc_strided(const float *A, int64_t lda, int64_t sA, const float *B, int64_t ldb, int64_t sB, float *C,
                          int64_t ldc, int64_t sC, int64_t M, int64_t N, int K, int assign, int count, cudaStream_t s,
                          fh_error_info *err) {
    GemmArgs g;
    g.A = reinterpret_cast<const float2 *>(A);
    g.lda = lda;
    g.sA = sA;
    g.B = reinterpret_cast<const float2 *>(B);
    g.ldb = ldb;
    g.sB = sB;
    g.C = reinterpret_cast<float2 *>(C);
    g.ldc = ldc;
    g.sC = sC;
    g.M = M;
    g.N = N;
    g.K = K;
    g.assign = assign;
    return gemm_tc_launch(g, count, s, err);
}

fh_status gemm_tc_check(fh_error_info *err) {
    int dev = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    if (!g_err_flag[dev]) return FH_OK;
    int flag = 0;
    FHB_CUDA(cudaMemcpy(&flag, g_err_flag[dev], sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset(g_err_flag[dev], 0, sizeof(int));
        return fail(err, FH_ERR_DEVICE_TIMEOUT, "a tensor-core wait ran out of its iteration limit");
    }
    return FH_OK;
}

}  // namespace fhb
