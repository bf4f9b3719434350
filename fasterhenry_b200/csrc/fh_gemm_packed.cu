// Deep trailing update of the FP32 complex LU on the 5th-generation tensor
// cores, from pre-split operands:
//
//     C (M x N) -= A (M x K) B (K x N)        complex, FP32 storage
//
// Every FP32 operand value is split once into two BF16 terms (x = hi + lo)
// by a pack kernel, which also lays the terms out in the tcgen05 canonical
// K-major no-swizzle layout: for each 128-row (A) or 128-column (B) block and
// each 16-wide k chunk, four 4 KB tiles (re hi, re lo, im hi, im lo) of
// 8-row x 16-byte core matrices, 16 KB contiguous.  The update kernel then
// never touches an operand with its own threads:
//
//   warp 0, one lane   producer: cp.async.bulk of the A and B chunk (2 x 16
//                      KB) into a 6-stage shared-memory ring, completion
//                      counted by the stage's mbarrier (expect_tx);
//   warp 1, one lane   MMA issuer: 12 tcgen05.mma (kind::f16, M128 N128 K16)
//                      per chunk -- Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br,
//                      each real product hi*hi + hi*lo + lo*hi, the minus sign
//                      from the A-negate bit -- then tcgen05.commit to the
//                      stage's "empty" barrier;
//   warps 2..9         epilogue: tcgen05.ld of the accumulators, C -= acc with
//                      coalesced loads/stores (lane = row, 256 B per column
//                      per warp); two warps per TMEM lane quarter, one per
//                      column half, 16 loads in flight per thread.
//
// The kernel is persistent (one CTA per SM, a static round-robin over tiles)
// and the accumulators are double-buffered in TMEM (2 x 256 of the 512
// columns), so the epilogue of tile i overlaps the MMAs of tile i+1.  With
// K = 512 a tile is 384 MMAs (about 25k cycles) against 256 KB of C traffic,
// which puts the update on the tensor-core side of the roofline.
//
// No cluster launch and no multicast: every bulk copy is a plain global ->
// own-CTA shared-memory load.  Every mbarrier wait is bounded; a wait that
// runs out sets the error flag, the role stops, the MMA issuer and the
// producer wait (bounded) for their operations in flight, and the TMEM is
// freed before the CTA exits.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "fh_lu.cuh"

namespace fhb {

namespace {

constexpr int kTile = 128;                        // rows / columns of a complex C tile
constexpr int kChunk = 16;                        // complex k per stage
constexpr int kOpTileBytes = kTile * kChunk * 2;  // one bf16 operand tile (128 x 16): 4 KB
constexpr int kOpBytes = 4 * kOpTileBytes;        // re hi, re lo, im hi, im lo: 16 KB
constexpr int kStageBytes = 2 * kOpBytes;         // A and B: 32 KB
constexpr int kStages = 6;
constexpr int kAccCols = 2 * kTile;  // Re (columns 0..127) + Im (128..255)
constexpr int kTmemCols = 2 * kAccCols;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 32 * (2 + kEpiWarps);
constexpr int kBarBytes = 256;
constexpr int kSmemBytes = kStages * kStageBytes + 1024 + kBarBytes;
constexpr int kGroupRows = 16;  // row blocks per raster group (L2 working set)
constexpr long long kSpinLimit = 1LL << 24;

enum { ReH = 0, ReL, ImH, ImL };

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// SM100 shared-memory matrix descriptor, K-major, no swizzle: start>>4 at
// [0,14), LBO>>4 at [16,30), SBO>>4 at [32,46), version 1 at [46,48).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    constexpr uint32_t lbo = (kTile / 8) * 128;  // next 8-wide k group
    constexpr uint32_t sbo = 128;                // next 8-row group
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// kind::f16, BF16 x BF16 -> F32, K-major A and B, M = N = 128, optional A negate.
__host__ __device__ constexpr uint32_t instr_desc(bool negate_a) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((negate_a ? 1u : 0u) << 13) | ((uint32_t)(kTile >> 3) << 17) |
           ((uint32_t)(kTile >> 4) << 24);
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

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait for the completion of the phase with the given parity.
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

// Plain (non-multicast) bulk copy global -> this CTA's shared memory.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack2(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }

__device__ __forceinline__ void split(float x, uint16_t &hi, uint16_t &lo) {
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

// Byte offset of (row r, k group j) inside a 4 KB tile: [j][r/8][r%8][8 bf16].
__device__ __forceinline__ uint32_t tile_off(int r, int j) {
    return (uint32_t)(j * (kTile / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16);
}

// Splits 8 complex values (consecutive k of one row) into the four tiles of
// one operand chunk at `dst`.
__device__ __forceinline__ void split_store8(const float2 *v, uint8_t *dst, uint32_t off) {
    uint16_t rh[8], rl[8], ih[8], il[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        split(v[k].x, rh[k], rl[k]);
        split(v[k].y, ih[k], il[k]);
    }
    *reinterpret_cast<uint4 *>(dst + ReH * kOpTileBytes + off) =
        make_uint4(pack2(rh[0], rh[1]), pack2(rh[2], rh[3]), pack2(rh[4], rh[5]), pack2(rh[6], rh[7]));
    *reinterpret_cast<uint4 *>(dst + ReL * kOpTileBytes + off) =
        make_uint4(pack2(rl[0], rl[1]), pack2(rl[2], rl[3]), pack2(rl[4], rl[5]), pack2(rl[6], rl[7]));
    *reinterpret_cast<uint4 *>(dst + ImH * kOpTileBytes + off) =
        make_uint4(pack2(ih[0], ih[1]), pack2(ih[2], ih[3]), pack2(ih[4], ih[5]), pack2(ih[6], ih[7]));
    *reinterpret_cast<uint4 *>(dst + ImL * kOpTileBytes + off) =
        make_uint4(pack2(il[0], il[1]), pack2(il[2], il[3]), pack2(il[4], il[5]), pack2(il[6], il[7]));
}

// Packs the A operand: element (row r, k) at A[f sA + r + k lda], rows
// [0, M), k in [0, K).  Block (rb * nchunks + c, f), 256 threads: thread t
// takes row rb*128 + t%128 and k group t/128 of chunk c.  Rows >= M are zero.
__global__ void __launch_bounds__(256) pack_a_kernel(const float2 *__restrict__ A, int64_t lda, int64_t sA,
                                                     int64_t M, int nchunks, int rblocks, uint8_t *__restrict__ out) {
    const int rb = blockIdx.x / nchunks, c = blockIdx.x % nchunks, f = blockIdx.y;
    const int r = threadIdx.x & 127, j = threadIdx.x >> 7;
    const int64_t row = (int64_t)rb * kTile + r;
    const float2 *src = A + (int64_t)f * sA + row + (int64_t)(c * kChunk + 8 * j) * lda;
    float2 v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = row < M ? __ldg(src + (int64_t)k * lda) : make_float2(0.f, 0.f);
    uint8_t *dst = out + (((int64_t)f * rblocks + rb) * nchunks + c) * kOpBytes;
    split_store8(v, dst, tile_off(r, j));
}

// Packs the B operand: element (k, column n) at B[f sB + k + n ldb], columns
// [0, N).  Thread t takes column cb*128 + t%128 (8 consecutive k: one 64-byte
// run).  Columns >= N are zero.
__global__ void __launch_bounds__(256) pack_b_kernel(const float2 *__restrict__ B, int64_t ldb, int64_t sB,
                                                     int64_t N, int nchunks, int cblocks, uint8_t *__restrict__ out) {
    const int cb = blockIdx.x / nchunks, c = blockIdx.x % nchunks, f = blockIdx.y;
    const int n = threadIdx.x & 127, j = threadIdx.x >> 7;
    const int64_t col = (int64_t)cb * kTile + n;
    const float2 *src = B + (int64_t)f * sB + (int64_t)(c * kChunk + 8 * j) + col * ldb;
    float2 v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = col < N ? __ldg(src + k) : make_float2(0.f, 0.f);
    uint8_t *dst = out + (((int64_t)f * cblocks + cb) * nchunks + c) * kOpBytes;
    split_store8(v, dst, tile_off(n, j));
}

struct PackedArgs {
    const uint8_t *Ap;  // [f][row block][chunk] 16 KB
    const uint8_t *Bp;  // [f][column block][chunk] 16 KB
    float2 *C;          // (r, n) at C[f sC + r + n ldc]
    int64_t ldc, sC;
    int64_t M, N;
    int rblocks, cblocks, nchunks;
    long long tiles;  // count * tiles per matrix
    // With a tile table: the (row block, column block) of each of a matrix's
    // per_matrix tiles, packed rb | cb << 16, in schedule order.
    const uint32_t *table;
    long long per_matrix;
};

// Tile t -> (matrix, row block, column block).  Within a matrix, groups of
// kGroupRows row blocks; inside a group the row block runs fastest, so the
// CTAs of one wave share a few A blocks and a few B blocks.
__device__ __forceinline__ void tile_coords(const PackedArgs &g, long long t, int &f, int &rb, int &cb) {
    if (g.table) {
        f = (int)(t / g.per_matrix);
        const uint32_t e = g.table[t - (long long)f * g.per_matrix];
        rb = (int)(e & 0xffffu);
        cb = (int)(e >> 16);
        return;
    }
    const long long per = (long long)g.rblocks * g.cblocks;
    f = (int)(t / per);
    const long long r = t - (long long)f * per;
    const long long group_tiles = (long long)kGroupRows * g.cblocks;
    const int grp = (int)(r / group_tiles);
    const int within = (int)(r - (long long)grp * group_tiles);
    const int rows = min(kGroupRows, g.rblocks - grp * kGroupRows);
    cb = within / rows;
    rb = grp * kGroupRows + within % rows;
}

__global__ void __launch_bounds__(kThreads, 1) packed_update_kernel(PackedArgs g, int *__restrict__ err_flag) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kStages * kStageBytes);
    uint64_t *full = bars;                     // [kStages]
    uint64_t *empty = bars + kStages;          // [kStages]
    uint64_t *tfull = bars + 2 * kStages;      // [2]
    uint64_t *tempty = bars + 2 * kStages + 2; // [2]
    uint64_t *drain = bars + 2 * kStages + 4;  // [1]
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 5);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&tfull[b]), 1);
            mbar_init(smem_u32(&tempty[b]), kEpiWarps);
        }
        mbar_init(smem_u32(drain), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- producer ----------------
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued = 0, last_phase = 0;  // per-stage bits: ever issued, phase of the last issue
            for (long long t = blockIdx.x; t < g.tiles && ok; t += gridDim.x) {
                int f, rb, cb;
                tile_coords(g, t, f, rb, cb);
                const uint8_t *a_src = g.Ap + (((int64_t)f * g.rblocks + rb) * g.nchunks) * kOpBytes;
                const uint8_t *b_src = g.Bp + (((int64_t)f * g.cblocks + cb) * g.nchunks) * kOpBytes;
                for (int c = 0; c < g.nchunks; ++c) {
                    if (!mbar_wait(smem_u32(&empty[stage]), phase ^ 1u)) {
                        ok = false;
                        break;
                    }
                    const uint32_t dst = smem_u32(smem + stage * kStageBytes);
                    const uint32_t bar = smem_u32(&full[stage]);
                    mbar_expect_tx(bar, kStageBytes);
                    bulk_load(dst, a_src + (int64_t)c * kOpBytes, kOpBytes, bar);
                    bulk_load(dst + kOpBytes, b_src + (int64_t)c * kOpBytes, kOpBytes, bar);
                    issued |= 1u << stage;
                    last_phase = (last_phase & ~(1u << stage)) | (phase << stage);
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            if (!ok) {
                atomicExch(err_flag, 1);
                // Let the copies already issued land before the CTA exits.
                for (int s = 0; s < kStages; ++s)
                    if (issued >> s & 1u) mbar_wait(smem_u32(&full[s]), last_phase >> s & 1u);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            int stage = 0;
            uint32_t phase = 0;
            uint32_t n_tile = 0;
            bool issued = false;
            const uint32_t pos = instr_desc(false), neg = instr_desc(true);
            for (long long t = blockIdx.x; t < g.tiles && ok; t += gridDim.x, ++n_tile) {
                const uint32_t buf = n_tile & 1u, use = n_tile >> 1;
                if (!mbar_wait(smem_u32(&tempty[buf]), (use & 1u) ^ 1u)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_re = tmem + buf * kAccCols, d_im = d_re + kTile;
                for (int c = 0; c < g.nchunks; ++c) {
                    if (!mbar_wait(smem_u32(&full[stage]), phase)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t s = smem_u32(smem + stage * kStageBytes);
                    auto da = [&](int tile) { return smem_desc(s + tile * kOpTileBytes); };
                    auto db = [&](int tile) { return smem_desc(s + kOpBytes + tile * kOpTileBytes); };
                    const uint32_t acc = c > 0 ? 1u : 0u;
                    // Re += Ar Br - Ai Bi
                    mma_bf16(d_re, da(ReH), db(ReH), pos, acc);
                    mma_bf16(d_re, da(ReH), db(ReL), pos, 1u);
                    mma_bf16(d_re, da(ReL), db(ReH), pos, 1u);
                    mma_bf16(d_re, da(ImH), db(ImH), neg, 1u);
                    mma_bf16(d_re, da(ImH), db(ImL), neg, 1u);
                    mma_bf16(d_re, da(ImL), db(ImH), neg, 1u);
                    // Im += Ar Bi + Ai Br
                    mma_bf16(d_im, da(ReH), db(ImH), pos, acc);
                    mma_bf16(d_im, da(ReH), db(ImL), pos, 1u);
                    mma_bf16(d_im, da(ReL), db(ImH), pos, 1u);
                    mma_bf16(d_im, da(ImH), db(ReH), pos, 1u);
                    mma_bf16(d_im, da(ImH), db(ReL), pos, 1u);
                    mma_bf16(d_im, da(ImL), db(ReH), pos, 1u);
                    issued = true;
                    mma_commit(smem_u32(&empty[stage]));  // the stage is free once these MMAs have read it
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(smem_u32(&tfull[buf]));
            }
            if (!ok) {
                atomicExch(err_flag, 1);
                if (issued) {
                    mma_commit(smem_u32(drain));
                    mbar_wait(smem_u32(drain), 0u);
                }
            }
        }
    } else {
        // ---------------- epilogue ----------------
        const int quarter = warp & 3;        // TMEM lanes 32*quarter.. (hardware: warp id % 4)
        const int half = (warp - 2) >> 2;    // column half of the tile
        const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
        uint32_t n_tile = 0;
        for (long long t = blockIdx.x; t < g.tiles; t += gridDim.x, ++n_tile) {
            const uint32_t buf = n_tile & 1u, use = n_tile >> 1;
            int f, rb, cb;
            tile_coords(g, t, f, rb, cb);
            if (!mbar_wait(smem_u32(&tfull[buf]), use & 1u)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const int64_t row = (int64_t)rb * kTile + quarter * 32 + lane;
            const int64_t col0 = (int64_t)cb * kTile + half * (kTile / 2);
            const bool row_ok = row < g.M;
            float2 *p = g.C + (int64_t)f * g.sC + row + col0 * g.ldc;
            const int ncols = (int)max((int64_t)0, min((int64_t)(kTile / 2), g.N - col0));
            const uint32_t t_re = tmem + buf * kAccCols + lane_off + half * (kTile / 2);
            const uint32_t t_im = t_re + kTile;
#pragma unroll 1
            for (int step = 0; step < kTile / 2 / 16; ++step) {
                uint32_t re[16], im[16];
                float2 cur[16];
                tmem_ld16(t_re + step * 16, re);
                tmem_ld16(t_im + step * 16, im);
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) {
                    const int cc = step * 16 + jj;
                    cur[jj] = (row_ok && cc < ncols) ? __ldcs(p + (int64_t)cc * g.ldc) : make_float2(0.f, 0.f);
                }
                tmem_wait_ld();
                if (step + 1 == kTile / 2 / 16) {
                    // All of this warp's accumulator reads are complete: release the buffer.
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_u32(&tempty[buf]));
                }
                if (row_ok) {
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const int cc = step * 16 + jj;
                        if (cc < ncols)
                            __stcs(p + (int64_t)cc * g.ldc, make_float2(cur[jj].x - __uint_as_float(re[jj]),
                                                                        cur[jj].y - __uint_as_float(im[jj])));
                    }
                }
            }
        }
        if (!ok && lane == 0) atomicExch(err_flag, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

int *g_flag[64] = {nullptr};
int g_sms[64] = {0};

}  // namespace

size_t packed_operand_bytes(int64_t rows, int K, int count) {
    const int64_t blocks = (rows + kTile - 1) / kTile;
    return (size_t)count * (size_t)blocks * (size_t)(K / kChunk) * kOpBytes;
}

fh_status gemm_tc_packed_update(const float *A, int64_t lda, int64_t sA, const float *B, int64_t ldb, int64_t sB,
                                float *C, int64_t ldc, int64_t sC, int64_t M, int64_t N, int K, int count,
                                void *pack_a, void *pack_b, cudaStream_t s, fh_error_info *err, int lower_from) {
    if (K % kChunk || K <= 0) return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update needs K a positive multiple of 16");
    if (M <= 0 || N <= 0 || count <= 0) return FH_OK;
    if (!pack_a || !pack_b) return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update needs operand scratch");
    int dev = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    static std::mutex init_mu;  // first use on a device may race between host threads
    std::unique_lock<std::mutex> lk(init_mu);
    if (!g_flag[dev]) {
        FHB_CUDA(cudaMalloc(&g_flag[dev], sizeof(int)));
        FHB_CUDA(cudaMemset(g_flag[dev], 0, sizeof(int)));
        FHB_CUDA(cudaFuncSetAttribute(packed_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
        FHB_CUDA(cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    }
    lk.unlock();
    const int nchunks = K / kChunk;
    const int rblocks = (int)((M + kTile - 1) / kTile), cblocks = (int)((N + kTile - 1) / kTile);
    uint8_t *pa = reinterpret_cast<uint8_t *>(pack_a), *pb = reinterpret_cast<uint8_t *>(pack_b);
    const bool prof = prof_on();
    if (prof) prof_begin(s, FH_PROF_PACK);
    pack_a_kernel<<<dim3((unsigned)(rblocks * nchunks), (unsigned)count), 256, 0, s>>>(
        reinterpret_cast<const float2 *>(A), lda, sA, M, nchunks, rblocks, pa);
    pack_b_kernel<<<dim3((unsigned)(cblocks * nchunks), (unsigned)count), 256, 0, s>>>(
        reinterpret_cast<const float2 *>(B), ldb, sB, N, nchunks, cblocks, pb);
    if (prof) prof_end(s, FH_PROF_PACK, 16.0 * (double)(M + N) * K * count);
    FHB_CUDA(cudaGetLastError());
    PackedArgs g;
    g.Ap = pa;
    g.Bp = pb;
    g.C = reinterpret_cast<float2 *>(C);
    g.ldc = ldc;
    g.sC = sC;
    g.M = M;
    g.N = N;
    g.rblocks = rblocks;
    g.cblocks = cblocks;
    g.nchunks = nchunks;
    g.table = nullptr;
    g.per_matrix = (long long)rblocks * cblocks;
    double entries = (double)M * (double)N;  // complex C entries updated per matrix
    uint32_t *d_table = nullptr;
    if (lower_from >= 0 && lower_from < cblocks) {
        // Lower-triangle form (symmetric trailing matrix, C rows and columns
        // on the same blocks): column blocks below lower_from in full, the
        // rest only on and below the diagonal block; the same grouped order
        // as the full schedule (row blocks fastest inside groups of
        // kGroupRows), invalid tiles left out.
        std::vector<uint32_t> table;
        table.reserve((size_t)rblocks * cblocks);
        entries = 0.0;
        for (int g0 = 0; g0 < rblocks; g0 += kGroupRows) {
            const int rows = std::min(kGroupRows, rblocks - g0);
            for (int cb = 0; cb < cblocks; ++cb)
                for (int r = 0; r < rows; ++r) {
                    const int rb = g0 + r;
                    if (cb < lower_from || rb >= cb) {
                        table.push_back((uint32_t)rb | ((uint32_t)cb << 16));
                        entries += (double)std::min<int64_t>(kTile, M - (int64_t)rb * kTile) *
                                   (double)std::min<int64_t>(kTile, N - (int64_t)cb * kTile);
                    }
                }
        }
        if (rblocks > 0xffff || cblocks > 0xffff)
            return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update tile table overflow");
        FHB_CUDA(cache_alloc((void **)&d_table, table.size() * 4, s));
        FHB_CUDA(cudaMemcpyAsync(d_table, table.data(), table.size() * 4, cudaMemcpyHostToDevice, s));
        g.table = d_table;
        g.per_matrix = (long long)table.size();
    }
    g.tiles = (long long)count * g.per_matrix;
    const int grid = (int)std::min<long long>(g.tiles, (long long)std::max(1, g_sms[dev]));
    if (prof) prof_begin(s, FH_PROF_GEMM_TC);
    packed_update_kernel<<<grid, kThreads, kSmemBytes, s>>>(g, g_flag[dev]);
    if (prof) prof_end(s, FH_PROF_GEMM_TC, 8.0 * entries * (double)K * count);
    cudaError_t le = cudaGetLastError();
    if (d_table) cache_free(d_table, s);  // stream-ordered: after the kernel
    if (le != cudaSuccess) return fail(err, FH_ERR_CUDA, std::string("packed update launch failed: ") + cudaGetErrorString(le));
    return FH_OK;
}

fh_status gemm_tc_packed_check(fh_error_info *err) {
    int dev = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    if (!g_flag[dev]) return FH_OK;
    int flag = 0;
    FHB_CUDA(cudaMemcpy(&flag, g_flag[dev], sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset(g_flag[dev], 0, sizeof(int));
        return fail(err, FH_ERR_DEVICE_TIMEOUT, "a tensor-core wait of the packed update ran out of its iteration limit");
    }
    return FH_OK;
}

}  // namespace fhb
