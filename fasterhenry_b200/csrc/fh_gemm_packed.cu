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
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
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
constexpr int kRing = 8;  // tile numbers in flight from the producer to the MMA and epilogue warps
constexpr int kBarBytes = 512;
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

__device__ __forceinline__ uint32_t tile_off(int r, int j) {
    return (uint32_t)(j * (kTile / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16);
}

// Splits 8 complex values (k consecutive) into the four 16-byte core-matrix
// rows (re hi, re lo, im hi, im lo) at offset `off` of the four tiles at dst.
__device__ __forceinline__ void split_store8(const float2 *v, uint8_t *dst, uint32_t off) {
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        split2(v[2 * q].x, v[2 * q + 1].x, rh[q], rl[q]);
        split2(v[2 * q].y, v[2 * q + 1].y, ih[q], il[q]);
    }
    *reinterpret_cast<uint4 *>(dst + ReH * kOpTileBytes + off) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
    *reinterpret_cast<uint4 *>(dst + ReL * kOpTileBytes + off) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
    *reinterpret_cast<uint4 *>(dst + ImH * kOpTileBytes + off) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
    *reinterpret_cast<uint4 *>(dst + ImL * kOpTileBytes + off) = make_uint4(il[0], il[1], il[2], il[3]);
}

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
    // With a tile counter the CTAs draw tiles from it (atomicAdd) instead of
    // taking every gridDim.x-th: two grids on different streams then share
    // one update, each CTA running until the counter passes the last tile.
    int *next;
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
    // Drawn tiles (with a tile counter): ring slot n % kRing holds the CTA's
    // n-th tile (-1: none left); idfull[slot] completes when the producer has
    // written it, idempty[slot] when the MMA warp and every epilogue warp
    // have read it.
    uint64_t *idfull = bars + 2 * kStages + 5;           // [kRing]
    uint64_t *idempty = bars + 2 * kStages + 5 + kRing;  // [kRing]
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 5 + 2 * kRing);
    volatile int *ring = reinterpret_cast<volatile int *>(tmem_slot + 2);  // [kRing]

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
        for (int r = 0; r < kRing; ++r) {
            mbar_init(smem_u32(&idfull[r]), 1);
            mbar_init(smem_u32(&idempty[r]), 1 + kEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    // The n-th tile of a consumer (the MMA thread, or a whole epilogue warp
    // through its lane 0): -1 when none is left or a wait for the
    // producer's draw ran out (ok cleared).
    auto consumer_tile = [&](uint32_t n, bool warp_wide) -> long long {
        if (!g.next) {
            const long long t = blockIdx.x + (long long)n * gridDim.x;
            return t < g.tiles ? t : -1;
        }
        long long t = -1;
        int good = 1;
        if (!warp_wide || lane == 0) {
            const uint32_t slot = n % kRing, parity = (n / kRing) & 1u;
            good = mbar_wait(smem_u32(&idfull[slot]), parity) ? 1 : 0;
            if (good) {
                t = ring[slot];
                mbar_arrive(smem_u32(&idempty[slot]));
            }
        }
        if (warp_wide) {
            t = __shfl_sync(0xffffffffu, t, 0);
            good = __shfl_sync(0xffffffffu, good, 0);
        }
        if (!good) ok = false;
        return t;
    };

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- producer ----------------
            int stage = 0;
            uint32_t phase = 0;
            uint32_t issued = 0, last_phase = 0;  // per-stage bits: ever issued, phase of the last issue
            for (uint32_t n = 0; ok; ++n) {
                long long t;
                if (g.next) {
                    const uint32_t slot = n % kRing, parity = (n / kRing) & 1u;
                    if (!mbar_wait(smem_u32(&idempty[slot]), parity ^ 1u)) {
                        ok = false;
                        break;
                    }
                    const int d = atomicAdd(g.next, 1);
                    t = d < g.tiles ? d : -1;
                    ring[slot] = (int)t;
                    mbar_arrive(smem_u32(&idfull[slot]));
                } else {
                    t = blockIdx.x + (long long)n * gridDim.x;
                    if (t >= g.tiles) t = -1;
                }
                if (t < 0) break;
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
            for (;; ++n_tile) {
                if (consumer_tile(n_tile, false) < 0) break;
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
        for (uint32_t n_tile = 0;; ++n_tile) {
            const long long t = consumer_tile(n_tile, true);
            if (t < 0) break;
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

// ---------------------------------------------------------------------------
// The rows below a super-panel of the factorization without pivoting.
//
// For a factored super-panel [K0, E) (W = E - K0 columns, D = L_D U_D) and
// the rows [E, m) below it, in place:
//
//     L21 = A21 X,    X = U_D^{-1}  (W x W upper triangular, packed as a B operand)
//
// and with L21 everything else the super-panel step needs from it: the matrix
// is complex symmetric and factored without interchanges, so U = diag(U) L^T
// and U12 = diag(d) L21^T (d_k = U_kk) is written over the rows [K0, E) of the
// trailing columns (unless no solve reads it); and the one operand of the deep update is written
// packed: P = L21 diag(s) by 128-row blocks, s_k a square root of d_k, so
// that L21 U12 = P P^T and the update takes P's tiles for both A (row
// blocks) and B (column blocks).
//
// A work item is one 128-row block of one matrix; its output column blocks
// are formed from the last to the first, block j from the k chunks
// [0, 8 (j + 1)) (X is upper triangular), so the FP32 write of a block never
// reaches a column that a later block of the item reads, and items own
// disjoint rows.  Roles:
//   warp 13, one lane  loader: per chunk, one 2D tensor copy (no multicast)
//                      of the raw FP32 rows into a ring of raw slots -- box
//                      128 rows x 16 columns of the batch seen as an m x
//                      (count m) array of 8-byte elements, rows past m
//                      filled with zeros (a tensor map needs a column stride
//                      that is a multiple of 16 bytes: m even);
//   warps 0..3         splitters: thread t reads row t of the chunk from the
//                      raw slot into registers and releases the slot; once
//                      the MMAs are done with the A/X stage, thread 0 starts
//                      the plain bulk copy of the X chunk into it and every
//                      thread stores its row as BF16 hi/lo into the four A
//                      tiles, then a proxy fence and an arrival on `afull`.
//                      The raw ring and the A/X ring are separate, so a raw
//                      slot is reused after the split, not after the MMAs;
//   warp 12, one lane  TMEM allocation and the MMA issuer: 12 tcgen05.mma per
//                      chunk into one of two TMEM accumulators;
//   warps 4..11        epilogue: tcgen05.ld, then L21 and U12 in FP32 and the
//                      packed tile of P.
// An A/X stage is reused once the MMAs that read it have completed
// (`empty`), a raw slot once the splitters have read it.  No cluster launch
// and no multicast.  Every wait is bounded; a wait that runs out sets the
// error flag and stops the role, and the loader, the splitters' copy thread
// and the MMA issuer wait (bounded) for their operations in flight before
// the TMEM is freed.
constexpr int kPsRawBytes = kChunk * kTile * 8;                   // 16 columns x 128 rows of complex FP32
constexpr int kPsStageBytes = 2 * kOpBytes;                        // packed A, X: 32 KB
constexpr int kPsStages = 4;                                       // A/X ring
constexpr int kPsRawSlots = 4;                                     // raw ring
constexpr int kPsThreads = 32 * 14;
// A staging tile per epilogue warp for U12 (32 rows x 16 complex, XOR-swizzled).
constexpr int kPsU12Bytes = kEpiWarps * 32 * 16 * 8;
constexpr int kPsSmemBytes =
    kPsStages * kPsStageBytes + kPsRawSlots * kPsRawBytes + kPsU12Bytes + 1024 + kBarBytes;
static_assert(kPsSmemBytes <= 227 * 1024, "panel-solve shared memory");

struct PanelSolveArgs {
    float2 *A;             // the batch: (r, c) of matrix f at A[f mm + r + c m]
    int64_t m, mm, K0, E;
    int W, nbw, nch;       // super-panel width, its 128-blocks and 16-chunks
    const uint8_t *Xp;     // X packed: [f][column block][chunk] 16 KB
    const float2 *dvec;    // d_k = U_kk of the super-panel: [f][W]
    const float2 *svec;    // s_k, s_k^2 = d_k: [f][W]
    int write_u12;         // 0: U12 is not written (no solve reads it)
    uint8_t *P;            // packed output L21 diag(s): [f][row block][chunk] 16 KB
    int rblocks;           // 128-row blocks of [E, m)
    long long items;       // count * rblocks
};

__device__ __forceinline__ void tensor_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__global__ void __launch_bounds__(kPsThreads, 1)
    panel_solve_kernel(PanelSolveArgs g, const __grid_constant__ CUtensorMap rows_map, int *__restrict__ err_flag) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint8_t *raw_base = smem + kPsStages * kPsStageBytes;
    float2 *u12_stage = reinterpret_cast<float2 *>(raw_base + kPsRawSlots * kPsRawBytes);
    uint64_t *bars = reinterpret_cast<uint64_t *>(raw_base + kPsRawSlots * kPsRawBytes + kPsU12Bytes);
    uint64_t *rfull = bars;                           // [kPsRawSlots] loader: raw rows landed
    uint64_t *rempty = rfull + kPsRawSlots;           // [kPsRawSlots] splitters: raw rows read
    uint64_t *xfull = rempty + kPsRawSlots;           // [kPsStages] X chunk landed
    uint64_t *afull = xfull + kPsStages;              // [kPsStages] splitters: A tiles written
    uint64_t *empty = afull + kPsStages;              // [kPsStages] MMA commit
    uint64_t *tfull = empty + kPsStages;              // [2]
    uint64_t *tempty = tfull + 2;                     // [2]
    uint64_t *drain = tempty + 2;                     // [1]
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    // A/X stage: packed A (4 tiles) | X chunk (4 tiles); raw slots apart, so a
    // raw slot is free again as soon as the splitters have read it
    auto stage_a = [&](int st) { return smem + st * kPsStageBytes; };
    auto stage_b = [&](int st) { return smem + st * kPsStageBytes + kOpBytes; };
    auto stage_raw = [&](int rs) { return raw_base + rs * kPsRawBytes; };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 12) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int rs = 0; rs < kPsRawSlots; ++rs) {
            mbar_init(smem_u32(&rfull[rs]), 1);
            mbar_init(smem_u32(&rempty[rs]), 128);
        }
        for (int st = 0; st < kPsStages; ++st) {
            mbar_init(smem_u32(&xfull[st]), 1);
            mbar_init(smem_u32(&afull[st]), 128);
            mbar_init(smem_u32(&empty[st]), 1);
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

    if (warp == 13) {
        if (lane == 0) {
            // raw rows only: one 2D tensor copy per chunk into the raw ring
            int rs = 0;
            uint32_t phase = 0, issued = 0, last_phase = 0;
            for (long long t = blockIdx.x; t < g.items && ok; t += gridDim.x) {
                const int f = (int)(t / g.rblocks), rb = (int)(t % g.rblocks);
                const int x = (int)(g.E + (int64_t)rb * kTile);  // first row (even: a 16-byte boundary)
                const int y0 = (int)((int64_t)f * g.m + g.K0);  // column K0 of matrix f
                for (int j = g.nbw - 1; j >= 0 && ok; --j)
                    for (int c = 0; c < 8 * (j + 1); ++c) {
                        if (!mbar_wait(smem_u32(&rempty[rs]), phase ^ 1u)) {
                            ok = false;
                            break;
                        }
                        const uint32_t bar = smem_u32(&rfull[rs]);
                        mbar_expect_tx(bar, kPsRawBytes);
                        tensor_load_2d(smem_u32(stage_raw(rs)), &rows_map, x, y0 + c * kChunk, bar);
                        issued |= 1u << rs;
                        last_phase = (last_phase & ~(1u << rs)) | (phase << rs);
                        if (++rs == kPsRawSlots) {
                            rs = 0;
                            phase ^= 1u;
                        }
                    }
            }
            if (!ok) {
                atomicExch(err_flag, 1);
                for (int r = 0; r < kPsRawSlots; ++r)
                    if (issued >> r & 1u) mbar_wait(smem_u32(&rfull[r]), last_phase >> r & 1u);
            }
        }
    } else if (warp < 4) {
        // splitters: raw rows -> registers (the raw slot is released at once),
        // then, once the MMAs are done with the A/X stage, the X chunk's bulk
        // copy (thread 0) and the BF16 hi/lo A tiles
        const int tr = threadIdx.x;  // row of the block
        int rs = 0, stage = 0;
        uint32_t rphase = 0, phase = 0, xissued = 0, xlast = 0;
        for (long long t = blockIdx.x; t < g.items && ok; t += gridDim.x) {
            const int f = (int)(t / g.rblocks);
            for (int j = g.nbw - 1; j >= 0 && ok; --j)
                for (int c = 0; c < 8 * (j + 1); ++c) {
                    if (!mbar_wait(smem_u32(&rfull[rs]), rphase)) {
                        ok = false;
                        break;
                    }
                    // raw tile: column kk of the chunk at kk * 128, rows contiguous (zeros past m)
                    const float2 *raw = reinterpret_cast<const float2 *>(stage_raw(rs));
                    float2 v[kChunk];
#pragma unroll
                    for (int kk = 0; kk < kChunk; ++kk) v[kk] = raw[kk * kTile + tr];
                    mbar_arrive(smem_u32(&rempty[rs]));
                    if (++rs == kPsRawSlots) {
                        rs = 0;
                        rphase ^= 1u;
                    }
                    if (!mbar_wait(smem_u32(&empty[stage]), phase ^ 1u)) {
                        ok = false;
                        break;
                    }
                    if (tr == 0) {
                        const uint32_t bar = smem_u32(&xfull[stage]);
                        mbar_expect_tx(bar, kOpBytes);
                        bulk_load(smem_u32(stage_b(stage)), g.Xp + (((int64_t)f * g.nbw + j) * g.nch + c) * kOpBytes,
                                  kOpBytes, bar);
                        xissued |= 1u << stage;
                        xlast = (xlast & ~(1u << stage)) | (phase << stage);
                    }
                    uint8_t *dst = stage_a(stage);
                    split_store8(v, dst, tile_off(tr, 0));
                    split_store8(v + 8, dst, tile_off(tr, 1));
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    mbar_arrive(smem_u32(&afull[stage]));
                    if (++stage == kPsStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
        }
        if (!ok) {
            atomicExch(err_flag, 1);
            if (tr == 0)
                for (int st = 0; st < kPsStages; ++st)
                    if (xissued >> st & 1u) mbar_wait(smem_u32(&xfull[st]), xlast >> st & 1u);
        }
    } else if (warp == 12) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0, n_tile = 0;
            bool issued = false;
            const uint32_t pos = instr_desc(false), neg = instr_desc(true);
            for (long long t = blockIdx.x; t < g.items && ok; t += gridDim.x)
                for (int j = g.nbw - 1; j >= 0 && ok; --j, ++n_tile) {
                    const uint32_t buf = n_tile & 1u, use = n_tile >> 1;
                    if (!mbar_wait(smem_u32(&tempty[buf]), (use & 1u) ^ 1u)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d_re = tmem + buf * kAccCols, d_im = d_re + kTile;
                    for (int c = 0; c < 8 * (j + 1); ++c) {
                        if (!mbar_wait(smem_u32(&xfull[stage]), phase) || !mbar_wait(smem_u32(&afull[stage]), phase)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t sa = smem_u32(stage_a(stage)), sb = smem_u32(stage_b(stage));
                        auto da = [&](int tile) { return smem_desc(sa + tile * kOpTileBytes); };
                        auto db = [&](int tile) { return smem_desc(sb + tile * kOpTileBytes); };
                        const uint32_t acc = c > 0 ? 1u : 0u;
                        mma_bf16(d_re, da(ReH), db(ReH), pos, acc);
                        mma_bf16(d_re, da(ReH), db(ReL), pos, 1u);
                        mma_bf16(d_re, da(ReL), db(ReH), pos, 1u);
                        mma_bf16(d_re, da(ImH), db(ImH), neg, 1u);
                        mma_bf16(d_re, da(ImH), db(ImL), neg, 1u);
                        mma_bf16(d_re, da(ImL), db(ImH), neg, 1u);
                        mma_bf16(d_im, da(ReH), db(ImH), pos, acc);
                        mma_bf16(d_im, da(ReH), db(ImL), pos, 1u);
                        mma_bf16(d_im, da(ReL), db(ImH), pos, 1u);
                        mma_bf16(d_im, da(ImH), db(ReH), pos, 1u);
                        mma_bf16(d_im, da(ImH), db(ReL), pos, 1u);
                        mma_bf16(d_im, da(ImL), db(ReH), pos, 1u);
                        issued = true;
                        mma_commit(smem_u32(&empty[stage]));
                        if (++stage == kPsStages) {
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
        const int quarter = warp & 3;       // TMEM lanes 32*quarter.. (hardware: warp id % 4)
        const int half = (warp - 4) >> 2;   // column half of the output block
        const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
        const int tr = quarter * 32 + lane;  // row of the block
        uint32_t n_tile = 0;
        for (long long t = blockIdx.x; t < g.items && ok; t += gridDim.x) {
            const int f = (int)(t / g.rblocks), rb = (int)(t % g.rblocks);
            const int64_t row = g.E + (int64_t)rb * kTile + tr;
            const bool valid = row < g.m;
            float2 *Af = g.A + (int64_t)f * g.mm;
            for (int j = g.nbw - 1; j >= 0; --j, ++n_tile) {
                const uint32_t buf = n_tile & 1u, use = n_tile >> 1;
                if (!mbar_wait(smem_u32(&tfull[buf]), use & 1u)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t t_re = tmem + buf * kAccCols + lane_off + half * (kTile / 2);
                const uint32_t t_im = t_re + kTile;
#pragma unroll 1
                for (int step = 0; step < kTile / 2 / 16; ++step) {
                    const int kc = j * kTile + half * (kTile / 2) + step * 16;  // column in the super-panel
                    uint32_t re[16], im[16];
                    tmem_ld16(t_re + step * 16, re);
                    tmem_ld16(t_im + step * 16, im);
                    float2 d[16];
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) d[jj] = __ldg(g.dvec + (int64_t)f * g.W + kc + jj);
                    tmem_wait_ld();
                    if (step + 1 == kTile / 2 / 16) {
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(smem_u32(&tempty[buf]));
                    }
                    float2 l[16], u[16];
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        l[jj] = make_float2(__uint_as_float(re[jj]), __uint_as_float(im[jj]));
                        u[jj] = make_float2(d[jj].x * l[jj].x - d[jj].y * l[jj].y, d[jj].x * l[jj].y + d[jj].y * l[jj].x);
                    }
                    if (valid) {
                        float2 *pl = Af + row + (g.K0 + kc) * g.m;  // L21: down the columns, coalesced over lanes
#pragma unroll
                        for (int jj = 0; jj < 16; ++jj) pl[(int64_t)jj * g.m] = l[jj];
                    }
                    if (g.write_u12) {
                        // U12: the thread's 16 entries lie down column `row`; the
                        // warp's tile goes through shared memory (column jj of row
                        // r at r * 16 + (jj ^ (r % 16))) so that each store covers
                        // 16 consecutive entries of two columns.
                        float2 *stg = u12_stage + (warp - 4) * 512;
#pragma unroll
                        for (int jj = 0; jj < 16; ++jj) stg[lane * 16 + (jj ^ (lane & 15))] = u[jj];
                        __syncwarp();
                        const int64_t row_base = g.E + (int64_t)rb * kTile + quarter * 32;
#pragma unroll
                        for (int q = 0; q < 16; ++q) {
                            const int rr = 2 * q + (lane >> 4), kk = lane & 15;
                            const int64_t r_abs = row_base + rr;
                            const float2 v = stg[rr * 16 + (kk ^ (rr & 15))];
                            if (r_abs < g.m) Af[(g.K0 + kc + kk) + r_abs * g.m] = v;
                        }
                        __syncwarp();
                    }
                    // P = L21 diag(s): one operand for both sides of C -= P P^T
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const float2 sq = __ldg(g.svec + (int64_t)f * g.W + kc + jj);
                        u[jj] = make_float2(sq.x * l[jj].x - sq.y * l[jj].y, sq.x * l[jj].y + sq.y * l[jj].x);
                    }
                    const int64_t tile = ((int64_t)f * g.rblocks + rb) * g.nch + kc / kChunk;
                    split_store8(u, g.P + tile * kOpBytes, tile_off(tr, 0));
                    split_store8(u + 8, g.P + tile * kOpBytes, tile_off(tr, 1));
                }
            }
        }
        if (!ok && lane == 0) atomicExch(err_flag, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 12) {
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

namespace {
// First use on a device: the error flag, the kernels' shared-memory limits,
// the SM count.
fh_status packed_init(int *dev_out, fh_error_info *err) {
    int dev = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    static std::mutex init_mu;  // first use on a device may race between host threads
    std::lock_guard<std::mutex> lk(init_mu);
    if (!g_flag[dev]) {
        FHB_CUDA(cudaMalloc(&g_flag[dev], sizeof(int)));
        FHB_CUDA(cudaMemset(g_flag[dev], 0, sizeof(int)));
        FHB_CUDA(cudaFuncSetAttribute(packed_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
        FHB_CUDA(cudaFuncSetAttribute(panel_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPsSmemBytes));
        FHB_CUDA(cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    }
    *dev_out = dev;
    return FH_OK;
}
}  // namespace

fh_status gemm_tc_packed_schedule(PackedSchedule &ps, const void *pack_a, const void *pack_b, float *C, int64_t ldc,
                                  int64_t sC, int64_t M, int64_t N, int K, int count, int lower_from, int col_lo,
                                  int col_hi, cudaStream_t s, fh_error_info *err) {
    ps = PackedSchedule{};
    if (K % kChunk || K <= 0) return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update needs K a positive multiple of 16");
    if (M <= 0 || N <= 0 || count <= 0) return FH_OK;
    if (!pack_a || !pack_b) return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update needs packed operands");
    int dev = 0;
    fh_status st = packed_init(&dev, err);
    if (st) return st;
    const int rblocks = (int)((M + kTile - 1) / kTile), cblocks = (int)((N + kTile - 1) / kTile);
    if (col_hi < 0 || col_hi > cblocks) col_hi = cblocks;
    col_lo = std::max(0, col_lo);
    if (col_lo >= col_hi) return FH_OK;
    ps.pack_a = pack_a;
    ps.pack_b = pack_b;
    ps.C = C;
    ps.ldc = ldc;
    ps.sC = sC;
    ps.M = M;
    ps.N = N;
    ps.K = K;
    ps.count = count;
    ps.per_matrix = (long long)rblocks * cblocks;
    ps.entries = (double)M * (double)N;  // complex C entries updated per matrix
    const bool ranged = col_lo > 0 || col_hi < cblocks;
    if ((lower_from >= 0 && lower_from < cblocks) || ranged) {
        if (lower_from < 0 || lower_from > cblocks) lower_from = cblocks;  // a range of full column blocks
        // Lower-triangle form (symmetric trailing matrix, C rows and columns
        // on the same blocks): column blocks below lower_from in full, the
        // rest only on and below the diagonal block (lower_from = 0: the
        // lower triangle of tiles), over the column blocks [col_lo, col_hi);
        // the same grouped order as the full schedule (row blocks fastest
        // inside groups of kGroupRows), the other tiles left out.
        if (rblocks > 0xffff || cblocks > 0xffff)
            return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update tile table overflow");
        std::vector<uint32_t> table;
        table.reserve((size_t)rblocks * (col_hi - col_lo));
        ps.entries = 0.0;
        for (int g0 = 0; g0 < rblocks; g0 += kGroupRows) {
            const int rows = std::min(kGroupRows, rblocks - g0);
            for (int cb = col_lo; cb < col_hi; ++cb)
                for (int r = 0; r < rows; ++r) {
                    const int rb = g0 + r;
                    if (cb < lower_from || rb >= cb) {
                        table.push_back((uint32_t)rb | ((uint32_t)cb << 16));
                        ps.entries += (double)std::min<int64_t>(kTile, M - (int64_t)rb * kTile) *
                                      (double)std::min<int64_t>(kTile, N - (int64_t)cb * kTile);
                    }
                }
        }
        ps.per_matrix = (long long)table.size();
        if (table.empty()) return FH_OK;
        FHB_CUDA(cache_alloc((void **)&ps.table, table.size() * 4, s));
        FHB_CUDA(cudaMemcpyAsync(ps.table, table.data(), table.size() * 4, cudaMemcpyHostToDevice, s));
    }
    ps.tiles = (long long)count * ps.per_matrix;
    return FH_OK;
}

fh_status gemm_tc_packed_launch(const PackedSchedule &ps, int grid, int *next, cudaStream_t s, fh_error_info *err,
                                int prof_class) {
    if (ps.tiles <= 0) return FH_OK;
    if (next && ps.tiles > INT32_MAX) return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update tile counter overflow");
    int dev = 0;
    fh_status st = packed_init(&dev, err);
    if (st) return st;
    const int rblocks = (int)((ps.M + kTile - 1) / kTile), cblocks = (int)((ps.N + kTile - 1) / kTile);
    PackedArgs g;
    g.Ap = reinterpret_cast<const uint8_t *>(ps.pack_a);
    g.Bp = reinterpret_cast<const uint8_t *>(ps.pack_b);
    g.C = reinterpret_cast<float2 *>(ps.C);
    g.ldc = ps.ldc;
    g.sC = ps.sC;
    g.M = ps.M;
    g.N = ps.N;
    g.rblocks = rblocks;
    g.cblocks = cblocks;
    g.nchunks = ps.K / kChunk;
    g.tiles = ps.tiles;
    g.table = ps.table;
    g.per_matrix = ps.per_matrix;
    g.next = next;
    if (grid <= 0) grid = std::max(1, g_sms[dev]);
    grid = (int)std::min<long long>(ps.tiles, grid);
    const bool prof = prof_class >= 0 && prof_on();
    if (prof) prof_begin(s, prof_class);
    packed_update_kernel<<<grid, kThreads, kSmemBytes, s>>>(g, g_flag[dev]);
    if (prof) prof_end(s, prof_class, 8.0 * ps.entries * (double)ps.K * ps.count);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return fail(err, FH_ERR_CUDA, std::string("packed update launch failed: ") + cudaGetErrorString(le));
    return FH_OK;
}

void gemm_tc_packed_release(PackedSchedule &ps, cudaStream_t s) {
    if (ps.table) cache_free(ps.table, s);  // stream-ordered: after the launches before it on s
    ps.table = nullptr;
    ps.tiles = 0;
}

int gemm_tc_sm_count() {
    int dev = 0;
    if (packed_init(&dev, nullptr)) return 1;
    return std::max(1, g_sms[dev]);
}

fh_status gemm_tc_packed_run(const void *pack_a, const void *pack_b, float *C, int64_t ldc, int64_t sC, int64_t M,
                             int64_t N, int K, int count, cudaStream_t s, fh_error_info *err, int lower_from, int col_lo,
                             int col_hi) {
    PackedSchedule ps;
    fh_status st = gemm_tc_packed_schedule(ps, pack_a, pack_b, C, ldc, sC, M, N, K, count, lower_from, col_lo, col_hi, s,
                                           err);
    if (!st) st = gemm_tc_packed_launch(ps, 0, nullptr, s, err);
    gemm_tc_packed_release(ps, s);
    return st;
}

fh_status gemm_tc_packed_update(const float *A, int64_t lda, int64_t sA, const float *B, int64_t ldb, int64_t sB,
                                float *C, int64_t ldc, int64_t sC, int64_t M, int64_t N, int K, int count,
                                void *pack_a, void *pack_b, cudaStream_t s, fh_error_info *err, int lower_from) {
    if (K % kChunk || K <= 0) return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update needs K a positive multiple of 16");
    if (M <= 0 || N <= 0 || count <= 0) return FH_OK;
    if (!pack_a || !pack_b) return fail(err, FH_ERR_INVALID_ARGUMENT, "packed update needs operand scratch");
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
    return gemm_tc_packed_run(pa, pb, C, ldc, sC, M, N, K, count, s, err, lower_from);
}

fh_status gemm_tc_pack_b(const float *B, int64_t ldb, int64_t sB, int64_t N, int K, int count, void *out,
                         cudaStream_t s, fh_error_info *err) {
    if (K % kChunk || K <= 0) return fail(err, FH_ERR_INVALID_ARGUMENT, "packing needs K a positive multiple of 16");
    if (N <= 0 || count <= 0) return FH_OK;
    const int nchunks = K / kChunk, cblocks = (int)((N + kTile - 1) / kTile);
    pack_b_kernel<<<dim3((unsigned)(cblocks * nchunks), (unsigned)count), 256, 0, s>>>(
        reinterpret_cast<const float2 *>(B), ldb, sB, N, nchunks, cblocks, reinterpret_cast<uint8_t *>(out));
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

namespace {
// The driver's tensor-map encoder, looked up once through the runtime.
PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    }();
    return fn;
}
}  // namespace

fh_status encode_column_tiles(void *map, const float *a, int64_t m, int count, int box_rows, int box_cols,
                              fh_error_info *err) {
    // The batch as an m x (count m) array of 8-byte elements (complex FP32),
    // column stride 8 m bytes; rows past m read as zeros.
    PFN_cuTensorMapEncodeTiled encode = tensor_map_encoder();
    if (!encode) return fail(err, FH_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)count * (cuuint64_t)m};
    const cuuint64_t strides[1] = {(cuuint64_t)m * 8};
    const cuuint32_t box[2] = {(cuuint32_t)box_rows, (cuuint32_t)box_cols};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult cr = encode(static_cast<CUtensorMap *>(map), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                               const_cast<float *>(a), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS)
        return fail(err, FH_ERR_CUDA, "tensor map of the batch rejected (driver error " + std::to_string((int)cr) + ")");
    return FH_OK;
}

bool panel_solve_supported(int64_t m) { return m % 2 == 0 && m * 8 < ((int64_t)1 << 40); }

fh_status gemm_tc_panel_solve(float *a, int64_t m, int count, int64_t K0, int W, const void *xpack, const float *dvec,
                              const float *svec, void *pack, bool write_u12, cudaStream_t s, fh_error_info *err) {
    const int64_t E = K0 + W;
    if (W <= 0 || W % kTile || W > 4 * kTile || K0 < 0 || K0 % 2 || E > m)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "panel solve needs a super-panel of 128-column blocks (at most 4)");
    if (!panel_solve_supported(m) || (int64_t)count * m > INT32_MAX)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "panel solve needs an even order (16-byte column stride)");
    if (E == m || count <= 0) return FH_OK;
    if (!xpack || !dvec || !svec || !pack)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "panel solve needs the packed inverse, the diagonal and outputs");
    int dev = 0;
    fh_status st = packed_init(&dev, err);
    if (st) return st;
    CUtensorMap rows_map;
    st = encode_column_tiles(&rows_map, a, m, count, kTile, kChunk, err);
    if (st) return st;
    PanelSolveArgs g;
    g.A = reinterpret_cast<float2 *>(a);
    g.m = m;
    g.mm = m * m;
    g.K0 = K0;
    g.E = E;
    g.W = W;
    g.nbw = W / kTile;
    g.nch = W / kChunk;
    g.Xp = reinterpret_cast<const uint8_t *>(xpack);
    g.dvec = reinterpret_cast<const float2 *>(dvec);
    g.svec = reinterpret_cast<const float2 *>(svec);
    g.write_u12 = write_u12 ? 1 : 0;
    g.P = reinterpret_cast<uint8_t *>(pack);
    g.rblocks = (int)((m - E + kTile - 1) / kTile);
    g.items = (long long)count * g.rblocks;
    const int grid = (int)std::min<long long>(g.items, (long long)std::max(1, g_sms[dev]));
    const bool prof = prof_on();
    // complex MACs of the triangular product (block j of each 128 rows takes K = 128 (j + 1))
    const double macs = (double)(m - E) * kTile * kTile * (g.nbw * (g.nbw + 1) / 2) * count;
    if (prof) prof_begin(s, FH_PROF_PANEL_SOLVE);
    panel_solve_kernel<<<grid, kPsThreads, kPsSmemBytes, s>>>(g, rows_map, g_flag[dev]);
    if (prof) prof_end(s, FH_PROF_PANEL_SOLVE, 24.0 * macs);  // BF16 tensor flops (3 products x 8)
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return fail(err, FH_ERR_CUDA, std::string("panel solve launch failed: ") + cudaGetErrorString(le));
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
