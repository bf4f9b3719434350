// Near-pair search of the precorrected-FFT set-up on the device
// (replaces the reference's near_pairs, pfft/near.rs:41-106).
//
// The reference bins every filament into the uniform bins its bounding box
// overlaps, then for each filament i collects the filaments j >= i found in
// the bins that its box grown by the radius overlaps, and keeps j when the
// separating-axis gap of the two bars is below the radius.  The bins are a
// search structure only; which pairs are found depends on their geometry
// (lower corner, size, counts), so it is computed here exactly as the
// reference computes it.  The device form:
//
//   near_boxes_kernel   bounding box of every bar (the reference's reach sum)
//   cub reductions      the boxes' lower and upper corners -> host: bin size
//                       and counts by the reference's coarsening loop
//   bin_count_kernel,   (bin, filament) entries of every box, radix-sorted by
//   bin_emit_kernel     bin; per-bin starts from a histogram and a scan
//   near_rows_kernel    a warp per filament i walks its query bins, lanes over
//                       the bins' entries; a candidate j is taken only in the
//                       first bin (lowest x, y, z) common to i's query range
//                       and j's own range, so each pair is seen once without a
//                       per-row set; then the separating-axis gap (fh_geom.cuh,
//                       the reference's operation order) and the direction
//                       cosine (orthogonal pairs, |cos| < 1e-14, have neither
//                       an exact value nor a grid approximation and are not
//                       listed).  Run twice: counts, then the pairs.
//   one radix sort      of (i, j) keys: rows ascending in j.
#include <cub/cub.cuh>

#include <cmath>
#include <limits>
#include <vector>

#include "fh_geom.cuh"
#include "fh_pfft.h"

namespace fhb {
namespace {

constexpr double kOrthogonalCos = 1e-14;  // near.rs:25
constexpr int kNearWarps = 8;             // warps (rows) per CTA of near_rows_kernel

struct Bins {
    double lo[3];
    double size;
    int64_t dims[3];
};

__global__ void near_boxes_kernel(const DevFil *__restrict__ fil, int64_t n, double *__restrict__ lo,
                                  double *__restrict__ hi) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const DevFil &f = fil[i];
        double reach[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < 3; ++k)
            for (int a = 0; a < 3; ++a) reach[a] = __dadd_rn(reach[a], __dmul_rn(fabs(f.axes[3 * k + a]), f.half[k]));
        for (int a = 0; a < 3; ++a) {
            lo[a * n + i] = __dsub_rn(f.centre[a], reach[a]);
            hi[a * n + i] = __dadd_rn(f.centre[a], reach[a]);
        }
    }
}

__device__ __forceinline__ int64_t bin_cell(const Bins &b, double x, int a) {
    const double c = floor(__ddiv_rn(__dsub_rn(x, b.lo[a]), b.size));
    const int64_t v = c > 0.0 ? (int64_t)c : 0;
    return v < b.dims[a] - 1 ? v : b.dims[a] - 1;
}

__device__ __forceinline__ int64_t bin_index(const Bins &b, int64_t x, int64_t y, int64_t z) {
    return (x * b.dims[1] + y) * b.dims[2] + z;
}

// Bins overlapped by filament i's box (and the per-bin histogram).
__global__ void bin_count_kernel(const double *__restrict__ lo, const double *__restrict__ hi, int64_t n, Bins b,
                                 int64_t *__restrict__ count, unsigned *__restrict__ per_bin) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t f[3], l[3];
        for (int a = 0; a < 3; ++a) {
            f[a] = bin_cell(b, lo[a * n + i], a);
            l[a] = bin_cell(b, hi[a * n + i], a);
        }
        count[i] = (l[0] - f[0] + 1) * (l[1] - f[1] + 1) * (l[2] - f[2] + 1);
        for (int64_t x = f[0]; x <= l[0]; ++x)
            for (int64_t y = f[1]; y <= l[1]; ++y)
                for (int64_t z = f[2]; z <= l[2]; ++z) atomicAdd(per_bin + bin_index(b, x, y, z), 1u);
    }
}

__global__ void bin_emit_kernel(const double *__restrict__ lo, const double *__restrict__ hi, int64_t n, Bins b,
                                const int64_t *__restrict__ offset, uint32_t *__restrict__ key,
                                uint32_t *__restrict__ val) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t f[3], l[3];
        for (int a = 0; a < 3; ++a) {
            f[a] = bin_cell(b, lo[a * n + i], a);
            l[a] = bin_cell(b, hi[a * n + i], a);
        }
        int64_t o = offset[i];
        for (int64_t x = f[0]; x <= l[0]; ++x)
            for (int64_t y = f[1]; y <= l[1]; ++y)
                for (int64_t z = f[2]; z <= l[2]; ++z) {
                    key[o] = (uint32_t)bin_index(b, x, y, z);
                    val[o] = (uint32_t)i;
                    ++o;
                }
    }
}

// A warp per filament i.  Pass 0 writes the row's pair count to row_count[i];
// pass 1 writes the row's pairs (as (i << 32 | j) keys and their direction
// cosines) from out_off[i] on.
template <int kPass>
__global__ void __launch_bounds__(32 * kNearWarps)
    near_rows_kernel(const DevFil *__restrict__ fil, const double *__restrict__ lo, const double *__restrict__ hi,
                     int64_t n, Bins b, double radius, const int64_t *__restrict__ bin_start,
                     const uint32_t *__restrict__ bin_fil, int64_t *__restrict__ row_count,
                     const int64_t *__restrict__ out_off, unsigned long long *__restrict__ out_key,
                     double *__restrict__ out_cos) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * kNearWarps;
    for (int64_t i = (int64_t)blockIdx.x * kNearWarps + (threadIdx.x >> 5); i < n; i += warps) {
        const DevFil &fi = fil[i];
        int64_t fq[3], lq[3];
        for (int a = 0; a < 3; ++a) {
            fq[a] = bin_cell(b, __dsub_rn(lo[a * n + i], radius), a);
            lq[a] = bin_cell(b, __dadd_rn(hi[a * n + i], radius), a);
        }
        int64_t count = 0;
        int64_t base = kPass ? out_off[i] : 0;
        for (int64_t x = fq[0]; x <= lq[0]; ++x)
            for (int64_t y = fq[1]; y <= lq[1]; ++y)
                for (int64_t z = fq[2]; z <= lq[2]; ++z) {
                    const int64_t bin = bin_index(b, x, y, z);
                    const int64_t t0 = bin_start[bin], t1 = bin_start[bin + 1];
                    for (int64_t t = t0; t < t1; t += 32) {
                        bool keep = false;
                        double c = 0.0;
                        uint32_t j = 0;
                        if (t + lane < t1) {
                            j = bin_fil[t + lane];
                            if ((int64_t)j >= i) {
                                // the first bin of the overlap of i's query range and j's range
                                const int64_t jx = bin_cell(b, lo[j], 0), jy = bin_cell(b, lo[n + j], 1),
                                              jz = bin_cell(b, lo[2 * n + j], 2);
                                const bool first = x == (jx > fq[0] ? jx : fq[0]) && y == (jy > fq[1] ? jy : fq[1]) &&
                                                   z == (jz > fq[2] ? jz : fq[2]);
                                if (first) {
                                    const DevFil &fj = fil[j];
                                    keep = (int64_t)j == i || separation(fi, fj) < radius;
                                    if (keep) {
                                        c = ndot(fi.axes, fj.axes);
                                        keep = !(fabs(c) < kOrthogonalCos);
                                    }
                                }
                            }
                        }
                        const unsigned mask = __ballot_sync(0xffffffffu, keep);
                        if (kPass && keep) {
                            const int64_t o = base + __popc(mask & ((1u << lane) - 1u));
                            out_key[o] = ((unsigned long long)i << 32) | j;
                            out_cos[o] = c;
                        }
                        base += __popc(mask);
                        count += __popc(mask);
                    }
                }
        if (!kPass && lane == 0) row_count[i] = count;
    }
}

__global__ void near_split_pairs_kernel(const unsigned long long *__restrict__ key, int64_t np,
                                        int2 *__restrict__ pairs) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x)
        pairs[t] = make_int2((int)(key[t] >> 32), (int)(key[t] & 0xffffffffu));
}

unsigned grid_of(int64_t work, int threads) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads, 148 * 32));
}

// Stream-ordered scratch released at the end of the search.
struct Temp {
    cudaStream_t s;
    std::vector<void *> held;
    template <class T>
    cudaError_t get(T **p, size_t count) {
        void *q = nullptr;
        cudaError_t e = cache_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), s);
        if (e == cudaSuccess) held.push_back(q);
        *p = static_cast<T *>(q);
        return e;
    }
    ~Temp() {
        for (void *q : held) cache_free(q, s);
    }
};

}  // namespace

fh_status near_pairs_device(const DevFil *d_fil, int64_t n, double radius, cudaStream_t s, NearPairs &out,
                            fh_error_info *err) {
    out = NearPairs();
    out.n = n;
    FHB_CUDA(cache_alloc(reinterpret_cast<void **>(&out.off), sizeof(int64_t) * (size_t)(n + 1), s));
    FHB_CUDA(cudaMemsetAsync(out.off, 0, sizeof(int64_t) * (size_t)(n + 1), s));
    if (n == 0) return FH_OK;
    if (n > (int64_t)UINT32_MAX) return fail(err, FH_ERR_PFFT, "near-pair search: too many filaments");
    Temp tmp{s, {}};
    double *d_lo, *d_hi, *d_red;
    FHB_CUDA(tmp.get(&d_lo, (size_t)(3 * n)));
    FHB_CUDA(tmp.get(&d_hi, (size_t)(3 * n)));
    FHB_CUDA(tmp.get(&d_red, 6));
    near_boxes_kernel<<<grid_of(n, 256), 256, 0, s>>>(d_fil, n, d_lo, d_hi);
    FHB_CUDA(cudaGetLastError());
    // Overall box (min / max are exact, so the reduction order does not matter).
    size_t rb = 0;
    FHB_CUDA(cub::DeviceReduce::Min(nullptr, rb, d_lo, d_red, (int)n, s));
    size_t rb2 = 0;
    FHB_CUDA(cub::DeviceReduce::Max(nullptr, rb2, d_hi, d_red, (int)n, s));
    rb = std::max(rb, rb2);
    void *d_rt;
    FHB_CUDA(tmp.get(reinterpret_cast<uint8_t **>(&d_rt), rb));
    for (int a = 0; a < 3; ++a) {
        FHB_CUDA(cub::DeviceReduce::Min(d_rt, rb, d_lo + a * n, d_red + a, (int)n, s));
        FHB_CUDA(cub::DeviceReduce::Max(d_rt, rb, d_hi + a * n, d_red + 3 + a, (int)n, s));
    }
    double red[6];
    FHB_CUDA(cudaMemcpyAsync(red, d_red, sizeof red, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    // Bin geometry, near.rs:57-66.
    Bins b;
    double extent[3];
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = red[a];
        extent[a] = red[3 + a] - red[a];
    }
    const double emax = std::max(extent[0], std::max(extent[1], extent[2]));
    b.size = std::max(std::max(radius, emax * 1e-9), std::numeric_limits<double>::min());
    auto set_dims = [&]() {
        for (int a = 0; a < 3; ++a) b.dims[a] = (int64_t)std::floor(extent[a] / b.size) + 1;
    };
    set_dims();
    while (b.dims[0] * b.dims[1] * b.dims[2] > 8 * n + 64) {
        b.size *= 1.5;
        set_dims();
    }
    const int64_t nbins = b.dims[0] * b.dims[1] * b.dims[2];
    // (bin, filament) entries sorted by bin.
    int64_t *d_count, *d_off;
    unsigned *d_per_bin;
    int64_t *d_bin_start;
    FHB_CUDA(tmp.get(&d_count, (size_t)n + 1));
    FHB_CUDA(tmp.get(&d_off, (size_t)n + 1));
    FHB_CUDA(tmp.get(&d_per_bin, (size_t)nbins + 1));
    FHB_CUDA(tmp.get(&d_bin_start, (size_t)nbins + 1));
    FHB_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int64_t) * ((size_t)n + 1), s));
    FHB_CUDA(cudaMemsetAsync(d_per_bin, 0, sizeof(unsigned) * ((size_t)nbins + 1), s));
    bin_count_kernel<<<grid_of(n, 256), 256, 0, s>>>(d_lo, d_hi, n, b, d_count, d_per_bin);
    FHB_CUDA(cudaGetLastError());
    size_t sb = 0, sb2 = 0;
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb, d_count, d_off, (int)(n + 1), s));
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb2, d_per_bin, d_bin_start, (int)(nbins + 1), s));
    sb = std::max(sb, sb2);
    void *d_st;
    FHB_CUDA(tmp.get(reinterpret_cast<uint8_t **>(&d_st), sb));
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(d_st, sb, d_count, d_off, (int)(n + 1), s));
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(d_st, sb, d_per_bin, d_bin_start, (int)(nbins + 1), s));
    int64_t entries = 0;
    FHB_CUDA(cudaMemcpyAsync(&entries, d_off + n, sizeof entries, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    if (entries > (int64_t)INT32_MAX) return fail(err, FH_ERR_PFFT, "near-pair search: too many bin entries");
    uint32_t *d_key, *d_key2, *d_val, *d_val2;
    FHB_CUDA(tmp.get(&d_key, (size_t)entries));
    FHB_CUDA(tmp.get(&d_key2, (size_t)entries));
    FHB_CUDA(tmp.get(&d_val, (size_t)entries));
    FHB_CUDA(tmp.get(&d_val2, (size_t)entries));
    bin_emit_kernel<<<grid_of(n, 256), 256, 0, s>>>(d_lo, d_hi, n, b, d_off, d_key, d_val);
    FHB_CUDA(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 32 && (int64_t(1) << end_bit) < nbins) ++end_bit;
    size_t kb = 0;
    FHB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, kb, d_key, d_key2, d_val, d_val2, (int)entries, 0, end_bit, s));
    void *d_kt;
    FHB_CUDA(tmp.get(reinterpret_cast<uint8_t **>(&d_kt), kb));
    FHB_CUDA(cub::DeviceRadixSort::SortPairs(d_kt, kb, d_key, d_key2, d_val, d_val2, (int)entries, 0, end_bit, s));
    // Rows: counts, offsets, pairs.
    int64_t *d_rows;
    FHB_CUDA(tmp.get(&d_rows, (size_t)n + 1));
    FHB_CUDA(cudaMemsetAsync(d_rows, 0, sizeof(int64_t) * ((size_t)n + 1), s));
    const unsigned row_blocks = (unsigned)std::min<int64_t>((n + kNearWarps - 1) / kNearWarps, 148 * 64);
    near_rows_kernel<0><<<row_blocks, 32 * kNearWarps, 0, s>>>(d_fil, d_lo, d_hi, n, b, radius, d_bin_start, d_val2,
                                                              d_rows, nullptr, nullptr, nullptr);
    FHB_CUDA(cudaGetLastError());
    size_t ob = 0;
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, ob, d_rows, out.off, (int)(n + 1), s));
    void *d_ot;
    FHB_CUDA(tmp.get(reinterpret_cast<uint8_t **>(&d_ot), ob));
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(d_ot, ob, d_rows, out.off, (int)(n + 1), s));
    int64_t np = 0;
    FHB_CUDA(cudaMemcpyAsync(&np, out.off + n, sizeof np, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    out.count = np;
    FHB_CUDA(cache_alloc(reinterpret_cast<void **>(&out.pairs), sizeof(int2) * (size_t)std::max<int64_t>(np, 1), s));
    FHB_CUDA(cache_alloc(reinterpret_cast<void **>(&out.cos), sizeof(double) * (size_t)std::max<int64_t>(np, 1), s));
    if (np) {
        unsigned long long *d_pk, *d_pk2;
        double *d_pc;
        FHB_CUDA(tmp.get(&d_pk, (size_t)np));
        FHB_CUDA(tmp.get(&d_pk2, (size_t)np));
        FHB_CUDA(tmp.get(&d_pc, (size_t)np));
        near_rows_kernel<1><<<row_blocks, 32 * kNearWarps, 0, s>>>(d_fil, d_lo, d_hi, n, b, radius, d_bin_start,
                                                                  d_val2, nullptr, out.off, d_pk, d_pc);
        FHB_CUDA(cudaGetLastError());
        int key_bits = 33;
        while (key_bits < 64 && (int64_t(1) << (key_bits - 32)) < n) ++key_bits;
        size_t pb = 0;
        FHB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, pb, d_pk, d_pk2, d_pc, out.cos, (int)np, 0, key_bits, s));
        void *d_pt;
        FHB_CUDA(tmp.get(reinterpret_cast<uint8_t **>(&d_pt), pb));
        FHB_CUDA(cub::DeviceRadixSort::SortPairs(d_pt, pb, d_pk, d_pk2, d_pc, out.cos, (int)np, 0, key_bits, s));
        near_split_pairs_kernel<<<grid_of(np, 256), 256, 0, s>>>(d_pk2, np, out.pairs);
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(cudaStreamSynchronize(s));
    return FH_OK;
}

void near_pairs_free(NearPairs &p, cudaStream_t s) {
    if (p.off) cache_free(p.off, s);
    if (p.pairs) cache_free(p.pairs, s);
    if (p.cos) cache_free(p.cos, s);
    p = NearPairs();
}

}  // namespace fhb

using namespace fhb;

extern "C" fh_status fh_test_near_pairs(const fh_filament *filaments, size_t n, double radius, int64_t *off,
                                        int64_t *cols, size_t cap, size_t *total, fh_error_info *err) {
    clear_error(err);
    if ((n && (!filaments || !off)) || !total) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    if (!(radius >= 0.0 && std::isfinite(radius))) return fail(err, FH_ERR_INVALID_ARGUMENT, "invalid radius");
    fh_status st = ensure_device(err);
    if (st) return st;
    cudaStream_t s = nullptr;
    FHB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{s};
    std::vector<DevFil> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = make_devfil(filaments[i]);
    DevFil *d_fil = nullptr;
    FHB_CUDA(cache_alloc(reinterpret_cast<void **>(&d_fil), sizeof(DevFil) * std::max<size_t>(n, 1), s));
    struct FilGuard {
        DevFil *p;
        cudaStream_t s;
        ~FilGuard() { cache_free(p, s); }
    } fg{d_fil, s};
    if (n) FHB_CUDA(cudaMemcpyAsync(d_fil, h.data(), sizeof(DevFil) * n, cudaMemcpyHostToDevice, s));
    NearPairs near;
    st = near_pairs_device(d_fil, (int64_t)n, radius, s, near, err);
    struct NearGuard {
        NearPairs *p;
        cudaStream_t s;
        ~NearGuard() { near_pairs_free(*p, s); }
    } ng{&near, s};
    if (st) return st;
    *total = (size_t)near.count;
    FHB_CUDA(cudaMemcpyAsync(off, near.off, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
    if (near.count && cols && (size_t)near.count <= cap) {
        std::vector<int2> pairs((size_t)near.count);
        FHB_CUDA(cudaMemcpyAsync(pairs.data(), near.pairs, sizeof(int2) * pairs.size(), cudaMemcpyDeviceToHost, s));
        FHB_CUDA(cudaStreamSynchronize(s));
        for (size_t k = 0; k < pairs.size(); ++k) cols[k] = pairs[k].y;
    }
    FHB_CUDA(cudaStreamSynchronize(s));
    return FH_OK;
}
