// The precorrected-FFT operator on the device: y = L x without forming L
// (pfft/mod.rs:482-560 of the reference).
//
//   y = C x + mu0/4pi sum_c d_c . W^T (K (*) (W (d_c . x)))
//
// per product, for `count` vectors at once:
//   1. near_kernel        y = C x (CSR rows of precorrected near pairs; warp
//                         per filament, every vector from one pass over the
//                         row);
//   2. spread_kernel      the grid sources q_{v,c}(g) = sum_i W_ig d_ic x_vi,
//                         one thread per grid point over the transposed
//                         projection (no atomics), written to compact complex
//                         grids (two real sources per grid: real and imaginary
//                         part) in the convolution's precision;
//   3. fftconv_run        the aperiodic convolution K (*) q by pruned
//                         mixed-radix transforms on the 2N-1 padded torus
//                         (fh_fftconv.cu; FP64 or FP32);
//   4. interp_kernel      y_vi += mu0/4pi sum_c d_ic sum_g W_ig phi_{v,c}(g),
//                         warp per filament, from the compact grids.
//
// The near-field corrections C_ij = L_ij(exact) - mu0/4pi cos_ij G_ij are
// built at set-up from the device's grid approximations G_ij and the exact
// partial inductances of the same pairs, evaluated by the device fill in
// pair-list mode; the upper triangle is mirrored into full rows (near.rs:
// 263-298).  The kernel spectrum is the forward transform of the wrapped
// kernel 1/|r_g - r_h| on the padded grid, real for an even kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <string>

#include "fh_device.cuh"
#include "fh_pfft.h"

namespace fhb {

namespace {

constexpr double kMu0Over4PiP = 1e-7;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class T>
cudaError_t upload(T **d, const std::vector<T> &h, cudaStream_t s) {
    cudaError_t e = cudaMalloc((void **)d, std::max<size_t>(1, h.size()) * sizeof(T));
    if (e != cudaSuccess) return e;
    if (h.empty()) return cudaSuccess;
    return cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

// ---------------------------------------------------------------------------
// Products.
// ---------------------------------------------------------------------------
struct ApplyArgs {
    int64_t n, G, P;
    int64_t n1, n2, m1, m2;  // unpadded / padded extents of axes 1 and 2
    int ncomp;
    int comp[3];
    int count;
};

// y_v = C x_v, warp per row; the row is read once for up to kNearVec vectors.
constexpr int kNearVec = 4;
__global__ void __launch_bounds__(256) near_kernel(const int64_t *__restrict__ off, const uint32_t *__restrict__ col,
                                                   const double *__restrict__ val, const double *__restrict__ x,
                                                   double *__restrict__ y, int64_t n, int count) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < n; row += warps) {
        const int64_t b = off[row], e = off[row + 1];
        for (int v0 = 0; v0 < count; v0 += kNearVec) {
            const int nv = count - v0 < kNearVec ? count - v0 : kNearVec;
            double acc[kNearVec] = {0.0, 0.0, 0.0, 0.0};
            for (int64_t k = b + lane; k < e; k += 32) {
                const double a = val[k];
                const int64_t c = col[k];
#pragma unroll
                for (int v = 0; v < kNearVec; ++v)
                    if (v < nv) acc[v] += a * x[(int64_t)(v0 + v) * n + c];
            }
#pragma unroll
            for (int v = 0; v < kNearVec; ++v) {
                double t = acc[v];
                for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
                if (lane == 0 && v < nv) y[(int64_t)(v0 + v) * n + row] = t;
            }
        }
    }
}

// Grid sources into compact complex grids: real source r = v * ncomp + c
// goes to grid r / 2, part r % 2, at the grid index g.  T: the convolution's
// precision.
template <class T>
__global__ void __launch_bounds__(256) spread_kernel(const int64_t *__restrict__ off,
                                                     const uint32_t *__restrict__ fil,
                                                     const double *__restrict__ w, const double *__restrict__ dir,
                                                     const double *__restrict__ x, T *__restrict__ work,
                                                     ApplyArgs a) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.G; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = off[g], e = off[g + 1];
        for (int v = 0; v < a.count; ++v) {
            const double *xv = x + (int64_t)v * a.n;
            double q[3] = {0.0, 0.0, 0.0};
            for (int64_t t = b; t < e; ++t) {
                const uint32_t f = fil[t];
                const double s = w[t] * xv[f];
                for (int c = 0; c < a.ncomp; ++c) q[c] += s * dir[3 * (int64_t)f + a.comp[c]];
            }
            for (int c = 0; c < a.ncomp; ++c) {
                const int r = v * a.ncomp + c;
                work[2 * ((int64_t)(r >> 1) * a.G + g) + (r & 1)] = (T)q[c];
            }
        }
        // the unused imaginary part of an odd number of sources
        if ((a.count * a.ncomp) & 1) work[2 * ((int64_t)((a.count * a.ncomp) >> 1) * a.G + g) + 1] = (T)0;
    }
}

// y_vi += mu0/4pi sum_c d_ic sum_g W_ig phi_{v,c}(g), warp per filament, from
// the compact potential grids.
template <class T>
__global__ void __launch_bounds__(256) interp_kernel(const int64_t *__restrict__ off, const uint32_t *__restrict__ idx,
                                                     const double *__restrict__ w, const double *__restrict__ dir,
                                                     const T *__restrict__ work, double *__restrict__ y,
                                                     ApplyArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < a.n; i += warps) {
        const int64_t b = off[i], e = off[i + 1];
        for (int v = 0; v < a.count; ++v) {
            double far = 0.0;
            for (int c = 0; c < a.ncomp; ++c) {
                const int r = v * a.ncomp + c;
                const T *grid = work + 2 * (int64_t)(r >> 1) * a.G + (r & 1);
                double sum = 0.0;
                for (int64_t t = b + lane; t < e; t += 32) sum += w[t] * (double)grid[2 * (int64_t)idx[t]];
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
                far += dir[3 * i + a.comp[c]] * sum;
            }
            if (lane == 0) y[(int64_t)v * a.n + i] += kMu0Over4PiP * far;
        }
    }
}

// The convolution's work buffer of `bytes`, from the device cache (grown on
// demand; the old buffer goes back to the cache, stream-ordered).
fh_status ensure_work(PfftDevice &op, size_t bytes, fh_error_info *err) {
    if (op.work_bytes >= bytes) return FH_OK;
    cudaStream_t s = (cudaStream_t)op.stream;
    if (op.d_work) cache_free(op.d_work, s);
    op.d_work = nullptr;
    op.work_bytes = 0;
    if (cache_alloc(&op.d_work, bytes, s) != cudaSuccess) {
        cudaGetLastError();
        return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    op.work_bytes = bytes;
    return FH_OK;
}

inline unsigned blocks_for(int64_t work, int threads, int64_t cap = 148 * 16) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads, cap));
}

}  // namespace

fh_status pfft_apply_impl(PfftDevice &op, const double *d_x, double *d_y, int count, fh_error_info *err,
                          bool full_precision);

PfftDevice::~PfftDevice() {
    cudaStream_t s = (cudaStream_t)stream;
    fftconv_free(conv, s);
    fftconv_free(conv64, s);
    if (d_work) cache_free(d_work, s);
    void *ptrs[] = {d_dir, d_proj_off, d_proj_idx, d_proj_w, d_spread_off, d_spread_fil,
                    d_spread_w, d_near_off, d_near_col, d_near_val};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (own_stream && stream) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
}

size_t PfftDevice::memory_bytes() const {
    return (size_t)projection_entries * 2 * (4 + 8) + (size_t)(n + 1 + G + 1) * 8 + (size_t)near_entries * (4 + 8) +
           (size_t)(n + 1) * 8 + (size_t)n * 3 * 8 + (size_t)P * 8 + work_bytes;
}

fh_status pfft_build(const fh_filament *fil, int64_t n, const PfftConfig &cfg, void *stream, PfftDevice &op,
                     fh_error_info *err) {
    const double t0 = now_s();
    PfftSetup st;
    fh_status e = pfft_setup(fil, n, cfg, st, err);
    if (e) return e;
    const double t1 = now_s();
    op.setup_host_s = t1 - t0;
    if (stream) {
        op.stream = stream;
    } else {
        cudaStream_t s;
        FHB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        op.stream = s;
        op.own_stream = true;
    }
    cudaStream_t s = (cudaStream_t)op.stream;
    op.n = n;
    if (n == 0) return FH_OK;
    op.grid = st.grid;
    for (int a = 0; a < 3; ++a) op.padded[a] = st.padded[a];
    op.G = st.grid.len();
    op.P = op.padded[0] * op.padded[1] * op.padded[2];
    op.components = st.components;

    // Near pairs (device search), projections, their transpose and the grid
    // approximations of the near pairs on the device; then the exact near
    // pairs (device fill, pair list) and the near-field matrix.
    std::vector<DevFil> hf((size_t)n);
    for (int64_t i = 0; i < n; ++i) hf[i] = make_devfil(fil[i]);
    DevFil *d_fil = nullptr;
    double *d_exact = nullptr;
    NearPairs near;
    struct Release {
        cudaStream_t s;
        DevFil **fil;
        double **exact;
        NearPairs *near;
        ~Release() {
            if (*fil) cudaFree(*fil);
            if (*exact) cudaFree(*exact);
            near_pairs_free(*near, s);
        }
    } release{s, &d_fil, &d_exact, &near};
    FHB_CUDA(upload(&d_fil, hf, s));
    const double tn = now_s();
    e = near_pairs_device(d_fil, n, st.radius, s, near, err);
    if (e) return e;
    op.setup_near_s = now_s() - tn;
    PfftDeviceSetup ds;
    e = pfft_device_setup(st, fil, near, s, ds, err);
    op.d_proj_off = ds.proj_off;
    op.d_proj_idx = ds.proj_idx;
    op.d_proj_w = ds.proj_w;
    op.d_spread_off = ds.spread_off;
    op.d_spread_fil = ds.spread_fil;
    op.d_spread_w = ds.spread_w;
    struct FreeGrid {
        double *p;
        ~FreeGrid() {
            if (p) cudaFree(p);
        }
    } free_grid{ds.pair_grid};
    if (e) return e;
    op.projection_entries = ds.entries;
    const int64_t np = near.count;
    FHB_CUDA(cudaMalloc(&d_exact, sizeof(double) * std::max<int64_t>(np, 1)));
    if (np) {
        e = device_fill_pairs(d_fil, n, near.pairs, np, d_exact, s, nullptr, err);
        if (e) return e;
    }
    e = pfft_near_csr(n, np, near.pairs, d_exact, ds.pair_grid, near.cos, s, &op.d_near_off, &op.d_near_col,
                      &op.d_near_val, &op.near_entries, err);
    if (e) return e;
    FHB_CUDA(upload(&op.d_dir, st.directions, s));

    // The convolution's twiddles and the kernel's spectrum.
    FftConvShape shape;
    for (int a = 0; a < 3; ++a) {
        shape.n[a] = op.grid.dims[a];
        shape.m[a] = op.padded[a];
    }
    op.fft_fp32 = cfg.fft_fp32;
    e = op.fft_fp32 ? fftconv_setup<float>(shape, op.grid.spacing, op.conv, s, err)
                    : fftconv_setup<double>(shape, op.grid.spacing, op.conv, s, err);
    if (e) return e;
    if (op.fft_fp32) {
        e = fftconv_setup<double>(shape, op.grid.spacing, op.conv64, s, err);
        if (e) return e;
    }
    FHB_CUDA(cudaStreamSynchronize(s));
    op.setup_device_s = now_s() - t1;
    return FH_OK;
}

// Algorithmic bytes of one product of `count` vectors: the near-field CSR
// read once (12 B per entry), both passes over the projection (12 B per entry
// each), the vectors, and per complex grid (element size E: 8 B in FP32, 16 B
// in FP64) the pruned transform chain of fh_fftconv.cu: the sources A written
// and read, B = n0 n1 m2 and C = n0 m1 m2 written and read twice each, the
// spectrum (P reals), and the potentials A written and read.
double pfft_apply_bytes(const PfftDevice &op, int count, bool full_precision) {
    const int ncomp = (int)op.components.size();
    const double grids = (double)((count * ncomp + 1) / 2);
    const double E = op.fft_fp32 && !full_precision ? 8.0 : 16.0;
    const FftConvShape &sh = op.conv.shape;
    const double A = (double)sh.n[0] * sh.n[1] * sh.n[2], B = (double)sh.n[0] * sh.n[1] * sh.m[2],
                 C = (double)sh.n[0] * sh.m[1] * sh.m[2], P = (double)op.P;
    const double conv = E * (4.0 * A + 4.0 * B + 4.0 * C) + (E / 2.0) * P;
    return 12.0 * (double)op.near_entries + 24.0 * (double)op.projection_entries + 32.0 * (double)op.n * count +
           grids * conv;
}

fh_status pfft_apply(PfftDevice &op, const double *d_x, double *d_y, int count, fh_error_info *err,
                     bool full_precision) {
    if (op.n == 0 || count <= 0) return FH_OK;
    prof_begin((cudaStream_t)op.stream, FH_PROF_PFFT_APPLY);
    fh_status st = pfft_apply_impl(op, d_x, d_y, count, err, full_precision);
    prof_end((cudaStream_t)op.stream, FH_PROF_PFFT_APPLY, pfft_apply_bytes(op, count, full_precision));
    return st;
}

namespace {
template <class T>
fh_status apply_far(PfftDevice &op, const FftConvTables &conv, const double *d_x, double *d_y, int count,
                    fh_error_info *err) {
    cudaStream_t s = (cudaStream_t)op.stream;
    const int ncomp = (int)op.components.size();
    const int grids = (count * ncomp + 1) / 2;
    fh_status e = ensure_work(op, sizeof(T) * 2 * fftconv_work_elems(conv.shape) * (size_t)grids, err);
    if (e) return e;
    ApplyArgs a;
    a.n = op.n;
    a.G = op.G;
    a.P = op.P;
    a.n1 = op.grid.dims[1];
    a.n2 = op.grid.dims[2];
    a.m1 = op.padded[1];
    a.m2 = op.padded[2];
    a.ncomp = ncomp;
    for (int c = 0; c < 3; ++c) a.comp[c] = c < ncomp ? op.components[c] : 0;
    a.count = count;
    T *work = static_cast<T *>(op.d_work);
    spread_kernel<T><<<blocks_for(op.G, 256), 256, 0, s>>>(op.d_spread_off, op.d_spread_fil, op.d_spread_w, op.d_dir,
                                                            d_x, work, a);
    FHB_CUDA(cudaGetLastError());
    e = fftconv_run<T>(conv, work, grids, s, err);
    if (e) return e;
    interp_kernel<T><<<blocks_for(op.n * 32, 256), 256, 0, s>>>(op.d_proj_off, op.d_proj_idx, op.d_proj_w, op.d_dir,
                                                                 work, d_y, a);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}
}  // namespace

fh_status pfft_apply_impl(PfftDevice &op, const double *d_x, double *d_y, int count, fh_error_info *err,
                          bool full_precision) {
    cudaStream_t s = (cudaStream_t)op.stream;
    near_kernel<<<blocks_for(op.n * 32, 256), 256, 0, s>>>(op.d_near_off, op.d_near_col, op.d_near_val, d_x, d_y,
                                                             op.n, count);
    FHB_CUDA(cudaGetLastError());
    if (op.components.empty()) return FH_OK;
    if (op.fft_fp32 && !full_precision) return apply_far<float>(op, op.conv, d_x, d_y, count, err);
    return apply_far<double>(op, op.fft_fp32 ? op.conv64 : op.conv, d_x, d_y, count, err);
}

}  // namespace fhb
