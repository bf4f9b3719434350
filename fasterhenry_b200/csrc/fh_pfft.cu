// The precorrected-FFT operator on the device: y = L x without forming L
// (pfft/mod.rs:482-560 of the reference).
//
//   y = C x + mu0/4pi sum_c d_c . W^T (K (*) (W (d_c . x)))
//
// per product, for `count` vectors at once:
//   1. near_kernel        y = C x (CSR rows of precorrected near pairs; warp
//                         per filament);
//   2. spread_kernel      the grid sources q_{v,c}(g) = sum_i W_ig d_ic x_vi,
//                         one thread per grid point over the transposed
//                         projection (no atomics), written straight into the
//                         zero-padded complex grids: two real sources per
//                         complex grid (real and imaginary part);
//   3. cuFFT Z2Z forward over every padded grid, spectrum_kernel multiplies by
//      the kernel's real spectrum (with the 1/P of the inverse), cuFFT inverse:
//      the aperiodic convolution K (*) q on a 2N-1 padded torus (fft.rs:1-30);
//   4. interp_kernel      y_vi += mu0/4pi sum_c d_ic sum_g W_ig phi_{v,c}(g),
//                         warp per filament, read from the padded grids.
//
// The near-field corrections C_ij = L_ij(exact) - mu0/4pi cos_ij G_ij are
// built at set-up from the host's grid approximations G_ij and the exact
// partial inductances of the same pairs, evaluated by the device fill in
// pair-list mode; the upper triangle is mirrored into full rows (near.rs:
// 263-298).  The kernel spectrum is the forward transform of the wrapped
// kernel 1/|r_g - r_h| on the padded grid, real for an even kernel.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <chrono>
#include <string>

#include "fh_device.cuh"
#include "fh_pfft.h"

namespace fhb {

namespace {

constexpr double kMu0Over4PiP = 1e-7;

#define FHB_CUFFT(call)                                                                        \
    do {                                                                                       \
        cufftResult r_ = (call);                                                               \
        if (r_ != CUFFT_SUCCESS)                                                               \
            return ::fhb::fail(err, FH_ERR_CUDA, std::string(#call " failed: cufft status ") + \
                                                     std::to_string((int)r_));                 \
    } while (0)

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
// Kernel spectrum: the wrapped kernel on the padded grid, then (after the
// forward transform) its real part times 1 / P.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool wrapped_offset(int64_t k, int64_t n, int64_t m, int64_t &d) {
    if (k < n) {
        d = k;
        return true;
    }
    if (k + n > m) {
        d = k - m;
        return true;
    }
    return false;
}

__global__ void kernel_grid_kernel(cufftDoubleComplex *__restrict__ out, int64_t n0, int64_t n1, int64_t n2,
                                   int64_t m0, int64_t m1, int64_t m2, double spacing) {
    const int64_t total = m0 * m1 * m2;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = p % m2, rest = p / m2, j = rest % m1, i = rest / m1;
        int64_t di, dj, dk;
        double v = 0.0;
        if (wrapped_offset(i, n0, m0, di) && wrapped_offset(j, n1, m1, dj) && wrapped_offset(k, n2, m2, dk)) {
            const double r2 = (double)(di * di + dj * dj + dk * dk);
            v = r2 == 0.0 ? 0.0 : 1.0 / (spacing * sqrt(r2));
        }
        out[p] = make_cuDoubleComplex(v, 0.0);
    }
}

__global__ void spectrum_extract_kernel(const cufftDoubleComplex *__restrict__ in, double *__restrict__ spectrum,
                                        int64_t total) {
    const double scale = 1.0 / (double)total;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x)
        spectrum[p] = in[p].x * scale;
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

// y_v = C x_v, warp per row.
__global__ void __launch_bounds__(256) near_kernel(const int64_t *__restrict__ off, const uint32_t *__restrict__ col,
                                                   const double *__restrict__ val, const double *__restrict__ x,
                                                   double *__restrict__ y, int64_t n, int count) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < n; row += warps) {
        const int64_t b = off[row], e = off[row + 1];
        for (int v = 0; v < count; ++v) {
            const double *xv = x + (int64_t)v * n;
            double acc = 0.0;
            for (int64_t k = b + lane; k < e; k += 32) acc += val[k] * xv[col[k]];
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if (lane == 0) y[(int64_t)v * n + row] = acc;
        }
    }
}

// Grid sources into the padded complex grids: real source r = v * ncomp + c
// goes to grid r / 2, part r % 2, at padded position (i m1 + j) m2 + k.
__global__ void __launch_bounds__(256) spread_kernel(const int64_t *__restrict__ off,
                                                     const uint32_t *__restrict__ fil,
                                                     const double *__restrict__ w, const double *__restrict__ dir,
                                                     const double *__restrict__ x, double *__restrict__ work,
                                                     ApplyArgs a) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.G; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = off[g], e = off[g + 1];
        if (b == e) continue;
        const int64_t k = g % a.n2, rest = g / a.n2, j = rest % a.n1, i = rest / a.n1;
        const int64_t pp = (i * a.m1 + j) * a.m2 + k;
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
                work[2 * ((int64_t)(r >> 1) * a.P + pp) + (r & 1)] = q[c];
            }
        }
    }
}

__global__ void spectrum_kernel(cufftDoubleComplex *__restrict__ work, const double *__restrict__ spectrum,
                                int64_t P, int64_t grids) {
    const int64_t total = P * grids;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const double s = spectrum[t % P];
        cufftDoubleComplex z = work[t];
        z.x *= s;
        z.y *= s;
        work[t] = z;
    }
}

// y_vi += mu0/4pi sum_c d_ic sum_g W_ig phi_{v,c}(g), warp per filament.
__global__ void __launch_bounds__(256) interp_kernel(const int64_t *__restrict__ off, const uint32_t *__restrict__ idx,
                                                     const double *__restrict__ w, const double *__restrict__ dir,
                                                     const double *__restrict__ work, double *__restrict__ y,
                                                     ApplyArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < a.n; i += warps) {
        const int64_t b = off[i], e = off[i + 1];
        for (int v = 0; v < a.count; ++v) {
            double far = 0.0;
            for (int c = 0; c < a.ncomp; ++c) {
                const int r = v * a.ncomp + c;
                const double *grid = work + 2 * (int64_t)(r >> 1) * a.P + (r & 1);
                double sum = 0.0;
                for (int64_t t = b + lane; t < e; t += 32) {
                    const int64_t g = idx[t];
                    const int64_t k = g % a.n2, rest = g / a.n2, jj = rest % a.n1, ii = rest / a.n1;
                    sum += w[t] * grid[2 * ((ii * a.m1 + jj) * a.m2 + k)];
                }
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
                far += dir[3 * i + a.comp[c]] * sum;
            }
            if (lane == 0) y[(int64_t)v * a.n + i] += kMu0Over4PiP * far;
        }
    }
}

fh_status get_plan(PfftDevice &op, int batch, cufftHandle *out, fh_error_info *err) {
    for (auto &p : op.plans)
        if (p.first == batch) {
            *out = (cufftHandle)p.second;
            return FH_OK;
        }
    cufftHandle plan;
    int dims[3] = {(int)op.padded[0], (int)op.padded[1], (int)op.padded[2]};
    FHB_CUFFT(cufftPlanMany(&plan, 3, dims, nullptr, 1, (int)op.P, nullptr, 1, (int)op.P, CUFFT_Z2Z, batch));
    FHB_CUFFT(cufftSetStream(plan, (cudaStream_t)op.stream));
    op.plans.push_back({batch, (int)plan});
    *out = plan;
    return FH_OK;
}

fh_status ensure_work(PfftDevice &op, size_t bytes, fh_error_info *err) {
    if (op.work_bytes >= bytes) return FH_OK;
    if (op.d_work) cudaFree(op.d_work);
    op.d_work = nullptr;
    op.work_bytes = 0;
    if (cudaMalloc(&op.d_work, bytes) != cudaSuccess) {
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

fh_status pfft_apply_impl(PfftDevice &op, const double *d_x, double *d_y, int count, fh_error_info *err);

PfftDevice::~PfftDevice() {
    for (auto &p : plans) cufftDestroy((cufftHandle)p.second);
    void *ptrs[] = {d_dir, d_proj_off, d_proj_idx, d_proj_w, d_spread_off, d_spread_fil,
                    d_spread_w, d_near_off, d_near_col, d_near_val, d_spectrum, d_work};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (own_stream && stream) cudaStreamDestroy((cudaStream_t)stream);
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

    // Kernel spectrum.
    FHB_CUDA(cudaMalloc(&op.d_spectrum, sizeof(double) * op.P));
    e = ensure_work(op, sizeof(cufftDoubleComplex) * (size_t)op.P, err);
    if (e) return e;
    cufftDoubleComplex *work = reinterpret_cast<cufftDoubleComplex *>(op.d_work);
    kernel_grid_kernel<<<blocks_for(op.P, 256), 256, 0, s>>>(work, op.grid.dims[0], op.grid.dims[1], op.grid.dims[2],
                                                              op.padded[0], op.padded[1], op.padded[2],
                                                              op.grid.spacing);
    FHB_CUDA(cudaGetLastError());
    cufftHandle plan;
    e = get_plan(op, 1, &plan, err);
    if (e) return e;
    FHB_CUFFT(cufftExecZ2Z(plan, work, work, CUFFT_FORWARD));
    spectrum_extract_kernel<<<blocks_for(op.P, 256), 256, 0, s>>>(work, op.d_spectrum, op.P);
    FHB_CUDA(cudaGetLastError());
    FHB_CUDA(cudaStreamSynchronize(s));
    op.setup_device_s = now_s() - t1;
    return FH_OK;
}

// Algorithmic bytes of one product of `count` vectors: the near-field CSR
// (12 B per entry) and both passes over the projection (12 B per entry each),
// the vectors, and per padded complex grid its zeroing, three axis passes of
// each transform (read + write), the spectrum product (read, write, spectrum).
double pfft_apply_bytes(const PfftDevice &op, int count) {
    const int ncomp = (int)op.components.size();
    const double grids = (double)((count * ncomp + 1) / 2);
    return 12.0 * (double)op.near_entries + 24.0 * (double)op.projection_entries + 32.0 * (double)op.n * count +
           grids * (double)op.P * (16.0 + 2.0 * 3.0 * 32.0 + 40.0);
}

fh_status pfft_apply(PfftDevice &op, const double *d_x, double *d_y, int count, fh_error_info *err) {
    if (op.n == 0 || count <= 0) return FH_OK;
    prof_begin((cudaStream_t)op.stream, FH_PROF_PFFT_APPLY);
    fh_status st = pfft_apply_impl(op, d_x, d_y, count, err);
    prof_end((cudaStream_t)op.stream, FH_PROF_PFFT_APPLY, pfft_apply_bytes(op, count));
    return st;
}

fh_status pfft_apply_impl(PfftDevice &op, const double *d_x, double *d_y, int count, fh_error_info *err) {
    cudaStream_t s = (cudaStream_t)op.stream;
    near_kernel<<<blocks_for(op.n * 32, 256), 256, 0, s>>>(op.d_near_off, op.d_near_col, op.d_near_val, d_x, d_y,
                                                             op.n, count);
    FHB_CUDA(cudaGetLastError());
    const int ncomp = (int)op.components.size();
    if (ncomp == 0) return FH_OK;
    const int real_grids = count * ncomp;
    const int grids = (real_grids + 1) / 2;
    fh_status e = ensure_work(op, sizeof(cufftDoubleComplex) * (size_t)op.P * grids, err);
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
    double *work = reinterpret_cast<double *>(op.d_work);
    FHB_CUDA(cudaMemsetAsync(work, 0, sizeof(cufftDoubleComplex) * (size_t)op.P * grids, s));
    spread_kernel<<<blocks_for(op.G, 256), 256, 0, s>>>(op.d_spread_off, op.d_spread_fil, op.d_spread_w, op.d_dir, d_x,
                                                         work, a);
    FHB_CUDA(cudaGetLastError());
    cufftHandle plan;
    e = get_plan(op, grids, &plan, err);
    if (e) return e;
    cufftDoubleComplex *cw = reinterpret_cast<cufftDoubleComplex *>(op.d_work);
    FHB_CUFFT(cufftExecZ2Z(plan, cw, cw, CUFFT_FORWARD));
    spectrum_kernel<<<blocks_for(op.P * grids, 256), 256, 0, s>>>(cw, op.d_spectrum, op.P, grids);
    FHB_CUDA(cudaGetLastError());
    FHB_CUFFT(cufftExecZ2Z(plan, cw, cw, CUFFT_INVERSE));
    interp_kernel<<<blocks_for(op.n * 32, 256), 256, 0, s>>>(op.d_proj_off, op.d_proj_idx, op.d_proj_w, op.d_dir, work,
                                                               d_y, a);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

}  // namespace fhb
