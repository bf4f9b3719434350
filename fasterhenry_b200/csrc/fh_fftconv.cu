// The pFFT convolution K (*) q on the device, without a library FFT: pruned
// mixed-radix (2, 3, 4, 5) Stockham transforms in shared memory, in FP32 or
// FP64 (pfft/fft.rs:155-320 of the reference, re-designed for the GPU).
//
// The sources q live on the n0 x n1 x n2 grid; the aperiodic convolution
// needs transforms of length m_a >= 2 n_a - 1 per axis (a torus of 2^a 3^b
// 5^c points).  Only n0 n1 lines carry data along axis 2, only n0 planes
// along axis 1, and only n0 planes of the result are read back, so the
// transform is pruned axis by axis (the reference prunes the same way):
//
//   1. axis 2 forward  A[n0][n1][n2]  -> B[n0][n1][m2]   (n0 n1 lines)
//   2. axis 1 forward  B[n0][n1][m2]  -> C[n0][m1][m2]   (n0 m2 lines)
//   3. axis 0 forward, times the kernel's real spectrum, axis 0 inverse, in
//      place in C (m1 m2 lines of n0 points in, n0 points out)
//   4. axis 1 inverse  C[n0][m1][m2]  -> B[n0][n1][m2]
//   5. axis 2 inverse  B[n0][n1][m2]  -> A[n0][n1][n2]   (the potentials)
//
// Each step is one launch of fft_lines_kernel: a CTA loads a tile of lines
// into shared memory (consecutive lines when they are contiguous, else
// consecutive columns, so every global access is a run of adjacent
// elements), zero-pads them to m, runs one Stockham pass per radix between
// two shared buffers, and writes the first `keep` outputs.  Two real source
// fields travel in one complex grid (real and imaginary parts), as in the
// reference's convolver.  The kernel's spectrum is computed at set-up by the
// same kernels (unpruned, FP64) from the wrapped kernel grid; it is real
// because the wrapped kernel is even.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "fh_device.cuh"
#include "fh_fftconv.h"

namespace fhb {
namespace {

// Threads per CTA: 512 for FP32 (two CTAs, 32 warps per SM), 256 for FP64
// (whose wider lines leave fewer butterflies per tile).
template <class T>
constexpr int fft_threads() {
    return sizeof(T) == 4 ? 512 : 256;
}
constexpr size_t kFftSmemBudget = 100 * 1024;  // two CTAs per SM
constexpr double kPi = 3.14159265358979323846;

template <class T>
struct Cplx;
template <>
struct Cplx<float> {
    using type = float2;
};
template <>
struct Cplx<double> {
    using type = double2;
};

template <class V>
__device__ __forceinline__ V cmul(V a, V b) {
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// R-point DFT of v in place, W = exp(sign 2 pi i / R).
template <int R, class V, class T>
__device__ __forceinline__ void small_dft(V (&v)[R], int sign) {
    if constexpr (R == 2) {
        V a = v[0], b = v[1];
        v[0].x = a.x + b.x;
        v[0].y = a.y + b.y;
        v[1].x = a.x - b.x;
        v[1].y = a.y - b.y;
    } else if constexpr (R == 4) {
        const V a = v[0], b = v[1], c = v[2], d = v[3];
        V s0, s1, d0, d1;
        s0.x = a.x + c.x, s0.y = a.y + c.y;
        d0.x = a.x - c.x, d0.y = a.y - c.y;
        s1.x = b.x + d.x, s1.y = b.y + d.y;
        d1.x = b.x - d.x, d1.y = b.y - d.y;
        // (b - d) times sign * i
        V jd;
        jd.x = -(T)sign * d1.y;
        jd.y = (T)sign * d1.x;
        v[0].x = s0.x + s1.x, v[0].y = s0.y + s1.y;
        v[2].x = s0.x - s1.x, v[2].y = s0.y - s1.y;
        v[1].x = d0.x + jd.x, v[1].y = d0.y + jd.y;
        v[3].x = d0.x - jd.x, v[3].y = d0.y - jd.y;
    } else {
        // cos and sin of 2 pi k / R, k = 0 .. R-1
        constexpr double c3[3] = {1.0, -0.5, -0.5};
        constexpr double s3[3] = {0.0, 0.86602540378443864676, -0.86602540378443864676};
        constexpr double c5[5] = {1.0, 0.30901699437494742410, -0.80901699437494742410, -0.80901699437494742410,
                                  0.30901699437494742410};
        constexpr double s5[5] = {0.0, 0.95105651629515357212, 0.58778525229247312917, -0.58778525229247312917,
                                  -0.95105651629515357212};
        V out[R];
#pragma unroll
        for (int b = 0; b < R; ++b) {
            V acc = v[0];
#pragma unroll
            for (int a = 1; a < R; ++a) {
                const int e = (a * b) % R;
                const T c = (T)(R == 3 ? c3[e] : c5[e]);
                const T s = (T)sign * (T)(R == 3 ? s3[e] : s5[e]);
                acc.x += v[a].x * c - v[a].y * s;
                acc.y += v[a].x * s + v[a].y * c;
            }
            out[b] = acc;
        }
#pragma unroll
        for (int b = 0; b < R; ++b) v[b] = out[b];
    }
}

// One Stockham pass of radix R over `lines` interleaved lines of length m
// (element t of line l at t * lines + l), src -> dst; tw holds
// exp(-2 pi i t / m) in shared memory.
template <int R, class V, class T>
__device__ void stockham_pass(const V *__restrict__ src, V *__restrict__ dst, int m, int lines, int Ns,
                              const V *__restrict__ tw, int sign) {
    const int nb = m / R;
    const int tw_step = m / (Ns * R);
    for (int idx = threadIdx.x; idx < nb * lines; idx += blockDim.x) {
        const int line = idx % lines, j = idx / lines;
        V v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * lines + line];
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; ++r) {
            V w = tw[k * r * tw_step];
            if (sign > 0) w.y = -w.y;
            v[r] = cmul(v[r], w);
        }
        small_dft<R, V, T>(v, sign);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[(base + r * Ns) * lines + line] = v[r];
    }
}

// The transform of `lines` lines of length m held in a (interleaved), with b
// as the second buffer; returns the buffer holding the result.
template <class V, class T>
__device__ V *stockham(V *a, V *b, int m, int lines, const FftAxis &ax, const V *__restrict__ tw, int sign) {
    int Ns = 1;
    for (int f = 0; f < ax.nfac; ++f) {
        const int R = ax.fac[f];
        __syncthreads();
        if (R == 4)
            stockham_pass<4, V, T>(a, b, m, lines, Ns, tw, sign);
        else if (R == 2)
            stockham_pass<2, V, T>(a, b, m, lines, Ns, tw, sign);
        else if (R == 3)
            stockham_pass<3, V, T>(a, b, m, lines, Ns, tw, sign);
        else
            stockham_pass<5, V, T>(a, b, m, lines, Ns, tw, sign);
        Ns *= R;
        V *t = a;
        a = b;
        b = t;
    }
    __syncthreads();
    return a;
}

// One pruned axis transform over a batch of arrays.  An array holds
// `outer` x len x `inner` complex elements (len = n_in for the input, keep
// for the output); line (o, c) is elements (o len + t) inner + c.  Lines are
// tiled `tile` at a time: consecutive o when inner == 1 (each line
// contiguous), else consecutive c.  With `spectrum`, the forward transform is
// multiplied by spectrum[t inner + c] (real) and transformed back (sign
// flipped) before the write.  in and out may be the same array (the fused
// axis-0 step): a CTA reads its whole tile before it writes, and tiles are
// disjoint.
template <class T>
__global__ void __launch_bounds__(fft_threads<T>())
    fft_lines_kernel(const typename Cplx<T>::type *in, typename Cplx<T>::type *out,
                     int64_t in_stride, int64_t out_stride, int64_t outer, int64_t inner, int n_in, int keep,
                     FftAxis ax, const typename Cplx<T>::type *__restrict__ tw_global, int sign, int tile,
                     const T *__restrict__ spectrum) {
    using V = typename Cplx<T>::type;
    extern __shared__ __align__(16) unsigned char fft_smem[];
    V *bufa = reinterpret_cast<V *>(fft_smem);
    V *bufb = bufa + (size_t)tile * ax.m;
    V *tw = bufb + (size_t)tile * ax.m;  // the twiddles, read by every pass
    const int m = ax.m;
    for (int t = threadIdx.x; t < m; t += blockDim.x) tw[t] = tw_global[t];
    const V *src = in + (int64_t)blockIdx.y * in_stride;
    V *dst = out + (int64_t)blockIdx.y * out_stride;
    const bool contiguous = inner == 1;
    const int64_t tiles = contiguous ? (outer + tile - 1) / tile : outer * ((inner + tile - 1) / tile);
    for (int64_t tt = blockIdx.x; tt < tiles; tt += gridDim.x) {
        int64_t o0, c0;
        int lines;
        if (contiguous) {
            o0 = tt * tile;
            c0 = 0;
            lines = (int)(outer - o0 < tile ? outer - o0 : (int64_t)tile);
        } else {
            const int64_t per = (inner + tile - 1) / tile;
            o0 = tt / per;
            c0 = (tt % per) * tile;
            lines = (int)(inner - c0 < tile ? inner - c0 : (int64_t)tile);
        }
        __syncthreads();  // the previous tile's reads of the buffers are done
        // load (zero-padded to m)
        for (int idx = threadIdx.x; idx < lines * m; idx += blockDim.x) {
            int l, t;
            if (contiguous) {
                l = idx / m;
                t = idx % m;
            } else {
                t = idx / lines;
                l = idx % lines;
            }
            V v;
            v.x = v.y = (T)0;
            if (t < n_in)
                v = contiguous ? src[(o0 + l) * (int64_t)n_in + t] : src[(o0 * n_in + t) * inner + c0 + l];
            bufa[t * lines + l] = v;
        }
        V *res = stockham<V, T>(bufa, bufb, m, lines, ax, tw, sign);
        if (spectrum) {
            for (int idx = threadIdx.x; idx < lines * m; idx += blockDim.x) {
                const int t = idx / lines, l = idx % lines;
                const T s = spectrum[(int64_t)t * inner + c0 + l];
                V v = res[idx];
                v.x *= s;
                v.y *= s;
                res[idx] = v;
            }
            V *other = res == bufa ? bufb : bufa;
            res = stockham<V, T>(res, other, m, lines, ax, tw, -sign);
        }
        for (int idx = threadIdx.x; idx < lines * keep; idx += blockDim.x) {
            int l, t;
            if (contiguous) {
                l = idx / keep;
                t = idx % keep;
            } else {
                t = idx / lines;
                l = idx % lines;
            }
            const V v = res[t * lines + l];
            if (contiguous)
                dst[(o0 + l) * (int64_t)keep + t] = v;
            else
                dst[(o0 * keep + t) * inner + c0 + l] = v;
        }
    }
}

// The wrapped kernel 1 / (h |d|) on the padded grid (zero at the origin and
// beyond the unpadded extent), FP64 complex.
__global__ void wrapped_kernel_kernel(double2 *__restrict__ out, int64_t n0, int64_t n1, int64_t n2, int64_t m0,
                                      int64_t m1, int64_t m2, double spacing) {
    const int64_t total = m0 * m1 * m2;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = p % m2, rest = p / m2, j = rest % m1, i = rest / m1;
        auto wrap = [](int64_t t, int64_t n, int64_t m, int64_t &d) {
            if (t < n) {
                d = t;
                return true;
            }
            if (t + n > m) {
                d = t - m;
                return true;
            }
            return false;
        };
        int64_t di, dj, dk;
        double v = 0.0;
        if (wrap(i, n0, m0, di) && wrap(j, n1, m1, dj) && wrap(k, n2, m2, dk)) {
            const double r2 = (double)(di * di + dj * dj + dk * dk);
            v = r2 == 0.0 ? 0.0 : 1.0 / (spacing * sqrt(r2));
        }
        out[p] = make_double2(v, 0.0);
    }
}

template <class T>
__global__ void spectrum_store_kernel(const double2 *__restrict__ in, T *__restrict__ out, int64_t total) {
    const double scale = 1.0 / (double)total;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x)
        out[p] = (T)(in[p].x * scale);
}

unsigned blocks_of(int64_t work, int threads, int64_t cap = 148 * 16) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads, cap));
}

// Lines per CTA: as many as two buffers of them and the twiddles fit the
// shared-memory budget, up to about 8,192 points per tile (short lines come
// many to a tile).
template <class T>
int tile_for(int m) {
    const size_t elem = sizeof(typename Cplx<T>::type);
    const size_t per = 2 * elem * (size_t)m;
    const size_t want = std::max<size_t>(16, 8192 / (size_t)m);
    const size_t room = kFftSmemBudget > elem * (size_t)m ? kFftSmemBudget - elem * (size_t)m : 0;
    return (int)std::max<size_t>(1, std::min<size_t>(want, room / per));
}

// One axis step: outer x n_in x inner -> outer x keep x inner, `batch` arrays.
template <class T>
fh_status axis_step(const void *in, void *out, int64_t in_stride, int64_t out_stride, int64_t outer, int64_t inner,
                    int n_in, int keep, const FftAxis &ax, const void *tw, int sign, const T *spectrum, int batch,
                    cudaStream_t s, fh_error_info *err) {
    using V = typename Cplx<T>::type;
    const int tile = tile_for<T>(ax.m);
    const size_t smem = sizeof(V) * ((2 * (size_t)tile + 1) * ax.m);
    if (smem > 227 * 1024)
        return fail(err, FH_ERR_PFFT, "pFFT convolution: axis length " + std::to_string(ax.m) +
                                          " does not fit the transform kernel's shared memory");
    const int64_t tiles = inner == 1 ? (outer + tile - 1) / tile : outer * ((inner + tile - 1) / tile);
    FHB_CUDA(cudaFuncSetAttribute(fft_lines_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, 148 * 8));
    fft_lines_kernel<T><<<dim3(gx, (unsigned)batch), fft_threads<T>(), smem, s>>>(
        static_cast<const V *>(in), static_cast<V *>(out), in_stride, out_stride, outer, inner, n_in, keep, ax,
        static_cast<const V *>(tw), sign, tile, spectrum);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

}  // namespace

bool fft_axis_plan(int64_t m, FftAxis &ax) {
    ax = FftAxis();
    if (m < 1 || m > kFftMaxLength) return false;
    ax.m = (int)m;
    int64_t r = m;
    // radix 4 first, then 2, 3, 5
    for (int p : {4, 2, 3, 5})
        while (r % p == 0) {
            if (ax.nfac == kFftMaxFactors) return false;
            ax.fac[ax.nfac++] = p;
            r /= p;
        }
    return r == 1;
}

size_t fftconv_work_elems(const FftConvShape &sh) {
    const int64_t a = sh.n[0] * sh.n[1] * sh.n[2];
    const int64_t b = sh.n[0] * sh.n[1] * sh.m[2];
    const int64_t c = sh.n[0] * sh.m[1] * sh.m[2];
    return (size_t)(a + b + c);
}

template <class T>
fh_status fftconv_setup(const FftConvShape &sh, double spacing, FftConvTables &tab, cudaStream_t s,
                        fh_error_info *err) {
    using V = typename Cplx<T>::type;
    for (int a = 0; a < 3; ++a)
        if (!fft_axis_plan(sh.m[a], tab.axis[a]))
            return fail(err, FH_ERR_PFFT,
                        "pFFT convolution: padded axis length " + std::to_string((long long)sh.m[a]) +
                            " is not a 2^a 3^b 5^c length up to " + std::to_string(kFftMaxLength));
    // Twiddle tables exp(-2 pi i t / m), computed in FP64 on the host.
    for (int a = 0; a < 3; ++a) {
        const int64_t m = sh.m[a];
        std::vector<double2> h64((size_t)m);
        for (int64_t t = 0; t < m; ++t) {
            const double ang = -2.0 * kPi * (double)t / (double)m;
            h64[(size_t)t] = make_double2(std::cos(ang), std::sin(ang));
        }
        std::vector<V> h((size_t)m);
        for (int64_t t = 0; t < m; ++t) {
            h[(size_t)t].x = (T)h64[(size_t)t].x;
            h[(size_t)t].y = (T)h64[(size_t)t].y;
        }
        FHB_CUDA(cache_alloc(&tab.tw[a], sizeof(V) * (size_t)m, s));
        FHB_CUDA(cudaMemcpyAsync(tab.tw[a], h.data(), sizeof(V) * (size_t)m, cudaMemcpyHostToDevice, s));
        if (sizeof(T) == 4) {
            FHB_CUDA(cache_alloc(&tab.tw64[a], sizeof(double2) * (size_t)m, s));
            FHB_CUDA(cudaMemcpyAsync(tab.tw64[a], h64.data(), sizeof(double2) * (size_t)m, cudaMemcpyHostToDevice, s));
        } else {
            tab.tw64[a] = tab.tw[a];
        }
        FHB_CUDA(cudaStreamSynchronize(s));
    }
    // Spectrum: unpruned FP64 forward transform of the wrapped kernel.
    const int64_t P = sh.m[0] * sh.m[1] * sh.m[2];
    double2 *grid = nullptr, *tmp = nullptr;
    FHB_CUDA(cache_alloc(reinterpret_cast<void **>(&grid), sizeof(double2) * (size_t)P, s));
    FHB_CUDA(cache_alloc(reinterpret_cast<void **>(&tmp), sizeof(double2) * (size_t)P, s));
    struct Release {
        void *a, *b;
        cudaStream_t s;
        ~Release() {
            cache_free(a, s);
            cache_free(b, s);
        }
    } release{grid, tmp, s};
    wrapped_kernel_kernel<<<blocks_of(P, 256), 256, 0, s>>>(grid, sh.n[0], sh.n[1], sh.n[2], sh.m[0], sh.m[1],
                                                           sh.m[2], spacing);
    FHB_CUDA(cudaGetLastError());
    const int64_t m0 = sh.m[0], m1 = sh.m[1], m2 = sh.m[2];
    fh_status e = axis_step<double>(grid, tmp, 0, 0, m0 * m1, 1, (int)m2, (int)m2, tab.axis[2], tab.tw64[2], -1,
                                    nullptr, 1, s, err);
    if (!e)
        e = axis_step<double>(tmp, grid, 0, 0, m0, m2, (int)m1, (int)m1, tab.axis[1], tab.tw64[1], -1, nullptr, 1, s,
                              err);
    if (!e)
        e = axis_step<double>(grid, tmp, 0, 0, 1, m1 * m2, (int)m0, (int)m0, tab.axis[0], tab.tw64[0], -1, nullptr, 1,
                              s, err);
    if (e) return e;
    FHB_CUDA(cache_alloc(&tab.spectrum, sizeof(T) * (size_t)P, s));
    spectrum_store_kernel<T><<<blocks_of(P, 256), 256, 0, s>>>(tmp, static_cast<T *>(tab.spectrum), P);
    FHB_CUDA(cudaGetLastError());
    FHB_CUDA(cudaStreamSynchronize(s));
    tab.shape = sh;
    tab.fp32 = sizeof(T) == 4;
    return FH_OK;
}

template <class T>
fh_status fftconv_run(const FftConvTables &tab, void *work, int grids, cudaStream_t s, fh_error_info *err) {
    using V = typename Cplx<T>::type;
    const FftConvShape &sh = tab.shape;
    const int64_t n0 = sh.n[0], n1 = sh.n[1], n2 = sh.n[2], m1 = sh.m[1], m2 = sh.m[2];
    const int64_t sa = n0 * n1 * n2, sb = n0 * n1 * m2, sc = n0 * m1 * m2;
    V *A = static_cast<V *>(work);
    V *B = A + sa * grids;
    V *C = B + sb * grids;
    const T *spec = static_cast<const T *>(tab.spectrum);
    fh_status e = axis_step<T>(A, B, sa, sb, n0 * n1, 1, (int)n2, (int)m2, tab.axis[2], tab.tw[2], -1, nullptr, grids,
                               s, err);
    if (!e)
        e = axis_step<T>(B, C, sb, sc, n0, m2, (int)n1, (int)m1, tab.axis[1], tab.tw[1], -1, nullptr, grids, s, err);
    if (!e)
        e = axis_step<T>(C, C, sc, sc, 1, m1 * m2, (int)n0, (int)n0, tab.axis[0], tab.tw[0], -1, spec, grids, s, err);
    if (!e)
        e = axis_step<T>(C, B, sc, sb, n0, m2, (int)m1, (int)n1, tab.axis[1], tab.tw[1], +1, nullptr, grids, s, err);
    if (!e)
        e = axis_step<T>(B, A, sb, sa, n0 * n1, 1, (int)m2, (int)n2, tab.axis[2], tab.tw[2], +1, nullptr, grids, s,
                         err);
    return e;
}

void fftconv_free(FftConvTables &tab, cudaStream_t s) {
    for (int a = 0; a < 3; ++a) {
        if (tab.tw64[a] && tab.tw64[a] != tab.tw[a]) cache_free(tab.tw64[a], s);
        if (tab.tw[a]) cache_free(tab.tw[a], s);
        tab.tw[a] = tab.tw64[a] = nullptr;
    }
    if (tab.spectrum) cache_free(tab.spectrum, s);
    tab.spectrum = nullptr;
}

template fh_status fftconv_setup<float>(const FftConvShape &, double, FftConvTables &, cudaStream_t, fh_error_info *);
template fh_status fftconv_setup<double>(const FftConvShape &, double, FftConvTables &, cudaStream_t,
                                         fh_error_info *);
template fh_status fftconv_run<float>(const FftConvTables &, void *, int, cudaStream_t, fh_error_info *);
template fh_status fftconv_run<double>(const FftConvTables &, void *, int, cudaStream_t, fh_error_info *);

}  // namespace fhb

using namespace fhb;

extern "C" fh_status fh_test_grid_convolution(const int64_t *n, const int64_t *m, double spacing, int32_t fp32,
                                              const double *sources, int32_t fields, double *potentials,
                                              fh_error_info *err) {
    clear_error(err);
    if (!n || !m || !sources || !potentials || fields < 1)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument or no fields");
    FftConvShape sh;
    for (int a = 0; a < 3; ++a) {
        if (n[a] < 1 || m[a] < 2 * n[a] - 1)
            return fail(err, FH_ERR_INVALID_ARGUMENT, "padded axis shorter than 2 n - 1");
        sh.n[a] = n[a];
        sh.m[a] = m[a];
    }
    fh_status st = ensure_device(err);
    if (st) return st;
    cudaStream_t s = nullptr;
    FHB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct Guard {
        cudaStream_t s;
        FftConvTables tab;
        void *work = nullptr;
        ~Guard() {
            cudaStreamSynchronize(s);
            if (work) cache_free(work, s);
            fftconv_free(tab, s);
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } g{s};
    st = fp32 ? fftconv_setup<float>(sh, spacing, g.tab, s, err) : fftconv_setup<double>(sh, spacing, g.tab, s, err);
    if (st) return st;
    const int grids = (fields + 1) / 2;
    const int64_t G = sh.n[0] * sh.n[1] * sh.n[2];
    const size_t elem = fp32 ? 4 : 8;
    FHB_CUDA(cache_alloc(&g.work, 2 * elem * fftconv_work_elems(sh) * (size_t)grids, s));
    // fields as real / imaginary parts of the complex source grids
    std::vector<double> h((size_t)(2 * G * grids), 0.0);
    for (int f = 0; f < fields; ++f)
        for (int64_t p = 0; p < G; ++p) h[(size_t)(2 * ((f / 2) * G + p) + (f & 1))] = sources[(size_t)(f * G + p)];
    if (fp32) {
        std::vector<float> hf(h.begin(), h.end());
        FHB_CUDA(cudaMemcpyAsync(g.work, hf.data(), 4 * hf.size(), cudaMemcpyHostToDevice, s));
        st = fftconv_run<float>(g.tab, g.work, grids, s, err);
        if (st) return st;
        FHB_CUDA(cudaMemcpyAsync(hf.data(), g.work, 4 * hf.size(), cudaMemcpyDeviceToHost, s));
        FHB_CUDA(cudaStreamSynchronize(s));
        std::copy(hf.begin(), hf.end(), h.begin());
    } else {
        FHB_CUDA(cudaMemcpyAsync(g.work, h.data(), 8 * h.size(), cudaMemcpyHostToDevice, s));
        st = fftconv_run<double>(g.tab, g.work, grids, s, err);
        if (st) return st;
        FHB_CUDA(cudaMemcpyAsync(h.data(), g.work, 8 * h.size(), cudaMemcpyDeviceToHost, s));
        FHB_CUDA(cudaStreamSynchronize(s));
    }
    for (int f = 0; f < fields; ++f)
        for (int64_t p = 0; p < G; ++p) potentials[(size_t)(f * G + p)] = h[(size_t)(2 * ((f / 2) * G + p) + (f & 1))];
    return FH_OK;
}
