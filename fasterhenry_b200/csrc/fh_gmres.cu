// Device GMRES (see fh_gmres.cuh).  The Arnoldi loop, the rotations and the
// stopping rule follow gmres.rs:91-215; every vector operation is a kernel
// on the solver's stream, and the host reads back one Hessenberg column and
// one norm per Arnoldi step.
#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "fh_gmres.cuh"

namespace fhb {

namespace {

constexpr int kRB = 256;  // reduction blocks (fixed: the combination order never depends on n's scheduling)
constexpr int kRT = 256;  // threads per block

// Layout of GmresWork::red (doubles).
constexpr int kMaxPartial = 2 * kRB;            // kRB
constexpr int kSumPartial = 3 * kRB;            // kRB
constexpr int kScale = 4 * kRB;                 // 1
constexpr int kSum = 4 * kRB + 1;               // 1
constexpr int kRedLen = 4 * kRB + 8;

using cplx = std::complex<double>;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

__global__ void __launch_bounds__(kRT) maxabs_partial_kernel(const double2 *__restrict__ v, int64_t n,
                                                             double *__restrict__ partial) {
    __shared__ double sh[kRT];
    double m = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kRT + threadIdx.x; i < n; i += (int64_t)kRB * kRT) {
        const double a = hypot(v[i].x, v[i].y);
        m = fmax(m, a);
        if (a != a) m = a;  // NaN propagates
    }
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = kRT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double o = sh[threadIdx.x + s];
            sh[threadIdx.x] = (o != o) ? o : fmax(sh[threadIdx.x], o);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(kRT) max_final_kernel(const double *__restrict__ partial, double *__restrict__ out) {
    __shared__ double sh[kRT];
    sh[threadIdx.x] = partial[threadIdx.x];
    __syncthreads();
    for (int s = kRT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double o = sh[threadIdx.x + s];
            sh[threadIdx.x] = (o != o) ? o : fmax(sh[threadIdx.x], o);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// sum |v_i / scale|^2 (gmres.rs:234-241: the scaled norm).
__global__ void __launch_bounds__(kRT) sumsq_partial_kernel(const double2 *__restrict__ v, int64_t n,
                                                            const double *__restrict__ scale,
                                                            double *__restrict__ partial) {
    __shared__ double sh[kRT];
    const double sc = *scale;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kRT + threadIdx.x; i < n; i += (int64_t)kRB * kRT) {
        const double a = v[i].x / sc, b = v[i].y / sc;
        acc += a * a + b * b;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kRT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(kRT) sum_final_kernel(const double *__restrict__ partial, double *__restrict__ out) {
    __shared__ double sh[kRT];
    sh[threadIdx.x] = partial[threadIdx.x];
    __syncthreads();
    for (int s = kRT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// The projections of w on the cnt basis vectors V_0 .. V_cnt-1 at once
// (classical Gram-Schmidt): per block and vector k, the partial sum of
// conj(V_k[i]) w[i] over the block's rows (warp shuffles, then the warps in
// order) into partial[2 (k kRB + block)].
__global__ void __launch_bounds__(kRT) multidot_partial_kernel(const double2 *__restrict__ V,
                                                               const double2 *__restrict__ w, int64_t n, int cnt,
                                                               double *__restrict__ partial) {
    __shared__ double2 sh[kRT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < cnt; ++k) {
        const double2 *vk = V + (size_t)k * n;
        double2 acc = make_double2(0.0, 0.0);
        for (int64_t i = (int64_t)blockIdx.x * kRT + threadIdx.x; i < n; i += (int64_t)kRB * kRT) {
            const double2 a = vk[i], b = w[i];
            acc = cadd(acc, make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x));
        }
        for (int o = 16; o > 0; o >>= 1) {
            acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
        }
        if (lane == 0) sh[warp] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double2 t = sh[0];
            for (int q = 1; q < kRT / 32; ++q) t = cadd(t, sh[q]);
            partial[2 * ((size_t)k * kRB + blockIdx.x)] = t.x;
            partial[2 * ((size_t)k * kRB + blockIdx.x) + 1] = t.y;
        }
        __syncthreads();
    }
}

// h[k] = the sum of vector k's kRB partials (block k, fixed tree).
__global__ void __launch_bounds__(kRT) multidot_final_kernel(const double *__restrict__ partial,
                                                             double2 *__restrict__ h) {
    __shared__ double2 sh[kRT];
    const size_t base = (size_t)blockIdx.x * kRB;
    sh[threadIdx.x] = make_double2(partial[2 * (base + threadIdx.x)], partial[2 * (base + threadIdx.x) + 1]);
    __syncthreads();
    for (int s = kRT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = cadd(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) h[blockIdx.x] = sh[0];
}

// w -= sum_k h[k] V_k, the terms taken in increasing k.
__global__ void multi_axpy_kernel(double2 *__restrict__ w, const double2 *__restrict__ V,
                                  const double2 *__restrict__ h, int cnt, int64_t n) {
    extern __shared__ double2 hs[];
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) hs[k] = h[k];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 y = w[i];
        for (int k = 0; k < cnt; ++k) {
            const double2 a = hs[k], b = V[(size_t)k * n + i];
            y.x += -a.x * b.x + a.y * b.y;
            y.y += -a.x * b.y - a.y * b.x;
        }
        w[i] = y;
    }
}

// y += a x (a from the host).
__global__ void axpy_kernel(double2 *__restrict__ y, const double2 *__restrict__ x, double2 a, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 b = x[i];
        double2 v = y[i];
        v.x += a.x * b.x - a.y * b.y;
        v.y += a.x * b.y + a.y * b.x;
        y[i] = v;
    }
}

__global__ void div_real_kernel(double2 *__restrict__ out, const double2 *__restrict__ in, double s, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = make_double2(in[i].x / s, in[i].y / s);
}

__global__ void sub_kernel(double2 *__restrict__ r, const double2 *__restrict__ b, const double2 *__restrict__ ax,
                           int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = make_double2(b[i].x - ax[i].x, b[i].y - ax[i].y);
}

__global__ void add_kernel(double2 *__restrict__ x, const double2 *__restrict__ c, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = make_double2(x[i].x + c[i].x, x[i].y + c[i].y);
}

inline unsigned grid_of(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

// The reference's complex division (num-complex): (a conj(b)) / |b|^2.
cplx cdiv_ref(cplx a, cplx b) {
    const double ns = b.real() * b.real() + b.imag() * b.imag();
    return cplx((a.real() * b.real() + a.imag() * b.imag()) / ns, (a.imag() * b.real() - a.real() * b.imag()) / ns);
}
cplx cmul_ref(cplx a, cplx b) {
    return cplx(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

// The rotation G = [c s; -conj(s) c] with G [a; b] = [r; 0] (gmres.rs:244-257).
void givens(cplx a, cplx b, double &c, cplx &s, cplx &r) {
    const double abs_a = std::hypot(a.real(), a.imag()), abs_b = std::hypot(b.real(), b.imag());
    if (abs_b == 0.0) {
        c = 1.0;
        s = 0.0;
        r = a;
        return;
    }
    if (abs_a == 0.0) {
        c = 0.0;
        s = 1.0;
        r = b;
        return;
    }
    const double length = std::hypot(abs_a, abs_b);
    const cplx phase(a.real() / abs_a, a.imag() / abs_a);
    c = abs_a / length;
    s = cmul_ref(phase, cplx(b.real() / length, -b.imag() / length));
    r = cplx(phase.real() * length, phase.imag() * length);
}

struct Norm {
    double scale = 0, sum = 0;
    double value() const { return (scale == 0.0 || !std::isfinite(scale)) ? scale : scale * std::sqrt(sum); }
};

}  // namespace

GmresWork::~GmresWork() {
    void *p[] = {V, w, r, t, u, h, red, part};
    for (void *q : p)
        if (q) cudaFree(q);
}

fh_status GmresWork::ensure(int64_t n_, int restart_, fh_error_info *err) {
    if (n_ <= n && restart_ <= restart && V) return FH_OK;
    void *p[] = {V, w, r, t, u, h, red, part};
    for (void *q : p)
        if (q) cudaFree(q);
    V = w = r = t = u = h = nullptr;
    red = part = nullptr;
    n = n_;
    restart = restart_;
    auto alloc = [&](void **q, size_t bytes) { return cudaMalloc(q, std::max<size_t>(bytes, 16)); };
    if (alloc((void **)&V, sizeof(double2) * (size_t)(restart + 1) * n) != cudaSuccess ||
        alloc((void **)&w, sizeof(double2) * n) != cudaSuccess || alloc((void **)&r, sizeof(double2) * n) != cudaSuccess ||
        alloc((void **)&t, sizeof(double2) * n) != cudaSuccess || alloc((void **)&u, sizeof(double2) * n) != cudaSuccess ||
        alloc((void **)&h, sizeof(double2) * 2 * (restart + 1)) != cudaSuccess ||
        alloc((void **)&red, sizeof(double) * kRedLen) != cudaSuccess ||
        alloc((void **)&part, sizeof(double) * 2 * kRB * (size_t)(restart + 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation of the GMRES workspace failed");
    }
    return FH_OK;
}

fh_status gmres_solve(int64_t n, const DeviceOp &apply, const DeviceOp &precondition, const double2 *d_b, double2 *d_x,
                      const GmresParams &params, cudaStream_t s, GmresWork &work, GmresOutcome *out,
                      fh_error_info *err) {
    GmresOutcome oc;
    const int restart = (int)std::max<int64_t>(1, std::min<int64_t>(params.restart, n));
    fh_status st = work.ensure(n, restart, err);
    if (st) return st;
    auto norm_of = [&](const double2 *v, Norm &nm) -> fh_status {
        maxabs_partial_kernel<<<kRB, kRT, 0, s>>>(v, n, work.red + kMaxPartial);
        max_final_kernel<<<1, kRT, 0, s>>>(work.red + kMaxPartial, work.red + kScale);
        sumsq_partial_kernel<<<kRB, kRT, 0, s>>>(v, n, work.red + kScale, work.red + kSumPartial);
        sum_final_kernel<<<1, kRT, 0, s>>>(work.red + kSumPartial, work.red + kSum);
        FHB_CUDA(cudaGetLastError());
        double hv[2];
        FHB_CUDA(cudaMemcpyAsync(hv, work.red + kScale, sizeof hv, cudaMemcpyDeviceToHost, s));
        FHB_CUDA(cudaStreamSynchronize(s));
        nm.scale = hv[0];
        nm.sum = hv[1];
        return FH_OK;
    };
    auto residual = [&](double &rn) -> fh_status {
        fh_status e = apply(d_x, work.t, err);
        if (e) return e;
        sub_kernel<<<grid_of(n), 256, 0, s>>>(work.r, d_b, work.t, n);
        FHB_CUDA(cudaGetLastError());
        Norm nm;
        e = norm_of(work.r, nm);
        rn = nm.value();
        return e;
    };
    Norm bn;
    st = norm_of(d_b, bn);
    if (st) return st;
    const double b_norm = bn.value();
    if (b_norm == 0.0) {
        FHB_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double2) * n, s));
        FHB_CUDA(cudaStreamSynchronize(s));
        oc.converged = true;
        if (out) *out = oc;
        return FH_OK;
    }
    const double target = params.tolerance * b_norm;
    int64_t iterations = 0;
    double r_norm = 0.0;
    st = residual(r_norm);
    if (st) return st;
    std::vector<cplx> hcol_dev(2 * (size_t)(restart + 1));
    for (;;) {
        oc.iterations = iterations;
        oc.relative_residual = r_norm / b_norm;
        if (r_norm <= target) {
            oc.converged = true;
            break;
        }
        if (iterations >= params.max_iterations || !std::isfinite(r_norm)) {
            oc.converged = false;
            break;
        }
        // One Arnoldi cycle from the current residual.
        div_real_kernel<<<grid_of(n), 256, 0, s>>>(work.V, work.r, r_norm, n);
        FHB_CUDA(cudaGetLastError());
        std::vector<std::vector<cplx>> hess;
        std::vector<std::pair<double, cplx>> rot;
        std::vector<cplx> g((size_t)restart + 1, cplx(0.0, 0.0));
        g[0] = cplx(r_norm, 0.0);
        while ((int)hess.size() < restart && iterations < params.max_iterations) {
            const int j = (int)hess.size();
            double2 *vj = work.V + (size_t)j * n;
            st = precondition(vj, work.u, err);
            if (st) return st;
            st = apply(work.u, work.w, err);
            if (st) return st;
            iterations += 1;
            // Classical Gram-Schmidt twice: each pass projects w on all of
            // V_0 .. V_j in one product and removes them in one update (the
            // reference's modified Gram-Schmidt applied twice reaches the same
            // orthogonality; three launches per pass instead of three per
            // basis vector).
            for (int pass = 0; pass < 2; ++pass) {
                double2 *hp = work.h + pass * (restart + 1);
                multidot_partial_kernel<<<kRB, kRT, 0, s>>>(work.V, work.w, n, j + 1, work.part);
                multidot_final_kernel<<<j + 1, kRT, 0, s>>>(work.part, hp);
                multi_axpy_kernel<<<grid_of(n), 256, sizeof(double2) * (j + 1), s>>>(work.w, work.V, hp, j + 1, n);
            }
            FHB_CUDA(cudaGetLastError());
            Norm wn;
            st = norm_of(work.w, wn);
            if (st) return st;
            const double next_norm = wn.value();
            FHB_CUDA(cudaMemcpyAsync(hcol_dev.data(), work.h, sizeof(double2) * 2 * (restart + 1),
                                     cudaMemcpyDeviceToHost, s));
            FHB_CUDA(cudaStreamSynchronize(s));
            std::vector<cplx> column((size_t)j + 2, cplx(0.0, 0.0));
            for (int pass = 0; pass < 2; ++pass)
                for (int k = 0; k <= j; ++k) column[k] += hcol_dev[pass * (restart + 1) + k];
            column[j + 1] = cplx(next_norm, 0.0);
            for (size_t i = 0; i < rot.size(); ++i) {
                const double c = rot[i].first;
                const cplx sr = rot[i].second;
                const cplx a = column[i], b = column[i + 1];
                column[i] = cplx(a.real() * c, a.imag() * c) + cmul_ref(sr, b);
                column[i + 1] = cplx(b.real() * c, b.imag() * c) - cmul_ref(std::conj(sr), a);
            }
            double c;
            cplx sr, rr;
            givens(column[j], column[j + 1], c, sr, rr);
            column[j] = rr;
            column[j + 1] = cplx(0.0, 0.0);
            rot.push_back({c, sr});
            const cplx gj = g[j];
            g[j] = cplx(gj.real() * c, gj.imag() * c);
            g[j + 1] = -cmul_ref(std::conj(sr), gj);
            hess.push_back(column);
            if (next_norm == 0.0 || std::abs(g[j + 1]) <= target) break;
            div_real_kernel<<<grid_of(n), 256, 0, s>>>(work.V + (size_t)(j + 1) * n, work.w, next_norm, n);
            FHB_CUDA(cudaGetLastError());
        }
        // Back substitution, then x += M (V y).
        const int steps = (int)hess.size();
        std::vector<cplx> y((size_t)steps);
        for (int i = steps - 1; i >= 0; --i) {
            cplx sum = g[i];
            for (int k = i + 1; k < steps; ++k) sum -= cmul_ref(hess[k][i], y[k]);
            y[i] = cdiv_ref(sum, hess[i][i]);
        }
        FHB_CUDA(cudaMemsetAsync(work.u, 0, sizeof(double2) * n, s));
        for (int k = 0; k < steps; ++k)
            axpy_kernel<<<grid_of(n), 256, 0, s>>>(work.u, work.V + (size_t)k * n, make_double2(y[k].real(), y[k].imag()),
                                                   n);
        FHB_CUDA(cudaGetLastError());
        st = precondition(work.u, work.t, err);
        if (st) return st;
        add_kernel<<<grid_of(n), 256, 0, s>>>(d_x, work.t, n);
        FHB_CUDA(cudaGetLastError());
        st = residual(r_norm);
        if (st) return st;
    }
    if (out) *out = oc;
    return FH_OK;
}

}  // namespace fhb
