// Matrix-free port impedance (iterative.rs of the reference): GMRES on the
// precorrected-FFT operator, never forming L or Z_ee.
//
//   Z(w) = Z_pp - Z_ep^T Z_ee^-1 Z_ep,   Z_ee x = M_e (R c + j w L c),  c = M_e^T x
//
// Assembly (IterativeSystem::assemble, iterative.rs:155-239): discretize, loop
// basis, the pFFT operator, the port columns Z_ep / Z_pp from one operator
// product per port (R and L are frequency independent), and the Jacobi
// diagonal of M_e R M_e^T and M_e L M_e^T (exact sum_a sum_b s_a s_b L_ab for
// loops of at most 32 branches, the self terms otherwise; the pair values
// come from the device fill in pair-list mode).
// Per frequency (iterative.rs:269-302, 454-485): one Jacobi-preconditioned
// GMRES solve per port on the device, each Z_ee product being a scatter to
// branch currents, one pFFT product of the real and imaginary parts
// together, the branch drops and a gather back to loops; then the Schur
// complement with a plain transpose and Z <- (Z + Z^T) / 2.  At f = 0 the
// system is M_e R M_e^T and no pFFT product runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <memory>
#include <string>
#include <vector>

#include "fh_cx.cuh"
#include "fh_device.cuh"
#include "fh_gmres.cuh"
#include "fh_pfft.h"

using namespace fhb;

namespace {

constexpr double kTauI = 6.283185307179586;
constexpr size_t kExactDiagonalMaxLoop = 32;  // iterative.rs:97

double wall_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// c_b = sum over the internal loops through branch b of sign x_loop, in loop
// order (transposed loop basis; iterative.rs:403-411).
__global__ void scatter_kernel(const double2 *__restrict__ x, const int64_t *__restrict__ off,
                               const int32_t *__restrict__ loop, const double *__restrict__ sign,
                               double2 *__restrict__ c, int64_t n) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n; b += (int64_t)gridDim.x * blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        for (int64_t k = off[b]; k < off[b + 1]; ++k) {
            const double2 v = x[loop[k]];
            const double s = sign[k];
            acc.x += v.x * s;
            acc.y += v.y * s;
        }
        c[b] = acc;
    }
}

// Real and imaginary parts as two real vectors (one pFFT product of both).
__global__ void split_kernel(const double2 *__restrict__ c, double *__restrict__ parts, int64_t n) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n; b += (int64_t)gridDim.x * blockDim.x) {
        parts[b] = c[b].x;
        parts[n + b] = c[b].y;
    }
}

// drop_b = r_b c_b + j w (L c)_b  (iterative.rs:432-451); w = 0 skips L.
__global__ void drop_kernel(const double2 *__restrict__ c, const double *__restrict__ r,
                            const double *__restrict__ flux, double omega, double2 *__restrict__ drop, int64_t n) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n; b += (int64_t)gridDim.x * blockDim.x) {
        const double rb = r[b];
        if (flux)
            drop[b] = make_double2(rb * c[b].x - omega * flux[n + b], rb * c[b].y + omega * flux[b]);
        else
            drop[b] = make_double2(c[b].x * rb, c[b].y * rb);
    }
}

// y_i = sum over loop i's branches of sign v_b, in row order (iterative.rs:488-505).
__global__ void gather_kernel(const double2 *__restrict__ v, const int64_t *__restrict__ row_ptr,
                              const int32_t *__restrict__ branch, const double *__restrict__ sign,
                              double2 *__restrict__ y, int64_t loops) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < loops; i += (int64_t)gridDim.x * blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            const double2 t = v[branch[k]];
            const double s = sign[k];
            acc.x += t.x * s;
            acc.y += t.y * s;
        }
        y[i] = acc;
    }
}

// Jacobi: out = v / d (num-complex division).
__global__ void jacobi_kernel(const double2 *__restrict__ v, const double2 *__restrict__ d, double2 *__restrict__ out,
                              int64_t m) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const Cx<double> q = cdiv(Cx<double>{v[i].x, v[i].y}, Cx<double>{d[i].x, d[i].y});
        out[i] = make_double2(q.re, q.im);
    }
}

// y = A x for a dense column-major complex matrix (GMRES tests).
__global__ void dense_matvec_kernel(const double2 *__restrict__ a, const double2 *__restrict__ x,
                                    double2 *__restrict__ y, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        for (int64_t k = 0; k < n; ++k) {
            const double2 m = a[i + k * n], v = x[k];
            acc.x += m.x * v.x - m.y * v.y;
            acc.y += m.x * v.y + m.y * v.x;
        }
        y[i] = acc;
    }
}

inline unsigned grid_n(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

template <class T>
cudaError_t put(T **d, const std::vector<T> &h, cudaStream_t s) {
    cudaError_t e = cudaMalloc((void **)d, std::max<size_t>(1, h.size()) * sizeof(T));
    if (e != cudaSuccess || h.empty()) return e;
    return cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

using cplx = std::complex<double>;

}  // namespace

struct fh_iterative {
    Discretized disc;
    LoopBasis loops;
    std::vector<double> resistances;
    int64_t n = 0, m = 0, p = 0, nloops = 0;
    fh_counts counts{};
    fh_timing timing{};
    GmresParams gp;
    PfftDevice op;
    cudaStream_t stream = nullptr;
    // Host blocks of M R M^T and M L M^T (column-major (m x p), (p x p)).
    std::vector<double> r_ep, l_ep, r_pp, l_pp, r_diag, l_diag;
    // Device: loop basis rows and its transpose over the internal loops.
    int64_t *d_row_ptr = nullptr, *d_t_off = nullptr;
    int32_t *d_branch = nullptr, *d_t_loop = nullptr;
    double *d_sign = nullptr, *d_t_sign = nullptr, *d_r = nullptr;
    double2 *d_c = nullptr, *d_drop = nullptr, *d_diag = nullptr, *d_b = nullptr, *d_x = nullptr;
    double *d_parts = nullptr, *d_flux = nullptr;
    // refinement of the FP32-convolution solves: residual, correction, product
    double2 *d_res = nullptr, *d_cor = nullptr, *d_ax = nullptr;
    GmresWork work;
    double operator_s = 0;
    // Currents (built on first use): segment / conductor layout, the loop
    // basis transposed over all loops, (w, h, R) per filament, outputs.
    ConductorLayout layout;
    int64_t *d_col_ptr = nullptr, *d_first = nullptr, *d_segi = nullptr;
    int32_t *d_col_loop = nullptr;
    double *d_col_sign = nullptr, *d_whr = nullptr, *d_ip = nullptr, *d_ib = nullptr, *d_dens = nullptr,
           *d_pow = nullptr, *d_segc = nullptr, *d_segp = nullptr, *d_segpk = nullptr;
    ~fh_iterative() {
        void *ptrs[] = {d_row_ptr, d_t_off, d_branch, d_t_loop, d_sign,  d_t_sign, d_r,    d_c,    d_drop,
                        d_diag,    d_b,     d_x,      d_parts,  d_flux,  d_res,    d_cor,  d_ax,   d_col_ptr,
                        d_first,   d_segi,  d_col_loop, d_col_sign, d_whr, d_ip,   d_ib,   d_dens, d_pow,
                        d_segc,    d_segp,  d_segpk};
        for (void *q : ptrs)
            if (q) cudaFree(q);
    }
};

namespace {

// r = b - y (refinement residual) and x += d (its correction).
__global__ void sub_kernel(const double2 *__restrict__ b, const double2 *__restrict__ y, double2 *__restrict__ r,
                           int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = make_double2(b[i].x - y[i].x, b[i].y - y[i].y);
}
__global__ void axpy_kernel(double2 *__restrict__ x, const double2 *__restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = make_double2(x[i].x + d[i].x, x[i].y + d[i].y);
}

// Z_ee x (f > 0: omega > 0) or M_e R M_e^T x (omega == 0).  full_precision:
// an operator with the FP32 grid convolution convolves in FP64.
fh_status apply_ee(fh_iterative *s, double omega, const double2 *x, double2 *y, fh_error_info *err,
                   bool full_precision = false) {
    const int64_t n = s->n;
    scatter_kernel<<<grid_n(n), 256, 0, s->stream>>>(x, s->d_t_off, s->d_t_loop, s->d_t_sign, s->d_c, n);
    FHB_CUDA(cudaGetLastError());
    const double *flux = nullptr;
    if (omega != 0.0) {
        split_kernel<<<grid_n(n), 256, 0, s->stream>>>(s->d_c, s->d_parts, n);
        FHB_CUDA(cudaGetLastError());
        fh_status st = pfft_apply(s->op, s->d_parts, s->d_flux, 2, err, full_precision);
        if (st) return st;
        flux = s->d_flux;
    }
    drop_kernel<<<grid_n(n), 256, 0, s->stream>>>(s->d_c, s->d_r, flux, omega, s->d_drop, n);
    gather_kernel<<<grid_n(s->m), 256, 0, s->stream>>>(s->d_drop, s->d_row_ptr, s->d_branch, s->d_sign, y, s->m);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

// sum_a sum_b s_a s_b L_ab over one loop, or the self terms alone for long
// loops (iterative.rs:516-536).  `self` per branch, `mutual` the loop's
// (k < l) pairs in row order.
double loop_inductance(const int32_t *br, size_t len, const double *self_l, const double *mutual, const double *sg) {
    double own = 0.0;
    for (size_t k = 0; k < len; ++k) own += self_l[br[k]];
    if (len > kExactDiagonalMaxLoop) return own;
    double mut = 0.0;
    size_t q = 0;
    for (size_t k = 0; k < len; ++k)
        for (size_t l = k + 1; l < len; ++l) mut += sg[k] * sg[l] * mutual[q++];
    return own + 2.0 * mut;
}

// GMRES with the FP32 grid convolution, refined against the FP64 operator:
// x = 0; repeat r = b - A x (FP64 convolution), stop when |r| <= tol |b|,
// else solve A d = r by GMRES with the FP32 convolution to a relative
// residual of max(tol, 1e-5) (about the FP32 product's own accuracy) and
// x += d.  The outcome counts all inner iterations and reports the FP64
// relative residual.
constexpr int kMaxRefinements = 12;
fh_status refined_solve(fh_iterative *s, double omega, const DeviceOp &apply, const DeviceOp &precondition,
                        double2 *x, GmresOutcome *out, fh_error_info *err) {
    const int64_t m = s->m;
    cudaStream_t cs = s->stream;
    if (!s->d_res) {
        FHB_CUDA(cudaMalloc(&s->d_res, sizeof(double2) * m));
        FHB_CUDA(cudaMalloc(&s->d_cor, sizeof(double2) * m));
        FHB_CUDA(cudaMalloc(&s->d_ax, sizeof(double2) * m));
    }
    std::vector<double2> hb((size_t)m), hr((size_t)m);
    FHB_CUDA(cudaMemcpyAsync(hb.data(), s->d_b, sizeof(double2) * m, cudaMemcpyDeviceToHost, cs));
    FHB_CUDA(cudaStreamSynchronize(cs));
    auto norm = [&](const std::vector<double2> &v) {
        double t = 0.0;
        for (const double2 &z : v) t += z.x * z.x + z.y * z.y;
        return std::sqrt(t);
    };
    const double bnorm = norm(hb);
    *out = GmresOutcome();
    if (bnorm == 0.0) {
        out->converged = true;
        return FH_OK;
    }
    GmresParams inner = s->gp;
    inner.tolerance = std::max(s->gp.tolerance, 1e-5);
    int64_t used = 0;
    for (int k = 0; k <= kMaxRefinements; ++k) {
        fh_status st = apply_ee(s, omega, x, s->d_ax, err, true);
        if (st) return st;
        sub_kernel<<<grid_n(m), 256, 0, cs>>>(s->d_b, s->d_ax, s->d_res, m);
        FHB_CUDA(cudaGetLastError());
        FHB_CUDA(cudaMemcpyAsync(hr.data(), s->d_res, sizeof(double2) * m, cudaMemcpyDeviceToHost, cs));
        FHB_CUDA(cudaStreamSynchronize(cs));
        const double rel = norm(hr) / bnorm;
        out->relative_residual = rel;
        out->iterations = used;
        if (rel <= s->gp.tolerance) {
            out->converged = true;
            return FH_OK;
        }
        if (k == kMaxRefinements || used >= s->gp.max_iterations) break;
        inner.max_iterations = (int)std::max<int64_t>(1, s->gp.max_iterations - used);
        FHB_CUDA(cudaMemsetAsync(s->d_cor, 0, sizeof(double2) * m, cs));
        GmresOutcome oc;
        st = gmres_solve(m, apply, precondition, s->d_res, s->d_cor, inner, cs, s->work, &oc, err);
        if (st) return st;
        used += oc.iterations;
        axpy_kernel<<<grid_n(m), 256, 0, cs>>>(x, s->d_cor, m);
        FHB_CUDA(cudaGetLastError());
    }
    out->converged = false;
    return FH_OK;
}

// Z_ee x = b for the right-hand side in s->d_b, x starting from zero: one
// Jacobi-preconditioned GMRES solve on the pFFT operator (iterative.rs:
// 269-288, 347-367), refined against the FP64 convolution when the operator
// convolves in FP32.
fh_status solve_ee(fh_iterative *s, double omega, double2 *x, GmresOutcome *oc, fh_error_info *err) {
    const int64_t m = s->m;
    cudaStream_t cs = s->stream;
    std::vector<double2> diag((size_t)m);
    for (int64_t i = 0; i < m; ++i) diag[i] = make_double2(s->r_diag[i], omega * s->l_diag[i]);
    FHB_CUDA(cudaMemcpyAsync(s->d_diag, diag.data(), sizeof(double2) * m, cudaMemcpyHostToDevice, cs));
    DeviceOp apply = [&](const double2 *in, double2 *out, fh_error_info *e) { return apply_ee(s, omega, in, out, e); };
    DeviceOp precondition = [&](const double2 *in, double2 *out, fh_error_info *e) {
        jacobi_kernel<<<grid_n(m), 256, 0, cs>>>(in, s->d_diag, out, m);
        cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess) return fail(e, FH_ERR_CUDA, std::string("jacobi: ") + cudaGetErrorString(ce));
        return FH_OK;
    };
    FHB_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * m, cs));
    fh_status st = s->op.fft_fp32 ? refined_solve(s, omega, apply, precondition, x, oc, err)
                                  : gmres_solve(m, apply, precondition, s->d_b, x, s->gp, cs, s->work, oc, err);
    // Also keeps `diag` alive until its copy has run.
    cudaError_t ce = cudaStreamSynchronize(cs);
    if (st) return st;
    FHB_CUDA(ce);
    return FH_OK;
}

// SolveError::NotConverged (iterative.rs:368-375) for the first failing solve.
fh_status not_converged(fh_error_info *err, double f, int64_t port, const GmresOutcome &oc) {
    fh_status e = fail(err, FH_ERR_NOT_CONVERGED,
                       "GMRES did not converge at " + std::to_string(f) + " Hz for port " + std::to_string(port) +
                           " after " + std::to_string(oc.iterations) + " iterations (relative residual " +
                           std::to_string(oc.relative_residual) + ")",
                       port, -1, f);
    if (err) {
        err->iterations = oc.iterations;
        err->residual = oc.relative_residual;
    }
    return e;
}

// Device buffers of the currents for one frequency, built on first use.
fh_status prepare_currents(fh_iterative *s, fh_error_info *err) {
    if (s->d_col_ptr) return FH_OK;
    cudaStream_t cs = s->stream;
    const int64_t n = s->n, p = s->p, nseg = (int64_t)s->layout.conductor_of_segment.size();
    TransposedLoops cols;
    transpose_loops(s->loops, n, s->nloops, cols);
    std::vector<double> whr((size_t)(3 * n));
    for (int64_t k = 0; k < n; ++k) {
        whr[(size_t)(3 * k)] = s->disc.filaments[(size_t)k].width;
        whr[(size_t)(3 * k + 1)] = s->disc.filaments[(size_t)k].height;
        whr[(size_t)(3 * k + 2)] = s->resistances[(size_t)k];
    }
    FHB_CUDA(put(&s->d_col_ptr, cols.offset, cs));
    FHB_CUDA(put(&s->d_col_loop, cols.loop, cs));
    FHB_CUDA(put(&s->d_col_sign, cols.sign, cs));
    FHB_CUDA(put(&s->d_whr, whr, cs));
    FHB_CUDA(put(&s->d_first, s->layout.segment_first, cs));
    auto alloc = [&](void **q, size_t bytes) { return cudaMalloc(q, std::max<size_t>(bytes, 16)); };
    if (alloc((void **)&s->d_ip, 16 * (size_t)p) || alloc((void **)&s->d_ib, 16 * (size_t)n) ||
        alloc((void **)&s->d_dens, 8 * (size_t)n) || alloc((void **)&s->d_pow, 8 * (size_t)n) ||
        alloc((void **)&s->d_segc, 16 * (size_t)nseg) || alloc((void **)&s->d_segp, 8 * (size_t)nseg) ||
        alloc((void **)&s->d_segpk, 8 * (size_t)nseg) || alloc((void **)&s->d_segi, 8 * (size_t)nseg)) {
        cudaGetLastError();
        return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation of the currents buffers failed");
    }
    FHB_CUDA(cudaStreamSynchronize(cs));
    return FH_OK;
}

}  // namespace

extern "C" {

void fh_gmres_default_params(fh_gmres_params *params) {
    if (!params) return;
    params->tolerance = 1e-10;
    params->restart = 100;
    params->max_iterations = 5000;
}

fh_status fh_iterative_create(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segments, size_t n_segments,
                              const fh_port *ports, size_t n_ports, const fh_discretization *disc,
                              const fh_pfft_params *pfft, const fh_gmres_params *gmres, fh_iterative **out,
                              fh_error_info *err) {
    clear_error(err);
    if (!out) return fail(err, FH_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (n_ports && !ports) return fail(err, FH_ERR_INVALID_ARGUMENT, "null ports");
    const double t0 = wall_s();
    std::unique_ptr<fh_iterative> s(new fh_iterative);
    fh_gmres_params g;
    fh_gmres_default_params(&g);
    if (gmres) g = *gmres;
    if (!(g.tolerance > 0.0) || g.restart < 1 || g.max_iterations < 0)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "GMRES tolerance must be positive and restart at least 1");
    s->gp.tolerance = g.tolerance;
    s->gp.restart = g.restart;
    s->gp.max_iterations = g.max_iterations;
    fh_pfft_params pp;
    fh_pfft_default_params(&pp);
    if (pfft) pp = *pfft;
    PfftConfig cfg;
    cfg.fixed_spacing = pp.spacing_kind == 1;
    cfg.cells_per_filament = pp.cells_per_filament;
    cfg.spacing = pp.spacing;
    cfg.near_field_radius = pp.near_field_radius;
    cfg.order = pp.interpolation_order;
    if (pp.fft_precision != 0 && pp.fft_precision != 1)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "fft_precision must be 0 (FP64) or 1 (FP32)");
    cfg.fft_fp32 = pp.fft_precision == 1;
    fh_status st = discretize_geometry(nodes, n_nodes, segments, n_segments, disc, s->disc, err);
    if (st) return st;
    st = build_loops(segments, n_segments, n_nodes, s->disc.per_segment.data(), ports, n_ports, s->loops, err);
    if (st) return st;
    st = ensure_device(err);
    if (st) return st;
    FHB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    cudaStream_t cs = s->stream;
    const int64_t n = (int64_t)s->disc.filaments.size();
    s->n = n;
    s->nloops = s->loops.rows();
    s->m = s->loops.internal;
    s->p = s->nloops - s->m;
    const int64_t m = s->m, p = s->p, L = s->nloops;
    for (const fh_filament &f : s->disc.filaments) s->resistances.push_back(f.length / (f.sigma * (f.width * f.height)));

    const double t_op = wall_s();
    st = pfft_build(s->disc.filaments.data(), n, cfg, cs, s->op, err);
    if (st) return st;
    s->operator_s = wall_s() - t_op;

    // Port columns: one operator product per port.
    const auto &rp = s->loops.row_ptr;
    const auto &br = s->loops.branch;
    const auto &sg = s->loops.sign;
    s->r_ep.assign((size_t)m * p, 0.0);
    s->l_ep.assign((size_t)m * p, 0.0);
    s->r_pp.assign((size_t)p * p, 0.0);
    s->l_pp.assign((size_t)p * p, 0.0);
    if (p > 0 && n > 0) {
        double *d_cur = nullptr, *d_fl = nullptr;
        FHB_CUDA(cudaMalloc(&d_cur, sizeof(double) * n));
        std::unique_ptr<void, decltype(&cudaFree)> g1(d_cur, &cudaFree);
        FHB_CUDA(cudaMalloc(&d_fl, sizeof(double) * n));
        std::unique_ptr<void, decltype(&cudaFree)> g2(d_fl, &cudaFree);
        std::vector<double> current((size_t)n), flux((size_t)n), drop((size_t)n);
        for (int64_t q = 0; q < p; ++q) {
            std::fill(current.begin(), current.end(), 0.0);
            for (int64_t k = rp[m + q]; k < rp[m + q + 1]; ++k) current[br[k]] += sg[k];
            FHB_CUDA(cudaMemcpyAsync(d_cur, current.data(), sizeof(double) * n, cudaMemcpyHostToDevice, cs));
            st = pfft_apply(s->op, d_cur, d_fl, 1, err);
            if (st) return st;
            FHB_CUDA(cudaMemcpyAsync(flux.data(), d_fl, sizeof(double) * n, cudaMemcpyDeviceToHost, cs));
            FHB_CUDA(cudaStreamSynchronize(cs));
            for (int64_t b = 0; b < n; ++b) drop[b] = current[b] * s->resistances[b];
            for (int64_t i = 0; i < L; ++i) {
                double rv = 0.0, lv = 0.0;
                for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
                    rv += drop[br[k]] * sg[k];
                    lv += flux[br[k]] * sg[k];
                }
                if (i < m) {
                    s->r_ep[i + q * m] = rv;
                    s->l_ep[i + q * m] = lv;
                } else {
                    s->r_pp[(i - m) + q * p] = rv;
                    s->l_pp[(i - m) + q * p] = lv;
                }
            }
        }
        // Symmetric in exact arithmetic; made so to the last bit (iterative.rs:199-200).
        std::vector<double> r2 = s->r_pp, l2 = s->l_pp;
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) {
                s->r_pp[a + b * p] = (r2[a + b * p] + r2[b + a * p]) * 0.5;
                s->l_pp[a + b * p] = (l2[a + b * p] + l2[b + a * p]) * 0.5;
            }
    }

    // Jacobi diagonal: self terms of every branch and the pairs of short loops.
    std::vector<int2> pairs;
    for (int64_t b = 0; b < n; ++b) pairs.push_back(make_int2((int)b, (int)b));
    for (int64_t i = 0; i < m; ++i) {
        const size_t len = (size_t)(rp[i + 1] - rp[i]);
        if (len > kExactDiagonalMaxLoop) continue;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
            for (int64_t l = k + 1; l < rp[i + 1]; ++l) pairs.push_back(make_int2(br[k], br[l]));
    }
    std::vector<double> values(pairs.size(), 0.0);
    if (!pairs.empty()) {
        std::vector<DevFil> hf((size_t)n);
        for (int64_t i = 0; i < n; ++i) hf[i] = make_devfil(s->disc.filaments[i]);
        DevFil *d_fil = nullptr;
        int2 *d_pairs = nullptr;
        double *d_vals = nullptr;
        FHB_CUDA(put(&d_fil, hf, cs));
        std::unique_ptr<void, decltype(&cudaFree)> g1(d_fil, &cudaFree);
        FHB_CUDA(put(&d_pairs, pairs, cs));
        std::unique_ptr<void, decltype(&cudaFree)> g2(d_pairs, &cudaFree);
        FHB_CUDA(cudaMalloc(&d_vals, sizeof(double) * pairs.size()));
        std::unique_ptr<void, decltype(&cudaFree)> g3(d_vals, &cudaFree);
        st = device_fill_pairs(d_fil, n, d_pairs, (int64_t)pairs.size(), d_vals, cs, nullptr, err);
        if (st) return st;
        FHB_CUDA(cudaMemcpyAsync(values.data(), d_vals, sizeof(double) * pairs.size(), cudaMemcpyDeviceToHost, cs));
        FHB_CUDA(cudaStreamSynchronize(cs));
    }
    s->r_diag.assign((size_t)m, 0.0);
    s->l_diag.assign((size_t)m, 0.0);
    size_t cursor = (size_t)n;
    for (int64_t i = 0; i < m; ++i) {
        const size_t len = (size_t)(rp[i + 1] - rp[i]);
        double r = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) r += s->resistances[br[k]];
        s->r_diag[i] = r;
        const double *mutual = values.data() + cursor;
        s->l_diag[i] = loop_inductance(&br[rp[i]], len, values.data(), mutual, &sg[rp[i]]);
        if (len <= kExactDiagonalMaxLoop) cursor += len * (len - 1) / 2;
    }

    // Device copies of the loop basis, its transpose over internal loops, R.
    TransposedLoops internal;
    transpose_loops(s->loops, n, m, internal);
    FHB_CUDA(put(&s->d_row_ptr, rp, cs));
    FHB_CUDA(put(&s->d_branch, br, cs));
    FHB_CUDA(put(&s->d_sign, sg, cs));
    FHB_CUDA(put(&s->d_t_off, internal.offset, cs));
    FHB_CUDA(put(&s->d_t_loop, internal.loop, cs));
    FHB_CUDA(put(&s->d_t_sign, internal.sign, cs));
    FHB_CUDA(put(&s->d_r, s->resistances, cs));
    auto alloc = [&](void **q, size_t bytes) { return cudaMalloc(q, std::max<size_t>(bytes, 16)); };
    if (alloc((void **)&s->d_c, sizeof(double2) * n) || alloc((void **)&s->d_drop, sizeof(double2) * n) ||
        alloc((void **)&s->d_diag, sizeof(double2) * m) || alloc((void **)&s->d_b, sizeof(double2) * m) ||
        alloc((void **)&s->d_x, sizeof(double2) * m * std::max<int64_t>(p, 1)) ||
        alloc((void **)&s->d_parts, sizeof(double) * 2 * n) || alloc((void **)&s->d_flux, sizeof(double) * 2 * n)) {
        cudaGetLastError();
        return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation of the iterative system failed");
    }
    FHB_CUDA(cudaStreamSynchronize(cs));
    conductor_layout(segments, n_segments, n_nodes, s->disc.per_segment.data(), s->layout);
    s->counts = fh_counts{(int64_t)n_nodes, (int64_t)n_segments, n, L, m, p};
    s->timing.inductance_s = s->operator_s;
    s->timing.assembly_s = wall_s() - t0;
    s->timing.total_s = s->timing.assembly_s;
    *out = s.release();
    return FH_OK;
}

fh_status fh_iterative_counts(const fh_iterative *s, fh_counts *out) {
    if (!s || !out) return FH_ERR_INVALID_ARGUMENT;
    *out = s->counts;
    return FH_OK;
}

fh_status fh_iterative_timing(const fh_iterative *s, fh_timing *out) {
    if (!s || !out) return FH_ERR_INVALID_ARGUMENT;
    *out = s->timing;
    return FH_OK;
}

fh_status fh_iterative_pfft_stats(const fh_iterative *s, fh_pfft_stats *out) {
    if (!s || !out) return FH_ERR_INVALID_ARGUMENT;
    const PfftDevice &d = s->op;
    out->filaments = d.n;
    out->grid_spacing = d.grid.spacing;
    for (int a = 0; a < 3; ++a) {
        out->grid_dims[a] = d.grid.dims[a];
        out->fft_dims[a] = d.padded[a];
    }
    out->projection_entries = d.projection_entries;
    out->near_entries = d.near_entries;
    out->memory_bytes = (int64_t)d.memory_bytes();
    out->setup_host_s = d.setup_host_s;
    out->setup_device_s = d.setup_device_s;
    return FH_OK;
}

fh_status fh_iterative_sweep(fh_iterative *s, const double *freqs, size_t nf, double *z_out,
                             fh_gmres_outcome *outcomes, fh_error_info *err) {
    clear_error(err);
    if (!s || (nf && (!freqs || !z_out))) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    for (size_t k = 0; k < nf; ++k)
        if (!(std::isfinite(freqs[k]) && freqs[k] >= 0.0))
            return fail(err, FH_ERR_INVALID_FREQUENCY,
                        "frequency " + std::to_string(k) + " is " + std::to_string(freqs[k]) +
                            " Hz; frequencies must be finite and non-negative",
                        (int64_t)k, -1, freqs[k]);
    const double t0 = wall_s();
    const int64_t m = s->m, p = s->p;
    cudaStream_t cs = s->stream;
    for (size_t fi = 0; fi < nf; ++fi) {
        const double f = freqs[fi];
        const double omega = f == 0.0 ? 0.0 : kTauI * f;
        std::vector<cplx> z((size_t)p * p);
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b)
                z[a + b * p] = cplx(s->r_pp[a + b * p], omega * s->l_pp[a + b * p]);
        if (m > 0) {
            std::vector<double2> rhs((size_t)m);
            std::vector<double2> xs((size_t)m * p);
            for (int64_t q = 0; q < p; ++q) {
                for (int64_t i = 0; i < m; ++i) rhs[i] = make_double2(s->r_ep[i + q * m], omega * s->l_ep[i + q * m]);
                FHB_CUDA(cudaMemcpyAsync(s->d_b, rhs.data(), sizeof(double2) * m, cudaMemcpyHostToDevice, cs));
                GmresOutcome oc;
                fh_status st = solve_ee(s, omega, s->d_x + q * m, &oc, err);
                if (st) return st;
                if (outcomes) {
                    outcomes[fi * p + q].iterations = oc.iterations;
                    outcomes[fi * p + q].relative_residual = oc.relative_residual;
                    outcomes[fi * p + q].converged = oc.converged ? 1 : 0;
                }
                if (!oc.converged) return not_converged(err, f, q, oc);
            }
            FHB_CUDA(cudaMemcpyAsync(xs.data(), s->d_x, sizeof(double2) * m * p, cudaMemcpyDeviceToHost, cs));
            FHB_CUDA(cudaStreamSynchronize(cs));
            // Z = Z_pp - Z_ep^T X (plain transpose: Z is complex symmetric).
            for (int64_t a = 0; a < p; ++a)
                for (int64_t b = 0; b < p; ++b) {
                    cplx acc(0.0, 0.0);
                    for (int64_t i = 0; i < m; ++i) {
                        const cplx ep(s->r_ep[i + a * m], omega * s->l_ep[i + a * m]);
                        const cplx xv(xs[i + b * m].x, xs[i + b * m].y);
                        acc += cplx(ep.real() * xv.real() - ep.imag() * xv.imag(),
                                    ep.real() * xv.imag() + ep.imag() * xv.real());
                    }
                    z[a + b * p] -= acc;
                }
        }
        // (Z + Z^T) / 2, then finiteness (iterative.rs:291-301).
        bool finite = true;
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = 0; b < p; ++b) {
                const cplx v = (z[a + b * p] + z[b + a * p]) * 0.5;
                finite = finite && std::isfinite(v.real()) && std::isfinite(v.imag());
                // Row-major output like impedance_ohm[k][a][b].
                z_out[2 * ((fi * p + a) * p + b)] = v.real();
                z_out[2 * ((fi * p + a) * p + b) + 1] = v.imag();
            }
        if (!finite)
            return fail(err, FH_ERR_SINGULAR, "the impedance at " + std::to_string(f) + " Hz is not finite", -1, -1, f);
    }
    s->timing.solve_s = wall_s() - t0;
    s->timing.total_s = s->timing.assembly_s + s->timing.solve_s;
    return FH_OK;
}

fh_status fh_iterative_filaments(const fh_iterative *s, fh_filament *out, size_t capacity) {
    if (!s || !out) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null argument");
    if (capacity < s->disc.filaments.size()) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "buffer too small");
    std::copy(s->disc.filaments.begin(), s->disc.filaments.end(), out);
    return FH_OK;
}

fh_status fh_iterative_layout(const fh_iterative *s, int64_t *segment_of_filament, int64_t *conductor_of_segment,
                              int64_t *conductor_count) {
    if (!s) return fail(nullptr, FH_ERR_INVALID_ARGUMENT, "null system");
    const ConductorLayout &l = s->layout;
    if (segment_of_filament) std::copy(l.segment_of_filament.begin(), l.segment_of_filament.end(), segment_of_filament);
    if (conductor_of_segment)
        std::copy(l.conductor_of_segment.begin(), l.conductor_of_segment.end(), conductor_of_segment);
    if (conductor_count) *conductor_count = l.conductors;
    return FH_OK;
}

// IterativeSystem::currents (iterative.rs:316-377 with solve.rs:1110-1149):
// per frequency one GMRES solve Z_ee x = Z_ep I_p, internal loop currents
// -x, port voltages V_p = Z_pp I_p + Z_ep^T I_e, then the same branch
// currents, densities, powers, segment sums and conductor peaks as the dense
// path.
fh_status fh_iterative_currents(fh_iterative *s, const double *freqs, size_t nf, const double *excitation,
                                size_t n_excitation, double *filament_current, double *current_density,
                                double *power_w, double *segment_current, double *segment_power_w,
                                int64_t *conductor_peak_filament, double *conductor_peak_density,
                                fh_power_balance *balance, fh_gmres_outcome *outcomes, fh_error_info *err) {
    clear_error(err);
    if (!s || (nf && !freqs) || (n_excitation && !excitation))
        return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    for (size_t k = 0; k < nf; ++k)
        if (!(std::isfinite(freqs[k]) && freqs[k] >= 0.0))
            return fail(err, FH_ERR_INVALID_FREQUENCY,
                        "frequency " + std::to_string(k) + " is " + std::to_string(freqs[k]) +
                            " Hz; frequencies must be finite and non-negative",
                        (int64_t)k, -1, freqs[k]);
    const int64_t n = s->n, m = s->m, p = s->p;
    const int64_t nseg = (int64_t)s->layout.conductor_of_segment.size(), ncond = s->layout.conductors;
    bool finite = (int64_t)n_excitation == p;
    for (size_t q = 0; q < 2 * n_excitation && finite; ++q) finite = std::isfinite(excitation[q]);
    if (!finite)
        return fail(err, FH_ERR_INVALID_EXCITATION,
                    "excitation must have one finite entry per port (" + std::to_string(p) + "), got " +
                        std::to_string(n_excitation) + " entries",
                    p, (int64_t)n_excitation);
    if (nf == 0) return FH_OK;
    fh_status st = prepare_currents(s, err);
    if (st) return st;
    cudaStream_t cs = s->stream;
    std::vector<cplx> ip((size_t)p);
    for (int64_t q = 0; q < p; ++q) ip[(size_t)q] = cplx(excitation[2 * q], excitation[2 * q + 1]);
    FHB_CUDA(cudaMemcpyAsync(s->d_ip, excitation, 16 * (size_t)p, cudaMemcpyHostToDevice, cs));
    std::vector<double2> rhs((size_t)m), x((size_t)m);
    std::vector<double> segp((size_t)nseg), segpk((size_t)nseg);
    std::vector<int64_t> segi((size_t)nseg);
    const double t0 = wall_s();
    for (size_t fi = 0; fi < nf; ++fi) {
        const double f = freqs[fi];
        const double omega = f == 0.0 ? 0.0 : kTauI * f;
        auto ep = [&](int64_t i, int64_t q) { return cplx(s->r_ep[i + q * m], omega * s->l_ep[i + q * m]); };
        GmresOutcome oc;
        oc.converged = true;
        if (m > 0) {
            for (int64_t i = 0; i < m; ++i) {
                cplx acc(0.0, 0.0);
                for (int64_t q = 0; q < p; ++q) acc += ep(i, q) * ip[(size_t)q];
                rhs[(size_t)i] = make_double2(acc.real(), acc.imag());
            }
            FHB_CUDA(cudaMemcpyAsync(s->d_b, rhs.data(), sizeof(double2) * m, cudaMemcpyHostToDevice, cs));
            st = solve_ee(s, omega, s->d_x, &oc, err);
            if (st) return st;
            if (outcomes) {
                outcomes[fi].iterations = oc.iterations;
                outcomes[fi].relative_residual = oc.relative_residual;
                outcomes[fi].converged = oc.converged ? 1 : 0;
            }
            if (!oc.converged) return not_converged(err, f, 0, oc);
        } else if (outcomes) {
            outcomes[fi] = fh_gmres_outcome{0, 0.0, 1};
        }
        st = launch_currents(reinterpret_cast<const double *>(s->d_x), s->d_ip, m, (int)p, true, n, 1, s->d_col_ptr,
                             s->d_col_loop, s->d_col_sign, s->d_whr, s->d_first, nseg, s->d_ib, s->d_dens, s->d_pow,
                             s->d_segc, s->d_segp, s->d_segpk, s->d_segi, cs, err);
        if (st) return st;
        if (m > 0) FHB_CUDA(cudaMemcpyAsync(x.data(), s->d_x, sizeof(double2) * m, cudaMemcpyDeviceToHost, cs));
        FHB_CUDA(cudaMemcpyAsync(segp.data(), s->d_segp, 8 * (size_t)nseg, cudaMemcpyDeviceToHost, cs));
        FHB_CUDA(cudaMemcpyAsync(segpk.data(), s->d_segpk, 8 * (size_t)nseg, cudaMemcpyDeviceToHost, cs));
        FHB_CUDA(cudaMemcpyAsync(segi.data(), s->d_segi, 8 * (size_t)nseg, cudaMemcpyDeviceToHost, cs));
        if (filament_current)
            FHB_CUDA(cudaMemcpyAsync(filament_current + 2 * fi * n, s->d_ib, 16 * (size_t)n, cudaMemcpyDeviceToHost, cs));
        if (current_density)
            FHB_CUDA(cudaMemcpyAsync(current_density + fi * n, s->d_dens, 8 * (size_t)n, cudaMemcpyDeviceToHost, cs));
        if (power_w) FHB_CUDA(cudaMemcpyAsync(power_w + fi * n, s->d_pow, 8 * (size_t)n, cudaMemcpyDeviceToHost, cs));
        if (segment_current)
            FHB_CUDA(cudaMemcpyAsync(segment_current + 2 * fi * nseg, s->d_segc, 16 * (size_t)nseg,
                                     cudaMemcpyDeviceToHost, cs));
        FHB_CUDA(cudaStreamSynchronize(cs));
        // V_p = Z_pp I_p + Z_ep^T I_e with I_e = -x (solve.rs:1128).
        bool ok = true;
        std::vector<cplx> v((size_t)p);
        for (int64_t a = 0; a < p; ++a) {
            cplx acc(0.0, 0.0);
            for (int64_t b = 0; b < p; ++b)
                acc += cplx(s->r_pp[a + b * p], omega * s->l_pp[a + b * p]) * ip[(size_t)b];
            for (int64_t i = 0; i < m; ++i) acc -= ep(i, a) * cplx(x[(size_t)i].x, x[(size_t)i].y);
            v[(size_t)a] = acc;
            ok = ok && std::isfinite(acc.real()) && std::isfinite(acc.imag());
        }
        for (int64_t i = 0; i < m && ok; ++i) ok = std::isfinite(x[(size_t)i].x) && std::isfinite(x[(size_t)i].y);
        if (!ok)
            return fail(err, FH_ERR_SINGULAR, "the currents at " + std::to_string(f) + " Hz are not finite",
                        (int64_t)fi, -1, f);
        if (segment_power_w) std::copy(segp.begin(), segp.end(), segment_power_w + fi * nseg);
        // Conductor peaks: segments are contiguous in filament order, so the
        // first strictly larger segment peak is the first filament of
        // largest |J|.
        std::vector<double> best((size_t)ncond, -1.0);
        std::vector<int64_t> at((size_t)ncond, -1);
        double dissipated = 0.0;
        for (int64_t g = 0; g < nseg; ++g) {
            dissipated += segp[(size_t)g];
            const int64_t c = s->layout.conductor_of_segment[(size_t)g];
            if (segi[(size_t)g] >= 0 && (at[(size_t)c] < 0 || segpk[(size_t)g] > best[(size_t)c])) {
                best[(size_t)c] = segpk[(size_t)g];
                at[(size_t)c] = segi[(size_t)g];
            }
        }
        if (conductor_peak_filament) std::copy(at.begin(), at.end(), conductor_peak_filament + fi * ncond);
        if (conductor_peak_density) std::copy(best.begin(), best.end(), conductor_peak_density + fi * ncond);
        if (balance) {
            double input = 0.0;
            for (int64_t a = 0; a < p; ++a) input += (std::conj(ip[(size_t)a]) * v[(size_t)a]).real();
            input *= 0.5;
            const double scale = std::max(dissipated, input);
            balance[fi] = fh_power_balance{dissipated, input, scale > 0.0 ? std::fabs(dissipated - input) / scale : 0.0};
        }
    }
    s->timing.solve_s = wall_s() - t0;
    return FH_OK;
}

void fh_iterative_destroy(fh_iterative *s) {
    if (!s) return;
    cudaStream_t cs = s->stream;
    delete s;
    if (cs) cudaStreamDestroy(cs);
}

fh_status fh_test_gmres_dense(const double *a, size_t n, const double *b, double *x, const double *precond,
                              const fh_gmres_params *params, fh_gmres_outcome *outcome, fh_error_info *err) {
    clear_error(err);
    if (!a || !b || !x || !params) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    fh_status st = ensure_device(err);
    if (st) return st;
    cudaStream_t cs;
    FHB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, decltype(&cudaStreamDestroy)> sg(cs, &cudaStreamDestroy);
    double2 *d_a = nullptr, *d_m = nullptr, *d_b = nullptr, *d_x = nullptr;
    FHB_CUDA(cudaMalloc(&d_a, sizeof(double2) * n * n));
    std::unique_ptr<void, decltype(&cudaFree)> g1(d_a, &cudaFree);
    FHB_CUDA(cudaMalloc(&d_m, sizeof(double2) * n * n));
    std::unique_ptr<void, decltype(&cudaFree)> g2(d_m, &cudaFree);
    FHB_CUDA(cudaMalloc(&d_b, sizeof(double2) * n));
    std::unique_ptr<void, decltype(&cudaFree)> g3(d_b, &cudaFree);
    FHB_CUDA(cudaMalloc(&d_x, sizeof(double2) * n));
    std::unique_ptr<void, decltype(&cudaFree)> g4(d_x, &cudaFree);
    FHB_CUDA(cudaMemcpyAsync(d_a, a, sizeof(double2) * n * n, cudaMemcpyHostToDevice, cs));
    if (precond) FHB_CUDA(cudaMemcpyAsync(d_m, precond, sizeof(double2) * n * n, cudaMemcpyHostToDevice, cs));
    FHB_CUDA(cudaMemcpyAsync(d_b, b, sizeof(double2) * n, cudaMemcpyHostToDevice, cs));
    FHB_CUDA(cudaMemcpyAsync(d_x, x, sizeof(double2) * n, cudaMemcpyHostToDevice, cs));
    const int64_t nn = (int64_t)n;
    DeviceOp apply = [&](const double2 *in, double2 *out, fh_error_info *) {
        dense_matvec_kernel<<<grid_n(nn), 256, 0, cs>>>(d_a, in, out, nn);
        return FH_OK;
    };
    DeviceOp pre = [&](const double2 *in, double2 *out, fh_error_info *) {
        if (precond)
            dense_matvec_kernel<<<grid_n(nn), 256, 0, cs>>>(d_m, in, out, nn);
        else
            cudaMemcpyAsync(out, in, sizeof(double2) * nn, cudaMemcpyDeviceToDevice, cs);
        return FH_OK;
    };
    GmresParams gp;
    gp.tolerance = params->tolerance;
    gp.restart = params->restart;
    gp.max_iterations = params->max_iterations;
    GmresWork work;
    GmresOutcome oc;
    st = gmres_solve(nn, apply, pre, d_b, d_x, gp, cs, work, &oc, err);
    if (st) return st;
    FHB_CUDA(cudaMemcpyAsync(x, d_x, sizeof(double2) * n, cudaMemcpyDeviceToHost, cs));
    FHB_CUDA(cudaStreamSynchronize(cs));
    if (outcome) {
        outcome->iterations = oc.iterations;
        outcome->relative_residual = oc.relative_residual;
        outcome->converged = oc.converged ? 1 : 0;
    }
    return FH_OK;
}

}  // extern "C"
