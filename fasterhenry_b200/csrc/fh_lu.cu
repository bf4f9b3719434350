// Batched blocked right-looking complex LU with partial pivoting.
//
// The algorithm is the reference's (fasterhenry/src/dense.rs:43-190: PA = LU,
// pivot = first row of largest |re| + |im|, multipliers scaled by the
// reciprocal of the pivot, zero pivot -> Singular), re-arranged for the GPU:
//
//   * every launch works on all frequencies of a sweep at once (grid.y /
//     grid.z = matrix index), so one panel step is a handful of launches for
//     the whole batch instead of one factorization per thread;
//   * per panel column: a pivot search (one block per row chunk, the last
//     block to finish reduces the partials and swaps the rows inside the
//     panel) and a fused scale + rank-1 update of the panel;
//   * after the panel: row interchanges of the trailing columns, a TRSM for
//     U12 and the GEMM A22 -= L21 U12.  The GEMM is FP64 SIMT here (the FP64
//     form) or split-BF16 x3 on the tensor cores (fh_gemm_tc.cu, FP32 form).
//   * interchanges are never applied to the columns left of the panel: the
//     forward substitution applies each panel's interchanges to the
//     right-hand side just before that panel's L columns are used, which is
//     the same elimination order.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdio>

#include "fh_cx.cuh"
#include "fh_lu.cuh"

namespace fhb {

namespace {

// ---------------------------------------------------------------------------
// Pivot search for column j (rows j..m-1) of every matrix.  The last block of
// a matrix to finish reduces the partials, records the pivot, flags a zero
// pivot and swaps rows j and pivot across the panel's columns.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) pivot_kernel(Cx<T> *__restrict__ a, int64_t m, int j, int k0, int ncols,
                                                    int *__restrict__ pivots, int *__restrict__ singular,
                                                    double *__restrict__ pval, int *__restrict__ pidx,
                                                    unsigned *__restrict__ tickets, int chunks) {
    const int f = blockIdx.y;
    Cx<T> *A = a + (int64_t)f * m * m;
    double best = -1.0;
    int bi = INT_MAX;
    for (int64_t r = j + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
        Cx<T> v = A[r + (int64_t)j * m];
        const double n1 = (double)(fabs(v.re) + fabs(v.im));  // |re| + |im| in T
        if (n1 > best || (n1 == best && r < bi)) {
            best = n1;
            bi = (int)r;
        }
    }
    auto better = [](double v2, int i2, double v1, int i1) { return v2 > v1 || (v2 == v1 && i2 < i1); };
    for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_down_sync(0xffffffffu, best, o);
        int i2 = __shfl_down_sync(0xffffffffu, bi, o);
        if (better(v2, i2, best, bi)) {
            best = v2;
            bi = i2;
        }
    }
    __shared__ double sv[8];
    __shared__ int si[8];
    __shared__ bool s_last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sv[warp] = best;
        si[warp] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
            if (better(sv[w], si[w], best, bi)) {
                best = sv[w];
                bi = si[w];
            }
        pval[f * chunks + blockIdx.x] = best;
        pidx[f * chunks + blockIdx.x] = bi;
        __threadfence();
        unsigned ticket = atomicAdd(&tickets[f], 1u);
        s_last = ticket == (unsigned)(chunks - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __shared__ int s_piv;
    if (threadIdx.x == 0) {
        __threadfence();
        double b = -1.0;
        int i = INT_MAX;
        for (int c = 0; c < chunks; ++c) {
            double v2 = ((volatile double *)pval)[f * chunks + c];
            int i2 = ((volatile int *)pidx)[f * chunks + c];
            if (better(v2, i2, b, i)) {
                b = v2;
                i = i2;
            }
        }
        int p = j;
        if (b == 0.0) singular[f] = 1;  // exactly zero pivot (dense.rs:166-168)
        else if (b > 0.0) p = i;       // all-NaN column: keep the diagonal
        pivots[(int64_t)f * m + j] = p;
        tickets[f] = 0;
        s_piv = p;
    }
    __syncthreads();
    const int p = s_piv;
    if (p != j)
        for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
            Cx<T> *col = A + (int64_t)(k0 + c) * m;
            Cx<T> t = col[j];
            col[j] = col[p];
            col[p] = t;
        }
}

// Scale column j below the pivot by 1/pivot and apply the rank-1 update to
// the panel columns j+1 .. k0+ncols-1 (dense.rs:176-186).
template <class T>
__global__ void __launch_bounds__(256) panel_update_kernel(Cx<T> *__restrict__ a, int64_t m, int j, int k0, int ncols) {
    const int f = blockIdx.y;
    Cx<T> *A = a + (int64_t)f * m * m;
    __shared__ Cx<T> prow[128];
    const int rest = k0 + ncols - j;  // columns j .. k0+ncols-1
    for (int c = threadIdx.x; c < rest; c += blockDim.x) prow[c] = A[j + (int64_t)(j + c) * m];
    __syncthreads();
    const Cx<T> one{(T)1, (T)0};
    const Cx<T> inv = cdiv(one, prow[0]);
    for (int64_t i = j + 1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        Cx<T> l = cmul(A[i + (int64_t)j * m], inv);
        A[i + (int64_t)j * m] = l;
        for (int c = 1; c < rest; ++c) {
            Cx<T> y = A[i + (int64_t)(j + c) * m];
            csubmul(y, prow[c], l);
            A[i + (int64_t)(j + c) * m] = y;
        }
    }
}

// Row interchanges of rows [k0, k0+nb), in order, applied to columns [c0, c1).
template <class T>
__global__ void __launch_bounds__(256) swap_kernel(Cx<T> *__restrict__ a, int64_t m, int k0, int nb, int64_t c0,
                                                   int64_t c1, const int *__restrict__ pivots) {
    const int f = blockIdx.y;
    Cx<T> *A = a + (int64_t)f * m * m;
    const int *piv = pivots + (int64_t)f * m;
    for (int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += (int64_t)gridDim.x * blockDim.x) {
        Cx<T> *col = A + c * m;
        for (int jj = 0; jj < nb; ++jj) {
            int p = piv[k0 + jj];
            if (p != k0 + jj) {
                Cx<T> t = col[k0 + jj];
                col[k0 + jj] = col[p];
                col[p] = t;
            }
        }
    }
}

// U12 = L11^{-1} A12 for columns [k0+nb, m): 64 columns per block, L11 and
// the block's columns staged in shared memory.
template <class T>
__global__ void __launch_bounds__(64) trsm_kernel(Cx<T> *__restrict__ a, int64_t m, int k0, int nb) {
    extern __shared__ unsigned char smem_raw[];
    Cx<T> *Ls = reinterpret_cast<Cx<T> *>(smem_raw);  // [nb][nb] (row r, col k) at r*nb + k
    Cx<T> *Bs = Ls + nb * nb;                          // [nb][64]
    const int f = blockIdx.y;
    Cx<T> *A = a + (int64_t)f * m * m;
    const int64_t c0 = (int64_t)k0 + nb + (int64_t)blockIdx.x * 64;
    for (int idx = threadIdx.x; idx < nb * nb; idx += 64) {
        int r = idx % nb, k = idx / nb;
        Ls[r * nb + k] = A[(k0 + r) + (int64_t)(k0 + k) * m];
    }
    const int64_t col = c0 + threadIdx.x;
    for (int idx = threadIdx.x; idx < nb * 64; idx += 64) {
        int r = idx % nb, cc = idx / nb;
        int64_t c = c0 + cc;
        Bs[r * 64 + cc] = c < m ? A[(k0 + r) + c * m] : Cx<T>{0, 0};
    }
    __syncthreads();
    if (col < m) {
        for (int k = 0; k < nb; ++k) {
            Cx<T> xk = Bs[k * 64 + threadIdx.x];
            for (int r = k + 1; r < nb; ++r) {
                Cx<T> y = Bs[r * 64 + threadIdx.x];
                csubmul(y, xk, Ls[r * nb + k]);
                Bs[r * 64 + threadIdx.x] = y;
            }
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nb * 64; idx += 64) {
        int r = idx % nb, cc = idx / nb;
        int64_t c = c0 + cc;
        if (c < m) A[(k0 + r) + c * m] = Bs[r * 64 + cc];
    }
}

// A22 -= L21 U12 (SIMT).  Tile 64 x 64, K = nb <= 64; 256 threads, each a
// 4 x 4 block of outputs interleaved with stride 16.
template <class T>
__global__ void __launch_bounds__(256) gemm_update_kernel(Cx<T> *__restrict__ a, int64_t m, int k0, int nb) {
    extern __shared__ unsigned char smem_raw[];
    Cx<T> *Ls = reinterpret_cast<Cx<T> *>(smem_raw);  // [nb][64]  Ls[k*64 + i]
    Cx<T> *Us = Ls + nb * 64;                          // [nb][64]  Us[k*64 + j]
    const int f = blockIdx.z;
    Cx<T> *A = a + (int64_t)f * m * m;
    const int64_t base = (int64_t)k0 + nb;
    const int64_t i0 = base + (int64_t)blockIdx.y * 64, j0 = base + (int64_t)blockIdx.x * 64;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < nb * 64; idx += 256) {
        int ii = idx % 64, k = idx / 64;
        int64_t row = i0 + ii;
        Ls[k * 64 + ii] = row < m ? A[row + (int64_t)(k0 + k) * m] : Cx<T>{0, 0};
        int kk = idx % nb, jj = idx / nb;
        int64_t col = j0 + jj;
        Us[kk * 64 + jj] = col < m ? A[(k0 + kk) + col * m] : Cx<T>{0, 0};
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;
    T accr[4][4], acci[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) accr[r][c] = acci[r][c] = (T)0;
    for (int k = 0; k < nb; ++k) {
        Cx<T> l[4], u[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) l[r] = Ls[k * 64 + tx + 16 * r];
#pragma unroll
        for (int c = 0; c < 4; ++c) u[c] = Us[k * 64 + ty + 16 * c];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                accr[r][c] += l[r].re * u[c].re - l[r].im * u[c].im;
                acci[r][c] += l[r].re * u[c].im + l[r].im * u[c].re;
            }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        int64_t col = j0 + ty + 16 * c;
        if (col >= m) continue;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            int64_t row = i0 + tx + 16 * r;
            if (row >= m) continue;
            Cx<T> y = A[row + col * m];
            y.re -= accr[r][c];
            y.im -= acci[r][c];
            A[row + col * m] = y;
        }
    }
}

// ---------------------------------------------------------------------------
// Solves.  x: count x nrhs columns of length m (matrix f, rhs q at
// x + (f*nrhs + q)*m).
// ---------------------------------------------------------------------------
// Forward, one panel: apply the panel's interchanges, then L11 (unit).
// L11 and the touched entries of x are staged in shared memory; the
// interchanges run in order on one thread but only touch shared memory (an
// interchange with a row below the panel uses the value of that row
// preloaded in parallel, indexed by its first occurrence in the pivot list).
// With pivots == nullptr the interchanges were applied by fwd_swap_kernel.
// Dynamic shared memory: nb*nb complex + 3*nb complex + 2*nb ints.
template <class T>
__global__ void __launch_bounds__(128) fwd_panel_kernel(const Cx<T> *__restrict__ a, int64_t m, int nrhs, int k0,
                                                        int nb, const int *__restrict__ pivots,
                                                        Cx<T> *__restrict__ x) {
    extern __shared__ unsigned char smem_raw[];
    Cx<T> *Ls = reinterpret_cast<Cx<T> *>(smem_raw);  // Ls[r * nb + k]
    Cx<T> *xs = Ls + nb * nb;
    Cx<T> *ext = xs + nb;
    int *piv = reinterpret_cast<int *>(ext + nb);
    int *first = piv + nb;
    const int f = blockIdx.x / nrhs;
    const Cx<T> *A = a + (int64_t)f * m * m;
    Cx<T> *X = x + (int64_t)blockIdx.x * m;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < nb * nb; idx += blockDim.x) {
        const int r = idx % nb, k = idx / nb;
        Ls[r * nb + k] = A[(k0 + r) + (int64_t)(k0 + k) * m];
    }
    for (int t = tid; t < nb; t += blockDim.x) {
        xs[t] = X[k0 + t];
        if (pivots) piv[t] = pivots[(int64_t)f * m + k0 + t];
    }
    __syncthreads();
    if (pivots) {
        for (int t = tid; t < nb; t += blockDim.x) {
            const int p = piv[t];
            int fst = t;
            if (p >= k0 + nb) {
                for (int q = 0; q < t; ++q)
                    if (piv[q] == p) {
                        fst = q;
                        break;
                    }
                if (fst == t) ext[t] = X[p];
            }
            first[t] = fst;
        }
        __syncthreads();
        if (tid == 0) {
            for (int jj = 0; jj < nb; ++jj) {
                const int p = piv[jj];
                if (p == k0 + jj) continue;
                Cx<T> &other = p < k0 + nb ? xs[p - k0] : ext[first[jj]];
                const Cx<T> tmp = xs[jj];
                xs[jj] = other;
                other = tmp;
            }
        }
        __syncthreads();
        for (int t = tid; t < nb; t += blockDim.x)
            if (piv[t] >= k0 + nb && first[t] == t) X[piv[t]] = ext[t];
    }
    for (int k = 0; k < nb; ++k) {
        const Cx<T> xk = xs[k];
        for (int r = k + 1 + tid; r < nb; r += blockDim.x) {
            Cx<T> y = xs[r];
            csubmul(y, xk, Ls[r * nb + k]);
            xs[r] = y;
        }
        __syncthreads();
    }
    for (int r = tid; r < nb; r += blockDim.x) X[k0 + r] = xs[r];
}

// Forward, interchanges only: rows [g0, g0+wg) of a swap group, applied in
// order to x, with the same shared-memory staging as fwd_panel_kernel.
// Dynamic shared memory: 2*wg complex + 2*wg ints.
template <class T>
__global__ void __launch_bounds__(128) fwd_swap_kernel(int64_t m, int nrhs, int g0, int wg,
                                                       const int *__restrict__ pivots, Cx<T> *__restrict__ x) {
    extern __shared__ unsigned char smem_raw[];
    Cx<T> *xs = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *ext = xs + wg;
    int *piv = reinterpret_cast<int *>(ext + wg);
    int *first = piv + wg;
    const int f = blockIdx.x / nrhs;
    Cx<T> *X = x + (int64_t)blockIdx.x * m;
    const int tid = threadIdx.x;
    for (int t = tid; t < wg; t += blockDim.x) {
        xs[t] = X[g0 + t];
        piv[t] = pivots[(int64_t)f * m + g0 + t];
    }
    __syncthreads();
    for (int t = tid; t < wg; t += blockDim.x) {
        const int p = piv[t];
        int fst = t;
        if (p >= g0 + wg) {
            for (int q = 0; q < t; ++q)
                if (piv[q] == p) {
                    fst = q;
                    break;
                }
            if (fst == t) ext[t] = X[p];
        }
        first[t] = fst;
    }
    __syncthreads();
    if (tid == 0) {
        for (int jj = 0; jj < wg; ++jj) {
            const int p = piv[jj];
            if (p == g0 + jj) continue;
            Cx<T> &other = p < g0 + wg ? xs[p - g0] : ext[first[jj]];
            const Cx<T> tmp = xs[jj];
            xs[jj] = other;
            other = tmp;
        }
    }
    __syncthreads();
    for (int t = tid; t < wg; t += blockDim.x) {
        if (piv[t] >= g0 + wg && first[t] == t) X[piv[t]] = ext[t];
        X[g0 + t] = xs[t];
    }
}

// Backward, one panel: U11 (non-unit upper), staged in shared memory.
template <class T>
__global__ void __launch_bounds__(128) bwd_panel_kernel2(const Cx<T> *__restrict__ a, int64_t m, int nrhs, int k0,
                                                         int nb, Cx<T> *__restrict__ x) {
    extern __shared__ unsigned char smem_raw[];
    Cx<T> *Us = reinterpret_cast<Cx<T> *>(smem_raw);  // Us[r * nb + k]
    Cx<T> *xs = Us + nb * nb;
    const int f = blockIdx.x / nrhs;
    const Cx<T> *A = a + (int64_t)f * m * m;
    Cx<T> *X = x + (int64_t)blockIdx.x * m;
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        const int r = idx % nb, k = idx / nb;
        Us[r * nb + k] = A[(k0 + r) + (int64_t)(k0 + k) * m];
    }
    for (int r = threadIdx.x; r < nb; r += blockDim.x) xs[r] = X[k0 + r];
    __syncthreads();
    for (int k = nb - 1; k >= 0; --k) {
        if (threadIdx.x == 0) xs[k] = cdiv(xs[k], Us[k * nb + k]);
        __syncthreads();
        const Cx<T> xk = xs[k];
        for (int r = threadIdx.x; r < k; r += blockDim.x) {
            Cx<T> y = xs[r];
            csubmul(y, xk, Us[r * nb + k]);
            xs[r] = y;
        }
        __syncthreads();
    }
    for (int r = threadIdx.x; r < nb; r += blockDim.x) X[k0 + r] = xs[r];
}

// The diagonal block of a factorization without pivoting, in one CTA per
// matrix: the LU of the nb x nb block at (k0, k0) in place (L unit lower below
// the diagonal, U on and above it), then L^{-1} into linv and U^{-1} into
// uinv (matrix f at + f * mstride, column-major with leading dimension nb);
// optionally U^{-1} also into x2 (matrix f at + f * stride2, leading dimension
// ld2) and the diagonal of U into dv (matrix f at + f * dstride).
// For A = R + jwL with R and L symmetric positive definite (a mesh impedance
// matrix) elimination without pivoting is stable (the growth factor is
// bounded); a zero or non-finite pivot of any other matrix shows as a
// non-finite refinement correction, and the caller falls back to the pivoted
// FP64 factorization.
//
// Each of the 512 threads keeps 32 entries in registers: rows lane + 32 i
// (i < 4) of columns warp + 16 j (j < 8), so a column belongs to one warp and a
// row to one lane of every warp.  Step k of the elimination reads column k
// and row k of the block as step k - 1 left them; the owners write those
// entries to a shared double buffer right after their own update of step
// k - 1 (with the reciprocal of the next pivot), so a step costs one barrier.
// The LU is one kernel (diag_lu_kernel); the two inverses, which need only
// the factors, run as two CTAs per matrix of a second (diag_inv_kernel).
// The steps run in eight segments of 16 (a template per segment): inside one,
// the row group and the column slot of k are constants, so the row groups and
// column slots a step does not touch are left out at compile time and every
// register index is a constant.  The inverses run in the same registers with
// the factors kept in shared memory: X = L^{-1} by forward elimination on the
// rows of I (row k of X is final before step k), Y = U^{-1} backward (row k
// scaled by 1 / U_kk at step k, every thread scaling the published row).
constexpr int kDiagThreads = 512;
constexpr int kDiagSmemExtra = 2 * 128 + 2 * 128 + 128 + 2;  // complex entries besides the nb x nb factors
using Cf = Cx<float>;

// y -= f x as four fused multiply-adds.
__device__ __forceinline__ void cfms(Cf &y, Cf f, Cf x) {
    y.re = fmaf(-f.re, x.re, y.re);
    y.re = fmaf(f.im, x.im, y.re);
    y.im = fmaf(-f.re, x.im, y.im);
    y.im = fmaf(-f.im, x.re, y.im);
}
// 1 / p = conj(p) / |p|^2 with one reciprocal.
__device__ __forceinline__ Cf crcp(Cf p) {
    const float s = __frcp_rn(p.re * p.re + p.im * p.im);
    return Cf{p.re * s, -p.im * s};
}

struct DiagSmem {
    Cf *S;     // the factors, column-major, ld nb
    Cf *colb;  // [2][128]
    Cf *rowb;  // [2][128], column c of a row at (c % 16) * 8 + c / 16 (diag_row_slot)
    Cf *dinv;  // [128]: 1 / U_kk
    Cf *pinv;  // [2]: 1 / pivot of the step
};

// Position of column c in a row buffer: the 8 columns a thread owns (warp +
// 16 j) are adjacent, so a row's owner lane writes them with four 16-byte
// stores and the readers of a column slot read one broadcast address.
__device__ __forceinline__ int diag_row_slot(int c) { return (c & 15) * 8 + (c >> 4); }

// Row group I of a lane's registers into its 8 slots of the row buffer rn.
template <int I>
__device__ __forceinline__ void diag_store_row(const Cf (&v)[4][8], int warp, Cf *rn) {
    float4 *d = reinterpret_cast<float4 *>(rn + warp * 8);
#pragma unroll
    for (int q = 0; q < 4; ++q) d[q] = make_float4(v[I][2 * q].re, v[I][2 * q].im, v[I][2 * q + 1].re, v[I][2 * q + 1].im);
}

// Column k1 (slot J, rows >= k1) and row k1 (group I) of the block into cn /
// rn, and 1 / a(k1, k1) into *pn.  The row is written whole: its columns
// < k1 are never read.
template <int J, int I>
__device__ __forceinline__ void diag_publish(const Cf (&v)[4][8], int k1, int nb, int lane, int warp, Cf *cn, Cf *rn,
                                             Cf *pn) {
    if (warp == (k1 & 15)) {
#pragma unroll
        for (int i = I; i < 4; ++i) {
            const int r = lane + 32 * i;
            if (r >= k1 && r < nb) cn[r] = v[i][J];
        }
    }
    if (lane == (k1 & 31)) {
        diag_store_row<I>(v, warp, rn);
        if (warp == (k1 & 15)) *pn = crcp(v[I][J]);
    }
}

// LU steps k in [16 JS, 16 JS + 16):  l_r = a_rk / a_kk,  a_rc -= l_r a_kc  (r, c > k).
template <int JS>
__device__ __forceinline__ void diag_lu_segment(Cf (&v)[4][8], int nb, int lane, int warp, const DiagSmem &sm) {
    constexpr int IS = JS / 2;  // row group of k
    const Cf zero{0.f, 0.f};
#pragma unroll 1
    for (int kk = 0; kk < 16; ++kk) {
        const int k = 16 * JS + kk;
        if (k >= nb) return;  // uniform
        const int b = k & 1, k1 = k + 1;
        const Cf inv = sm.pinv[b];
        Cf l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            l[i] = zero;
            const int r = lane + 32 * i;
            if (i >= IS && (i > IS || r > k) && r < nb) l[i] = cmul(sm.colb[b * 128 + r], inv);
        }
#pragma unroll
        for (int j = JS; j < 8; ++j) {
            const int c = warp + 16 * j;
            if (j == JS && warp <= kk) {
                if (warp == kk) {  // column k takes the multipliers
#pragma unroll
                    for (int i = IS; i < 4; ++i)
                        if (i > IS || lane + 32 * i > k) v[i][j] = l[i];
                }
                continue;
            }
            if (c >= nb) continue;
            const Cf u = sm.rowb[b * 128 + warp * 8 + j];
#pragma unroll
            for (int i = IS; i < 4; ++i) cfms(v[i][j], l[i], u);  // l = 0 on rows <= k
        }
        if (k1 < nb) {
            Cf *cn = sm.colb + (b ^ 1) * 128, *rn = sm.rowb + (b ^ 1) * 128;
            if (kk < 15) {
                diag_publish<JS, IS>(v, k1, nb, lane, warp, cn, rn, sm.pinv + (b ^ 1));
            } else if constexpr (JS < 7) {
                diag_publish<JS + 1, (JS + 1) / 2>(v, k1, nb, lane, warp, cn, rn, sm.pinv + (b ^ 1));
            }
        }
        __syncthreads();
    }
}

// Row k + 1 (group I) of X into rn: its owner's registers hold the whole
// row (columns <= k as step k left them, 1 at k + 1, zeros after).
template <int I>
__device__ __forceinline__ void diag_publish_xrow(const Cf (&v)[4][8], int k, int lane, int warp, Cf *rn) {
    if (lane == ((k + 1) & 31)) diag_store_row<I>(v, warp, rn);
}

// X = L^{-1} steps k in [16 JS, 16 JS + 16):  X[r][:] -= L[r][k] X[k][:]  (r > k; X[k][c] = 0 for c > k).
template <int JS>
__device__ __forceinline__ void diag_linv_segment(Cf (&v)[4][8], int nb, int lane, int warp, const DiagSmem &sm) {
    constexpr int IS = JS / 2;
    const Cf zero{0.f, 0.f};
#pragma unroll 1
    for (int kk = 0; kk < 16; ++kk) {
        const int k = 16 * JS + kk;
        if (k + 1 >= nb) return;  // uniform
        const int b = k & 1;
        Cf *rn = sm.rowb + (b ^ 1) * 128;
        Cf lk[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            lk[i] = zero;
            const int r = lane + 32 * i;
            if (i >= IS && (i > IS || r > k) && r < nb) lk[i] = sm.S[r + k * nb];
        }
#pragma unroll
        for (int j = 0; j <= JS; ++j) {
            if (j == JS && warp > kk) continue;  // columns c <= k only
            const Cf xk = sm.rowb[b * 128 + warp * 8 + j];
#pragma unroll
            for (int i = IS; i < 4; ++i) cfms(v[i][j], lk[i], xk);
        }
        if (kk < 15) {
            diag_publish_xrow<IS>(v, k, lane, warp, rn);
        } else if constexpr (JS < 7) {
            diag_publish_xrow<(JS + 1) / 2>(v, k, lane, warp, rn);
        }
        __syncthreads();
    }
}

// Row km (group I) of Y before its scaling into rn: its owner's registers
// hold the whole row (zeros before km, 1 at km, columns >= k as step k left
// them).
template <int I>
__device__ __forceinline__ void diag_publish_yrow(const Cf (&v)[4][8], int km, int lane, int warp, Cf *rn) {
    if (lane == (km & 31)) diag_store_row<I>(v, warp, rn);
}

// Y = U^{-1} steps k = 16 JS + 15 .. 16 JS:  Y[k][:] /= U_kk;  Y[r][:] -= U[r][k] Y[k][:]  (r < k;
// Y[k][c] = 0 for c < k).  t counts the steps taken (buffer parity).
template <int JS>
__device__ __forceinline__ void diag_uinv_segment(Cf (&v)[4][8], int nb, int lane, int warp, const DiagSmem &sm,
                                                  int &t) {
    constexpr int IS = JS / 2;
    const Cf zero{0.f, 0.f};
#pragma unroll 1
    for (int kk = 15; kk >= 0; --kk) {
        const int k = 16 * JS + kk;
        if (k >= nb) continue;  // uniform
        const int b = t & 1, km = k - 1;
        ++t;
        Cf *rn = sm.rowb + (b ^ 1) * 128;
        const Cf inv = sm.dinv[k];
        Cf uk[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            uk[i] = zero;
            const int r = lane + 32 * i;
            if (i <= IS && (i < IS || r < k)) uk[i] = sm.S[r + k * nb];
        }
#pragma unroll
        for (int j = JS; j < 8; ++j) {
            const int c = warp + 16 * j;
            if (j == JS && warp < kk) continue;  // columns c >= k only
            if (c >= nb) continue;
            const Cf yk = cmul(sm.rowb[b * 128 + warp * 8 + j], inv);
#pragma unroll
            for (int i = 0; i <= IS; ++i) cfms(v[i][j], uk[i], yk);  // uk = 0 on rows >= k
            if (lane == (k & 31)) v[IS][j] = yk;                       // row k, scaled
        }
        if (km >= 0) {
            if (kk > 0) {
                diag_publish_yrow<IS>(v, km, lane, warp, rn);
            } else if constexpr (JS > 0) {
                diag_publish_yrow<(16 * JS - 1) / 32>(v, km, lane, warp, rn);
            }
        }
        __syncthreads();
    }
}

// Principal square root of z, by the cancellation-free pair of formulas
// (t = sqrt((|z| + |Re z|) / 2), the other part Im z / 2t), in FP64.
__device__ __forceinline__ Cf csqrt_principal(Cf z) {
    const double a = z.re, b = z.im, r = hypot(a, b);
    if (r == 0.0) return Cf{0.f, 0.f};
    const double t = sqrt(0.5 * (r + fabs(a)));
    if (a >= 0.0) return Cf{(float)t, (float)(b / (2.0 * t))};
    return Cf{(float)(fabs(b) / (2.0 * t)), (float)copysign(t, b)};
}

// LU of the block in place (the diagonal of U into dv and its principal
// square roots into sv, when given); one CTA per matrix.
__global__ void __launch_bounds__(kDiagThreads, 1)
    diag_lu_kernel(Cx<float> *__restrict__ a, int64_t m, int64_t k0, int nb, Cx<float> *__restrict__ dv,
                   Cx<float> *__restrict__ sv, int64_t dstride) {
    __shared__ __align__(16) Cf bufs[2 * 128 + 2 * 128 + 2];
    DiagSmem sm;
    sm.S = nullptr;
    sm.colb = bufs;
    sm.rowb = bufs + 256;
    sm.dinv = nullptr;
    sm.pinv = bufs + 512;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Cf *A = a + (int64_t)blockIdx.x * m * m + k0 + k0 * m;
    const Cf zero{0.f, 0.f};
    Cf v[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int r = lane + 32 * i, c = warp + 16 * j;
            v[i][j] = (r < nb && c < nb) ? A[r + (int64_t)c * m] : zero;
        }
    diag_publish<0, 0>(v, 0, nb, lane, warp, sm.colb, sm.rowb, sm.pinv);  // column 0, row 0, 1 / a_00
    __syncthreads();
    diag_lu_segment<0>(v, nb, lane, warp, sm);
    diag_lu_segment<1>(v, nb, lane, warp, sm);
    diag_lu_segment<2>(v, nb, lane, warp, sm);
    diag_lu_segment<3>(v, nb, lane, warp, sm);
    diag_lu_segment<4>(v, nb, lane, warp, sm);
    diag_lu_segment<5>(v, nb, lane, warp, sm);
    diag_lu_segment<6>(v, nb, lane, warp, sm);
    diag_lu_segment<7>(v, nb, lane, warp, sm);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int r = lane + 32 * i, c = warp + 16 * j;
            if (r < nb && c < nb) {
                A[r + (int64_t)c * m] = v[i][j];
                if (dv && r == c) {
                    dv[(int64_t)blockIdx.x * dstride + r] = v[i][j];
                    sv[(int64_t)blockIdx.x * dstride + r] = csqrt_principal(v[i][j]);
                }
            }
        }
}

// The inverses of the factored block's L (blockIdx.y == 0, into linv) and U
// (blockIdx.y == 1, into uinv and optionally x2), in parallel: CTA (f, y).
__global__ void __launch_bounds__(kDiagThreads, 1)
    diag_inv_kernel(const Cx<float> *__restrict__ a, int64_t m, int64_t k0, int nb, Cx<float> *__restrict__ linv,
                    Cx<float> *__restrict__ uinv, int64_t mstride, Cx<float> *__restrict__ x2, int64_t ld2,
                    int64_t stride2) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DiagSmem sm;
    sm.colb = reinterpret_cast<Cf *>(smem_raw);  // the buffers first: 16-byte aligned for any nb
    sm.rowb = sm.colb + 256;
    sm.dinv = sm.rowb + 256;
    sm.pinv = sm.dinv + 128;
    sm.S = sm.pinv + 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool upper = blockIdx.y == 1;
    const Cf *A = a + (int64_t)blockIdx.x * m * m + k0 + k0 * m;
    const Cf zero{0.f, 0.f}, one{1.f, 0.f};
    for (int idx = threadIdx.x; idx < nb * nb; idx += kDiagThreads) {
        const int r = idx % nb, c = idx / nb;
        sm.S[idx] = A[r + (int64_t)c * m];
    }
    __syncthreads();
    if (threadIdx.x < nb) sm.dinv[threadIdx.x] = crcp(sm.S[threadIdx.x + threadIdx.x * nb]);
    // the first row the elimination reads: row 0 of I (X) or row nb - 1 of I (Y, before scaling)
    if (threadIdx.x < 128) sm.rowb[diag_row_slot(threadIdx.x)] = (int)threadIdx.x == (upper ? nb - 1 : 0) ? one : zero;
    Cf v[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) v[i][j] = (lane + 32 * i == warp + 16 * j) ? one : zero;
    __syncthreads();
    Cf *out;
    if (!upper) {
        diag_linv_segment<0>(v, nb, lane, warp, sm);
        diag_linv_segment<1>(v, nb, lane, warp, sm);
        diag_linv_segment<2>(v, nb, lane, warp, sm);
        diag_linv_segment<3>(v, nb, lane, warp, sm);
        diag_linv_segment<4>(v, nb, lane, warp, sm);
        diag_linv_segment<5>(v, nb, lane, warp, sm);
        diag_linv_segment<6>(v, nb, lane, warp, sm);
        diag_linv_segment<7>(v, nb, lane, warp, sm);
        out = linv + (int64_t)blockIdx.x * mstride;
    } else {
        int t = 0;
        diag_uinv_segment<7>(v, nb, lane, warp, sm, t);
        diag_uinv_segment<6>(v, nb, lane, warp, sm, t);
        diag_uinv_segment<5>(v, nb, lane, warp, sm, t);
        diag_uinv_segment<4>(v, nb, lane, warp, sm, t);
        diag_uinv_segment<3>(v, nb, lane, warp, sm, t);
        diag_uinv_segment<2>(v, nb, lane, warp, sm, t);
        diag_uinv_segment<1>(v, nb, lane, warp, sm, t);
        diag_uinv_segment<0>(v, nb, lane, warp, sm, t);
        out = uinv + (int64_t)blockIdx.x * mstride;
    }
    Cf *out2 = upper && x2 ? x2 + (int64_t)blockIdx.x * stride2 : nullptr;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int r = lane + 32 * i, c = warp + 16 * j;
            if (r < nb && c < nb) {
                out[r + c * nb] = v[i][j];
                if (out2) out2[r + (int64_t)c * ld2] = v[i][j];
            }
        }
}

// Linv = L11^{-1} for the unit lower triangle of panel [k0, k0+nb) of every
// matrix (column-major nb x nb, leading dimension nb, matrix f at
// linv + f * mstride).  The columns of the inverse are independent
// triangular solves, so CTA (f, c) forms columns [32c, 32c + 32) of matrix f:
// X starts as those columns of the identity and is reduced column by column
// of L11 (right-looking forward substitution),
//     for k: X[r][j] -= L[r][k] X[k][j]   for r > k,
// lane = column, warps over rows, X in shared memory, column k+1 of L11
// (contiguous in memory) fetched while step k computes.
// Grid (count, ceil(nb / 32)), 256 threads; dynamic shared memory
// (32 nb + 2 nb) complex.
// U[k, c] = U[k, k] L[c, k] for rows k in [K0, K0 + W) and columns c in
// [E, c1): U12 of a symmetric matrix factored without pivoting (U = D L^T).
// 32 x 32 tiles through shared memory, so both the reads of L (down a column)
// and the writes of U (along a row) are coalesced.
__global__ void u12_from_l21_kernel(Cx<float> *__restrict__ a, int64_t m, int64_t K0, int W, int64_t E, int64_t c1) {
    __shared__ Cx<float> t[32][33];
    Cx<float> *A = a + (int64_t)blockIdx.z * m * m;
    const int64_t c0 = E + (int64_t)blockIdx.x * 32, k0 = K0 + (int64_t)blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const int64_t c = c0 + tx, k = k0 + r;
        if (c < c1 && k < K0 + W) t[r][tx] = A[c + k * m];  // L[c, k]
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int64_t k = k0 + tx, c = c0 + r;
        if (c < c1 && k < K0 + W) A[k + c * m] = cmul(A[k + k * m], t[tx][r]);
    }
}

// pivots[f m + k] = k: the identity interchanges of a factorization without pivoting.
__global__ void identity_pivots_kernel(int *__restrict__ pivots, int64_t total, int64_t m) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x)
        pivots[t] = (int)(t % m);
}

template <class T>
__global__ void __launch_bounds__(256) tri_inverse_kernel(const Cx<T> *__restrict__ a, int64_t m, int k0, int nb,
                                                          Cx<T> *__restrict__ linv, int64_t mstride) {
    extern __shared__ unsigned char smem_raw[];
    Cx<T> *X = reinterpret_cast<Cx<T> *>(smem_raw);  // X[r * 32 + lane]
    Cx<T> *col = X + 32 * nb;                          // two staged columns of L11
    const int f = blockIdx.x, j0 = blockIdx.y * 32, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int j = j0 + lane;
    const Cx<T> *A = a + (int64_t)f * m * m + k0 + (int64_t)k0 * m;  // L11(r, k) at A[r + k m]
    for (int idx = tid; idx < 32 * nb; idx += blockDim.x)
        X[idx] = Cx<T>{(idx / 32 == j0 + idx % 32) ? (T)1 : (T)0, (T)0};
    if (j0 < nb)
        for (int r = tid; r < nb; r += blockDim.x) col[(j0 & 1) * nb + r] = A[r + (int64_t)j0 * m];
    __syncthreads();
    // Columns k < j0 of L do not touch these columns of X (their rows k are zero).
    for (int k = j0; k + 1 < nb; ++k) {
        const Cx<T> *ck = col + (k & 1) * nb;
        Cx<T> nxt{(T)0, (T)0};
        const bool fetch = k + 2 < nb && tid < nb;
        if (fetch) nxt = A[tid + (int64_t)(k + 1) * m];
        if (j <= k && j < nb) {
            const Cx<T> xk = X[k * 32 + lane];
            for (int r = k + 1 + warp; r < nb; r += 8) {
                Cx<T> x = X[r * 32 + lane];
                csubmul(x, ck[r], xk);
                X[r * 32 + lane] = x;
            }
        }
        if (fetch) col[((k + 1) & 1) * nb + tid] = nxt;
        __syncthreads();
    }
    Cx<T> *out = linv + (int64_t)f * mstride;
    for (int idx = tid; idx < 32 * nb; idx += blockDim.x) {
        const int r = idx % nb, c = idx / nb;
        if (j0 + c < nb) out[r + (int64_t)(j0 + c) * nb] = X[r * 32 + c];
    }
}

// Uinv = U11^{-1} for the upper triangle (non-unit) of panel [k0, k0+nb),
// same layout and grid.  Backward, column by column of U11 from the last
// that reaches these columns:
//     X[k][j] /= U[k][k];   X[r][j] -= U[r][k] X[k][j]   for r < k.
template <class T>
__global__ void __launch_bounds__(256) tri_inverse_upper_kernel(const Cx<T> *__restrict__ a, int64_t m, int k0,
                                                                int nb, Cx<T> *__restrict__ uinv, int64_t mstride) {
    extern __shared__ unsigned char smem_raw[];
    Cx<T> *X = reinterpret_cast<Cx<T> *>(smem_raw);  // X[r * 32 + lane]
    Cx<T> *col = X + 32 * nb;
    const int f = blockIdx.x, j0 = blockIdx.y * 32, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int j = j0 + lane;
    const Cx<T> *A = a + (int64_t)f * m * m + k0 + (int64_t)k0 * m;  // U11(r, k) at A[r + k m]
    for (int idx = tid; idx < 32 * nb; idx += blockDim.x)
        X[idx] = Cx<T>{(idx / 32 == j0 + idx % 32) ? (T)1 : (T)0, (T)0};
    const int klast = min(nb - 1, j0 + 31);  // rows k > klast of these columns are zero
    for (int r = tid; r <= klast; r += blockDim.x) col[(klast & 1) * nb + r] = A[r + (int64_t)klast * m];
    __syncthreads();
    const Cx<T> one{(T)1, (T)0};
    for (int k = klast; k >= 0; --k) {
        const Cx<T> *ck = col + (k & 1) * nb;
        Cx<T> nxt{(T)0, (T)0};
        const bool fetch = k > 0 && tid < k;
        if (fetch) nxt = A[tid + (int64_t)(k - 1) * m];
        const bool active = j >= k && j < nb;
        Cx<T> xk{(T)0, (T)0};
        if (active) {
            xk = cmul(X[k * 32 + lane], cdiv(one, ck[k]));
            for (int r = warp; r < k; r += 8) {
                Cx<T> x = X[r * 32 + lane];
                csubmul(x, ck[r], xk);
                X[r * 32 + lane] = x;
            }
        }
        if (fetch) col[((k - 1) & 1) * nb + tid] = nxt;
        __syncthreads();
        // Row k is read by every warp above; it is final once all have read it,
        // and no later step reads it again.
        if (active && warp == 0) X[k * 32 + lane] = xk;
    }
    __syncthreads();
    Cx<T> *out = uinv + (int64_t)f * mstride;
    for (int idx = tid; idx < 32 * nb; idx += blockDim.x) {
        const int r = idx % nb, c = idx / nb;
        if (j0 + c < nb) out[r + (int64_t)(j0 + c) * nb] = X[r * 32 + c];
    }
}

// C = A B (assign) or C -= A B for general strided complex operands, SIMT.
// Tile 64 x 64, K <= 64 staged whole in shared memory; 256 threads, 4 x 4
// outputs each.  In the assign form C may alias B when M <= 64.
template <class T>
struct SimtArgs {
    const Cx<T> *A;
    int64_t lda, sA;
    const Cx<T> *B;
    int64_t ldb, sB;
    Cx<T> *C;
    int64_t ldc, sC;
    int64_t M, N;
    int K;
    int assign;
};

template <class T>
__global__ void __launch_bounds__(256) gemm_simt_kernel(SimtArgs<T> g) {
    extern __shared__ unsigned char smem_raw[];
    Cx<T> *Ls = reinterpret_cast<Cx<T> *>(smem_raw);  // [K][64]
    Cx<T> *Us = Ls + g.K * 64;                         // [K][64]
    const int f = blockIdx.z;
    const Cx<T> *Aop = g.A + (int64_t)f * g.sA;
    const Cx<T> *Bop = g.B + (int64_t)f * g.sB;
    Cx<T> *C = g.C + (int64_t)f * g.sC;
    const int64_t i0 = (int64_t)blockIdx.y * 64, j0 = (int64_t)blockIdx.x * 64;
    const int tid = threadIdx.x, K = g.K;
    for (int idx = tid; idx < K * 64; idx += 256) {
        const int ii = idx % 64, k = idx / 64;
        Ls[k * 64 + ii] = i0 + ii < g.M ? Aop[(i0 + ii) + (int64_t)k * g.lda] : Cx<T>{0, 0};
        const int kk = idx % K, jj = idx / K;
        Us[kk * 64 + jj] = j0 + jj < g.N ? Bop[kk + (j0 + jj) * g.ldb] : Cx<T>{0, 0};
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;
    T accr[4][4], acci[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) accr[r][c] = acci[r][c] = (T)0;
    for (int k = 0; k < K; ++k) {
        Cx<T> l[4], u[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) l[r] = Ls[k * 64 + tx + 16 * r];
#pragma unroll
        for (int c = 0; c < 4; ++c) u[c] = Us[k * 64 + ty + 16 * c];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                accr[r][c] += l[r].re * u[c].re - l[r].im * u[c].im;
                acci[r][c] += l[r].re * u[c].im + l[r].im * u[c].re;
            }
    }
    if (g.assign) __syncthreads();  // every B load of this CTA precedes any C store
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int64_t col = j0 + ty + 16 * c;
        if (col >= g.N) continue;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int64_t row = i0 + tx + 16 * r;
            if (row >= g.M) continue;
            Cx<T> *p = C + row + col * g.ldc;
            if (g.assign) {
                *p = Cx<T>{accr[r][c], acci[r][c]};
            } else {
                Cx<T> y = *p;
                y.re -= accr[r][c];
                y.im -= acci[r][c];
                *p = y;
            }
        }
    }
}

// x[r] -= sum_c A[r, k0 + c] x[k0 + c] for r in [r0, r1).
template <class T>
__global__ void __launch_bounds__(256) gemv_update_kernel(const Cx<T> *__restrict__ a, int64_t m, int nrhs, int k0,
                                                          int nb, int64_t r0, int64_t r1, Cx<T> *__restrict__ x) {
    const int g = blockIdx.y;  // (f, q)
    const int f = g / nrhs;
    const Cx<T> *A = a + (int64_t)f * m * m;
    Cx<T> *X = x + (int64_t)g * m;
    __shared__ Cx<T> xs[128];
    for (int c = threadIdx.x; c < nb; c += blockDim.x) xs[c] = X[k0 + c];
    __syncthreads();
    for (int64_t r = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < r1; r += (int64_t)gridDim.x * blockDim.x) {
        Cx<T> y = X[r];
        for (int c = 0; c < nb; ++c) csubmul(y, xs[c], A[r + (int64_t)(k0 + c) * m]);
        X[r] = y;
    }
}

// ---------------------------------------------------------------------------
// System formation and FP64 residual.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) form_kernel(const double *__restrict__ R, const double *__restrict__ L, int64_t ld,
                                                   int64_t m, const double *__restrict__ omega, int count,
                                                   Cx<T> *__restrict__ a) {
    const int64_t total = m * m;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t % m, j = t / m;
        const double r = R[i + j * ld], l = L[i + j * ld];
        for (int f = 0; f < count; ++f) a[(int64_t)f * total + t] = Cx<T>{(T)r, (T)(omega[f] * l)};
    }
}

// FP32 form, two consecutive entries per 16-byte store (mo * mo even, batch
// 16-byte aligned).  A CTA takes kFormPer x 256 consecutive entry pairs,
// reads their R and L once and writes them frequency by frequency, so each
// frequency's plane receives one contiguous 16 KB run per CTA.  With
// lower_tiles, pairs whose entries both lie in 128 x 128 tiles above the
// diagonal are skipped.  The formed matrix has order mo >= m: entries outside
// the leading m x m block are those of the identity (the border of an odd
// order, see the mixed sweep).
constexpr int kFormPer = 4;
__global__ void __launch_bounds__(256) form_pair_kernel(const double *__restrict__ R, const double *__restrict__ L,
                                                        int64_t ld, int64_t m, int64_t mo,
                                                        const double *__restrict__ omega, int count,
                                                        float4 *__restrict__ a, int lower_tiles) {
    const int64_t pairs = mo * mo / 2, chunk = 256 * kFormPer;
    for (int64_t base = (int64_t)blockIdx.x * chunk; base < pairs; base += (int64_t)gridDim.x * chunk) {
        double r0[kFormPer], l0[kFormPer], r1[kFormPer], l1[kFormPer];
        bool keep[kFormPer];
#pragma unroll
        for (int k = 0; k < kFormPer; ++k) {
            const int64_t t = base + k * 256 + threadIdx.x;
            keep[k] = t < pairs;
            if (!keep[k]) continue;
            const int64_t e = 2 * t, i = e % mo, j = e / mo;
            const int64_t i1 = i + 1 == mo ? 0 : i + 1, j1 = i + 1 == mo ? j + 1 : j;  // entry e + 1
            if (lower_tiles && (i >> 7) < (j >> 7) && (i1 >> 7) < (j1 >> 7)) {
                keep[k] = false;
                continue;
            }
            const bool in0 = i < m && j < m, in1 = i1 < m && j1 < m;
            r0[k] = in0 ? R[i + j * ld] : (i == j ? 1.0 : 0.0);
            l0[k] = in0 ? L[i + j * ld] : 0.0;
            r1[k] = in1 ? R[i1 + j1 * ld] : (i1 == j1 ? 1.0 : 0.0);
            l1[k] = in1 ? L[i1 + j1 * ld] : 0.0;
        }
        for (int f = 0; f < count; ++f) {
            const double w = __ldg(omega + f);
            float4 *plane = a + (int64_t)f * pairs + base + threadIdx.x;
#pragma unroll
            for (int k = 0; k < kFormPer; ++k)
                if (keep[k])
                    __stcs(plane + k * 256,
                           make_float4((float)r0[k], (float)(w * l0[k]), (float)r1[k], (float)(w * l1[k])));
        }
    }
}

template <class T>
__global__ void rhs_kernel(const double *__restrict__ R, const double *__restrict__ L, int64_t ld, int64_t m, int64_t p,
                           const double *__restrict__ omega, int count, Cx<T> *__restrict__ b) {
    const int64_t total = m * p;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total * count;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int f = (int)(t / total);
        const int64_t e = t % total, i = e % m, q = e / m;
        const double r = R[i + (m + q) * ld], l = L[i + (m + q) * ld];
        b[t] = Cx<T>{(T)r, (T)(omega[f] * l)};
    }
}

// r = b - (R + j w L) x for every (frequency f, port column q), b = Z_ep
// column q; x and r hold column g = f p + q at g m.  R x and L x are real
// matrices times complex columns: a register-tiled FP64 product, block tile
// 32 rows x 32 columns g, k in stages of 16 staged in shared memory (double
// buffered, the next stage's loads in flight during the current one), thread
// tile 4 rows x 2 columns for both R and L.  Each accumulator sums over k in
// increasing order.  With `part`, the k stages are split into gridDim.z
// contiguous ranges (CTA z takes range z) and each CTA writes its sums
// (R x re, im, L x re, im) to part[(z G + g) m + row]; residual_finish_kernel
// then adds the ranges in order, so the result does not depend on the
// schedule.  The split keeps every SM busy when the row tiles alone are few
// or uneven across the SMs.
// kDenseR false: R x comes precomputed in rx (the loop-basis product) and the
// pass reads L alone.
constexpr int kResRows = 32, kResCols = 32, kResK = 16, kResThreads = 128, kResMaxSplits = 16;
template <bool kDenseR>
__global__ void __launch_bounds__(kResThreads) residual_kernel(const double *__restrict__ R,
                                                               const double *__restrict__ L, int64_t ld, int64_t m,
                                                               int64_t p, const double *__restrict__ omega, int count,
                                                               const Cx<double> *__restrict__ x,
                                                               Cx<double> *__restrict__ r, double4 *__restrict__ part,
                                                               const Cx<double> *__restrict__ rx) {
    __shared__ double Rs[2][kResK][kResRows], Ls[2][kResK][kResRows];
    __shared__ Cx<double> Xs[2][kResK][kResCols + 1];  // padded: the stores run down k
    const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
    const int64_t i0 = (int64_t)blockIdx.x * kResRows;
    const int64_t g0 = (int64_t)blockIdx.y * kResCols, G = (int64_t)count * p;
    double rv[4], lv[4];
    Cx<double> xv[4];
    auto load = [&](int64_t k0) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int idx = tid + kResThreads * e;
            const int row = idx & 31, k = idx >> 5;
            const int64_t i = i0 + row, kk = k0 + k;
            const bool in = i < m && kk < m;
            if (kDenseR) rv[e] = in ? R[i + kk * ld] : 0.0;
            lv[e] = in ? L[i + kk * ld] : 0.0;
            const int kx = idx & 15, g = idx >> 4;
            const int64_t kkx = k0 + kx;
            xv[e] = (g0 + g < G && kkx < m) ? x[(g0 + g) * m + kkx] : Cx<double>{0.0, 0.0};
        }
    };
    auto store = [&](int b) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int idx = tid + kResThreads * e;
            if (kDenseR) Rs[b][idx >> 5][idx & 31] = rv[e];
            Ls[b][idx >> 5][idx & 31] = lv[e];
            Xs[b][idx & 15][idx >> 4] = xv[e];
        }
    };
    Cx<double> ar[4][2], al[4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) ar[i][j] = al[i][j] = Cx<double>{0.0, 0.0};
    const int64_t all_stages = (m + kResK - 1) / kResK, per = (all_stages + gridDim.z - 1) / gridDim.z;
    const int64_t s_begin = min(all_stages, (int64_t)blockIdx.z * per), s_end = min(all_stages, s_begin + per);
    load(s_begin * kResK);
    store(0);
    __syncthreads();
    for (int64_t st = s_begin; st < s_end; ++st) {
        const int b = (int)((st - s_begin) & 1);
        if (st + 1 < s_end) load((st + 1) * kResK);
#pragma unroll
        for (int k = 0; k < kResK; ++k) {
            double rk[4], lk[4];
            Cx<double> xk[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                rk[i] = kDenseR ? Rs[b][k][tx + 8 * i] : 0.0;
                lk[i] = Ls[b][k][tx + 8 * i];
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) xk[j] = Xs[b][k][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    if (kDenseR) {
                        ar[i][j].re += rk[i] * xk[j].re;
                        ar[i][j].im += rk[i] * xk[j].im;
                    }
                    al[i][j].re += lk[i] * xk[j].re;
                    al[i][j].im += lk[i] * xk[j].im;
                }
        }
        if (st + 1 < s_end) store(b ^ 1);
        __syncthreads();
    }
    if (part) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int64_t g = g0 + ty + 16 * j;
            if (g >= G) continue;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t row = i0 + tx + 8 * i;
                if (row < m)
                    part[((int64_t)blockIdx.z * G + g) * m + row] =
                        make_double4(ar[i][j].re, ar[i][j].im, al[i][j].re, al[i][j].im);
            }
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int64_t g = g0 + ty + 16 * j;
        if (g >= G) continue;
        const int f = (int)(g / p);
        const int64_t q = g % p;
        const double w = omega[f];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t row = i0 + tx + 8 * i;
            if (row >= m) continue;
            const double br = R[row + (m + q) * ld], bl = L[row + (m + q) * ld];
            // (R + jwL) x = R x + j w (L x)
            const Cx<double> rxv = kDenseR ? ar[i][j] : rx[g * m + row];
            const double ax_re = rxv.re - w * al[i][j].im;
            const double ax_im = rxv.im + w * al[i][j].re;
            r[g * m + row] = Cx<double>{br - ax_re, w * bl - ax_im};
        }
    }
}

// The split residual's second pass: the k ranges' sums added in range order,
// then r as in residual_kernel.
__global__ void residual_finish_kernel(const double *__restrict__ R, const double *__restrict__ L, int64_t ld,
                                       int64_t m, int64_t p, const double *__restrict__ omega, int count, int splits,
                                       const double4 *__restrict__ part, Cx<double> *__restrict__ r,
                                       const Cx<double> *__restrict__ rx) {
    const int64_t G = (int64_t)count * p, total = G * m;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = t / m, row = t % m;
        double4 a = part[t];
        for (int z = 1; z < splits; ++z) {
            const double4 b = part[(int64_t)z * total + t];
            a.x += b.x;
            a.y += b.y;
            a.z += b.z;
            a.w += b.w;
        }
        const int f = (int)(g / p);
        const int64_t q = g % p;
        const double w = omega[f];
        const double br = R[row + (m + q) * ld], bl = L[row + (m + q) * ld];
        if (rx) {  // R x from the loop basis (the split sums hold zeros there)
            a.x = rx[t].re;
            a.y = rx[t].im;
        }
        const double ax_re = a.x - w * a.w, ax_im = a.y + w * a.z;
        r[t] = Cx<double>{br - ax_re, w * bl - ax_im};
    }
}

// Z_f[i][j] = pp[i][j] - sum_k ep[k][i] x_f[k][j]; one block per (f, i, j).
__global__ void __launch_bounds__(256) schur_kernel(const double *__restrict__ R, const double *__restrict__ L,
                                                    int64_t ld, int64_t m, int64_t p, const double *__restrict__ omega,
                                                    const Cx<double> *__restrict__ x, Cx<double> *__restrict__ z) {
    const int64_t g = blockIdx.x;
    const int f = (int)(g / (p * p));
    const int64_t ij = g % (p * p), i = ij / p, j = ij % p;
    const double w = omega[f];
    double sre = 0.0, sim = 0.0;
    const Cx<double> *X = x + ((int64_t)f * p + j) * m;
    for (int64_t k = threadIdx.x; k < m; k += blockDim.x) {
        const double er = R[k + (m + i) * ld], el = w * L[k + (m + i) * ld];
        const Cx<double> xv = X[k];
        sre += er * xv.re - el * xv.im;
        sim += er * xv.im + el * xv.re;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sre += __shfl_down_sync(0xffffffffu, sre, o);
        sim += __shfl_down_sync(0xffffffffu, sim, o);
    }
    __shared__ double s1[8], s2[8];
    if ((threadIdx.x & 31) == 0) {
        s1[threadIdx.x >> 5] = sre;
        s2[threadIdx.x >> 5] = sim;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a += s1[k];
            b += s2[k];
        }
        const double pr = R[(m + i) + (m + j) * ld], pl = w * L[(m + i) + (m + j) * ld];
        Cx<double> out{pr - a, pl - b};
        if (w == 0.0) out.im = 0.0;  // DC: the real resistive network (solve.rs:811-815)
        z[((int64_t)f * p + i) * p + j] = out;
    }
}

__global__ void c64_to_c32_kernel(const double *__restrict__ s, float *__restrict__ d, int64_t n) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * n; t += (int64_t)gridDim.x * blockDim.x)
        d[t] = (float)s[t];
}
__global__ void add_c32_kernel(double *__restrict__ x, const float *__restrict__ d, int64_t n) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * n; t += (int64_t)gridDim.x * blockDim.x)
        x[t] += (double)d[t];
}
// The same between columns of m entries (FP64) and columns of mo > m entries
// (FP32, the bordered system): the border entries are written as zero / not
// read back.  t runs over the FP32 side's interleaved values.
__global__ void c64_to_c32_border_kernel(const double *__restrict__ s, float *__restrict__ d, int64_t m, int64_t mo,
                                         int64_t cols) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * mo * cols;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t >> 1, col = e / mo, i = e - col * mo;
        d[t] = i < m ? (float)s[2 * (col * m + i) + (t & 1)] : 0.0f;
    }
}
__global__ void add_c32_border_kernel(double *__restrict__ x, const float *__restrict__ d, int64_t m, int64_t mo,
                                      int64_t cols) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * m * cols;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t >> 1, col = e / m, i = e - col * m;
        x[t] += (double)d[2 * (col * mo + i) + (t & 1)];
    }
}
template <class T>
__global__ void max_abs_kernel(const T *__restrict__ v, int64_t per, double *__restrict__ out) {
    const T *V = v + (int64_t)blockIdx.x * per;
    double mx = 0.0;
    for (int64_t t = threadIdx.x; t < per; t += blockDim.x) mx = fmax(mx, (double)fabs(V[t]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    __shared__ double s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) mx = fmax(mx, s[k]);
        out[blockIdx.x] = mx;
    }
}

inline int grid_for(int64_t work, int threads, int cap = 148 * 32) {
    int64_t g = (work + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

// Look-ahead sizing: SMs left to the front while the deep update runs (at
// least one per matrix, for the one-CTA-per-matrix diagonal kernels, and at
// most a quarter of the GPU), and the smallest second part of an update, in
// tiles per SM, worth splitting the update for (a 128 x 128 tile at K = 512
// takes about 19 us of an SM; a front, about 1 ms on the whole GPU).
constexpr int kAheadMinSpare = 16;
constexpr int kAheadMinWaves = 16;

// Two-level blocked factorization of an FP32 batch on the tensor cores.
//
// For each super-panel [K0, E) of `outer` columns:
//   for each nb-wide panel [j0, j0+nb) inside it
//     cooperative panel factorization (rows j0.., its own columns);
//     its interchanges on the super-panel's other columns;
//     Linv_j = (unit L_jj)^{-1};  U = Linv_j A[j0 block, j0+nb..E);
//     A[j0+nb.., j0+nb..E) -= L[j0+nb.., panel] U       (K = nb)
//   all interchanges of the super-panel, in order, on columns [E, m);
//   U12 = L11^{-1} A12 block by block (Linv_j, then the rows below it inside
//   the super-panel);
//   A22 -= L21 U12 with K = outer from packed operands.
//
// The deep update moves the same 16 bytes of C per entry as a one-panel
// update but does outer/nb times the arithmetic on them, which lifts it off
// the HBM roofline.  The interchange convention differs from the one-level
// path only inside a super-panel (all of its L columns carry all of its
// interchanges), hence lu_solve(group = outer).
fh_status lu_factor_deep(LuBatch<float> &b, LuWork &w, int nb, cudaStream_t s, fh_error_info *err) {
    using C = Cx<float>;
    C *a = reinterpret_cast<C *>(b.a);
    const int64_t m = b.m, mm = m * m;
    const int count = b.count;
    const int outer = w.outer;
    if (nb % 16 || nb > 128 || outer % nb || !w.coop || !w.linv || !w.pack_a)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "two-level factorization needs nb | outer, nb <= 128 and scratch");
    const size_t inv_smem = sizeof(C) * (34 * (size_t)nb);
    const dim3 inv_grid((unsigned)count, (unsigned)((nb + 31) / 32));
    FHB_CUDA(cudaFuncSetAttribute(tri_inverse_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)inv_smem));
    FHB_CUDA(cudaFuncSetAttribute(tri_inverse_upper_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)inv_smem));
    auto at = [&](int64_t r, int64_t c) { return b.a + 2 * (r + c * m); };
    // Inverses of the diagonal blocks, slot j0 / nb (count * nb * nb each).
    auto slot = [&](void *base, int64_t j0) { return reinterpret_cast<C *>(base) + (size_t)(j0 / nb) * count * nb * nb; };
    auto swaps = [&](int64_t k0, int n, int64_t c0, int64_t c1) {
        if (c1 > c0)
            swap_kernel<float><<<dim3(grid_for(c1 - c0, 256, 1024), count), 256, 0, s>>>(a, m, (int)k0, n, c0, c1,
                                                                                        b.pivots);
    };
    fh_status st = FH_OK;
    const bool nopivot = w.nopivot;
    // The closing coop_check reads this flag whether or not a cooperative
    // panel ran (the factorization without pivoting runs none).
    FHB_CUDA(cudaMemsetAsync(w.coop->error, 0, sizeof(int), s));
    if (nopivot) {
        if (!w.uinv) return fail(err, FH_ERR_INVALID_ARGUMENT, "the factorization without pivoting needs uinv");
        const size_t diag_smem = sizeof(C) * ((size_t)nb * nb + kDiagSmemExtra);
        FHB_CUDA(cudaFuncSetAttribute(diag_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem));
        const int64_t total = (int64_t)count * m;
        identity_pivots_kernel<<<grid_for(total, 256, 1024), 256, 0, s>>>(b.pivots, total, m);
        FHB_CUDA(cudaGetLastError());
    }
    // Without pivoting and with the scratch for it, the rows below each
    // super-panel are left to one tensor-core pass (gemm_tc_panel_solve);
    // the per-block steps then stop at the super-panel's last row.
    const bool fused = nopivot && w.xinv && w.xpack && w.tbuf && w.dvec && nb == 128 && outer % nb == 0 &&
                       panel_solve_supported(m) && (int64_t)count * m <= INT32_MAX;
    // the fused pass packs one operand for both sides; otherwise B has its own
    if (!fused && !w.pack_b)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "two-level factorization needs a packed B operand scratch");
    C *xinv = reinterpret_cast<C *>(w.xinv), *dvec = reinterpret_cast<C *>(w.dvec);
    C *svec = fused ? dvec + (int64_t)count * outer : nullptr;
    // X's blocks below its diagonal are read as zeros and never written.
    if (fused) FHB_CUDA(cudaMemsetAsync(w.xinv, 0, sizeof(C) * (size_t)count * outer * outer, s));
    // Look-ahead (fused form, with a second stream and a tile counter): the
    // diagonal region of each super-panel, its X and the packing of X (the
    // "front", a chain of small launches of one or two CTAs per matrix) run
    // on `side`, overlapping the previous super-panel's deep update.  That
    // update goes in two parts on s: first the next super-panel's column
    // blocks on every SM (the front needs them), then the rest from the tile
    // counter on all SMs but `spare`; when the front is done, a grid of
    // `spare` CTAs on the side stream joins the rest from the same counter.
    // The rows-below pass stays on s (it needs the whole GPU and the packed
    // operand, which the update reads until it ends).  A deep update too
    // short to hide a front runs whole, without the split.
    const bool ahead = fused && w.side && w.tile_counter;
    const int sms = ahead ? gemm_tc_sm_count() : 0;
    const int spare = std::min(sms / 4, std::max(count, kAheadMinSpare));
    cudaEvent_t ev_go = nullptr, ev_done = nullptr;  // s -> side: the front may start; side -> s: front (+ helper) done
    PackedSchedule rest;                             // the deep update's second part, waiting for its helper grid
    struct AheadRelease {
        cudaEvent_t *a, *b;
        PackedSchedule *ps;
        cudaStream_t s;
        ~AheadRelease() {
            if (ps->table) gemm_tc_packed_release(*ps, s);
            if (*a) cudaEventDestroy(*a);
            if (*b) cudaEventDestroy(*b);
        }
    } ahead_release{&ev_go, &ev_done, &rest, s};
    if (ahead) {
        FHB_CUDA(cudaEventCreateWithFlags(&ev_go, cudaEventDisableTiming));
        FHB_CUDA(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
        FHB_CUDA(cudaEventRecord(ev_go, s));  // the set-up above, before the first front
        FHB_CUDA(cudaStreamWaitEvent(w.side, ev_go, 0));
    }
    // After a front: the helper grid of the update it overlapped, then s waits
    // for both.
    auto join_front = [&]() -> fh_status {
        if (rest.tiles > 0) {
            const fh_status hs = gemm_tc_packed_launch(rest, spare, w.tile_counter, w.side, err, -1);
            if (hs) return hs;
        }
        FHB_CUDA(cudaEventRecord(ev_done, w.side));
        FHB_CUDA(cudaStreamWaitEvent(s, ev_done, 0));
        if (rest.tiles > 0 || rest.table) gemm_tc_packed_release(rest, s);
        return FH_OK;
    };
    for (int64_t K0 = 0; K0 < m; K0 += outer) {
        const cudaStream_t sx = ahead ? w.side : s;  // the front's stream
        const int W = (int)std::min<int64_t>(outer, m - K0);
        const int64_t E = K0 + W;
        const bool below = fused && E < m;  // rows below this super-panel go to the fused pass
        const int64_t rend = below ? E : m;  // rows the per-block steps update
        for (int64_t j0 = K0; j0 < E; j0 += nb) {
            const int wj = (int)std::min<int64_t>(nb, E - j0);
            const int64_t r1 = j0 + wj;  // first row / column after the panel
            C *linv = slot(w.linv, j0);
            const int64_t mstride = (int64_t)nb * nb;  // a partial last block keeps the full slot stride
            prof_begin(sx, FH_PROF_PANEL);
            if (nopivot) {
                // LU of the diagonal block and the inverses of its L and U
                // (with the fused pass: U^-1 also into X's diagonal block, and
                // U's diagonal into dvec).
                const int64_t o = j0 - K0;
                diag_lu_kernel<<<(unsigned)count, kDiagThreads, 0, sx>>>(a, m, j0, wj, below ? dvec + o : nullptr,
                                                                        below ? svec + o : nullptr, W);
                diag_inv_kernel<<<dim3((unsigned)count, 2), kDiagThreads, sizeof(C) * ((size_t)wj * wj + kDiagSmemExtra),
                                  sx>>>(a, m, j0, wj, linv, slot(w.uinv, j0), mstride, below ? xinv + o + o * W : nullptr,
                                       W, (int64_t)W * W);
                st = cudaGetLastError() == cudaSuccess ? FH_OK
                                                       : fail(err, FH_ERR_CUDA, "diagonal block factorization launch failed");
            } else {
                st = panel_coop<float>(b, j0, wj, *w.coop, sx, err);
            }
            prof_end(sx, FH_PROF_PANEL, 0.0);
            if (st) return st;
            prof_begin(sx, FH_PROF_TRSM);
            if (!nopivot) {
                tri_inverse_kernel<float><<<inv_grid, 256, inv_smem, sx>>>(a, m, (int)j0, wj, linv, mstride);
                if (w.uinv)
                    tri_inverse_upper_kernel<float><<<inv_grid, 256, inv_smem, sx>>>(a, m, (int)j0, wj,
                                                                                    slot(w.uinv, j0), mstride);
            }
            if (r1 >= m) {
                prof_end(sx, FH_PROF_TRSM, 0.0);
                break;
            }
            if (nopivot) {
                // L21 = A21 U11^-1 for the rows below the block (in place: each
                // tile of L21 reads exactly its own rows of A21).
                if (rend > r1)
                    st = gemm_tc_strided(at(r1, j0), m, mm, reinterpret_cast<const float *>(slot(w.uinv, j0)), wj,
                                         mstride, at(r1, j0), m, mm, rend - r1, wj, wj, 1, count, sx, err);
                if (st) return st;
            } else {
                swaps(j0, wj, K0, j0);
                swaps(j0, wj, r1, E);
            }
            if (r1 < E && nopivot) {
                // U12 inside the super-panel = D L21^T from the L21 just formed,
                // so nothing reads the upper tiles of a diagonal region, which
                // the symmetric deep updates leave out.
                const dim3 tg((unsigned)((E - r1 + 31) / 32), (unsigned)((wj + 31) / 32), (unsigned)count);
                u12_from_l21_kernel<<<tg, dim3(32, 8), 0, sx>>>(a, m, j0, wj, r1, E);
                st = cudaGetLastError() == cudaSuccess ? FH_OK : fail(err, FH_ERR_CUDA, "U12 transpose launch failed");
            } else if (r1 < E) {
                st = gemm_tc_strided(reinterpret_cast<const float *>(linv), wj, mstride, at(j0, r1), m, mm,
                                     at(j0, r1), m, mm, wj, E - r1, wj, 1, count, sx, err);
            }
            prof_end(sx, FH_PROF_TRSM, 4.0 * (double)wj * wj * (double)(E - r1) * count);
            if (st) return st;
            if (r1 < E) {
                prof_begin(sx, FH_PROF_GEMM_TC_INNER);
                st = gemm_tc_strided(at(r1, j0), m, mm, at(j0, r1), m, mm, at(r1, r1), m, mm, rend - r1, E - r1, wj, 0,
                                     count, sx, err);
                prof_end(sx, FH_PROF_GEMM_TC_INNER, 8.0 * (double)(rend - r1) * (double)(E - r1) * wj * count);
                if (st) return st;
            }
        }
        if (E >= m) break;
        const int64_t n2 = m - E;
        if (below) {
            // X = U_D^{-1} from the block inverses on its diagonal, by block
            // rows from the bottom: row i right of its diagonal block is
            //     X_i,(i+1..) = -X_ii (U_i,(i+1..) X_(i+1..),(i+1..))
            // (X_(i+1..),(i+1..) upper triangular and already formed): two
            // products per block row.
            const int nbw = W / nb;
            auto xat = [&](int bi, int bj) {
                return reinterpret_cast<float *>(xinv + (int64_t)bi * nb + (int64_t)bj * nb * W);
            };
            float *t = reinterpret_cast<float *>(w.tbuf);
            const int64_t ww = (int64_t)W * W, tt = (int64_t)nb * (W - nb);
            prof_begin(sx, FH_PROF_TRSM);
            for (int bi = nbw - 2; bi >= 0 && !st; --bi) {
                const int rest_cols = (nbw - 1 - bi) * nb;  // columns right of the diagonal block
                st = gemm_tc_strided(at(K0 + (int64_t)bi * nb, K0 + (int64_t)(bi + 1) * nb), m, mm, xat(bi + 1, bi + 1),
                                     W, ww, t, nb, tt, nb, rest_cols, rest_cols, 1, count, sx, err);
                if (!st)
                    st = gemm_tc_strided(xat(bi, bi), W, ww, t, nb, tt, xat(bi, bi + 1), W, ww, nb, rest_cols, nb, 2,
                                         count, sx, err);
            }
            if (!st) st = gemm_tc_pack_b(reinterpret_cast<float *>(xinv), W, ww, W, W, count, w.xpack, sx, err);
            prof_end(sx, FH_PROF_TRSM, 0.0);
            if (st) return st;
            if (ahead) {
                st = join_front();
                if (st) return st;
            }
            // L21 = A21 X for every row below, U12 = D L21^T, P = L21 S packed.
            st = gemm_tc_panel_solve(b.a, m, count, K0, W, w.xpack, reinterpret_cast<const float *>(dvec),
                                     reinterpret_cast<const float *>(svec), w.pack_a, w.upper, s, err);
            if (st) return st;
            // C -= P P^T, only the tiles on and below the diagonal: every U
            // entry is formed from L (steps inside each diagonal region, panel
            // solve beyond).
            // With the look-ahead: the next super-panel's column blocks first,
            // then the front of that super-panel may start.
            const int next_blocks = (int)((std::min<int64_t>(outer, n2) + 127) / 128);
            const int64_t rest_blocks = (n2 + 127) / 128 - next_blocks;
            const double rest_tiles = (double)count * (double)rest_blocks * (double)(rest_blocks + 1) / 2.0;
            if (!ahead || rest_tiles < (double)kAheadMinWaves * sms) {
                st = gemm_tc_packed_run(w.pack_a, w.pack_a, at(E, E), m, mm, n2, n2, W, count, s, err, 0);
                if (st) return st;
                if (ahead) {
                    FHB_CUDA(cudaEventRecord(ev_go, s));
                    FHB_CUDA(cudaStreamWaitEvent(w.side, ev_go, 0));
                }
                continue;
            }
            st = gemm_tc_packed_run(w.pack_a, w.pack_a, at(E, E), m, mm, n2, n2, W, count, s, err, 0, 0, next_blocks);
            if (st) return st;
            // The counter and the rest's tile table are in place (on s)
            // before the side stream, whose helper grid reads both, goes on.
            FHB_CUDA(cudaMemsetAsync(w.tile_counter, 0, sizeof(int), s));
            st = gemm_tc_packed_schedule(rest, w.pack_a, w.pack_a, at(E, E), m, mm, n2, n2, W, count, 0, next_blocks, -1,
                                         s, err);
            if (st) return st;
            FHB_CUDA(cudaEventRecord(ev_go, s));
            FHB_CUDA(cudaStreamWaitEvent(w.side, ev_go, 0));
            st = gemm_tc_packed_launch(rest, sms - spare, w.tile_counter, s, err, FH_PROF_GEMM_TC_SHARED);
            if (st) return st;
            continue;
        }
        prof_begin(s, FH_PROF_TRSM);
        if (nopivot) {
            // Symmetric trailing matrix: U12 = D L21^T (D the diagonal of U11).
            const dim3 tg((unsigned)((n2 + 31) / 32), (unsigned)((W + 31) / 32), (unsigned)count);
            u12_from_l21_kernel<<<tg, dim3(32, 8), 0, s>>>(a, m, K0, W, E, m);
            FHB_CUDA(cudaGetLastError());
            prof_end(s, FH_PROF_TRSM, 0.0);
            // Only the tiles on and below the diagonal of the trailing matrix
            // are read from here on: every U entry of the later super-panels,
            // inside their diagonal blocks too, is formed from L.
            st = gemm_tc_packed_update(at(E, K0), m, mm, at(K0, E), m, mm, at(E, E), m, mm, n2, n2, W, count,
                                       w.pack_a, w.pack_b, s, err, 0);
            if (st) return st;
            continue;
        }
        swaps(K0, W, E, m);
        for (int64_t j0 = K0; j0 < E && !st; j0 += nb) {
            const C *linv = slot(w.linv, j0);
            st = gemm_tc_strided(reinterpret_cast<const float *>(linv), nb, (int64_t)nb * nb, at(j0, E), m, mm,
                                 at(j0, E), m, mm, nb, n2, nb, 1, count, s, err);
            if (!st && j0 + nb < E)
                st = gemm_tc_strided(at(j0 + nb, j0), m, mm, at(j0, E), m, mm, at(j0 + nb, E), m, mm, E - j0 - nb,
                                     n2, nb, 0, count, s, err);
        }
        prof_end(s, FH_PROF_TRSM, 4.0 * (double)W * W * (double)n2 * count);
        if (st) return st;
        st = gemm_tc_packed_update(at(E, K0), m, mm, at(K0, E), m, mm, at(E, E), m, mm, n2, n2, W, count, w.pack_a,
                                   w.pack_b, s, err);
        if (st) return st;
        FHB_CUDA(cudaGetLastError());
    }
    if (ahead) {  // the last front (the final diagonal region) and any helper, before what follows on s
        st = join_front();
        if (st) return st;
    }
    FHB_CUDA(cudaGetLastError());
    return coop_check(*w.coop, s, err);
}

}  // namespace

template <class T>
fh_status lu_factor(LuBatch<T> &b, LuWork &w, int nb, TrailingUpdate mode, cudaStream_t s, fh_error_info *err) {
    using C = Cx<T>;
    C *a = reinterpret_cast<C *>(b.a);
    const int64_t m = b.m;
    if (m == 0 || b.count == 0) return FH_OK;
    if constexpr (sizeof(T) == 4) {
        if (w.outer > nb && mode == TrailingUpdate::TensorBf16x3) return lu_factor_deep(b, w, nb, s, err);
    }
    // Shared-memory budget of the TRSM / SIMT update kernels: 64 columns in
    // FP64, 128 in FP32.
    const int nb_max = sizeof(T) == 8 ? 64 : 128;
    if (nb > nb_max || nb < 1)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "panel width must be in 1.." + std::to_string(nb_max));
    const size_t trsm_smem = sizeof(C) * (size_t)nb * (nb + 64);
    const size_t gemm_smem = sizeof(C) * (size_t)nb * 128;
    FHB_CUDA(cudaFuncSetAttribute(trsm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem));
    FHB_CUDA(cudaFuncSetAttribute(gemm_update_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem));
    for (int64_t k0 = 0; k0 < m; k0 += nb) {
        const int w_nb = (int)std::min<int64_t>(nb, m - k0);
        prof_begin(s, FH_PROF_PANEL);
        if (w.coop) {
            fh_status st = panel_coop<T>(b, k0, w_nb, *w.coop, s, err);
            if (st) return st;
        }
        for (int c = 0; c < w_nb && !w.coop; ++c) {
            const int j = (int)(k0 + c);
            const int chunks = std::min(w.max_chunks, (int)((m - j + 1023) / 1024));
            pivot_kernel<T><<<dim3(chunks, b.count), 256, 0, s>>>(a, m, j, (int)k0, w_nb, b.pivots, b.singular,
                                                                  w.partial_val, w.partial_idx, w.tickets, chunks);
            if (j + 1 < m) {
                const int ublocks = (int)std::max<int64_t>(1, std::min<int64_t>((m - j - 1 + 255) / 256, 64));
                panel_update_kernel<T><<<dim3(ublocks, b.count), 256, 0, s>>>(a, m, j, (int)k0, w_nb);
            }
        }
        const int64_t c0 = k0 + w_nb;
        prof_end(s, FH_PROF_PANEL, 0.0);
        if (c0 >= m) break;
        const int64_t ncols = m - c0;
        prof_begin(s, FH_PROF_TRSM);
        swap_kernel<T><<<dim3(grid_for(ncols, 256, 1024), b.count), 256, 0, s>>>(a, m, (int)k0, w_nb, c0, m,
                                                                                  b.pivots);
        const bool tc_apply = mode == TrailingUpdate::TensorBf16x3 && sizeof(T) == 4 && w_nb % 16 == 0;
        if (w.linv && (tc_apply || w_nb <= 64)) {
            // U12 = L11^{-1} A12 as an explicit triangular inverse times A12:
            // the product runs as a GEMM (tensor cores in the mixed form).
            C *linv = reinterpret_cast<C *>(w.linv);
            const size_t inv_smem = sizeof(C) * (34 * (size_t)w_nb);
            FHB_CUDA(cudaFuncSetAttribute(tri_inverse_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)inv_smem));
            tri_inverse_kernel<T><<<dim3((unsigned)b.count, (unsigned)((w_nb + 31) / 32)), 256, inv_smem, s>>>(
                a, m, (int)k0, w_nb, linv, (int64_t)w_nb * w_nb);
            if (tc_apply) {
                fh_status st = gemm_tc_tri_apply(reinterpret_cast<const float *>(w.linv), w_nb,
                                                 reinterpret_cast<float *>(b.a), m, b.count, k0, s, err);
                if (st) return st;
            } else {
                fh_status st = gemm_simt_assign<T>(linv, w_nb, b.a, m, b.count, k0, w_nb, s, err);
                if (st) return st;
            }
        } else {
            trsm_kernel<T><<<dim3((unsigned)((ncols + 63) / 64), b.count), 64, trsm_smem, s>>>(a, m, (int)k0, w_nb);
        }
        prof_end(s, FH_PROF_TRSM, 4.0 * (double)w_nb * w_nb * ncols * b.count);
        // complex GEMM: 8 real flops per complex multiply-add
        const double flops = 8.0 * (double)ncols * (double)ncols * (double)w_nb * (double)b.count;
        if (mode == TrailingUpdate::TensorBf16x3 && sizeof(T) == 4 && w_nb == nb) {
            prof_begin(s, FH_PROF_GEMM_TC);
            fh_status st = gemm_tc_update(reinterpret_cast<float *>(b.a), m, b.count, k0, nb, s, err);
            prof_end(s, FH_PROF_GEMM_TC, flops);
            if (st) return st;
        } else if constexpr (sizeof(T) == 8) {
            prof_begin(s, FH_PROF_GEMM_FP64);
            fh_status st = dmma_update(b.a, m, b.count, k0, w_nb, s, err);
            prof_end(s, FH_PROF_GEMM_FP64, flops);
            if (st) return st;
        } else {
            prof_begin(s, FH_PROF_GEMM_FP32);
            const unsigned tiles = (unsigned)((ncols + 63) / 64);
            gemm_update_kernel<T><<<dim3(tiles, tiles, b.count), 256, gemm_smem, s>>>(a, m, (int)k0, w_nb);
            prof_end(s, FH_PROF_GEMM_FP32, flops);
        }
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(cudaGetLastError());
    if (w.coop) return coop_check(*w.coop, s, err);
    return FH_OK;
}

template <class T>
fh_status gemm_simt_update(T *av, int64_t m, int count, int64_t k0, int nb, cudaStream_t s, fh_error_info *err) {
    const int64_t ncols = m - k0 - nb;
    if (ncols <= 0) return FH_OK;
    if constexpr (sizeof(T) == 8) return dmma_update(av, m, count, k0, nb, s, err);
    const size_t gemm_smem = sizeof(Cx<T>) * (size_t)nb * 128;
    FHB_CUDA(cudaFuncSetAttribute(gemm_update_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem));
    const unsigned tiles = (unsigned)((ncols + 63) / 64);
    gemm_update_kernel<T><<<dim3(tiles, tiles, count), 256, gemm_smem, s>>>(reinterpret_cast<Cx<T> *>(av), m, (int)k0,
                                                                             nb);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}
// U12 = Linv A12 for the panel [k0, k0+nb): C aliases B (rows k0..k0+nb of
// the columns right of the panel); nb <= 64 so that one CTA row covers M.
template <class T>
fh_status gemm_simt_assign(const void *linv, int nb, T *av, int64_t m, int count, int64_t k0, int K, cudaStream_t s,
                           fh_error_info *err) {
    const int64_t c0 = k0 + nb;
    if (c0 >= m) return FH_OK;
    if (nb > 64) return fail(err, FH_ERR_INVALID_ARGUMENT, "SIMT triangular apply needs nb <= 64");
    Cx<T> *A = reinterpret_cast<Cx<T> *>(av);
    SimtArgs<T> g;
    g.A = reinterpret_cast<const Cx<T> *>(linv);
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
    g.K = K;
    g.assign = 1;
    const size_t smem = sizeof(Cx<T>) * (size_t)K * 128;
    FHB_CUDA(cudaFuncSetAttribute(gemm_simt_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    gemm_simt_kernel<T><<<dim3((unsigned)((g.N + 63) / 64), 1, count), 256, smem, s>>>(g);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}
template fh_status gemm_simt_assign<float>(const void *, int, float *, int64_t, int, int64_t, int, cudaStream_t,
                                           fh_error_info *);
template fh_status gemm_simt_assign<double>(const void *, int, double *, int64_t, int, int64_t, int, cudaStream_t,
                                            fh_error_info *);

template fh_status gemm_simt_update<float>(float *, int64_t, int, int64_t, int, cudaStream_t, fh_error_info *);
template fh_status gemm_simt_update<double>(double *, int64_t, int, int64_t, int, cudaStream_t, fh_error_info *);

template <class T>
fh_status lu_solve(const LuBatch<T> &b, T *xv, int nrhs, int nb, cudaStream_t s, fh_error_info *err, int group) {
    using C = Cx<T>;
    const C *a = reinterpret_cast<const C *>(b.a);
    C *x = reinterpret_cast<C *>(xv);
    const int64_t m = b.m;
    if (m == 0) return FH_OK;
    if (group <= nb) group = nb;
    if (group % nb || group > 4096)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "interchange group must be a multiple of the panel width");
    const int groups = b.count * nrhs;
    const size_t fwd_smem = sizeof(C) * ((size_t)nb * nb + 3 * (size_t)nb) + 2 * sizeof(int) * (size_t)nb;
    const size_t bwd_smem = sizeof(C) * ((size_t)nb * nb + (size_t)nb);
    const size_t swap_smem = (2 * sizeof(C) + 2 * sizeof(int)) * (size_t)group;
    FHB_CUDA(cudaFuncSetAttribute(fwd_panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem));
    FHB_CUDA(cudaFuncSetAttribute(bwd_panel_kernel2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bwd_smem));
    FHB_CUDA(cudaFuncSetAttribute(fwd_swap_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)swap_smem));
    prof_begin(s, FH_PROF_SOLVE);
    for (int64_t g0 = 0; g0 < m; g0 += group) {
        const int wg = (int)std::min<int64_t>(group, m - g0);
        if (group > nb) fwd_swap_kernel<T><<<groups, 128, swap_smem, s>>>(m, nrhs, (int)g0, wg, b.pivots, x);
        for (int64_t k0 = g0; k0 < g0 + wg; k0 += nb) {
            const int w_nb = (int)std::min<int64_t>(nb, g0 + wg - k0);
            fwd_panel_kernel<T><<<groups, 128, fwd_smem, s>>>(a, m, nrhs, (int)k0, w_nb,
                                                              group > nb ? nullptr : b.pivots, x);
            if (k0 + w_nb < m)
                gemv_update_kernel<T><<<dim3(grid_for(m - k0 - w_nb, 256, 64), groups), 256, 0, s>>>(
                    a, m, nrhs, (int)k0, w_nb, k0 + w_nb, m, x);
        }
    }
    const int64_t last = ((m - 1) / nb) * nb;
    for (int64_t k0 = last; k0 >= 0; k0 -= nb) {
        const int w_nb = (int)std::min<int64_t>(nb, m - k0);
        bwd_panel_kernel2<T><<<groups, 128, bwd_smem, s>>>(a, m, nrhs, (int)k0, w_nb, x);
        if (k0 > 0)
            gemv_update_kernel<T><<<dim3(grid_for(k0, 256, 64), groups), 256, 0, s>>>(a, m, nrhs, (int)k0, w_nb, 0,
                                                                                      k0, x);
    }
    prof_end(s, FH_PROF_SOLVE, 8.0 * (double)m * (double)m * nrhs * b.count);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

template <class T>
fh_status form_system(const double *Rm, const double *Lm, int64_t ld, int64_t m, const double *omega, int count, T *a,
                      cudaStream_t s, fh_error_info *err, bool lower_tiles, int64_t mo) {
    if (m == 0) return FH_OK;
    if (mo <= 0) mo = m;
    if (mo < m) return fail(err, FH_ERR_INVALID_ARGUMENT, "form_system: the formed order is below the system's");
    prof_begin(s, FH_PROF_FORM);
    bool pairs = false;
    if constexpr (sizeof(T) == 4) pairs = (mo * mo) % 2 == 0 && (reinterpret_cast<uintptr_t>(a) & 15) == 0;
    if (pairs)
        form_pair_kernel<<<grid_for((mo * mo / 2 + kFormPer - 1) / kFormPer, 256, 148 * 16), 256, 0, s>>>(
            Rm, Lm, ld, m, mo, omega, count, reinterpret_cast<float4 *>(a), lower_tiles ? 1 : 0);
    else if (mo == m)
        form_kernel<T><<<grid_for(m * m, 256, 148 * 16), 256, 0, s>>>(Rm, Lm, ld, m, omega, count,
                                                                       reinterpret_cast<Cx<T> *>(a));
    else
        return fail(err, FH_ERR_INVALID_ARGUMENT, "form_system: a bordered system needs the paired FP32 form");
    // bytes written: every entry of every frequency (about half with lower_tiles)
    prof_end(s, FH_PROF_FORM, (double)mo * (double)mo * count * 2.0 * sizeof(T));
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

template <class T>
fh_status form_rhs(const double *Rm, const double *Lm, int64_t ld, int64_t m, int64_t p, const double *omega, int count,
                   T *b, cudaStream_t s, fh_error_info *err) {
    if (m == 0 || p == 0) return FH_OK;
    rhs_kernel<T><<<grid_for(m * p * count, 256), 256, 0, s>>>(Rm, Lm, ld, m, p, omega, count,
                                                               reinterpret_cast<Cx<T> *>(b));
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

// t[g n + b] = R_b sum over the internal loops of branch b of s x[g m + loop].
__global__ void sparse_rt_kernel(const Cx<double> *__restrict__ x, int64_t m, int64_t n, int64_t G,
                                 const int64_t *__restrict__ t_off, const int32_t *__restrict__ t_loop,
                                 const double *__restrict__ t_sign, const double *__restrict__ R,
                                 Cx<double> *__restrict__ t) {
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < G * n;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = idx / n, b = idx % n;
        double re = 0.0, im = 0.0;
        for (int64_t e = t_off[b]; e < t_off[b + 1]; ++e) {
            const Cx<double> v = x[g * m + t_loop[e]];
            re += t_sign[e] * v.re;
            im += t_sign[e] * v.im;
        }
        t[idx] = Cx<double>{R[b] * re, R[b] * im};
    }
}
// y[g m + i] = sum over the branches of loop i of s t[g n + branch].
__global__ void sparse_ry_kernel(const Cx<double> *__restrict__ t, int64_t m, int64_t n, int64_t G,
                                 const int64_t *__restrict__ row_ptr, const int32_t *__restrict__ branch,
                                 const double *__restrict__ sign, Cx<double> *__restrict__ y) {
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < G * m;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = idx / m, i = idx % m;
        double re = 0.0, im = 0.0;
        for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
            const Cx<double> v = t[g * n + branch[e]];
            re += sign[e] * v.re;
            im += sign[e] * v.im;
        }
        y[idx] = Cx<double>{re, im};
    }
}

int residual_splits(int64_t m, int64_t p, int count) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const int64_t tiles = ((m + kResRows - 1) / kResRows) * (((int64_t)count * p + kResCols - 1) / kResCols);
    const int64_t stages = (m + kResK - 1) / kResK;
    // about 16 CTAs per SM over the launch, each range at least 16 stages
    const int64_t want = (16 * (int64_t)sms + tiles - 1) / std::max<int64_t>(1, tiles);
    return (int)std::max<int64_t>(1, std::min<int64_t>({want, kResMaxSplits, stages / 16}));
}

size_t residual_scratch_bytes(int64_t m, int64_t p, int count) {
    const int splits = residual_splits(m, p, count);
    return splits > 1 ? (size_t)splits * (size_t)count * (size_t)p * (size_t)m * sizeof(double4) : 0;
}

fh_status residual_fp64(const double *Rm, const double *Lm, int64_t ld, int64_t m, int64_t p, const double *omega,
                        int count, const double *x, double *r, double *rnorm, cudaStream_t s, fh_error_info *err,
                        void *scratch, const SparseR *sr) {
    if (m == 0) return FH_OK;
    const int64_t cols = (int64_t)count * p;
    const int splits = scratch ? residual_splits(m, p, count) : 1;
    double4 *part = splits > 1 ? static_cast<double4 *>(scratch) : nullptr;
    prof_begin(s, FH_PROF_RESIDUAL);
    const Cx<double> *rx = nullptr;
    if (sr) {
        Cx<double> *t = reinterpret_cast<Cx<double> *>(sr->t), *y = reinterpret_cast<Cx<double> *>(sr->y);
        sparse_rt_kernel<<<grid_for(cols * sr->n, 256), 256, 0, s>>>(reinterpret_cast<const Cx<double> *>(x), m,
                                                                     sr->n, cols, sr->t_off, sr->t_loop, sr->t_sign,
                                                                     sr->R, t);
        sparse_ry_kernel<<<grid_for(cols * m, 256), 256, 0, s>>>(t, m, sr->n, cols, sr->row_ptr, sr->branch, sr->sign,
                                                                 y);
        rx = y;
    }
    const dim3 rgrid((unsigned)((m + kResRows - 1) / kResRows), (unsigned)((cols + kResCols - 1) / kResCols),
                     (unsigned)(part ? splits : 1));
    if (rx)
        residual_kernel<false><<<rgrid, kResThreads, 0, s>>>(Rm, Lm, ld, m, p, omega, count,
                                                             reinterpret_cast<const Cx<double> *>(x),
                                                             reinterpret_cast<Cx<double> *>(r), part, rx);
    else
        residual_kernel<true><<<rgrid, kResThreads, 0, s>>>(Rm, Lm, ld, m, p, omega, count,
                                                            reinterpret_cast<const Cx<double> *>(x),
                                                            reinterpret_cast<Cx<double> *>(r), part, nullptr);
    if (part)
        residual_finish_kernel<<<grid_for(cols * m, 256), 256, 0, s>>>(Rm, Lm, ld, m, p, omega, count, splits, part,
                                                                      reinterpret_cast<Cx<double> *>(r), rx);
    prof_end(s, FH_PROF_RESIDUAL, (sr ? 8.0 : 16.0) * (double)m * (double)m);  // bytes: L (and R) read once
    FHB_CUDA(cudaGetLastError());
    if (rnorm) {
        max_abs_kernel<double><<<count, 256, 0, s>>>(r, 2 * m * p, rnorm);
        FHB_CUDA(cudaGetLastError());
    }
    return FH_OK;
}

fh_status schur(const double *Rm, const double *Lm, int64_t ld, int64_t m, int64_t p, const double *omega, int count,
                const double *x, double *z, cudaStream_t s, fh_error_info *err) {
    if (p == 0 || count == 0) return FH_OK;
    schur_kernel<<<(unsigned)(count * p * p), 256, 0, s>>>(Rm, Lm, ld, m, p, omega,
                                                           reinterpret_cast<const Cx<double> *>(x),
                                                           reinterpret_cast<Cx<double> *>(z));
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

fh_status convert_c64_to_c32(const double *src, float *dst, int64_t n, cudaStream_t s, fh_error_info *err, int64_t m,
                             int64_t mo) {
    if (!n) return FH_OK;
    if (mo > m && m > 0) {
        const int64_t cols = n / m;
        c64_to_c32_border_kernel<<<grid_for(2 * mo * cols, 256), 256, 0, s>>>(src, dst, m, mo, cols);
    } else {
        c64_to_c32_kernel<<<grid_for(2 * n, 256), 256, 0, s>>>(src, dst, n);
    }
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

fh_status add_c32_to_c64(double *x, const float *d, int64_t n, cudaStream_t s, fh_error_info *err, int64_t m,
                         int64_t mo) {
    if (!n) return FH_OK;
    if (mo > m && m > 0) {
        const int64_t cols = n / m;
        add_c32_border_kernel<<<grid_for(2 * m * cols, 256), 256, 0, s>>>(x, d, m, mo, cols);
    } else {
        add_c32_kernel<<<grid_for(2 * n, 256), 256, 0, s>>>(x, d, n);
    }
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

fh_status max_abs_per_matrix(const double *v, int64_t per, int count, double *out, cudaStream_t s, fh_error_info *err) {
    if (!count) return FH_OK;
    max_abs_kernel<double><<<count, 256, 0, s>>>(v, per, out);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

fh_status max_abs_per_matrix_f32(const float *v, int64_t per, int count, double *out, cudaStream_t s,
                                 fh_error_info *err) {
    if (!count) return FH_OK;
    max_abs_kernel<float><<<count, 256, 0, s>>>(v, per, out);
    FHB_CUDA(cudaGetLastError());
    return FH_OK;
}

template fh_status lu_factor<double>(LuBatch<double> &, LuWork &, int, TrailingUpdate, cudaStream_t, fh_error_info *);
template fh_status lu_factor<float>(LuBatch<float> &, LuWork &, int, TrailingUpdate, cudaStream_t, fh_error_info *);
template fh_status lu_solve<double>(const LuBatch<double> &, double *, int, int, cudaStream_t, fh_error_info *, int);
template fh_status lu_solve<float>(const LuBatch<float> &, float *, int, int, cudaStream_t, fh_error_info *, int);
template fh_status form_system<double>(const double *, const double *, int64_t, int64_t, const double *, int, double *,
                                       cudaStream_t, fh_error_info *, bool, int64_t);
template fh_status form_system<float>(const double *, const double *, int64_t, int64_t, const double *, int, float *,
                                      cudaStream_t, fh_error_info *, bool, int64_t);
template fh_status form_rhs<double>(const double *, const double *, int64_t, int64_t, int64_t, const double *, int,
                                    double *, cudaStream_t, fh_error_info *);
template fh_status form_rhs<float>(const double *, const double *, int64_t, int64_t, int64_t, const double *, int,
                                   float *, cudaStream_t, fh_error_info *);

}  // namespace fhb
