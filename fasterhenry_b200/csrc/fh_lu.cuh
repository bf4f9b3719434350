// Batched blocked complex LU with partial pivoting (device), its solves, the
// FP64 residual of R + jwL, and the Schur complement.
#pragma once

#include <cuda_runtime.h>

#include "fh_device.cuh"

namespace fhb {

// A batch of `count` column-major complex matrices of order m (leading
// dimension m), stored back to back with stride m*m complex entries.
// T is double (FP64 form) or float (mixed form).
template <class T>
struct LuBatch {
    T *a = nullptr;          // interleaved complex, count * m * m
    int *pivots = nullptr;   // count * m: row interchanged with row k
    int *singular = nullptr; // count flags (zero pivot met)
    int64_t m = 0;
    int count = 0;
};

// Scratch of the cooperative panel factorization (fh_panel.cu).
struct CoopScratch {
    unsigned *barrier = nullptr;  // arrivals, generation
    int *error = nullptr;         // set when a bounded grid barrier gives up
    double *cand_val = nullptr;   // pivot candidates, count * per_matrix * 2
    int *cand_row = nullptr;
    void *cand_data = nullptr;    // candidate rows, count * per_matrix * 2 * 128 complex
    void *rowj = nullptr;         // row j of each matrix, count * 2 * 128 complex
    int per_matrix = 0;           // CTAs per matrix
    bool cluster = false;         // the CTAs of a matrix form one thread-block cluster
};

// Workspace for the factorization (pivot search partials).  With `coop`
// set, panels are factored by the cooperative kernel; without it, one column
// at a time (pivot search + rank-1 update launches).
struct LuWork {
    double *partial_val = nullptr;
    int *partial_idx = nullptr;
    unsigned *tickets = nullptr;
    int max_chunks = 0;
    const CoopScratch *coop = nullptr;
    // count * nb * nb complex T: with it, U12 = L11^{-1} A12 is formed from
    // the explicit triangular inverse and a GEMM; without it, by the
    // column-at-a-time TRSM kernel.  With `outer` set it holds one slot per
    // nb-block of the matrix (ceil(m / nb) slots, slot j0 / nb, matrices
    // back to back within a slot), kept for lu_solve_inv.
    void *linv = nullptr;
    // With `outer` set: the inverses of the diagonal nb x nb blocks of U,
    // laid out like linv (optional; lu_solve_inv needs them).
    void *uinv = nullptr;
    // Two-level blocking (FP32 form on the tensor cores): super-panels of
    // `outer` columns are factored with nb-wide panels and updates confined
    // to the super-panel; the rest of the matrix then takes one deep update
    // with K = outer from the packed operands in pack_a / pack_b
    // (packed_operand_bytes(m, outer, count) each).  Row interchanges of a
    // panel are applied to every column of its super-panel, so lu_solve must
    // be called with group = outer.
    int outer = 0;
    void *pack_a = nullptr;
    void *pack_b = nullptr;
    // Two-level form without pivoting (for matrices with symmetric positive
    // definite real and imaginary parts): each diagonal block is factored
    // in shared memory and L21 = A21 U11^-1 formed on the tensor cores;
    // pivots are the identity.
    bool nopivot = false;
    // With the no-pivot form: whether U12 beyond each super-panel's diagonal
    // region is written in FP32.  A solve that takes U_ij = D_i L_ji^T
    // (lu_solve_flow) reads no U entry outside the diagonal regions.
    bool upper = true;
    // Scratch of the factorization without pivoting, for the rows below each
    // super-panel (one super-panel at a time; outer = W columns):
    //   xinv  count * W * W complex FP32: X = U_D^{-1} of the super-panel's
    //         diagonal block D (column-major, leading dimension W);
    //   xpack packed_operand_bytes(W, W, count): X packed as a B operand;
    //   tbuf  count * nb * (W - nb) complex FP32: one block row product;
    //   dvec  2 * count * W complex FP32: the diagonal d of U_D, then its
    //         principal square roots s (matrix f's at count * W + f * W).
    // With all four set, L21, U12 and the packed operand of the deep update
    // come from one tensor-core pass over the rows below (gemm_tc_panel_solve).
    void *xinv = nullptr;
    void *xpack = nullptr;
    void *tbuf = nullptr;
    void *dvec = nullptr;
    // Look-ahead of the fused form (both given): each super-panel's diagonal
    // region, X and its packing run on `side` while the bulk of the previous
    // deep update runs on the factorization's stream on all SMs but a few,
    // drawing its tiles from tile_counter; when the side stream's work is
    // done a second grid on it joins the update and takes those SMs back.
    cudaStream_t side = nullptr;
    int *tile_counter = nullptr;
};

// Cooperative panel: sizing, binding of a scratch block, launch, error check.
// `share`: the number of cooperative launches that may run at once on the
// device (concurrent sweeps); each is sized to 1 / share of the resident
// capacity so that all of them are co-resident together.
template <class T>
fh_status coop_plan(int count, int64_t m, int *per_matrix, size_t *bytes, fh_error_info *err, int share = 1);
template <class T>
void coop_bind(void *mem, int count, int per_matrix, CoopScratch &cs, int share = 1);
// Whether coop_plan's per_matrix CTAs of type T run as one cluster per
// matrix: when every cluster of `count` matrices (times `share` concurrent
// sweeps) is resident at once.
template <class T>
bool coop_cluster(int count, int per_matrix, int share = 1);
template <class T>
fh_status panel_coop(LuBatch<T> &b, int64_t K0, int nb, const CoopScratch &cs, cudaStream_t s, fh_error_info *err);
fh_status coop_check(const CoopScratch &cs, cudaStream_t s, fh_error_info *err);

// How the trailing update A22 -= L21 U12 is computed for the FP32 form.
enum class TrailingUpdate { Simt, TensorBf16x3 };

template <class T>
fh_status lu_factor(LuBatch<T> &b, LuWork &w, int nb, TrailingUpdate mode, cudaStream_t s, fh_error_info *err);

// One trailing update A22 -= L21 U12 of the panel [k0, k0+nb) on the tensor
// cores (split-BF16 x3), for every matrix of an FP32 batch.
fh_status gemm_tc_update(float *a, int64_t m, int count, int64_t k0, int nb, cudaStream_t s, fh_error_info *err);
// Reports (and clears) a bounded tensor-core wait that ran out.
fh_status gemm_tc_check(fh_error_info *err);
// General strided form of the same kernel: C (M x N) -= A (M x K) B (K x N)
// (assign == 0), C = A B (assign == 1; C may alias B when M <= 128, or A when
// N <= 128) or C = -A B (assign == 2, same aliasing rule).
// Complex FP32 operands, element (r, k) of A at A[2 (f sA + r + k lda)].
fh_status gemm_tc_strided(const float *A, int64_t lda, int64_t sA, const float *B, int64_t ldb, int64_t sB, float *C,
                          int64_t ldc, int64_t sC, int64_t M, int64_t N, int K, int assign, int count, cudaStream_t s,
                          fh_error_info *err);
// Bytes of one packed operand (rows rounded up to 128, K a multiple of 16).
size_t packed_operand_bytes(int64_t rows, int K, int count);
// C (M x N) -= A (M x K) B (K x N), complex FP32, strided as above: both
// operands split into BF16 hi/lo and packed into pack_a / pack_b, then the
// persistent warp-specialized tensor-core kernel (fh_gemm_packed.cu).
fh_status gemm_tc_packed_update(const float *A, int64_t lda, int64_t sA, const float *B, int64_t ldb, int64_t sB,
                                float *C, int64_t ldc, int64_t sC, int64_t M, int64_t N, int K, int count,
                                void *pack_a, void *pack_b, cudaStream_t s, fh_error_info *err, int lower_from = -1);
// The deep update from operands already packed (layout of pack_a / pack_b
// above), one CTA per SM.  lower_from >= 0: column blocks (of 128) below it
// in full, the rest on and below the diagonal tile only; col_lo / col_hi
// restrict it to the column blocks in [col_lo, col_hi) (col_hi < 0: to the
// end).
fh_status gemm_tc_packed_run(const void *pack_a, const void *pack_b, float *C, int64_t ldc, int64_t sC, int64_t M,
                             int64_t N, int K, int count, cudaStream_t s, fh_error_info *err, int lower_from = -1,
                             int col_lo = 0, int col_hi = -1);
// The same update as a schedule (its tile table on the device) launched as
// one or more grids: with a tile counter (zeroed before the first launch,
// in stream order) the grids draw tiles from it, so a grid on a second
// stream can join an update already running on fewer SMs.  The release
// frees the table in stream order on s, after every launch it follows.
struct PackedSchedule {
    const void *pack_a = nullptr, *pack_b = nullptr;
    float *C = nullptr;
    int64_t ldc = 0, sC = 0, M = 0, N = 0;
    int K = 0, count = 0;
    uint32_t *table = nullptr;
    long long per_matrix = 0, tiles = 0;
    double entries = 0.0;  // complex C entries per matrix
};
fh_status gemm_tc_packed_schedule(PackedSchedule &ps, const void *pack_a, const void *pack_b, float *C, int64_t ldc,
                                  int64_t sC, int64_t M, int64_t N, int K, int count, int lower_from, int col_lo,
                                  int col_hi, cudaStream_t s, fh_error_info *err);
// grid <= 0: one CTA per SM; next: the tile counter or nullptr (every
// grid-th tile per CTA).  prof_class: the event profiler's class of the
// launch, or -1 to leave it out (a grid joining an update whose first grid
// is timed: its time lies inside that grid's, its work is counted there).
fh_status gemm_tc_packed_launch(const PackedSchedule &ps, int grid, int *next, cudaStream_t s, fh_error_info *err,
                                int prof_class = FH_PROF_GEMM_TC);
void gemm_tc_packed_release(PackedSchedule &ps, cudaStream_t s);
int gemm_tc_sm_count();
// Packs B (K x N, element (k, n) at B[2 (f sB + k + n ldb)]) as a B operand.
fh_status gemm_tc_pack_b(const float *B, int64_t ldb, int64_t sB, int64_t N, int K, int count, void *out,
                         cudaStream_t s, fh_error_info *err);
// For the factored super-panel [K0, K0 + W) of a complex symmetric batch
// factored without interchanges and the rows below it: L21 = A21 X in place
// (X = U_D^{-1}, xpack from gemm_tc_pack_b), U12 = diag(d) L21^T over the
// super-panel's rows of the trailing columns (if write_u12), and P = L21 diag(s) packed into
// pack (s_k^2 = d_k): the deep update C -= L21 U12 = P P^T takes P as both
// its A and its B operand.  The rows are read by 2D tensor copies, so the
// order m must be even (a column stride of 16-byte multiples).
bool panel_solve_supported(int64_t m);
fh_status gemm_tc_panel_solve(float *a, int64_t m, int count, int64_t K0, int W, const void *xpack, const float *dvec,
                              const float *svec, void *pack, bool write_u12, cudaStream_t s, fh_error_info *err);
fh_status gemm_tc_packed_check(fh_error_info *err);
// One SIMT trailing update (FP32 or FP64), for tests.
template <class T>
fh_status gemm_simt_update(T *a, int64_t m, int count, int64_t k0, int nb, cudaStream_t s, fh_error_info *err);
// The FP64 form of the same update on the FP64 tensor cores (mma.sync m8n8k4
// f64, fh_dmma.cu): A22 -= L21 U12 for panel [k0, k0 + nb) of `count`
// complex column-major m x m matrices.
fh_status dmma_update(double *a, int64_t m, int count, int64_t k0, int nb, cudaStream_t s, fh_error_info *err);
// U12 = Linv A12 of panel [k0, k0+nb) in place (tensor cores / SIMT).
fh_status gemm_tc_tri_apply(const float *linv, int nb, float *a, int64_t m, int count, int64_t k0, cudaStream_t s,
                            fh_error_info *err);
template <class T>
fh_status gemm_simt_assign(const void *linv, int nb, T *a, int64_t m, int count, int64_t k0, int K, cudaStream_t s,
                           fh_error_info *err);

// Solve with the factors in place: x (count x m x nrhs, column-major per
// matrix, stride m*nrhs) is overwritten.  `group` is the span of columns
// whose L entries carry each other's row interchanges (nb for the one-level
// factorization, LuWork::outer for the two-level one).
template <class T>
fh_status lu_solve(const LuBatch<T> &b, T *x, int nrhs, int nb, cudaStream_t s, fh_error_info *err, int group = 0);

// Cooperative forward + backward solve with the two-level FP32 factors
// (fh_trisolve.cu): one launch, groups of CTAs per (matrix, right-hand side)
// meeting at their own bounded barriers, diagonal blocks applied through the
// inverses kept in LuWork::linv / uinv.
struct SolveScratch {
    unsigned *barrier = nullptr;
    int *error = nullptr;  // must start at zero
    int groups = 0;        // count * nrhs
    int per_group = 0;     // CTAs per group; 0 = the batch does not fit one launch
};
fh_status trisolve_plan(int groups, int64_t m, int *per_group, size_t *bytes, fh_error_info *err, int share = 1);
void trisolve_bind(void *mem, int groups, int per_group, SolveScratch &ss);
fh_status lu_solve_inv(const LuBatch<float> &b, const void *linv, const void *uinv, float *x, int nrhs, int nb,
                       int group, const SolveScratch &ss, cudaStream_t s, fh_error_info *err);
fh_status trisolve_check(const SolveScratch &ss, cudaStream_t s, fh_error_info *err);

// Tensor map (a CUtensorMap, 64-byte aligned, at map) of a batch of count
// column-major m x m complex FP32 matrices seen as one m x (count m) array
// of 8-byte elements, box box_rows x box_cols; m must be even.
fh_status encode_column_tiles(void *map, const float *a, int64_t m, int count, int box_rows, int box_cols,
                              fh_error_info *err);

// Dataflow form of the same solves for factors without interchanges
// (fh_flowsolve.cu): a flag per 128-row block instead of barriers, the
// factor tiles loaded by TMA.  The scratch (flowsolve_plan's bytes) must be
// zeroed once per batch; per_group = 0 means the batch does not fit one
// launch or the order is odd (the barrier-based solve is used instead).
struct FlowScratch {
    unsigned *flags = nullptr;  // [group][2][nblk]
    int *error = nullptr;
    int groups = 0, per_group = 0, nblk = 0;
    unsigned epoch = 0;  // the flag value of the last launch
};
fh_status flowsolve_plan(int groups, int64_t m, int *per_group, size_t *bytes, fh_error_info *err, int share = 1);
void flowsolve_bind(void *mem, int groups, int per_group, int64_t m, FlowScratch &fs);
fh_status lu_solve_flow(const LuBatch<float> &b, const void *linv, const void *uinv, float *x, int nrhs,
                        FlowScratch &fs, cudaStream_t s, fh_error_info *err);
fh_status flowsolve_check(const FlowScratch &fs, cudaStream_t s, fh_error_info *err);

// A_f = R + j w_f L for the top-left m x m block of R_m, L_m (ld = loops),
// written as T complex into a (count x m x m).  With lower_tiles (FP32, for
// the two-level factorization without pivoting, which forms every U entry it
// reads from L) the 128 x 128 tiles above the diagonal are not written.  With
// mo > m (FP32 only) each matrix has order mo and is bordered by the identity:
// [A_f 0; 0 I].
template <class T>
fh_status form_system(const double *Rm, const double *Lm, int64_t ld, int64_t m, const double *omega, int count,
                      T *a, cudaStream_t s, fh_error_info *err, bool lower_tiles = false, int64_t mo = 0);

// Right-hand sides b_f = Z_ep (m x p) at each frequency, as T complex.
template <class T>
fh_status form_rhs(const double *Rm, const double *Lm, int64_t ld, int64_t m, int64_t p, const double *omega,
                   int count, T *b, cudaStream_t s, fh_error_info *err);

// r_f = b_f - (R_ee + j w_f L_ee) x_f in FP64 for all f at once (one pass
// over R_ee and L_ee).  x, b, r: count x m x p complex double.  Also returns
// per-frequency max-norms of r and b through rnorm/bnorm (device, count each).
// With scratch (residual_scratch_bytes; 0 means none is used) the k range is
// split across CTAs and the ranges' sums are added in a fixed order.
size_t residual_scratch_bytes(int64_t m, int64_t p, int count);
// R_ee through the loop basis, R_ee = M_e diag(R) M_e^T: y = M_e (R (M_e^T x))
// costs O(loop entries) per column instead of the m^2 of the dense R_ee.
// row_ptr / branch / sign: the basis rows (the first m used); t_off /
// t_loop / t_sign: per branch (n + 1 offsets) its internal loops in
// increasing order; R: branch resistances; t (G x n) and y (G x m complex)
// scratch, G = count p.
struct SparseR {
    const int64_t *row_ptr = nullptr;
    const int32_t *branch = nullptr;
    const double *sign = nullptr;
    const int64_t *t_off = nullptr;
    const int32_t *t_loop = nullptr;
    const double *t_sign = nullptr;
    const double *R = nullptr;
    int64_t n = 0;
    double *t = nullptr;
    double *y = nullptr;
};
// With sr, R_ee x comes from the loop basis and the dense pass reads L_ee only.
fh_status residual_fp64(const double *Rm, const double *Lm, int64_t ld, int64_t m, int64_t p, const double *omega,
                        int count, const double *x, double *r, double *rnorm, cudaStream_t s, fh_error_info *err,
                        void *scratch = nullptr, const SparseR *sr = nullptr);

// Z_f = Z_pp - Z_ep^T X_f (p x p complex, row-major per frequency).
fh_status schur(const double *Rm, const double *Lm, int64_t ld, int64_t m, int64_t p, const double *omega, int count,
                const double *x, double *z, cudaStream_t s, fh_error_info *err);

// Elementwise helpers.  With mo > m, the FP64 side holds columns of m
// entries and the FP32 side columns of mo entries (the bordered system):
// conversion writes the border entries as zero, the addition skips them.
fh_status convert_c64_to_c32(const double *src, float *dst, int64_t n_complex, cudaStream_t s, fh_error_info *err,
                             int64_t m = 0, int64_t mo = 0);
fh_status add_c32_to_c64(double *x, const float *d, int64_t n_complex, cudaStream_t s, fh_error_info *err,
                         int64_t m = 0, int64_t mo = 0);
fh_status max_abs_per_matrix(const double *v, int64_t per_matrix, int count, double *out, cudaStream_t s,
                             fh_error_info *err);
fh_status max_abs_per_matrix_f32(const float *v, int64_t per_matrix, int count, double *out, cudaStream_t s,
                                 fh_error_info *err);

}  // namespace fhb
