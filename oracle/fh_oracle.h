/*
 * CPU oracle for the fasterhenry PEEC dense path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++17 restatement of the reference algorithm (2AMLogic/fasterhenry,
 * Rust) for the path geometry -> filaments -> loop basis -> partial-inductance
 * fill -> congruence -> per-frequency complex LU + Schur complement.  Each
 * function in fh_oracle.cpp cites the reference file:line it restates.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline and
 * reference legs) may load this library, and only as the checker or as the
 * timed CPU baseline.  The product library (fasterhenry_b200/) never links,
 * loads or calls it.
 *
 * Parity pinning: the reference cannot be built here (no Rust toolchain), so
 * the restatement is pinned against the reference's own known-answer tests
 * (unit-cube self-potential, closed-form self inductances, Grover/Rosa
 * limits, circuit identities); see tests/test_oracle_known_answers.py and
 * tests/golden/known_answers.json.
 */
#ifndef FH_ORACLE_H
#define FH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Segment as stored in a geometry: node indices plus the cross-section. */
typedef struct orc_segment {
    long long a, b;
    double width, height, sigma;
    long long has_width_dir;
    double width_dir[3];
} orc_segment;

/* Per-segment grid (nw x nh, ratios >= 1). */
typedef struct orc_axis_grading {
    long long nw, nh;
    double width_ratio, height_ratio;
} orc_axis_grading;

/* kind: 0 uniform, 1 per-segment, 2 graded, 3 skin-depth, 4 per-segment graded */
typedef struct orc_discretization {
    long long kind;
    long long nw, nh;
    double ratio;
    double frequency_hz, target_skin_depths;
    long long max_per_axis;
    const orc_axis_grading *per_segment;
    long long per_segment_len;
} orc_discretization;

/* Filament record: 19 doubles
 * [0..3) start, [3..6) end, [6] length, [7..10) length dir, [10..13) width dir,
 * [13..16) height dir, [16] width, [17] height, [18] sigma */
#define ORC_FILAMENT_DOUBLES 19

/* Methods (inductance/mod.rs:130) */
enum { ORC_ORTHOGONAL = 0, ORC_BAR_CLOSED_FORM = 1, ORC_ALIGNED_QUADRATURE = 2,
       ORC_POINT_QUADRATURE = 3, ORC_SAMPLED_FILAMENTS = 4 };

/* Status codes (subset of SolveError / KernelError variants) */
enum { ORC_OK = 0, ORC_ERR_ARGUMENT = 1, ORC_ERR_DISCRETIZE = 2, ORC_ERR_COINCIDENT = 3,
       ORC_ERR_NOT_FINITE = 4, ORC_ERR_MESH = 5, ORC_ERR_GRADING = 6, ORC_ERR_FREQUENCY = 7,
       ORC_ERR_SINGULAR = 8 };

void orc_gauss_rule(int n, double *nodes, double *weights);
int orc_order_for(double tolerance, int max_order, double half_extent, double distance);

int orc_discretize(const double *nodes, long long nnode, const orc_segment *segs, long long nseg,
                   const orc_discretization *disc, double *filaments, long long cap,
                   long long *nfil, long long *per_segment);

/* Loop basis as CSR rows (branch, sign). */
int orc_mesh(const orc_segment *segs, long long nseg, long long nnode, const long long *per_segment,
             const long long *ports, long long nport, long long *row_ptr, long long *cols,
             double *signs, long long cap_rows, long long cap_nnz, long long *nrows,
             long long *nnz, long long *internal);

int orc_mutual(const double *fa, const double *fb, double *value, int *method, int *resolved);
double orc_self_inductance(const double *f);
void orc_bar_integral(const double *qx, const double *qy, const double *qz, double *value,
                      double *relative_error);
double orc_aligned_quadrature(const double *length2, const double *width2,
                              const double *height2, const double *offset3);
double orc_lines_parallel(double l1, double l2, double offset, double rho, int *ok);
double orc_lines_skew(const double *a0, const double *a1, const double *b0, const double *b1,
                      double sin_min, int *ok);
double orc_separation(const double *fa, const double *fb);

/* n x n partial inductance matrix, column-major; methods (optional, n*n, int8). */
int orc_fill(const double *filaments, long long n, double *L, signed char *methods, int threads,
             long long *err_i, long long *err_j);

/* The fill with every dispatch decision (method, orders, closed-form
 * acceptance, aligned-quadrature break points and panel tree) taken on
 * `nominal` and the arithmetic done on `perturbed` (same count and order):
 * the frozen-dispatch evaluation that finite-difference checks of the
 * impedance gradient differentiate.  Sampled-filament pairs: ORC_ERR_ARGUMENT. */
int orc_fill_frozen(const double *nominal, const double *perturbed, long long n, double *L, int threads);
/* The same for rows[0..nrows) of the matrix: out[r * n + j] = L(rows[r], j). */
int orc_fill_frozen_rows(const double *nominal, const double *perturbed, long long n, const long long *rows,
                         long long nrows, double *out, int threads);

/* Solve a (n x n, complex interleaved, column-major) x = b in place (b: n x nrhs).
 * Returns ORC_ERR_SINGULAR on an exactly zero pivot. */
int orc_lu_solve(double *a, long long n, double *b, long long nrhs, int threads);
// near_pairs (pfft/near.rs:41-106) in CSR form; *total may exceed cap.
int orc_near_pairs(const double *filaments, long long n, double radius, long long *off, long long *cols,
                   long long cap, long long *total);
// The same solve through the reference's column-at-a-time sweeps on one thread
// (dense.rs:98-190); equal bits to orc_lu_solve.
int orc_lu_solve_plain(double *a, long long n, double *b, long long nrhs);

/* Whole dense system (MeshSystem). */
typedef struct orc_system orc_system;
int orc_system_assemble(const double *nodes, long long nnode, const orc_segment *segs,
                        long long nseg, const long long *ports, long long nport,
                        const orc_discretization *disc, int threads, orc_system **out,
                        double *timing3 /* inductance_s, assembly_s, fill pairs */);
void orc_system_counts(const orc_system *s, long long *counts6);
/* R_m, L_m as full (loops x loops) column-major; filaments (n x 19). */
void orc_system_blocks(const orc_system *s, double *r_mesh, double *l_mesh);
void orc_system_filaments(const orc_system *s, double *filaments);
void orc_system_inductance(const orc_system *s, double *L);
/* Z at one frequency: p x p complex interleaved, row-major (impedance_ohm[i][j]). */
int orc_system_impedance(const orc_system *s, double frequency, double *z, int threads);
void orc_system_free(orc_system *s);

#ifdef __cplusplus
}
#endif
#endif
