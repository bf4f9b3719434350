/*
 * fasterhenry_b200 — C ABI of the B200 (sm_100a) PEEC extraction path.
 *
 * The reference (2AMLogic/fasterhenry) is a Rust library; its hot path is the
 * dense extraction
 *     geometry -> filaments -> loop basis M -> partial inductance L (fill)
 *     -> R_m = M R M^T, L_m = M L M^T (congruence)
 *     -> per frequency: Z(w) = Z_pp - Z_ep^T (R_ee + jwL_ee)^-1 Z_ep  (LU + Schur)
 * plus the matrix-free pFFT + GMRES alternative.  Each entry point below
 * names the reference interface it replaces (paths relative to the reference
 * project root).  A Rust crate binds these with `extern "C"` declarations;
 * the Python package binds them with ctypes.
 *
 * Conventions
 *   - Plain pointers and sizes; all buffers are caller-owned HOST memory
 *     unless a function says otherwise.  Opaque handles own device memory.
 *   - SI units: metres, S/m, hertz, ohms, henries.
 *   - Complex numbers are interleaved (re, im) doubles.
 *   - Every function returns an fh_status; on failure the optional
 *     fh_error_info out-struct carries the payload the reference's
 *     SolveError / KernelError variant would carry, and fh_last_error()
 *     returns a thread-local message.
 *   - There is no CPU fallback: without a usable CUDA device every compute
 *     entry point returns FH_ERR_NO_DEVICE.
 */
#ifndef FASTERHENRY_B200_H
#define FASTERHENRY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FH_ABI_VERSION 1

/* Status codes.  The FH_ERR_* values between 10 and 29 map 1:1 onto the
 * reference's error variants: SolveError (fasterhenry/src/solve.rs:567-637),
 * KernelError (fasterhenry/src/inductance/mod.rs:93-115), MeshError
 * (fasterhenry/src/mesh.rs:94-144), DiscretizeError
 * (fasterhenry/src/filament.rs:141-190), GeometryError
 * (fasterhenry/src/geometry.rs:296-324). */
typedef enum fh_status {
    FH_OK = 0,
    FH_ERR_INVALID_ARGUMENT = 1,   /* null pointer, size mismatch (reference: panic) */
    FH_ERR_NO_DEVICE = 2,          /* no CUDA device / extension unusable */
    FH_ERR_CUDA = 3,               /* a CUDA runtime call failed */
    FH_ERR_OUT_OF_MEMORY = 4,      /* device allocation failed */
    FH_ERR_DEVICE_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    FH_ERR_GEOMETRY = 10,          /* GeometryError::{NonFiniteNode, DanglingNode, InvalidSegment} */
    FH_ERR_DISCRETIZE = 11,        /* SolveError::Discretize{segment, source} */
    FH_ERR_KERNEL_COINCIDENT = 12, /* KernelError::CoincidentSamples{first, second} */
    FH_ERR_KERNEL_NOT_FINITE = 13, /* KernelError::NotFinite{first, second} */
    FH_ERR_MESH = 14,              /* SolveError::Mesh(MeshError) */
    FH_ERR_INVALID_GRADING = 15,   /* SolveError::InvalidGrading */
    FH_ERR_INVALID_FREQUENCY = 16, /* SolveError::InvalidFrequency{index, value} */
    FH_ERR_SINGULAR = 17,          /* SolveError::Singular{frequency} */
    FH_ERR_NOT_CONVERGED = 18,     /* SolveError::NotConverged{frequency, port, iterations, residual};
                                      also: mixed-precision refinement that did not reach its target */
    FH_ERR_PFFT = 19,              /* SolveError::Pfft(PfftError) */
    FH_ERR_INVALID_EXCITATION = 20,/* SolveError::InvalidExcitation */
    FH_ERR_COUPLING = 21,          /* SolveError::Coupling(CouplingError), kind in detail (FH_COUPLING_*) */
    FH_ERR_UNSUPPORTED = 30        /* a path this build does not provide */
} fh_status;

/* MeshError sub-codes carried in fh_error_info.detail for FH_ERR_MESH. */
enum {
    FH_MESH_NO_PORTS = 1,
    FH_MESH_UNKNOWN_PORT_NODE = 2,
    FH_MESH_DEGENERATE_PORT = 3,
    FH_MESH_PORT_NOT_CONNECTED = 4,
    FH_MESH_SEGMENT_COUNT_MISMATCH = 5,
    FH_MESH_EMPTY_SEGMENT = 6
};

/* CouplingError kinds (coupling.rs:93-130) carried in fh_error_info.detail for
 * FH_ERR_COUPLING: a declared group no segment belongs to; more group tags than
 * segments (index_a = segments, index_b = tags); a non-transitive declaration
 * (index_a, index_b = the two groups, in order of first appearance). */
enum {
    FH_COUPLING_UNKNOWN_GROUP = 1,
    FH_COUPLING_SEGMENT_COUNT_MISMATCH = 2,
    FH_COUPLING_NON_TRANSITIVE = 3
};

/* Payload of a failure (all fields optional / -1 when not applicable). */
typedef struct fh_error_info {
    int32_t status;       /* the fh_status returned */
    int32_t detail;       /* sub-code (MeshError kind, ...) */
    int64_t index_a;      /* segment / node / first filament / frequency index / port */
    int64_t index_b;      /* second filament / node */
    double frequency;     /* Singular / NotConverged / InvalidFrequency value */
    int64_t iterations;   /* NotConverged */
    double residual;      /* NotConverged relative residual */
} fh_error_info;

/* Node, geometry.rs:20-60. */
typedef struct fh_node {
    double x, y, z;
} fh_node;

/* SegmentDef, geometry.rs:226-270: node indices, cross-section, conductivity,
 * optional width direction (has_width_dir != 0). */
typedef struct fh_segment_def {
    int64_t a, b;
    double width, height, sigma;
    int64_t has_width_dir;
    double width_dir[3];
} fh_segment_def;

/* Port, mesh.rs:67-92: current enters at `positive`, leaves at `negative`. */
typedef struct fh_port {
    int64_t positive, negative;
} fh_port;

/* Filament record, filament.rs:33-139: 19 doubles. */
typedef struct fh_filament {
    double start[3], end[3];
    double length;
    double dir_length[3], dir_width[3], dir_height[3];
    double width, height, sigma;
} fh_filament;

/* Discretization, solve.rs:409-510. */
typedef enum fh_discretization_kind {
    FH_DISC_UNIFORM = 0,
    FH_DISC_PER_SEGMENT = 1,
    FH_DISC_GRADED = 2,
    FH_DISC_SKIN_DEPTH = 3,
    FH_DISC_PER_SEGMENT_GRADED = 4
} fh_discretization_kind;

typedef struct fh_axis_grading {
    int64_t nw, nh;
    double width_ratio, height_ratio;
} fh_axis_grading;

typedef struct fh_discretization {
    int64_t kind;                  /* fh_discretization_kind */
    int64_t nw, nh;                /* UNIFORM / GRADED */
    double ratio;                  /* GRADED / SKIN_DEPTH */
    double frequency_hz;           /* SKIN_DEPTH */
    double target_skin_depths;     /* SKIN_DEPTH */
    int64_t max_per_axis;          /* SKIN_DEPTH (reference default 32) */
    const fh_axis_grading *per_segment; /* PER_SEGMENT(_GRADED): one per segment */
    int64_t per_segment_len;
} fh_discretization;

/* SolverChoice, solve.rs:169-193; DENSE_PATH_MAX_FILAMENTS = 10000 (solve.rs:133). */
typedef enum fh_solver_choice {
    FH_SOLVER_AUTO = 0,
    FH_SOLVER_DENSE = 1,
    FH_SOLVER_ITERATIVE = 2
} fh_solver_choice;
#define FH_DENSE_PATH_MAX_FILAMENTS 10000

/* How the per-frequency complex LU is computed (no reference counterpart:
 * the reference always runs the FP64 form). */
typedef enum fh_precision {
    FH_PRECISION_FP64 = 0,          /* FP64 blocked LU, partial pivoting (dense.rs) */
    FH_PRECISION_MIXED_BF16X3 = 1,  /* FP32 panels, split-BF16 x3 tensor-core trailing
                                       updates, FP64-residual iterative refinement */
    FH_PRECISION_MIXED_FP32 = 2     /* FP32 factors with FP32 SIMT trailing updates,
                                       FP64-residual iterative refinement */
} fh_precision;

/* Counts, result.rs:110-126. */
typedef struct fh_counts {
    int64_t nodes, segments, filaments, meshes, internal_meshes, ports;
} fh_counts;

/* Timing, result.rs:129-141, plus device-event phase times. */
typedef struct fh_timing {
    double inductance_s;   /* fill */
    double assembly_s;     /* discretize + mesh + fill + congruence */
    double solve_s;        /* sweep */
    double total_s;
} fh_timing;

/* Per-sweep report; arrays are optional (NULL) and have nf entries. */
typedef struct fh_sweep_report {
    int32_t *refinement_iterations;  /* mixed form: iterations per frequency */
    double *residual;                /* final relative residual ||b - Ax|| / ||b|| per frequency */
    double solve_s;                  /* device time of the sweep */
    double factor_s;                 /* device time of the factorizations */
    double refine_s;                 /* device time of the refinement */
} fh_sweep_report;

typedef struct fh_system fh_system;

/* ---- library ---------------------------------------------------------- */

/* ABI version and build string. */
int32_t fh_abi_version(void);
const char *fh_build_info(void);
/* Thread-local message for the last failing call on this thread. */
const char *fh_last_error(void);
/* Number of usable sm_100 devices (0 when none). */
int32_t fh_device_count(void);

/* Device memory of finished systems is kept in a per-device cache (a
 * stream-ordered pool) and reused by later systems; this hands the idle part
 * back to the driver (the analogue of emptying a framework's allocator
 * cache).  Waits for the devices to finish their work first. */
fh_status fh_release_cached_memory(void);

/* ---- host model (no device use) --------------------------------------- */

/* Discretize a geometry into filaments.  Replaces discretize_geometry
 * (fasterhenry/src/solve.rs:947-978) over discretize (filament.rs:320) /
 * discretize_graded_per_axis (filament.rs:478).  Call with filaments == NULL
 * to get *n_filaments; per_segment (optional, nseg entries) gets the bundle
 * sizes. */
fh_status fh_discretize(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segments,
                        size_t n_segments, const fh_discretization *disc, fh_filament *filaments,
                        size_t capacity, size_t *n_filaments, int64_t *per_segment,
                        fh_error_info *err);

/* Loop basis as CSR rows of (branch, sign).  Replaces MeshMatrix::build
 * (fasterhenry/src/mesh.rs:170-263).  Call with row_ptr == NULL to size. */
fh_status fh_mesh_build(const fh_segment_def *segments, size_t n_segments, size_t n_nodes,
                        const int64_t *per_segment, const fh_port *ports, size_t n_ports,
                        int64_t *row_ptr, int64_t *branch, double *sign, size_t cap_rows,
                        size_t cap_nnz, size_t *n_rows, size_t *nnz, size_t *n_internal,
                        fh_error_info *err);

/* SolverChoice::resolve (solve.rs:181-190): 0 dense, 1 iterative. */
int32_t fh_solver_resolve(fh_solver_choice choice, size_t filaments);

/* ---- GPU kernels exposed as library calls ----------------------------- */

/* Symmetric n x n partial-inductance matrix, column-major, on cuda:0.
 * Replaces partial_inductance_matrix (fasterhenry/src/inductance/batch.rs:246).
 * `methods` (optional, n*n int8) receives the inductance::Method per entry
 * (0 Orthogonal, 1 BarClosedForm, 2 AlignedQuadrature, 3 PointQuadrature,
 * 4 SampledFilaments). */
fh_status fh_partial_inductance_matrix(const fh_filament *filaments, size_t n, double *L,
                                       int8_t *methods, fh_error_info *err);

/* Solve a x = b for complex a (n x n, column-major) and b (n x nrhs,
 * column-major) with the device FP64 blocked LU (partial pivoting).
 * Replaces dense::lu_solve (fasterhenry/src/dense.rs:43).  x may alias b. */
fh_status fh_lu_solve_c64(const double *a, size_t n, const double *b, size_t nrhs, double *x,
                          fh_error_info *err);

/* The same FP64 LU solve for callers that cannot allocate device memory while
 * they solve (for example an application that hands all device memory to its
 * own pool, whose accounting a cudaMalloc would bypass, or a latency-critical
 * loop that must not cudaMalloc/cudaFree).  No counterpart in the reference.
 *   a: DEVICE pointer, n x n complex column-major; consumed as workspace
 *      (overwritten with the LU factors), like the reference's lu_solve.
 *   b: DEVICE pointer, n x nrhs complex column-major; overwritten with x.
 *   stream: a cudaStream_t (NULL = the legacy default stream).
 * Allocates nothing: its scratch (pivots, pivot-search partials, flags) is a
 * file-scope device array sized for n <= FH_NOALLOC_MAX_ORDER; larger n is
 * rejected with FH_ERR_INVALID_ARGUMENT.  The first call in each device
 * context looks up the array's address.  All calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller.  The
 * call blocks the host until the solve has finished on `stream` (it copies
 * the zero-pivot flag back and synchronizes the stream), so it must not be
 * made while `stream`, or the legacy stream, is being captured into a CUDA
 * graph. */
#define FH_NOALLOC_MAX_ORDER 65536
fh_status fh_lu_solve_c64_noalloc(double *a, size_t n, double *b, size_t nrhs, void *stream,
                                  fh_error_info *err);

/* ---- the dense system (MeshSystem) ------------------------------------ */

/* Assemble: discretize, loop basis, fill L on the device, congruence
 * R_m = M R M^T, L_m = M L M^T kept resident in HBM.  Replaces
 * MeshSystem::assemble (fasterhenry/src/solve.rs:680-766).  `choice` is
 * resolved with fh_solver_resolve; a choice that resolves to the iterative
 * path returns FH_ERR_UNSUPPORTED here: the matrix-free path has its own
 * handle, fh_iterative_create (the reference's IterativeSystem). */
fh_status fh_system_create(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segments,
                           size_t n_segments, const fh_port *ports, size_t n_ports,
                           const fh_discretization *disc, fh_solver_choice choice,
                           fh_system **out, fh_error_info *err);

void fh_system_destroy(fh_system *sys);

/* Coupling (coupling.rs:150-215): the group of each segment and the group
 * pairs whose mutual inductance is kept.  truncate = 0 is Coupling::all_pairs
 * (group names ignored, every pair kept); truncate = 1 keeps every group with
 * itself and the declared pairs, and stores zero for every other filament
 * pair without evaluating it.  A NULL or empty name is the default group;
 * segments past n_segment_groups are in the default group. */
typedef struct fh_coupling {
    const char *const *segment_groups;
    size_t n_segment_groups;
    int32_t truncate;
    const char *const *couples; /* 2 x n_couples group names */
    size_t n_couples;
} fh_coupling;

/* MeshSystem::assemble_with_coupling (solve.rs:703-766): the coupling is
 * checked against the geometry first (FH_ERR_COUPLING), then as
 * fh_system_create with the truncated pairs left out of the fill.  A NULL
 * coupling is Coupling::all_pairs. */
fh_status fh_system_create_coupled(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segments,
                                   size_t n_segments, const fh_port *ports, size_t n_ports,
                                   const fh_discretization *disc, const fh_coupling *coupling,
                                   fh_solver_choice choice, fh_system **out, fh_error_info *err);

/* TruncationWarning (coupling.rs:132-148): a truncated group pair whose
 * bounding boxes lie closer than the larger box diagonal.  Groups are
 * numbered in order of first appearance over the segments. */
typedef struct fh_truncation_warning {
    int64_t group_a, group_b;
    double separation, extent;
} fh_truncation_warning;

/* The assembled system's coupling: PairMask::kept_pairs / total_pairs
 * (inductance/batch.rs:88-117) and Coupling::truncation_warnings
 * (coupling.rs:285-318), `count` of them written up to `capacity`. */
fh_status fh_system_coupling(const fh_system *sys, int64_t *kept_pairs, int64_t *total_pairs,
                             fh_truncation_warning *warnings, size_t capacity, size_t *count);

fh_status fh_system_counts(const fh_system *sys, fh_counts *counts);
fh_status fh_system_timing(const fh_system *sys, fh_timing *timing);

/* Host copies of the assembled data (MeshSystem::filaments, ::filament_resistances). */
fh_status fh_system_filaments(const fh_system *sys, fh_filament *out, size_t capacity);
fh_status fh_system_resistances(const fh_system *sys, double *out, size_t capacity);
/* R_m and L_m as full (meshes x meshes) column-major host matrices. */
fh_status fh_system_mesh_matrices(const fh_system *sys, double *r_mesh, double *l_mesh);
/* Device pointer of L_m (meshes x meshes, column-major, FP64); valid until destroy. */
fh_status fh_system_device_l_mesh(const fh_system *sys, const double **l_mesh, const double **r_mesh);

/* Z(w) at every frequency: z_out is nf x p x p complex (interleaved), row-major
 * per frequency like SweepResult.impedance_ohm[k][i][j] (result.rs:47-66).
 * Replaces MeshSystem::sweep (solve.rs:881-893) / sweep_impedances
 * (solve.rs:1039-1079): frequencies are validated first (InvalidFrequency
 * names the first bad index), and the first failing frequency in list order
 * is reported.  All frequencies are factorized in batched launches. */
fh_status fh_sweep(fh_system *sys, const double *frequencies_hz, size_t nf, fh_precision precision,
                   double *z_out, fh_sweep_report *report, fh_error_info *err);

/* Batched sweep of independent systems (no reference counterpart: the
 * reference sweeps one MeshSystem at a time).  System i is swept over its own
 * frequencies freqs[i][0..nf[i]) into z_out[i] (nf[i] x p_i x p_i), as
 * fh_sweep would.  In the mixed precisions every (system, frequency) of the
 * systems with at most FH_BATCH_MAX_ORDER internal loops is solved in ONE
 * persistent launch (FP32 factors without interchanges, FP64-residual
 * refinement, work items largest first, tile shapes per order bucket from an
 * autotuner whose table is kept in a JSON file: $FH_AUTOTUNE_CACHE, else the
 * user's cache directory); an item whose refinement does not converge is
 * redone in FP64.  Larger systems, and every system in FP64, are swept as by
 * fh_sweep, up to `concurrency` (<= 0: 4) at once on their own streams.  On
 * failure the first failing system (lowest index) is reported, its index in
 * fh_error_info.detail. */
#define FH_BATCH_MAX_ORDER 1024
fh_status fh_batch_sweep(fh_system *const *systems, size_t k, const double *const *freqs, const size_t *nf,
                         fh_precision precision, double *const *z_out, int32_t concurrency, fh_error_info *err);

/* One frequency (MeshSystem::impedance, solve.rs:806-830). */
fh_status fh_impedance(fh_system *sys, double frequency_hz, fh_precision precision, double *z_out,
                       fh_error_info *err);

/* ---- filament currents and power (currents.rs) -------------------------- */

/* Layout, currents.rs:128-170: the segment of every filament (n), the
 * conductor (connected component of the segment graph, numbered by first
 * segment) of every segment (n_segments), and the conductor count. */
fh_status fh_system_layout(const fh_system *sys, int64_t *segment_of_filament, int64_t *conductor_of_segment,
                           int64_t *conductor_count);

/* PowerBalance, currents.rs:97-106 (time-average power of peak phasors). */
typedef struct fh_power_balance {
    double dissipated_w;
    double input_w;
    double relative_residual;
} fh_power_balance;

/* MeshSystem::currents (solve.rs:845-868 with currents.rs:172-274) at nf
 * frequencies for one port-current excitation (p complex phasors, peak
 * amperes): internal loop currents -Z_ee^-1 Z_ep I_p, branch currents
 * M^T [I_e; I_p], |J| = |I| / (w h) and P = |I|^2 R / 2 per filament, sums
 * per segment, the filament of largest |J| per conductor (first in filament
 * order on ties), and the power balance against 1/2 Re(I_p^H V_p).  The
 * frequencies are factorized in batches as by fh_sweep (precision as there).
 * Every output is optional (NULL):
 *   filament_current   nf x n complex (interleaved)
 *   current_density    nf x n (A/m^2)
 *   power_w            nf x n
 *   segment_current    nf x n_segments complex
 *   segment_power_w    nf x n_segments
 *   conductor_peak_filament, conductor_peak_density   nf x conductors
 *   balance            nf
 * Errors: FH_ERR_INVALID_FREQUENCY (first bad index), FH_ERR_INVALID_EXCITATION
 * (a non-finite entry; index_a = the port count, index_b = the entries
 * given), FH_ERR_SINGULAR. */
fh_status fh_currents(fh_system *sys, const double *frequencies_hz, size_t nf, const double *excitation,
                      size_t n_excitation, fh_precision precision, double *filament_current, double *current_density,
                      double *power_w, double *segment_current, double *segment_power_w,
                      int64_t *conductor_peak_filament, double *conductor_peak_density, fh_power_balance *balance,
                      fh_error_info *err);

/* ---- impedance gradient (no reference counterpart) --------------------- */

/* A geometric parameter: the width or the thickness of segment `index`, or a
 * coordinate of node `index` (node coordinates are not provided: moving a
 * node rotates the segments that meet there, and the derivative of the
 * integrals under a rotation is not built; FH_ERR_UNSUPPORTED). */
typedef enum fh_param_kind {
    FH_PARAM_WIDTH = 0,
    FH_PARAM_THICKNESS = 1,
    FH_PARAM_NODE_X = 2,
    FH_PARAM_NODE_Y = 3,
    FH_PARAM_NODE_Z = 4
} fh_param_kind;

typedef struct fh_param_spec {
    int32_t kind; /* fh_param_kind */
    int32_t reserved;
    int64_t index;
} fh_param_spec;

typedef struct fh_gradient_report {
    double solve_s;           /* FP64 factorization and solve for the loop currents */
    double derivative_fill_s; /* device time of the derivative fill */
    double contract_s;        /* device time of the products with the branch currents */
    double total_s;           /* wall time of the call */
    int64_t pairs;            /* filament pairs differentiated (upper triangle) */
} fh_gradient_report;

/* dZ/dp at one frequency for np parameters, by the stationary (adjoint) form
 * dZ_ab/dp = I_a^T (dR/dp + j w dL/dp) I_b with the branch currents I of unit
 * port currents: one FP64 solve, one derivative fill of all filament pairs,
 * one product per derivative matrix.  Derivatives are those of the
 * evaluation as dispatched at the nominal geometry (method, Gauss orders,
 * closed-form acceptance, quadrature panels, and the discretization's
 * filament counts and grading held fixed).  Parameters: a segment's width
 * or thickness, or a node's x or y.  A node moving in the xy plane turns the
 * segments that meet there about z and changes their length; those segments
 * must lie in a plane z = const with z along their width or height, else
 * FH_ERR_UNSUPPORTED (so is FH_PARAM_NODE_Z, and a coordinate parameter
 * whose moving filaments have a parallel partner of another segment with
 * cross-sections meeting along the length, such as collinear segments end
 * to end).  z_out (optional): p x p Z; dz_out: np x p x p complex
 * (interleaved), row-major per parameter, in ohm per metre.  report
 * optional. */
fh_status fh_gradient(fh_system *sys, double frequency_hz, const fh_param_spec *params, size_t np, double *z_out,
                      double *dz_out, fh_gradient_report *report, fh_error_info *err);

/* Test hook: the derivative fill of a filament set.  tangents: n x 4 (sw, sh,
 * gw, gh per filament: d centre / d w = sw * width axis, d width / d w = gw,
 * and the same for the thickness); Dw, Dh: n x n column-major with
 * D[a + b n] = dL_ab / d(side a). */
fh_status fh_test_inductance_gradient(const fh_filament *filaments, const double *tangents, size_t n, double *Dw,
                                      double *Dh, fh_error_info *err);

/* Test hook: the coordinate derivative fill of a filament set (every filament
 * moving; segment[i] numbers the segment of filament i).  Dl, Dp, Ds, Dr:
 * n x n column-major, D[a + b n] = dL_ab / d(coordinate of a): translation
 * of its centre along its length axis (Dl) and along z x l normalized (Dp),
 * stretch of its length about its centre (Ds), rotation about the z axis
 * through its centre (Dr).  Pairs of one segment carry Ds only; the diagonal
 * of Ds is half of dL_aa / d length. */
fh_status fh_test_coordinate_gradient(const fh_filament *filaments, const int32_t *segment, size_t n, double *Dl,
                                      double *Dp, double *Ds, double *Dr, fh_error_info *err);

/* Test hook: the device near-pair search of the precorrected-FFT set-up
 * (pfft/near.rs:41-106) for a filament set and a radius in metres: for each
 * filament i the filaments j >= i (i included) with a separating-axis gap
 * below the radius and non-orthogonal directions, ascending.  off: n + 1
 * row offsets; cols: capacity `cap` column indices; *total: the pair count
 * (may exceed cap, then only off is complete). */
fh_status fh_test_near_pairs(const fh_filament *filaments, size_t n, double radius, int64_t *off, int64_t *cols,
                             size_t cap, size_t *total, fh_error_info *err);

/* Test hook: the pFFT grid convolution on its own.  `fields` real source
 * grids n[0] x n[1] x n[2] (axis 2 fastest, field f at sources + f G) are
 * convolved with the kernel 1 / (spacing |d|) (zero at d = 0) on the padded
 * torus m[0] x m[1] x m[2] (m_a >= 2 n_a - 1, 2^a 3^b 5^c) by the library's
 * own transforms, fp32 != 0 in FP32; potentials like sources. */
fh_status fh_test_grid_convolution(const int64_t *n, const int64_t *m, double spacing, int32_t fp32,
                                   const double *sources, int32_t fields, double *potentials, fh_error_info *err);

/* Fill statistics of an assembled system: pairs per method and device time
 * per fill kernel (no reference counterpart; diagnostics). */
typedef struct fh_fill_stats {
    int64_t pairs, orthogonal, point_quadrature, closed_form, aligned_quadrature, sampled;
    int64_t distinct_aligned_keys;
    double point_evaluations;
    double ms_classify, ms_point, ms_closed_form, ms_aligned_quadrature, ms_sampled, ms_congruence;
    int64_t truncated;  /* pairs dropped by the coupling (never evaluated, zero in L) */
    int64_t distinct_point_keys;  /* point-quadrature pairs evaluated (one per geometry up to translation) */
} fh_fill_stats;
fh_status fh_system_fill_stats(const fh_system *sys, fh_fill_stats *stats);

/* ---- test hooks (no reference counterpart) ----------------------------- */

/* One trailing update A22 -= L21 U12 of an LU panel [k0, k0+nb) applied to
 * `count` complex FP32 matrices of order m (interleaved, column-major, back
 * to back), in place on a host copy.  mode 0: FP32 SIMT; mode 1: split-BF16
 * x3 on the tensor cores (nb a multiple of 16); mode 2: split-BF16 x3 from
 * packed operands on the persistent tensor-core kernel (nb a multiple of 16). */
fh_status fh_test_trailing_update(float *a, int64_t m, int32_t count, int64_t k0, int32_t nb, int32_t mode,
                                  fh_error_info *err);

/* ---- device-event profiler (no reference counterpart) ------------------ */

/* Kernel classes timed when profiling is on. */
typedef enum fh_profile_class {
    FH_PROF_GEMM_FP64 = 0,      /* trailing update A22 -= L21 U12, FP64 SIMT */
    FH_PROF_GEMM_FP32 = 1,      /* trailing update, FP32 SIMT */
    FH_PROF_GEMM_TC = 2,        /* trailing update, split-BF16 x3 tcgen05 (deep update of a super-panel) */
    FH_PROF_PANEL = 3,          /* panel factorization (pivot search + rank-1 updates) */
    FH_PROF_TRSM = 4,           /* row interchanges + U12 triangular solve */
    FH_PROF_SOLVE = 5,          /* forward/backward substitution */
    FH_PROF_RESIDUAL = 6,       /* FP64 residual of R + jwL */
    FH_PROF_PACK = 7,           /* BF16 split + packing of the deep update's operands */
    FH_PROF_GEMM_TC_INNER = 8,  /* tensor-core updates inside a super-panel and of its U12 rows */
    FH_PROF_PFFT_APPLY = 9,     /* one precorrected-FFT product (near field, spread, FFTs, interpolation) */
    FH_PROF_PANEL_SOLVE = 10,   /* rows below a super-panel: L21 = A21 U^-1, U12 and the packed operands */
    FH_PROF_FORM = 11,          /* the sweep's systems R + jwL (and right-hand sides) formed from R_m, L_m */
    FH_PROF_SOLVE_FLOW = 12,    /* dataflow forward/backward solve of the two-level factors (flags per block) */
    FH_PROF_SOLVE_BARRIER = 13, /* barrier-based forward/backward solve of the two-level factors */
    FH_PROF_BATCH = 14,         /* the persistent batched solve of many small systems (fh_batch_sweep, mixed) */
    FH_PROF_GEMM_TC_SHARED = 15, /* the second part of a split deep update, on the SMs the look-ahead leaves it */
    FH_PROF_CLASSES = 16
} fh_profile_class;

void fh_profile_enable(int32_t on);
void fh_profile_reset(void);
/* Totals since the last reset: launches, device milliseconds (sum of
 * per-launch event durations) and algorithmic work (flops). */
fh_status fh_profile_read(int32_t cls, int64_t *launches, double *ms, double *work);
/* Time (ms, from the launches recorded since fh_profile_enable) during which
 * a launch of a class in mask_a (bit 1 << class) ran, a launch of a class in
 * mask_b ran, and both ran at once (launches on different streams: the
 * factorization's look-ahead).  Each launch counts from the event before it
 * to the event after it on its stream. */
fh_status fh_profile_overlap(uint32_t mask_a, uint32_t mask_b, double *ms_a, double *ms_b, double *ms_both);

/* ---- outputs (host) ---------------------------------------------------- */

/* SweepResult JSON (result.rs:1-40, schema_version 1).  port_names may be NULL.
 * Writes at most `capacity` bytes (NUL-terminated) and sets *length to the
 * full length; call with buf == NULL to size. */
fh_status fh_sweep_json(const fh_port *ports, const char *const *port_names, size_t n_ports,
                        const double *frequencies_hz, size_t nf, const double *z,
                        const fh_counts *counts, const fh_timing *timing, char *buf,
                        size_t capacity, size_t *length);

/* MAT v4 Zc.mat (fasterhenry-cli/src/mat.rs:31-100) written to `path`. */
fh_status fh_write_zc_mat(const char *path, size_t n_ports, const double *frequencies_hz, size_t nf,
                          const double *z);

/* SPICE subcircuit at frequency index k (fasterhenry-cli/src/spice.rs:64-135). */
fh_status fh_spice_subckt(size_t n_ports, const double *frequencies_hz, size_t nf, const double *z,
                          size_t k, const char *name, char *buf, size_t capacity, size_t *length);

/* ---- matrix-free path: precorrected FFT operator and GMRES ------------- */

/* PfftParams (pfft/mod.rs:183-232).  spacing_kind 0 = GridSpacing::Auto with
 * cells_per_filament, 1 = GridSpacing::Fixed(spacing, metres);
 * near_field_radius in grid spacings (>= interpolation_order + 1). */
typedef struct fh_pfft_params {
    int32_t spacing_kind;
    int32_t interpolation_order;
    double cells_per_filament;
    double spacing;
    double near_field_radius;
    /* Precision of the grid convolution (no reference counterpart; the
     * reference convolves in FP64): 0 = FP64, 1 = FP32.  Projection,
     * interpolation and the near-field precorrection stay FP64. */
    int32_t fft_precision;
    int32_t reserved;
} fh_pfft_params;

/* PfftParams::default(): Auto 8 cells per filament, radius 8, order 5; FP64
 * convolution. */
void fh_pfft_default_params(fh_pfft_params *params);

/* PfftStats (pfft/mod.rs:255-272) plus the set-up time split. */
typedef struct fh_pfft_stats {
    int64_t filaments;
    double grid_spacing;
    int64_t grid_dims[3];
    int64_t fft_dims[3];
    int64_t projection_entries;
    int64_t near_entries;
    int64_t memory_bytes;
    double setup_host_s;   /* parameters and the grid (host) */
    double setup_device_s; /* near-pair search, projections, precorrection, exact near pairs, kernel spectrum */
    double setup_near_s;   /* the near-pair search alone (part of setup_device_s) */
} fh_pfft_stats;

typedef struct fh_pfft fh_pfft;

/* PfftOperator::new (pfft/mod.rs:332-478).  Errors: FH_ERR_PFFT
 * (PfftError::InvalidParameter / GridTooLarge), FH_ERR_KERNEL_* for a near
 * pair (PfftError::Kernel). */
fh_status fh_pfft_create(const fh_filament *filaments, size_t n, const fh_pfft_params *params, fh_pfft **out,
                         fh_error_info *err);
/* PfftOperator::apply (pfft/mod.rs:482-529): y = L x for `count` vectors of
 * length n (host arrays, vector v at x + v n). */
fh_status fh_pfft_apply(fh_pfft *op, const double *x, double *y, size_t count, fh_error_info *err);
/* PfftOperator::stats (pfft/mod.rs:563-597). */
fh_status fh_pfft_get_stats(const fh_pfft *op, fh_pfft_stats *stats);
void fh_pfft_destroy(fh_pfft *op);

/* GmresParams (gmres.rs:32-58). */
typedef struct fh_gmres_params {
    double tolerance;       /* ||b - A x|| <= tolerance ||b||; default 1e-10 */
    int32_t restart;        /* Krylov dimension between restarts; default 100 */
    int32_t max_iterations; /* cap on products with A over all restarts; default 5000 */
} fh_gmres_params;
void fh_gmres_default_params(fh_gmres_params *params);

/* GmresOutcome (gmres.rs:61-73). */
typedef struct fh_gmres_outcome {
    int64_t iterations;
    double relative_residual;
    int32_t converged;
} fh_gmres_outcome;

typedef struct fh_iterative fh_iterative;

/* IterativeSystem::assemble (iterative.rs:155-239): discretization, loop
 * basis, pFFT operator, port columns and the Jacobi diagonal.  Null params
 * mean the defaults.  Errors as fh_system_create plus FH_ERR_PFFT. */
fh_status fh_iterative_create(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segments,
                              size_t n_segments, const fh_port *ports, size_t n_ports,
                              const fh_discretization *disc, const fh_pfft_params *pfft,
                              const fh_gmres_params *gmres, fh_iterative **out, fh_error_info *err);
fh_status fh_iterative_counts(const fh_iterative *sys, fh_counts *out);
/* inductance_s = operator set-up, assembly_s, solve_s of the last sweep. */
fh_status fh_iterative_timing(const fh_iterative *sys, fh_timing *out);
/* IterativeSystem::operator_stats (iterative.rs:259). */
fh_status fh_iterative_pfft_stats(const fh_iterative *sys, fh_pfft_stats *out);
/* IterativeSystem::sweep / solve (iterative.rs:269-302, 379-398): z_out is
 * nf x p x p interleaved complex, row-major per frequency; `outcomes`
 * (optional) nf x p GMRES outcomes.  FH_ERR_NOT_CONVERGED carries the
 * frequency, port (index_a), iterations and relative residual of the first
 * failing solve; FH_ERR_SINGULAR a non-finite Z. */
fh_status fh_iterative_sweep(fh_iterative *sys, const double *frequencies_hz, size_t nf, double *z_out,
                             fh_gmres_outcome *outcomes, fh_error_info *err);
/* The discretized filaments (n, as fh_system_filaments) and the segment /
 * conductor layout (as fh_system_layout) of an iterative system. */
fh_status fh_iterative_filaments(const fh_iterative *sys, fh_filament *out, size_t capacity);
fh_status fh_iterative_layout(const fh_iterative *sys, int64_t *segment_of_filament, int64_t *conductor_of_segment,
                              int64_t *conductor_count);
/* IterativeSystem::currents (iterative.rs:316-377 with solve.rs:1110-1149):
 * per frequency one Jacobi-preconditioned GMRES solve Z_ee x = Z_ep I_p on
 * the pFFT operator, internal loop currents -x, port voltages
 * V_p = Z_pp I_p + Z_ep^T I_e; outputs and errors as fh_currents, plus the
 * GMRES outcome of every frequency (`outcomes`, optional, nf) and
 * FH_ERR_NOT_CONVERGED (port index 0) as fh_iterative_sweep. */
fh_status fh_iterative_currents(fh_iterative *sys, const double *frequencies_hz, size_t nf, const double *excitation,
                                size_t n_excitation, double *filament_current, double *current_density,
                                double *power_w, double *segment_current, double *segment_power_w,
                                int64_t *conductor_peak_filament, double *conductor_peak_density,
                                fh_power_balance *balance, fh_gmres_outcome *outcomes, fh_error_info *err);
void fh_iterative_destroy(fh_iterative *sys);

/* Test hook (no reference counterpart): the device GMRES on a dense complex
 * system a (n x n column-major, interleaved), right preconditioner `precond`
 * (n x n, or NULL for none); x holds the initial guess and receives the
 * solution. */
fh_status fh_test_gmres_dense(const double *a, size_t n, const double *b, double *x, const double *precond,
                              const fh_gmres_params *params, fh_gmres_outcome *outcome, fh_error_info *err);

#ifdef __cplusplus
}
#endif
#endif /* FASTERHENRY_B200_H */
