// Restarted, right-preconditioned GMRES on device vectors (gmres.rs:91-215
// of the reference): Gram-Schmidt applied twice (classical, each pass one
// multi-vector product and one update; the reference applies modified
// Gram-Schmidt twice), complex Givens
// rotations, the true residual recomputed at every restart.  Vectors are
// complex doubles on the device; the small Hessenberg problem lives on the
// host.  Reductions (inner products, norms) use a fixed grid and a fixed
// combination order, so a solve is a deterministic function of its inputs.
#pragma once

#include <cuda_runtime.h>

#include <functional>

#include "fh_device.cuh"

namespace fhb {

struct GmresParams {
    double tolerance = 1e-10;  // gmres.rs:45
    int restart = 100;         // gmres.rs:47
    int max_iterations = 5000; // gmres.rs:49
};

struct GmresOutcome {
    int64_t iterations = 0;
    double relative_residual = 0.0;
    bool converged = false;
};

// out = op(in) for device vectors of length n, enqueued on the solver's stream.
using DeviceOp = std::function<fh_status(const double2 *in, double2 *out, fh_error_info *err)>;

// Device workspace of a solve of order n with a given restart length.
struct GmresWork {
    int64_t n = 0;
    int restart = 0;
    double2 *V = nullptr;    // (restart + 1) x n basis
    double2 *w = nullptr, *r = nullptr, *t = nullptr, *u = nullptr;
    double2 *h = nullptr;    // 2 x (restart + 1) projections of one Arnoldi step
    double *red = nullptr;   // reduction partials and results
    double *part = nullptr;  // per-block partial projections, 2 x kRB x (restart + 1)
    ~GmresWork();
    fh_status ensure(int64_t n_, int restart_, fh_error_info *err);
};

// Solves A x = b; x holds the initial guess on entry.  b, x: device.
fh_status gmres_solve(int64_t n, const DeviceOp &apply, const DeviceOp &precondition, const double2 *d_b, double2 *d_x,
                      const GmresParams &params, cudaStream_t s, GmresWork &work, GmresOutcome *out,
                      fh_error_info *err);

}  // namespace fhb
