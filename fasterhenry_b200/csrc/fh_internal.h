// Internal declarations shared by the host model (fh_host.cpp) and the
// device side (fh_*.cu).  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fasterhenry_b200.h"

namespace fhb {

// Records `msg` as this thread's fh_last_error() and fills `err`.
fh_status fail(fh_error_info *err, fh_status status, const std::string &msg, int64_t a = -1,
               int64_t b = -1, double frequency = 0.0, int32_t detail = 0);
void clear_error(fh_error_info *err);

struct Vec3 {
    double x, y, z;
};

// Filament bundles of every segment, in segment order.
struct Discretized {
    std::vector<fh_filament> filaments;
    std::vector<int64_t> per_segment;
};

fh_status validate_geometry(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segs,
                            size_t n_segs, fh_error_info *err);
fh_status discretize_geometry(const fh_node *nodes, size_t n_nodes, const fh_segment_def *segs,
                              size_t n_segs, const fh_discretization *disc, Discretized &out,
                              fh_error_info *err);

// n-point Gauss-Legendre rule on [-1, 1] (gauss.rs:25-75), nodes ascending.
void gauss_rule(int n, double *nodes, double *weights);

// Loop basis, CSR.
struct LoopBasis {
    std::vector<int64_t> row_ptr;
    std::vector<int32_t> branch;
    std::vector<double> sign;
    int64_t internal = 0;
    int64_t rows() const { return (int64_t)row_ptr.size() - 1; }
};
fh_status build_loops(const fh_segment_def *segs, size_t n_segs, size_t n_nodes,
                      const int64_t *per_segment, const fh_port *ports, size_t n_ports,
                      LoopBasis &out, fh_error_info *err);

// Conductor layout (currents.rs:128-170): the segment of every filament, the
// first filament of every segment (n_segs + 1 entries), and the conductor of
// every segment, conductors being the connected components of the segment
// graph numbered in order of their first segment.
struct ConductorLayout {
    std::vector<int64_t> segment_of_filament, segment_first, conductor_of_segment;
    int64_t conductors = 0;
};
void conductor_layout(const fh_segment_def *segs, size_t n_segs, size_t n_nodes, const int64_t *per_segment,
                      ConductorLayout &out);

// The loop basis transposed over its first `rows` loops: per branch (n + 1
// offsets) the (loop, sign) entries in increasing loop order, which is the
// order in which a row-by-row scatter of the basis adds them.
struct TransposedLoops {
    std::vector<int64_t> offset;
    std::vector<int32_t> loop;
    std::vector<double> sign;
};
void transpose_loops(const LoopBasis &basis, int64_t n, int64_t rows, TransposedLoops &out);

// Coupling resolved against a segment count (coupling.rs:323-380): group of
// each segment (numbered by first appearance), names, and the symmetric
// groups x groups table of kept pairs.
struct CouplingResolved {
    bool all_pairs = true;
    std::vector<int32_t> of_segment;
    std::vector<std::string> names;
    std::vector<uint8_t> couples;
    int64_t groups() const { return (int64_t)names.size(); }
};
fh_status resolve_coupling(const fh_coupling *c, size_t n_segs, CouplingResolved &out, fh_error_info *err);
// Truncated group pairs closer than their extent (coupling.rs:285-318).
std::vector<fh_truncation_warning> coupling_warnings(const CouplingResolved &r, const fh_node *nodes,
                                                     const fh_segment_def *segs, size_t n_segs);
// PairMask::kept_pairs (inductance/batch.rs:88-112) for per-segment filament counts.
int64_t coupling_kept_pairs(const CouplingResolved &r, const int64_t *per_segment, size_t n_segs);

}  // namespace fhb
