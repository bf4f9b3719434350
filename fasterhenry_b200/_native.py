"""ctypes binding of ``libfhb200.so`` (the C ABI in include/fasterhenry_b200.h).

The library is loaded from this package directory only (built in-tree by
``fasterhenry_b200/build.py``).  There is no CPU fallback: if the library is
missing or no B200 is present, the compute entry points raise.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfhb200.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int64_p = ctypes.POINTER(ctypes.c_int64)


class Node(ctypes.Structure):
    _fields_ = [("x", ctypes.c_double), ("y", ctypes.c_double), ("z", ctypes.c_double)]


class SegmentDef(ctypes.Structure):
    _fields_ = [("a", ctypes.c_int64), ("b", ctypes.c_int64), ("width", ctypes.c_double),
                ("height", ctypes.c_double), ("sigma", ctypes.c_double), ("has_width_dir", ctypes.c_int64),
                ("width_dir", ctypes.c_double * 3)]


class Port(ctypes.Structure):
    _fields_ = [("positive", ctypes.c_int64), ("negative", ctypes.c_int64)]


class Filament(ctypes.Structure):
    _fields_ = [("start", ctypes.c_double * 3), ("end", ctypes.c_double * 3), ("length", ctypes.c_double),
                ("dir_length", ctypes.c_double * 3), ("dir_width", ctypes.c_double * 3),
                ("dir_height", ctypes.c_double * 3), ("width", ctypes.c_double), ("height", ctypes.c_double),
                ("sigma", ctypes.c_double)]


class AxisGrading(ctypes.Structure):
    _fields_ = [("nw", ctypes.c_int64), ("nh", ctypes.c_int64), ("width_ratio", ctypes.c_double),
                ("height_ratio", ctypes.c_double)]


class Discretization(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int64), ("nw", ctypes.c_int64), ("nh", ctypes.c_int64), ("ratio", ctypes.c_double),
                ("frequency_hz", ctypes.c_double), ("target_skin_depths", ctypes.c_double),
                ("max_per_axis", ctypes.c_int64), ("per_segment", ctypes.POINTER(AxisGrading)),
                ("per_segment_len", ctypes.c_int64)]


class ErrorInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("detail", ctypes.c_int32), ("index_a", ctypes.c_int64),
                ("index_b", ctypes.c_int64), ("frequency", ctypes.c_double), ("iterations", ctypes.c_int64),
                ("residual", ctypes.c_double)]


class Counts(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("nodes", "segments", "filaments", "meshes", "internal_meshes", "ports")]


class Timing(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("inductance_s", "assembly_s", "solve_s", "total_s")]


class SweepReport(ctypes.Structure):
    _fields_ = [("refinement_iterations", ctypes.POINTER(ctypes.c_int32)), ("residual", c_double_p),
                ("solve_s", ctypes.c_double), ("factor_s", ctypes.c_double), ("refine_s", ctypes.c_double)]


class PfftParams(ctypes.Structure):
    _fields_ = [("spacing_kind", ctypes.c_int32), ("interpolation_order", ctypes.c_int32),
                ("cells_per_filament", ctypes.c_double), ("spacing", ctypes.c_double),
                ("near_field_radius", ctypes.c_double), ("fft_precision", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class PfftStats(ctypes.Structure):
    _fields_ = [("filaments", ctypes.c_int64), ("grid_spacing", ctypes.c_double), ("grid_dims", ctypes.c_int64 * 3),
                ("fft_dims", ctypes.c_int64 * 3), ("projection_entries", ctypes.c_int64),
                ("near_entries", ctypes.c_int64), ("memory_bytes", ctypes.c_int64), ("setup_host_s", ctypes.c_double),
                ("setup_device_s", ctypes.c_double), ("setup_near_s", ctypes.c_double)]


class GmresParams(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("restart", ctypes.c_int32), ("max_iterations", ctypes.c_int32)]


class ParamSpec(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("reserved", ctypes.c_int32), ("index", ctypes.c_int64)]


class PowerBalance(ctypes.Structure):
    _fields_ = [("dissipated_w", ctypes.c_double), ("input_w", ctypes.c_double),
                ("relative_residual", ctypes.c_double)]


class GradientReport(ctypes.Structure):
    _fields_ = [("solve_s", ctypes.c_double), ("derivative_fill_s", ctypes.c_double), ("contract_s", ctypes.c_double),
                ("total_s", ctypes.c_double), ("pairs", ctypes.c_int64)]


class GmresOutcome(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("relative_residual", ctypes.c_double), ("converged", ctypes.c_int32)]


# Status codes (fh_status)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_NO_DEVICE = 2
ERR_CUDA = 3
ERR_OUT_OF_MEMORY = 4
ERR_DEVICE_TIMEOUT = 5
ERR_GEOMETRY = 10
ERR_DISCRETIZE = 11
ERR_KERNEL_COINCIDENT = 12
ERR_KERNEL_NOT_FINITE = 13
ERR_MESH = 14
ERR_INVALID_GRADING = 15
ERR_INVALID_FREQUENCY = 16
ERR_SINGULAR = 17
ERR_NOT_CONVERGED = 18
ERR_PFFT = 19
ERR_INVALID_EXCITATION = 20
ERR_COUPLING = 21
ERR_UNSUPPORTED = 30

EXPORTS = [
    "fh_abi_version", "fh_build_info", "fh_last_error", "fh_device_count", "fh_discretize", "fh_mesh_build",
    "fh_solver_resolve", "fh_partial_inductance_matrix", "fh_lu_solve_c64", "fh_system_create", "fh_system_destroy",
    "fh_system_counts", "fh_system_timing", "fh_system_filaments", "fh_system_resistances",
    "fh_system_mesh_matrices", "fh_system_device_l_mesh", "fh_sweep", "fh_impedance", "fh_sweep_json",
    "fh_write_zc_mat", "fh_spice_subckt", "fh_system_fill_stats", "fh_profile_enable", "fh_profile_reset",
    "fh_profile_read", "fh_profile_overlap", "fh_pfft_default_params", "fh_pfft_create", "fh_pfft_apply", "fh_pfft_get_stats",
    "fh_pfft_destroy", "fh_gmres_default_params", "fh_iterative_create", "fh_iterative_counts", "fh_iterative_timing",
    "fh_iterative_pfft_stats", "fh_iterative_sweep", "fh_iterative_destroy", "fh_test_gmres_dense",
    "fh_batch_sweep", "fh_gradient", "fh_test_inductance_gradient", "fh_release_cached_memory", "fh_test_near_pairs",
    "fh_test_grid_convolution",
    "fh_system_layout", "fh_currents", "fh_system_create_coupled", "fh_system_coupling", "fh_iterative_filaments",
    "fh_iterative_layout", "fh_iterative_currents", "fh_test_coordinate_gradient",
]

PROFILE_CLASSES = ["gemm_fp64", "gemm_fp32", "gemm_tc", "panel", "trsm", "solve", "residual", "pack", "gemm_tc_inner",
                   "pfft_apply", "panel_solve", "form", "solve_flow", "solve_barrier", "batch", "gemm_tc_shared"]


class FillStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("pairs", "orthogonal", "point_quadrature", "closed_form",
                                              "aligned_quadrature", "sampled", "distinct_aligned_keys")] + \
               [(k, ctypes.c_double) for k in ("point_evaluations", "ms_classify", "ms_point", "ms_closed_form",
                                               "ms_aligned_quadrature", "ms_sampled", "ms_congruence")] + \
               [("truncated", ctypes.c_int64), ("distinct_point_keys", ctypes.c_int64)]


class CouplingSpec(ctypes.Structure):
    _fields_ = [("segment_groups", ctypes.POINTER(ctypes.c_char_p)), ("n_segment_groups", ctypes.c_size_t),
                ("truncate", ctypes.c_int32), ("couples", ctypes.POINTER(ctypes.c_char_p)),
                ("n_couples", ctypes.c_size_t)]


class TruncationWarning(ctypes.Structure):
    _fields_ = [("group_a", ctypes.c_int64), ("group_b", ctypes.c_int64), ("separation", ctypes.c_double),
                ("extent", ctypes.c_double)]

_lib = None


def load():
    """Loads the in-tree library (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("fasterhenry_b200 native library not built: %s (run python -m fasterhenry_b200.build)"
                      % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    ei = P(ErrorInfo)
    sz = ctypes.c_size_t
    L.fh_abi_version.restype = ctypes.c_int32
    L.fh_build_info.restype = ctypes.c_char_p
    L.fh_last_error.restype = ctypes.c_char_p
    L.fh_device_count.restype = ctypes.c_int32
    L.fh_discretize.argtypes = [P(Node), sz, P(SegmentDef), sz, P(Discretization), P(Filament), sz, P(sz), c_int64_p, ei]
    L.fh_mesh_build.argtypes = [P(SegmentDef), sz, sz, c_int64_p, P(Port), sz, c_int64_p, c_int64_p, c_double_p, sz, sz,
                                P(sz), P(sz), P(sz), ei]
    L.fh_solver_resolve.argtypes = [ctypes.c_int, sz]
    L.fh_solver_resolve.restype = ctypes.c_int32
    L.fh_partial_inductance_matrix.argtypes = [P(Filament), sz, c_double_p, P(ctypes.c_int8), ei]
    L.fh_lu_solve_c64.argtypes = [c_double_p, sz, c_double_p, sz, c_double_p, ei]
    L.fh_system_create.argtypes = [P(Node), sz, P(SegmentDef), sz, P(Port), sz, P(Discretization), ctypes.c_int,
                                   P(ctypes.c_void_p), ei]
    L.fh_pfft_default_params.argtypes = [P(PfftParams)]
    L.fh_pfft_default_params.restype = None
    L.fh_pfft_create.argtypes = [P(Filament), sz, P(PfftParams), P(ctypes.c_void_p), ei]
    L.fh_pfft_apply.argtypes = [ctypes.c_void_p, c_double_p, c_double_p, sz, ei]
    L.fh_pfft_get_stats.argtypes = [ctypes.c_void_p, P(PfftStats)]
    L.fh_pfft_destroy.argtypes = [ctypes.c_void_p]
    L.fh_pfft_destroy.restype = None
    L.fh_gmres_default_params.argtypes = [P(GmresParams)]
    L.fh_gmres_default_params.restype = None
    L.fh_iterative_create.argtypes = [P(Node), sz, P(SegmentDef), sz, P(Port), sz, P(Discretization), P(PfftParams),
                                      P(GmresParams), P(ctypes.c_void_p), ei]
    L.fh_iterative_counts.argtypes = [ctypes.c_void_p, P(Counts)]
    L.fh_iterative_timing.argtypes = [ctypes.c_void_p, P(Timing)]
    L.fh_iterative_pfft_stats.argtypes = [ctypes.c_void_p, P(PfftStats)]
    L.fh_iterative_sweep.argtypes = [ctypes.c_void_p, c_double_p, sz, c_double_p, P(GmresOutcome), ei]
    L.fh_iterative_destroy.argtypes = [ctypes.c_void_p]
    L.fh_iterative_destroy.restype = None
    L.fh_test_gmres_dense.argtypes = [c_double_p, sz, c_double_p, c_double_p, c_double_p, P(GmresParams),
                                      P(GmresOutcome), ei]
    L.fh_batch_sweep.argtypes = [P(ctypes.c_void_p), sz, P(c_double_p), P(sz), ctypes.c_int, P(c_double_p),
                                 ctypes.c_int32, ei]
    L.fh_gradient.argtypes = [ctypes.c_void_p, ctypes.c_double, P(ParamSpec), sz, c_double_p, c_double_p,
                              P(GradientReport), ei]
    L.fh_test_inductance_gradient.argtypes = [P(Filament), c_double_p, sz, c_double_p, c_double_p, ei]
    L.fh_test_near_pairs.argtypes = [P(Filament), sz, ctypes.c_double, c_int64_p, c_int64_p, sz, P(sz), ei]
    L.fh_test_grid_convolution.argtypes = [c_int64_p, c_int64_p, ctypes.c_double, ctypes.c_int32, c_double_p,
                                           ctypes.c_int32, c_double_p, ei]
    L.fh_system_layout.argtypes = [ctypes.c_void_p, c_int64_p, c_int64_p, c_int64_p]
    L.fh_system_create_coupled.argtypes = [P(Node), sz, P(SegmentDef), sz, P(Port), sz, P(Discretization),
                                           P(CouplingSpec), ctypes.c_int, P(ctypes.c_void_p), ei]
    L.fh_system_coupling.argtypes = [ctypes.c_void_p, c_int64_p, c_int64_p, P(TruncationWarning), sz, P(sz)]
    L.fh_currents.argtypes = [ctypes.c_void_p, c_double_p, sz, c_double_p, sz, ctypes.c_int, c_double_p, c_double_p,
                              c_double_p, c_double_p, c_double_p, c_int64_p, c_double_p, P(PowerBalance), ei]
    L.fh_test_coordinate_gradient.argtypes = [P(Filament), ctypes.POINTER(ctypes.c_int32), sz, c_double_p, c_double_p,
                                              c_double_p, c_double_p, ei]
    L.fh_iterative_filaments.argtypes = [ctypes.c_void_p, P(Filament), sz]
    L.fh_iterative_layout.argtypes = [ctypes.c_void_p, c_int64_p, c_int64_p, c_int64_p]
    L.fh_iterative_currents.argtypes = [ctypes.c_void_p, c_double_p, sz, c_double_p, sz, c_double_p, c_double_p,
                                        c_double_p, c_double_p, c_double_p, c_int64_p, c_double_p, P(PowerBalance),
                                        P(GmresOutcome), ei]
    L.fh_system_destroy.argtypes = [ctypes.c_void_p]
    L.fh_system_destroy.restype = None
    L.fh_system_counts.argtypes = [ctypes.c_void_p, P(Counts)]
    L.fh_system_timing.argtypes = [ctypes.c_void_p, P(Timing)]
    L.fh_system_filaments.argtypes = [ctypes.c_void_p, P(Filament), sz]
    L.fh_system_resistances.argtypes = [ctypes.c_void_p, c_double_p, sz]
    L.fh_system_mesh_matrices.argtypes = [ctypes.c_void_p, c_double_p, c_double_p]
    L.fh_system_device_l_mesh.argtypes = [ctypes.c_void_p, P(c_double_p), P(c_double_p)]
    L.fh_sweep.argtypes = [ctypes.c_void_p, c_double_p, sz, ctypes.c_int, c_double_p, P(SweepReport), ei]
    L.fh_impedance.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, c_double_p, ei]
    L.fh_sweep_json.argtypes = [P(Port), P(ctypes.c_char_p), sz, c_double_p, sz, c_double_p, P(Counts), P(Timing),
                                ctypes.c_char_p, sz, P(sz)]
    L.fh_write_zc_mat.argtypes = [ctypes.c_char_p, sz, c_double_p, sz, c_double_p]
    L.fh_spice_subckt.argtypes = [sz, c_double_p, sz, c_double_p, sz, ctypes.c_char_p, ctypes.c_char_p, sz, P(sz)]
    L.fh_test_trailing_update.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int64, ctypes.c_int32,
                                          ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ei]
    L.fh_system_fill_stats.argtypes = [ctypes.c_void_p, P(FillStats)]
    L.fh_profile_enable.argtypes = [ctypes.c_int32]
    L.fh_profile_enable.restype = None
    L.fh_profile_reset.restype = None
    L.fh_profile_read.argtypes = [ctypes.c_int32, c_int64_p, c_double_p, c_double_p]
    L.fh_profile_overlap.argtypes = [ctypes.c_uint32, ctypes.c_uint32, c_double_p, c_double_p, c_double_p]
    _lib = L
    return L


def last_error() -> str:
    return load().fh_last_error().decode("utf-8", "replace")
