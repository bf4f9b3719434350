"""Python host interface mirroring the reference library surface.

Names, argument meanings and error behaviour follow the reference's public
API (fasterhenry/src/lib.rs:77-118): ``Geometry`` / ``Node`` / ``SegmentDef``
(geometry.rs), ``Port`` (mesh.rs), ``Discretization`` (solve.rs:409-510),
``SolverChoice`` (solve.rs:169-193), ``MeshSystem.assemble`` / ``.sweep`` /
``.impedance`` (solve.rs:680-893), ``solve`` (solve.rs:931),
``partial_inductance_matrix`` (inductance/batch.rs:246), ``lu_solve``
(dense.rs:43) and ``SweepResult`` (result.rs:47) with its JSON, MAT v4 and
SPICE writers (fasterhenry-cli/src/{main,mat,spice}.rs).  Everything that
computes runs through the C ABI on the GPU; nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import enum
import json
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N

MU0 = 4.0e-7 * np.pi
DENSE_PATH_MAX_FILAMENTS = 10_000


# ---------------------------------------------------------------------------
# Errors (SolveError, KernelError, MeshError, GeometryError, DiscretizeError)
# ---------------------------------------------------------------------------
class FasterHenryError(RuntimeError):
    status = -1

    def __init__(self, message: str, info: Optional[N.ErrorInfo] = None):
        super().__init__(message)
        self.info = info


class NoDevice(FasterHenryError):
    status = N.ERR_NO_DEVICE


class CudaError(FasterHenryError):
    status = N.ERR_CUDA


class OutOfMemory(FasterHenryError):
    status = N.ERR_OUT_OF_MEMORY


class GeometryError(FasterHenryError):
    status = N.ERR_GEOMETRY


class DiscretizeError(FasterHenryError):
    status = N.ERR_DISCRETIZE


class KernelError(FasterHenryError):
    @property
    def first(self) -> int:
        return int(self.info.index_a) if self.info else 0

    @property
    def second(self) -> int:
        return int(self.info.index_b) if self.info else 0


class CoincidentSamples(KernelError):
    status = N.ERR_KERNEL_COINCIDENT


class NotFinite(KernelError):
    status = N.ERR_KERNEL_NOT_FINITE


class MeshError(FasterHenryError):
    status = N.ERR_MESH


class InvalidGrading(FasterHenryError):
    status = N.ERR_INVALID_GRADING


class InvalidFrequency(FasterHenryError):
    status = N.ERR_INVALID_FREQUENCY

    @property
    def index(self) -> int:
        return int(self.info.index_a)

    @property
    def value(self) -> float:
        return float(self.info.frequency)


class Singular(FasterHenryError):
    status = N.ERR_SINGULAR

    @property
    def frequency(self) -> float:
        return float(self.info.frequency)


class NotConverged(FasterHenryError):
    status = N.ERR_NOT_CONVERGED


class CouplingError(FasterHenryError):
    """SolveError::Coupling(CouplingError) (coupling.rs:93-130): ``kind`` is
    "unknown_group", "segment_count_mismatch" or "non_transitive"."""
    status = N.ERR_COUPLING

    @property
    def kind(self) -> str:
        return {1: "unknown_group", 2: "segment_count_mismatch", 3: "non_transitive"}.get(
            int(self.info.detail) if self.info else 0, "")


class InvalidExcitation(FasterHenryError):
    """SolveError::InvalidExcitation{expected, got} (solve.rs:592-599)."""
    status = N.ERR_INVALID_EXCITATION

    @property
    def expected(self) -> int:
        return int(self.info.index_a)

    @property
    def got(self) -> int:
        return int(self.info.index_b)


class Unsupported(FasterHenryError):
    status = N.ERR_UNSUPPORTED


class PfftError(FasterHenryError):
    """PfftError::{InvalidParameter, GridTooLarge} (pfft/mod.rs:234-253)."""
    status = N.ERR_PFFT


class InvalidArgument(FasterHenryError, ValueError):
    status = N.ERR_INVALID_ARGUMENT


_ERRORS = {c.status: c for c in (NoDevice, CudaError, OutOfMemory, GeometryError, DiscretizeError, CoincidentSamples,
                                 NotFinite, MeshError, InvalidGrading, InvalidFrequency, Singular, NotConverged,
                                 Unsupported, InvalidArgument, PfftError, InvalidExcitation,
                                 CouplingError)}


def _check(status: int, info: Optional[N.ErrorInfo] = None) -> None:
    if status == N.OK:
        return
    cls = _ERRORS.get(status, FasterHenryError)
    raise cls(N.last_error() or ("status %d" % status), info)


# ---------------------------------------------------------------------------
# Geometry model (geometry.rs, mesh.rs)
# ---------------------------------------------------------------------------
@dataclasses.dataclass(frozen=True)
class Node:
    x: float
    y: float
    z: float


@dataclasses.dataclass(frozen=True)
class SegmentDef:
    a: int
    b: int
    width: float
    height: float
    sigma: float
    width_dir: Optional[Tuple[float, float, float]] = None


@dataclasses.dataclass(frozen=True)
class Port:
    positive: int
    negative: int
    name: Optional[str] = None


class Geometry:
    """Nodes and the segments joining them (geometry.rs:338-467).  Validation
    of nodes and segments happens in ``add_node`` / ``add_segment``, with the
    reference's error conditions."""

    def __init__(self):
        self.nodes: List[Node] = []
        self.segments: List[SegmentDef] = []

    @classmethod
    def from_parts(cls, nodes: Sequence, segments: Sequence) -> "Geometry":
        g = cls()
        for n in nodes:
            g.add_node(n if isinstance(n, Node) else Node(*n))
        for s in segments:
            g.add_segment(s)
        return g

    def add_node(self, node) -> int:
        node = node if isinstance(node, Node) else Node(*node)
        if not all(np.isfinite([node.x, node.y, node.z])):
            raise GeometryError("node %d has a non-finite coordinate" % len(self.nodes))
        self.nodes.append(node)
        return len(self.nodes) - 1

    def add_segment(self, seg) -> int:
        if isinstance(seg, dict):
            seg = SegmentDef(seg["a"], seg["b"], seg["width"], seg["height"], seg["sigma"], seg.get("width_dir"))
        idx = len(self.segments)
        # Validate through the library's own rule (Segment::validate).  With
        # both ends in range only the segment's own two nodes take part (the
        # nodes are finite by add_node), so they alone are passed; adding a
        # segment then costs O(1) instead of O(nodes).
        n = len(self.nodes)
        if 0 <= seg.a < n and 0 <= seg.b < n:
            ends = [self.nodes[seg.a]] if seg.a == seg.b else [self.nodes[seg.a], self.nodes[seg.b]]
            local = dataclasses.replace(seg, a=0, b=0 if seg.a == seg.b else 1)
            nodes, segs, count = _nodes(ends), _segments([local]), len(ends)
        else:
            nodes, segs, count = _nodes(self.nodes), _segments([seg]), n
        disc = _disc({"kind": "uniform", "nw": 1, "nh": 1})[0]
        cnt = ctypes.c_size_t()
        info = N.ErrorInfo()
        st = N.load().fh_discretize(nodes, count, segs, 1, ctypes.byref(disc), None, 0, ctypes.byref(cnt),
                                    None, ctypes.byref(info))
        if st == N.ERR_GEOMETRY:
            msg = N.last_error().replace("segment 0", "segment %d" % idx)
            raise GeometryError(msg, info)
        _check(st, info)
        self.segments.append(seg)
        return idx

    def segment_count(self) -> int:
        return len(self.segments)

    @classmethod
    def from_deck(cls, deck) -> "Geometry":
        return cls.from_parts(deck.nodes, deck.segments)


def _nodes(nodes: Sequence) -> ctypes.Array:
    arr = (N.Node * max(1, len(nodes)))()
    for i, n in enumerate(nodes):
        if isinstance(n, Node):
            arr[i].x, arr[i].y, arr[i].z = n.x, n.y, n.z
        else:
            arr[i].x, arr[i].y, arr[i].z = n
    return arr


def _segments(segs: Sequence) -> ctypes.Array:
    arr = (N.SegmentDef * max(1, len(segs)))()
    for i, s in enumerate(segs):
        if isinstance(s, dict):
            s = SegmentDef(s["a"], s["b"], s["width"], s["height"], s["sigma"], s.get("width_dir"))
        arr[i].a, arr[i].b = s.a, s.b
        arr[i].width, arr[i].height, arr[i].sigma = s.width, s.height, s.sigma
        arr[i].has_width_dir = 0 if s.width_dir is None else 1
        if s.width_dir is not None:
            for k in range(3):
                arr[i].width_dir[k] = s.width_dir[k]
    return arr


def _ports(ports: Sequence) -> ctypes.Array:
    arr = (N.Port * max(1, len(ports)))()
    for i, p in enumerate(ports):
        if isinstance(p, Port):
            arr[i].positive, arr[i].negative = p.positive, p.negative
        else:
            arr[i].positive, arr[i].negative = p[0], p[1]
    return arr


# ---------------------------------------------------------------------------
# Discretization and SolverChoice (solve.rs:169-510)
# ---------------------------------------------------------------------------
class Discretization:
    """Constructors mirror the reference's variants; the value is a dict
    (the form the synthetic decks in ``fixtures`` use)."""

    @staticmethod
    def uniform(nw: int, nh: int) -> dict:
        return {"kind": "uniform", "nw": nw, "nh": nh}

    @staticmethod
    def per_segment(grids: Sequence[Tuple[int, int]]) -> dict:
        return {"kind": "per_segment", "grids": [tuple(g) for g in grids]}

    @staticmethod
    def graded(nw: int, nh: int, ratio: float) -> dict:
        return {"kind": "graded", "nw": nw, "nh": nh, "ratio": ratio}

    @staticmethod
    def skin_depth(frequency_hz: float, target_skin_depths: float, ratio: float, max_per_axis: int = 32) -> dict:
        return {"kind": "skin_depth", "frequency_hz": frequency_hz, "target_skin_depths": target_skin_depths,
                "ratio": ratio, "max_per_axis": max_per_axis}

    @staticmethod
    def per_segment_graded(grids: Sequence[Tuple[int, int, float, float]]) -> dict:
        return {"kind": "per_segment_graded", "grids": [tuple(g) for g in grids]}


_KIND = {"uniform": 0, "per_segment": 1, "graded": 2, "skin_depth": 3, "per_segment_graded": 4}


def _disc(d: dict):
    c = N.Discretization()
    c.kind = _KIND[d["kind"]]
    c.nw, c.nh = d.get("nw", 0), d.get("nh", 0)
    c.ratio = d.get("ratio", 1.0)
    c.frequency_hz = d.get("frequency_hz", 0.0)
    c.target_skin_depths = d.get("target_skin_depths", 0.0)
    c.max_per_axis = d.get("max_per_axis", 32)
    grids = d.get("grids", [])
    arr = (N.AxisGrading * max(1, len(grids)))()
    for i, g in enumerate(grids):
        arr[i].nw, arr[i].nh = g[0], g[1]
        arr[i].width_ratio = g[2] if len(g) > 2 else 1.0
        arr[i].height_ratio = g[3] if len(g) > 3 else 1.0
    c.per_segment = ctypes.cast(arr, ctypes.POINTER(N.AxisGrading))
    c.per_segment_len = len(grids)
    return c, arr


class SolverChoice(enum.IntEnum):
    AUTO = 0
    DENSE = 1
    ITERATIVE = 2

    def resolve(self, filaments: int) -> str:
        return "dense" if N.load().fh_solver_resolve(int(self), filaments) == 0 else "iterative"


class Precision(enum.IntEnum):
    """FP64: the reference's FP64 LU.  MIXED_BF16X3: FP32 factors with
    split-BF16 x3 tensor-core trailing updates and FP64-residual refinement."""
    FP64 = 0
    MIXED_BF16X3 = 1
    MIXED_FP32 = 2


# ---------------------------------------------------------------------------
# Filaments and the fill
# ---------------------------------------------------------------------------
FILAMENT_FIELDS = 19


def _fil_array(filaments: np.ndarray) -> ctypes.Array:
    f = np.ascontiguousarray(filaments, dtype=np.float64).reshape(-1, FILAMENT_FIELDS)
    arr = (N.Filament * max(1, len(f)))()
    ctypes.memmove(arr, f.ctypes.data, f.nbytes)
    return arr


def discretize(geometry, discretization: dict) -> Tuple[np.ndarray, np.ndarray]:
    """Filaments (n x 19: start, end, length, length/width/height unit
    vectors, width, height, sigma) and the per-segment bundle sizes."""
    nodes, segs = _geom_arrays(geometry)
    disc, keep = _disc(discretization)
    cnt = ctypes.c_size_t()
    info = N.ErrorInfo()
    nseg = len(geometry.segments)
    per = np.zeros(max(1, nseg), dtype=np.int64)
    L = N.load()
    _check(L.fh_discretize(nodes, len(geometry.nodes), segs, nseg, ctypes.byref(disc), None, 0, ctypes.byref(cnt),
                           None, ctypes.byref(info)), info)
    out = (N.Filament * max(1, cnt.value))()
    _check(L.fh_discretize(nodes, len(geometry.nodes), segs, nseg, ctypes.byref(disc), out, cnt.value,
                           ctypes.byref(cnt), per.ctypes.data_as(N.c_int64_p), ctypes.byref(info)), info)
    arr = np.frombuffer(out, dtype=np.float64, count=cnt.value * FILAMENT_FIELDS).reshape(-1, FILAMENT_FIELDS).copy()
    return arr, per[:nseg].copy()


def _geom_arrays(geometry):
    return _nodes(geometry.nodes), _segments(geometry.segments)


def partial_inductance_matrix(filaments: np.ndarray, methods: bool = False):
    """Symmetric partial-inductance matrix of the filaments (batch.rs:246),
    evaluated on the GPU.  With ``methods=True`` also returns the per-entry
    inductance::Method ids."""
    f = np.ascontiguousarray(filaments, dtype=np.float64).reshape(-1, FILAMENT_FIELDS)
    n = len(f)
    Lm = np.zeros((n, n), order="F")
    meth = np.zeros((n, n), dtype=np.int8, order="F") if methods else None
    info = N.ErrorInfo()
    _check(N.load().fh_partial_inductance_matrix(_fil_array(f), n, Lm.ctypes.data_as(N.c_double_p),
                                                 meth.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)) if methods else None,
                                                 ctypes.byref(info)), info)
    return (Lm, meth) if methods else Lm


def mutual_inductance(a: np.ndarray, b: np.ndarray) -> float:
    """Partial mutual inductance of two filaments (inductance/mod.rs:215)."""
    return float(partial_inductance_matrix(np.stack([a, b]))[0, 1])


def self_inductance(f: np.ndarray) -> float:
    """Partial self inductance (inductance/mod.rs:196)."""
    return float(partial_inductance_matrix(np.asarray(f).reshape(1, -1))[0, 0])


def lu_solve(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Solve a x = b (complex) with the device FP64 blocked LU (dense.rs:43).
    Raises Singular on an exactly zero pivot."""
    a = np.asarray(a, dtype=np.complex128)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise InvalidArgument("lu_solve: the matrix must be square")
    bb = np.asarray(b, dtype=np.complex128)
    vec = bb.ndim == 1
    if bb.ndim == 0 or bb.shape[0] != a.shape[0]:
        raise InvalidArgument("lu_solve: right-hand side has the wrong number of rows")
    bb = bb.reshape(a.shape[0], -1)
    af = np.asfortranarray(a)
    bf = np.asfortranarray(bb)
    x = np.zeros_like(bf, order="F")
    info = N.ErrorInfo()
    _check(N.load().fh_lu_solve_c64(af.ctypes.data_as(N.c_double_p), a.shape[0], bf.ctypes.data_as(N.c_double_p),
                                    bf.shape[1], x.ctypes.data_as(N.c_double_p), ctypes.byref(info)), info)
    return x.reshape(-1) if vec else x


def mesh_matrix(geometry, per_segment: Sequence[int], ports: Sequence):
    """Loop basis M as CSR (row_ptr, branch, sign, internal_count)
    (mesh.rs:170)."""
    segs = _segments(geometry.segments)
    per = np.ascontiguousarray(per_segment, dtype=np.int64)
    pts = _ports(ports)
    nrows, nnz, nint = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
    info = N.ErrorInfo()
    L = N.load()
    _check(L.fh_mesh_build(segs, len(geometry.segments), len(geometry.nodes), per.ctypes.data_as(N.c_int64_p), pts,
                           len(ports), None, None, None, 0, 0, ctypes.byref(nrows), ctypes.byref(nnz),
                           ctypes.byref(nint), ctypes.byref(info)), info)
    rp = np.zeros(nrows.value + 1, dtype=np.int64)
    br = np.zeros(nnz.value, dtype=np.int64)
    sg = np.zeros(nnz.value)
    _check(L.fh_mesh_build(segs, len(geometry.segments), len(geometry.nodes), per.ctypes.data_as(N.c_int64_p), pts,
                           len(ports), rp.ctypes.data_as(N.c_int64_p), br.ctypes.data_as(N.c_int64_p),
                           sg.ctypes.data_as(N.c_double_p), len(rp), len(br), ctypes.byref(nrows), ctypes.byref(nnz),
                           ctypes.byref(nint), ctypes.byref(info)), info)
    return rp, br, sg, nint.value


# ---------------------------------------------------------------------------
# The dense system (MeshSystem) and the sweep result
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class SweepResult:
    """result.rs:47-104: impedance_ohm[k][i][j] is Z at frequencies_hz[k]."""
    ports: List[Port]
    frequencies_hz: List[float]
    impedance_ohm: np.ndarray          # (nf, p, p) complex
    counts: Dict[str, int]
    timing: Optional[Dict[str, float]] = None
    refinement_iterations: Optional[List[int]] = None
    residuals: Optional[List[float]] = None
    precision: Precision = Precision.FP64

    SCHEMA_VERSION = 1

    def resistance(self, index: int) -> np.ndarray:
        return self.impedance_ohm[index].real.copy()

    def inductance(self, index: int) -> Optional[np.ndarray]:
        omega = 2.0 * np.pi * self.frequencies_hz[index]
        return None if omega == 0.0 else self.impedance_ohm[index].imag / omega

    def without_timing(self) -> "SweepResult":
        return dataclasses.replace(self, timing=None)

    def _z_interleaved(self) -> np.ndarray:
        z = np.ascontiguousarray(self.impedance_ohm, dtype=np.complex128)
        return z.view(np.float64).reshape(-1)

    def to_json(self) -> str:
        """The reference's JSON document (schema_version 1), formatted by the
        library (serde_json float formatting)."""
        ports = _ports(self.ports)
        names = (ctypes.c_char_p * max(1, len(self.ports)))()
        for i, p in enumerate(self.ports):
            names[i] = (p.name.encode() if isinstance(p, Port) and p.name else None)
        f = np.ascontiguousarray(self.frequencies_hz, dtype=np.float64)
        z = self._z_interleaved()
        c = N.Counts(*[self.counts[k] for k in ("nodes", "segments", "filaments", "meshes", "internal_meshes", "ports")])
        t = None
        if self.timing is not None:
            t = N.Timing(*[self.timing[k] for k in ("inductance_s", "assembly_s", "solve_s", "total_s")])
        L = N.load()
        length = ctypes.c_size_t()
        args = [ports, names, len(self.ports), f.ctypes.data_as(N.c_double_p), len(f), z.ctypes.data_as(N.c_double_p),
                ctypes.byref(c), ctypes.byref(t) if t is not None else None]
        _check(L.fh_sweep_json(*args, None, 0, ctypes.byref(length)))
        buf = ctypes.create_string_buffer(length.value + 1)
        _check(L.fh_sweep_json(*args, buf, length.value + 1, ctypes.byref(length)))
        return buf.value.decode()

    def write_zc_mat(self, path: str) -> None:
        f = np.ascontiguousarray(self.frequencies_hz, dtype=np.float64)
        z = self._z_interleaved()
        _check(N.load().fh_write_zc_mat(path.encode(), len(self.ports), f.ctypes.data_as(N.c_double_p), len(f),
                                        z.ctypes.data_as(N.c_double_p)))

    def spice_subckt(self, frequency_index: int, name: str) -> str:
        f = np.ascontiguousarray(self.frequencies_hz, dtype=np.float64)
        z = self._z_interleaved()
        L = N.load()
        length = ctypes.c_size_t()
        args = [len(self.ports), f.ctypes.data_as(N.c_double_p), len(f), z.ctypes.data_as(N.c_double_p),
                frequency_index, name.encode()]
        _check(L.fh_spice_subckt(*args, None, 0, ctypes.byref(length)))
        buf = ctypes.create_string_buffer(length.value + 1)
        _check(L.fh_spice_subckt(*args, buf, length.value + 1, ctypes.byref(length)))
        return buf.value.decode()


class MeshSystem:
    """Assembled dense system resident on the GPU (solve.rs:643-893)."""

    def __init__(self, handle, geometry, ports):
        self._h = handle
        self.ports = [p if isinstance(p, Port) else Port(p[0], p[1]) for p in ports]
        c = N.Counts()
        _check(N.load().fh_system_counts(handle, ctypes.byref(c)))
        self._counts = {k: int(getattr(c, k)) for k, _ in N.Counts._fields_}

    @classmethod
    def assemble(cls, geometry, ports: Sequence, discretization: dict,
                 solver: SolverChoice = SolverChoice.DENSE, coupling: Optional["Coupling"] = None) -> "MeshSystem":
        """MeshSystem::assemble, or assemble_with_coupling (solve.rs:680-766)
        when ``coupling`` is given."""
        nodes, segs = _geom_arrays(geometry)
        pts = _ports(ports)
        disc, keep = _disc(discretization)
        h = ctypes.c_void_p()
        info = N.ErrorInfo()
        spec, hold = (coupling._spec() if coupling is not None else (None, None))
        _check(N.load().fh_system_create_coupled(nodes, len(geometry.nodes), segs, len(geometry.segments), pts,
                                                 len(ports), ctypes.byref(disc),
                                                 ctypes.byref(spec) if spec is not None else None, int(solver),
                                                 ctypes.byref(h), ctypes.byref(info)), info)
        out = cls(h, geometry, ports)
        out.coupling = coupling if coupling is not None else Coupling.all_pairs()
        return out

    def kept_pairs(self) -> Tuple[int, int]:
        """(kept, total) filament pairs of the fill: PairMask::kept_pairs and
        total_pairs (inductance/batch.rs:88-117)."""
        kept, total = ctypes.c_int64(), ctypes.c_int64()
        _check(N.load().fh_system_coupling(self._h, ctypes.byref(kept), ctypes.byref(total), None, 0, None))
        return int(kept.value), int(total.value)

    def truncation_warnings(self) -> List["TruncationWarning"]:
        """Truncated group pairs closer than their extent
        (Coupling::truncation_warnings, coupling.rs:285-318)."""
        count = ctypes.c_size_t()
        L = N.load()
        _check(L.fh_system_coupling(self._h, None, None, None, 0, ctypes.byref(count)))
        buf = (N.TruncationWarning * max(1, count.value))()
        _check(L.fh_system_coupling(self._h, None, None, buf, count.value, ctypes.byref(count)))
        names = getattr(self, "coupling", Coupling.all_pairs()).group_names(self._counts["segments"])
        return [TruncationWarning((names[buf[k].group_a], names[buf[k].group_b]), buf[k].separation, buf[k].extent)
                for k in range(count.value)]

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.load().fh_system_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def counts(self) -> Dict[str, int]:
        return dict(self._counts)

    def timing(self) -> Dict[str, float]:
        t = N.Timing()
        _check(N.load().fh_system_timing(self._h, ctypes.byref(t)))
        return {k: float(getattr(t, k)) for k, _ in N.Timing._fields_}

    def filaments(self) -> np.ndarray:
        n = self._counts["filaments"]
        out = (N.Filament * max(1, n))()
        _check(N.load().fh_system_filaments(self._h, out, n))
        return np.frombuffer(out, dtype=np.float64, count=n * FILAMENT_FIELDS).reshape(-1, FILAMENT_FIELDS).copy()

    def filament_resistances(self) -> np.ndarray:
        n = self._counts["filaments"]
        out = np.zeros(max(1, n))
        _check(N.load().fh_system_resistances(self._h, out.ctypes.data_as(N.c_double_p), n))
        return out[:n]

    def mesh_matrices(self) -> Tuple[np.ndarray, np.ndarray]:
        loops = self._counts["meshes"]
        r = np.zeros((loops, loops), order="F")
        l = np.zeros((loops, loops), order="F")
        _check(N.load().fh_system_mesh_matrices(self._h, r.ctypes.data_as(N.c_double_p), l.ctypes.data_as(N.c_double_p)))
        return r, l

    def sweep(self, frequencies: Sequence[float], precision: Precision = Precision.FP64) -> SweepResult:
        f = np.ascontiguousarray(frequencies, dtype=np.float64)
        p = self._counts["ports"]
        z = np.zeros((len(f), p, p), dtype=np.complex128)
        iters = np.zeros(max(1, len(f)), dtype=np.int32)
        resid = np.zeros(max(1, len(f)))
        rep = N.SweepReport(iters.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), resid.ctypes.data_as(N.c_double_p))
        info = N.ErrorInfo()
        _check(N.load().fh_sweep(self._h, f.ctypes.data_as(N.c_double_p), len(f), int(precision),
                                 z.ctypes.data_as(N.c_double_p), ctypes.byref(rep), ctypes.byref(info)), info)
        timing = self.timing()
        return SweepResult(self.ports, [float(x) for x in f], z, self.counts(), timing,
                           [int(x) for x in iters[:len(f)]] if precision != Precision.FP64 else None,
                           [float(x) for x in resid[:len(f)]] if precision != Precision.FP64 else None, precision)

    def impedance(self, frequency: float, precision: Precision = Precision.FP64) -> np.ndarray:
        return self.sweep([frequency], precision).impedance_ohm[0]

    def layout(self) -> Tuple[np.ndarray, np.ndarray, int]:
        """(segment of every filament, conductor of every segment, conductor
        count): the Layout of currents.rs:128-170."""
        n, nseg = self._counts["filaments"], self._counts["segments"]
        sof = np.zeros(max(1, n), dtype=np.int64)
        cos = np.zeros(max(1, nseg), dtype=np.int64)
        nc = ctypes.c_int64()
        _check(N.load().fh_system_layout(self._h, sof.ctypes.data_as(N.c_int64_p), cos.ctypes.data_as(N.c_int64_p),
                                         ctypes.byref(nc)))
        return sof[:n], cos[:nseg], int(nc.value)

    def currents(self, frequency, excitation: Optional[Sequence[complex]] = None,
                 precision: Precision = Precision.FP64):
        """Filament currents for the port-current phasors ``excitation``
        (default: 1 A into port 1, the other ports open) at one frequency or a
        list of them (MeshSystem::currents, solve.rs:845-868): one
        CurrentSolution per frequency."""
        return _solve_currents(self, frequency, excitation,
                               lambda *a: N.load().fh_currents(self._h, *a[:4], int(precision), *a[4:]))

    def gradient(self, frequency: float, params: Optional[Sequence["Param"]] = None) -> "GradientResult":
        """dZ/dp at one frequency by the stationary (adjoint) form
        (fh_gradient): one FP64 solve for the loop currents, one derivative
        fill, one product per derivative matrix.  ``params`` defaults to
        every segment's width, then every segment's thickness."""
        if params is None:
            nseg = self._counts["segments"]
            params = [Param("width", s) for s in range(nseg)] + [Param("thickness", s) for s in range(nseg)]
        params = list(params)
        spec = (N.ParamSpec * max(1, len(params)))()
        for k, q in enumerate(params):
            spec[k].kind = Param.KINDS[q.kind]
            spec[k].index = int(q.index)
        p = self._counts["ports"]
        z = np.zeros((p, p), dtype=np.complex128)
        dz = np.zeros((max(1, len(params)), p, p), dtype=np.complex128)
        rep = N.GradientReport()
        info = N.ErrorInfo()
        _check(N.load().fh_gradient(self._h, float(frequency), spec, len(params), z.ctypes.data_as(N.c_double_p),
                                    dz.ctypes.data_as(N.c_double_p), ctypes.byref(rep), ctypes.byref(info)), info)
        return GradientResult(float(frequency), params, z, dz[:len(params)],
                              {k: (int(getattr(rep, k)) if k == "pairs" else float(getattr(rep, k)))
                               for k, _ in N.GradientReport._fields_})


DEFAULT_GROUP = ""


class Coupling:
    """Segment group names and the group pairs whose mutual inductance is
    kept (Coupling, coupling.rs:150-283).  ``Coupling.all_pairs()`` keeps
    everything; ``Coupling.truncated(groups)`` keeps each group with itself
    and the pairs declared with ``coupled``, and the fill never evaluates the
    rest (they are zero in L).  Validation (unknown groups, too many tags,
    non-transitive declarations) happens at assembly (CouplingError)."""

    def __init__(self, segment_groups: Optional[Sequence[str]] = None, couples: Optional[List[Tuple[str, str]]] = None):
        self.segment_groups = list(segment_groups or [])
        self._couples = None if couples is None else [tuple(c) for c in couples]

    @classmethod
    def all_pairs(cls) -> "Coupling":
        return cls()

    @classmethod
    def truncated(cls, segment_groups: Sequence[str]) -> "Coupling":
        return cls(segment_groups, [])

    def coupled(self, a: str, b: str) -> "Coupling":
        return Coupling(self.segment_groups, (self._couples or []) + [(a, b)])

    def is_all_pairs(self) -> bool:
        return self._couples is None

    def is_trivial(self) -> bool:
        return not self.segment_groups and self._couples is None

    def group_of(self, index: int) -> str:
        return self.segment_groups[index] if index < len(self.segment_groups) else DEFAULT_GROUP

    def couples(self, a: str, b: str) -> bool:
        if self._couples is None or a == b:
            return True
        return any((x == a and y == b) or (x == b and y == a) for x, y in self._couples)

    def group_names(self, segment_count: int) -> List[str]:
        """Group names in order of first appearance over the segments."""
        names: List[str] = []
        for k in range(segment_count):
            g = self.group_of(k)
            if g not in names:
                names.append(g)
        return names

    def to_json(self) -> dict:
        """The serde form of the reference (coupling.rs:166-175): absent
        fields are the defaults, so all_pairs() is ``{}``."""
        d: dict = {}
        if self.segment_groups:
            d["segment_groups"] = list(self.segment_groups)
        if self._couples is not None:
            d["couples"] = [list(c) for c in self._couples]
        return d

    @classmethod
    def from_json(cls, d: dict) -> "Coupling":
        unknown = set(d) - {"segment_groups", "couples"}
        if unknown:
            raise InvalidArgument("unknown coupling field(s): %s" % ", ".join(sorted(unknown)))
        couples = d.get("couples")
        return cls(d.get("segment_groups", []), None if couples is None else [tuple(c) for c in couples])

    def __eq__(self, other) -> bool:
        return isinstance(other, Coupling) and self.to_json() == other.to_json()

    def _spec(self):
        enc = [g.encode() for g in self.segment_groups]
        groups = (ctypes.c_char_p * max(1, len(enc)))(*enc)
        flat = [x.encode() for c in (self._couples or []) for x in c]
        pairs = (ctypes.c_char_p * max(1, len(flat)))(*flat)
        spec = N.CouplingSpec(groups, len(enc), 0 if self._couples is None else 1, pairs, len(self._couples or []))
        return spec, (enc, groups, flat, pairs)


@dataclasses.dataclass
class TruncationWarning:
    """A truncated group pair closer than one extent (coupling.rs:132-160)."""
    groups: Tuple[str, str]
    separation: float
    extent: float

    def __str__(self) -> str:
        name = lambda g: "(default)" if g == "" else "'%s'" % g
        ratio = self.separation / self.extent if self.extent > 0 else float("inf")
        return ("mutual inductance between groups %s and %s is truncated, but they are only %.3e m apart — %.2fx "
                "their %.3e m extent; truncation is justified from about 10x"
                % (name(self.groups[0]), name(self.groups[1]), self.separation, ratio, self.extent))


CURRENTS_CSV_HEADER = ("frequency_hz,filament,segment,conductor,x_m,y_m,z_m,"
                       "current_re_a,current_im_a,current_abs_a,j_abs_a_per_m2,power_w")


def unit_excitation(ports: int) -> List[complex]:
    """1 A into port 1, every other port open (currents.rs:121-128)."""
    return [1.0 + 0j if k == 0 else 0j for k in range(ports)]


def _solve_currents(system, frequency, excitation, call):
    """The shared envelope of MeshSystem.currents and IterativeSystem.currents:
    output arrays, the C call (``call(freqs, nf, excitation, n_excitation,
    outputs..., balance, [outcomes,] info)`` with the system's own extras
    bound), and one CurrentSolution per frequency."""
    single = np.ndim(frequency) == 0
    f = np.ascontiguousarray(np.atleast_1d(frequency), dtype=np.float64)
    c = system.counts()
    p, n, nseg = c["ports"], c["filaments"], c["segments"]
    if excitation is None:
        excitation = unit_excitation(p)
    exc = np.ascontiguousarray(np.asarray(excitation, dtype=np.complex128).ravel())
    sof, cos, ncond = system.layout()
    nf = len(f)
    cur = np.zeros((nf, n), dtype=np.complex128)
    dens = np.zeros((nf, n))
    pw = np.zeros((nf, n))
    segc = np.zeros((nf, nseg), dtype=np.complex128)
    segp = np.zeros((nf, nseg))
    pk = np.zeros((nf, max(1, ncond)), dtype=np.int64)
    pkd = np.zeros((nf, max(1, ncond)))
    bal = (N.PowerBalance * max(1, nf))()
    info = N.ErrorInfo()
    dp = lambda a: a.ctypes.data_as(N.c_double_p)
    _check(call(dp(f), nf, exc.ctypes.data_as(N.c_double_p) if len(exc) else None, len(exc), dp(cur), dp(dens),
                dp(pw), dp(segc), dp(segp), pk.ctypes.data_as(N.c_int64_p), dp(pkd), bal, ctypes.byref(info)), info)
    fil = system.filaments()
    centres = 0.5 * (fil[:, 0:3] + fil[:, 3:6])
    out = []
    for k in range(nf):
        out.append(CurrentSolution(float(f[k]), exc.copy(), cur[k], dens[k], pw[k], sof, cos, centres, segc[k],
                                   segp[k], pk[k, :ncond], pkd[k, :ncond],
                                   {"dissipated_w": bal[k].dissipated_w, "input_w": bal[k].input_w,
                                    "relative_residual": bal[k].relative_residual}))
    return out[0] if single else out


@dataclasses.dataclass
class CurrentSolution:
    """All currents of one frequency and excitation (CurrentSolution,
    currents.rs:107-119), held as arrays: phasor currents (peak amperes),
    |J| in A/m^2 and time-average power P = |I|^2 R / 2 per filament, sums
    per segment, the filament of largest |J| per conductor, and the power
    balance."""
    frequency_hz: float
    excitation: np.ndarray
    current: np.ndarray
    current_density: np.ndarray
    power_w: np.ndarray
    segment_of_filament: np.ndarray
    conductor_of_segment: np.ndarray
    location: np.ndarray
    segment_current: np.ndarray
    segment_power_w: np.ndarray
    peak_filament: np.ndarray
    peak_current_density: np.ndarray
    power_balance: Dict[str, float]

    @property
    def segments(self) -> List[dict]:
        return [{"segment": s, "conductor": int(self.conductor_of_segment[s]),
                 "current": complex(self.segment_current[s]), "power_w": float(self.segment_power_w[s])}
                for s in range(len(self.segment_current))]

    @property
    def conductors(self) -> List[dict]:
        return [{"conductor": c, "peak_current_density": float(self.peak_current_density[c]),
                 "filament": int(self.peak_filament[c]), "location": [float(x) for x in self.location[self.peak_filament[c]]]}
                for c in range(len(self.peak_filament))]

    def csv_rows(self) -> List[str]:
        """Rows of the CLI's --currents CSV for this frequency (fasterhenry-cli/src/lib.rs:238-276)."""
        rows = []
        for k in range(len(self.current)):
            s = int(self.segment_of_filament[k])
            i = self.current[k]
            x, y, z = self.location[k]
            rows.append(",".join([_rust_e(self.frequency_hz), str(k), str(s), str(int(self.conductor_of_segment[s])),
                                  _rust_e(x), _rust_e(y), _rust_e(z), _rust_e(i.real), _rust_e(i.imag), _rust_e(abs(i)),
                                  _rust_e(self.current_density[k]), _rust_e(self.power_w[k])]))
        return rows

    def json_block(self) -> dict:
        """One entry of the CLI's ``currents.by_frequency`` JSON block."""
        seg = [{"segment": d["segment"], "conductor": d["conductor"],
                "current": [d["current"].real, d["current"].imag], "power_w": d["power_w"]} for d in self.segments]
        return {"frequency_hz": self.frequency_hz, "power_balance": dict(self.power_balance),
                "conductors": self.conductors, "segments": seg}


def _rust_e(x: float) -> str:
    """Rust's ``{:e}`` formatting of an f64: the shortest mantissa that reads
    back to the same value, exponent without padding or plus sign (1e6,
    2.5e-3, 0e0)."""
    x = float(x)
    if x != x:
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    if x == 0.0:
        return "-0e0" if math.copysign(1.0, x) < 0 else "0e0"
    for prec in range(17):
        cand = "%.*e" % (prec, x)
        if float(cand) == x:
            break
    m, e = cand.split("e")
    if "." in m:
        m = m.rstrip("0").rstrip(".")
    return "%se%d" % (m, int(e))


@dataclasses.dataclass(frozen=True)
class Param:
    """A geometric parameter of dZ/dp: the "width" or "thickness" of segment
    ``index``, or the "x" / "y" coordinate of node ``index`` (its segments in
    a plane z = const; "z" is rejected with Unsupported)."""
    kind: str
    index: int

    KINDS = {"width": 0, "thickness": 1, "x": 2, "y": 3, "z": 4}


@dataclasses.dataclass
class GradientResult:
    """Z (p x p) and dZ/dp (one p x p matrix per parameter, ohm per metre) at
    one frequency.  ``resistance_gradient`` and ``inductance_gradient`` are
    d Re Z / dp and d (Im Z / omega) / dp (zero frequency: inductance
    gradient undefined, reported as NaN)."""
    frequency_hz: float
    params: List[Param]
    impedance_ohm: np.ndarray
    gradient: np.ndarray
    report: Dict[str, float]

    @property
    def resistance_gradient(self) -> np.ndarray:
        return self.gradient.real

    @property
    def inductance_gradient(self) -> np.ndarray:
        w = 2.0 * np.pi * self.frequency_hz
        return self.gradient.imag / w if w > 0 else np.full(self.gradient.shape, np.nan)


def inductance_gradient(filaments: np.ndarray, tangents: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """The derivative fill on its own (fh_test_inductance_gradient): for
    filaments (n x 19) and their tangents (n x 4: sw, sh, gw, gh), returns
    (Dw, Dh) with D[a, b] = dL_ab / d(side a)."""
    f = np.ascontiguousarray(filaments, dtype=np.float64).reshape(-1, FILAMENT_FIELDS)
    fil = _fil_array(f)
    n = len(f)
    t = np.ascontiguousarray(tangents, dtype=np.float64).reshape(n, 4) if n else np.zeros((1, 4))
    dw = np.zeros((n, n), order="F")
    dh = np.zeros((n, n), order="F")
    info = N.ErrorInfo()
    _check(N.load().fh_test_inductance_gradient(fil, t.ctypes.data_as(N.c_double_p), n,
                                                dw.ctypes.data_as(N.c_double_p), dh.ctypes.data_as(N.c_double_p),
                                                ctypes.byref(info)), info)
    return dw, dh


def coordinate_gradient(filaments: np.ndarray, segment: Sequence[int]) -> Tuple[np.ndarray, ...]:
    """The coordinate derivative fill on its own
    (fh_test_coordinate_gradient): for filaments (n x 19) and the segment of
    each, returns (Dl, Dp, Ds, Dr) with D[a, b] = dL_ab / d(coordinate of a):
    translation along a's length axis, along z x l, stretch of its length,
    rotation about z through its centre."""
    f = np.ascontiguousarray(filaments, dtype=np.float64).reshape(-1, FILAMENT_FIELDS)
    fil = _fil_array(f)
    n = len(f)
    seg = np.ascontiguousarray(segment, dtype=np.int32).reshape(-1) if n else np.zeros(1, dtype=np.int32)
    outs = [np.zeros((n, n), order="F") for _ in range(4)]
    info = N.ErrorInfo()
    _check(N.load().fh_test_coordinate_gradient(fil, seg.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), n,
                                                *[o.ctypes.data_as(N.c_double_p) for o in outs],
                                                ctypes.byref(info)), info)
    return tuple(outs)


def near_pairs(filaments: np.ndarray, radius: float) -> Tuple[np.ndarray, np.ndarray]:
    """The device near-pair search of the pFFT set-up on its own
    (fh_test_near_pairs, pfft/near.rs:41-106): for each filament i the
    filaments j >= i within `radius` (separating-axis gap) whose directions
    are not orthogonal, ascending.  Returns (off, cols) as CSR arrays."""
    f = np.ascontiguousarray(filaments, dtype=np.float64).reshape(-1, FILAMENT_FIELDS)
    fil = _fil_array(f)
    n = len(f)
    off = np.zeros(n + 1, dtype=np.int64)
    total = ctypes.c_size_t(0)
    cap = max(64 * n, 1)
    for _ in range(2):
        cols = np.zeros(cap, dtype=np.int64)
        info = N.ErrorInfo()
        _check(N.load().fh_test_near_pairs(fil, n, float(radius), off.ctypes.data_as(N.c_int64_p),
                                           cols.ctypes.data_as(N.c_int64_p), cap, ctypes.byref(total),
                                           ctypes.byref(info)), info)
        if total.value <= cap:
            return off, cols[:total.value]
        cap = total.value
    raise RuntimeError("near_pairs: capacity")


def grid_convolution(sources: np.ndarray, padded: Sequence[int], spacing: float, fp32: bool = False) -> np.ndarray:
    """The pFFT grid convolution on its own (fh_test_grid_convolution):
    ``sources`` (fields x n0 x n1 x n2) convolved with 1 / (spacing |d|) on
    the padded torus ``padded`` by the library's own transforms."""
    q = np.ascontiguousarray(sources, dtype=np.float64)
    if q.ndim == 3:
        q = q[None]
    n = np.array(q.shape[1:], dtype=np.int64)
    m = np.ascontiguousarray(padded, dtype=np.int64)
    out = np.zeros_like(q)
    info = N.ErrorInfo()
    _check(N.load().fh_test_grid_convolution(n.ctypes.data_as(N.c_int64_p), m.ctypes.data_as(N.c_int64_p),
                                             float(spacing), 1 if fp32 else 0, q.ctypes.data_as(N.c_double_p),
                                             q.shape[0], out.ctypes.data_as(N.c_double_p), ctypes.byref(info)), info)
    return out


def solve(geometry, ports: Sequence, discretization: dict, frequencies: Sequence[float],
          precision: Precision = Precision.FP64, solver: SolverChoice = SolverChoice.DENSE,
          iterative: Optional[IterativeParams] = None) -> SweepResult:
    """MeshSystem.assemble followed by MeshSystem.sweep (solve.rs:931-938),
    or IterativeSystem when ``solver`` resolves to the iterative path
    (SolverChoice::resolve, solve.rs:169-193)."""
    n = len(discretize(geometry, discretization)[0]) if solver == SolverChoice.AUTO else 0
    path = solver.resolve(n) if solver != SolverChoice.DENSE else "dense"
    if path == "iterative":
        with IterativeSystem.assemble(geometry, ports, discretization, iterative) as system:
            return system.sweep(frequencies)
    with MeshSystem.assemble(geometry, ports, discretization) as system:
        return system.sweep(frequencies, precision)


def batch_sweep(systems: Sequence["MeshSystem"], frequencies: Sequence[Sequence[float]],
                precision: Precision = Precision.MIXED_BF16X3, concurrency: int = 4) -> List[SweepResult]:
    """Sweeps many independent systems (uneven sizes) at once: each over its
    own frequencies, up to ``concurrency`` concurrently on the device
    (fh_batch_sweep).  Results as MeshSystem.sweep, in input order."""
    k = len(systems)
    if len(frequencies) != k:
        raise InvalidArgument("one frequency list per system")
    f_arrays = [np.ascontiguousarray(f, dtype=np.float64) for f in frequencies]
    z_arrays = [np.zeros((len(f), s.counts()["ports"], s.counts()["ports"]), dtype=np.complex128)
                for s, f in zip(systems, f_arrays)]
    handles = (ctypes.c_void_p * max(1, k))(*[s._h for s in systems])
    fptr = (N.c_double_p * max(1, k))(*[f.ctypes.data_as(N.c_double_p) for f in f_arrays])
    nfs = (ctypes.c_size_t * max(1, k))(*[len(f) for f in f_arrays])
    zptr = (N.c_double_p * max(1, k))(*[z.ctypes.data_as(N.c_double_p) for z in z_arrays])
    info = N.ErrorInfo()
    _check(N.load().fh_batch_sweep(handles, k, fptr, nfs, int(precision), zptr, int(concurrency),
                                   ctypes.byref(info)), info)
    return [SweepResult(s.ports, [float(x) for x in f], z, s.counts(), s.timing(), None, None, precision)
            for s, f, z in zip(systems, f_arrays, z_arrays)]


# ---------------------------------------------------------------------------
# Matrix-free path: the precorrected-FFT operator (pfft/mod.rs)
# ---------------------------------------------------------------------------
@dataclasses.dataclass(frozen=True)
class PfftParams:
    """PfftParams (pfft/mod.rs:183-232).  ``spacing`` None means
    GridSpacing::Auto with ``cells_per_filament``; a float is
    GridSpacing::Fixed in metres.  ``fft_fp32`` runs the grid convolution in
    FP32 instead of FP64 (projection, interpolation and the near-field
    precorrection stay FP64)."""
    cells_per_filament: float = 8.0
    spacing: Optional[float] = None
    near_field_radius: float = 8.0
    interpolation_order: int = 5
    fft_fp32: bool = False

    def _native(self) -> N.PfftParams:
        p = N.PfftParams()
        p.spacing_kind = 0 if self.spacing is None else 1
        p.interpolation_order = int(self.interpolation_order)
        p.cells_per_filament = float(self.cells_per_filament)
        p.spacing = float(self.spacing or 0.0)
        p.near_field_radius = float(self.near_field_radius)
        p.fft_precision = 1 if self.fft_fp32 else 0
        return p


class PfftOperator:
    """Matrix-free partial-inductance operator: ``apply(x)`` = L x without
    forming L (PfftOperator::new / apply / stats, pfft/mod.rs:332-597).
    Set-up on the host and the device; products on the device."""

    def __init__(self, filaments: np.ndarray, params: Optional[PfftParams] = None):
        f = np.ascontiguousarray(filaments, dtype=np.float64).reshape(-1, FILAMENT_FIELDS)
        self._n = len(f)
        arr = _fil_array(f)
        p = (params or PfftParams())._native()
        h = ctypes.c_void_p()
        info = N.ErrorInfo()
        _check(N.load().fh_pfft_create(arr, self._n, ctypes.byref(p), ctypes.byref(h), ctypes.byref(info)), info)
        self._h = h

    def __len__(self) -> int:
        return self._n

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.load().fh_pfft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def apply(self, x: np.ndarray) -> np.ndarray:
        """L x for one vector (length n) or several (count x n)."""
        x = np.asarray(x, dtype=np.float64)
        one = x.ndim == 1
        xs = np.ascontiguousarray(x.reshape(1, -1) if one else x)
        if xs.shape[1] != self._n:
            raise InvalidArgument("pFFT operator of dimension %d applied to a vector of length %d"
                                  % (self._n, xs.shape[1]))
        y = np.zeros_like(xs)
        info = N.ErrorInfo()
        _check(N.load().fh_pfft_apply(self._h, xs.ctypes.data_as(N.c_double_p), y.ctypes.data_as(N.c_double_p),
                                      xs.shape[0], ctypes.byref(info)), info)
        return y[0] if one else y

    def stats(self) -> Dict[str, object]:
        s = N.PfftStats()
        _check(N.load().fh_pfft_get_stats(self._h, ctypes.byref(s)))
        return {"filaments": int(s.filaments), "grid_spacing": float(s.grid_spacing),
                "grid_dims": [int(v) for v in s.grid_dims], "fft_dims": [int(v) for v in s.fft_dims],
                "projection_entries": int(s.projection_entries), "near_entries": int(s.near_entries),
                "memory_bytes": int(s.memory_bytes), "setup_host_s": float(s.setup_host_s),
                "setup_device_s": float(s.setup_device_s), "setup_near_s": float(s.setup_near_s)}


@dataclasses.dataclass(frozen=True)
class GmresParams:
    """GmresParams (gmres.rs:32-58)."""
    tolerance: float = 1e-10
    restart: int = 100
    max_iterations: int = 5000

    def _native(self) -> N.GmresParams:
        g = N.GmresParams()
        g.tolerance, g.restart, g.max_iterations = float(self.tolerance), int(self.restart), int(self.max_iterations)
        return g


@dataclasses.dataclass(frozen=True)
class IterativeParams:
    """IterativeParams (iterative.rs:100-107)."""
    pfft: PfftParams = PfftParams()
    gmres: GmresParams = GmresParams()


@dataclasses.dataclass(frozen=True)
class GmresOutcome:
    """GmresOutcome (gmres.rs:61-73)."""
    iterations: int
    relative_residual: float
    converged: bool


class IterativeSystem:
    """Matrix-free port impedance: GMRES on the precorrected-FFT operator
    (IterativeSystem, iterative.rs:109-409).  Same results as MeshSystem to
    the pFFT far-field accuracy and the GMRES tolerance."""

    def __init__(self, handle, ports):
        self._h = handle
        self.ports = [p if isinstance(p, Port) else Port(p[0], p[1]) for p in ports]
        self.last_outcomes: List[List[GmresOutcome]] = []

    @classmethod
    def assemble(cls, geometry, ports: Sequence, discretization: dict,
                 params: Optional[IterativeParams] = None) -> "IterativeSystem":
        params = params or IterativeParams()
        nodes, segs = _geom_arrays(geometry)
        pts = _ports(ports)
        disc, keep = _disc(discretization)
        pp, gp = params.pfft._native(), params.gmres._native()
        h = ctypes.c_void_p()
        info = N.ErrorInfo()
        _check(N.load().fh_iterative_create(nodes, len(geometry.nodes), segs, len(geometry.segments), pts, len(ports),
                                            ctypes.byref(disc), ctypes.byref(pp), ctypes.byref(gp), ctypes.byref(h),
                                            ctypes.byref(info)), info)
        return cls(h, ports)

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.load().fh_iterative_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def counts(self) -> Dict[str, int]:
        c = N.Counts()
        _check(N.load().fh_iterative_counts(self._h, ctypes.byref(c)))
        return {k: int(getattr(c, k)) for k, _ in N.Counts._fields_}

    def timing(self) -> Dict[str, float]:
        t = N.Timing()
        _check(N.load().fh_iterative_timing(self._h, ctypes.byref(t)))
        return {k: float(getattr(t, k)) for k, _ in N.Timing._fields_}

    def operator_stats(self) -> Dict[str, object]:
        s = N.PfftStats()
        _check(N.load().fh_iterative_pfft_stats(self._h, ctypes.byref(s)))
        return {"filaments": int(s.filaments), "grid_spacing": float(s.grid_spacing),
                "grid_dims": [int(v) for v in s.grid_dims], "fft_dims": [int(v) for v in s.fft_dims],
                "projection_entries": int(s.projection_entries), "near_entries": int(s.near_entries),
                "memory_bytes": int(s.memory_bytes), "setup_host_s": float(s.setup_host_s),
                "setup_device_s": float(s.setup_device_s), "setup_near_s": float(s.setup_near_s)}

    def sweep(self, frequencies: Sequence[float]) -> SweepResult:
        f = np.ascontiguousarray(frequencies, dtype=np.float64)
        p = len(self.ports)
        z = np.zeros((len(f), p, p), dtype=np.complex128)
        oc = (N.GmresOutcome * max(1, len(f) * p))()
        info = N.ErrorInfo()
        _check(N.load().fh_iterative_sweep(self._h, f.ctypes.data_as(N.c_double_p), len(f),
                                           z.ctypes.data_as(N.c_double_p), oc, ctypes.byref(info)), info)
        self.last_outcomes = [[GmresOutcome(int(oc[k * p + q].iterations), float(oc[k * p + q].relative_residual),
                                            bool(oc[k * p + q].converged)) for q in range(p)] for k in range(len(f))]
        return SweepResult(self.ports, [float(x) for x in f], z, self.counts(), self.timing())

    def impedance(self, frequency: float) -> np.ndarray:
        return self.sweep([frequency]).impedance_ohm[0]

    def solve(self, frequency: float) -> Tuple[np.ndarray, List[GmresOutcome]]:
        """Z at one frequency with the GMRES outcome of every port."""
        z = self.impedance(frequency)
        return z, self.last_outcomes[0]

    def filaments(self) -> np.ndarray:
        n = self.counts()["filaments"]
        out = (N.Filament * max(1, n))()
        _check(N.load().fh_iterative_filaments(self._h, out, n))
        return np.frombuffer(out, dtype=np.float64, count=n * FILAMENT_FIELDS).reshape(-1, FILAMENT_FIELDS).copy()

    def layout(self) -> Tuple[np.ndarray, np.ndarray, int]:
        """(segment of every filament, conductor of every segment, conductor
        count), as MeshSystem.layout."""
        c = self.counts()
        n, nseg = c["filaments"], c["segments"]
        sof = np.zeros(max(1, n), dtype=np.int64)
        cos = np.zeros(max(1, nseg), dtype=np.int64)
        nc = ctypes.c_int64()
        _check(N.load().fh_iterative_layout(self._h, sof.ctypes.data_as(N.c_int64_p),
                                            cos.ctypes.data_as(N.c_int64_p), ctypes.byref(nc)))
        return sof[:n], cos[:nseg], int(nc.value)

    def currents(self, frequency, excitation: Optional[Sequence[complex]] = None):
        """Filament currents for the port-current phasors ``excitation``
        (default: 1 A into port 1) at one frequency or a list of them
        (IterativeSystem::currents, iterative.rs:316-377): one GMRES solve
        per frequency, one CurrentSolution per frequency; the GMRES outcomes
        land in ``last_outcomes`` (one list of one outcome per frequency)."""
        nf = len(np.atleast_1d(frequency))
        oc = (N.GmresOutcome * max(1, nf))()
        out = _solve_currents(self, frequency, excitation,
                              lambda *a: N.load().fh_iterative_currents(self._h, *a[:-1], oc, a[-1]))
        self.last_outcomes = [[GmresOutcome(int(oc[k].iterations), float(oc[k].relative_residual),
                                            bool(oc[k].converged))] for k in range(nf)]
        return out


def gmres_dense(a: np.ndarray, b: np.ndarray, x0: Optional[np.ndarray] = None,
                precondition: Optional[np.ndarray] = None, params: Optional[GmresParams] = None):
    """The device GMRES on a dense complex system (test hook of the solver
    that IterativeSystem uses).  Returns (x, GmresOutcome)."""
    a = np.asfortranarray(a, dtype=np.complex128)
    n = a.shape[0]
    b = np.ascontiguousarray(b, dtype=np.complex128)
    x = np.ascontiguousarray(np.zeros(n, dtype=np.complex128) if x0 is None else x0, dtype=np.complex128)
    m = None if precondition is None else np.asfortranarray(precondition, dtype=np.complex128)
    g = (params or GmresParams())._native()
    oc = N.GmresOutcome()
    info = N.ErrorInfo()
    _check(N.load().fh_test_gmres_dense(a.ctypes.data_as(N.c_double_p), n, b.ctypes.data_as(N.c_double_p),
                                        x.ctypes.data_as(N.c_double_p),
                                        None if m is None else m.ctypes.data_as(N.c_double_p), ctypes.byref(g),
                                        ctypes.byref(oc), ctypes.byref(info)), info)
    return x, GmresOutcome(int(oc.iterations), float(oc.relative_residual), bool(oc.converged))


def skin_depth(frequency_hz: float, sigma: float) -> float:
    return 1.0 / np.sqrt(np.pi * frequency_hz * MU0 * sigma)


def device_count() -> int:
    return int(N.load().fh_device_count())


def build_info() -> str:
    return N.load().fh_build_info().decode()


def release_cached_memory() -> None:
    """Hands the device memory that finished systems left in the library's
    cache back to the driver (fh_release_cached_memory)."""
    _check(N.load().fh_release_cached_memory())


def fill_stats(system: "MeshSystem") -> Dict[str, float]:
    """Pairs per method and device time per fill kernel of an assembled system."""
    s = N.FillStats()
    _check(N.load().fh_system_fill_stats(system._h, ctypes.byref(s)))
    return {k: (int(getattr(s, k)) if t is ctypes.c_int64 else float(getattr(s, k))) for k, t in N.FillStats._fields_}


class Profiler:
    """Device-event profile of the extraction kernels (per kernel class:
    launches, milliseconds, algorithmic flops)."""

    def __enter__(self):
        L = N.load()
        L.fh_profile_reset()
        L.fh_profile_enable(1)
        return self

    def __exit__(self, *exc):
        N.load().fh_profile_enable(0)

    @staticmethod
    def read() -> Dict[str, Dict[str, float]]:
        L = N.load()
        out = {}
        for i, name in enumerate(N.PROFILE_CLASSES):
            launches, ms, work = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
            _check(L.fh_profile_read(i, ctypes.byref(launches), ctypes.byref(ms), ctypes.byref(work)))
            out[name] = {"launches": int(launches.value), "ms": float(ms.value), "work": float(work.value)}
        return out

    @staticmethod
    def overlap(a, b) -> Dict[str, float]:
        """Milliseconds during which a launch of the classes named in `a` ran,
        of those in `b`, and both at once (fh_profile_overlap): the
        factorization's look-ahead runs the diagonal regions ("panel",
        "trsm", "gemm_tc_inner") beside the deep update ("gemm_tc")."""
        idx = {name: i for i, name in enumerate(N.PROFILE_CLASSES)}
        ma = sum(1 << idx[n] for n in a)
        mb = sum(1 << idx[n] for n in b)
        x, y, both = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(N.load().fh_profile_overlap(ma, mb, ctypes.byref(x), ctypes.byref(y), ctypes.byref(both)))
        return {"a_ms": float(x.value), "b_ms": float(y.value), "both_ms": float(both.value)}
