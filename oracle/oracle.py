"""ctypes binding of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's dense extraction path on the CPU (see
fh_oracle.cpp for the file:line each routine follows).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline/reference legs import
this module, and only as the checker or the timed CPU baseline; the product
(fasterhenry_b200) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

ORTHOGONAL, BAR_CLOSED_FORM, ALIGNED_QUADRATURE, POINT_QUADRATURE, SAMPLED_FILAMENTS = range(5)
METHOD_NAMES = ["Orthogonal", "BarClosedForm", "AlignedQuadrature", "PointQuadrature",
                "SampledFilaments"]


class Segment(ctypes.Structure):
    _fields_ = [("a", ctypes.c_longlong), ("b", ctypes.c_longlong), ("width", ctypes.c_double),
                ("height", ctypes.c_double), ("sigma", ctypes.c_double),
                ("has_width_dir", ctypes.c_longlong), ("width_dir", ctypes.c_double * 3)]


class AxisGrading(ctypes.Structure):
    _fields_ = [("nw", ctypes.c_longlong), ("nh", ctypes.c_longlong),
                ("width_ratio", ctypes.c_double), ("height_ratio", ctypes.c_double)]


class Discretization(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_longlong), ("nw", ctypes.c_longlong), ("nh", ctypes.c_longlong),
                ("ratio", ctypes.c_double), ("frequency_hz", ctypes.c_double),
                ("target_skin_depths", ctypes.c_double), ("max_per_axis", ctypes.c_longlong),
                ("per_segment", ctypes.POINTER(AxisGrading)), ("per_segment_len", ctypes.c_longlong)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        lp = ctypes.POINTER(ctypes.c_longlong)
        L.orc_gauss_rule.argtypes = [ctypes.c_int, dp, dp]
        L.orc_order_for.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.orc_order_for.restype = ctypes.c_int
        L.orc_discretize.argtypes = [dp, ctypes.c_longlong, ctypes.POINTER(Segment), ctypes.c_longlong,
                                     ctypes.POINTER(Discretization), dp, ctypes.c_longlong, lp, lp]
        L.orc_mesh.argtypes = [ctypes.POINTER(Segment), ctypes.c_longlong, ctypes.c_longlong, lp, lp,
                               ctypes.c_longlong, lp, lp, dp, ctypes.c_longlong, ctypes.c_longlong,
                               lp, lp, lp]
        L.orc_mutual.argtypes = [dp, dp, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.orc_self_inductance.argtypes = [dp]
        L.orc_self_inductance.restype = ctypes.c_double
        L.orc_bar_integral.argtypes = [dp, dp, dp, dp, dp]
        L.orc_aligned_quadrature.argtypes = [dp, dp, dp, dp]
        L.orc_aligned_quadrature.restype = ctypes.c_double
        L.orc_lines_parallel.argtypes = [ctypes.c_double] * 4 + [ctypes.POINTER(ctypes.c_int)]
        L.orc_lines_parallel.restype = ctypes.c_double
        L.orc_lines_skew.argtypes = [dp, dp, dp, dp, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
        L.orc_lines_skew.restype = ctypes.c_double
        L.orc_separation.argtypes = [dp, dp]
        L.orc_separation.restype = ctypes.c_double
        L.orc_fill.argtypes = [dp, ctypes.c_longlong, dp, ctypes.POINTER(ctypes.c_byte), ctypes.c_int, lp, lp]
        L.orc_lu_solve.argtypes = [dp, ctypes.c_longlong, dp, ctypes.c_longlong, ctypes.c_int]
        L.orc_lu_solve_plain.argtypes = [dp, ctypes.c_longlong, dp, ctypes.c_longlong]
        L.orc_near_pairs.argtypes = [dp, ctypes.c_longlong, ctypes.c_double, lp, lp, ctypes.c_longlong, lp]
        L.orc_fill_frozen.argtypes = [dp, dp, ctypes.c_longlong, dp, ctypes.c_int]
        L.orc_fill_frozen_rows.argtypes = [dp, dp, ctypes.c_longlong, lp, ctypes.c_longlong, dp, ctypes.c_int]
        L.orc_system_assemble.argtypes = [dp, ctypes.c_longlong, ctypes.POINTER(Segment), ctypes.c_longlong,
                                          lp, ctypes.c_longlong, ctypes.POINTER(Discretization),
                                          ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), dp]
        L.orc_system_counts.argtypes = [ctypes.c_void_p, lp]
        L.orc_system_blocks.argtypes = [ctypes.c_void_p, dp, dp]
        L.orc_system_filaments.argtypes = [ctypes.c_void_p, dp]
        L.orc_system_inductance.argtypes = [ctypes.c_void_p, dp]
        L.orc_system_impedance.argtypes = [ctypes.c_void_p, ctypes.c_double, dp, ctypes.c_int]
        L.orc_system_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _lp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))


def default_threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


class OracleError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__("oracle %s failed with status %d" % (what, status))
        self.status = status


def _check(status: int, what: str) -> None:
    if status:
        raise OracleError(status, what)


# ---------------------------------------------------------------------------
# Deck marshalling
# ---------------------------------------------------------------------------
_KINDS = {"uniform": 0, "per_segment": 1, "graded": 2, "skin_depth": 3, "per_segment_graded": 4}


def _marshal(deck):
    nodes = np.ascontiguousarray(np.array(deck.nodes, dtype=np.float64).reshape(-1, 3))
    segs = (Segment * max(1, len(deck.segments)))()
    for i, s in enumerate(deck.segments):
        segs[i].a, segs[i].b = s["a"], s["b"]
        segs[i].width, segs[i].height, segs[i].sigma = s["width"], s["height"], s["sigma"]
        wd = s.get("width_dir")
        segs[i].has_width_dir = 0 if wd is None else 1
        if wd is not None:
            segs[i].width_dir[0], segs[i].width_dir[1], segs[i].width_dir[2] = wd
    d = deck.discretization
    disc = Discretization()
    disc.kind = _KINDS[d["kind"]]
    disc.nw, disc.nh = d.get("nw", 0), d.get("nh", 0)
    disc.ratio = d.get("ratio", 1.0)
    disc.frequency_hz = d.get("frequency_hz", 0.0)
    disc.target_skin_depths = d.get("target_skin_depths", 0.0)
    disc.max_per_axis = d.get("max_per_axis", 32)
    grids = d.get("grids", [])
    arr = (AxisGrading * max(1, len(grids)))()
    for i, g in enumerate(grids):
        arr[i].nw, arr[i].nh = g[0], g[1]
        arr[i].width_ratio = g[2] if len(g) > 2 else 1.0
        arr[i].height_ratio = g[3] if len(g) > 3 else 1.0
    disc.per_segment = ctypes.cast(arr, ctypes.POINTER(AxisGrading))
    disc.per_segment_len = len(grids)
    ports = np.ascontiguousarray(np.array(deck.ports, dtype=np.int64).reshape(-1, 2))
    return nodes, segs, disc, arr, ports


def discretize(deck) -> Tuple[np.ndarray, np.ndarray]:
    L = lib()
    nodes, segs, disc, keep, _ = _marshal(deck)
    cap = 1
    out = np.zeros((cap, 19))
    nfil = ctypes.c_longlong(0)
    per = np.zeros(max(1, len(deck.segments)), dtype=np.int64)
    st = L.orc_discretize(_dp(nodes), len(nodes), segs, len(deck.segments), ctypes.byref(disc), _dp(out), cap,
                          ctypes.byref(nfil), _lp(per))
    if st and nfil.value > cap:
        out = np.zeros((nfil.value, 19))
        st = L.orc_discretize(_dp(nodes), len(nodes), segs, len(deck.segments), ctypes.byref(disc), _dp(out),
                              nfil.value, ctypes.byref(nfil), _lp(per))
    _check(st, "discretize")
    return out[: nfil.value].copy(), per[: len(deck.segments)].copy()


def mesh(deck, per_segment: np.ndarray):
    """Loop basis as (row_ptr, cols, signs, internal)."""
    L = lib()
    nodes, segs, disc, keep, ports = _marshal(deck)
    per = np.ascontiguousarray(per_segment, dtype=np.int64)
    cap_rows, cap_nnz = int(per.sum()) + len(deck.ports) + len(deck.segments) + 2, 4 * int(per.sum()) + 8 * (len(deck.segments) + 8) * (len(deck.ports) + len(deck.segments) + 1)
    row_ptr = np.zeros(cap_rows, dtype=np.int64)
    cols = np.zeros(cap_nnz, dtype=np.int64)
    signs = np.zeros(cap_nnz)
    nrows, nnz, internal = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    st = L.orc_mesh(segs, len(deck.segments), len(nodes), _lp(per), _lp(ports), len(deck.ports), _lp(row_ptr),
                    _lp(cols), _dp(signs), cap_rows, cap_nnz, ctypes.byref(nrows), ctypes.byref(nnz),
                    ctypes.byref(internal))
    _check(st, "mesh")
    return row_ptr[: nrows.value + 1].copy(), cols[: nnz.value].copy(), signs[: nnz.value].copy(), internal.value


def mutual(fa: np.ndarray, fb: np.ndarray) -> Tuple[float, int, bool]:
    L = lib()
    fa = np.ascontiguousarray(fa, dtype=np.float64)
    fb = np.ascontiguousarray(fb, dtype=np.float64)
    v, m, r = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    _check(L.orc_mutual(_dp(fa), _dp(fb), ctypes.byref(v), ctypes.byref(m), ctypes.byref(r)), "mutual")
    return v.value, m.value, bool(r.value)


def self_inductance(f: np.ndarray) -> float:
    f = np.ascontiguousarray(f, dtype=np.float64)
    return lib().orc_self_inductance(_dp(f))


def bar_integral(qx, qy, qz) -> Tuple[float, float]:
    a = [np.ascontiguousarray(q, dtype=np.float64) for q in (qx, qy, qz)]
    v, r = ctypes.c_double(), ctypes.c_double()
    lib().orc_bar_integral(_dp(a[0]), _dp(a[1]), _dp(a[2]), ctypes.byref(v), ctypes.byref(r))
    return v.value, r.value


def aligned_quadrature(length, width, height, offset) -> float:
    a = [np.ascontiguousarray(q, dtype=np.float64) for q in (length, width, height, offset)]
    return lib().orc_aligned_quadrature(_dp(a[0]), _dp(a[1]), _dp(a[2]), _dp(a[3]))


def lines_parallel(l1, l2, offset, rho) -> Optional[float]:
    ok = ctypes.c_int()
    v = lib().orc_lines_parallel(l1, l2, offset, rho, ctypes.byref(ok))
    return v if ok.value else None


def lines_skew(a0, a1, b0, b1, sin_min=0.0) -> Optional[float]:
    a = [np.ascontiguousarray(q, dtype=np.float64) for q in (a0, a1, b0, b1)]
    ok = ctypes.c_int()
    v = lib().orc_lines_skew(_dp(a[0]), _dp(a[1]), _dp(a[2]), _dp(a[3]), sin_min, ctypes.byref(ok))
    return v if ok.value else None


def gauss_rule(n: int) -> Tuple[np.ndarray, np.ndarray]:
    x, w = np.zeros(n), np.zeros(n)
    lib().orc_gauss_rule(n, _dp(x), _dp(w))
    return x, w


def order_for(tolerance: float, max_order: int, half: float, distance: float) -> Optional[int]:
    r = lib().orc_order_for(tolerance, max_order, half, distance)
    return r if r else None


def fill(filaments: np.ndarray, threads: Optional[int] = None, methods: bool = False):
    filaments = np.ascontiguousarray(filaments, dtype=np.float64)
    n = len(filaments)
    Lm = np.zeros((n, n), order="F")
    meth = np.zeros((n, n), dtype=np.int8, order="F") if methods else None
    ei, ej = ctypes.c_longlong(), ctypes.c_longlong()
    mp = meth.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)) if methods else None
    st = lib().orc_fill(_dp(filaments), n, Lm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), mp,
                        threads or default_threads(), ctypes.byref(ei), ctypes.byref(ej))
    _check(st, "fill")
    return (Lm, meth) if methods else Lm


def fill_frozen(nominal: np.ndarray, perturbed: np.ndarray, threads: Optional[int] = None) -> np.ndarray:
    """L of ``perturbed`` with every dispatch decision taken on ``nominal``
    (the evaluation that finite differences of the gradient differentiate)."""
    a = np.ascontiguousarray(nominal, dtype=np.float64)
    b = np.ascontiguousarray(perturbed, dtype=np.float64)
    assert a.shape == b.shape
    n = len(a)
    Lm = np.zeros((n, n), order="F")
    _check(lib().orc_fill_frozen(_dp(a), _dp(b), n, Lm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 threads or default_threads()), "fill_frozen")
    return Lm


def fill_frozen_rows(nominal: np.ndarray, perturbed: np.ndarray, rows: Sequence[int],
                     threads: Optional[int] = None) -> np.ndarray:
    """Rows of fill_frozen: out[r, j] = L(rows[r], j)."""
    a = np.ascontiguousarray(nominal, dtype=np.float64)
    b = np.ascontiguousarray(perturbed, dtype=np.float64)
    r = np.ascontiguousarray(rows, dtype=np.int64)
    n = len(a)
    out = np.zeros((len(r), n))
    _check(lib().orc_fill_frozen_rows(_dp(a), _dp(b), n, _lp(r), len(r), _dp(out), threads or default_threads()),
           "fill_frozen_rows")
    return out


def lu_solve(a: np.ndarray, b: np.ndarray, threads: Optional[int] = None, plain: bool = False) -> np.ndarray:
    """Solve a x = b with the reference's blocked partial-pivoting LU (complex).

    ``plain=True`` runs the reference's column-at-a-time sweeps (dense.rs:98-190)
    on one thread; the default runs the same per-entry operations in cache
    blocks on all threads, and both give the same bits."""
    a = np.array(a, dtype=np.complex128, order="F", copy=True)
    b2 = np.array(b, dtype=np.complex128, order="F", copy=True)
    if b2.ndim == 1:
        b2 = b2.reshape(-1, 1, order="F")
    n = a.shape[0]
    if plain:
        st = lib().orc_lu_solve_plain(_dp(a), n, _dp(b2), b2.shape[1])
    else:
        st = lib().orc_lu_solve(_dp(a), n, _dp(b2), b2.shape[1], threads or default_threads())
    _check(st, "lu_solve")
    return b2.reshape(b.shape) if np.ndim(b) == 1 else b2


def near_pairs(filaments: np.ndarray, radius: float):
    """pfft/near.rs:41-106: for each filament i, the j >= i (i included) whose
    separating-axis gap is below `radius`, ascending.  Returns (off, cols) as
    CSR arrays."""
    f = np.ascontiguousarray(filaments, dtype=np.float64)
    n = len(f)
    off = np.zeros(n + 1, dtype=np.int64)
    total = ctypes.c_longlong(0)
    cap = max(16 * n, 1)
    for _ in range(2):
        cols = np.zeros(cap, dtype=np.int64)
        _check(lib().orc_near_pairs(_dp(f), n, float(radius), _lp(off), _lp(cols), cap, ctypes.byref(total)),
               "near_pairs")
        if total.value <= cap:
            return off, cols[:total.value]
        cap = total.value
    raise RuntimeError("near_pairs: capacity")


class System:
    """The oracle's MeshSystem: assemble once, then impedance(f) per frequency."""

    def __init__(self, deck, threads: Optional[int] = None):
        L = lib()
        self.threads = threads or default_threads()
        nodes, segs, disc, keep, ports = _marshal(deck)
        h = ctypes.c_void_p()
        t = np.zeros(3)
        st = L.orc_system_assemble(_dp(nodes), len(nodes), segs, len(deck.segments), _lp(ports), len(deck.ports),
                                   ctypes.byref(disc), self.threads, ctypes.byref(h), _dp(t))
        _check(st, "assemble")
        self._h = h
        self.inductance_s, self.assembly_s = float(t[0]), float(t[1])
        c = np.zeros(6, dtype=np.int64)
        L.orc_system_counts(h, _lp(c))
        self.counts = dict(zip(["nodes", "segments", "filaments", "meshes", "internal_meshes", "ports"],
                               [int(x) for x in c]))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_system_free(self._h)
            self._h = None

    def blocks(self) -> Tuple[np.ndarray, np.ndarray]:
        loops = self.counts["meshes"]
        r = np.zeros((loops, loops), order="F")
        l = np.zeros((loops, loops), order="F")
        lib().orc_system_blocks(self._h, r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                l.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return r, l

    def filaments(self) -> np.ndarray:
        f = np.zeros((self.counts["filaments"], 19))
        lib().orc_system_filaments(self._h, _dp(f))
        return f

    def inductance(self) -> np.ndarray:
        n = self.counts["filaments"]
        Lm = np.zeros((n, n), order="F")
        lib().orc_system_inductance(self._h, Lm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return Lm

    def impedance(self, frequency: float) -> np.ndarray:
        p = self.counts["ports"]
        z = np.zeros((p, p), dtype=np.complex128)
        _check(lib().orc_system_impedance(self._h, frequency, z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          self.threads), "impedance")
        return z

    def sweep(self, frequencies: Sequence[float]) -> np.ndarray:
        return np.stack([self.impedance(f) for f in frequencies])


def currents(deck, frequency: float, excitation, threads: Optional[int] = None) -> dict:
    """Filament currents, densities, powers, segment sums, conductor peaks and
    the power balance at one frequency (MeshSystem::currents, solve.rs:
    1110-1149, with currents.rs:128-274), restated with numpy on the
    oracle's own matrices and LU."""
    system = System(deck, threads)
    R, L = system.blocks()
    fil = system.filaments()
    m, p = system.counts["internal_meshes"], system.counts["ports"]
    w = 2 * np.pi * frequency
    Z = R + 1j * w * L
    ee, ep, pp = Z[:m, :m], Z[:m, m:], Z[m:, m:]
    current = np.asarray(excitation, dtype=np.complex128)
    internal = -lu_solve(ee, ep @ current) if m else np.zeros(0, dtype=np.complex128)
    voltage = pp @ current + ep.T @ internal
    fil_all, per = discretize(deck)
    row_ptr, cols, signs, _ = mesh(deck, per)
    branch = np.zeros(len(fil), dtype=np.complex128)
    loops = np.concatenate([internal, current])
    for i, x in enumerate(loops):  # currents.rs:183-190: row by row
        for k in range(row_ptr[i], row_ptr[i + 1]):
            branch[cols[k]] += x * signs[k]
    # Layout, currents.rs:137-170.
    nodes = len(deck.nodes)
    parent = list(range(nodes))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x
    for sd in deck.segments:
        a, b = find(sd["a"]), find(sd["b"])
        if a != b:
            parent[a] = b
    roots, cond_of_seg = [], []
    for sd in deck.segments:
        r = find(sd["a"])
        if r not in roots:
            roots.append(r)
        cond_of_seg.append(roots.index(r))
    seg_of_fil = np.repeat(np.arange(len(per)), per)
    res = fil[:, 6] / (fil[:, 18] * (fil[:, 16] * fil[:, 17]))
    density = np.abs(branch) / (fil[:, 16] * fil[:, 17])
    power = 0.5 * (branch.real ** 2 + branch.imag ** 2) * res
    seg_cur = np.zeros(len(per), dtype=np.complex128)
    seg_pow = np.zeros(len(per))
    peaks = [None] * len(roots)
    dissipated = 0.0
    for k in range(len(fil)):
        s = seg_of_fil[k]
        dissipated += power[k]
        seg_cur[s] += branch[k]
        seg_pow[s] += power[k]
        c = cond_of_seg[s]
        if peaks[c] is None or density[k] > peaks[c][0]:
            peaks[c] = (density[k], k)
    inp = 0.5 * float(np.sum((np.conj(current) * voltage).real))
    scale = max(dissipated, inp)
    return {"current": branch, "density": density, "power": power, "segment_current": seg_cur,
            "segment_power": seg_pow, "peak_filament": np.array([pk[1] for pk in peaks]),
            "peak_density": np.array([pk[0] for pk in peaks]), "conductor_of_segment": np.array(cond_of_seg),
            "balance": {"dissipated_w": dissipated, "input_w": inp,
                        "relative_residual": abs(dissipated - inp) / scale if scale > 0 else 0.0}}
