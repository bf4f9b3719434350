"""Ground planes: a thick rectangular sheet meshed into bars that join the
centres of adjacent cells, with holes, graded contact regions and
equipotential patches (the reference's GroundPlane, fasterhenry/src/plane.rs;
the FastHenry ``G`` statement of the deck reader).

A plane is host-side geometry: it adds nodes and segments to a
:class:`~fasterhenry_b200.api.Geometry`, and the GPU path then treats its bars
like any other segments (fill, loop basis, sweep or the matrix-free path).

Cell layout (plane.rs:835-937, 610-785):

* ``nx x ny`` background cells over ``[lo, hi]``; each :class:`ContactRegion`
  adds, per axis, a band of uniform fine cells, and the cells outside a band
  grow geometrically by its ratio until they reach the background cell.
  Bands that overlap or lie closer than one fine cell merge (finest cell,
  gentlest ratio); a band that spans the whole axis at the background count
  is the background itself and is dropped.
* A node sits at every live cell centre, at mid-thickness; an x-directed bar
  joins horizontally adjacent centres with width ``dy_j``, a y-directed bar
  vertically adjacent ones with width ``dx_i``, both ``thickness`` high.
* :class:`Hole` shapes remove cells (and so their bars); an
  :class:`Equipotential` ties the live cells whose centres it covers into
  one node at their mean position, and the bars inside it are not built.

Coordinates are metres; x/y are plane coordinates (the plane is parallel to
the xy plane, top surface at ``z_top``).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

from . import api as A

MAX_AXIS_CELLS = 100_000  # plane.rs:479
EPS = 2.220446049250313e-16


class PlaneError(A.InvalidArgument):
    """A ground plane that cannot be meshed (PlaneError, plane.rs:417-476)."""


# ---------------------------------------------------------------------------
# Shapes
# ---------------------------------------------------------------------------
@dataclasses.dataclass(frozen=True)
class Hole:
    """A hole (plane.rs:214-281).  ``kind`` is "rect" (cells whose centre is
    strictly inside ``lo .. hi``), "point" (cells whose closed extent contains
    ``at``) or "circle" (cells whose centre is within ``radius`` of ``centre``,
    boundary included)."""
    kind: str
    lo: Tuple[float, float] = (0.0, 0.0)
    hi: Tuple[float, float] = (0.0, 0.0)
    at: Tuple[float, float] = (0.0, 0.0)
    centre: Tuple[float, float] = (0.0, 0.0)
    radius: float = 0.0

    @staticmethod
    def rect(lo, hi) -> "Hole":
        return Hole("rect", lo=(float(lo[0]), float(lo[1])), hi=(float(hi[0]), float(hi[1])))

    @staticmethod
    def point(at) -> "Hole":
        return Hole("point", at=(float(at[0]), float(at[1])))

    @staticmethod
    def circle(centre, radius: float) -> "Hole":
        return Hole("circle", centre=(float(centre[0]), float(centre[1])), radius=float(radius))

    def removes(self, c, bounds) -> bool:
        if self.kind == "rect":
            return self.lo[0] < c[0] < self.hi[0] and self.lo[1] < c[1] < self.hi[1]
        if self.kind == "point":
            (x0, y0), (x1, y1) = bounds
            return x0 <= self.at[0] <= x1 and y0 <= self.at[1] <= y1
        if self.kind == "circle":
            return math.hypot(c[0] - self.centre[0], c[1] - self.centre[1]) <= self.radius
        raise PlaneError("unknown hole shape %r" % self.kind)


@dataclasses.dataclass(frozen=True)
class ContactRegion:
    """A locally refined patch (plane.rs:282-335): ``cells`` uniform fine
    cells per axis inside ``lo .. hi``, growing outward by ``ratio`` per cell
    (per axis) back to the background cell."""
    lo: Tuple[float, float]
    hi: Tuple[float, float]
    cells: Tuple[int, int]
    ratio: Tuple[float, float]

    @staticmethod
    def new(lo, hi, cells, ratio: float) -> "ContactRegion":
        return ContactRegion((float(lo[0]), float(lo[1])), (float(hi[0]), float(hi[1])),
                             (int(cells[0]), int(cells[1])), (float(ratio), float(ratio)))

    @staticmethod
    def graded_per_axis(lo, hi, cells, ratio) -> "ContactRegion":
        return ContactRegion((float(lo[0]), float(lo[1])), (float(hi[0]), float(hi[1])),
                             (int(cells[0]), int(cells[1])), (float(ratio[0]), float(ratio[1])))

    @staticmethod
    def centred(centre, side: float, cells: int, ratio: float) -> "ContactRegion":
        half = side / 2.0
        return ContactRegion.new((centre[0] - half, centre[1] - half), (centre[0] + half, centre[1] + half),
                                 (cells, cells), ratio)


@dataclasses.dataclass(frozen=True)
class Equipotential:
    """A patch of plane tied to one node (plane.rs:350-378): every live cell
    whose centre lies in the closed rectangle ``lo .. hi``."""
    lo: Tuple[float, float]
    hi: Tuple[float, float]

    @staticmethod
    def centred(centre, widths) -> "Equipotential":
        return Equipotential((centre[0] - widths[0] / 2.0, centre[1] - widths[1] / 2.0),
                             (centre[0] + widths[0] / 2.0, centre[1] + widths[1] / 2.0))

    def ties(self, c) -> bool:
        return self.lo[0] <= c[0] <= self.hi[0] and self.lo[1] <= c[1] <= self.hi[1]


# ---------------------------------------------------------------------------
# Axis layout
# ---------------------------------------------------------------------------
def contact_slack(lo: float, hi: float) -> float:
    """Overlap below which a contact only touches the footprint on an axis
    (plane.rs:610-614): the larger of 1e-9 of the span and 32 ulps of the
    largest coordinate."""
    return max(1e-9 * abs(hi - lo), 32.0 * EPS * max(abs(lo), abs(hi)))


def cells_no_coarser_than(span: float, fine: float) -> int:
    """ceil(span / fine), at least 1, with a quotient within 1e-9 (relative)
    of an integer taken as that integer (plane.rs:626-638)."""
    q = span / fine
    if math.isnan(q):
        return 1
    if math.isinf(q):
        return MAX_AXIS_CELLS + 1  # refused by the per-axis limit
    # nearest integer, halves away from zero (q - floor(q) is exact)
    a = abs(q)
    r = math.floor(a)
    if a - r >= 0.5:
        r += 1
    r = math.copysign(r, q)
    cells = r if abs(q - r) <= 1e-9 * r else math.ceil(q)
    return max(int(cells), 1)


@dataclasses.dataclass
class _Band:
    start: float
    end: float
    cells: int
    ratio: float

    def fine(self) -> float:
        return (self.end - self.start) / self.cells


def _gap_edges(edges: List[float], start: float, stop: float, left, right, coarse: float) -> None:
    """Cells filling start .. stop (plane.rs:646-709): extents grow by the
    bordering bands' ratios from each refined side, capped at the background
    cell; the fewest cells that cover the gap, scaled to fill it."""
    gap = stop - start
    if gap <= 0.0:
        return

    def target(side, k):
        if side is None:
            return math.inf
        fine, ratio = side
        return min(fine * ratio ** (k + 1), coarse)

    def extents(count):
        out = []
        for i in range(count):
            e = min(target(left, i), target(right, count - 1 - i))
            out.append(e if math.isfinite(e) else coarse)
        return out

    def covered(count):
        s = 0.0
        for e in extents(count):
            s += e
        return s

    hi_count = 1
    while covered(hi_count) < gap:
        if hi_count > MAX_AXIS_CELLS:
            raise PlaneError("graded plane mesh needs more than %d cells on one axis: coarsen the contacts"
                             % MAX_AXIS_CELLS)
        hi_count *= 2
    lo_count = 1
    while lo_count < hi_count:
        mid = lo_count + (hi_count - lo_count) // 2
        if covered(mid) >= gap:
            hi_count = mid
        else:
            lo_count = mid + 1
    ext = extents(hi_count)
    total = 0.0
    for e in ext:
        total += e
    cursor = start
    for e in ext:
        cursor += gap * e / total
        edges.append(cursor)
    edges[-1] = stop


def axis_edges(lo: float, hi: float, background: int, bands: Sequence[_Band]) -> List[float]:
    """Cell edges of one axis (plane.rs:711-800)."""
    coarse = (hi - lo) / background
    bands = [b for b in bands if not (b.start <= lo and b.end >= hi and b.cells == background)]
    if not bands:
        return [lo + i * coarse for i in range(background)] + [hi]
    bands = sorted(bands, key=lambda b: b.start)
    merged: List[_Band] = []
    for b in bands:
        if merged and b.start <= merged[-1].end + min(merged[-1].fine(), b.fine()):
            last = merged[-1]
            fine = min(last.fine(), b.fine())
            last.end = max(last.end, b.end)
            last.ratio = min(last.ratio, b.ratio)
            last.cells = cells_no_coarser_than(last.end - last.start, fine)
        else:
            merged.append(_Band(b.start, b.end, b.cells, b.ratio))
    if sum(b.cells for b in merged) > MAX_AXIS_CELLS:
        raise PlaneError("graded plane mesh needs more than %d cells on one axis: coarsen the contacts"
                         % MAX_AXIS_CELLS)
    edges = [lo]
    cursor = lo
    for k, b in enumerate(merged):
        prev = merged[k - 1] if k else None
        _gap_edges(edges, cursor, b.start, None if prev is None else (prev.fine(), prev.ratio),
                   (b.fine(), b.ratio), coarse)
        fine = b.fine()
        for c in range(1, b.cells + 1):
            edges.append(b.start + c * fine)
        edges[-1] = b.end
        cursor = b.end
        if len(edges) > MAX_AXIS_CELLS:
            raise PlaneError("graded plane mesh needs more than %d cells on one axis: coarsen the contacts"
                             % MAX_AXIS_CELLS)
    last = merged[-1]
    _gap_edges(edges, cursor, hi, (last.fine(), last.ratio), None, coarse)
    if len(edges) - 1 > MAX_AXIS_CELLS:
        raise PlaneError("graded plane mesh needs more than %d cells on one axis: coarsen the contacts"
                         % MAX_AXIS_CELLS)
    return edges


# ---------------------------------------------------------------------------
# The mesh and the plane
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class PlaneMesh:
    """Cell edges per axis and the nodes' depth (plane.rs:503-600)."""
    x: List[float]
    y: List[float]
    z: float

    def nx(self) -> int:
        return len(self.x) - 1

    def ny(self) -> int:
        return len(self.y) - 1

    def dx(self, i: int) -> float:
        return self.x[i + 1] - self.x[i]

    def dy(self, j: int) -> float:
        return self.y[j + 1] - self.y[j]

    def centre(self, i: int, j: int) -> Tuple[float, float, float]:
        return ((self.x[i] + self.x[i + 1]) / 2.0, (self.y[j] + self.y[j + 1]) / 2.0, self.z)

    def cell_bounds(self, i: int, j: int):
        return (self.x[i], self.y[j]), (self.x[i + 1], self.y[j + 1])

    def bars(self) -> int:
        return 2 * self.nx() * self.ny() - self.nx() - self.ny()


def _find(parent: List[int], k: int) -> int:
    while parent[k] != k:
        parent[k] = parent[parent[k]]
        k = parent[k]
    return k


@dataclasses.dataclass
class GroundPlane:
    """A ground plane (plane.rs:386-415): footprint ``lo .. hi`` (x, y), top
    surface ``z_top``, ``thickness`` downward, ``nx x ny`` background cells,
    conductivity ``sigma``, and its holes, contact regions and
    equipotential patches."""
    lo: Tuple[float, float]
    hi: Tuple[float, float]
    z_top: float
    thickness: float
    nx: int
    ny: int
    sigma: float
    holes: List[Hole] = dataclasses.field(default_factory=list)
    contacts: List[ContactRegion] = dataclasses.field(default_factory=list)
    equipotentials: List[Equipotential] = dataclasses.field(default_factory=list)

    def mesh(self) -> PlaneMesh:
        """The cell layout (plane.rs:850-937); independent of the holes."""
        if self.nx < 1 or self.ny < 1:
            raise PlaneError("ground plane needs nx, ny >= 1 (got %d, %d)" % (self.nx, self.ny))
        if not (self.hi[0] > self.lo[0] and self.hi[1] > self.lo[1]):
            raise PlaneError("ground plane extent is degenerate (lo %r, hi %r)" % (list(self.lo), list(self.hi)))
        bands: List[List[_Band]] = [[], []]
        for c in self.contacts:
            for r in c.ratio:
                if not (math.isfinite(r) and r >= 1.0):
                    raise PlaneError("contact decay ratio must be finite and >= 1 (got %r)" % r)
            if c.cells[0] < 1 or c.cells[1] < 1:
                raise PlaneError("contact region needs cells >= 1 on both axes (got %r)" % list(c.cells))
            if not (c.hi[0] > c.lo[0] and c.hi[1] > c.lo[1]):
                raise PlaneError("contact region extent is degenerate (lo %r, hi %r)" % (list(c.lo), list(c.hi)))
            for a in range(2):
                fine = (c.hi[a] - c.lo[a]) / c.cells[a]
                start = max(c.lo[a], self.lo[a])
                end = min(c.hi[a], self.hi[a])
                if end - start <= contact_slack(self.lo[a], self.hi[a]):
                    raise PlaneError("contact region (lo %r, hi %r) lies outside the plane footprint"
                                     % (list(c.lo), list(c.hi)))
                if start - self.lo[a] < fine:
                    start = self.lo[a]
                if self.hi[a] - end < fine:
                    end = self.hi[a]
                bands[a].append(_Band(start, end, cells_no_coarser_than(end - start, fine), c.ratio[a]))
        return PlaneMesh(axis_edges(self.lo[0], self.hi[0], self.nx, bands[0]),
                         axis_edges(self.lo[1], self.hi[1], self.ny, bands[1]),
                         self.z_top - self.thickness / 2.0)

    def _holed(self, c, bounds) -> bool:
        return any(h.removes(c, bounds) for h in self.holes)

    def _ties(self, mesh: PlaneMesh):
        """Equipotential class of every live cell and each class's node
        position (plane.rs:944-1003)."""
        nx, ny = mesh.nx(), mesh.ny()
        root = list(range(len(self.equipotentials)))
        cell = [[None] * ny for _ in range(nx)]
        if not self.equipotentials:
            return root, cell, []
        for i in range(nx):
            for j in range(ny):
                c = mesh.centre(i, j)
                if self._holed(c, mesh.cell_bounds(i, j)):
                    continue
                for k, region in enumerate(self.equipotentials):
                    if not region.ties(c):
                        continue
                    k = _find(root, k)
                    if cell[i][j] is None:
                        cell[i][j] = k
                    else:
                        first = _find(root, cell[i][j])
                        root[k] = first
                        cell[i][j] = first
        total = [[0.0, 0.0, 0.0] for _ in self.equipotentials]
        tied = [0] * len(self.equipotentials)
        for i in range(nx):
            for j in range(ny):
                if cell[i][j] is None:
                    continue
                k = _find(root, cell[i][j])
                cell[i][j] = k
                c = mesh.centre(i, j)
                for a in range(3):
                    total[k][a] += c[a]
                tied[k] += 1
        node_at = [tuple(t / n for t in s) if n else None for s, n in zip(total, tied)]
        return root, cell, node_at

    def build_into(self, geometry: "A.Geometry", max_width=(None, None)) -> List[List[Optional[int]]]:
        """Adds the plane's nodes and bars to ``geometry`` (plane.rs:1055-1155)
        and returns the node of every cell, ``[i][j]`` (None where a hole
        removed it).  ``max_width`` optionally caps the widths of the x- and
        y-directed bars (the narrowed-bar form)."""
        def cap(axis, width):
            return width if max_width[axis] is None else min(max_width[axis], width)

        mesh = self.mesh()
        nx, ny = mesh.nx(), mesh.ny()
        _, tie_of, node_at = self._ties(mesh)
        tie_node: List[Optional[int]] = [None] * len(self.equipotentials)
        centres: List[List[Optional[int]]] = [[None] * ny for _ in range(nx)]
        for i in range(nx):
            for j in range(ny):
                c = mesh.centre(i, j)
                if self._holed(c, mesh.cell_bounds(i, j)):
                    continue
                k = tie_of[i][j]
                if k is None:
                    centres[i][j] = geometry.add_node(A.Node(*c))
                elif tie_node[k] is None:
                    tie_node[k] = geometry.add_node(A.Node(*node_at[k]))
                    centres[i][j] = tie_node[k]
                else:
                    centres[i][j] = tie_node[k]
        for i in range(nx):
            for j in range(ny):
                here = centres[i][j]
                if here is None:
                    continue
                if i + 1 < nx:
                    right = centres[i + 1][j]
                    if right is not None and right != here:
                        geometry.add_segment(A.SegmentDef(here, right, cap(0, mesh.dy(j)), self.thickness,
                                                          self.sigma))
                if j + 1 < ny:
                    up = centres[i][j + 1]
                    if up is not None and up != here:
                        geometry.add_segment(A.SegmentDef(here, up, cap(1, mesh.dx(i)), self.thickness,
                                                          self.sigma))
        return centres

    def equipotential_node(self, centres, index: int) -> Optional[int]:
        """The node that equipotential ``index`` ties its cells to, None if it
        ties no live cell (plane.rs:1020-1046)."""
        if not 0 <= index < len(self.equipotentials):
            raise IndexError("equipotential %d is not one of this plane's %d" % (index, len(self.equipotentials)))
        root, cell, _ = self._ties(self.mesh())
        r = _find(root, index)
        for i, column in enumerate(cell):
            for j, k in enumerate(column):
                if k == r:
                    return centres[i][j]
        return None

    def contains(self, point, tolerance: float) -> bool:
        """Inside the footprint and depth, with ``tolerance`` of slack
        (plane.rs:1178-1187)."""
        bottom = self.z_top - self.thickness
        return (self.lo[0] - tolerance <= point[0] <= self.hi[0] + tolerance
                and self.lo[1] - tolerance <= point[1] <= self.hi[1] + tolerance
                and bottom - tolerance <= point[2] <= self.z_top + tolerance)

    def attach(self, centres, point) -> int:
        """The live cell-centre node nearest to ``point`` in xy, first in
        (i, j) order on a tie (plane.rs:1197-1222)."""
        mesh = self.mesh()
        best = None
        for i, column in enumerate(centres):
            for j, node in enumerate(column):
                if node is None:
                    continue
                c = mesh.centre(i, j)
                d = math.hypot(c[0] - point[0], c[1] - point[1])
                if best is None or d < best[0]:
                    best = (d, node)
        if best is None:
            raise PlaneError("ground plane extent is degenerate (lo %r, hi %r)" % (list(self.lo), list(self.hi)))
        return best[1]
