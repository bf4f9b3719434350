"""Synthetic decks for the extraction path: square spirals and meanders.

The builders return a :class:`Deck` — nodes, segment definitions, ports and a
discretization — in the same form the reference's ``Geometry`` /
``SegmentDef`` / ``Port`` / ``Discretization`` take (fasterhenry/src/
geometry.rs:338-467, mesh.rs:67-92, solve.rs:409-510).  All lengths in metres.

* :func:`square_spiral` lays segments head to tail in the winding order of
  the reference's test fixture (fasterhenry/tests/common/mod.rs:116-134):
  directions +x, +y, -x, -y, the side growing by one pitch after every second
  segment.
* :func:`meander` is a chain of parallel legs along +-x joined by short
  connectors along +y, the last connector being the lead-out
  (fasterhenry/benches/support.rs:64-83 builds the same shape).
* :func:`random_spirals` draws the batched uneven-geometry set from a
  SplitMix64 stream (the generator of fasterhenry/src/dense.rs:197-208).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

COPPER = 5.8e7
UM = 1e-6


@dataclasses.dataclass
class Deck:
    """A geometry plus its ports and discretization."""

    nodes: List[Tuple[float, float, float]]
    segments: List[dict]
    ports: List[Tuple[int, int]]
    discretization: dict
    name: str = ""

    def segment_count(self) -> int:
        return len(self.segments)


def segment(a: int, b: int, width: float, height: float, sigma: float = COPPER,
            width_dir: Optional[Sequence[float]] = None) -> dict:
    return {"a": a, "b": b, "width": width, "height": height, "sigma": sigma,
            "width_dir": None if width_dir is None else tuple(float(x) for x in width_dir)}


def uniform(nw: int, nh: int) -> dict:
    return {"kind": "uniform", "nw": nw, "nh": nh}


def per_segment(grids: Sequence[Tuple[int, int]]) -> dict:
    return {"kind": "per_segment", "grids": [(int(a), int(b)) for a, b in grids]}


def graded(nw: int, nh: int, ratio: float) -> dict:
    return {"kind": "graded", "nw": nw, "nh": nh, "ratio": ratio}


def skin_depth(frequency_hz: float, target_skin_depths: float, ratio: float,
               max_per_axis: int = 32) -> dict:
    return {"kind": "skin_depth", "frequency_hz": frequency_hz,
            "target_skin_depths": target_skin_depths, "ratio": ratio,
            "max_per_axis": max_per_axis}


def per_segment_graded(grids: Sequence[Tuple[int, int, float, float]]) -> dict:
    return {"kind": "per_segment_graded",
            "grids": [(int(a), int(b), float(c), float(d)) for a, b, c, d in grids]}


def spiral_lengths(turns: int, start_len: float, pitch: float) -> List[float]:
    out, length = [], start_len
    for k in range(4 * turns):
        out.append(length)
        if k % 2 == 1:
            length += pitch
    return out


def square_spiral(turns: int, width: float, spacing: float, thickness: float, outer: float,
                  discretization: dict, z: float = 0.0, sigma: float = COPPER,
                  name: str = "spiral") -> Deck:
    """``turns``-turn square spiral whose longest side is ``outer``.

    Pitch ``P = width + spacing``; the first side is ``outer - (2 turns - 1) P``
    so that the last pair of sides is ``outer`` long.
    """
    pitch = width + spacing
    start = outer - (2 * turns - 1) * pitch
    if start <= 0:
        raise ValueError("spiral closes on itself: first side would be %g" % start)
    directions = [(1.0, 0.0), (0.0, 1.0), (-1.0, 0.0), (0.0, -1.0)]
    x, y = 0.0, 0.0
    nodes = [(x, y, z)]
    segs = []
    for k, length in enumerate(spiral_lengths(turns, start, pitch)):
        dx, dy = directions[k % 4]
        x, y = x + dx * length, y + dy * length
        nodes.append((x, y, z))
        segs.append(segment(k, k + 1, width, thickness, sigma))
    return Deck(nodes, segs, [(0, len(segs))], discretization, name)


def meander(legs: int, leg_length: float, pitch: float, width: float, thickness: float,
            discretization: dict, sigma: float = COPPER, name: str = "meander") -> Deck:
    """``legs`` parallel legs along +-x, ``pitch`` apart, joined by ``pitch``-long
    connectors along +y; ``2 legs`` segments in one chain, port across the ends."""
    nodes = [(0.0, 0.0, 0.0)]
    segs = []
    for leg in range(legs):
        y = leg * pitch
        x_far = leg_length if leg % 2 == 0 else 0.0
        for (x, yy) in ((x_far, y), (x_far, y + pitch)):
            nodes.append((x, yy, 0.0))
            segs.append(segment(len(nodes) - 2, len(nodes) - 1, width, thickness, sigma))
    return Deck(nodes, segs, [(0, len(nodes) - 1)], discretization, name)


# ---------------------------------------------------------------------------
# The named workloads
# ---------------------------------------------------------------------------

def c1_spiral() -> Tuple[Deck, List[float]]:
    """4-turn square spiral, 10 um wide, 2 um thick, 5 um spacing, 300 um
    outer side, z = 0, 16 segments at 5 x 3 (240 filaments), 10 log-spaced
    frequencies 1e6..1e10 Hz."""
    deck = square_spiral(4, 10 * UM, 5 * UM, 2 * UM, 300 * UM, uniform(5, 3), name="c1_spiral")
    return deck, logspace(6, 10, 10)


def c2_meander() -> Tuple[Deck, List[float]]:
    """40 legs of 1 mm at 40 um pitch (80 segments), 20 um x 5 um copper, 10 x 3
    per segment (2,400 filaments), 32 log-spaced frequencies 1e5..1e10 Hz."""
    deck = meander(40, 1e-3, 40 * UM, 20 * UM, 5 * UM, uniform(10, 3), name="c2_meander")
    return deck, logspace(5, 10, 32)


def metric_meander() -> Tuple[Deck, List[float]]:
    """The meander above scaled to 167 legs (334 segments, 10,020 filaments,
    9,686 internal loops), 32 log-spaced frequencies 1e5..1e10 Hz."""
    deck = meander(167, 1e-3, 40 * UM, 20 * UM, 5 * UM, uniform(10, 3), name="meander_10k")
    return deck, logspace(5, 10, 32)


def metric_meander_odd() -> Tuple[Deck, List[float]]:
    """The metric meander with its sixth segment on a 29 x 1 grid instead of
    10 x 3: 10,019 filaments and an odd order, 9,685 internal loops; the same
    32 frequencies."""
    base, freqs = metric_meander()
    grids = [(10, 3)] * base.segment_count()
    grids[5] = (29, 1)
    deck = Deck(list(base.nodes), [dict(sg) for sg in base.segments], list(base.ports), per_segment(grids),
                "meander_10k_odd")
    return deck, freqs


def meander_legs(legs: int, nw: int = 10, nh: int = 3) -> Deck:
    return meander(legs, 1e-3, 40 * UM, 20 * UM, 5 * UM, uniform(nw, nh), name="meander_%d" % legs)


def c4_spiral(target_skin_depths: float = 0.1, ratio: float = 1.4, max_per_axis: int = 32) -> Deck:
    """6-turn spiral, 15 um wide, 5 um spacing, 3 um thick, 500 um outer side,
    skin-depth graded at 1 GHz.  The defaults (cells at most 0.1 skin depth,
    grading ratio 1.4) give 17 x 9 filaments per segment, 3,672 in all; its
    gradient parameters are the 24 widths and 24 thicknesses."""
    return square_spiral(6, 15 * UM, 5 * UM, 3 * UM, 500 * UM,
                         skin_depth(1e9, target_skin_depths, ratio, max_per_axis), name="c4_spiral")


ISLAND_SIDE = 10e-3
ISLAND_EXTENT = math.sqrt(2.0) * ISLAND_SIDE


def two_islands(separation: float) -> Tuple[Deck, List[str]]:
    """Two nearly closed square loops (side 10 mm, trace 0.4 mm x 35 um, the
    left side broken by a gap of side / 20 that holds the port), bounding
    boxes ``separation`` apart along x; uniform 2 x 1.  Returns the deck and
    the group tag of each segment ("a" x 4, "b" x 4).  The coupling fixture of
    fasterhenry/tests/coupling.rs:33-75."""
    nodes: List[Tuple[float, float, float]] = []
    segs, ports = [], []
    gap = ISLAND_SIDE / 20.0
    for x0 in (0.0, ISLAND_SIDE + separation):
        base = len(nodes)
        for (x, y) in ((0.0, 0.0), (ISLAND_SIDE, 0.0), (ISLAND_SIDE, ISLAND_SIDE), (0.0, ISLAND_SIDE), (0.0, gap)):
            nodes.append((x0 + x, y, 0.0))
        for k in range(4):
            segs.append(segment(base + k, base + k + 1, 0.4e-3, 35e-6))
        ports.append((base, base + 4))
    return Deck(nodes, segs, ports, uniform(2, 1), "two_islands"), ["a"] * 4 + ["b"] * 4


def with_segment(deck: Deck, index: int, **changes) -> Deck:
    """A copy of ``deck`` with segment ``index``'s fields replaced."""
    segs = [dict(s) for s in deck.segments]
    segs[index].update(changes)
    return Deck(list(deck.nodes), segs, list(deck.ports), dict(deck.discretization), deck.name)


def logspace(lo: float, hi: float, count: int) -> List[float]:
    if count == 1:
        return [10.0 ** lo]
    return [10.0 ** (lo + (hi - lo) * k / (count - 1)) for k in range(count)]


class SplitMix64:
    """SplitMix64 (Steele, Lea & Flood 2014), the stream of the reference's
    dense-LU tests (fasterhenry/src/dense.rs:197-208)."""

    def __init__(self, seed: int):
        self.state = seed & 0xFFFFFFFFFFFFFFFF

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        return z ^ (z >> 31)

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))

    def integer(self, lo: int, hi: int) -> int:
        return lo + self.next_u64() % (hi - lo + 1)


def random_spirals(count: int = 64, seed: int = 2026) -> List[Deck]:
    """Seeded uneven spirals: turns in {2..8}, width 5-20 um, spacing 3-10 um,
    thickness 1-4 um, outer side 150-600 um, nw in {3..10}, nh in {2, 3}.
    Draws whose first side would be shorter than two pitches are rejected
    (the spiral would close on itself)."""
    rng = SplitMix64(seed)
    decks = []
    while len(decks) < count:
        turns = rng.integer(2, 8)
        width = rng.uniform(5, 20) * UM
        spacing = rng.uniform(3, 10) * UM
        thickness = rng.uniform(1, 4) * UM
        outer = rng.uniform(150, 600) * UM
        nw = rng.integer(3, 10)
        nh = rng.integer(2, 3)
        pitch = width + spacing
        if outer - (2 * turns - 1) * pitch < 2 * pitch:
            continue
        decks.append(square_spiral(turns, width, spacing, thickness, outer, uniform(nw, nh),
                                   name="spiral_%d" % len(decks)))
    return decks


# ---------------------------------------------------------------------------
# Random filament clouds (the pFFT accuracy fixtures)
# ---------------------------------------------------------------------------

def cloud_side(n: int) -> float:
    """Side of the cube holding n filaments at 400 filaments per 1,000 mm^3."""
    return 10e-3 * (n / 400.0) ** (1.0 / 3.0)


def cloud_bars(n: int, side: float, manhattan: bool, seed: int):
    """n bars of length 0.5-1.5 mm in a cube of side `side`, axis-aligned
    (random axis and sense) or in general position, cross-sections
    0.1-0.3 x 0.05-0.15 mm; drawn from SplitMix64(seed)."""
    r = SplitMix64(seed)
    nodes, segs = [], []
    for _ in range(n):
        a = [side * r.uniform(0.0, 1.0) for _ in range(3)]
        length = 1e-3 * (0.5 + r.uniform(0.0, 1.0))
        if manhattan:
            d = [0.0, 0.0, 0.0]
            d[min(2, int(r.uniform(0.0, 1.0) * 3.0))] = -1.0 if r.uniform(0.0, 1.0) < 0.5 else 1.0
        else:
            v = [r.uniform(-0.5, 0.5) for _ in range(3)]
            norm = math.sqrt(sum(c * c for c in v))
            d = [c / norm for c in v]
        b = [a[k] + length * d[k] for k in range(3)]
        width = 0.1e-3 + 0.2e-3 * r.uniform(0.0, 1.0)
        height = 0.05e-3 + 0.1e-3 * r.uniform(0.0, 1.0)
        nodes += [tuple(a), tuple(b)]
        segs.append(segment(len(nodes) - 2, len(nodes) - 1, width, height))
    return nodes, segs


def cloud_deck(n: int, manhattan: bool, seed: int, side: Optional[float] = None) -> Deck:
    """The cloud as a deck of unconnected one-filament segments (no ports)."""
    nodes, segs = cloud_bars(n, cloud_side(n) if side is None else side, manhattan, seed)
    return Deck(nodes, segs, [], uniform(1, 1), "cloud_%d" % n)


def scaling_meander(bars: int, pitch: float = 100e-6, width: float = 20e-6, thickness: float = 10e-6,
                    nw: int = 2, nh: int = 2) -> Deck:
    """A square meander of `bars` runs along +-x, each cut into `bars`
    collinear segments one pitch long, joined by one-pitch jogs along +y
    (bars (bars + 1) segments; 4 bars (bars + 1) filaments at 2 x 2).  One
    port spans the chain.  bars = 157 gives 99,224 filaments, bars = 49
    gives 9,800."""
    nodes = [(0.0, 0.0, 0.0)]
    segs = []

    def add(x, y):
        nodes.append((x, y, 0.0))
        segs.append(segment(len(nodes) - 2, len(nodes) - 1, width, thickness))

    for bar in range(bars):
        y = bar * pitch
        for step in range(1, bars + 1):
            along = step if bar % 2 == 0 else bars - step
            add(along * pitch, y)
        add((bars if bar % 2 == 0 else 0) * pitch, y + pitch)
    return Deck(nodes, segs, [(0, len(nodes) - 1)], uniform(nw, nh), "scaling_meander_%d" % bars)


def meander_over_plane(bars: int, plane_side: float = 4e-3, cells: int = 64, gap: float = 50e-6,
                       plane_thickness: float = 10e-6, hole_side: float = 0.5e-3) -> Deck:
    """The square meander of `bars` runs (scaling_meander, 2 x 2 per segment)
    over a copper ground plane: a `plane_side` square centred under the
    meander, top surface `gap` below the meander's bottom face,
    `plane_thickness` thick, meshed `cells` x `cells` (one filament per bar)
    with one square hole of side `hole_side` at its centre.  The plane is not
    connected to the meander: it carries the induced (eddy) currents.
    bars = 157 with the defaults is the matrix-free large case (99,224
    meander filaments plus 8,060 plane bars); bars = 49 its dense-checkable
    subset."""
    from .api import Geometry, Node, SegmentDef
    from .plane import GroundPlane, Hole
    base = scaling_meander(bars)
    thickness = base.segments[0]["height"]
    centre = bars * 100e-6 / 2.0
    half = plane_side / 2.0
    g = Geometry()
    plane = GroundPlane((centre - half, centre - half), (centre + half, centre + half),
                        -thickness / 2.0 - gap, plane_thickness, cells, cells, COPPER,
                        holes=[Hole.rect((centre - hole_side / 2.0, centre - hole_side / 2.0),
                                         (centre + hole_side / 2.0, centre + hole_side / 2.0))])
    plane.build_into(g)
    offset = len(g.nodes)
    nodes = [(nd.x, nd.y, nd.z) for nd in g.nodes] + list(base.nodes)
    segs = [segment(sd.a, sd.b, sd.width, sd.height, sd.sigma) for sd in g.segments]
    nplane = len(segs)
    segs += [dict(sg, a=sg["a"] + offset, b=sg["b"] + offset) for sg in base.segments]
    ports = [(a + offset, b + offset) for a, b in base.ports]
    grids = [(1, 1)] * nplane + [(2, 2)] * len(base.segments)
    return Deck(nodes, segs, ports, per_segment(grids), "meander_%d_over_plane" % bars)

