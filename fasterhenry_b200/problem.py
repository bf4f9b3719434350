"""The problem document and the FastHenry `.inp` deck reader: the front end
that turns an input file into geometry, ports, discretization, coupling and
frequencies for the C ABI (fasterhenry-cli/src/problem.rs:1-50; the deck
dialect of fasterhenry-cli/src/inp.rs:1-600 and docs/input-format.md).

* :class:`Problem` is the JSON problem document: ``geometry`` (``nodes`` of
  ``x, y, z``; ``segments`` of ``a, b, width, height, sigma[, width_dir]``),
  ``ports`` (``positive, negative[, name]``), ``discretization`` (one of
  ``uniform``, ``per_segment``, ``graded``, ``skin_depth``,
  ``per_segment_graded``), optional ``coupling`` and ``frequencies_hz``, in
  SI units, unknown keys rejected at every level.
* :func:`parse_deck` reads the deck subset: ``.title``, ``.units`` (required),
  ``.default``, ``N`` nodes, ``E`` segments (``w h nwinc nhinc rw rh wx wy wz
  sigma|rho group``), ``.external``, ``.freq``, ``.equiv``, ``.couples``,
  ``.end``; ``*`` comments and ``+`` continuations; directives and node names
  case-insensitive.  Ground planes (fasterhenry-cli/src/inp.rs:53-200,
  2410-2790, 3981-4050, 4329-4398, 4437-4650) in both ``G`` grammars: the
  FastHenry corner-point form (``x1= .. z3= thick= seg1= seg2= segwid1=
  segwid2= sigma=|rho= nhinc= relx= rely= relz= file=NONE``, in-plane nodes
  ``N<name> (x, y, z)``, ``hole rect|point|circle``, ``contact rect`` in its
  six- and seven-value spellings, ``contact decay_rect``, ``contact point``,
  ``contact line``, ``contact trace`` along x or y, the named contact areas
  ``contact equiv_rect N<name>`` and ``contact connection N<name>``, and
  ``contact initial_grid`` / ``initial_mesh_grid``) and the extension form
  (``G<name> x1 y1 z1 x2 y2 z2 t nx= ny= nhinc= sigma=|rho=`` with ``.hole``
  and ``.contact``); the plane meshes come first in the geometry, segment and
  port endpoints inside a plane's slab (or joined to an in-plane node) land
  on its nearest live cell centre, a named contact area's node on the one
  node its cells are tied to, and only declared nodes still referenced as
  themselves are kept.  Other plane clauses (a diagonal ``contact trace``,
  user-defined hole shapes, hierarchy files, tilted planes) are rejected by
  name with the statement's line number.
* ``parse_deck(text, fasthenry_compat=True)`` (and
  :func:`parse_deck_reporting`, which also returns the :class:`DeckWarning`
  list) reads third-party decks the way FastHenry does, each default stated
  in a warning on its line: the title line, metres without ``.units``, the
  long unit spellings, copper, FastHenry's sweep rules and the plane
  defaults.
* :func:`load` picks the reader by file extension (``.inp``/``.fh`` decks,
  anything else JSON), and :func:`run` assembles and sweeps a problem
  (fasterhenry-cli/src/lib.rs:183-230).
"""
from __future__ import annotations

import dataclasses
import json
import math
import os
import re
from typing import Dict, List, Optional, Sequence, Tuple

from . import api as A
from . import plane as PL

UNITS = {"km": 1e3, "m": 1.0, "cm": 1e-2, "mm": 1e-3, "um": 1e-6, "in": 0.0254, "mils": 2.54e-5, "mil": 2.54e-5}
DISCRETIZATION_KINDS = ("uniform", "per_segment", "graded", "skin_depth", "per_segment_graded")


class ProblemError(A.InvalidArgument):
    """A malformed problem document."""


class DeckError(A.InvalidArgument):
    """A deck line the reader rejects; ``line`` is 1-based (0: the whole deck)."""

    def __init__(self, line: int, message: str):
        super().__init__("line %d: %s" % (line, message))
        self.line = line


@dataclasses.dataclass(frozen=True)
class DeckWarning:
    """A deck line read under a stated assumption: the FastHenry defaults the
    ``fasthenry_compat`` mode applies (inp.rs ParseWarning); ``line`` as in
    :class:`DeckError`."""
    line: int
    message: str

    def __str__(self) -> str:
        return "line %d: %s" % (self.line, self.message)


# FastHenry's defaults, applied only in the compat mode (inp.rs:816, 1408,
# 4814-4822): copper where a conductor names no conductivity, a contact cell
# as wide as its rectangle clamped to 0.99 of it, ndec=0 read as 0.01, and
# points up to 0.1 % above fmax kept.
COPPER_SIGMA = 5.8e7
COMPAT_CELL_CLAMP = 0.99
COMPAT_ZERO_NDEC = 0.01
COMPAT_FMAX_SLACK = 1.001
# Unit spellings FastHenry reads at the right scale (its prefix match), read
# in the compat mode with a warning (inp.rs:757-792).
_COMPAT_UNITS = {"meter": ("m", 1.0), "meters": ("m", 1.0), "metre": ("m", 1.0), "metres": ("m", 1.0),
                 "kilometer": ("km", 1e3), "kilometers": ("km", 1e3), "kilometre": ("km", 1e3),
                 "kilometres": ("km", 1e3), "inch": ("in", 0.0254), "inches": ("in", 0.0254)}


# ---------------------------------------------------------------------------
# The JSON problem document
# ---------------------------------------------------------------------------
def _keys(obj, allowed, required, where):
    if not isinstance(obj, dict):
        raise ProblemError("%s must be an object" % where)
    for k in obj:
        if k not in allowed:
            raise ProblemError("unknown field `%s` in %s" % (k, where))
    for k in required:
        if k not in obj:
            raise ProblemError("missing field `%s` in %s" % (k, where))


def _num(v, where) -> float:
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise ProblemError("%s must be a number" % where)
    return float(v)


def _count(v, where) -> int:
    if isinstance(v, bool) or not isinstance(v, int) or v < 0:
        raise ProblemError("%s must be a non-negative integer" % where)
    return int(v)


@dataclasses.dataclass
class Problem:
    """A complete input: geometry, ports, discretization, coupling and the
    frequency sweep (fasterhenry-cli/src/problem.rs:13-36)."""
    nodes: List[Tuple[float, float, float]]
    segments: List[dict]
    ports: List[Tuple[int, int, Optional[str]]]
    discretization: dict
    frequencies_hz: List[float]
    coupling: "A.Coupling" = dataclasses.field(default_factory=lambda: A.Coupling.all_pairs())
    title: Optional[str] = None

    # -- JSON --------------------------------------------------------------
    @classmethod
    def from_json(cls, doc) -> "Problem":
        if isinstance(doc, (str, bytes)):
            doc = json.loads(doc)
        _keys(doc, ("geometry", "ports", "discretization", "coupling", "frequencies_hz"),
              ("geometry", "ports", "discretization", "frequencies_hz"), "the problem document")
        g = doc["geometry"]
        _keys(g, ("nodes", "segments"), (), "geometry")
        nodes = []
        for i, n in enumerate(g.get("nodes", [])):
            _keys(n, ("x", "y", "z"), ("x", "y", "z"), "node %d" % i)
            nodes.append(tuple(_num(n[k], "node %d %s" % (i, k)) for k in ("x", "y", "z")))
        segs = []
        for i, s in enumerate(g.get("segments", [])):
            _keys(s, ("a", "b", "width", "height", "sigma", "width_dir"), ("a", "b", "width", "height", "sigma"),
                  "segment %d" % i)
            seg = {"a": _count(s["a"], "segment %d a" % i), "b": _count(s["b"], "segment %d b" % i),
                   "width": _num(s["width"], "segment %d width" % i),
                   "height": _num(s["height"], "segment %d height" % i),
                   "sigma": _num(s["sigma"], "segment %d sigma" % i), "width_dir": None}
            if "width_dir" in s:
                wd = s["width_dir"]
                if not (isinstance(wd, list) and len(wd) == 3):
                    raise ProblemError("segment %d width_dir must be [x, y, z]" % i)
                seg["width_dir"] = tuple(_num(x, "segment %d width_dir" % i) for x in wd)
            segs.append(seg)
        if not isinstance(doc["ports"], list):
            raise ProblemError("ports must be an array")
        ports = []
        for i, p in enumerate(doc["ports"]):
            _keys(p, ("positive", "negative", "name"), ("positive", "negative"), "port %d" % i)
            name = p.get("name")
            if name is not None and not isinstance(name, str):
                raise ProblemError("port %d name must be a string" % i)
            ports.append((_count(p["positive"], "port %d positive" % i), _count(p["negative"], "port %d negative" % i),
                          name))
        disc = _discretization_from_json(doc["discretization"])
        freqs = doc["frequencies_hz"]
        if not isinstance(freqs, list):
            raise ProblemError("frequencies_hz must be an array")
        coupling = A.Coupling.from_json(doc["coupling"]) if "coupling" in doc else A.Coupling.all_pairs()
        return cls(nodes, segs, ports, disc, [_num(f, "frequencies_hz") for f in freqs], coupling)

    def to_json(self) -> dict:
        out = {
            "geometry": {
                "nodes": [{"x": x, "y": y, "z": z} for (x, y, z) in self.nodes],
                "segments": [dict({k: s[k] for k in ("a", "b", "width", "height", "sigma")},
                                  **({"width_dir": list(s["width_dir"])} if s.get("width_dir") is not None else {}))
                             for s in self.segments]},
            "ports": [dict({"positive": a, "negative": b}, **({"name": n} if n is not None else {}))
                      for (a, b, n) in self.ports],
            "discretization": _discretization_to_json(self.discretization),
            "frequencies_hz": list(self.frequencies_hz),
        }
        if not self.coupling.is_trivial():
            out["coupling"] = self.coupling.to_json()
        return out

    # -- to the library ------------------------------------------------------
    def geometry(self) -> "A.Geometry":
        return A.Geometry.from_parts(self.nodes, [A.SegmentDef(s["a"], s["b"], s["width"], s["height"], s["sigma"],
                                                               s.get("width_dir")) for s in self.segments])

    def port_list(self) -> List["A.Port"]:
        return [A.Port(a, b, n) for (a, b, n) in self.ports]


def _discretization_from_json(d) -> dict:
    if not isinstance(d, dict) or len(d) != 1:
        raise ProblemError("discretization must be an object with exactly one of %s" % ", ".join(DISCRETIZATION_KINDS))
    (kind, v), = d.items()
    if kind == "uniform":
        _keys(v, ("nw", "nh"), ("nw", "nh"), "discretization.uniform")
        return {"kind": "uniform", "nw": _count(v["nw"], "nw"), "nh": _count(v["nh"], "nh")}
    if kind == "graded":
        _keys(v, ("nw", "nh", "ratio"), ("nw", "nh", "ratio"), "discretization.graded")
        return {"kind": "graded", "nw": _count(v["nw"], "nw"), "nh": _count(v["nh"], "nh"),
                "ratio": _num(v["ratio"], "ratio")}
    if kind == "skin_depth":
        keys = ("frequency_hz", "target_skin_depths", "ratio", "max_per_axis")
        _keys(v, keys, keys, "discretization.skin_depth")
        return {"kind": "skin_depth", "frequency_hz": _num(v["frequency_hz"], "frequency_hz"),
                "target_skin_depths": _num(v["target_skin_depths"], "target_skin_depths"),
                "ratio": _num(v["ratio"], "ratio"), "max_per_axis": _count(v["max_per_axis"], "max_per_axis")}
    if kind == "per_segment":
        if not isinstance(v, list):
            raise ProblemError("discretization.per_segment must be an array")
        grids = []
        for i, g in enumerate(v):
            _keys(g, ("nw", "nh"), ("nw", "nh"), "discretization.per_segment[%d]" % i)
            grids.append((_count(g["nw"], "nw"), _count(g["nh"], "nh")))
        return {"kind": "per_segment", "grids": grids}
    if kind == "per_segment_graded":
        if not isinstance(v, list):
            raise ProblemError("discretization.per_segment_graded must be an array")
        grids = []
        keys = ("nw", "nh", "width_ratio", "height_ratio")
        for i, g in enumerate(v):
            _keys(g, keys, keys, "discretization.per_segment_graded[%d]" % i)
            grids.append((_count(g["nw"], "nw"), _count(g["nh"], "nh"), _num(g["width_ratio"], "width_ratio"),
                          _num(g["height_ratio"], "height_ratio")))
        return {"kind": "per_segment_graded", "grids": grids}
    raise ProblemError("unknown discretization `%s`; expected one of %s" % (kind, ", ".join(DISCRETIZATION_KINDS)))


def _discretization_to_json(d: dict) -> dict:
    k = d["kind"]
    if k == "uniform":
        return {"uniform": {"nw": d["nw"], "nh": d["nh"]}}
    if k == "graded":
        return {"graded": {"nw": d["nw"], "nh": d["nh"], "ratio": d["ratio"]}}
    if k == "skin_depth":
        return {"skin_depth": {"frequency_hz": d["frequency_hz"], "target_skin_depths": d["target_skin_depths"],
                               "ratio": d["ratio"], "max_per_axis": d.get("max_per_axis", 32)}}
    if k == "per_segment":
        return {"per_segment": [{"nw": a, "nh": b} for a, b in d["grids"]]}
    return {"per_segment_graded": [{"nw": g[0], "nh": g[1], "width_ratio": g[2], "height_ratio": g[3]}
                                   for g in d["grids"]]}


# ---------------------------------------------------------------------------
# The `.inp` deck
# ---------------------------------------------------------------------------
def frequency_sweep(fmin: float, fmax: float, ndec: float, compat: bool = False) -> List[float]:
    """`.freq fmin fmax ndec`: n = floor(ndec log10(fmax/fmin)) + 1 points
    f(k) = fmin 10^(k/ndec), the exact fmin 10^q where k/ndec is whole
    (inp.rs:509-526, 4829-4896).  ``compat`` keeps the points up to 0.1 %
    above fmax and an fmin above fmax gives no point (FastHenry's rule)."""
    if not (math.isfinite(fmin) and math.isfinite(fmax)) or fmin < 0 or fmax < 0:
        raise ValueError("frequencies must be finite and >= 0")
    if not (math.isfinite(ndec) and ndec > 0):
        raise ValueError("ndec must be > 0, got %r" % ndec)
    if fmax < fmin and not compat:
        raise ValueError("fmax (%r) is below fmin (%r)" % (fmax, fmin))
    if fmin == fmax:
        return [fmin]
    if fmin == 0.0:
        raise ValueError("fmin = 0 is only allowed as the single-frequency case (.freq fmin=0 fmax=0 runs the DC "
                         "solve)")
    # compat keeps points up to 0.1 % above fmax, as FastHenry does
    ceiling = COMPAT_FMAX_SLACK * fmax if compat else fmax
    if fmin > ceiling:
        return []
    # the last step the rule admits, with 1e-9 of slack for rounding, and
    # each point's exponent snapped to a whole decade within 1e-9
    # (inp.rs:4833-4896)
    last = ndec * (math.log10(ceiling) - math.log10(fmin))
    if last + 1.0 > MAX_SWEEP_POINTS:
        raise ValueError("the sweep would have about %.3e points (at most %g); lower ndec or narrow fmin..fmax"
                         % (last + 1.0, MAX_SWEEP_POINTS))

    def point(k):
        exponent = k / ndec
        whole = _round_half_away(exponent)
        if abs(exponent - whole) <= 1e-9 * max(abs(whole), 1.0):
            return fmin * _pow10i(int(whole))
        return fmin * 10.0 ** exponent

    if compat:
        # one candidate past the rule's last step, each checked against the
        # ceiling
        out = []
        for k in range(int(math.floor(last + 1e-9)) + 2):
            f = point(k)
            if f > ceiling:
                break
            out.append(f)
        return out
    return [point(k) for k in range(int(math.floor(last + 1e-9)) + 1)]


MAX_SWEEP_POINTS = 1e7


def _round_half_away(x: float) -> float:
    """f64::round: the nearest integer, halves away from zero."""
    a = abs(x)
    r = math.floor(a)
    if a - r >= 0.5:    # a - floor(a) is exact
        r += 1
    return math.copysign(r, x)


def _pow10i(k: int) -> float:
    """10^k by repeated squaring in binary (f64::powi's scheme); exact for
    the powers of ten a float holds exactly."""
    base, result, e = 10.0, 1.0, abs(k)
    while e:
        if e & 1:
            result *= base
        base *= base
        e >>= 1
    return result if k >= 0 else 1.0 / result


_FIELDS = {"x", "y", "z", "w", "h", "nwinc", "nhinc", "rw", "rh", "wx", "wy", "wz", "sigma", "rho"}
_LENGTHS = {"x", "y", "z", "w", "h"}


def _split_statements(text: str, compat: bool = False):
    """Logical lines: comments dropped, '+' lines joined onto the previous
    statement (keeping the first line's number).  In the compat mode the
    physical first line is the deck's title, whatever it holds, and is not
    read as a statement (inp.rs:3504-3560).  Returns (title, statements,
    number of the last line)."""
    out: List[Tuple[int, str]] = []
    lines = text.splitlines()
    title = None
    start = 0
    if compat and lines:
        title = " ".join(lines[0].split()) or None
        start = 1
    for no, raw in enumerate(lines[start:], start + 1):
        line = raw.strip()
        if not line or line.startswith("*"):
            continue
        if line.startswith("+"):
            if not out:
                raise DeckError(no, "a continuation line with nothing to continue")
            out[-1] = (out[-1][0], out[-1][1] + " " + line[1:])
            continue
        out.append((no, line))
    return title, out, len(lines)


def _tokens(body: str) -> List[str]:
    """Whitespace-separated tokens with whitespace around '=' removed."""
    body = re.sub(r"\s*=\s*", "=", body.strip())
    return body.split()


def _number(tok: str, line: int) -> float:
    try:
        return float(tok)
    except ValueError:
        raise DeckError(line, "'%s' is not a number" % tok) from None


def _assignments(tokens: Sequence[str], line: int, allowed) -> Dict[str, str]:
    out: Dict[str, str] = {}
    for t in tokens:
        if "=" not in t:
            raise DeckError(line, "expected <field>=<value>, got '%s'" % t)
        k, v = t.split("=", 1)
        k = k.lower()
        if not v:
            raise DeckError(line, "'%s=' has no value" % k)
        if k not in allowed:
            raise DeckError(line, "unknown field '%s'" % k)
        out[k] = v
    if "sigma" in out and "rho" in out:
        raise DeckError(line, "give either sigma= or rho=, not both")
    return out


_PLANE_ITEM = re.compile(r"\s*(?:(?P<key>[A-Za-z_][A-Za-z0-9_]*)\s*=\s*(?P<val>[^\s(]+)|"
                         r"(?P<group>\([^)]*\))|(?P<word>[^\s(]+))")


def _plane_items(body: str, line: int) -> List[Tuple[str, str]]:
    """A G statement's body as items: ("key", "k=v"), ("group", "a, b, c")
    and ("word", w)."""
    out: List[Tuple[str, str]] = []
    pos = 0
    body = body.strip()
    while pos < len(body):
        m = _PLANE_ITEM.match(body, pos)
        if not m or m.end() == pos:
            raise DeckError(line, "cannot read the ground plane statement near '%s'" % body[pos:pos + 20])
        if m.group("key"):
            out.append(("key", m.group("key").lower() + "=" + m.group("val")))
        elif m.group("group"):
            out.append(("group", m.group("group")[1:-1]))
        else:
            out.append(("word", m.group("word")))
        pos = m.end()
        while pos < len(body) and body[pos].isspace():
            pos += 1
    return out


def _group_values(text: str, line: int, unit: float) -> List[float]:
    vals = [v.strip() for v in text.split(",")]
    if any(not v for v in vals):
        raise DeckError(line, "an empty value in '(%s)'" % text)
    return [_number(v, line) * unit for v in vals]


@dataclasses.dataclass
class _PlaneSpec:
    name: str
    plane: "PL.GroundPlane"
    nhinc: int
    line: int
    mid_z: float
    axis1: int = 0
    bar_width: Tuple[Optional[float], Optional[float]] = (None, None)


def _plane_extension(head: str, toks: List[str], line: int, unit: float, sigma_default, compat: bool = False,
                     warn=None) -> _PlaneSpec:
    """G<name> x1 y1 z1 x2 y2 z2 t [nx=] [ny=] [nhinc=] [sigma=|rho=]
    (inp.rs:4329-4398): footprint corners, TOP surface z, thickness down."""
    if len(toks) < 7:
        raise DeckError(line, "expected G<name> x1 y1 z1 x2 y2 z2 thickness [nx=..] [ny=..] [nhinc=..], or the "
                              "FastHenry corner-point form G<name> x1=.. y1=.. z1=.. x2=.. ... thick=.. seg1=.. seg2=..")
    x1, y1, z1, x2, y2, z2, t = [_number(v, line) * unit for v in toks[:7]]
    vals = _assignments(toks[7:], line, {"nx", "ny", "nhinc", "sigma", "rho"})
    nx = _deck_count(vals.get("nx", "1"), "nx", line)
    ny = _deck_count(vals.get("ny", "1"), "ny", line)
    nhinc = _deck_count(vals.get("nhinc", "1"), "nhinc", line)
    sigma = _plane_sigma(vals, line, unit, sigma_default, head, compat, warn)
    if nx < 1 or ny < 1:
        raise DeckError(line, "ground plane '%s' needs nx and ny >= 1 (got nx=%d, ny=%d)" % (head, nx, ny))
    plane = PL.GroundPlane((min(x1, x2), min(y1, y2)), (max(x1, x2), max(y1, y2)), max(z1, z2), t, nx, ny, sigma)
    return _PlaneSpec(head, plane, nhinc, line, max(z1, z2) - t / 2.0)


def _rho_sigma(text: str, unit: float, line: int) -> float:
    """A resistivity per deck unit as a conductivity in S/m: 1/rho first,
    then the unit, as the reference's reader does (inp.rs:976-987), so that
    sigma = 1/rho spellings give bit-identical conductivities."""
    r = _number(text, line)
    if r <= 0:
        raise DeckError(line, "rho must be positive")
    return 1.0 / r / unit


def _plane_sigma(vals, line, unit, sigma_default, head, compat=False, warn=None):
    if "sigma" in vals:
        return _number(vals["sigma"], line) / unit
    if "rho" in vals:
        return _rho_sigma(vals["rho"], unit, line)
    if sigma_default is None:
        if compat:
            warn(line, "ground plane '%s' has no conductivity; using copper (5.8e7 S/m, FastHenry default)" % head)
            return COPPER_SIGMA
        raise DeckError(line, "ground plane '%s' has no conductivity: set sigma= or rho= here or in .default" % head)
    return sigma_default


def _finite(tok: str, line: int) -> float:
    v = _number(tok, line)
    if not math.isfinite(v):
        raise DeckError(line, "'%s' is not finite" % tok)
    return v


def _deck_count(text: str, what: str, line: int) -> int:
    """A whole number >= 1 (inp.rs:956-967 parse_count)."""
    if not re.fullmatch(r"\+?[0-9]+", text):
        raise DeckError(line, "'%s' is not a valid %s (a whole number >= 1)" % (text, what))
    v = int(text)
    if v < 1:
        raise DeckError(line, "%s must be >= 1, got %d" % (what, v))
    return v


def _shown(x: float) -> str:
    """A length in a message: shortest round-trip digits, positional (the
    reference prints its f64 values that way)."""
    import numpy as np
    return np.format_float_positional(x, unique=True, trim="-")


def _clause_values(text: str) -> List[str]:
    """A clause's value list: fields separated by commas, whitespace or
    both, empty fields dropped (inp.rs:1073-1124 read_list)."""
    return [v for v in re.split(r"[\s,]+", text.strip()) if v]


def _node_fields(text: str) -> List[str]:
    """An in-plane node's value list with its empty fields kept ("" for a
    field between two commas, or after a trailing one)."""
    parts = text.split(",")
    out: List[str] = []
    for part in parts:
        words = part.split()
        if words:
            out.extend(words)
        elif len(parts) > 1:
            out.append("")
    return out


# The clauses of a corner-point G statement and what they carry, as the
# reference's reader accepts them (inp.rs:2061-2168 apply_clause).
_CONTACT_SHAPES = ("'contact rect (x, y, z, xwidth, ywidth, xcell, ycell)' or '(x1, y1, z1, x2, y2, z2)', "
                   "'contact decay_rect (x, y, z, xwidth, ywidth, xcell, ycell, xmaxcell, ymaxcell)', "
                   "'contact point (x, y, z, xcell, ycell)', 'contact line (x0, y0, z0, x1, y1, z1, xcell, ycell)', "
                   "'contact trace (x0, y0, z0, x1, y1, z1, trace_width, scale_factor)' along x or y, "
                   "'contact equiv_rect N<name> (x, y, z, xwidth, ywidth)', "
                   "'contact connection N<name> (x, y, z, xwidth, ywidth, ratio)', "
                   "'contact initial_grid (n1, n2)' and 'contact initial_mesh_grid (n1, n2)'")


@dataclasses.dataclass
class _Refine:
    """A `contact point` / `line` (and each of a trace's five lines): the
    locus's two ends (x, y, z) and the largest cell wanted, in the plane's
    own (p1->p2, p2->p3) axes."""
    ends: List[List[float]]
    cell: List[float]


def _trace_lines(ends, width: float, along: int, axis1: int) -> List[_Refine]:
    """The documented expansion of an axis-aligned `contact trace` into five
    `contact line`s (inp.rs:1552-1579): at offsets 0 and +-w/2 across the
    trace with cells (length, w/2), and at +-3w/2 with cells (length, w)."""
    across = 1 - along
    length = abs(ends[1][along] - ends[0][along])
    along_slot = 0 if along == axis1 else 1
    out = []
    for offset, across_cell in ((0.0, width / 2.0), (width / 2.0, width / 2.0), (-width / 2.0, width / 2.0),
                                (1.5 * width, width), (-1.5 * width, width)):
        moved = [list(e) for e in ends]
        for e in moved:
            e[across] += offset
        cell = [0.0, 0.0]
        cell[along_slot] = length
        cell[1 - along_slot] = across_cell
        out.append(_Refine(moved, cell))
    return out


def _plane_corner_form(head: str, body: str, line: int, unit: float, sigma_default, compat: bool = False,
                       warn=None):
    """The FastHenry corner-point G statement (inp.rs:1686-2790).  Returns the
    plane and its in-plane nodes [(name, position, equipotential index or
    None)]; a node that a `contact equiv_rect` / `contact connection`
    declares names its contact area, the others attach to the nearest live
    cell.  Corner points, `thick`, `seg1`/`seg2` (or `contact initial_grid`),
    `segwid1`/`segwid2`, `sigma`/`rho`, `nhinc`, `relx`/`rely`/`relz` and
    `file=NONE` are read; every other field or clause is rejected by name."""
    items = _plane_items(body, line)
    # relx / rely / relz move every node, hole and contact coordinate of the
    # statement (not its corner points), wherever they are written; the last
    # value of a repeated key wins (inp.rs:1982-2001).
    offset = [0.0, 0.0, 0.0]
    for kind, text in items:
        if kind == "key":
            key, val = text.split("=", 1)
            if key in ("relx", "rely", "relz"):
                offset["xyz".index(key[3])] = _finite(val, line) * unit

    def triple(vals, what):
        return [_finite(v, line) * unit + offset[a] for a, v in enumerate(vals[:3])]

    def widths_of(vals, what):
        out = []
        for a in range(2):
            w = _finite(vals[3 + a], line) * unit
            if w <= 0:
                raise DeckError(line, "%s: %swidth=%s must be > 0 - it is the rectangle's full width about its "
                                      "centre, not a corner" % (what, "xy"[a], _shown(w)))
            out.append(w)
        return out

    # the compat mode's notes about this statement's clauses, given after
    # the statement's own copper note
    pending: List[str] = []

    def clamped(what, v):
        """[xwidth, ywidth, xcell, ycell]: in the compat mode a cell as wide
        as its rectangle is clamped to 0.99 of the width (inp.rs:1364-1406)."""
        for a in range(2):
            if compat and v[2 + a] > 0 and v[2 + a] >= v[a]:
                written, v[2 + a] = v[2 + a], COMPAT_CELL_CLAMP * v[a]
                pending.append("ground plane '%s': %s: %scell=%s metres is not smaller than %swidth=%s metres; "
                               "clamped to %s x %swidth = %s metres, as FastHenry does (--fasthenry-compat)"
                               % (head, what, "xy"[a], _shown(written), "xy"[a], _shown(v[a]), COMPAT_CELL_CLAMP,
                                  "xy"[a], _shown(v[2 + a])))
        return v

    def node_name(name, what):
        if name is None:
            raise DeckError(line, "%s names the node it ties: write it as '%s N<name> (...)'"
                            % (what, what.strip("'")))
        if not name.lower().startswith("n"):
            raise DeckError(line, "%s: '%s' is not a node name (node names start with 'N', as in '%s Ncontact "
                                  "(...)')" % (what, name, what.strip("'")))
        return name.lower()

    keys: Dict[str, str] = {}
    seg: List[Optional[int]] = [None, None]
    initial_grid: Optional[str] = None
    meshed_grid = False
    segwid: List[Optional[float]] = [None, None]
    file_none = False
    nodes: List[Tuple[str, List[float], Optional[int]]] = []
    hole_rects, hole_points, hole_circles = [], [], []
    contact_rects, contact_decays, contact_lines, contact_traces, contact_equivs = [], [], [], [], []
    corner_keys = {"%s%d" % (a, i) for a in "xyz" for i in (1, 2, 3)}
    k = 0
    while k < len(items):
        kind, text = items[k]
        if kind == "key":
            key, val = text.split("=", 1)
            if key in ("seg1", "seg2"):
                if initial_grid is not None:
                    raise DeckError(line, "ground plane '%s': '%s' and %s both set this plane's cell counts (%s's "
                                          "values are seg1 and seg2), so give one or the other"
                                    % (head, key, initial_grid, initial_grid))
                seg[key == "seg2"] = _deck_count(val, key, line)
            elif key in ("segwid1", "segwid2"):
                w = _finite(val, line) * unit
                if w <= 0:
                    raise DeckError(line, "ground plane '%s': '%s' needs a width > 0 (got '%s=%s')"
                                    % (head, key, key, val))
                segwid[key == "segwid2"] = w
            elif key == "file":
                if val.upper() != "NONE":
                    raise DeckError(line, "ground plane '%s': 'file=%s' names a nonuniform-discretization file, "
                                          "which this reader does not read (only 'file=NONE' is accepted); give "
                                          "the discretization on the statement with 'seg1'/'seg2' or 'contact "
                                          "initial_grid (n1, n2)' and the contact clauses" % (head, val))
                file_none = True
            elif key == "rh":
                raise DeckError(line, "ground plane '%s': 'rh' (filaments graded through the thickness) is not "
                                      "supported; plane filaments are uniform, so use 'nhinc' alone" % head)
            elif key in ("nx", "ny"):
                raise DeckError(line, "ground plane '%s': the corner-point form counts cells with 'seg1'/'seg2' "
                                      "('%s' belongs to the 'G<name> x1 y1 z1 x2 y2 z2 t' extension form)"
                                % (head, key))
            elif key in corner_keys or key in ("thick", "sigma", "rho", "nhinc", "relx", "rely", "relz"):
                keys[key] = val
            else:
                raise DeckError(line, "unknown ground-plane parameter '%s' (supported: x1..z3, thick, seg1, seg2, "
                                      "segwid1, segwid2, sigma, rho, nhinc, relx, rely, relz, file=NONE)" % key)
            k += 1
            continue
        if kind == "group":
            raise DeckError(line, "ground plane '%s': a value list '(%s)' belongs to no clause" % (head, text))
        low = text.lower()
        if low in ("hole", "contact"):
            if k + 1 >= len(items) or items[k + 1][0] != "word":
                raise DeckError(line, "'%s' needs a shape name, as in '%s rect (...)'" % (low, low))
            shape = items[k + 1][1].lower()
            what = "'%s %s'" % (low, shape)
            name = None
            j = k + 2
            if j + 1 < len(items) and items[j][0] == "word" and items[j + 1][0] == "group":
                name = items[j][1]
                j += 1
            if j >= len(items) or items[j][0] != "group":
                raise DeckError(line, "%s needs a parenthesised value list, as in '(x, y, z)'" % what)
            vals = _clause_values(items[j][1])
            k = j + 1
            if name is not None and (low, shape) not in (("contact", "equiv_rect"), ("contact", "connection")):
                raise DeckError(line, "%s takes no node name, but '%s' stands before its value list; only "
                                      "'contact equiv_rect' and 'contact connection' name a node" % (what, name))

            def arity(n, form):
                if len(vals) != n:
                    raise DeckError(line, "%s takes %d values (%s), got %d" % (what, n, form, len(vals)))

            if low == "hole" and shape == "rect":
                arity(6, "x1, y1, z1, x2, y2, z2")
                hole_rects.append((triple(vals[:3], what), triple(vals[3:6], what)))
            elif low == "hole" and shape == "point":
                arity(3, "x, y, z")
                hole_points.append(triple(vals, what))
            elif low == "hole" and shape == "circle":
                arity(4, "x, y, z, r")
                r = _finite(vals[3], line) * unit
                if r < 0:
                    raise DeckError(line, "%s: r=%s metres must be >= 0" % (what, _shown(r)))
                hole_circles.append((triple(vals, what), r))
            elif low == "contact" and shape == "rect" and len(vals) == 7:
                contact_decays.append(("'contact rect'", triple(vals, what),
                                       clamped(what, [_finite(v, line) * unit for v in vals[3:7]]) + [-1.0, -1.0]))
            elif low == "contact" and shape == "rect" and len(vals) == 6:
                contact_rects.append((triple(vals[:3], what), triple(vals[3:6], what)))
            elif low == "contact" and shape == "rect":
                raise DeckError(line, "'contact rect' takes 7 values (x, y, z, xwidth, ywidth, xcell, ycell) or 6 "
                                      "(x1, y1, z1, x2, y2, z2), got %d" % len(vals))
            elif low == "contact" and shape == "decay_rect":
                arity(9, "x, y, z, xwidth, ywidth, xcell, ycell, xmaxcell, ymaxcell")
                v = clamped(what, [_finite(x, line) * unit for x in vals[3:7]])
                limits = []
                for a in range(2):
                    raw = _finite(vals[7 + a], line)
                    if raw == 0:
                        raise DeckError(line, "%s: %smaxcell=0 is neither a cell size nor the 'no limit' sentinel; "
                                              "give a positive cell size, or a negative value to decay all the way "
                                              "to the plane's background cell" % (what, "xy"[a]))
                    limits.append(raw * unit if raw > 0 else -1.0)
                contact_decays.append(("'contact decay_rect'", triple(vals, what), v + limits))
            elif low == "contact" and shape in ("point", "line"):
                n = 5 if shape == "point" else 8
                arity(n, "x, y, z, xcell, ycell" if shape == "point" else "x0, y0, z0, x1, y1, z1, xcell, ycell")
                first = triple(vals[:3], what)
                ends = [first, list(first)] if shape == "point" else [first, triple(vals[3:6], what)]
                cell = [_finite(x, line) * unit for x in vals[n - 2:n]]
                for a in range(2):
                    if cell[a] <= 0:
                        raise DeckError(line, "%s: %scell=%s metres must be > 0 - it is the largest cell wanted "
                                              "along the %s" % (what, "xy"[a], _shown(cell[a]), shape))
                contact_lines.append((what, _Refine(ends, cell)))
            elif low == "contact" and shape == "trace":
                arity(8, "x0, y0, z0, x1, y1, z1, trace_width, scale_factor")
                ends = [triple(vals[:3], what), triple(vals[3:6], what)]
                width = _finite(vals[6], line) * unit
                if width <= 0:
                    raise DeckError(line, "%s: trace_width=%s metres must be > 0" % (what, _shown(width)))
                scale = _finite(vals[7], line)
                if scale <= 0:
                    raise DeckError(line, "%s: scale_factor=%s must be > 0 - it magnifies the cells under the "
                                          "trace" % (what, _shown(scale)))
                dx, dy = abs(ends[1][0] - ends[0][0]), abs(ends[1][1] - ends[0][1])
                if dx == 0.0 and dy == 0.0:
                    raise DeckError(line, "%s has zero length, so it has no direction to refine across; use "
                                          "'contact point (x, y, z, xcell, ycell)' for a point" % what)
                if dy <= 1e-9 * dx:
                    along = 0
                elif dx <= 1e-9 * dy:
                    along = 1
                elif compat:
                    along = None    # refined as its padded bounding box
                    pending.append("ground plane '%s': diagonal 'contact trace' approximated by refining its padded "
                                   "bounding box (a tensor-product refinement), not FastHenry's staircase "
                                   "refinement; cells (trace_width/2)*scale_factor^min(|tan t|, |cot t|)" % head)
                else:
                    raise DeckError(line, "%s from (%s, %s) to (%s, %s) metres is not parallel to x or y; a "
                                          "diagonal 'contact trace' is not supported, because its published "
                                          "description does not fix the cell size under it. Refine under it with "
                                          "'contact line (x0, y0, z0, x1, y1, z1, xcell, ycell)', which refines a "
                                          "diagonal line's bounding box to the cell you choose"
                                    % (what, _shown(ends[0][0]), _shown(ends[0][1]), _shown(ends[1][0]),
                                       _shown(ends[1][1])))
                contact_traces.append((ends, width, along, scale))
            elif low == "contact" and shape in ("equiv_rect", "connection"):
                n = 5 if shape == "equiv_rect" else 6
                arity(n, "x, y, z, xwidth, ywidth" + ("" if n == 5 else ", ratio"))
                centre, widths = triple(vals, what), widths_of(vals, what)
                if shape == "connection":
                    ratio = _finite(vals[5], line)
                    if ratio <= 1.0:
                        raise DeckError(line, "%s: ratio=%s must be > 1 - it divides the rectangle's widths into "
                                              "the contact's own cells (xwidth/ratio, ywidth/ratio)"
                                        % (what, _shown(ratio)))
                nm = node_name(name, what)
                contact_equivs.append((what, nm, centre, widths))
                if shape == "connection":
                    # an equiv_rect plus a decay_rect over the same rectangle
                    # with cells widths / ratio and no outward limit
                    contact_decays.append(("'contact connection'", centre,
                                           widths + [widths[0] / ratio, widths[1] / ratio, -1.0, -1.0]))
            elif low == "contact" and shape in ("initial_grid", "initial_mesh_grid"):
                arity(2, "cells along p1->p2, cells along p2->p3: what 'seg1' and 'seg2' set")
                if initial_grid is not None:
                    raise DeckError(line, "ground plane '%s': %s sets the initial discretization %s has already "
                                          "set on this statement; give one of the two clauses"
                                    % (head, what, initial_grid))
                if seg[0] is not None or seg[1] is not None:
                    raise DeckError(line, "ground plane '%s': %s and 'seg1'/'seg2' both set this plane's cell "
                                          "counts (its values are seg1 and seg2), so give one or the other"
                                    % (head, what))
                seg = [_deck_count(vals[0], "cell count along p1->p2", line),
                       _deck_count(vals[1], "cell count along p2->p3", line)]
                initial_grid = what
                meshed_grid = shape == "initial_mesh_grid"
            elif low == "contact" and shape == "circle":
                raise DeckError(line, "ground plane '%s': 'contact circle' is not supported, and no contact shape "
                                      "of that name is documented ('circle' is a hole shape: 'hole circle (x, y, "
                                      "z, r)'); refine the disc's bounding square instead with 'contact decay_rect "
                                      "(x, y, z, 2r, 2r, xcell, ycell, xmaxcell, ymaxcell)', or use 'contact point "
                                      "(x, y, z, xcell, ycell)' at its centre" % head)
            elif low == "hole":
                raise DeckError(line, "ground plane '%s': 'hole %s' is not supported; the holes are 'hole rect "
                                      "(x1, y1, z1, x2, y2, z2)', 'hole point (x, y, z)' and 'hole circle (x, y, "
                                      "z, r)'" % (head, shape))
            else:
                raise DeckError(line, "ground plane '%s': 'contact %s' is not supported; the contacts are %s"
                                % (head, shape, _CONTACT_SHAPES))
            continue
        if k + 1 < len(items) and items[k + 1][0] == "group":
            if not low.startswith("n"):
                raise DeckError(line, "'%s (...)' is not an in-plane node declaration: node names start with 'N'"
                                % text)
            fields = _node_fields(items[k + 1][1])
            empty = [i for i, f in enumerate(fields) if f == ""]
            if empty and not compat:
                raise DeckError(line, "in-plane node '%s' has an empty coordinate field; write every coordinate "
                                      "(x, y, z) (an empty field reads as 0 only in the compat mode)" % text)
            if empty:
                # compat: one empty field reads as 0, before the offset
                # (inp.rs:2008-2059)
                if len(fields) != 3 or len(empty) > 1:
                    raise DeckError(line, "in-plane node '%s' needs 3 coordinates (x, y, z) with at most one empty "
                                          "field, got %d value(s) of which %d empty" % (text, len(fields), len(empty)))
                fields[empty[0]] = "0"
                pending.append("ground plane '%s': in-plane node '%s' has an empty %s coordinate, read as 0 (before "
                               "the statement's relx/rely/relz offset)" % (head, text, "xyz"[empty[0]]))
            if len(fields) != 3:
                raise DeckError(line, "in-plane node '%s' needs (x, y, z), got %d values" % (text, len(fields)))
            nodes.append((low, triple(fields, "in-plane node '%s'" % text), None))
            k += 2
            continue
        raise DeckError(line, "'%s' is not a ground-plane parameter (expected <field>=<value>, 'N<name> (x, y, z)', "
                              "'hole <shape> (...)' or 'contact <shape> (...)')" % text)
    if "sigma" in keys and "rho" in keys:
        raise DeckError(line, "give either sigma= or rho=, not both")
    pts = []
    for i in (1, 2, 3):
        p = []
        for a in "xyz":
            key = "%s%d" % (a, i)
            if key not in keys:
                raise DeckError(line, "ground plane '%s' is missing '%s' (the corner points are x1..z1, x2..z2, "
                                      "x3..z3)" % (head, key))
            p.append(_number(keys[key], line) * unit)
        pts.append(p)
    e1 = (pts[1][0] - pts[0][0], pts[1][1] - pts[0][1])
    e2 = (pts[2][0] - pts[1][0], pts[2][1] - pts[1][1])
    tol = 1e-9 * (abs(e1[0]) + abs(e1[1]) + abs(e2[0]) + abs(e2[1]))
    if abs(pts[1][2] - pts[0][2]) > tol or abs(pts[2][2] - pts[0][2]) > tol:
        raise DeckError(line, "ground plane '%s' is not parallel to the xy plane; tilted planes are not supported"
                        % head)

    def axis_of(e):
        big = (abs(e[0]) > tol, abs(e[1]) > tol)
        return 0 if big == (True, False) else (1 if big == (False, True) else None)

    a1, a2 = axis_of(e1), axis_of(e2)
    if a1 is None or a2 is None or a1 == a2:
        raise DeckError(line, "ground plane '%s': the corner points do not form an axis-aligned rectangle" % head)
    root_cell = compat and file_none and seg == [None, None] and initial_grid is None
    if root_cell:
        # file=NONE and no grid at all: one root cell, refined only by the
        # contact clauses (inp.rs:2399-2404, 2460-2463)
        seg = [1, 1]
    for i in (0, 1):
        if seg[i] is None:
            raise DeckError(line, "ground plane '%s' has no 'seg%d' (cells along %s)"
                            % (head, i + 1, ("p1->p2", "p2->p3")[i]))
    cells = [0, 0]
    cells[a1], cells[a2] = seg[0], seg[1]
    if "thick" not in keys:
        raise DeckError(line, "ground plane '%s' has no 'thick' (its thickness)" % head)
    thick = abs(_finite(keys["thick"], line)) * unit
    if thick <= 0:
        raise DeckError(line, "ground plane '%s' needs a thickness > 0" % head)
    sigma = _plane_sigma(keys, line, unit, sigma_default, head, compat, warn)
    if root_cell:
        warn(line, "ground plane '%s' has 'file=NONE' and no 'seg1'/'seg2' or 'contact initial_grid': its initial "
                   "grid is a single cell (as 'contact initial_grid (1, 1)'), refined only by its 'contact' clauses"
             % head)
    nhinc = _deck_count(keys["nhinc"], "nhinc", line) if "nhinc" in keys else 1
    lo = (min(p[0] for p in pts), min(p[1] for p in pts))
    hi = (max(p[0] for p in pts), max(p[1] for p in pts))
    origin = (pts[0][0], pts[0][1])
    mid_z = pts[0][2]

    def in_slab(what, z):
        if abs(z - mid_z) > thick + 1e-15:
            raise DeckError(line, "%s: z=%r is not in ground plane '%s'" % (what, z, head))

    def contains(p):
        return lo[0] - tol <= p[0] <= hi[0] + tol and lo[1] - tol <= p[1] <= hi[1] + tol

    def on_plane(what, p):
        in_slab(what, p[2])
        if not contains(p):
            raise DeckError(line, "%s: (%s, %s) metres is outside ground plane '%s'"
                            % (what, _shown(p[0]), _shown(p[1]), head))

    def plane_pair(pair):
        return list(pair) if a1 == 0 else [pair[1], pair[0]]

    def background(a):
        return (hi[a] - lo[a]) / cells[a]

    def footprint(what, corners):
        in_slab(what, corners[0][2])
        in_slab(what, corners[1][2])
        rlo = (min(corners[0][0], corners[1][0]), min(corners[0][1], corners[1][1]))
        rhi = (max(corners[0][0], corners[1][0]), max(corners[0][1], corners[1][1]))
        if not (rhi[0] > rlo[0] and rhi[1] > rlo[1]):
            raise DeckError(line, "%s is degenerate: its two corners share an x or a y" % what)
        return rlo, rhi

    def misses(rlo, rhi):
        return any(rhi[a] < lo[a] - tol or rlo[a] > hi[a] + tol for a in range(2))

    def touches(rlo, rhi):
        return any(min(rhi[a], hi[a]) - max(rlo[a], lo[a]) <= PL.contact_slack(lo[a], hi[a]) for a in range(2))

    def refine_region(refine):
        """The region a refinement locus asks for (inp.rs:3201-3246): its
        bounding box padded by half a cell, cut into cells no coarser than
        the cell, graded outward at ratio 2.  An axis the background already
        meets spans the whole plane at its own cell count; None when both
        axes are met or the region misses the plane."""
        want = plane_pair(refine.cell)
        rlo, rhi, count = [0.0, 0.0], [0.0, 0.0], [0, 0]
        met = True
        for a in range(2):
            if want[a] >= background(a) * (1.0 - 1e-9):
                rlo[a], rhi[a], count[a] = lo[a], hi[a], cells[a]
                continue
            met = False
            p, q = refine.ends[0][a], refine.ends[1][a]
            rlo[a] = min(p, q) - want[a] / 2.0
            rhi[a] = max(p, q) + want[a] / 2.0
            count[a] = PL.cells_no_coarser_than(rhi[a] - rlo[a], want[a])
        if met or touches(rlo, rhi):
            return None
        return PL.ContactRegion.new(rlo, rhi, count, 2.0)

    nonuniform = (file_none or initial_grid is not None or
                  bool(contact_rects or contact_decays or contact_lines or contact_traces or contact_equivs))
    bar_width: List[Optional[float]] = [None, None]
    for i, width in enumerate(segwid):
        if width is None:
            continue
        if nonuniform and compat:
            pending.append("ground plane '%s': 'segwid%d' is ignored on a nonuniform plane (full-width bars are "
                           "used)" % (head, i + 1))
            continue
        if nonuniform:
            raise DeckError(line, "ground plane '%s': 'segwid%d' needs a uniform plane, but this plane's mesh is "
                                  "nonuniform ('file=NONE', 'contact initial_grid' or a 'contact' clause); drop "
                                  "'segwid%d'" % (head, i + 1, i + 1))
        bar_width[a1 if i == 0 else 1 - a1] = width

    holes = []
    if meshed_grid:
        # the checkerboard of `contact initial_mesh_grid` (inp.rs:2876-2911):
        # every cell whose two 1-based indices, counted from the p1 corner,
        # are even; cut into the initial grid before any refinement
        def holed(a):
            ascending = abs(origin[a] - lo[a]) <= abs(hi[a] - origin[a])
            out = []
            for index in range(1, cells[a], 2):
                from_lo = index if ascending else cells[a] - 1 - index
                out.append((lo[a] + from_lo * background(a), lo[a] + (from_lo + 1) * background(a)))
            return out
        for x0, x1 in holed(0):
            for y0, y1 in holed(1):
                holes.append(PL.Hole.rect((x0, y0), (x1, y1)))
    def outside(what, shape, effect):
        # a clause wholly off the footprint is kept (a hole) or dropped (a
        # contact) with a warning, not an error (inp.rs:2640-2760)
        pending.append("%s %s lies wholly outside ground plane '%s' (x %s to %s, y %s to %s metres), so it %s; "
                       "check its coordinates and the deck's .units"
                       % (what, shape, head, _shown(lo[0]), _shown(hi[0]), _shown(lo[1]), _shown(hi[1]), effect))

    def spanning(rlo, rhi):
        return "spanning (%s, %s) to (%s, %s) metres" % (_shown(rlo[0]), _shown(rlo[1]), _shown(rhi[0]),
                                                         _shown(rhi[1]))

    for corners in hole_rects:
        rlo, rhi = footprint("'hole rect'", corners)
        if misses(rlo, rhi):
            outside("'hole rect'", spanning(rlo, rhi), "removes nothing")
        holes.append(PL.Hole.rect(rlo, rhi))
    for p in hole_points:
        in_slab("'hole point'", p[2])
        if not contains(p):
            outside("'hole point'", "at (%s, %s) metres" % (_shown(p[0]), _shown(p[1])), "removes nothing")
        holes.append(PL.Hole.point((p[0], p[1])))
    for p, r in hole_circles:
        in_slab("'hole circle'", p[2])
        gap = math.hypot(max(lo[0] - p[0], p[0] - hi[0], 0.0), max(lo[1] - p[1], p[1] - hi[1], 0.0))
        if gap > r + tol:
            outside("'hole circle'", "centred at (%s, %s) metres with r=%s metres"
                    % (_shown(p[0]), _shown(p[1]), _shown(r)), "removes nothing")
        holes.append(PL.Hole.circle((p[0], p[1]), r))
    # contacts wholly outside the footprint, or only touching its boundary,
    # refine nothing and are dropped (inp.rs:2695-2760)
    contacts = []
    for corners in contact_rects:
        rlo, rhi = footprint("'contact rect'", corners)
        if misses(rlo, rhi):
            outside("'contact rect'", spanning(rlo, rhi), "refines nothing and is ignored")
            continue
        if touches(rlo, rhi):
            pending.append("'contact rect' %s only touches the boundary of ground plane '%s', so it refines "
                           "nothing and is ignored" % (spanning(rlo, rhi), head))
            continue
        contacts.append(PL.ContactRegion.new(rlo, rhi, (2, 2), 2.0))
    def decay_region(what, centre, widths, cell, limit):
        """The graded region of a decay rectangle (inp.rs:3060-3110), its
        widths, cells and limits given per global axis (-1: no limit)."""
        in_slab(what, centre[2])
        rlo, rhi, rc, ratio = [0.0, 0.0], [0.0, 0.0], [0, 0], [0.0, 0.0]
        for a in range(2):
            if not cell[a] > 0:
                raise DeckError(line, "%s: the cell sizes must be positive" % what)
            if not cell[a] < widths[a]:
                raise DeckError(line, "%s: a cell must be smaller than the rectangle's width" % what)
            half = widths[a] / 2.0
            rlo[a] = centre[a] - half
            rhi[a] = centre[a] + half
            rc[a] = PL.cells_no_coarser_than(widths[a], cell[a])
            ratio[a] = 1.0 / (1.0 - cell[a] / widths[a])
            if limit[a] >= 0 and limit[a] < background(a) * (1.0 - 1e-9):
                raise DeckError(line, "%s: a maxcell finer than ground plane '%s''s background cell (%r metres) "
                                      "is not supported; raise seg1/seg2" % (what, head, background(a)))
        return PL.ContactRegion.graded_per_axis(rlo, rhi, rc, ratio)

    for what, centre, v in contact_decays:
        region = decay_region(what, centre, plane_pair(v[0:2]), plane_pair(v[2:4]), plane_pair(v[4:6]))
        if misses(region.lo, region.hi):
            outside(what, spanning(region.lo, region.hi), "refines nothing and is ignored")
            continue
        if touches(region.lo, region.hi):
            pending.append("%s %s only touches the boundary of ground plane '%s', so it refines nothing and is "
                           "ignored" % (what, spanning(region.lo, region.hi), head))
            continue
        contacts.append(region)
    for what, refine in contact_lines:
        for p in refine.ends:
            on_plane(what, p)
        region = refine_region(refine)
        if region is not None:
            contacts.append(region)
    for ends, width, along, scale in contact_traces:
        for p in ends:
            on_plane("'contact trace'", p)
        if along is None:
            # compat: a diagonal trace is its bounding box padded by 3w/2,
            # cells (w/2) s^min(|tan|, |cot|), at most half the narrower
            # width, no outward limit (inp.rs:3167-3199)
            span = [abs(ends[1][0] - ends[0][0]), abs(ends[1][1] - ends[0][1])]
            ratio = min(span) / max(span)
            pad = 3.0 * width / 2.0
            widths = [span[0] + 2.0 * pad, span[1] + 2.0 * pad]
            c = min(width / 2.0 * scale ** ratio, min(widths) / 2.0)
            centre = [(ends[0][0] + ends[1][0]) / 2.0, (ends[0][1] + ends[1][1]) / 2.0, ends[0][2]]
            contacts.append(decay_region("'contact trace'", centre, widths, [c, c], [-1.0, -1.0]))
            continue
        for refine in _trace_lines(ends, width, along, a1):
            region = refine_region(refine)
            if region is not None:
                contacts.append(region)
    # a named contact area: one equipotential patch plus the in-plane node
    # that names it, at the rectangle's centre (inp.rs:2762-2776)
    equipotentials = []
    for what, name, centre, widths in contact_equivs:
        in_slab(what, centre[2])
        equipotentials.append(PL.Equipotential.centred((centre[0], centre[1]), plane_pair(widths)))
        nodes.append((name, centre, len(equipotentials) - 1))
    for name, pos, _ in nodes:
        if not contains(pos):
            raise DeckError(line, "in-plane node '%s' at (%s, %s) metres is outside ground plane '%s'"
                            % (name, _shown(pos[0]), _shown(pos[1]), head))
        in_slab("in-plane node '%s'" % name, pos[2])
    plane = PL.GroundPlane(lo, hi, mid_z + thick / 2.0, thick, cells[0], cells[1], sigma, holes, contacts,
                           equipotentials)
    for note in pending:
        warn(line, note)
    return _PlaneSpec(head, plane, nhinc, line, mid_z, a1, (bar_width[0], bar_width[1])), nodes


def parse_deck(text: str, fasthenry_compat: bool = False) -> Problem:
    """Parses a FastHenry `.inp` deck in this front end's subset into a
    :class:`Problem` (SI units).  ``fasthenry_compat`` reads third-party
    decks the way FastHenry does (inp.rs ParseOptions::fasthenry_compat):
    see :func:`parse_deck_reporting`, which also returns the warnings."""
    return parse_deck_reporting(text, fasthenry_compat)[0]


def parse_deck_reporting(text: str, fasthenry_compat: bool = False) -> Tuple[Problem, List[DeckWarning]]:
    """:func:`parse_deck` with the warnings of the compat mode's defaults, in
    line order.  The compat mode (inp.rs, its `--fasthenry-compat` rows):
    the physical first line is the title; a missing `.units` reads as
    metres and each `.units` applies from its own line on, in the long
    spellings FastHenry reads correctly too; a conductor without a
    conductivity is copper (5.8e7 S/m); `.equiv` of a node with itself is
    ignored; `.freq` reads an omitted ndec as 1 and ndec=0 as 0.01 and keeps
    points up to 0.1 % above fmax; on a ground plane one empty node
    coordinate reads as 0, a contact cell as wide as its rectangle is
    clamped to 0.99 of it, `segwid` on a nonuniform plane is ignored,
    `file=NONE` without a grid is one root cell, and a diagonal `contact
    trace` refines its padded bounding box.  Natively each of these is a
    line-numbered error."""
    compat = bool(fasthenry_compat)
    warnings: List[Tuple[int, int, DeckWarning]] = []   # (line, order, warning)

    def warn(line: int, message: str) -> None:
        warnings.append((line, len(warnings), DeckWarning(line, message)))

    first_line_title, statements, last_line = _split_statements(text, compat)
    unit: Optional[float] = None
    defaults: Dict[str, str] = {}
    defaults_unit: Dict[str, float] = {}
    node_index: Dict[str, int] = {}        # canonical lowercase name -> node slot
    alias: Dict[str, str] = {}             # name -> canonical name
    positions: List[Tuple[float, float, float]] = []
    segments: List[dict] = []
    seg_lines: List[int] = []
    grids: List[Tuple[int, int, float, float]] = []
    groups: List[str] = []
    ports: List[Tuple[str, str, Optional[str], int]] = []
    freqs: Optional[List[float]] = None
    couples: Optional[List[Tuple[str, str]]] = None   # the coupled group pairs of every .couples line
    couple_names: List[Tuple[int, str]] = []           # (line, group) of every group a .couples line names
    couples_first: Optional[int] = None
    couples_all = False
    title = first_line_title     # the compat mode's first line; a later .title replaces it
    ended = False
    planes: List[_PlaneSpec] = []
    plane_node: Dict[str, int] = {}        # in-plane node name -> plane index
    contact_area: Dict[str, int] = {}      # contact-area node name -> its equipotential on that plane

    def resolve(name: str, line: int) -> str:
        key = name.lower()
        key = alias.get(key, key)
        if key not in node_index:
            raise DeckError(line, "node '%s' is not defined (nodes must be declared before they are used)" % name)
        return key

    def field(vals: Dict[str, str], key: str, line: int) -> Optional[float]:
        """A field's value in metres / S/m from the line, else the default."""
        if key in vals:
            v, u = _number(vals[key], line), unit
        elif key in defaults:
            v, u = _number(defaults[key], line), defaults_unit[key]
        else:
            return None
        if key in ("nwinc", "nhinc"):
            return float(_deck_count(vals[key] if key in vals else defaults[key], key, line))
        if key in ("w", "h"):
            return abs(v * u)     # widths and heights are magnitudes (inp.rs:4140-4141)
        return v * u if key in _LENGTHS else v

    def default_sigma(line: int) -> Optional[float]:
        """The .default conductivity in S/m, or None."""
        if "sigma" in defaults:
            return _number(defaults["sigma"], line) / defaults_unit["sigma"]
        if "rho" in defaults:
            return _rho_sigma(defaults["rho"], defaults_unit["rho"], line)
        return None

    for line, stmt in statements:
        if ended:
            raise DeckError(line, "content after .end")
        head, _, rest = stmt.partition(" ")
        low = head.lower()
        if low == ".end":
            if rest.strip():
                raise DeckError(line, ".end takes no arguments")
            ended = True
            continue
        if low == ".title":
            title = " ".join(rest.split())
            continue
        if low == ".units":
            toks = rest.split()
            if len(toks) != 1:
                raise DeckError(line, "expected .units <unit>")
            u = toks[0].lower()
            if u not in UNITS:
                if not compat:
                    raise DeckError(line, "unknown unit '%s'; expected one of km, m, cm, mm, um, in, mils" % toks[0])
                if u.startswith("milli") or u.startswith("micron") or u.startswith("micromet"):
                    reads, documented = ("mils (2.54e-5 m)", "mm") if u.startswith("milli") else ("metres", "um")
                    raise DeckError(line, "'.units %s' is not a documented unit, and FastHenry misreads it as %s, "
                                          "which would scale every length wrongly; write '.units %s'"
                                    % (toks[0], reads, documented))
                if u not in _COMPAT_UNITS:
                    raise DeckError(line, "unknown unit '%s'; expected one of km, m, cm, mm, um, in, mils" % toks[0])
                documented, factor = _COMPAT_UNITS[u]
                warn(line, "'.units %s' is not one of the documented units (km, m, cm, mm, um, in, mils); reading "
                           "it as '%s', as FastHenry does" % (toks[0], documented))
                unit = factor
                continue
            if unit is not None and not compat:
                raise DeckError(line, "duplicate .units directive (.units may appear once)")
            # compat: each .units applies from its own line on; every value
            # read so far is already in metres and S/m
            unit = UNITS[u]
            continue
        if unit is None and (low in (".default", ".hole", ".contact") or low[:1] in ("n", "e", "g")):
            if not compat:
                raise DeckError(line, "a .units line must come before this line (the deck unit is required)")
            warn(line, "no .units directive before this line; reading lengths in metres, as FastHenry does")
            unit = 1.0
        if low == ".default":
            vals = _assignments(_tokens(rest), line, _FIELDS)
            for k, v in vals.items():
                if k in ("sigma", "rho"):
                    defaults.pop("rho" if k == "sigma" else "sigma", None)
                defaults[k] = v
                defaults_unit[k] = unit
            continue
        if low.startswith("n") and not low.startswith("."):
            name = low
            if name in node_index or name in alias:
                raise DeckError(line, "node '%s' is declared twice" % head)
            vals = _assignments(_tokens(rest), line, {"x", "y", "z"})
            xyz = []
            for k in ("x", "y", "z"):
                v = field(vals, k, line)
                if v is None:
                    raise DeckError(line, "node '%s': a coordinate is unset and no .default covers it (set it, or "
                                          ".default x=.. y=.. z=..)" % head)
                xyz.append(v)
            node_index[name] = len(positions)
            positions.append(tuple(xyz))
            continue
        if low.startswith("e") and not low.startswith("."):
            toks = _tokens(rest)
            if len(toks) < 2:
                raise DeckError(line, "a segment needs two node names")
            a, b = resolve(toks[0], line), resolve(toks[1], line)
            vals = _assignments(toks[2:], line, (_FIELDS - {"x", "y", "z"}) | {"group"})
            w, h = field(vals, "w", line), field(vals, "h", line)
            for what, v, key in (("width", w, "w"), ("height", h, "h")):
                if v is None:
                    raise DeckError(line, "segment '%s' has no %s: set %s= here or in .default" % (head, what, key))
            if "sigma" in vals or ("rho" not in vals and "sigma" in defaults):
                src, su = (vals, unit) if "sigma" in vals else (defaults, defaults_unit["sigma"])
                sigma = _number(src["sigma"], line) / su
            elif "rho" in vals or "rho" in defaults:
                src, su = (vals, unit) if "rho" in vals else (defaults, defaults_unit["rho"])
                sigma = _rho_sigma(src["rho"], su, line)
            elif compat:
                warn(line, "segment '%s' has no conductivity; using copper (5.8e7 S/m, FastHenry default)" % head)
                sigma = COPPER_SIGMA
            else:
                raise DeckError(line, "segment '%s' has no conductivity: set sigma= or rho= here or in .default"
                                % head)
            nw = int(field(vals, "nwinc", line) or 1)
            nh = int(field(vals, "nhinc", line) or 1)
            rw = field(vals, "rw", line) or 1.0
            rh = field(vals, "rh", line) or 1.0
            for key, r in (("rw", rw), ("rh", rh)):
                if r < 1.0:
                    raise DeckError(line, "'%s' must be >= 1, got %g" % (key, r))
            wdir = None
            if any(k in vals or k in defaults for k in ("wx", "wy", "wz")):
                wdir = tuple((field(vals, k, line) or 0.0) for k in ("wx", "wy", "wz"))
            segments.append({"a": a, "b": b, "width": w, "height": h, "sigma": sigma, "width_dir": wdir})
            seg_lines.append(line)
            grids.append((nw, nh, rw, rh))
            groups.append(vals.get("group", ""))
            continue
        if low == ".external":
            toks = rest.split()
            if len(toks) not in (2, 3):
                raise DeckError(line, ".external takes two node names and an optional label")
            pos, neg = resolve(toks[0], line), resolve(toks[1], line)
            label = toks[2] if len(toks) == 3 else "%s/%s" % (toks[0].lower(), toks[1].lower())
            ports.append((pos, neg, label, line))
            continue
        if low == ".freq":
            vals = _assignments(_tokens(rest), line, {"fmin", "fmax", "ndec"})
            # all three are required natively; compat reads FastHenry's
            # defaults for an omitted or zero ndec (inp.rs:3787-3870)
            if "fmin" not in vals or "fmax" not in vals or ("ndec" not in vals and not compat):
                raise DeckError(line, ".freq needs fmin=, fmax= and ndec=")
            fmin, fmax = _finite(vals["fmin"], line), _finite(vals["fmax"], line)
            if "ndec" not in vals:
                warn(line, ".freq has no ndec; using ndec=1 (FastHenry behavior)")
                ndec = 1.0
            else:
                ndec = _number(vals["ndec"], line)
            if ndec < 0:
                raise DeckError(line, "ndec must be > 0, got %s (a negative ndec steps away from fmax)"
                                % _shown(ndec))
            if ndec == 0:
                if not compat:
                    raise DeckError(line, "ndec must be > 0, got 0")
                warn(line, ".freq ndec=0 has no points per decade; using ndec=0.01 (FastHenry behavior)")
                ndec = COMPAT_ZERO_NDEC
            if compat and fmin > fmax >= 0.0:
                warn(line, (".freq fmin (%s) is above fmax (%s): the sweep is empty (FastHenry behavior)"
                            if fmin > COMPAT_FMAX_SLACK * fmax else
                            ".freq fmin (%s) is above fmax (%s) but within FastHenry's 0.1%% slack; solving fmin "
                            "alone") % (_shown(fmin), _shown(fmax)))
            try:
                freqs = frequency_sweep(fmin, fmax, ndec, compat)
            except ValueError as e:
                raise DeckError(line, str(e)) from None
            continue
        if low == ".equiv":
            names = [t.lower() for t in rest.split()]
            if len(names) < 2:
                raise DeckError(line, ".equiv joins two or more nodes")
            first = next((i for i, nm in enumerate(names) if alias.get(nm, nm) in node_index), None)
            if first is None:
                raise DeckError(line, ".equiv names no defined node (a name not yet defined becomes a pseudonym "
                                      "for a defined node in the same list)")
            canon = alias.get(names[first], names[first])
            for i, nm in enumerate(names):
                if i == first:
                    continue
                key = alias.get(nm, nm)
                if key == canon:
                    # one node named twice (inp.rs:3879-3930)
                    message = (".equiv of node '%s' with itself" % nm if nm == names[first] else
                               ".equiv of node '%s' with itself: '%s' and '%s' already name one node"
                               % (nm, nm, names[first]))
                    if compat:
                        warn(line, message + "; ignored (--fasthenry-compat)")
                        continue
                    raise DeckError(line, message)
                if key in node_index:
                    # a defined node becomes an alias of the canonical one
                    for k2, v2 in list(alias.items()):
                        if v2 == key:
                            alias[k2] = canon
                    alias[key] = canon
                else:
                    alias[nm] = canon
            continue
        if low == ".couples":
            # `.couples all`, or the groups of one line coupled pairwise with
            # each other (not with other lines' groups); the two forms do not
            # mix (inp.rs:3933-3979)
            toks = rest.split()
            if not toks:
                raise DeckError(line, "expected .couples all | .couples <group> <group> ...")
            if couples_first is None:
                couples_first = line
            conflict = ("conflicting .couples declarations (the first is on line %d): 'all' cannot be combined "
                        "with named groups" % couples_first)
            if toks[0].lower() == "all":
                if len(toks) != 1:
                    raise DeckError(line, "'.couples all' takes no group names (it couples everything)")
                if couples is not None:
                    raise DeckError(line, conflict)
                couples_all = True
                continue
            if couples_all:
                raise DeckError(line, conflict)
            couples = couples or []
            for i, a in enumerate(toks):
                for b in toks[i + 1:]:
                    if a == b:
                        raise DeckError(line, "'.couples' lists group '%s' twice" % a)
                    couples.append((a, b))
                couple_names.append((line, a))
            continue
        if low.startswith("g") and not low.startswith("."):
            if any(pl.name.lower() == low for pl in planes):
                raise DeckError(line, "ground plane '%s' is declared twice" % head)
            first = rest.strip().split(None, 1)[0] if rest.strip() else ""
            try:
                float(first)
                bare = True
            except ValueError:
                bare = False
            if bare:
                planes.append(_plane_extension(head, _tokens(rest), line, unit, default_sigma(line), compat, warn))
            else:
                spec, pnodes = _plane_corner_form(head, rest, line, unit, default_sigma(line), compat, warn)
                for name, pos, area in pnodes:
                    if name in node_index or name in alias:
                        raise DeckError(line, "node '%s' is declared twice" % name)
                    node_index[name] = len(positions)
                    positions.append(tuple(pos))
                    plane_node[name] = len(planes)
                    if area is not None:
                        contact_area[name] = area
                planes.append(spec)
            continue
        if low in (".hole", ".contact"):
            toks = _tokens(rest)
            if len(toks) < 5:
                raise DeckError(line, "expected %s G<name> x1 y1 x2 y2%s"
                                % (low, " [nx=..] [ny=..] [ratio=..]" if low == ".contact" else ""))
            target = [pl for pl in planes if pl.name.lower() == toks[0].lower()]
            if not target:
                raise DeckError(line, "'%s' names unknown ground plane '%s'" % (low, toks[0]))
            pl = target[0]
            b = [_number(t, line) * unit for t in toks[1:5]]
            lo = (min(b[0], b[2]), min(b[1], b[3]))
            hi = (max(b[0], b[2]), max(b[1], b[3]))
            if low == ".hole":
                if len(toks) != 5:
                    raise DeckError(line, "expected .hole G<name> x1 y1 x2 y2")
                pl.plane.holes.append(PL.Hole.rect(lo, hi))
            else:
                vals = _assignments(toks[5:], line, {"nx", "ny", "ratio"})
                cells = (_deck_count(vals.get("nx", "2"), "nx", line), _deck_count(vals.get("ny", "2"), "ny", line))
                ratio = _number(vals.get("ratio", "2"), line)
                if ratio < 1.0:
                    raise DeckError(line, "contact decay ratio must be >= 1 (got %s)" % vals["ratio"])
                pl.plane.contacts.append(PL.ContactRegion.new(lo, hi, cells, ratio))
            continue
        raise DeckError(line, "'%s' is not in the deck subset" % head)
    # the deck-level checks (inp.rs:4401-4435)
    if not ended:
        raise DeckError(last_line, "the deck has no .end directive")
    if unit is None and not compat:
        raise DeckError(last_line, "the deck has no .units directive (units are mandatory: .units <unit>, one of "
                                   "km, m, cm, mm, um, in, mils)")
    if not ports:
        raise DeckError(0, "the deck has no .external port")
    if freqs is None:
        raise DeckError(0, "the deck has no .freq sweep")
    if not segments and not planes:
        raise DeckError(0, "the deck has no conductor: no E segment and no G ground plane")
    # Assembly (inp.rs:4437-4620): the ground-plane meshes first, then the
    # declared nodes still referenced as themselves (in declaration order),
    # then the segments.  An endpoint whose .equiv class holds an in-plane
    # node lands on that plane's nearest live cell centre, and so does one
    # whose position lies in a plane's slab.
    geometry = A.Geometry()
    meshes = []
    plane_grids: List[Tuple[int, int, float, float]] = []
    for pl in planes:
        try:
            centres = pl.plane.build_into(geometry, pl.bar_width)
        except PL.PlaneError as e:
            raise DeckError(pl.line, str(e)) from None
        meshes.append(centres)
        plane_grids += [(1, pl.nhinc, 1.0, 1.0)] * (len(geometry.segments) - len(plane_grids))

    def area_node(nm: str) -> int:
        """The tie node of a named contact area (inp.rs:4663-4693); an area
        that holds no live cell centre is an error whether or not anything
        references it."""
        k = plane_node[nm]
        node = planes[k].plane.equipotential_node(meshes[k], contact_area[nm])
        if node is None:
            raise DeckError(planes[k].line, "ground plane '%s': the contact area named here covers no live cell of "
                                            "the plane's mesh, so it ties nothing; widen it, or refine the mesh so "
                                            "a cell centre falls inside it" % planes[k].name)
        return node

    for nm in sorted(contact_area, key=lambda k: node_index[k]):
        area_node(nm)
    # the in-plane node each .equiv class attaches through (inp.rs:4695-4731):
    # the first in declaration order, except that a named contact area wins
    # over a plain in-plane node of the same plane
    owner: Dict[str, str] = {}
    for nm, k in sorted(plane_node.items(), key=lambda kv: node_index[kv[0]]):
        canon = alias.get(nm, nm)
        if canon in owner and plane_node[owner[canon]] != k:
            raise DeckError(0, ".equiv joins in-plane nodes of two different ground planes; connect the planes "
                               "with a segment instead")
        if canon not in owner or (owner[canon] not in contact_area and nm in contact_area):
            owner[canon] = nm

    def snapped(nm: str) -> Optional[int]:
        canon = alias.get(nm, nm)
        if canon in owner:
            pnode = owner[canon]
            if pnode in contact_area:
                return area_node(pnode)
            k = plane_node[pnode]
            return planes[k].plane.attach(meshes[k], positions[node_index[pnode]])
        pos = positions[node_index[canon]]
        for k, pl in enumerate(planes):
            if pl.plane.contains(pos, 0.0):
                return pl.plane.attach(meshes[k], pos)
        return None

    seg_ends = [(snapped(sg["a"]), snapped(sg["b"])) for sg in segments]
    port_ends = [(snapped(p), snapped(n)) for (p, n, _, _) in ports]
    used = set()
    for (sa, sb), sg in zip(seg_ends, segments):
        if sa is None:
            used.add(alias.get(sg["a"], sg["a"]))
        if sb is None:
            used.add(alias.get(sg["b"], sg["b"]))
    for (sp, sn), (p, n, _, _) in zip(port_ends, ports):
        if sp is None:
            used.add(alias.get(p, p))
        if sn is None:
            used.add(alias.get(n, n))
    slot: Dict[str, int] = {}
    for nm in sorted(node_index, key=lambda k: node_index[k]):
        if nm in alias or nm not in used:
            continue
        slot[nm] = geometry.add_node(A.Node(*positions[node_index[nm]]))
    nodes = [(nd.x, nd.y, nd.z) for nd in geometry.nodes]

    def end(nm: str, snap: Optional[int]) -> int:
        return snap if snap is not None else slot[alias.get(nm, nm)]
    plane_segs = [{"a": sd.a, "b": sd.b, "width": sd.width, "height": sd.height, "sigma": sd.sigma,
                   "width_dir": None} for sd in geometry.segments]
    segs = plane_segs + [dict(sg, a=end(sg["a"], sa), b=end(sg["b"], sb))
                         for sg, (sa, sb) in zip(segments, seg_ends)]
    # every E segment through the library's own rule (a zero length, a
    # width direction along the segment, ...), reported on its own line
    # (inp.rs:4573-4581)
    check = A.Geometry.from_parts(nodes, [])
    for k, sg in enumerate(segs[len(plane_segs):]):
        try:
            check.add_segment(sg)
        except A.GeometryError as e:
            raise DeckError(seg_lines[k], str(e)) from None
    port_list = [(end(p, sp), end(n, sn), label) for (p, n, label, _), (sp, sn) in zip(ports, port_ends)]
    grids = plane_grids + grids
    groups = [""] * len(plane_grids) + groups
    if any(g[2] != 1.0 or g[3] != 1.0 for g in grids):
        disc = {"kind": "per_segment_graded", "grids": grids}
    elif grids and all(g[:2] == grids[0][:2] for g in grids):
        disc = {"kind": "uniform", "nw": grids[0][0], "nh": grids[0][1]}
    elif grids:
        disc = {"kind": "per_segment", "grids": [g[:2] for g in grids]}
    else:
        disc = {"kind": "uniform", "nw": 1, "nh": 1}
    if couples is not None:
        # groups named but carried by no segment are a typo (inp.rs:4767-4796)
        for cline, g in couple_names:
            if g not in groups:
                raise DeckError(cline, "'.couples' names group '%s', which no segment carries" % g)
        _check_transitive(groups, couples, couples_first)
        coupling = A.Coupling.truncated(groups)
        for a, b in couples:
            coupling = coupling.coupled(a, b)
    else:
        # without named .couples every pair couples, whatever groups the
        # segments carry
        coupling = A.Coupling.all_pairs()
    problem = Problem(nodes, segs, port_list, disc, freqs or [], coupling, title)
    return problem, [w for _, _, w in sorted(warnings, key=lambda t: (t[0], t[1]))]


def _check_transitive(groups: Sequence[str], pairs: Sequence[Tuple[str, str]], line: int) -> None:
    """The declared couples must be an equivalence: two groups coupled
    through others are coupled to each other too (coupling.rs:326-420
    Coupling::resolve and check_transitive, which the reference's reader
    applies to a deck's .couples lines).  Groups in order of first
    appearance over the segments; the error names the first pair, in that
    order, that is joined but not declared."""
    names: List[str] = []
    for g in groups:
        if g not in names:
            names.append(g)
    n = len(names)
    if n < 3:
        return
    index = {g: i for i, g in enumerate(names)}
    couples = [[a == b for b in range(n)] for a in range(n)]
    for a, b in pairs:
        couples[index[a]][index[b]] = couples[index[b]][index[a]] = True
    parent = list(range(n))

    def find(x: int) -> int:
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a in range(n):
        for b in range(a + 1, n):
            if couples[a][b]:
                ra, rb = find(a), find(b)
                if ra != rb:
                    parent[ra] = rb
    for a in range(n):
        for b in range(a + 1, n):
            if not couples[a][b] and find(a) == find(b):
                raise DeckError(line, "the .couples declarations are not transitive: groups '%s' and '%s' are "
                                      "coupled through other groups but not to each other; declare them together "
                                      "on one .couples line" % (names[a], names[b]))


def load(path: str, fasthenry_compat: bool = False) -> Problem:
    """A problem from a file: `.inp` / `.fh` as a deck (``fasthenry_compat``
    as in :func:`parse_deck_reporting`), anything else as the JSON document
    (fasterhenry-cli/src/lib.rs read_inputs)."""
    with open(path) as f:
        text = f.read()
    if os.path.splitext(path)[1].lower() in (".inp", ".fh"):
        return parse_deck(text, fasthenry_compat)
    return Problem.from_json(text)


def run(problem: Problem, precision: "A.Precision" = A.Precision.FP64,
        solver: "A.SolverChoice" = A.SolverChoice.AUTO, frequencies: Optional[Sequence[float]] = None):
    """Assemble and sweep a problem (fasterhenry-cli/src/lib.rs:183-230): the
    dense path with its coupling, or the matrix-free path when the solver
    choice resolves there (which couples every pair).  Returns the
    SweepResult and the truncation warnings."""
    freqs = list(problem.frequencies_hz if frequencies is None else frequencies)
    if not problem.ports:
        raise A.InvalidArgument("no ports: give .external in the deck or ports in the document")
    if not freqs:
        raise A.InvalidArgument("no frequencies: give .freq in the deck or frequencies_hz in the document")
    geometry = problem.geometry()
    ports = problem.port_list()
    n = len(A.discretize(geometry, problem.discretization)[0]) if solver == A.SolverChoice.AUTO else 0
    path = solver.resolve(n) if solver != A.SolverChoice.DENSE else "dense"
    if path == "iterative":
        if not problem.coupling.is_all_pairs():
            raise A.Unsupported("a truncating coupling is a dense-path feature; choose the dense solver")
        with A.IterativeSystem.assemble(geometry, ports, problem.discretization) as system:
            return system.sweep(freqs), []
    with A.MeshSystem.assemble(geometry, ports, problem.discretization, coupling=problem.coupling) as system:
        warnings = [str(w) for w in system.truncation_warnings()]
        return system.sweep(freqs, precision), warnings
