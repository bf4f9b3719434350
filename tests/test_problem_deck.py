"""The problem front end (fasterhenry_b200/problem.py): the JSON problem
document (docs/input-format.md of the reference) and the `.inp` deck subset
(fasterhenry-cli/src/inp.rs:12-600): units, defaults, nodes, segments,
ports, frequency sweeps, node equivalence, coupling groups and the errors
the reader reports with line numbers.  Host-only."""
import json
import math

import pytest

from fasterhenry_b200 import problem as P

DECK = """* a two-segment trace
.units mm
.default sigma=5.8e4 w=0.1 h=0.035
N1 x=0 y=0 z=0
N2 x = 1 y=0 z=0
N3 x=1 y=1 z=0
E1 N1 N2 nwinc=3 nhinc=2
E2 N2 n3 nwinc=3
+ nhinc=2
.external N1 N3
.freq fmin=1e3 fmax=1e6 ndec=10
.end
"""


def test_a_small_deck_reads_in_si_units():
    p = P.parse_deck(DECK)
    assert p.nodes == [(0.0, 0.0, 0.0), (1e-3, 0.0, 0.0), (1e-3, 1e-3, 0.0)]
    s = p.segments[0]
    assert s["a"] == 0 and s["b"] == 1
    assert math.isclose(s["width"], 1e-4, rel_tol=1e-15) and math.isclose(s["height"], 3.5e-5, rel_tol=1e-15)
    assert math.isclose(s["sigma"], 5.8e7, rel_tol=1e-15)
    assert p.discretization == {"kind": "uniform", "nw": 3, "nh": 2}
    assert p.ports == [(0, 2, "n1/n3")]
    assert len(p.frequencies_hz) == 31 and p.frequencies_hz[0] == 1e3 and p.frequencies_hz[30] == 1e6
    assert p.coupling.is_trivial()


def test_frequency_sweeps():
    assert P.frequency_sweep(1e3, 1e7, 0.5) == [1e3, 1e5, 1e7]
    assert P.frequency_sweep(5.0, 5.0, 3) == [5.0]
    assert P.frequency_sweep(0.0, 0.0, 1) == [0.0]
    with pytest.raises(ValueError):
        P.frequency_sweep(0.0, 1e3, 1)
    with pytest.raises(ValueError):
        P.frequency_sweep(1e3, 1e6, -1)
    f = P.frequency_sweep(1e6, 1e9, 1)
    assert f == [1e6, 1e7, 1e8, 1e9]
    # the reference reader's sweep answers (inp.rs tests 8779-8790): whole
    # decades exact at any ndec, the last point the stepped value, never fmax
    g = P.frequency_sweep(1e3, 1e7, 1.5)
    assert (g[0], g[3], g[6]) == (1e3, 1e5, 1e7)
    g = P.frequency_sweep(1e3, 9e3, 2.5)
    assert len(g) == 3 and g[2] < 9e3
    assert P.frequency_sweep(1.0, 9.995, 1) == [1.0]
    # a decade step that lands within rounding of a whole exponent is that
    # exact power of ten (3 / 0.1 is 30.000000000000004 in floating point)
    h = P.frequency_sweep(1.0, 1e3, 10.0 / 3.0 * 0.3 * 10.0)
    assert h[0] == 1.0 and h[-1] == 1e3
    with pytest.raises(ValueError, match="below fmin"):
        P.frequency_sweep(1e6, 1e3, 1)
    with pytest.raises(ValueError, match="ndec"):
        P.frequency_sweep(5.0, 5.0, -0.5)
    with pytest.raises(ValueError, match="points"):
        P.frequency_sweep(1.0, 1e300, 1e6)


@pytest.mark.parametrize("sweep,what", [
    ("fmin=1e3 fmax=1e6", "ndec="), ("fmin=1e3 fmax=1e6 ndec=0", "ndec must be > 0, got 0"),
    ("fmin=1e3 fmax=1e7 ndec=-1", "ndec"), ("fmin=1e3 fmax=1e3 ndec=-0.5", "ndec"),
    ("fmin=1e3 fmax=1e6 ndec=1 fstep=2", "unknown field"),
])
def test_freq_needs_all_three_fields_and_a_positive_ndec(sweep, what):
    deck = (".units m\nn1 x=0 y=0 z=0\nn2 x=1 y=0 z=0\ne1 n1 n2 w=1 h=1 sigma=1\n.external n1 n2\n.freq %s\n.end"
            % sweep)
    with pytest.raises(P.DeckError) as e:
        P.parse_deck(deck)
    assert e.value.line == 6 and what in str(e.value), str(e.value)


def test_resistivity_grading_and_per_segment_counts():
    deck = """.units um
N1 x=0 y=0 z=0
N2 x=100 y=0 z=0
N3 x=100 y=100 z=0
E1 N1 N2 w=10 h=2 rho=0.0172 nwinc=5 rw=2
E2 N2 N3 w=10 h=2 rho=0.0172 nwinc=4 nhinc=1
.external N1 N3 coil
.freq fmin=1e9 fmax=1e9 ndec=1
.end"""
    p = P.parse_deck(deck)
    # rho in ohm * um: sigma = 1 / (rho * 1e-6) S/m
    assert math.isclose(p.segments[0]["sigma"], 1.0 / (0.0172e-6), rel_tol=1e-15)
    assert p.discretization["kind"] == "per_segment_graded"
    assert p.discretization["grids"] == [(5, 1, 2.0, 1.0), (4, 1, 1.0, 1.0)]
    assert p.ports == [(0, 2, "coil")]
    p2 = P.parse_deck(deck.replace(" rw=2", ""))
    assert p2.discretization == {"kind": "per_segment", "grids": [(5, 1), (4, 1)]}


def test_equiv_joins_nodes_and_drops_the_alias():
    deck = """.units m
N1 x=0 y=0 z=0
N2 x=1 y=0 z=0
N3 x=1 y=0 z=0
N4 x=2 y=0 z=0
E1 N1 N2 w=0.1 h=0.1 sigma=1
E2 N3 N4 w=0.1 h=0.1 sigma=1
.equiv N2 N3 mid
.external N1 mid
.freq fmin=0 fmax=0 ndec=1
.end"""
    p = P.parse_deck(deck)
    assert len(p.nodes) == 3
    assert p.segments[0]["b"] == p.segments[1]["a"] == 1
    assert p.ports == [(0, 1, "n1/mid")]
    assert p.frequencies_hz == [0.0]


def test_width_direction_and_groups():
    deck = """.units m
.default w=0.1 h=0.05 sigma=1
N1 x=0 y=0 z=0
N2 x=0 y=0 z=1
N3 x=5 y=0 z=0
N4 x=5 y=0 z=1
E1 N1 N2 wy=1 group=left
E2 N3 N4 group=right
.external N1 N2
.external N3 N4
.couples left right
.freq fmin=1e6 fmax=1e6 ndec=1
.end"""
    p = P.parse_deck(deck)
    assert p.segments[0]["width_dir"] == (0.0, 1.0, 0.0) and p.segments[1]["width_dir"] is None
    assert p.coupling.segment_groups == ["left", "right"] and p.coupling.couples("left", "right")
    assert not p.coupling.is_all_pairs()
    p_all = P.parse_deck(deck.replace(".couples left right", ".couples all"))
    assert p_all.coupling.is_all_pairs()


@pytest.mark.parametrize("text,line,what", [
    ("N1 x=0\n.end", 1, ".units"),
    (".units mm\nN1 x=0 y=0 z=0\n", 2, ".end"),
    (".units mm\nN1 x=0 y=0 z=0\n.bogus\n.end", 3, "not in the deck subset"),
    (".units mm\nN1 x=0 y=0 z=0\nGplane x1=0\n.end", 3, "is missing 'y1'"),
    (".units mm\nGp 0 0 0 1 1 0 0.1 nx=2 ny=2 sigma=1\n.hole Gq 0 0 1 1\n.end", 3, "unknown ground plane 'Gq'"),
    (".units mm\nGp x1=0 y1=0 z1=0 x2=1 y2=0 z2=0 x3=1 y3=1 z3=0 thick=0.1 seg1=2 seg2=2 sigma=1 hole user1 (1, 2)\n.end", 2, "'hole user1' is not supported"),
    (".units mm\nN1 x=0 y=0 z=0\nE1 N1 N9 w=1 h=1 sigma=1\n.end", 3, "not defined"),
    (".units mm\nN1 x=0 y=0 z=0\nN2 x=1 y=0 z=0\nE1 N1 N2 w=1 h=1\n.end", 4, "conductivity"),
    (".units mm\nN1 x=0 y=0 z=0\nN2 x=1 y=0 z=0\nE1 N1 N2 w=1 h=1 sigma=1 rho=1\n.end", 4, "either"),
    (".units mm\nN1 x=0 y=0 z=0\nn1 x=1 y=0 z=0\n.end", 3, "twice"),
    (".units mm\nN1 x=0 y=0 z=0\n.end\nN2 x=1 y=0 z=0", 4, "after .end"),
    (".units furlong\n.end", 1, "unknown unit"),
    (".units m\nn1 x=0\n.end", 2, ".default"),
    (".units m\nn1 x=0 y=0 z=0\nn2 x=1 y=0 z=0\ne1 n1 n2 h=1 sigma=1\n.end", 4, "'e1' has no width"),
    (".units m\nn1 x=0 y=0 z=0\nn2 x=1 y=0 z=0\ne1 n1 n2 w=1 h=1 sigma=1 nwinc=2.5\n.end", 4, "nwinc"),
])
def test_errors_carry_the_line(text, line, what):
    with pytest.raises(P.DeckError) as e:
        P.parse_deck(text)
    assert e.value.line == line and what in str(e.value), str(e.value)


def test_json_document_round_trips_and_rejects_unknown_keys():
    p = P.parse_deck(DECK)
    doc = p.to_json()
    assert set(doc) == {"geometry", "ports", "discretization", "frequencies_hz"}
    assert doc["discretization"] == {"uniform": {"nw": 3, "nh": 2}}
    back = P.Problem.from_json(json.dumps(doc))
    assert back.nodes == p.nodes and back.segments == p.segments and back.ports == p.ports
    assert back.discretization == p.discretization and back.frequencies_hz == p.frequencies_hz
    bad = dict(doc, typo=1)
    with pytest.raises(P.ProblemError, match="typo"):
        P.Problem.from_json(bad)
    port_typo = dict(doc, ports=[{"positive": 0, "negative": 1, "nmae": "x"}])
    with pytest.raises(P.ProblemError, match="nmae"):
        P.Problem.from_json(port_typo)
    with pytest.raises(P.ProblemError, match="unknown discretization"):
        P.Problem.from_json(dict(doc, discretization={"fancy": {}}))
    sk = dict(doc, discretization={"skin_depth": {"frequency_hz": 1e9, "target_skin_depths": 0.5, "ratio": 2.0,
                                                  "max_per_axis": 32}})
    assert P.Problem.from_json(sk).discretization["kind"] == "skin_depth"
    coupled = dict(doc, coupling={"segment_groups": ["a", "b"], "couples": [["a", "b"]]})
    assert P.Problem.from_json(coupled).to_json()["coupling"] == coupled["coupling"]


def test_load_picks_the_reader_by_extension(tmp_path):
    deck = tmp_path / "trace.inp"
    deck.write_text(DECK)
    doc = tmp_path / "trace.json"
    doc.write_text(json.dumps(P.parse_deck(DECK).to_json()))
    a, b = P.load(str(deck)), P.load(str(doc))
    assert a.nodes == b.nodes and a.segments == b.segments


@pytest.mark.parametrize("unit", ["m", "mm", "um", "mils"])
@pytest.mark.parametrize("rho", ["0.0172", "1.72e-8", "3", "0.7"])
def test_rho_and_its_reciprocal_sigma_give_the_same_conductivity_bits(unit, rho):
    """1/rho first, then the unit (inp.rs:976-987): a deck written with
    sigma = the correctly rounded 1/rho reads to the very same conductivity,
    on a segment, in .default and on a ground plane."""
    sigma = repr(1.0 / float(rho))
    base = (".units %s\n%%s\nN1 x=0 y=0 z=0\nN2 x=1 y=0 z=0\nE1 N1 N2 w=0.1 h=0.1 %%s\n"
            "Gp x1=0 y1=-3 z1=-1 x2=2 y2=-3 z2=-1 x3=2 y3=-2 z3=-1 thick=0.1 seg1=2 seg2=1 %%s\n"
            ".external N1 N2\n.freq fmin=1 fmax=1 ndec=1\n.end" % unit)
    for default, line_field, plane_field in [("", "rho=%s" % rho, "rho=%s" % rho),
                                             (".default rho=%s" % rho, "", "")]:
        a = P.parse_deck(base % (default, line_field, plane_field))
        b = P.parse_deck(base % (default.replace("rho=" + rho, "sigma=" + sigma),
                                 line_field.replace("rho=" + rho, "sigma=" + sigma),
                                 plane_field.replace("rho=" + rho, "sigma=" + sigma)))
        assert [s["sigma"] for s in a.segments] == [s["sigma"] for s in b.segments]


COUPLE_DECK = """.units m
.default w=0.1 h=0.05 sigma=1
N1 x=0 y=0 z=0
N2 x=0 y=0 z=1
N3 x=5 y=0 z=0
N4 x=5 y=0 z=1
N5 x=10 y=0 z=0
N6 x=10 y=0 z=1
N7 x=15 y=0 z=0
N8 x=15 y=0 z=1
E1 N1 N2 group=a
E2 N3 N4 group=b
E3 N5 N6 group=c
E4 N7 N8 group=d
.external N1 N2
%s
.freq fmin=1e6 fmax=1e6 ndec=1
.end"""


def test_couples_pairs_the_groups_of_each_line_only():
    """inp.rs:3933-3979: a .couples line couples its own groups pairwise;
    two lines do not couple across each other."""
    p = P.parse_deck(COUPLE_DECK % ".couples a b\n.couples c d")
    c = p.coupling
    assert c.couples("a", "b") and c.couples("c", "d")
    assert not c.couples("a", "c") and not c.couples("b", "d")
    three = P.parse_deck(COUPLE_DECK % ".couples a b c").coupling
    assert three.couples("a", "c") and three.couples("b", "c") and not three.couples("a", "d")
    # groups without a named .couples line: every pair couples
    assert P.parse_deck(COUPLE_DECK % "").coupling.is_all_pairs()


@pytest.mark.parametrize("couples,line,what", [
    (".couples a b\n.couples all", 17, "conflicting .couples declarations (the first is on line 16)"),
    (".couples all\n.couples a b", 17, "conflicting"),
    (".couples all a", 16, "takes no group names"),
    (".couples a b a", 16, "lists group 'a' twice"),
    (".couples a zz", 16, "group 'zz', which no segment carries"),
    (".equiv N1 N1", 16, "with itself"),
    (".equiv N3 x\n.equiv x N3", 17, "with itself: 'n3' and 'x' already name one node"),
])
def test_couples_and_equiv_errors(couples, line, what):
    with pytest.raises(P.DeckError) as e:
        P.parse_deck(COUPLE_DECK % couples)
    assert e.value.line == line and what in str(e.value), str(e.value)


@pytest.mark.parametrize("segment,what", [
    ("e1 n1 n2 w=1 h=1 sigma=1 wx=1", "width"),   # width direction along the segment
    ("e1 n1 n3 w=1 h=1 sigma=1", "zero length"),
])
def test_a_segment_the_geometry_rejects_is_reported_on_its_line(segment, what):
    deck = (".units m\nn1 x=0 y=0 z=0\nn2 x=1 y=0 z=0\nn3 x=0 y=0 z=0\n%s\n.external n1 n2\n"
            ".freq fmin=1 fmax=1 ndec=1\n.end" % segment)
    with pytest.raises(P.DeckError) as e:
        P.parse_deck(deck)
    assert e.value.line == 5 and what in str(e.value), str(e.value)


def test_non_transitive_couples_lines_are_rejected():
    """fasterhenry-cli/tests/roundtrip.rs:645-674: a b and b c without a c."""
    with pytest.raises(P.DeckError) as e:
        P.parse_deck(COUPLE_DECK % ".couples a b\n.couples b c")
    assert "'a'" in str(e.value) and "'c'" in str(e.value) and e.value.line == 16
    # declared together, the three are one coupled set
    assert P.parse_deck(COUPLE_DECK % ".couples a b c").coupling.couples("a", "c")
