"""The deck reader pinned to the reference's own fixtures
(fasterhenry-cli/tests/data, copied byte for byte into tests/golden/decks):
the two-turn spiral as a `.inp` deck and as the equivalent JSON problem
document read to the same problem field by field
(fasterhenry-cli/tests/roundtrip.rs:18-30), and the two-port deck reads to
its stated geometry.  Host-only."""
import os

import pytest

from fasterhenry_b200 import problem as P

DECKS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "decks")


def load(name):
    return P.load(os.path.join(DECKS, name))


def test_spiral_deck_and_document_agree_field_by_field():
    a, b = load("spiral.inp"), load("spiral.json")
    assert a.nodes == b.nodes
    assert a.segments == b.segments
    assert a.ports == b.ports
    assert a.discretization == b.discretization
    assert a.frequencies_hz == b.frequencies_hz == [1e6, 1e7, 1e8, 1e9]
    assert a.coupling.is_trivial() and b.coupling.is_trivial()
    assert a.to_json() == b.to_json()


def test_spiral_deck_reads_its_stated_geometry():
    p = load("spiral.inp")
    assert len(p.nodes) == 9 and len(p.segments) == 8
    assert p.nodes[8] == (-2e-3, -2e-3, 0.0)
    for s in p.segments:
        assert (s["width"], s["height"], s["sigma"]) == (2e-4, 3.5e-5, 5.8e7)
    assert p.discretization == {"kind": "uniform", "nw": 3, "nh": 2}
    assert p.ports == [(0, 8, "spiral")]


def test_twobar_deck_reads_two_named_ports():
    p = load("twobar.inp")
    assert p.nodes == [(0.0, 0.0, 0.0), (5e-3, 0.0, 0.0), (0.0, 5e-4, 0.0), (5e-3, 5e-4, 0.0)]
    assert [(s["a"], s["b"]) for s in p.segments] == [(0, 1), (2, 3)]
    assert p.ports == [(0, 1, "barA"), (2, 3, "barB")]
    assert p.frequencies_hz == [1e6, 1e7, 1e8, 1e9]


# The two ```json example documents of the reference's docs/input-format.md
# (extracted in order by tests/golden/decks/copy_reference_decks.py), held to
# what fasterhenry-cli/tests/input_format_doc.rs asserts of them.
EXAMPLES = ["input_format_example_0.json", "input_format_example_1.json"]


def example_text(k):
    with open(os.path.join(DECKS, EXAMPLES[k])) as f:
        return f.read()


def test_every_documented_example_parses_and_the_first_is_the_minimal_one(oracle):
    import numpy as np
    from fasterhenry_b200 import fixtures as F
    for k in range(len(EXAMPLES)):
        prob = P.Problem.from_json(example_text(k))
        # the oracle (the reference's dense path, restated) solves it: one
        # p x p impedance per listed frequency
        deck = F.Deck(list(prob.nodes), [dict(s) for s in prob.segments], [(a, b) for a, b, _ in prob.ports],
                      dict(prob.discretization))
        system = oracle.System(deck)
        z = np.array([system.impedance(f) for f in prob.frequencies_hz])
        assert z.shape == (len(prob.frequencies_hz), len(prob.ports), len(prob.ports)), k
        assert np.all(np.isfinite(z)) and np.all(z[:, range(len(prob.ports)), range(len(prob.ports))].real > 0)
        # and the document round-trips
        assert P.Problem.from_json(prob.to_json()).to_json() == prob.to_json()
    minimal = P.Problem.from_json(example_text(0))
    assert len(minimal.segments) == 1 and len(minimal.ports) == 1 and minimal.coupling.is_trivial()
    second = P.Problem.from_json(example_text(1))
    assert [p[2] for p in second.ports] == ["coil", "sense"] and second.discretization["kind"] == "skin_depth"
    assert second.segments[3]["width_dir"] == (0.0, 0.0, 1.0)
    assert not second.coupling.is_all_pairs() and not second.coupling.couples("coil", "sense")


@pytest.mark.parametrize("level,anchor,insertion", [
    ("the top level", '"ports":', '"typo": true, '),
    ("geometry", '"nodes":', '"typo": true, '),
    ("a node", '"x": 0.0,', '"typo": true, '),
    ("a segment", '"a": 0,', '"typo": true, '),
    ("a port", '"positive": 0,', '"typo": true, '),
    ("coupling", '"frequencies_hz":', '"coupling": { "typo": true }, '),
    ("a discretization payload", '"nw": 3,', '"typo": 1, '),
])
def test_an_unknown_key_is_rejected_by_name_at_every_level(level, anchor, insertion):
    minimal = example_text(0)
    assert minimal.count(anchor) == 1, level
    with pytest.raises((P.ProblemError, ValueError)) as e:
        P.Problem.from_json(minimal.replace(anchor, insertion + anchor))
    assert "typo" in str(e.value), (level, str(e.value))
    misspelled = minimal.replace('"positive": 0,', '"nmae": "sense", "positive": 0,')
    with pytest.raises(P.ProblemError, match="nmae"):
        P.Problem.from_json(misspelled)


def test_plane_deck_matches_the_api_built_geometry():
    """fasterhenry-cli/tests/roundtrip.rs:187-265: a trace over an
    extension-form plane reads to exactly the geometry built through the
    plane library (the plane first, then the trace's top nodes, the trace
    and its two vias landing on the snapped cell centres), so the two solve
    to the same Z bit for bit; 20 x 6 cells give 20*6*2 - 20 - 6 bars plus
    the 3 segments, and 122 nodes once the via feet snap away."""
    from fasterhenry_b200 import api as A
    from fasterhenry_b200 import plane as PL
    deck = P.parse_deck(""".units mm
.default sigma=5.8e4
Gp 0 -3 0 10 3 0 0.035 nx=20 ny=6
n1 x=1 y=0 z=0.5
n2 x=9 y=0 z=0.5
n3 x=1 y=0 z=0
n4 x=9 y=0 z=0
e1 n1 n2 w=0.2 h=0.035 nwinc=2
e2 n1 n3 w=0.2 h=0.035
e3 n2 n4 w=0.2 h=0.035
.external n1 n2
.freq fmin=1e9 fmax=1e9 ndec=1
.end
""")
    w, t, sigma = 0.2 * 1e-3, 0.035 * 1e-3, 5.8e4 / 1e-3
    api = A.Geometry()
    plane = PL.GroundPlane((0.0, -3.0e-3), (10.0e-3, 3.0e-3), 0.0, t, 20, 6, sigma)
    centres = plane.build_into(api)
    xa, xb, zt = 1.0 * 1e-3, 9.0 * 1e-3, 0.5 * 1e-3
    snap_a, snap_b = plane.attach(centres, (xa, 0.0, 0.0)), plane.attach(centres, (xb, 0.0, 0.0))
    a, b = api.add_node(A.Node(xa, 0.0, zt)), api.add_node(A.Node(xb, 0.0, zt))
    api.add_segment(A.SegmentDef(a, b, w, t, sigma))
    for top, bottom in ((a, snap_a), (b, snap_b)):
        api.add_segment(A.SegmentDef(top, bottom, w, t, sigma))
    assert deck.nodes == [(n.x, n.y, n.z) for n in api.nodes]
    assert [(s["a"], s["b"], s["width"], s["height"], s["sigma"]) for s in deck.segments] == \
        [(s.a, s.b, s.width, s.height, s.sigma) for s in api.segments]
    grids = [(1, 1)] * len(api.segments)
    grids[len(api.segments) - 3] = (2, 1)
    assert deck.discretization == {"kind": "per_segment", "grids": grids}
    assert deck.ports[0][:2] == (a, b)
    assert len(deck.segments) == 20 * 6 * 2 - 20 - 6 + 3 and len(deck.nodes) == 20 * 6 + 2


@pytest.mark.parametrize("replacement", ["+ contact rect (11, 3, 0, 2, 2, 1, 1)",
                                         "+ contact rect (11.000000000000002, 3, 0, 2, 2, 1, 1)"])
def test_a_contact_rect_touching_the_plane_edge_is_dropped_with_a_warning(replacement):
    """fasterhenry-cli/tests/roundtrip.rs:774-805: the deck reads as if the
    clause were absent, with one warning."""
    with open(os.path.join(DECKS, "plane_fasthenry.inp")) as f:
        text = f.read()
    original = "+ contact rect (5, 3, 0, 2, 2, 1, 1)"
    assert original in text.splitlines()
    baseline, none = P.parse_deck_reporting(text.replace(original + "\n", ""))
    assert none == []
    deck, warnings = P.parse_deck_reporting(text.replace(original, replacement))
    assert len(warnings) == 1 and "ignored" in warnings[0].message
    assert deck.to_json() == baseline.to_json()
