"""The deck reader pinned to the reference's own fixtures
(fasterhenry-cli/tests/data, copied byte for byte into tests/golden/decks):
the two-turn spiral as a `.inp` deck and as the equivalent JSON problem
document read to the same problem field by field
(fasterhenry-cli/tests/roundtrip.rs:18-30), and the two-port deck reads to
its stated geometry.  Host-only."""
import os

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
