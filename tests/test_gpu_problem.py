"""Problems read through the front end (a `.inp` deck, the JSON document)
solve to the same Z as the same geometry built in code, and a deck's
coupling groups reach the truncated assembly."""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu


def spiral_deck_text(deck, freqs_line):
    lines = ["* C1 spiral as a deck", ".units um", ".default sigma=58 nwinc=5 nhinc=3"]
    for i, (x, y, z) in enumerate(deck.nodes):
        lines.append("N%d x=%r y=%r z=%r" % (i, x * 1e6, y * 1e6, z * 1e6))
    for k, s in enumerate(deck.segments):
        lines.append("E%d N%d N%d w=%r h=%r" % (k, s["a"], s["b"], s["width"] * 1e6, s["height"] * 1e6))
    a, b = deck.ports[0]
    lines += [".external N%d N%d spiral" % (a, b), freqs_line, ".end"]
    return "\n".join(lines) + "\n"


def test_deck_and_document_solve_like_the_code_built_geometry(fh):
    deck, freqs = F.c1_spiral()
    text = spiral_deck_text(deck, ".freq fmin=1e6 fmax=1e10 ndec=2.25")
    prob = fh.parse_deck(text)
    assert len(prob.frequencies_hz) == 10
    assert np.allclose(prob.frequencies_hz, freqs, rtol=1e-14, atol=0)
    res, warnings = fh.run(prob, fh.Precision.FP64, fh.SolverChoice.DENSE)
    assert warnings == [] and res.ports[0].name == "spiral"
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        ref = s.sweep(prob.frequencies_hz).impedance_ohm
    assert np.max(np.abs(res.impedance_ohm - ref) / np.abs(ref)) < 1e-12
    doc = fh.Problem.from_json(prob.to_json())
    res2, _ = fh.run(doc, fh.Precision.FP64, fh.SolverChoice.DENSE)
    assert np.array_equal(res2.impedance_ohm, res.impedance_ohm)


def test_deck_coupling_groups_truncate(fh):
    deck, groups = F.two_islands(0.5 * F.ISLAND_EXTENT)
    lines = [".units m", ".default sigma=5.8e7 nwinc=2 nhinc=1"]
    for i, (x, y, z) in enumerate(deck.nodes):
        lines.append("N%d x=%r y=%r z=%r" % (i, x, y, z))
    for k, s in enumerate(deck.segments):
        lines.append("E%d N%d N%d w=%r h=%r group=%s" % (k, s["a"], s["b"], s["width"], s["height"], groups[k]))
    for a, b in deck.ports:
        lines.append(".external N%d N%d" % (a, b))
    lines += [".couples a", ".freq fmin=1e9 fmax=1e9 ndec=1", ".end"]
    prob = fh.parse_deck("\n".join(lines))
    res, warnings = fh.run(prob, fh.Precision.FP64, fh.SolverChoice.DENSE)
    assert len(warnings) == 1 and "truncated" in warnings[0]
    z = res.impedance_ohm[0]
    assert z[0, 1] == 0 and z[1, 0] == 0
