"""The reference's deck fixtures (tests/golden/decks, copied from
fasterhenry-cli/tests/data) solved on the GPU: the spiral read from the `.inp`
deck and from the JSON document give bit-identical sweeps
(fasterhenry-cli/tests/roundtrip.rs:18-40), both within 1e-10 of the oracle,
with the physical checks of roundtrip.rs:42-62; the two-bar deck's 2 x 2 Z
against the oracle."""
import os

import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F
from fasterhenry_b200 import problem as P

pytestmark = pytest.mark.gpu

DECKS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "decks")


def load(name):
    return P.load(os.path.join(DECKS, name))


def oracle_sweep(oracle, prob, freqs):
    deck = F.Deck(list(prob.nodes), [dict(s) for s in prob.segments], [(a, b) for a, b, _ in prob.ports],
                  dict(prob.discretization))
    s = oracle.System(deck)
    return np.array([s.impedance(f) for f in freqs])


def test_spiral_deck_and_document_solve_bit_identically(fh, oracle):
    a, b = load("spiral.inp"), load("spiral.json")
    za, _ = fh.run(a, fh.Precision.FP64, fh.SolverChoice.DENSE)
    zb, _ = fh.run(b, fh.Precision.FP64, fh.SolverChoice.DENSE)
    assert np.array_equal(za.impedance_ohm, zb.impedance_ohm)
    assert za.ports[0].name == "spiral"
    ref = oracle_sweep(oracle, a, a.frequencies_hz)
    assert np.max(np.abs(za.impedance_ohm - ref) / np.abs(ref)) < 1e-10
    # physical checks of the reference's round-trip test
    dc, _ = fh.run(a, fh.Precision.FP64, fh.SolverChoice.DENSE, frequencies=[0.0])
    z_dc = dc.impedance_ohm[0, 0, 0]
    assert z_dc.imag == 0.0 and z_dc.real > 0.0
    rf = za.impedance_ohm[3, 0, 0]
    inductance = rf.imag / (2 * np.pi * a.frequencies_hz[3])
    assert 5e-9 <= inductance <= 200e-9
    assert rf.real > z_dc.real
    # the mixed form agrees with the FP64 form
    zm, _ = fh.run(a, fh.Precision.MIXED_BF16X3, fh.SolverChoice.DENSE)
    assert np.max(np.abs(zm.impedance_ohm - za.impedance_ohm) / np.abs(za.impedance_ohm)) < 1e-9


def test_twobar_deck_matches_the_oracle(fh, oracle):
    p = load("twobar.inp")
    res, _ = fh.run(p, fh.Precision.FP64, fh.SolverChoice.DENSE)
    z = res.impedance_ohm
    assert z.shape == (4, 2, 2)
    assert [q.name for q in res.ports] == ["barA", "barB"]
    ref = oracle_sweep(oracle, p, p.frequencies_hz)
    assert np.max(np.abs(z - ref)) / np.max(np.abs(ref)) < 1e-10
    assert np.max(np.abs(z[:, 0, 1] - z[:, 1, 0]) / np.abs(z[:, 0, 1])) < 1e-12
    assert np.all(z[:, 0, 1].imag > 0)  # positive mutual inductance of parallel bars


@pytest.mark.parametrize("a,b", [("plane_fasthenry.inp", "plane_extension.inp"),
                                 ("plane_decay_rect.inp", "plane_decay_extension.inp")])
def test_plane_deck_pairs_solve_bit_identically_and_match_the_oracle(fh, oracle, a, b):
    """fasterhenry-cli/tests/roundtrip.rs:384-480: the two G grammars of one
    plane give identical sweeps; both within 1e-10 of the oracle's dense Z."""
    pa, pb = load(a), load(b)
    za, _ = fh.run(pa, fh.Precision.FP64, fh.SolverChoice.DENSE)
    zb, _ = fh.run(pb, fh.Precision.FP64, fh.SolverChoice.DENSE)
    assert np.array_equal(za.impedance_ohm, zb.impedance_ohm)
    ref = oracle_sweep(oracle, pa, pa.frequencies_hz)
    assert np.max(np.abs(za.impedance_ohm - ref) / np.abs(ref)) < 1e-10
    # the via pair over the plane: resistive and inductive, inductance falling
    # as the plane's eddy currents take over
    z = za.impedance_ohm[:, 0, 0]
    assert np.all(z.real > 0) and np.all(z.imag > 0)


CLAUSE_DECK = """.units mm
.default sigma=5.8e4
Gp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=6 z3=0
+ thick=0.035 %s
Nt x=5 y=3 z=0.5
Nb x=5 y=3 z=0.2
Ev Nt Nb w=0.2 h=0.2
.equiv Nb Npad
.external Nt Nb
.freq fmin=1e6 fmax=1e9 ndec=1
.end
"""


def test_plane_contact_clauses_solve_like_their_spelled_out_forms_and_match_the_oracle(fh, oracle):
    """A `contact connection` deck and the same deck with its equiv_rect and
    decay_rect written out give bit-identical sweeps, within 1e-10 of the
    oracle's dense Z; so does a meshed initial grid refined under a trace,
    the via landing on a named contact area."""
    short = P.parse_deck(CLAUSE_DECK % "seg1=5 seg2=3\n+ contact connection Npad (5, 3, 0, 2, 2, 4)")
    spelled = P.parse_deck(CLAUSE_DECK % ("seg1=5 seg2=3\n+ contact equiv_rect Npad (5, 3, 0, 2, 2)\n"
                                          "+ contact decay_rect (5, 3, 0, 2, 2, 0.5, 0.5, -1, -1)"))
    za, _ = fh.run(short, fh.Precision.FP64, fh.SolverChoice.DENSE)
    zb, _ = fh.run(spelled, fh.Precision.FP64, fh.SolverChoice.DENSE)
    assert np.array_equal(za.impedance_ohm, zb.impedance_ohm)
    ref = oracle_sweep(oracle, short, short.frequencies_hz)
    assert np.max(np.abs(za.impedance_ohm - ref) / np.abs(ref)) < 1e-10
    meshed = P.parse_deck(CLAUSE_DECK % ("contact initial_mesh_grid (5, 3)\n"
                                         "+ contact trace (2, 1, 0, 8, 1, 0, 0.4, 1)\n"
                                         "+ contact equiv_rect Npad (5, 3, 0, 1, 1)"))
    zm, _ = fh.run(meshed, fh.Precision.FP64, fh.SolverChoice.DENSE)
    ref = oracle_sweep(oracle, meshed, meshed.frequencies_hz)
    assert np.max(np.abs(zm.impedance_ohm - ref) / np.abs(ref)) < 1e-10
    z = zm.impedance_ohm[:, 0, 0]
    assert np.all(z.real > 0) and np.all(z.imag > 0)
