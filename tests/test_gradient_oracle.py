"""CPU checks of the finite-difference machinery the gradient tests rest on:
the oracle's frozen-dispatch fill is the fill at the nominal geometry bit for
bit, it is smooth across the dispatch thresholds it freezes, and the
filament tangents (how each filament moves with its segment's width and
thickness) are the derivatives of the discretization."""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F


def tangents_of(filaments, deck, per):
    out = np.zeros((len(filaments), 4))
    i = 0
    for s, count in enumerate(per):
        seg = deck.segments[s]
        a = np.array(deck.nodes[seg["a"]])
        for _ in range(count):
            f = filaments[i]
            d = f[0:3] - a
            out[i] = [d @ f[10:13] / seg["width"], d @ f[13:16] / seg["height"], f[16] / seg["width"],
                      f[17] / seg["height"]]
            i += 1
    return out


@pytest.mark.parametrize("deck", [F.c1_spiral()[0], F.cloud_deck(80, True, 4),
                                  F.square_spiral(2, 10e-6, 5e-6, 2e-6, 150e-6, F.graded(4, 2, 1.5))])
def test_frozen_fill_is_the_fill_at_nominal(oracle, deck):
    fil, _ = oracle.discretize(deck)
    assert np.array_equal(oracle.fill_frozen(fil, fil), oracle.fill(fil))
    rows = [0, len(fil) // 2, len(fil) - 1]
    assert np.array_equal(oracle.fill_frozen_rows(fil, fil, rows), oracle.fill(fil)[rows])


def test_frozen_fill_rejects_sampled_pairs(oracle):
    fil, _ = oracle.discretize(F.cloud_deck(40, False, 2))
    _, methods = oracle.fill(fil, methods=True)
    assert np.any(methods == oracle.SAMPLED_FILAMENTS)
    with pytest.raises(oracle.OracleError):
        oracle.fill_frozen(fil, fil)


@pytest.mark.parametrize("disc", [F.uniform(3, 2), F.graded(5, 3, 1.6), F.skin_depth(1e9, 0.3, 1.3, 16)])
def test_tangents_are_derivatives_of_the_discretization(oracle, disc):
    deck = F.square_spiral(2, 12e-6, 5e-6, 3e-6, 160e-6, disc)
    fil, per = oracle.discretize(deck)
    tan = tangents_of(fil, deck, per)
    for s in (0, 5):
        for which, key in ((0, "width"), (1, "height")):
            base = deck.segments[s][key]
            h = 1e-6 * base
            fp, perp = oracle.discretize(F.with_segment(deck, s, **{key: base + h}))
            fm, perm = oracle.discretize(F.with_segment(deck, s, **{key: base - h}))
            assert np.array_equal(perp, per) and np.array_equal(perm, per)
            d = (fp - fm) / (2 * h)
            first = int(np.sum(per[:s]))
            rows = np.arange(first, first + per[s])
            axis = fil[rows, 10:13] if which == 0 else fil[rows, 13:16]
            # centre (start) moves along the axis by the s tangent, the extent by the g tangent
            assert np.allclose(d[rows, 0:3], tan[rows, which][:, None] * axis, rtol=0, atol=1e-8)
            assert np.allclose(d[rows, 16 + which], tan[rows, 2 + which], rtol=0, atol=1e-8)
            others = np.setdiff1d(np.arange(len(fil)), rows)
            assert np.all(d[others] == 0.0)
