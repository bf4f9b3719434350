"""Filament currents on the matrix-free path (IterativeSystem::currents,
iterative.rs:316-377): one GMRES solve Z_ee x = Z_ep I_p per frequency on the
pFFT operator, then the dense path's branch currents, densities, powers and
peaks.

The cases follow the reference's own currents tests (fasterhenry/tests/
currents.rs): a bar at DC carries a uniform |J| = I/A on both paths
(currents.rs:60-86); on a ring the two paths agree to 1e-5 and the
iterative power balance holds to 1e-7 at 0, 1e5 and 1e8 Hz
(currents.rs:111-133); with no internal loops the filament currents are the
port currents to 1e-12 (currents.rs:136-164); bad inputs are rejected
(currents.rs:166-189).  Beyond those, a spiral against the oracle's
currents, with the FP32 convolution too, and batched frequencies equal to
single calls."""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu

COPPER = 5.8e7


def max_diff(a, b):
    """currents.rs:45-56: the largest filament-current difference over the
    largest filament current of the first solution."""
    return np.max(np.abs(a.current - b.current)) / np.max(np.abs(a.current))


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def bar(length, width, height, disc):
    return F.Deck([(0, 0, 0), (length, 0, 0)], [F.segment(0, 1, width, height)], [(0, 1)], disc, "bar")


def ring(disc):
    s = 5e-3
    nodes = [(0, 0, 0), (s, 0, 0), (s, s, 0), (0, s, 0)]
    segs = [F.segment(i, (i + 1) % 4, 1e-3, 0.5e-3) for i in range(4)]
    return F.Deck(nodes, segs, [(0, 1)], disc, "ring")


def both(fh, deck, params=None):
    g = fh.Geometry.from_deck(deck)
    dense = fh.MeshSystem.assemble(g, deck.ports, deck.discretization)
    it = fh.IterativeSystem.assemble(g, deck.ports, deck.discretization, params)
    return dense, it


def test_bar_at_dc_has_uniform_density_on_both_paths(fh):
    deck = bar(10e-3, 1e-3, 35e-6, F.uniform(5, 3))
    area = 1e-3 * 35e-6
    dense, it = both(fh, deck)
    with dense, it:
        for sol in (dense.currents(0.0, [2.0]), it.currents(0.0, [2.0])):
            assert len(sol.current) == 15
            assert np.max(np.abs(sol.current_density - 2.0 / area)) < 1e-6 * 2.0 / area
            assert np.max(np.abs(sol.current.imag)) < 1e-12
            assert abs(sol.segment_current[0] - 2.0) < 1e-9
            assert len(sol.peak_filament) == 1
            assert abs(sol.peak_current_density[0] - 2.0 / area) < 1e-6 * 2.0 / area
            r = 10e-3 / (COPPER * area)
            assert abs(sol.power_balance["dissipated_w"] - 0.5 * 4.0 * r) < 1e-9 * r
            assert sol.power_balance["relative_residual"] < 1e-9
        assert it.last_outcomes[0][0].converged


@pytest.mark.parametrize("fft_fp32", [False, True])
def test_ring_paths_agree_and_balance_power(fh, fft_fp32):
    deck = ring(F.uniform(3, 2))
    params = fh.IterativeParams(pfft=fh.PfftParams(fft_fp32=fft_fp32))
    dense, it = both(fh, deck, params)
    with dense, it:
        for f in (0.0, 1e5, 1e8):
            a = dense.currents(f)
            b = it.currents(f)
            assert a.power_balance["relative_residual"] < 1e-9, f
            assert b.power_balance["relative_residual"] < 1e-7, (f, b.power_balance)
            assert max_diff(a, b) < 1e-5, (f, max_diff(a, b))
            # Kirchhoff: the direct path and the way round carry the port current.
            assert abs(b.segment_current[0] - b.segment_current[1] - 1.0) < 1e-6
            assert len(b.segment_current) == 4 and len(b.peak_filament) == 1


def test_no_internal_loops_gives_the_port_currents(fh):
    nodes = [(i * 1e-3, 0, 0) for i in range(4)]
    segs = [F.segment(0, 1, 1e-4, 1e-4), F.segment(2, 3, 1e-4, 1e-4)]
    deck = F.Deck(nodes, segs, [(0, 1), (2, 3)], F.uniform(1, 1), "two_bars")
    ex = [1.0, 0.5j]
    dense, it = both(fh, deck)
    with dense, it:
        a = dense.currents(1e6, ex)
        b = it.currents(1e6, ex)
    assert abs(b.current[0] - ex[0]) < 1e-12 and abs(b.current[1] - ex[1]) < 1e-12
    assert len(b.peak_filament) == 2
    assert b.power_balance["relative_residual"] < 1e-9
    assert max_diff(a, b) < 1e-12


def test_bad_inputs_are_rejected(fh):
    deck = bar(1e-3, 1e-4, 1e-4, F.uniform(1, 1))
    g = fh.Geometry.from_deck(deck)
    with fh.IterativeSystem.assemble(g, deck.ports, deck.discretization) as it:
        with pytest.raises(fh.InvalidExcitation):
            it.currents(0.0, [])
        with pytest.raises(fh.InvalidFrequency):
            it.currents(-1.0)
        with pytest.raises(fh.InvalidExcitation):
            it.currents(0.0, [complex(np.nan, 0.0)])


@pytest.mark.parametrize("fft_fp32", [False, True])
def test_spiral_currents_match_the_oracle(fh, oracle, fft_fp32):
    """The C1 spiral at three frequencies: filament currents, densities,
    powers and segment sums within the reference's iterative-vs-dense bound
    for currents (1e-5), the layout identical to the oracle's."""
    deck, freqs = F.c1_spiral()
    picks = [0.0, freqs[3], freqs[-1]]
    params = fh.IterativeParams(pfft=fh.PfftParams(fft_fp32=fft_fp32))
    with fh.IterativeSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization, params) as it:
        sols = it.currents(picks)
        outcomes = it.last_outcomes
    assert len(outcomes) == 3 and all(o[0].converged for o in outcomes)
    for f, sol in zip(picks, sols):
        ref = oracle.currents(deck, f, [1.0])
        assert rel(sol.current, ref["current"]) < 1e-5, f
        assert rel(sol.current_density, ref["density"]) < 1e-5, f
        assert rel(sol.power_w, ref["power"]) < 1e-5, f
        assert rel(sol.segment_current, ref["segment_current"]) < 1e-5, f
        assert np.array_equal(sol.conductor_of_segment, ref["conductor_of_segment"])
        assert np.allclose(sol.peak_current_density, ref["peak_density"], rtol=1e-5, atol=0)
        assert sol.power_balance["relative_residual"] < 1e-7, (f, sol.power_balance)


def test_batched_frequencies_equal_single_calls(fh):
    deck, freqs = F.c1_spiral()
    with fh.IterativeSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as it:
        many = it.currents(freqs[::4])
        one = [it.currents(f) for f in freqs[::4]]
    for a, b in zip(many, one):
        assert np.array_equal(a.current, b.current)
