"""Filament currents, densities, powers and the power balance
(MeshSystem::currents, solve.rs:845-868; currents.rs) against the oracle's
numpy restatement, plus the identities the reference's own tests use:
Kirchhoff along a series chain, the DC split by conductance, linearity in
the excitation, and a power balance at the LU's rounding (currents.rs:34-41:
"<~ 1e-9 on the validation fixtures")."""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("precision", ["FP64", "MIXED_BF16X3"])
def test_c1_currents_match_the_oracle(fh, oracle, precision):
    deck, freqs = F.c1_spiral()
    freqs = [0.0, freqs[3], freqs[-1]]
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        sols = s.currents(freqs, precision=getattr(fh.Precision, precision))
    for f, sol in zip(freqs, sols):
        ref = oracle.currents(deck, f, [1.0])
        assert rel(sol.current, ref["current"]) < 1e-10
        assert rel(sol.current_density, ref["density"]) < 1e-10
        assert rel(sol.power_w, ref["power"]) < 1e-10
        assert rel(sol.segment_current, ref["segment_current"]) < 1e-10
        assert rel(sol.segment_power_w, ref["segment_power"]) < 1e-10
        assert np.array_equal(sol.conductor_of_segment, ref["conductor_of_segment"])
        assert np.allclose(sol.peak_current_density, ref["peak_density"], rtol=1e-10, atol=0)
        bal = sol.power_balance
        assert abs(bal["input_w"] - ref["balance"]["input_w"]) <= 1e-10 * ref["balance"]["input_w"]
        assert bal["relative_residual"] < 1e-9, bal
        # a series chain: every segment carries the port current
        assert np.max(np.abs(np.abs(sol.segment_current) - 1.0)) < 1e-9


def test_two_ports_excitation_is_linear_and_matches_the_oracle(fh, oracle):
    base = F.meander_legs(4, nw=3, nh=2)
    nodes = base.nodes
    deck = F.Deck(nodes, base.segments, [(0, len(nodes) // 2), (len(nodes) // 2, len(nodes) - 1)],
                  base.discretization, "two_port")
    e1, e2 = np.array([1.0, 0.0]), np.array([0.0, 1.0])
    mix = np.array([0.3 - 0.2j, -1.5 + 0.7j])
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        a = s.currents(1e8, e1)
        b = s.currents(1e8, e2)
        c = s.currents(1e8, mix)
        z = s.impedance(1e8)
    assert rel(c.current, mix[0] * a.current + mix[1] * b.current) < 1e-12
    ref = oracle.currents(deck, 1e8, mix)
    assert rel(c.current, ref["current"]) < 1e-10
    assert np.array_equal(c.peak_filament, ref["peak_filament"])
    # input power is 1/2 Re(I^H Z I)
    assert abs(c.power_balance["input_w"] - 0.5 * np.real(np.conj(mix) @ z @ mix)) <= 1e-12 * c.power_balance["input_w"]
    assert c.power_balance["relative_residual"] < 1e-9


def test_dc_currents_split_by_conductance(fh):
    # A single bar, graded 5 x 3: at DC the filaments are in parallel and the
    # current divides in proportion to their areas (all share sigma and length).
    deck = F.Deck([(0, 0, 0), (1e-3, 0, 0)], [F.segment(0, 1, 30e-6, 6e-6)], [(0, 1)], F.graded(5, 3, 1.5), "bar")
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        sol = s.currents(0.0)
        fil = s.filaments()
    area = fil[:, 16] * fil[:, 17]
    assert np.allclose(sol.current.real, area / area.sum(), rtol=1e-12, atol=0)
    assert np.all(sol.current.imag == 0.0)
    assert np.allclose(sol.current_density, 1.0 / area.sum(), rtol=1e-12)


def test_batched_frequencies_equal_single_calls(fh):
    deck, freqs = F.c1_spiral()
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        many = s.currents(freqs)
        one = [s.currents(f) for f in freqs[::3]]
    for sol, single in zip(many[::3], one):
        assert rel(sol.current, single.current) < 1e-13


def test_csv_and_json_follow_the_cli(fh):
    deck, _ = F.c1_spiral()
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        sol = s.currents(1e9)
    rows = sol.csv_rows()
    assert fh.CURRENTS_CSV_HEADER.split(",")[0] == "frequency_hz" and len(fh.CURRENTS_CSV_HEADER.split(",")) == 12
    assert len(rows) == 240 and rows[0].startswith("1e9,0,0,0,")
    block = sol.json_block()
    assert set(block) == {"frequency_hz", "power_balance", "conductors", "segments"}
    assert len(block["segments"]) == 16 and len(block["conductors"]) == 1


def test_currents_argument_errors(fh):
    deck, _ = F.c1_spiral()
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        with pytest.raises(fh.InvalidExcitation) as e:
            s.currents(1e9, [1.0, 0.0])
        assert e.value.expected == 1 and e.value.got == 2
        with pytest.raises(fh.InvalidExcitation):
            s.currents(1e9, [complex(np.nan, 0)])
        with pytest.raises(fh.InvalidFrequency):
            s.currents([1e6, -1.0])
