"""Z(w) sweeps on the device vs the oracle's dense path.

Tolerances (relative, per Z entry): FP64 form 1e-10 against the oracle (the
reference's FP64 LU); mixed form (FP32 factors + FP64-residual refinement)
1e-9 against the oracle.
"""
import math

import numpy as np
import pytest

from conftest import load_golden
from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10
MIXED_RTOL = 1e-9


def rel_err(z, ref):
    return float(np.max(np.abs(z - ref) / np.abs(ref)))


def golden_z(name):
    g = load_golden(name)
    return g["frequencies_hz"], np.array(g["z_re"]) + 1j * np.array(g["z_im"])


@pytest.fixture(scope="module")
def c1_system(fh):
    deck, _ = F.c1_spiral()
    s = fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization)
    yield s
    s.close()


def test_c1_fp64_matches_golden(fh, c1_system):
    freqs, ref = golden_z("c1_z.json")
    z = c1_system.sweep(freqs, fh.Precision.FP64).impedance_ohm
    assert rel_err(z, ref) < FP64_RTOL


def test_c1_mixed_matches_golden(fh, c1_system):
    freqs, ref = golden_z("c1_z.json")
    r = c1_system.sweep(freqs, fh.Precision.MIXED_BF16X3)
    assert rel_err(r.impedance_ohm, ref) < MIXED_RTOL
    assert all(i >= 1 for i in r.refinement_iterations)


def test_c1_counts_and_mesh_matrices(fh, oracle, c1_system):
    deck, _ = F.c1_spiral()
    o = oracle.System(deck)
    assert c1_system.counts() == o.counts
    R, L = c1_system.mesh_matrices()
    Ro, Lo = o.blocks()
    assert np.array_equal(R, Ro)
    assert np.max(np.abs(L - Lo)) <= 1e-12 * np.max(np.abs(Lo))
    assert np.array_equal(L, L.T)


@pytest.mark.slow
def test_c2_meander_fp64_and_mixed(fh):
    deck, _ = F.c2_meander()
    freqs, ref = golden_z("c2_z.json")
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        z64 = s.sweep(freqs, fh.Precision.FP64).impedance_ohm
        rm = s.sweep(freqs, fh.Precision.MIXED_BF16X3)
    assert rel_err(z64, ref) < FP64_RTOL
    assert rel_err(rm.impedance_ohm, ref) < MIXED_RTOL
    assert all(i != -1 for i in rm.refinement_iterations), rm.refinement_iterations


def test_doc_example_bar(fh, known):
    k = known["bar_1mm_100um_20um_5x3"]
    g = fh.Geometry()
    a, b = g.add_node((0, 0, 0)), g.add_node((k["length"], 0, 0))
    g.add_segment(fh.SegmentDef(a, b, k["width"], k["height"], k["sigma"]))
    res = fh.solve(g, [fh.Port(a, b)], fh.Discretization.uniform(k["nw"], k["nh"]), k["frequencies_hz"])
    r_dc = res.resistance(0)[0, 0]
    assert abs(r_dc - k["length"] / (k["sigma"] * k["width"] * k["height"])) < 1e-9
    assert res.resistance(2)[0, 0] > r_dc
    l1 = res.inductance(1)[0, 0]
    assert 0.5e-9 < l1 < 1.5e-9
    assert res.inductance(0) is None


def test_doc_example_trace_dc(fh, known):
    k = known["trace_10mm_1mm_35um_5x2"]
    g = fh.Geometry.from_parts([(0, 0, 0), (k["length"], 0, 0)],
                               [fh.SegmentDef(0, 1, k["width"], k["height"], k["sigma"])])
    for prec in (fh.Precision.FP64, fh.Precision.MIXED_BF16X3):
        res = fh.solve(g, [fh.Port(0, 1)], fh.Discretization.uniform(5, 2), k["frequencies_hz"], prec)
        dc = res.impedance_ohm[0, 0, 0]
        want = k["length"] / (k["sigma"] * k["width"] * k["height"])
        assert abs(dc.real - want) < 1e-12 * want
        assert dc.imag == 0.0
        assert res.impedance_ohm[2, 0, 0].real > dc.real


def two_port():
    nodes = [(0, 0, 0), (2e-3, 0, 0), (0, 0.3e-3, 0), (2e-3, 0.3e-3, 0)]
    segs = [F.segment(0, 1, 0.2e-3, 35e-6), F.segment(2, 3, 0.2e-3, 35e-6)]
    return F.Deck(nodes, segs, [(0, 1), (2, 3)], F.uniform(3, 2), name="two_port")


def ring_deck():
    nodes = [(0, 0, 0), (1e-3, 0, 0), (1e-3, 1e-3, 0), (0, 1e-3, 0), (0, 2e-3, 0)]
    segs = [F.segment(0, 1, 1e-4, 2e-5), F.segment(1, 2, 1e-4, 2e-5), F.segment(2, 3, 1e-4, 2e-5),
            F.segment(3, 0, 1e-4, 2e-5), F.segment(3, 4, 1e-4, 2e-5)]
    return F.Deck(nodes, segs, [(0, 2), (4, 1)], F.uniform(2, 2), name="ring")


@pytest.mark.parametrize("make", [two_port, ring_deck,
                                  lambda: F.c4_spiral(0.5, 2.0),
                                  lambda: F.square_spiral(3, 10e-6, 5e-6, 2e-6, 200e-6, F.graded(5, 3, 2.0))])
def test_multiport_and_graded_decks_match_oracle(fh, oracle, make):
    deck = make()
    freqs = [0.0, 1e6, 1e8, 1e10]
    ref = oracle.System(deck).sweep(freqs)
    g = fh.Geometry.from_deck(deck)
    for prec, tol in ((fh.Precision.FP64, FP64_RTOL), (fh.Precision.MIXED_BF16X3, MIXED_RTOL)):
        z = fh.solve(g, deck.ports, deck.discretization, freqs, prec).impedance_ohm
        nz = np.abs(ref) > 0
        assert np.max(np.abs(z - ref)[nz] / np.abs(ref)[nz]) < tol
        assert np.all(z[0].imag == 0.0)
    if len(deck.ports) > 1:
        for zk in z[1:]:
            assert abs(zk[0, 1] - zk[1, 0]) <= 1e-9 * abs(zk[0, 1])


def test_invalid_frequency_reports_first_bad_index(fh, c1_system):
    with pytest.raises(fh.InvalidFrequency) as e:
        c1_system.sweep([1e6, -1.0, float("nan")])
    assert e.value.index == 1 and e.value.value == -1.0
    with pytest.raises(fh.InvalidFrequency):
        c1_system.sweep([float("inf")])


def test_iterative_choice_is_unsupported_not_silent(fh):
    deck, _ = F.c1_spiral()
    with pytest.raises(fh.Unsupported):
        fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization,
                               fh.SolverChoice.ITERATIVE)


def test_sweep_json_roundtrip(fh, c1_system):
    import json
    freqs, _ = golden_z("c1_z.json")
    r = c1_system.sweep(freqs[:3], fh.Precision.FP64)
    doc = json.loads(r.to_json())
    z = np.array([[[e["re"] + 1j * e["im"] for e in row] for row in m] for m in doc["impedance_ohm"]])
    assert np.array_equal(z, r.impedance_ohm)
    assert doc["provenance"]["counts"]["filaments"] == 240


@pytest.mark.parametrize("legs", [9, 18])
def test_two_level_mixed_matches_fp64(fh, legs):
    """Orders just above one and two 512-column super-panels (m = 522, 1,044):
    the two-level FP32 factorization (deep tensor-core updates, grouped
    interchanges in the forward solve) refines to the FP64 answer."""
    deck = F.meander_legs(legs)
    freqs = F.logspace(5, 10, 8)
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        assert s.counts()["internal_meshes"] == 58 * legs
        z64 = s.sweep(freqs, fh.Precision.FP64).impedance_ohm
        rm = s.sweep(freqs, fh.Precision.MIXED_BF16X3)
    assert rel_err(rm.impedance_ohm, z64) < MIXED_RTOL
    assert all(1 <= i <= 10 for i in rm.refinement_iterations), rm.refinement_iterations


def test_two_level_mixed_look_ahead(fh):
    """The 40-leg meander (m = 2,320, five super-panels) at 96 frequencies in
    one batch: the deep updates of the first two super-panels are long enough
    to be split (the next super-panel's columns first, the rest on all SMs but
    a few while the next diagonal region runs on the second stream, then a
    second grid joining from the same tile counter); the later ones run
    whole.  Every frequency refines without the FP64 fallback and Z matches
    the FP64 sweep."""
    deck = F.meander_legs(40)
    freqs = F.logspace(5, 10, 96)
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        assert s.counts()["internal_meshes"] == 2320
        z64 = s.sweep(freqs, fh.Precision.FP64).impedance_ohm
        with fh.Profiler() as prof:
            rm = s.sweep(freqs, fh.Precision.MIXED_BF16X3)
            profile = prof.read()
            ov = prof.overlap(["panel", "trsm", "gemm_tc_inner"], ["gemm_tc", "gemm_tc_shared"])
    assert rel_err(rm.impedance_ohm, z64) < MIXED_RTOL
    assert all(1 <= i <= 10 for i in rm.refinement_iterations), rm.refinement_iterations
    # four deep updates (super-panels with rows below) on all SMs, two of them
    # with a second part on the SMs the look-ahead leaves
    assert profile["gemm_tc"]["launches"] == 4, profile["gemm_tc"]
    assert profile["gemm_tc_shared"]["launches"] == 2, profile["gemm_tc_shared"]
    # the second and third diagonal regions ran while an update did
    assert 0.0 < ov["both_ms"] <= min(ov["a_ms"], ov["b_ms"]), ov


def test_two_level_mixed_odd_order(fh, oracle):
    """An odd order (m = 1,043: one segment of the 18-leg meander on a 29 x 1
    grid, 28 loops instead of 29) over three super-panels.  The FP32 system is
    bordered to the even order 1,044, so the rows-below pass and the dataflow
    solve (both need a 16-byte column stride) run as for even orders; the
    border entry of every correction stays zero and Z matches the oracle."""
    base = F.meander_legs(18)
    grids = [(10, 3)] * base.segment_count()
    grids[5] = (29, 1)
    deck = F.Deck(list(base.nodes), [dict(sg) for sg in base.segments], list(base.ports), F.per_segment(grids),
                  "meander_18_odd")
    freqs = F.logspace(5, 10, 6)
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        assert s.counts()["internal_meshes"] == 1043
        z64 = s.sweep(freqs, fh.Precision.FP64).impedance_ohm
        with fh.Profiler() as prof:
            rm = s.sweep(freqs, fh.Precision.MIXED_BF16X3)
            profile = prof.read()
    assert rel_err(rm.impedance_ohm, z64) < MIXED_RTOL
    assert all(1 <= i <= 10 for i in rm.refinement_iterations), rm.refinement_iterations
    assert profile["panel_solve"]["launches"] > 0 and profile["solve_flow"]["launches"] > 0
    assert profile["solve_barrier"]["launches"] == 0 and profile["solve"]["launches"] == 0
    ref = oracle.System(deck)
    for k in (0, len(freqs) - 1):
        assert rel_err(rm.impedance_ohm[k], ref.impedance(freqs[k])) < MIXED_RTOL


def test_two_level_mixed_strongly_coupled_loops(fh):
    """Two thick segments on a 40 x 30 grid (m = 2,398): every mesh loop of a
    segment shares the segment's first filament, so loops far apart in the
    ordering stay strongly coupled -- unlike a meander, where couplings decay
    fast with the distance between loops.  Every entry the factorization reads
    must carry all earlier updates for the refinement to converge without the
    FP64 fallback (iterations -1); this mesh is ill-conditioned enough that
    it takes 4 to 6 steps."""
    nodes = [(0.0, 0.0, 0.0), (200 * F.UM, 0.0, 0.0), (200 * F.UM, 200 * F.UM, 0.0)]
    segs = [F.segment(0, 1, 40 * F.UM, 30 * F.UM), F.segment(1, 2, 40 * F.UM, 30 * F.UM)]
    deck = F.Deck(nodes, segs, [(0, 2)], F.uniform(40, 30), "thick_bend")
    freqs = F.logspace(5, 10, 6)
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        assert s.counts()["internal_meshes"] > 2048  # at least four 512-column super-panels
        z64 = s.sweep(freqs, fh.Precision.FP64).impedance_ohm
        rm = s.sweep(freqs, fh.Precision.MIXED_BF16X3)
    assert rel_err(rm.impedance_ohm, z64) < MIXED_RTOL
    assert all(1 <= i <= 8 for i in rm.refinement_iterations), rm.refinement_iterations


def test_two_level_mixed_many_ports(fh):
    """Ten ports x 32 frequencies = 320 (matrix, right-hand side) pairs, more
    than one cooperative launch of the dataflow solve holds (two CTAs per SM
    at most), so the refinement solves with the barrier-based form.  That
    form reads U12, which the rows-below pass then writes (m = 1,044, even:
    the fused pass runs over two super-panels), while the dataflow solve
    takes U from L and leaves it unwritten."""
    base = F.meander_legs(18)
    a, b = base.ports[0]
    inner = [k for k in range(len(base.nodes)) if k not in (a, b)]
    ports = list(base.ports) + [(a, inner[i]) for i in np.linspace(2, len(inner) - 3, 9).astype(int)]
    deck = F.Deck(list(base.nodes), [dict(sg) for sg in base.segments], ports, dict(base.discretization),
                  "meander_18_ten_ports")
    freqs = F.logspace(5, 10, 32)
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        c = s.counts()
        assert c["internal_meshes"] == 1044 and c["ports"] == 10
        z64 = s.sweep(freqs, fh.Precision.FP64).impedance_ohm
        with fh.Profiler() as prof:
            rm = s.sweep(freqs, fh.Precision.MIXED_BF16X3)
            profile = prof.read()
    assert rel_err(rm.impedance_ohm, z64) < MIXED_RTOL
    assert all(1 <= i <= 10 for i in rm.refinement_iterations), rm.refinement_iterations
    # the dataflow solve did not run: the refinement solved with a form that
    # reads U12 (the barrier-based one, or the per-block one when that does not
    # fit either), so the rows-below pass wrote U12
    assert profile["solve_flow"]["launches"] == 0, profile
    assert profile["solve_barrier"]["launches"] + profile["solve"]["launches"] > 0, profile
