"""GMRES and the matrix-free IterativeSystem.

* The device GMRES against direct solutions on dense complex systems, with
  the cases of the reference's own solver tests (fasterhenry/src/gmres.rs
  tests): convergence to the direct solution, real systems staying real, a
  full Krylov space in at most n steps, an exact preconditioner in one step,
  a zero right-hand side without a product, and the iteration cap.
* IterativeSystem against the dense path (oracle golden Z) within the
  reference's 1e-4 bound (fasterhenry/tests/solve.rs:775), the DC limit with
  an exactly real Z, reciprocity, and NotConverged reporting.
"""
import numpy as np
import pytest

from conftest import load_golden
from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu


def complex_symmetric(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a = 0.5 * (a + a.T)
    return a + n * np.eye(n)


def test_complex_symmetric_system_converges_to_the_direct_solution(fh):
    a = complex_symmetric(40, 1)
    b = np.random.default_rng(2).standard_normal(40) + 1j * np.random.default_rng(3).standard_normal(40)
    x, oc = fh.gmres_dense(a, b)
    assert oc.converged and oc.relative_residual <= 1e-10, oc
    direct = np.linalg.solve(a, b)
    assert np.linalg.norm(x - direct) / np.linalg.norm(direct) < 1e-9


def test_real_system_stays_real_and_matches_the_direct_solution(fh):
    rng = np.random.default_rng(4)
    a = rng.standard_normal((30, 30)) + 30 * np.eye(30)
    b = rng.standard_normal(30)
    x, oc = fh.gmres_dense(a.astype(complex), b.astype(complex))
    assert oc.converged
    assert np.all(x.imag == 0.0)
    direct = np.linalg.solve(a, b)
    assert np.linalg.norm(x.real - direct) < 1e-9 * np.linalg.norm(direct)


def test_full_krylov_space_solves_exactly_in_n_steps(fh):
    n = 12
    rng = np.random.default_rng(5)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal(n) + 0j
    x, oc = fh.gmres_dense(a, b, params=fh.GmresParams(tolerance=1e-10, restart=n, max_iterations=5 * n))
    assert oc.converged and oc.iterations <= n, oc


def test_exact_preconditioner_converges_in_one_iteration(fh):
    a = complex_symmetric(25, 6)
    b = np.ones(25, dtype=complex)
    x, oc = fh.gmres_dense(a, b, precondition=np.linalg.inv(a))
    assert oc.converged and oc.iterations == 1, oc


def test_zero_right_hand_side_is_solved_without_a_product(fh):
    a = complex_symmetric(10, 7)
    x, oc = fh.gmres_dense(a, np.zeros(10, dtype=complex), x0=np.ones(10, dtype=complex))
    assert oc.iterations == 0 and oc.converged
    assert np.all(x == 0)


def test_iteration_cap_reports_non_convergence(fh):
    rng = np.random.default_rng(8)
    a = rng.standard_normal((50, 50)) + 1j * rng.standard_normal((50, 50)) + 2 * np.eye(50)
    b = rng.standard_normal(50) + 0j
    x, oc = fh.gmres_dense(a, b, params=fh.GmresParams(tolerance=1e-14, restart=10, max_iterations=3))
    assert not oc.converged and oc.iterations == 3 and oc.relative_residual < 1.0, oc


# ---------------------------------------------------------------------------
# IterativeSystem vs the dense path
# ---------------------------------------------------------------------------
def golden_z(name):
    g = load_golden(name)
    return g["frequencies_hz"], np.array(g["z_re"]) + 1j * np.array(g["z_im"])


@pytest.fixture(scope="module")
def c1_iterative(fh):
    deck, _ = F.c1_spiral()
    with fh.IterativeSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        yield s


def test_c1_iterative_matches_the_dense_golden(fh, c1_iterative):
    freqs, ref = golden_z("c1_z.json")
    z = c1_iterative.sweep(freqs).impedance_ohm
    rel = np.max(np.abs(z - ref) / np.abs(ref))
    assert rel < 1e-4, rel
    assert all(o.converged for row in c1_iterative.last_outcomes for o in row)
    st = c1_iterative.operator_stats()
    assert st["filaments"] == 240 and st["near_entries"] > 0


def test_dc_limit_is_real_and_matches_the_dense_resistance(fh, c1_iterative):
    deck, _ = F.c1_spiral()
    z_it = c1_iterative.impedance(0.0)
    assert np.all(z_it.imag == 0.0)
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as s:
        z_dense = s.impedance(0.0)
    assert abs(z_it[0, 0].real - z_dense[0, 0].real) <= 1e-8 * abs(z_dense[0, 0].real)


def test_two_ports_are_reciprocal_and_match_the_dense_path(fh, oracle):
    deck = F.meander_legs(6, nw=3, nh=2)
    nodes = deck.nodes
    ports = [(0, len(nodes) // 2), (len(nodes) // 2, len(nodes) - 1)]
    freqs = [1e7, 1e9]
    with fh.IterativeSystem.assemble(fh.Geometry.from_deck(deck), ports, deck.discretization) as s:
        z = s.sweep(freqs).impedance_ohm
        counts = s.counts()
    assert counts["ports"] == 2
    assert np.array_equal(z[:, 0, 1], z[:, 1, 0])
    o = oracle.System(F.Deck(nodes, deck.segments, ports, deck.discretization))
    ref = o.sweep(freqs)
    assert np.max(np.abs(z - ref)) / np.max(np.abs(ref)) < 1e-4


def test_not_converged_names_the_port_and_frequency(fh):
    deck, _ = F.c1_spiral()
    params = fh.IterativeParams(gmres=fh.GmresParams(tolerance=1e-14, restart=2, max_iterations=2))
    with fh.IterativeSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization, params) as s:
        with pytest.raises(fh.NotConverged) as e:
            s.impedance(1e9)
    assert e.value.info.index_a == 0 and e.value.info.frequency == 1e9
    assert e.value.info.iterations == 2


def test_solve_dispatches_on_the_solver_choice(fh):
    deck, freqs = F.c1_spiral()
    geometry = fh.Geometry.from_deck(deck)
    dense = fh.solve(geometry, deck.ports, deck.discretization, freqs[:2])
    it = fh.solve(geometry, deck.ports, deck.discretization, freqs[:2], solver=fh.SolverChoice.ITERATIVE)
    assert np.max(np.abs(it.impedance_ohm - dense.impedance_ohm) / np.abs(dense.impedance_ohm)) < 1e-4
    assert fh.SolverChoice.AUTO.resolve(240) == "dense"
    assert fh.SolverChoice.AUTO.resolve(20000) == "iterative"


def test_meander_over_a_ground_plane_matches_the_dense_path(fh):
    """A meander over a holed ground plane (the plane carries only induced
    currents): the matrix-free Z within the reference's 1e-4 of the dense FP64
    Z, with the grid convolution in FP64 and in FP32."""
    deck = F.meander_over_plane(12, plane_side=1.0e-3, cells=16, hole_side=0.2e-3)
    g = fh.Geometry.from_deck(deck)
    with fh.MeshSystem.assemble(g, deck.ports, deck.discretization) as d:
        z_dense = d.impedance(1e9)
    for fp32 in (False, True):
        params = fh.IterativeParams(pfft=fh.PfftParams(near_field_radius=8.0, interpolation_order=2, fft_fp32=fp32),
                                    gmres=fh.GmresParams(tolerance=1e-8))
        with fh.IterativeSystem.assemble(g, deck.ports, deck.discretization, params) as s:
            z_it = s.impedance(1e9)
        assert np.max(np.abs(z_it - z_dense) / np.abs(z_dense)) < 1e-4
    # the plane's eddy currents lower the meander's inductance
    bare = F.scaling_meander(12)
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(bare), bare.ports, bare.discretization) as d:
        z_bare = d.impedance(1e9)
    assert z_dense[0, 0].imag < z_bare[0, 0].imag
