"""The impedance gradient dZ/dp (widths and thicknesses of segments) against
central finite differences of the oracle with frozen dispatch.

There is no reference implementation of the gradient, so parity is pinned
by finite differences.  The oracle evaluates the perturbed geometry with every
dispatch decision taken on the nominal one (orc_fill_frozen: method, Gauss
orders, closed-form acceptance, the aligned quadrature's break points and
panel tree).  The central difference then differentiates one smooth function,
which is what the device's forward-mode derivative fill computes.

* The derivative fill on its own (fh_test_inductance_gradient) against
  entry-wise differences of the oracle's L on a random Manhattan cloud that
  holds point-quadrature, closed-form and aligned-quadrature pairs.
* dZ/dp of small decks against differences of the oracle's whole Z (the
  stationarity of Z in the loop currents is tested with it).
* The 6-turn, skin-graded spiral at 1 GHz (3,672 filaments, 48 parameters)
  against differences of the oracle's rows of L, contracted with the branch
  currents.
Bound: |dZ_adjoint - dZ_fd| <= 1e-6 max |dZ_fd|.
"""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu

MU0_4PI = 1e-7
TOL = 1e-6


def tangents_of(filaments, deck, per):
    """(sw, sh, gw, gh) per filament: how each moves with its segment's width
    and thickness (start = node a + W c_w w + H c_h h; own width f_w w)."""
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


def moved(filaments, tangents, which, step):
    """Filaments displaced by `step` along the width (which = 0) or thickness
    (which = 1) tangent."""
    f = filaments.copy()
    s, g = tangents[:, which], tangents[:, 2 + which]
    axis = f[:, 10:13] if which == 0 else f[:, 13:16]
    shift = (s * step)[:, None] * axis
    f[:, 0:3] += shift
    f[:, 3:6] += shift
    f[:, 16 + which] += g * step
    return f


def loop_matrix(oracle, deck, per, n):
    row_ptr, cols, signs, internal = oracle.mesh(deck, per)
    M = np.zeros((len(row_ptr) - 1, n))
    for r in range(len(row_ptr) - 1):
        for k in range(row_ptr[r], row_ptr[r + 1]):
            M[r, cols[k]] += signs[k]
    return M, internal


def resistances(f):
    return f[:, 6] / (f[:, 18] * (f[:, 16] * f[:, 17]))


def schur(M, m, R, L, omega):
    Zm = M @ (np.diag(R) + 1j * omega * L) @ M.T
    ee, ep, pp = Zm[:m, :m], Zm[:m, m:], Zm[m:, m:]
    return pp - ep.T @ np.linalg.solve(ee, ep)


# ---------------------------------------------------------------------------
# The derivative fill
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("seed", [3, 11])
def test_derivative_fill_matches_frozen_differences(fh, oracle, seed):
    deck = F.cloud_deck(120, True, seed)
    fil, per = oracle.discretize(deck)
    n = len(fil)
    rng = np.random.default_rng(seed)
    tan = rng.uniform(-1.0, 1.0, (n, 4))
    tan[:, 2:] = np.abs(tan[:, 2:])
    tan[::2] = 0.0  # even filaments fixed: isolates each side of a pair
    _, methods = oracle.fill(fil, methods=True)
    counts = np.bincount(methods.ravel(), minlength=5)
    assert counts[oracle.POINT_QUADRATURE] and counts[oracle.BAR_CLOSED_FORM], counts
    Dw, Dh = fh.inductance_gradient(fil, tan)
    scale = np.min(fil[:, 16:18])
    for which, D in ((0, Dw), (1, Dh)):
        h = 1e-4 * scale
        fd = (oracle.fill_frozen(fil, moved(fil, tan, which, h)) -
              oracle.fill_frozen(fil, moved(fil, tan, which, -h))) / (2 * h)
        total = D + D.T  # both filaments of a pair move
        err = np.max(np.abs(total - fd)) / np.max(np.abs(fd))
        assert err < TOL, (which, err)
        fixed = np.arange(n) % 2 == 0
        assert np.all(D[fixed][:, :] == 0.0)


def test_derivative_fill_covers_aligned_quadrature(fh, oracle):
    # Long, thin filaments side by side in one bundle: their closed form is
    # rejected (cancellation) and the aligned quadrature takes over.
    deck = F.Deck([(0, 0, 0), (2e-3, 0, 0)], [F.segment(0, 1, 20e-6, 4e-6)], [(0, 1)], F.graded(5, 3, 1.7), "bundle")
    fil, per = oracle.discretize(deck)
    _, methods = oracle.fill(fil, methods=True)
    assert np.any(methods == oracle.ALIGNED_QUADRATURE)
    tan = tangents_of(fil, deck, per)
    Dw, Dh = fh.inductance_gradient(fil, tan)
    for which, D in ((0, Dw), (1, Dh)):
        h = 1e-4 * deck.segments[0]["width" if which == 0 else "height"]
        fd = (oracle.fill_frozen(fil, moved(fil, tan, which, h)) -
              oracle.fill_frozen(fil, moved(fil, tan, which, -h))) / (2 * h)
        err = np.max(np.abs(D + D.T - fd)) / np.max(np.abs(fd))
        assert err < TOL, (which, err)


# ---------------------------------------------------------------------------
# dZ/dp of whole systems
# ---------------------------------------------------------------------------
def fd_gradient(oracle, deck, params, frequency, rel):
    """Central differences of the oracle's Z (frozen dispatch) per parameter."""
    fil0, per0 = oracle.discretize(deck)
    M, m = loop_matrix(oracle, deck, per0, len(fil0))
    omega = 2 * np.pi * frequency
    out = []
    for p in params:
        key = "width" if p.kind == "width" else "height"
        base = deck.segments[p.index][key]
        h = rel * base
        z = []
        for sgn in (1, -1):
            d = F.with_segment(deck, p.index, **{key: base + sgn * h})
            fil, per = oracle.discretize(d)
            assert np.array_equal(per, per0)
            L = oracle.fill_frozen(fil0, fil)
            z.append(schur(M, m, resistances(fil), L, omega))
        out.append((z[0] - z[1]) / (2 * h))
    return np.array(out)


@pytest.mark.parametrize("frequency", [1e6, 1e9])
def test_small_spiral_gradient_matches_differences_of_z(fh, oracle, frequency):
    deck = F.square_spiral(2, 10e-6, 5e-6, 2e-6, 150e-6, F.graded(4, 2, 1.5))
    geometry = fh.Geometry.from_deck(deck)
    params = [fh.Param(k, s) for k in ("width", "thickness") for s in range(len(deck.segments))]
    with fh.MeshSystem.assemble(geometry, deck.ports, deck.discretization) as system:
        g = system.gradient(frequency, params)
        z = system.impedance(frequency)
    assert np.allclose(g.impedance_ohm, z, rtol=1e-12, atol=0)
    fd = fd_gradient(oracle, deck, params, frequency, 1e-4)
    err = np.max(np.abs(g.gradient - fd)) / np.max(np.abs(fd))
    assert err < TOL, err
    if frequency < 1e7:  # near DC, wider or thicker conductors lower the resistance
        assert np.all(g.resistance_gradient[:, 0, 0] < 0)


def test_two_port_gradient_is_symmetric_and_matches_differences(fh, oracle):
    deck = F.meander_legs(4, nw=3, nh=2)
    nodes = deck.nodes
    deck = F.Deck(nodes, deck.segments, [(0, len(nodes) // 2), (len(nodes) // 2, len(nodes) - 1)],
                  deck.discretization, "two_port")
    params = [fh.Param("width", 0), fh.Param("thickness", 3), fh.Param("width", 6)]
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as system:
        g = system.gradient(1e8, params)
    assert np.array_equal(g.gradient[:, 0, 1], g.gradient[:, 1, 0])
    fd = fd_gradient(oracle, deck, params, 1e8, 1e-4)
    err = np.max(np.abs(g.gradient - fd)) / np.max(np.abs(fd))
    assert err < TOL, err


def test_dc_gradient_of_a_bar_is_the_resistance_derivative(fh):
    length, w, t, sigma = 1e-3, 20e-6, 5e-6, F.COPPER
    deck = F.Deck([(0, 0, 0), (length, 0, 0)], [F.segment(0, 1, w, t)], [(0, 1)], F.uniform(4, 3), "bar")
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as system:
        g = system.gradient(0.0)
    r = length / (sigma * w * t)
    assert abs(g.impedance_ohm[0, 0].real - r) <= 1e-12 * r
    dw, dt = g.gradient[0, 0, 0], g.gradient[1, 0, 0]
    assert abs(dw.real + r / w) <= 1e-10 * r / w and dw.imag == 0.0
    assert abs(dt.real + r / t) <= 1e-10 * r / t and dt.imag == 0.0


def test_c4_spiral_gradient_matches_differences_of_the_rows(fh, oracle):
    deck = F.c4_spiral()
    frequency = 1e9
    omega = 2 * np.pi * frequency
    geometry = fh.Geometry.from_deck(deck)
    with fh.MeshSystem.assemble(geometry, deck.ports, deck.discretization) as system:
        g = system.gradient(frequency)
        assert system.counts()["filaments"] == 3672
        R_m, L_m = system.mesh_matrices()
        m = system.counts()["internal_meshes"]
    assert g.gradient.shape == (48, 1, 1) and np.all(np.isfinite(g.gradient))
    assert g.report["pairs"] == 3672 * 3673 // 2
    fil0, per0 = oracle.discretize(deck)
    n = len(fil0)
    M, m2 = loop_matrix(oracle, deck, per0, n)
    assert m2 == m
    Zm = R_m + 1j * omega * L_m
    x = np.linalg.solve(Zm[:m, :m], Zm[:m, m:])
    Ib = M.T @ np.concatenate([-x, np.eye(Zm.shape[0] - m)])[:, 0]
    first = np.concatenate([[0], np.cumsum(per0)])
    checked = [(0, "width"), (0, "thickness"), (13, "width"), (23, "thickness")]
    for s, kind in checked:
        key = "width" if kind == "width" else "height"
        base = deck.segments[s][key]
        h = 1e-4 * base
        rows = np.arange(first[s], first[s + 1])
        dL, dR = 0.0, 0.0
        for sgn in (1, -1):
            fil, per = oracle.discretize(F.with_segment(deck, s, **{key: base + sgn * h}))
            assert np.array_equal(per, per0)
            Lr = oracle.fill_frozen_rows(fil0, fil, rows)
            dL = dL + sgn * Lr
            dR = dR + sgn * resistances(fil)[rows]
        Ir = Ib[rows]
        lpart = 2 * Ir @ (dL @ Ib) - Ir @ dL[:, rows] @ Ir
        fd = (1j * omega * lpart + np.sum(Ir * Ir * dR)) / (2 * h)
        k = s + (24 if kind == "thickness" else 0)
        adj = g.gradient[k, 0, 0]
        assert abs(adj - fd) <= TOL * abs(fd), (s, kind, adj, fd)


def test_gradient_argument_errors(fh):
    deck = F.square_spiral(2, 10e-6, 5e-6, 2e-6, 150e-6, F.uniform(2, 1))
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as system:
        with pytest.raises(fh.Unsupported):
            system.gradient(1e9, [fh.Param("z", 1)])
        with pytest.raises(fh.InvalidArgument):
            system.gradient(1e9, [fh.Param("width", 99)])
        with pytest.raises(fh.InvalidFrequency):
            system.gradient(-1.0, [fh.Param("width", 0)])
