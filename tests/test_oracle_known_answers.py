"""Pins the CPU oracle to the reference's own known answers.

The reference (Rust) cannot be built here, so the oracle's parity rests on
the closed forms, independent integrations and circuit identities that the
reference's tests assert; each test cites the assertion it restates.
"""
import math

import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

MU0 = 4e-7 * math.pi


def bar_x(oracle, l, w, h):
    deck = F.Deck([(0, 0, 0), (l, 0, 0)], [F.segment(0, 1, w, h)], [(0, 1)], F.uniform(1, 1))
    return oracle.discretize(deck)[0][0]


def filament(oracle, a, b, w, h, wdir=None):
    deck = F.Deck([tuple(a), tuple(b)], [F.segment(0, 1, w, h, width_dir=wdir)], [(0, 1)], F.uniform(1, 1))
    return oracle.discretize(deck)[0][0]


# --- independent references, written from the mathematics -----------------

def gl01(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * (x + 1.0), 0.5 * w


def reference_self(l, w, h):
    """Direct integration of the self-potential of an l x w x h box: the
    triangular density of coordinate differences, split into three pyramids
    with apex at the origin (Duffy), each smooth after the map."""
    radial, angular = gl01(4), gl01(56)
    e = [l, w, h]
    total = 0.0
    s, ws = radial
    t, wt = angular
    T1, T2 = np.meshgrid(t, t, indexing="ij")
    W12 = np.outer(wt, wt)
    for apex in range(3):
        i, j, k = apex, (apex + 1) % 3, (apex + 2) % 3
        for sv, wsv in zip(s, ws):
            p = [None] * 3
            p[i] = e[i] * sv
            p[j] = e[j] * sv * T1
            p[k] = e[k] * sv * T2
            r_over_s = np.sqrt(e[i] ** 2 + e[j] ** 2 * T1 ** 2 + e[k] ** 2 * T2 ** 2)
            density = (l - p[0]) * (w - p[1]) * (h - p[2])
            total += wsv * np.sum(W12 * density * sv / r_over_s)
    return 1e-7 * 8.0 * total * l * w * h / (w * h * w * h)


def ln_gmd_rectangle(w, h):
    a, b = w / h, h / w
    return (0.5 * math.log(w * w + h * h) - a * a / 12.0 * math.log1p(b * b) - b * b / 12.0 * math.log1p(a * a)
            + 2.0 / 3.0 * (a * math.atan(b) + b * math.atan(a)) - 25.0 / 12.0)


def mean_distance_rectangle(w, h):
    long, t = max(w, h), min(w, h) / max(w, h)
    s = math.hypot(t, 1.0)
    return long / 15.0 * (t ** 3 - 1.0 / (1.0 + s) + s * (3.0 - t * t)
                          + 2.5 * (t * t * math.log((1.0 + s) / t) + math.asinh(t) / t))


def thin_bar_self(l, w, h):
    return MU0 * l / (2 * math.pi) * (math.log(2 * l) - ln_gmd_rectangle(w, h) - 1.0
                                       + mean_distance_rectangle(w, h) / l - (w * w + h * h) / (24 * l * l))


def brute_lines(a0, a1, b0, b1, panels=8):
    x, wx = gl01(16)
    a0, a1, b0, b1 = map(np.asarray, (a0, a1, b0, b1))
    total = 0.0
    for pa in range(panels):
        s = (pa + x) / panels
        ws = wx / panels
        for pb in range(panels):
            t = (pb + x) / panels
            wt = wx / panels
            P = a0[None, :] + (a1 - a0)[None, :] * s[:, None]
            Q = b0[None, :] + (b1 - b0)[None, :] * t[:, None]
            r = np.linalg.norm(P[:, None, :] - Q[None, :, :], axis=2)
            total += np.sum(np.outer(ws, wt) / r)
    return total * np.linalg.norm(a1 - a0) * np.linalg.norm(b1 - b0)


# --- tests ------------------------------------------------------------------

def test_unit_cube_self_potential(oracle, known):
    v, rel = oracle.bar_integral([1, 0, 0, -1], [1, 0, 0, -1], [1, 0, 0, -1])
    k = known["unit_cube_self_potential"]
    s2, s3 = math.sqrt(2), math.sqrt(3)
    closed = 2 * ((1 + s2 - 2 * s3) / 5 - math.pi / 3 + math.log(1 + s2) + math.log(2 + s3))
    assert abs(v - k["value"]) < k["tolerance_abs"]
    assert abs(closed - k["value"]) < 1e-15
    assert rel < 1e-12


def test_reference_helpers_reproduce_known_constants(known):
    assert abs(math.exp(ln_gmd_rectangle(1, 1)) - known["gmd_square"]["value"]) < 1e-5
    assert abs(mean_distance_rectangle(1, 1) - known["mean_distance_square"]["value"]) < 1e-6
    cube = reference_self(1.0, 1.0, 1.0) / 1e-7
    assert abs(cube - known["unit_cube_self_potential"]["value"]) < 1e-11


def test_trace_self_inductance_doc_example(oracle, known):
    k = known["trace_self_inductance_10mm_1mm_35um"]
    f = bar_x(oracle, k["length"], k["width"], k["height"])
    assert abs(oracle.self_inductance(f) - k["value"]) < k["tolerance_abs"]


@pytest.mark.parametrize("l,w,h", [(1.0, 1.0, 1.0), (1.0, 0.5, 0.25), (4.0, 1.0, 1.0), (1.0, 3.0, 2.0),
                                   (2e-3, 1e-3, 0.5e-3), (5.0, 1.0, 2.0)])
def test_self_closed_form_matches_direct_integration(oracle, l, w, h):
    want = reference_self(l, w, h)
    q = lambda e: [e, 0.0, 0.0, -e]
    v, rel = oracle.bar_integral(q(l), q(w), q(h))
    assert rel < 1e-11
    assert abs(1e-7 * v / (w * h) ** 2 - want) / want < 1e-9
    assert abs(oracle.self_inductance(bar_x(oracle, l, w, h)) - want) / want < 1e-9


@pytest.mark.parametrize("l,w,h,tol", [(1.0, 1e-2, 1e-2, 1e-8), (1.0, 1e-2, 2e-3, 1e-8), (10e-3, 1e-3, 35e-6, 5e-6),
                                       (0.1, 1e-4, 1e-4, 1e-9), (1.0, 1e-5, 3e-6, 1e-9), (1.0, 1e-7, 1e-7, 1e-9),
                                       (1.0, 1e-3, 1e-7, 1e-9)])
def test_self_term_matches_grover_rosa(oracle, l, w, h, tol):
    got = oracle.self_inductance(bar_x(oracle, l, w, h))
    want = thin_bar_self(l, w, h)
    assert abs(got - want) / want < tol


def test_self_term_switches_methods_continuously(oracle):
    methods = set()
    for k in range(40):
        w = 10 ** (-0.1 * k)
        f = bar_x(oracle, 1.0, w, 0.5 * w)
        v, m, _ = oracle.mutual(f, f)
        methods.add(m)
        assert v == oracle.self_inductance(f)
        q = lambda e: [e, 0.0, 0.0, -e]
        exact, rel = oracle.bar_integral(q(1.0), q(w), q(0.5 * w))
        if rel < 1e-6:
            exact = 1e-7 * exact / (w * 0.5 * w) ** 2
            assert abs(v - exact) / exact < 2e-9 + rel
    assert {oracle.BAR_CLOSED_FORM, oracle.ALIGNED_QUADRATURE} <= methods


@pytest.mark.parametrize("l,rho", [(1.0, 0.1), (1.0, 1.0), (1.0, 25.0), (3e-3, 2e-6)])
def test_parallel_lines_match_textbook(oracle, l, rho):
    got = oracle.lines_parallel(l, l, 0.0, rho)
    want = 2.0 * (l * math.asinh(l / rho) - math.hypot(l, rho) + rho)
    assert abs(got - want) / want < 1e-12


@pytest.mark.parametrize("b0,b1", [((0.2, 0.5, 0.1), (1.1, 1.4, 0.3)), ((0.3, -0.4, 0.6), (0.1, 0.9, 0.4)),
                                   ((2.0, 0.0, 0.3), (2.5, 1.0, 0.0))])
def test_skew_lines_match_brute_force(oracle, b0, b1):
    a0, a1 = (0, 0, 0), (1, 0, 0)
    got = oracle.lines_skew(a0, a1, b0, b1)
    want = brute_lines(a0, a1, b0, b1)
    assert abs(got - want) / abs(want) < 1e-9


@pytest.mark.parametrize("offset", [[0.0, 0.2, 0.0], [0.0, 0.0, 0.1], [0.0, 0.2, 0.1], [0.3, 0.05, 0.02],
                                    [0.4, 0.5, 0.3], [1.0, 0.0, 0.0], [1.5, 0.0, 0.0]])
def test_aligned_quadrature_matches_closed_form(oracle, offset):
    length, width, height = [1.0, 1.0], [0.2, 0.2], [0.1, 0.1]

    def cd(e1, e2, o):
        s, d = 0.5 * (e1 + e2), 0.5 * (e1 - e2)
        return [o + s, o + d, o - d, o - s]

    want, rel = oracle.bar_integral(cd(*length, offset[0]), cd(*width, offset[1]), cd(*height, offset[2]))
    got = oracle.aligned_quadrature(length, width, height, offset)
    assert abs(got - want) / want < 1e-9 + rel


def test_gauss_rules_integrate_polynomials_exactly(oracle):
    for n in [1, 2, 3, 5, 8, 16, 33, 64]:
        x, w = oracle.gauss_rule(n)
        assert abs(w.sum() - 2.0) < 1e-13
        for p in range(0, min(2 * n - 1, 40) + 1):
            got = np.sum(0.5 * w * (0.5 * (x + 1)) ** p)
            assert abs(got - 1.0 / (p + 1)) < 1e-13


def test_order_table_monotone(oracle):
    assert oracle.order_for(1e-9, 64, 0.0, 1.0) == 1
    assert oracle.order_for(1e-9, 64, 1.0, 0.0) is None
    assert oracle.order_for(1e-9, 64, 1.0, float("nan")) is None
    far, mid, near = (oracle.order_for(1e-9, 64, 1.0, d) for d in (1e6, 10.0, 1.0))
    assert far == 1 and far <= mid < near


def test_antiparallel_filaments_have_negative_mutual(oracle):
    a = filament(oracle, (0, 0, 0), (1, 0, 0), 0.1, 0.05)
    b = filament(oracle, (0, 0.5, 0), (1, 0.5, 0), 0.1, 0.05)
    c = filament(oracle, (1, 0.5, 0), (0, 0.5, 0), 0.1, 0.05)
    mf, mb = oracle.mutual(a, b)[0], oracle.mutual(a, c)[0]
    assert mf > 0 and abs(mb + mf) / mf < 1e-12


def test_orthogonal_filaments_do_not_couple(oracle):
    a = filament(oracle, (0, 0, 0), (1, 0, 0), 0.1, 0.05)
    b = filament(oracle, (0.5, 0, 0), (0.5, 1, 0), 0.1, 0.05)
    v, m, _ = oracle.mutual(a, b)
    assert v == 0.0 and m == oracle.ORTHOGONAL


def test_far_field_tends_to_dipole(oracle):
    a = filament(oracle, (0, 0, 0), (1, 0, 0), 0.01, 0.01)
    for d in [10.0, 100.0, 1000.0]:
        b = filament(oracle, (0, d, 0), (1, d, 0), 0.01, 0.01)
        got = oracle.mutual(a, b)[0]
        want = 1e-7 / d
        assert abs(got - want) / want < 2.0 / d


def test_general_orientation_matches_fine_quadrature(oracle):
    a = filament(oracle, (0, 0, 0), (1, 0, 0), 0.05, 0.03)
    b = filament(oracle, (0.3, 1.2, 0.4), (1.1, 1.9, 0.2), 0.04, 0.06)
    got, m, res = oracle.mutual(a, b)
    assert m == oracle.POINT_QUADRATURE and res
    want = brute_lines(a[0:3], a[3:6], b[0:3], b[3:6], panels=4)
    cos = float(np.dot(a[7:10], b[7:10]))
    assert abs(got - 1e-7 * cos * want) / abs(got) < 1e-3  # thin-line limit of the bars


def test_lu_matches_numpy(oracle):
    rng = np.random.default_rng(3)
    for n in [1, 31, 32, 33, 65, 200]:
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        b = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
        x = oracle.lu_solve(a, b, threads=2)
        want = np.linalg.solve(a, b)
        assert np.max(np.abs(x - want)) / np.max(np.abs(want)) < 1e-10
        assert np.max(np.abs(a @ x - b)) / (np.max(np.abs(a)) * np.max(np.abs(x))) < 1e-14 * n


def test_lu_cache_blocked_equals_column_sweeps_bitwise(oracle):
    """The oracle's row-blocked, multi-threaded LU and the reference's
    column-at-a-time sweeps (dense.rs:98-190) on one thread give the same bits,
    including interchanges, ragged last panels and several right-hand sides."""
    rng = np.random.default_rng(11)
    for n, nrhs in [(1, 1), (2, 1), (31, 2), (32, 1), (33, 3), (64, 1), (97, 2), (300, 1), (517, 2)]:
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
        fast = np.ascontiguousarray(oracle.lu_solve(a, b, threads=4))
        plain = np.ascontiguousarray(oracle.lu_solve(a, b, plain=True))
        assert np.array_equal(fast.view(np.uint64), plain.view(np.uint64)), n


def test_lu_singular_is_reported(oracle):
    a = np.zeros((4, 4), dtype=complex)
    with pytest.raises(oracle.OracleError):
        oracle.lu_solve(a, np.ones(4, dtype=complex))


def test_bar_doc_example(oracle, known):
    k = known["bar_1mm_100um_20um_5x3"]
    deck = F.Deck([(0, 0, 0), (k["length"], 0, 0)], [F.segment(0, 1, k["width"], k["height"], k["sigma"])],
                  [(0, 1)], F.uniform(k["nw"], k["nh"]))
    s = oracle.System(deck, threads=2)
    z = s.sweep(k["frequencies_hz"])[:, 0, 0]
    r_dc = k["length"] / (k["sigma"] * k["width"] * k["height"])
    assert abs(z[0].real - r_dc) < k["r_dc_tolerance_abs"]
    l1 = z[1].imag / (2 * math.pi * 1e6)
    assert k["l_1mhz_bounds"][0] < l1 < k["l_1mhz_bounds"][1]
    assert z[2].real > z[0].real


def test_trace_doc_example(oracle, known):
    k = known["trace_10mm_1mm_35um_5x2"]
    deck = F.Deck([(0, 0, 0), (k["length"], 0, 0)], [F.segment(0, 1, k["width"], k["height"], k["sigma"])],
                  [(0, 1)], F.uniform(k["nw"], k["nh"]))
    z = oracle.System(deck, threads=2).sweep(k["frequencies_hz"])[:, 0, 0]
    r_dc = k["length"] / (k["sigma"] * k["width"] * k["height"])
    assert abs(z[0].real - r_dc) < 1e-12 * r_dc
    assert z[0].imag == 0.0
    assert z[2].real > z[0].real


def coupled_two_port():
    """Two parallel traces, one port each (reciprocity / passivity checks)."""
    nodes = [(0, 0, 0), (2e-3, 0, 0), (0, 0.3e-3, 0), (2e-3, 0.3e-3, 0)]
    segs = [F.segment(0, 1, 0.2e-3, 35e-6), F.segment(2, 3, 0.2e-3, 35e-6)]
    return F.Deck(nodes, segs, [(0, 1), (2, 3)], F.uniform(3, 2), name="two_port")


def test_reciprocity_and_passivity(oracle):
    z = oracle.System(coupled_two_port(), threads=2).sweep([1e6, 1e9])
    for zk in z:
        assert abs(zk[0, 1] - zk[1, 0]) <= 1e-10 * abs(zk[0, 1])
        assert np.all(np.linalg.eigvalsh(0.5 * (zk + zk.conj().T)) > 0)


def test_schur_equals_textbook_mesh_solve(oracle):
    deck = coupled_two_port()
    s = oracle.System(deck, threads=2)
    R, L = s.blocks()
    m = s.counts["internal_meshes"]
    f = 1e8
    A = R + 2j * math.pi * f * L
    # exciting port currents: the loop currents of the full mesh system
    want = A[m:, m:] - A[:m, m:].T @ np.linalg.solve(A[:m, :m], A[:m, m:])
    got = s.impedance(f)
    assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < 1e-12


def test_golden_c1_regenerates(oracle):
    from conftest import load_golden
    g = load_golden("c1_z.json")
    d, fr = F.c1_spiral()
    z = oracle.System(d, threads=2).sweep(fr)
    want = np.array(g["z_re"]) + 1j * np.array(g["z_im"])
    assert np.max(np.abs(z - want) / np.abs(want)) < 1e-13
