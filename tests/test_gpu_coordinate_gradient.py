"""The impedance gradient with respect to node coordinates (x, y).

A node moving in the xy plane turns the segments that meet there about z,
changes their length and moves their filaments.  The coordinate derivative
fill (fh_test_coordinate_gradient) gives, per filament pair, the partial
derivatives of L_ab with respect to a translation, a stretch and a rotation
of either filament; fh_gradient chains them to the node coordinates.  There
is no reference gradient, so parity is pinned by:

* pair derivatives against central differences of an independent
  brute-force integral (composite Gauss-Legendre over both volumes, numpy)
  for point-quadrature and aligned-quadrature pairs, parallel, antiparallel
  and orthogonal, rotations included;
* near orthogonal pairs against the oracle's bar integral (the reference's
  closed form, bar.rs) of the two boxes;
* a segment's own pairs (stretch only) against differences of the oracle's
  frozen-dispatch fill;
* the rigid-motion identities of every pair of filaments of different segments
  of a graded spiral;
* dZ/dx, dZ/dy of small decks: translation and rotation invariance of Z, and
  node motions that keep the deck Manhattan (a uniform in-plane scaling, a
  column of nodes moved together, a port's end node moved along its
  segment) against differences of the oracle's Z with frozen dispatch.
Bound: 1e-6 of the scale of each compared quantity.
"""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu

MU0_4PI = 1e-7
TOL = 1e-6
UM = 1e-6


# ---------------------------------------------------------------------------
# Boxes, filaments, brute force
# ---------------------------------------------------------------------------
def rot_z(v, eps):
    c, s = np.cos(eps), np.sin(eps)
    return np.array([c * v[0] - s * v[1], s * v[0] + c * v[1], v[2]])


class Box:
    def __init__(self, centre, length_dir, dims, width_dir=None):
        self.c = np.asarray(centre, dtype=float)
        l = np.asarray(length_dir, dtype=float)
        self.l = l / np.linalg.norm(l)
        w = np.cross([0.0, 0.0, 1.0], self.l) if width_dir is None else np.asarray(width_dir, dtype=float)
        self.w = w / np.linalg.norm(w)
        self.h = np.cross(self.l, self.w)
        self.dims = np.asarray(dims, dtype=float)

    def moved(self, kind, eps):
        b = Box(self.c, self.l, self.dims, self.w)
        if kind == "l":
            b.c = self.c + eps * self.l
        elif kind == "p":
            p = np.cross([0.0, 0.0, 1.0], self.l)
            b.c = self.c + eps * p / np.linalg.norm(p)
        elif kind == "s":
            b.dims = self.dims + np.array([eps, 0.0, 0.0])
        elif kind == "r":
            b.l, b.w, b.h = rot_z(self.l, eps), rot_z(self.w, eps), rot_z(self.h, eps)
        return b

    def filament(self, sigma=F.COPPER):
        half = 0.5 * self.dims[0] * self.l
        s, e = self.c - half, self.c + half
        return np.concatenate([s, e, [self.dims[0]], self.l, self.w, self.h, [self.dims[1], self.dims[2], sigma]])


def box_points(box, panels, order):
    x, wx = np.polynomial.legendre.leggauss(order)
    axes = []
    for d, m in zip(box.dims, panels):
        edges = np.linspace(-0.5 * d, 0.5 * d, m + 1)
        mid, half = 0.5 * (edges[1:] + edges[:-1]), 0.5 * (edges[1:] - edges[:-1])
        axes.append(((mid[:, None] + half[:, None] * x[None]).ravel(), (half[:, None] * wx[None]).ravel()))
    (s, ws), (t, wt), (u, wu) = axes
    S, T, U = np.meshgrid(s, t, u, indexing="ij")
    W = (ws[:, None, None] * wt[None, :, None] * wu[None, None, :]).ravel()
    P = box.c + S.ravel()[:, None] * box.l + T.ravel()[:, None] * box.w + U.ravel()[:, None] * box.h
    return P, W


def coupling(a, b, panels_a, panels_b, order):
    """int int 1 / |r - r'| over the two volumes."""
    pa, wa = box_points(a, panels_a, order)
    pb, wb = box_points(b, panels_b, order)
    total = 0.0
    for k in range(0, len(pa), 256):
        d = pa[k:k + 256, None, :] - pb[None, :, :]
        total += wa[k:k + 256] @ (1.0 / np.sqrt(np.einsum("ijk,ijk->ij", d, d))) @ wb
    return total


def brute_l(a, b, panels_a, panels_b, order):
    area = a.dims[1] * a.dims[2] * b.dims[1] * b.dims[2]
    return MU0_4PI * (a.l @ b.l) * coupling(a, b, panels_a, panels_b, order) / area


def device_d(fh, boxes, segments):
    fil = np.array([b.filament() for b in boxes])
    return fh.coordinate_gradient(fil, segments)


# ---------------------------------------------------------------------------
# Pair derivatives
# ---------------------------------------------------------------------------
PAIRS = {
    # B far from A along y: point quadrature
    "point_parallel": (Box([0, 0, 0], [1, 0, 0], [30 * UM, 2 * UM, 1 * UM]),
                       Box([5 * UM, 40 * UM, 0], [1, 0, 0], [20 * UM, 2 * UM, 1 * UM]), (4, 1, 1), (3, 1, 1)),
    # B near A (gap 7 um against a 40 um length): aligned quadrature with rotations
    "quad_parallel": (Box([0, 0, 0], [1, 0, 0], [40 * UM, 2 * UM, 1 * UM]),
                      Box([6 * UM, 9 * UM, 0.5 * UM], [1, 0, 0], [30 * UM, 2 * UM, 1 * UM]), (8, 1, 1), (6, 1, 1)),
    # the gap (3 um) 1.5 times the largest side: the sixth-order product rule
    "quad_parallel_near": (Box([0, 0, 0], [1, 0, 0], [40 * UM, 2 * UM, 1 * UM]),
                           Box([6 * UM, 5 * UM, 0.5 * UM], [1, 0, 0], [30 * UM, 2 * UM, 1 * UM]), (8, 1, 1),
                           (6, 1, 1)),
    "quad_antiparallel": (Box([0, 0, 0], [1, 0, 0], [40 * UM, 2 * UM, 1 * UM]),
                          Box([-4 * UM, -9 * UM, 0], [-1, 0, 0], [30 * UM, 2 * UM, 1 * UM]), (8, 1, 1), (6, 1, 1)),
    # orthogonal, far: point quadrature (the derivative is the rotation's alone)
    "point_ortho": (Box([0, 0, 0], [1, 0, 0], [20 * UM, 2 * UM, 1 * UM]),
                    Box([45 * UM, 30 * UM, 0], [0, 1, 0], [20 * UM, 2 * UM, 1 * UM]), (3, 1, 1), (3, 1, 1)),
    # orthogonal, the width along z on B: rotation frame from the height axis
    "point_ortho_standing": (Box([0, 0, 0], [1, 0, 0], [20 * UM, 2 * UM, 1 * UM]),
                             Box([40 * UM, 35 * UM, 0], [0, 1, 0], [20 * UM, 1 * UM, 2 * UM], [0, 0, 1]),
                             (3, 1, 1), (3, 1, 1)),
}


@pytest.mark.parametrize("name", sorted(PAIRS))
def test_pair_derivatives_match_brute_force_differences(fh, name):
    a, b, pa, pb = PAIRS[name]
    D = device_d(fh, [a, b], [0, 1])
    order = 5  # panels and order resolve the derivatives to about 1e-9
    scale_l = MU0_4PI * coupling(a, b, pa, pb, order) / (a.dims[1] * a.dims[2] * b.dims[1] * b.dims[2])
    steps = {"l": 1e-9, "p": 1e-9, "s": 1e-9, "r": 1e-5}
    size = max(a.dims[0], b.dims[0])
    for k, kind in enumerate("lpsr"):
        h = steps[kind]
        for side, (row, col) in ((0, (0, 1)), (1, (1, 0))):
            def l_at(eps):
                if side == 0:
                    return brute_l(a.moved(kind, eps), b, pa, pb, order)
                return brute_l(a, b.moved(kind, eps), pa, pb, order)
            fd = (l_at(h) - l_at(-h)) / (2 * h)
            got = D[k][row, col]
            scale = scale_l * (1.0 if kind == "r" else 1.0 / size)
            assert abs(got - fd) <= TOL * max(abs(fd), scale), (name, kind, side, got, fd)


def test_near_orthogonal_pair_matches_the_oracle_bar_integral(fh, oracle):
    # Two segments meeting at a corner: their filaments' boxes overlap there.
    a = Box([15 * UM, 0, 0], [1, 0, 0], [30 * UM, 4 * UM, 2 * UM])
    b = Box([30 * UM, 15 * UM, 0], [0, 1, 0], [30 * UM, 4 * UM, 2 * UM])
    D = device_d(fh, [a, b], [0, 1])
    # b as a box in a's frame: extents (4, 30, 2) um, offset (15, 15, 0) um.
    def corners(e1, e2, off):
        return [off + 0.5 * (e1 + e2), off + 0.5 * (e1 - e2), off - 0.5 * (e1 - e2), off - 0.5 * (e1 + e2)]
    ext_b = [4 * UM, 30 * UM, 2 * UM]
    off = b.c - a.c
    v, rel = oracle.bar_integral(corners(a.dims[0], ext_b[0], off[0]), corners(a.dims[1], ext_b[1], off[1]),
                                 corners(a.dims[2], ext_b[2], off[2]))
    bound = 1e-10
    if rel > 1e-10:  # the closed form's own estimate rejects it: the reference's aligned quadrature
        v = oracle.aligned_quadrature([a.dims[0], ext_b[0]], [a.dims[1], ext_b[1]], [a.dims[2], ext_b[2]], off)
        bound = 1e-8
    k = MU0_4PI / (a.dims[1] * a.dims[2] * b.dims[1] * b.dims[2])
    want_a = k * (np.cross([0, 0, 1], a.l) @ b.l) * v
    want_b = k * (np.cross([0, 0, 1], b.l) @ a.l) * v
    assert abs(D[3][0, 1] - want_a) <= bound * abs(want_a), (D[3][0, 1], want_a)
    assert abs(D[3][1, 0] - want_b) <= bound * abs(want_b), (D[3][1, 0], want_b)
    for k in range(3):
        assert D[k][0, 1] == 0.0 and D[k][1, 0] == 0.0


@pytest.mark.parametrize("gap_um,on_side", [(g, side) for g in (5.0, 13.0, 20.0) for side in (False, True)])
def test_orthogonal_pairs_apart_match_the_oracle_quadrature(fh, oracle, gap_um, on_side):
    """Long orthogonal boxes whose gap is 2.5, 6.5 and 10 times their largest
    cross-section side (2 um): too near for point quadrature and rejected by
    the closed form, so the coordinate fill integrates them -- by the product
    rule over both cross-sections of the perpendicular-segment integral.  A
    lies flat (B's length then runs along A's width axis) or on its side
    (width along z: B's length runs along A's height axis).  The rotation
    rates against the oracle's restatement of the reference's aligned
    quadrature of the two boxes in A's frame."""
    la, lb = 300 * UM, 250 * UM
    a = Box([0, 0, 0], [1, 0, 0], [la, 2 * UM, 1 * UM], [0, 0, 1] if on_side else None)
    b = Box([0.5 * la + gap_um * UM + 1 * UM, 0.5 * lb + 2 * UM, 0.2 * UM], [0, 1, 0], [lb, 2 * UM, 1 * UM])
    D = device_d(fh, [a, b], [0, 1])
    # b's box in a's frame: its extents along a's axes, its centre's offset
    axes_a = [a.l, a.w, a.h]
    ext_b = [sum(abs(ax @ bx) * d for bx, d in zip([b.l, b.w, b.h], b.dims)) for ax in axes_a]
    off = [ax @ (b.c - a.c) for ax in axes_a]
    v = oracle.aligned_quadrature([a.dims[0], ext_b[0]], [a.dims[1], ext_b[1]], [a.dims[2], ext_b[2]], off)
    k = MU0_4PI / (a.dims[1] * a.dims[2] * b.dims[1] * b.dims[2])
    want_a = k * (np.cross([0, 0, 1], a.l) @ b.l) * v
    want_b = k * (np.cross([0, 0, 1], b.l) @ a.l) * v
    assert abs(want_a) > 0 and abs(want_b) > 0
    assert abs(D[3][0, 1] - want_a) <= 1e-9 * abs(want_a), (D[3][0, 1], want_a)
    assert abs(D[3][1, 0] - want_b) <= 1e-9 * abs(want_b), (D[3][1, 0], want_b)
    for q in range(3):
        assert D[q][0, 1] == 0.0 and D[q][1, 0] == 0.0


def test_segment_pairs_carry_the_stretch_of_the_frozen_fill(fh, oracle):
    """A bundle of one segment: only Ds, equal to differences of the oracle's
    frozen fill with one filament stretched about its centre (the diagonal:
    half of the self term's rate)."""
    deck = F.Deck([(0, 0, 0), (300e-6, 0, 0)], [F.segment(0, 1, 12e-6, 3e-6)], [(0, 1)], F.graded(4, 2, 1.6),
                  "bundle")
    fil, per = oracle.discretize(deck)
    n = len(fil)
    Dl, Dp, Ds, Dr = fh.coordinate_gradient(fil, np.zeros(n, dtype=np.int32))
    assert not Dl.any() and not Dp.any() and not Dr.any()
    h = 1e-5 * fil[0, 6]
    for a in (0, 3, n - 1):
        def stretched(eps):
            f = fil.copy()
            f[a, 0:3] -= 0.5 * eps * f[a, 7:10]
            f[a, 3:6] += 0.5 * eps * f[a, 7:10]
            f[a, 6] += eps
            return oracle.fill_frozen(fil, f)
        fd = (stretched(h) - stretched(-h)) / (2 * h)
        row = Ds[a].copy()
        row[a] *= 2.0  # the diagonal holds half of the self term's rate
        err = np.max(np.abs(row - fd[a])) / np.max(np.abs(fd[a]))
        assert err < TOL, (a, err)


def test_rigid_motions_leave_every_pair_unchanged(fh, oracle):
    """For every pair of filaments of different segments of a graded spiral: a
    common translation and a common rotation about a's centre change
    nothing, so
      grad_a L + grad_b L = 0  and  Dr_a + Dr_b + (z x (c_b - c_a)) . grad_b L = 0
    (point, quadrature and orthogonal pairs alike)."""
    deck = F.square_spiral(3, 10e-6, 5e-6, 2e-6, 200e-6, F.graded(3, 2, 1.5))
    fil, per = oracle.discretize(deck)
    seg = np.repeat(np.arange(len(per)), per).astype(np.int32)
    Dl, Dp, Ds, Dr = fh.coordinate_gradient(fil, seg)
    n = len(fil)
    c = 0.5 * (fil[:, 0:3] + fil[:, 3:6])
    l = fil[:, 7:10]
    p = np.stack([-l[:, 1], l[:, 0], np.zeros(n)], axis=1)
    nrm = np.linalg.norm(p, axis=1)
    p = np.where(nrm[:, None] > 0, p / np.where(nrm > 0, nrm, 1.0)[:, None], 0.0)
    flat = np.abs(l[:, 2]) < 1e-12
    # gradient with respect to a's centre, in the plane: Dl l_a + Dp p_a
    ga = Dl[:, :, None] * l[:, None, :] + Dp[:, :, None] * p[:, None, :]
    pair = flat[:, None] & flat[None, :] & (seg[:, None] != seg[None, :])
    scale_t = np.max(np.abs(ga[pair]))
    trans = ga + np.transpose(ga, (1, 0, 2))
    assert np.max(np.abs(trans[pair])) <= TOL * scale_t
    t = c[None, :, :] - c[:, None, :]  # c_b - c_a
    zt = np.stack([-t[..., 1], t[..., 0], np.zeros_like(t[..., 0])], axis=-1)
    gb = np.transpose(ga, (1, 0, 2))  # grad wrt b's centre of L_ab
    rot = Dr + Dr.T + np.einsum("abk,abk->ab", zt, gb)
    scale_r = np.max(np.abs(Dr[pair]))
    assert np.max(np.abs(rot[pair])) <= TOL * scale_r, np.max(np.abs(rot[pair])) / scale_r


# ---------------------------------------------------------------------------
# dZ/dx, dZ/dy of decks
# ---------------------------------------------------------------------------
def loop_matrix(oracle, deck, per, n):
    row_ptr, cols, signs, internal = oracle.mesh(deck, per)
    M = np.zeros((len(row_ptr) - 1, n))
    for r in range(len(row_ptr) - 1):
        for k in range(row_ptr[r], row_ptr[r + 1]):
            M[r, cols[k]] += signs[k]
    return M, internal


def schur(M, m, R, L, omega):
    Zm = M @ (np.diag(R) + 1j * omega * L) @ M.T
    ee, ep, pp = Zm[:m, :m], Zm[:m, m:], Zm[m:, m:]
    return pp - ep.T @ np.linalg.solve(ee, ep)


def resistances(f):
    return f[:, 6] / (f[:, 18] * (f[:, 16] * f[:, 17]))


def with_nodes(deck, nodes):
    return F.Deck([tuple(v) for v in nodes], deck.segments, deck.ports, deck.discretization, deck.name)


def fd_of_motion(oracle, deck, motion, frequency, h):
    """Central difference of the oracle's Z (frozen dispatch) for node
    positions nodes + t * motion, t = +-h."""
    nodes = np.array(deck.nodes, dtype=float)
    fil0, per0 = oracle.discretize(deck)
    M, m = loop_matrix(oracle, deck, per0, len(fil0))
    omega = 2 * np.pi * frequency
    z = []
    for sgn in (1, -1):
        d = with_nodes(deck, nodes + sgn * h * motion)
        fil, per = oracle.discretize(d)
        assert np.array_equal(per, per0)
        z.append(schur(M, m, resistances(fil), oracle.fill_frozen(fil0, fil), omega))
    return (z[0] - z[1]) / (2 * h)


def node_gradient(fh, deck, frequency):
    params = [fh.Param(k, i) for i in range(len(deck.nodes)) for k in ("x", "y")]
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as system:
        g = system.gradient(frequency, params)
    return g.gradient.reshape(len(deck.nodes), 2, *g.gradient.shape[1:]), g


@pytest.mark.parametrize("frequency", [1e6, 1e9])
def test_spiral_node_gradient_is_invariant_and_matches_manhattan_motions(fh, oracle, frequency):
    deck = F.square_spiral(3, 10e-6, 5e-6, 2e-6, 200e-6, F.graded(4, 2, 1.5))
    dz, g = node_gradient(fh, deck, frequency)
    nodes = np.array(deck.nodes)
    scale = np.max(np.abs(dz))
    # translation and rotation of the whole deck change nothing
    assert np.max(np.abs(dz[:, 0].sum(axis=0))) <= TOL * scale
    assert np.max(np.abs(dz[:, 1].sum(axis=0))) <= TOL * scale
    rot = (nodes[:, 0, None, None] * dz[:, 1] - nodes[:, 1, None, None] * dz[:, 0]).sum(axis=0)
    size = np.max(np.abs(nodes))
    assert np.max(np.abs(rot)) <= TOL * scale * size, np.max(np.abs(rot)) / (scale * size)
    # Manhattan-preserving motions against the oracle
    motions = []
    scaling = np.zeros_like(nodes)
    scaling[:, :2] = nodes[:, :2]
    motions.append(scaling)
    column = np.zeros_like(nodes)
    column[nodes[:, 0] > 0.5 * size, 0] = 1.0
    motions.append(column)
    end = np.zeros_like(nodes)
    last = deck.segments[-1]
    direction = nodes[last["b"]] - nodes[last["a"]]
    end[last["b"]] = direction / np.linalg.norm(direction)
    motions.append(end)
    for motion in motions:
        adj = np.einsum("nk,nkab->ab", motion[:, :2], dz)
        h = 1e-9 / np.max(np.abs(motion[:, :2]))  # nodes move by at most 1 nm
        fd = fd_of_motion(oracle, deck, motion, frequency, h)
        err = np.max(np.abs(adj - fd)) / np.max(np.abs(fd))
        assert err < TOL, err


def test_two_port_meander_node_gradient(fh, oracle):
    base = F.meander_legs(3, nw=3, nh=2)
    nodes = base.nodes
    deck = F.Deck(nodes, base.segments, [(0, len(nodes) // 2), (len(nodes) // 2, len(nodes) - 1)],
                  base.discretization, "two_port")
    dz, g = node_gradient(fh, deck, 1e8)
    assert np.array_equal(dz[..., 0, 1], dz[..., 1, 0])
    arr = np.array(nodes)
    motion = np.zeros_like(arr)
    motion[arr[:, 1] > 0.5 * arr[:, 1].max(), 1] = 1.0  # the upper legs move up together
    adj = np.einsum("nk,nkab->ab", motion[:, :2], dz)
    fd = fd_of_motion(oracle, deck, motion, 1e8, 1e-9)
    err = np.max(np.abs(adj - fd)) / np.max(np.abs(fd))
    assert err < TOL, err


def test_node_parameters_are_validated(fh):
    deck, _ = F.c1_spiral()
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization) as system:
        with pytest.raises(fh.Unsupported):
            system.gradient(1e9, [fh.Param("z", 3)])
        with pytest.raises(fh.InvalidArgument):
            system.gradient(1e9, [fh.Param("x", len(deck.nodes))])
        g = system.gradient(1e9, [fh.Param("width", 0), fh.Param("x", 2), fh.Param("y", 2)])
        assert g.gradient.shape == (3, 1, 1)
        # a vertical segment's node cannot move in the plane
    vdeck = F.Deck([(0, 0, 0), (100e-6, 0, 0), (100e-6, 0, 50e-6)],
                   [F.segment(0, 1, 10e-6, 2e-6), F.segment(1, 2, 10e-6, 2e-6)], [(0, 2)], F.uniform(2, 1), "via")
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(vdeck), vdeck.ports, vdeck.discretization) as system:
        with pytest.raises(fh.Unsupported):
            system.gradient(1e9, [fh.Param("x", 2)])
        system.gradient(1e9, [fh.Param("x", 0)])
