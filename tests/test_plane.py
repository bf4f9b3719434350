"""Ground planes (fasterhenry_b200/plane.py) against the reference's plane
known answers (fasterhenry/src/plane.rs tests: counts and positions of the
5 x 3 test plane, the hole rules with their ties, the composition of an
arbitrary rule from point holes, graded contact regions, equipotential ties,
snapping), and the deck reader's two G grammars against the reference's own
fixture pairs (fasterhenry-cli/tests/roundtrip.rs:384-480): the corner-point
and extension spellings of one plane must read to the same problem.
Host-only."""
import math
import os

import pytest

from fasterhenry_b200 import api as A
from fasterhenry_b200 import plane as PL
from fasterhenry_b200 import problem as P

DECKS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "decks")


def test_plane(**kw):
    args = dict(lo=(0.0, 0.0), hi=(10e-3, 6e-3), z_top=0.0, thickness=35e-6, nx=5, ny=3, sigma=5.8e7)
    args.update(kw)
    return PL.GroundPlane(**args)


test_plane.__test__ = False


def build(plane):
    g = A.Geometry()
    return g, plane.build_into(g)


def test_mesh_counts_and_positions():
    g, c = build(test_plane())
    assert len(g.nodes) == 15 and len(g.segments) == 22
    n = g.nodes[c[0][0]]
    assert abs(n.x - 1e-3) < 1e-12 and abs(n.y - 1e-3) < 1e-12 and abs(n.z + 17.5e-6) < 1e-12
    assert all(x is not None for col in c for x in col)


def test_rect_holes_remove_cells_and_bars_with_an_open_boundary():
    g, c = build(test_plane(holes=[PL.Hole.rect((4.9e-3, 2.9e-3), (5.1e-3, 3.1e-3))]))
    assert c[2][1] is None and len(g.nodes) == 14 and len(g.segments) == 18
    g, _ = build(test_plane(holes=[PL.Hole.rect((5e-3, 0.0), (6e-3, 6e-3))]))
    assert len(g.nodes) == 15


def test_point_holes_and_their_tie():
    g, c = build(test_plane(holes=[PL.Hole.point((5.5e-3, 3.5e-3))]))
    assert c[2][1] is None and len(g.nodes) == 14 and len(g.segments) == 18
    g, c = build(test_plane(holes=[PL.Hole.point((4e-3, 3.5e-3))]))
    assert c[1][1] is None and c[2][1] is None and len(g.nodes) == 13
    g, c = build(test_plane(holes=[PL.Hole.point((50e-3, 3e-3))]))
    assert all(x is not None for col in c for x in col)


def test_circle_holes_are_closed():
    g, c = build(test_plane(holes=[PL.Hole.circle((5e-3, 1e-3), 2.5e-3)]))
    for i, j in [(1, 0), (2, 0), (3, 0), (2, 1)]:
        assert c[i][j] is None
    for i, j in [(0, 0), (4, 0), (0, 1), (1, 1), (3, 1), (4, 1)]:
        assert c[i][j] is not None
    assert len(g.nodes) == 11
    g, c = build(test_plane(holes=[PL.Hole.circle((5e-3, 1e-3), 2e-3)]))
    assert c[2][0] is None and c[1][0] is None and c[3][0] is None and c[2][1] is None
    g, c = build(test_plane(holes=[PL.Hole.circle((5e-3, 3e-3), 100e-3)]))
    assert len(g.nodes) == 0 and len(g.segments) == 0


def test_an_arbitrary_rule_composes_from_point_holes_on_uniform_and_graded_meshes():
    for contacts in ([], [PL.ContactRegion.centred((5e-3, 3e-3), 1e-3, 2, 2.0)]):
        plane = test_plane(contacts=contacts)
        mesh = plane.mesh()
        rule = (lambda i, j, c: (i + j) % 2 == 0) if not contacts else (lambda i, j, c: c[0] < 5e-3)
        cut = 0
        for i in range(mesh.nx()):
            for j in range(mesh.ny()):
                if rule(i, j, mesh.centre(i, j)):
                    c = mesh.centre(i, j)
                    plane.holes.append(PL.Hole.point((c[0], c[1])))
                    cut += 1
        g, live = build(plane)
        for i in range(mesh.nx()):
            for j in range(mesh.ny()):
                assert (live[i][j] is None) == rule(i, j, mesh.centre(i, j))
        assert len(g.nodes) == mesh.nx() * mesh.ny() - cut
        if not contacts:
            assert len(g.nodes) == 7


def test_an_equipotential_ties_its_cells_into_one_node():
    plane = test_plane(equipotentials=[PL.Equipotential((2e-3, 0.0), (8e-3, 4e-3))])
    g, c = build(plane)
    tie = c[1][0]
    for i, j in [(1, 0), (1, 1), (2, 0), (2, 1), (3, 0), (3, 1)]:
        assert c[i][j] == tie
    for i, j in [(0, 0), (4, 0), (0, 1), (4, 1), (0, 2), (2, 2), (4, 2)]:
        assert c[i][j] is not None and c[i][j] != tie
    assert len(g.nodes) == 15 - 6 + 1
    n = g.nodes[tie]
    assert abs(n.x - 5e-3) < 1e-12 and abs(n.y - 2e-3) < 1e-12 and abs(n.z + 17.5e-6) < 1e-12
    assert len(g.segments) == 22 - 7
    assert all(s.a != s.b for s in g.segments)
    assert plane.equipotential_node(c, 0) == tie
    assert plane.attach(c, (6.9e-3, 0.1e-3, 0.0)) == tie


def test_attach_and_contains():
    plane = test_plane(holes=[PL.Hole.point((1e-3, 1e-3))])
    g, c = build(plane)
    assert c[0][0] is None
    snapped = plane.attach(c, (0.9e-3, 1.9e-3, 0.0))
    assert snapped == c[0][1]
    plane = test_plane()
    assert plane.contains((1e-3, 1e-3, 0.0), 0.0) and plane.contains((1e-3, 1e-3, -35e-6), 0.0)
    assert plane.contains((10e-3, 1e-3, 0.0), 1e-15) and not plane.contains((10e-3 + 1e-9, 1e-3, 0.0), 1e-15)
    assert not plane.contains((1e-3, 1e-3, 1e-9), 0.0)


def test_degenerate_planes_are_errors():
    with pytest.raises(PL.PlaneError, match="nx, ny >= 1"):
        test_plane(nx=0).mesh()
    with pytest.raises(PL.PlaneError, match="degenerate"):
        test_plane(hi=(0.0, 6e-3)).mesh()


def test_uniform_edges_and_graded_contact_regions():
    mesh = test_plane().mesh()
    assert (mesh.nx(), mesh.ny()) == (5, 3) and mesh.bars() == 22
    assert all(abs(mesh.x[i] - i * 2e-3) < 1e-15 for i in range(5)) and mesh.x[5] == 10e-3 and mesh.y[3] == 6e-3
    mesh = test_plane(contacts=[PL.ContactRegion.centred((5e-3, 3e-3), 1e-3, 4, 2.0)]).mesh()
    fine = [i for i in range(mesh.nx()) if abs(mesh.dx(i) - 0.25e-3) < 1e-12]
    assert len(fine) == 4
    assert abs(mesh.x[fine[0]] - 4.5e-3) < 1e-12 and abs(mesh.x[fine[3] + 1] - 5.5e-3) < 1e-12
    assert all(mesh.dx(i) <= 2e-3 + 1e-12 for i in range(fine[0]))
    assert 1.0 <= mesh.dx(fine[0] - 1) / 0.25e-3 <= 2.0 + 1e-9
    assert mesh.ny() > 3 and mesh.x[0] == 0.0 and mesh.x[-1] == 10e-3 and mesh.y[-1] == 6e-3
    assert abs(sum(mesh.dx(i) for i in range(mesh.nx())) - 10e-3) < 1e-15
    # grading costs far less than refining everywhere
    graded = test_plane(nx=20, ny=12, contacts=[PL.ContactRegion.centred((5e-3, 3e-3), 0.5e-3, 4, 1.5)]).mesh()
    assert abs(min(graded.dx(i) for i in range(graded.nx())) - 0.125e-3) < 1e-12
    assert graded.bars() * 4 < test_plane(nx=80, ny=48).mesh().bars()
    # a unit ratio is a uniformly fine axis; per-axis ratios decay independently
    mesh = test_plane(contacts=[PL.ContactRegion.new((4e-3, 2e-3), (6e-3, 4e-3), (4, 4), 1.0)]).mesh()
    assert (mesh.nx(), mesh.ny()) == (20, 12)
    region = lambda r: PL.ContactRegion.graded_per_axis((4e-3, 2e-3), (6e-3, 4e-3), (4, 4), r)  # noqa: E731
    assert (lambda m: (m.nx(), m.ny()))(test_plane(contacts=[region((1.0, 4.0))]).mesh()) == (20, 6)
    assert (lambda m: (m.nx(), m.ny()))(test_plane(contacts=[region((4.0, 1.0))]).mesh()) == (8, 12)
    # a contact at the footprint edge is clipped and keeps its resolution
    mesh = test_plane(contacts=[PL.ContactRegion.new((-0.5e-3, -1e-3), (0.5e-3, 1e-3), (4, 8), 2.0)]).mesh()
    assert mesh.x[0] == 0.0 and mesh.y[0] == 0.0
    assert abs(mesh.dx(0) - 0.25e-3) < 1e-12 and abs(mesh.dx(1) - 0.25e-3) < 1e-12
    assert abs(mesh.dy(0) - 0.25e-3) < 1e-12


def test_contacts_compose_with_holes():
    plane = test_plane(contacts=[PL.ContactRegion.centred((5e-3, 3e-3), 1e-3, 2, 2.0)],
                       holes=[PL.Hole.rect((4.5e-3, 2.5e-3), (5.5e-3, 3.5e-3))])
    mesh = plane.mesh()
    g, c = build(plane)
    dead = 0
    for i in range(mesh.nx()):
        for j in range(mesh.ny()):
            x, y, _ = mesh.centre(i, j)
            inside = 4.5e-3 < x < 5.5e-3 and 2.5e-3 < y < 3.5e-3
            assert (c[i][j] is None) == inside
            dead += inside
    assert dead >= 4 and len(g.nodes) == mesh.nx() * mesh.ny() - dead
    assert len(g.segments) < mesh.bars()


def load(name):
    return P.load(os.path.join(DECKS, name))


@pytest.mark.parametrize("a,b", [("plane_fasthenry.inp", "plane_extension.inp"),
                                 ("plane_decay_rect.inp", "plane_decay_extension.inp")])
def test_the_two_plane_grammars_read_to_one_problem(a, b):
    pa, pb = load(a), load(b)
    assert pa.nodes == pb.nodes
    assert pa.segments == pb.segments
    assert pa.ports == pb.ports
    assert pa.discretization == pb.discretization
    assert pa.frequencies_hz == pb.frequencies_hz == [1e6, 1e7, 1e8]
    assert len(pa.nodes) > 5 * 3  # the contact region refines the plane


def test_plane_deck_structure():
    p = load("plane_extension.inp")
    # plane nodes first; the two vias end on snapped plane nodes and on their
    # own top nodes, which are the only declared nodes kept
    tops = [k for k, nd in enumerate(p.nodes) if math.isclose(nd[2], 0.5e-3)]
    assert len(tops) == 2 and tops == [len(p.nodes) - 2, len(p.nodes) - 1]
    vias = p.segments[-2:]
    assert {vias[0]["a"], vias[1]["a"]} == set(tops)
    for v in vias:
        assert v["b"] < tops[0] and abs(p.nodes[v["b"]][2]) < 1e-15
    assert p.ports == [(tops[0], tops[1], "plane")]
    # the hole (0.5..1.5, 4.5..5.5) mm removed the cell centred at (1, 5) mm
    assert not any(math.isclose(x, 1e-3) and math.isclose(y, 5e-3) for x, y, _ in p.nodes)
