"""The corner-point G statement's refinement and contact-area clauses
(fasterhenry_b200/problem.py), pinned to the equivalences the reference's
own reader tests state (fasterhenry-cli/src/inp.rs tests, 6082-7240,
8003-8097, 9455-9560):

* ``contact point`` / ``contact line`` are the ``.contact`` directive over
  their padded bounding box, an axis the background already meets spanning
  the whole plane at its own cell count;
* ``contact trace`` along x or y is its five documented ``contact line`` s;
* ``contact equiv_rect N<name>`` ties every live cell centre in its
  rectangle to one node, and ``contact connection`` is an ``equiv_rect``
  plus a ``decay_rect`` over the same rectangle;
* ``contact initial_grid (n1, n2)`` is ``seg1=n1 seg2=n2``, and
  ``contact initial_mesh_grid`` adds the checkerboard of even-indexed cells
  counted from the p1 corner;
* ``segwid1`` / ``segwid2`` cap the widths of the bars along p1->p2 and
  p2->p3;
* ``relx`` / ``rely`` / ``relz`` move every in-plane coordinate, not the
  corner points.

CPU only: the deck reader and the plane mesher are host code.
"""
import math

import pytest

from fasterhenry_b200 import api as A
from fasterhenry_b200 import plane as PL
from fasterhenry_b200 import problem as P

REFINE_PLANE = "Gp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=6 z3=0\n+ thick=0.04 seg1=5 seg2=3"


def plane_deck(statement, extra=""):
    return (".units mm\n.default sigma=5.8e4\n%s\nNt x=5 y=3 z=0.5\nNb x=5 y=3 z=0\nEv Nt Nb w=0.2 h=0.2\n%s\n"
            ".external Nt Nb\n.freq fmin=1 fmax=1 ndec=1\n.end\n" % (statement, extra))


def refine_deck(clause):
    return plane_deck(REFINE_PLANE + "\n+ " + clause)


def parse(text):
    return P.parse_deck(text)


def same(a, b):
    """The same geometry, ports and discretization, bit for bit."""
    return a.to_json() == b.to_json()


def same_mesh(a, b):
    """The same node count, segment count and node positions to 1e-15 m."""
    if len(a.nodes) != len(b.nodes) or len(a.segments) != len(b.segments):
        return False
    return all(abs(p[0] - q[0]) < 1e-15 and abs(p[1] - q[1]) < 1e-15 and p[2] == q[2]
               for p, q in zip(a.nodes, b.nodes))


def node_axis(problem, axis):
    vals = sorted(n[axis] for n in problem.nodes)
    out = []
    for v in vals:
        if not out or abs(v - out[-1]) >= 1e-12:
            out.append(v)
    return out


def error_of(text):
    with pytest.raises(P.DeckError) as e:
        parse(text)
    return e.value


# -- contact point / contact line -------------------------------------------
def test_contact_point_is_one_fine_cell_centred_on_the_point():
    point = parse(refine_deck("contact point (5, 3, 0, 0.5, 0.25)"))
    directive = parse(plane_deck(REFINE_PLANE, ".contact Gp 4.75 2.875 5.25 3.125 nx=1 ny=1 ratio=2"))
    assert same(point, directive)
    assert any(abs(n[0] - 5e-3) < 1e-12 and abs(n[1] - 3e-3) < 1e-12 for n in point.nodes)


def test_contact_point_never_coarsens_the_background():
    plain = parse(plane_deck(REFINE_PLANE))
    assert same(parse(refine_deck("contact point (5, 3, 0, 2, 3)")), plain)
    half = parse(refine_deck("contact point (5, 3, 0, 4, 0.5)"))
    assert same(half, parse(plane_deck(REFINE_PLANE, ".contact Gp 0 2.75 10 3.25 nx=5 ny=1 ratio=2")))


def test_a_met_axis_is_left_alone_even_off_the_grid_lines():
    plain = parse(plane_deck(REFINE_PLANE))
    unaligned = parse(refine_deck("contact point (5.3, 3, 0, 4, 0.5)"))
    assert node_axis(unaligned, 0) == node_axis(plain, 0)
    assert node_axis(unaligned, 1) != node_axis(plain, 1)
    fine = ".contact Gp 0.95 0.95 1.05 1.05 nx=1 ny=1 ratio=2"
    both = parse(plane_deck(REFINE_PLANE + "\n+ contact point (5.3, 3, 0, 4, 0.5)", fine))
    alone = parse(plane_deck(REFINE_PLANE, fine))
    assert node_axis(both, 0) == node_axis(alone, 0)
    assert node_axis(both, 1) != node_axis(alone, 1)


def test_contact_line_met_on_one_axis_leaves_that_axis_alone():
    plain = parse(plane_deck(REFINE_PLANE))
    strip = parse(refine_deck("contact line (2, 3.1, 0, 8, 3.1, 0, 0.5, 3)"))
    assert same(strip, parse(plane_deck(REFINE_PLANE, ".contact Gp 1.75 0 8.25 6 nx=13 ny=3 ratio=2")))
    assert node_axis(strip, 1) == node_axis(plain, 1) and node_axis(strip, 0) != node_axis(plain, 0)
    column = parse(refine_deck("contact line (5.3, 1, 0, 5.3, 5, 0, 4, 0.5)"))
    assert same(column, parse(plane_deck(REFINE_PLANE, ".contact Gp 0 0.75 10 5.25 nx=5 ny=9 ratio=2")))
    assert node_axis(column, 0) == node_axis(plain, 0)


def test_contact_point_at_the_plane_edge_keeps_its_cell_size():
    edge = parse(refine_deck("contact point (0.8, 3, 0, 1, 1)"))
    directive = parse(plane_deck(REFINE_PLANE, ".contact Gp 0.3 2.5 1.3 3.5 nx=1 ny=1 ratio=2"))
    assert same_mesh(edge, directive)
    parse(refine_deck("contact point (0, 0, 0, 0.5, 0.5)"))
    parse(refine_deck("contact point (10, 6, 0, 0.5, 0.5)"))


def test_contact_line_along_an_axis_is_a_padded_strip():
    strip = parse(refine_deck("contact line (2, 3, 0, 8, 3, 0, 0.5, 0.25)"))
    assert same(strip, parse(plane_deck(REFINE_PLANE, ".contact Gp 1.75 2.875 8.25 3.125 nx=13 ny=1 ratio=2")))
    assert same(parse(refine_deck("contact line (8, 3, 0, 2, 3, 0, 0.5, 0.25)")), strip)
    assert same(parse(refine_deck("contact line (5, 3, 0, 5, 3, 0, 0.5, 0.25)")),
                parse(refine_deck("contact point (5, 3, 0, 0.5, 0.25)")))


def test_contact_line_on_a_diagonal_refines_its_bounding_box():
    diagonal = parse(refine_deck("contact line (2, 1, 0, 8, 5, 0, 0.5, 0.5)"))
    assert same(diagonal, parse(plane_deck(REFINE_PLANE, ".contact Gp 1.75 0.75 8.25 5.25 nx=13 ny=9 ratio=2")))
    mesh = PL.GroundPlane((0.0, 0.0), (10e-3, 6e-3), 0.02e-3, 0.04e-3, 5, 3, 5.8e7, [],
                          [PL.ContactRegion.new((1.75e-3, 0.75e-3), (8.25e-3, 5.25e-3), (13, 9), 2.0)]).mesh()
    for step in range(601):
        t = step / 600.0
        x, y = 2e-3 + t * 6e-3, 1e-3 + t * 4e-3
        i = next(k for k in range(mesh.nx()) if mesh.x[k] - 1e-15 <= x <= mesh.x[k + 1] + 1e-15)
        j = next(k for k in range(mesh.ny()) if mesh.y[k] - 1e-15 <= y <= mesh.y[k + 1] + 1e-15)
        assert mesh.dx(i) <= 0.5e-3 + 1e-15 and mesh.dy(j) <= 0.5e-3 + 1e-15


@pytest.mark.parametrize("clause,what", [
    ("contact point (5, 3, 0)", "takes 5 values"),
    ("contact point (5, 3, 0, 1, 1, 1)", "takes 5 values"),
    ("contact line (1, 1, 0, 9, 5, 0, 0.2)", "takes 8 values"),
    ("contact point (5, 3, 0, 0, 1)", "xcell=0"),
    ("contact point (5, 3, 0, 1, -1)", "ycell=-0.001"),
    ("contact line (1, 1, 0, 9, 5, 0, 0.2, 0)", "ycell=0"),
    ("contact point (5, 3, 3, 1, 1)", "is not in ground plane 'Gp'"),
    ("contact line (1, 1, 0, 9, 5, 3, 0.2, 0.2)", "is not in ground plane 'Gp'"),
    ("contact point (11, 3, 0, 1, 1)", "is outside ground plane 'Gp'"),
    ("contact line (1, 1, 0, 9, 7, 0, 0.2, 0.2)", "is outside ground plane 'Gp'"),
    ("contact circle (5, 3, 0, 1)", "'contact circle' is not supported"),
    ("contact trace (1, 3, 0, 9, 3, 0, 0.2)", "takes 8 values"),
    ("contact trace (1, 3, 0, 9, 3, 0, 0.2, 1, 1)", "takes 8 values"),
    ("contact trace (1, 3, 0, 9, 3, 0, 0, 1)", "trace_width=0"),
    ("contact trace (1, 3, 0, 9, 3, 0, -0.2, 1)", "trace_width=-0.0002"),
    ("contact trace (1, 3, 0, 9, 3, 0, 0.2, 0)", "scale_factor=0"),
    ("contact trace (1, 3, 0, 9, 3, 0, 0.2, -1)", "scale_factor=-1"),
    ("contact trace (5, 3, 0, 5, 3, 0, 0.2, 1)", "zero length"),
    ("contact trace (1, 3, 0, 9, 3, 3, 0.2, 1)", "is not in ground plane 'Gp'"),
    ("contact trace (1, 3, 0, 11, 3, 0, 0.2, 1)", "is outside ground plane 'Gp'"),
    ("contact trace (1, 1, 0, 9, 5, 0, 0.2, 1)", "contact line (x0, y0, z0, x1, y1, z1, xcell, ycell)"),
    ("contact equiv_rect (5, 3, 0, 2, 2)", "names the node it ties"),
    ("contact connection (5, 3, 0, 2, 2, 2)", "names the node it ties"),
    ("contact equiv_rect Xpad (5, 3, 0, 2, 2)", "is not a node name"),
    ("contact equiv_rect Npad (4, 2, 0, 6, 4, 0)", "takes 5 values"),
    ("contact equiv_rect Npad (5, 3, 0, 0, 2)", "xwidth=0 must be > 0"),
    ("contact equiv_rect Npad (5, 3, 0, 2, -1)", "ywidth=-0.001 must be > 0"),
    ("contact equiv_rect Npad (5, 3, 3, 2, 2)", "is not in ground plane 'Gp'"),
    ("contact equiv_rect Npad (50, 3, 0, 2, 2)", "is outside ground plane 'Gp'"),
    ("contact connection Npad (5, 3, 0, 2, 2)", "takes 6 values"),
    ("contact connection Npad (5, 3, 0, 2, 2, 1)", "ratio=1 must be > 1"),
    ("hole rect Npad (0.5, 4.5, 0, 1.5, 5.5, 0)", "'hole rect' takes no node name"),
    ("contact rect Npad (4, 2, 0, 6, 4, 0)", "'contact rect' takes no node name"),
    ("contact equiv_rect Nt (5, 3, 0, 2, 2)", "twice"),
    ("contact equiv_rect Npad (2, 2, 0, 0.5, 0.5)", "covers no live cell"),
])
def test_clause_errors_name_what_they_reject_on_the_statement_line(clause, what):
    e = error_of(refine_deck(clause))
    assert what in str(e), str(e)
    # the statement's line; a node declared twice is reported where the
    # second declaration is read
    assert e.line == (6 if what == "twice" else 3), str(e)


# -- contact trace -----------------------------------------------------------
def test_contact_trace_along_x_is_the_documented_five_lines():
    trace = parse(refine_deck("contact trace (2, 3, 0, 8, 3, 0, 0.4, 1)"))
    lines = parse(refine_deck("contact line (2, 3, 0, 8, 3, 0, 6, 0.2)\n"
                              "+ contact line (2, 3.2, 0, 8, 3.2, 0, 6, 0.2)\n"
                              "+ contact line (2, 2.8, 0, 8, 2.8, 0, 6, 0.2)\n"
                              "+ contact line (2, 3.6, 0, 8, 3.6, 0, 6, 0.4)\n"
                              "+ contact line (2, 2.4, 0, 8, 2.4, 0, 6, 0.4)"))
    assert same_mesh(trace, lines)
    assert not same(trace, parse(plane_deck(REFINE_PLANE)))
    assert same(parse(refine_deck("contact trace (2, 3, 0, 8, 3, 0, 0.4, 7)")), trace)
    assert same(parse(refine_deck("contact trace (8, 3, 0, 2, 3, 0, 0.4, 1)")), trace)


def test_contact_trace_along_y_refines_across_it_only():
    trace = parse(refine_deck("contact trace (5, 1, 0, 5, 5, 0, 0.4, 3)"))
    lines = parse(refine_deck("contact line (5, 1, 0, 5, 5, 0, 0.2, 4)\n"
                              "+ contact line (5.2, 1, 0, 5.2, 5, 0, 0.2, 4)\n"
                              "+ contact line (4.8, 1, 0, 4.8, 5, 0, 0.2, 4)\n"
                              "+ contact line (5.6, 1, 0, 5.6, 5, 0, 0.4, 4)\n"
                              "+ contact line (4.4, 1, 0, 4.4, 5, 0, 0.4, 4)"))
    assert same_mesh(trace, lines)
    short = parse(refine_deck("contact trace (5, 2, 0, 5, 3, 0, 0.4, 1)"))
    short_lines = parse(refine_deck("contact line (5, 2, 0, 5, 3, 0, 0.2, 1)\n"
                                    "+ contact line (5.2, 2, 0, 5.2, 3, 0, 0.2, 1)\n"
                                    "+ contact line (4.8, 2, 0, 4.8, 3, 0, 0.2, 1)\n"
                                    "+ contact line (5.6, 2, 0, 5.6, 3, 0, 0.4, 1)\n"
                                    "+ contact line (4.4, 2, 0, 4.4, 3, 0, 0.4, 1)"))
    assert same_mesh(short, short_lines)


def test_contact_trace_along_the_plane_edge_is_accepted():
    edge = parse(refine_deck("contact trace (1, 0.1, 0, 9, 0.1, 0, 0.4, 1)"))
    assert not same(edge, parse(plane_deck(REFINE_PLANE)))
    assert any(abs(n[1] - 0.1e-3) <= 0.1e-3 + 1e-15 for n in edge.nodes)
    assert "is outside ground plane 'Gp'" in str(error_of(refine_deck("contact line (1, -0.5, 0, 9, -0.5, 0, 8, 0.4)")))


# -- named contact areas -----------------------------------------------------
AREA_DECK = """.units mm
.default sigma=5.8e4
Gp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=6 z3=0
+ thick=0.035 seg1=5 seg2=3
+ %s
Nt x=5 y=3 z=0.5
Nb x=5 y=3 z=0.2
Ev Nt Nb w=0.2 h=0.2
.equiv Nb Npad
.external Nt Nb
.freq fmin=1 fmax=1 ndec=1
.end
"""


def test_equiv_rect_ties_its_rectangle_to_the_node_it_names():
    deck = parse(AREA_DECK % "contact equiv_rect Npad (5, 3, 0, 6, 3)")
    plane = PL.GroundPlane((0.0, 0.0), (10e-3, 6e-3), 0.035e-3 / 2.0, 0.035e-3, 5, 3, 5.8e7,
                           equipotentials=[PL.Equipotential.centred((5e-3, 3e-3), (6e-3, 3e-3))])
    g = A.Geometry()
    centres = plane.build_into(g)
    tie = plane.equipotential_node(centres, 0)
    assert [centres[i][1] for i in (1, 2, 3)] == [tie] * 3
    # 15 cells in 13 nodes plus the via's top; 22 bars less the 2 inside the
    # patch, plus the via
    assert len(deck.nodes) == 13 + 1 and len(deck.segments) == 22 - 2 + 1
    assert len(deck.nodes) == len(g.nodes) + 1 and len(deck.segments) == len(g.segments) + 1
    assert deck.segments[-1]["b"] == tie
    assert abs(deck.nodes[tie][0] - 5e-3) < 1e-12 and abs(deck.nodes[tie][1] - 3e-3) < 1e-12


def test_a_contact_area_node_can_be_named_by_a_port():
    deck = parse(".units mm\n.default sigma=5.8e4\nGp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=6 z3=0\n"
                 "+ thick=0.035 seg1=5 seg2=3\n+ contact equiv_rect Npad (5, 3, 0, 6, 3)\n+ Nfar (9, 5, 0)\n"
                 ".external Npad Nfar\n.freq fmin=1 fmax=1 ndec=1\n.end\n")
    assert len(deck.nodes) == 13 and len(deck.ports) == 1
    assert deck.ports[0][0] != deck.ports[0][1]


def test_connection_is_an_equiv_rect_plus_a_decay_rect():
    shorthand = parse(AREA_DECK % "contact connection Npad (5, 3, 0, 2, 2, 4)")
    written_out = parse(AREA_DECK % ("contact equiv_rect Npad (5, 3, 0, 2, 2)\n"
                                     "+ contact decay_rect (5, 3, 0, 2, 2, 0.5, 0.5, -1, -1)"))
    assert same(shorthand, written_out)
    plane = PL.GroundPlane((0.0, 0.0), (10e-3, 6e-3), 0.035e-3 / 2.0, 0.035e-3, 5, 3, 5.8e7,
                           contacts=[PL.ContactRegion.graded_per_axis((4e-3, 2e-3), (6e-3, 4e-3), (4, 4),
                                                                      (1.0 / 0.75, 1.0 / 0.75))],
                           equipotentials=[PL.Equipotential.centred((5e-3, 3e-3), (2e-3, 2e-3))])
    g = A.Geometry()
    centres = plane.build_into(g)
    tie = plane.equipotential_node(centres, 0)
    assert sum(node == tie for column in centres for node in column) == 16
    assert len(shorthand.nodes) == len(g.nodes) + 1 and len(shorthand.segments) == len(g.segments) + 1


# -- the initial grid ----------------------------------------------------------
G_HEAD = "Gp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=6 z3=0\n+ thick=0.04 "


def test_the_initial_grid_is_seg1_and_seg2_and_is_not_transposed():
    grid = parse(plane_deck(G_HEAD + "contact initial_grid (5, 3)"))
    segments = parse(plane_deck(G_HEAD + "seg1=5 seg2=3"))
    assert same(grid, segments)
    assert not same(grid, parse(plane_deck(G_HEAD + "seg1=3 seg2=5")))
    rotated = parse(plane_deck("Gp x1=0 y1=0 z1=0 x2=0 y2=6 z2=0 x3=10 y3=6 z3=0\n"
                               "+ thick=0.04 contact initial_grid (3, 5)"))
    assert same(rotated, segments)
    assert same(parse(plane_deck(G_HEAD + "file=NONE contact initial_grid (5, 3)")), segments)


def test_the_meshed_initial_grid_holes_the_even_indexed_cells():
    meshed = parse(plane_deck(G_HEAD + "contact initial_mesh_grid (5, 3)"))
    by_hand = parse(plane_deck(G_HEAD + "seg1=5 seg2=3\n+ hole point (3, 3, 0)\n+ hole point (7, 3, 0)"))
    assert same(meshed, by_hand)
    assert len(parse(plane_deck(G_HEAD + "contact initial_grid (5, 3)")).segments) > len(meshed.segments)
    reversed_ = parse(plane_deck("Gp x1=10 y1=6 z1=0 x2=0 y2=6 z2=0 x3=0 y3=0 z3=0\n"
                                 "+ thick=0.04 contact initial_mesh_grid (5, 3)"))
    assert same(reversed_, meshed)


def test_the_meshed_initial_grid_numbers_cells_from_the_p1_corner():
    meshed = parse(plane_deck(G_HEAD + "contact initial_mesh_grid (4, 2)"))
    assert same(meshed, parse(plane_deck(G_HEAD + "seg1=4 seg2=2\n+ hole point (3.75, 4.5, 0)\n"
                                                  "+ hole point (8.75, 4.5, 0)")))
    far = "Gp x1=10 y1=6 z1=0 x2=0 y2=6 z2=0 x3=0 y3=0 z3=0\n+ thick=0.04 "
    reversed_ = parse(plane_deck(far + "contact initial_mesh_grid (4, 2)"))
    assert same(reversed_, parse(plane_deck(far + "seg1=4 seg2=2\n+ hole point (6.25, 1.5, 0)\n"
                                                  "+ hole point (1.25, 1.5, 0)")))
    assert not same(reversed_, meshed)


def test_the_meshed_initial_grid_of_a_single_row_has_no_holes():
    assert same(parse(plane_deck(G_HEAD + "contact initial_mesh_grid (5, 1)")),
                parse(plane_deck(G_HEAD + "seg1=5 seg2=1")))


@pytest.mark.parametrize("body,what", [
    ("seg1=5 seg2=3 contact initial_grid (5, 3)", "both set this plane's cell counts"),
    ("contact initial_grid (5, 3) seg1=5", "both set this plane's cell counts"),
    ("contact initial_mesh_grid (5, 3) seg2=3", "both set this plane's cell counts"),
    ("contact initial_grid (5, 3) contact initial_mesh_grid (5, 3)", "has already set"),
    ("contact initial_grid (5)", "takes 2 values"),
    ("contact initial_grid (5, 0)", "must be >= 1"),
    ("contact initial_grid (5, 2.5)", "not a valid"),
    ("seg1=5", "has no 'seg2'"),
    ("seg1=5 seg2=3 file=plane.hier", "'file=plane.hier'"),
    ("seg1=5 seg2=3 rh=2", "'rh'"),
    ("seg1=5 seg2=3 nx=2", "extension form"),
    ("seg1=5 seg2=3 bogus=1", "unknown ground-plane parameter 'bogus'"),
])
def test_the_initial_grid_and_the_plane_fields_reject_what_they_cannot_read(body, what):
    e = error_of(plane_deck(G_HEAD + body))
    assert what in str(e) and e.line == 3, str(e)


# -- segwid ------------------------------------------------------------------------
def bar_widths(problem, plane_bars):
    """Widths of the plane's x- and y-directed bars (the first segments)."""
    xs, ys = [], []
    for s in problem.segments[:plane_bars]:
        a, b = problem.nodes[s["a"]], problem.nodes[s["b"]]
        (xs if abs(b[0] - a[0]) > abs(b[1] - a[1]) else ys).append(s["width"])
    return xs, ys


def test_segwid_narrows_the_bars_of_its_own_direction_only():
    square = "Gp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=10 z3=0\n+ thick=0.04 seg1=4 seg2=4 "
    plain = parse(plane_deck(square))
    bars = len(plain.segments) - 1
    px, py = bar_widths(plain, bars)
    assert all(abs(w - 2.5e-3) < 1e-12 for w in px + py)
    for extra, wx, wy in [("segwid1=0.5 segwid2=0.5", 0.5e-3, 0.5e-3), ("segwid1=0.5", 0.5e-3, 2.5e-3),
                          ("segwid2=0.5", 2.5e-3, 0.5e-3), ("segwid2=3", 2.5e-3, 2.5e-3)]:
        deck = parse(plane_deck(square + extra))
        x, y = bar_widths(deck, bars)
        assert (len(x), len(y)) == (len(px), len(py)) and len(deck.segments) == len(plain.segments)
        assert all(abs(w - wx) < 1e-12 for w in x) and all(abs(w - wy) < 1e-12 for w in y), extra
    rotated = parse(plane_deck("Gp x1=0 y1=0 z1=0 x2=0 y2=10 z2=0 x3=10 y3=10 z3=0\n"
                               "+ thick=0.04 seg1=4 seg2=4 segwid1=0.5"))
    x, y = bar_widths(rotated, bars)
    assert all(abs(w - 0.5e-3) < 1e-12 for w in y) and all(abs(w - 2.5e-3) < 1e-12 for w in x)
    for extra in ("segwid1=0.5 file=NONE", "segwid1=0.5 contact point (5, 5, 0, 1, 1)"):
        assert "'segwid1'" in str(error_of(plane_deck(square + extra)))


# -- relx / rely / relz -----------------------------------------------------------
def rel_deck(d, fields):
    """Every in-plane coordinate of every clause kind moved by ``d``; the
    corner points stay (metres, so every sum is exact in binary)."""
    def p(x, y, z):
        return "%r, %r, %r" % (x + d[0], y + d[1], z + d[2])
    return (".units m\nG1 x1=0 y1=0 z1=0 x2=16 y2=0 z2=0 x3=16 y3=8 z3=0\n"
            "+ thick=0.5 seg1=8 seg2=4 sigma=1e6 %s\n"
            "+ N1 (%s)\n+ N2 (%s)\n+ hole rect (%s, %s)\n+ hole point (%s)\n+ hole circle (%s, 0.5)\n"
            "+ contact rect (%s, 2, 2, 0.5, 0.5)\n+ contact rect (%s, %s)\n"
            "+ contact decay_rect (%s, 1, 1, 0.25, 0.25, -1, -1)\n+ contact point (%s, 0.5, 0.5)\n"
            "+ contact line (%s, %s, 0.5, 0.5)\n+ contact trace (%s, %s, 0.25, 1)\n"
            "+ contact equiv_rect Na (%s, 1, 1)\n+ contact connection Nb (%s, 1, 1, 2)\n"
            ".external N1 N2\n.external Na Nb\n.freq fmin=1 fmax=1 ndec=1\n.end\n"
            % (fields, p(2.0, 2.0, 0.0), p(14.0, 4.0, 0.0), p(12.0, 6.0, 0.0), p(13.0, 7.0, 0.0),
               p(14.0, 1.0, 0.0), p(1.0, 7.0, 0.0), p(4.0, 4.0, 0.0), p(8.0, 1.0, 0.0), p(9.0, 2.0, 0.0),
               p(6.0, 6.0, 0.0), p(10.0, 4.0, 0.0), p(2.0, 5.0, 0.0), p(4.0, 5.0, 0.0), p(8.0, 3.0, 0.0),
               p(12.0, 3.0, 0.0), p(12.0, 4.0, 0.0), p(4.0, 1.0, 0.0)))


def test_rel_offset_equals_the_pre_shifted_deck():
    offset = (0.5, 0.25, 0.125)
    rel = parse(rel_deck((0.0, 0.0, 0.0), "relx=0.5 rely=0.25 relz=0.125"))
    assert same(rel, parse(rel_deck(offset, "")))
    assert not same(rel, parse(rel_deck((0.0, 0.0, 0.0), "")))
    for axis, field in enumerate(("relx=0.5", "rely=0.25", "relz=0.125")):
        d = [0.0, 0.0, 0.0]
        d[axis] = offset[axis]
        assert same(parse(rel_deck((0.0, 0.0, 0.0), field)), parse(rel_deck(d, ""))), field
    # written after the clauses, and repeated: the last value wins everywhere
    after = rel_deck((0.0, 0.0, 0.0), "").replace("\n.external N1 N2", "\n+ rely=0.25 relx=0.5\n.external N1 N2")
    expected = parse(rel_deck((0.5, 0.25, 0.0), ""))
    assert same(parse(after), expected)
    repeated = rel_deck((0.0, 0.0, 0.0), "relx=7 rely=0.25").replace(
        "\n.external N1 N2", "\n+ relx=3\n+ relx = 0.5\n.external N1 N2")
    assert same(parse(repeated), expected)


def test_rel_offset_leaves_the_corner_points_alone():
    assert same(parse(plane_deck(REFINE_PLANE + " relx=0.3 rely=-0.2 relz=0.01")), parse(plane_deck(REFINE_PLANE)))


def test_every_clause_kind_meshes_a_plane_the_solver_accepts():
    """The all-clauses deck becomes an ordinary geometry: finite positive
    bar sizes, every segment of nonzero length, the two ports on distinct
    nodes."""
    deck = parse(rel_deck((0.0, 0.0, 0.0), ""))
    for s in deck.segments:
        a, b = deck.nodes[s["a"]], deck.nodes[s["b"]]
        assert s["width"] > 0 and s["height"] > 0 and math.dist(a, b) > 0
    assert len(deck.ports) == 2 and all(p != n for p, n, _ in deck.ports)
