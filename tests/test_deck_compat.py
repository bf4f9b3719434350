"""The deck reader's FastHenry compatibility mode
(fasterhenry_b200/problem.py ``parse_deck_reporting(text, fasthenry_compat=True)``),
pinned to the answers of the reference reader's compat tests
(fasterhenry-cli/src/inp.rs tests 4937-5036, 5926-6027, 6707-6758, 7351-7380,
7840-7860, 8070-8110, 8791-8860, 9571-9900): each FastHenry default is
applied with a warning on its line, and natively each stays an error.
Host-only."""
import pytest

from fasterhenry_b200 import problem as P

BODY = """.units m
n1 x=0 y=0 z=0
n2 x=1e-3 y=0 z=0
e1 n1 n2 w=1e-3 h=1e-4 sigma=5.8e7
.external n1 n2
.freq fmin=1e3 fmax=1e3 ndec=1
.end
"""


def compat(text):
    return P.parse_deck_reporting(text, fasthenry_compat=True)


def same(a, b):
    return a.to_json() == b.to_json()


def test_the_first_line_is_the_title():
    with pytest.raises(P.DeckError) as e:
        P.parse_deck("A two-node test trace\n" + BODY)
    assert e.value.line == 1
    deck, warnings = compat("A two-node   test trace\n" + BODY)
    assert deck.title == "A two-node test trace" and warnings == []
    assert same(deck, P.parse_deck(BODY)) or deck.nodes == P.parse_deck(BODY).nodes
    plain = P.parse_deck(BODY)
    assert deck.nodes == plain.nodes and deck.segments == plain.segments and deck.frequencies_hz == plain.frequencies_hz
    # whatever line 1 holds: a .units there is swallowed, and the deck reads
    # in metres with a warning
    deck, warnings = compat(BODY)
    assert deck.title == ".units m" and len(warnings) == 1 and "no .units" in warnings[0].message
    assert compat("* comment-looking title\n" + BODY)[0].title == "* comment-looking title"
    assert compat("prose title\n" + BODY.replace(".units m", ".units m\n.title explicit  name"))[0].title == \
        "explicit name"
    for first in ("", "   ", "\t "):
        assert compat(first + "\n" + BODY)[0].title is None


def test_compat_keeps_physical_line_numbers():
    with pytest.raises(P.DeckError) as e:
        compat("title\n" + BODY.replace("n2 x=1e-3", "n2 bogus=1"))
    assert e.value.line == 4
    with pytest.raises(P.DeckError) as e:
        compat("title\n+ more\n" + BODY)
    assert e.value.line == 2 and "continuation" in str(e.value)
    for text in ("just a title", "just a title\n", "just a title\n\n* note\n", ""):
        with pytest.raises(P.DeckError, match="no .end directive"):
            compat(text)


UNITS_DECK = """title
.units %s
n1 x=0 y=0 z=0
n2 x=1 y=0 z=0
e1 n1 n2 w=0.1 h=0.1 sigma=1
.external n1 n2
.freq fmin=1 fmax=1 ndec=1
.end
"""


@pytest.mark.parametrize("spelling,documented", [("meter", "m"), ("Metres", "m"), ("kilometers", "km"),
                                                 ("inch", "in"), ("INCHES", "in")])
def test_long_unit_spellings_read_at_their_scale_with_a_warning(spelling, documented):
    deck, warnings = compat(UNITS_DECK % spelling)
    assert same(deck, compat(UNITS_DECK % documented)[0])
    assert len(warnings) == 1 and warnings[0].line == 2 and "'%s'" % documented in warnings[0].message
    with pytest.raises(P.DeckError):
        P.parse_deck((UNITS_DECK % spelling).split("\n", 1)[1])


@pytest.mark.parametrize("spelling,reads", [("millimeters", "mils"), ("milli", "mils"), ("microns", "metres"),
                                            ("micrometre", "metres")])
def test_spellings_fasthenry_misreads_are_errors(spelling, reads):
    with pytest.raises(P.DeckError) as e:
        compat(UNITS_DECK % spelling)
    assert e.value.line == 2 and reads in str(e.value)


def test_missing_units_is_metres_and_repeated_units_apply_forward():
    with_units = UNITS_DECK % "m"
    without = with_units.replace(".units m\n", "", 1)
    deck, warnings = compat(without)
    assert same(deck, compat(with_units)[0])
    assert len(warnings) == 1 and warnings[0].line == 2 and "metres" in warnings[0].message
    text = """title
.units mm
.default z=0 w=1 h=1 sigma=5.8e4
n1 x=0 y=0
.units m
n2 x=0.01 y=0
e1 n1 n2
e2 n1 n2 sigma=5.8e7 w=1e-3 h=1e-3
.units cm
n3 x=2 y=0
e3 n2 n3
.external n1 n3
.freq fmin=1 fmax=1 ndec=1
.end
"""
    deck, warnings = compat(text)
    assert warnings == []
    e1, e2, e3 = deck.segments
    length = lambda s: abs(deck.nodes[s["b"]][0] - deck.nodes[s["a"]][0])  # noqa: E731
    assert abs(length(e1) - 0.01) < 1e-15 and abs(e1["width"] - 1e-3) < 1e-18 and abs(e1["sigma"] - 5.8e7) < 1e-3
    assert abs(e2["sigma"] - 5.8e7) < 1e-3 and abs(length(e3) - 0.01) < 1e-15
    with pytest.raises(P.DeckError, match="duplicate .units"):
        P.parse_deck(text.split("\n", 1)[1])


def conductivity_deck(unit, default_fields, segment_fields):
    return ("title\n.units %s\n.default %s\nn1 x=0 y=0 z=0\nn2 x=1 y=0 z=0\ne1 n1 n2 w=0.1 h=0.1 %s\n"
            ".external n1 n2\n.freq fmin=1 fmax=1 ndec=1\n.end\n" % (unit, default_fields, segment_fields))


@pytest.mark.parametrize("unit", ["m", "mm", "mils"])
def test_a_conductor_without_conductivity_is_copper(unit):
    deck, warnings = compat(conductivity_deck(unit, "", ""))
    assert deck.segments[0]["sigma"] == P.COPPER_SIGMA
    assert [(w.line, w.message) for w in warnings] == \
        [(6, "segment 'e1' has no conductivity; using copper (5.8e7 S/m, FastHenry default)")]
    with pytest.raises(P.DeckError, match="no conductivity"):
        P.parse_deck(conductivity_deck(unit, "", "").split("\n", 1)[1])
    # a plane without one too, in both G grammars
    plane = ("title\n.units mm\nGp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=6 z3=0 thick=0.04 seg1=5 seg2=3\n"
             "Gq 0 0 -1 10 6 -1 0.04 nx=5 ny=3\nNt x=5 y=3 z=0.5\nNb x=5 y=3 z=0\nEv Nt Nb w=0.2 h=0.2 sigma=5.8e4\n"
             ".external Nt Nb\n.freq fmin=1 fmax=1 ndec=1\n.end\n")
    deck, warnings = compat(plane)
    assert [w.line for w in warnings] == [3, 4] and all("ground plane" in w.message for w in warnings)
    assert all(s["sigma"] == P.COPPER_SIGMA for s in deck.segments[:-1])


@pytest.mark.parametrize("fields", [("sigma=5.8e4", ""), ("rho=0.5", ""), ("", "sigma=2")])
def test_copper_yields_to_any_given_conductivity(fields):
    deck, warnings = compat(conductivity_deck("mm", *fields))
    assert warnings == [] and same(deck, P.parse_deck(conductivity_deck("mm", *fields).split("\n", 1)[1]))


def test_equiv_of_a_node_with_itself_is_ignored_with_a_warning():
    text = BODY.replace(".external", ".equiv n1 n1\n.external")
    with pytest.raises(P.DeckError, match="with itself"):
        P.parse_deck(text)
    deck, warnings = compat("title\n" + text)
    assert len(warnings) == 1 and warnings[0].line == 6 and "ignored" in warnings[0].message
    assert same(deck, compat("title\n" + BODY)[0])


SWEEP = ".units m\nn1 x=0 y=0 z=0\nn2 x=1 y=0 z=0\ne1 n1 n2 w=1 h=1 sigma=1\n.external n1 n2\n.freq %s\n.end\n"


def sweep_of(fields):
    deck, warnings = compat("title\n" + SWEEP % fields)
    return deck.frequencies_hz, warnings


def test_compat_sweeps():
    assert P.parse_deck(SWEEP % "fmin=1 fmax=9.995 ndec=1").frequencies_hz == [1.0]
    f, w = sweep_of("fmin=1 fmax=9.995 ndec=1")
    assert f == [1.0, 10.0] and w == []
    assert sweep_of("fmin=1 fmax=9.98 ndec=1")[0] == [1.0]
    f, w = sweep_of("fmin=1e3 fmax=1e7 ndec=0")
    assert f == [1e3] and len(w) == 1 and w[0].line == 7 and "ndec=0.01" in w[0].message
    f, w = sweep_of("fmin=1e3 fmax=1e6")
    assert f == [1e3, 1e4, 1e5, 1e6] and len(w) == 1 and "ndec=1" in w[0].message
    f, w = sweep_of("fmin=1e6 fmax=1e3 ndec=1")
    assert f == [] and len(w) == 1 and "empty" in w[0].message
    f, w = sweep_of("fmin=1.0005e6 fmax=1e6 ndec=1")
    assert f == [1.0005e6] and "slack" in w[0].message
    for fields in ("fmin=1e3 fmax=1e7 ndec=-1", "fmin=1e3 fmax=1e3 ndec=-0.5"):
        with pytest.raises(P.DeckError, match="ndec"):
            sweep_of(fields)
    with pytest.raises(P.DeckError, match="no .freq"):
        compat("title\n" + (SWEEP % "x=1").replace(".freq x=1\n", ""))


REFINE_PLANE = "Gp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=6 z3=0\n+ thick=0.04 seg1=5 seg2=3"


def plane_deck(statement, extra=""):
    return ("title\n.units mm\n.default sigma=5.8e4\n%s\nNt x=5 y=3 z=0.5\nNb x=5 y=3 z=0\nEv Nt Nb w=0.2 h=0.2\n%s\n"
            ".external Nt Nb\n.freq fmin=1 fmax=1 ndec=1\n.end\n" % (statement, extra))


def same_mesh(a, b):
    return (len(a.nodes) == len(b.nodes) and len(a.segments) == len(b.segments) and
            all(abs(p[0] - q[0]) < 1e-15 and abs(p[1] - q[1]) < 1e-15 and p[2] == q[2]
                for p, q in zip(a.nodes, b.nodes)))


@pytest.mark.parametrize("clause,explicit,axes", [
    ("contact decay_rect (5, 3, 0, 2, 2, 4, 4, 2, 2)", "contact decay_rect (5, 3, 0, 2, 2, 1.98, 1.98, 2, 2)", "xy"),
    ("contact decay_rect (5, 3, 0, 2, 2, 4, 4, -1, -1)", "contact decay_rect (5, 3, 0, 2, 2, 1.98, 1.98, -1, -1)",
     "xy"),
    ("contact rect (5, 3, 0, 2, 2, 2, 0.5)", "contact rect (5, 3, 0, 2, 2, 1.98, 0.5)", "x"),
])
def test_a_contact_cell_as_wide_as_its_rectangle_is_clamped(clause, explicit, axes):
    deck, warnings = compat(plane_deck(REFINE_PLANE + "\n+ " + clause))
    by_hand, none = compat(plane_deck(REFINE_PLANE + "\n+ " + explicit))
    assert none == [] and same_mesh(deck, by_hand)
    clamps = [w for w in warnings if "clamped" in w.message]
    assert [w.message.split(": ")[2][0] for w in clamps] == list(axes)
    with pytest.raises(P.DeckError):
        P.parse_deck(plane_deck(REFINE_PLANE + "\n+ " + clause).split("\n", 1)[1])


@pytest.mark.parametrize("span,k", [((4.0, 4.0 / 3.0 ** 0.5), 1.0 / 3.0 ** 0.5), ((4.0 / 3.0 ** 0.5, 4.0),
                                                                               1.0 / 3.0 ** 0.5), ((3.0, 3.0), 1.0)])
def test_a_diagonal_trace_refines_its_padded_bounding_box(span, k):
    w, s, x0, y0 = 0.4, 4.0, 2.0, 1.0
    trace, warnings = compat(plane_deck(REFINE_PLANE + "\n+ contact trace (%r, %r, 0, %r, %r, 0, %r, %r)"
                                        % (x0, y0, x0 + span[0], y0 + span[1], w, s)))
    cell = w / 2.0 * s ** k
    rect, _ = compat(plane_deck(REFINE_PLANE + "\n+ contact rect (%r, %r, 0, %r, %r, %r, %r)"
                                % (x0 + span[0] / 2.0, y0 + span[1] / 2.0, span[0] + 3.0 * w, span[1] + 3.0 * w,
                                   cell, cell)))
    assert same_mesh(trace, rect)
    assert not same(trace, compat(plane_deck(REFINE_PLANE))[0])
    assert len(warnings) == 1 and "diagonal 'contact trace'" in warnings[0].message
    with pytest.raises(P.DeckError, match="not parallel to x or y"):
        P.parse_deck(plane_deck(REFINE_PLANE + "\n+ contact trace (2, 1, 0, 6, 3, 0, 0.4, 4)").split("\n", 1)[1])


def test_file_none_without_a_grid_is_a_single_cell():
    g = "Gp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=6 z3=0\n+ thick=0.04"
    bare, warnings = compat(plane_deck(g + " file=NONE"))
    assert same(bare, compat(plane_deck(g + " contact initial_grid (1, 1)"))[0])
    assert len(warnings) == 1 and warnings[0].line == 4 and "single cell" in warnings[0].message
    refine = "contact rect (5, 3, 0, 4, 4, 1, 1)"
    refined, _ = compat(plane_deck(g + " file=NONE " + refine))
    assert same(refined, compat(plane_deck(g + " contact initial_grid (1, 1) " + refine))[0])
    assert not same(refined, bare)
    assert compat(plane_deck(g + " file=NONE seg1=2 seg2=2"))[1] == []
    with pytest.raises(P.DeckError, match="seg1"):
        P.parse_deck(plane_deck(g + " file=NONE").split("\n", 1)[1])


def test_segwid_on_a_nonuniform_plane_is_ignored():
    square = "Gp x1=0 y1=0 z1=0 x2=10 y2=0 z2=0 x3=10 y3=10 z3=0\n+ thick=0.04 seg1=4 seg2=4 "
    for extra in ("segwid1=0.5 file=NONE", "segwid1=0.5 contact point (5, 5, 0, 1, 1)"):
        deck, warnings = compat(plane_deck(square + extra))
        assert any("'segwid1' is ignored" in w.message for w in warnings)
        plane_bars = len(deck.segments) - 1
        assert all(s["width"] > 0.5e-3 + 1e-9 for s in deck.segments[:plane_bars])


def test_an_empty_in_plane_node_coordinate_is_zero():
    def deck(node):
        return ("title\n.units m\nG1 x1=0 y1=0 z1=0 x2=16 y2=0 z2=0 x3=16 y3=8 z3=0\n"
                "+ thick=0.5 seg1=8 seg2=4 sigma=1e6 relx=2\n+ %s\n+ N2 (12, 4, 0)\n.external N1 N2\n"
                ".freq fmin=1 fmax=1 ndec=1\n.end\n" % node)
    for node, axis, zero in [("N1 (, 2, 0)", "x", "N1 (0, 2, 0)"), ("N1 (-2, , 0)", "y", "N1 (-2, 0, 0)"),
                             ("N1 (,2,0)", "x", "N1 (0,2,0)"), ("N1 (-2,2,)", "z", "N1 (-2,2,0)")]:
        expected, none = compat(deck(zero))
        assert none == []
        got, warnings = compat(deck(node))
        assert same(got, expected), node
        assert len(warnings) == 1 and "empty %s coordinate" % axis in warnings[0].message
        with pytest.raises(P.DeckError, match="empty coordinate"):
            P.parse_deck(deck(node).split("\n", 1)[1])
    for node in ("N1 (, , 0)", "N1 (, 2)"):
        with pytest.raises(P.DeckError, match="at most one empty"):
            compat(deck(node))
