"""Host model (no device): discretization, loop basis, errors, SolverChoice and
the output formats, checked against the oracle and the reference's rules."""
import ctypes
import json
import math
import os
import re

import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

DECKS = [
    lambda: F.c1_spiral()[0],
    lambda: F.c2_meander()[0],
    lambda: F.c4_spiral(0.5, 2.0),
    lambda: F.square_spiral(3, 10e-6, 5e-6, 2e-6, 200e-6, F.graded(5, 3, 2.0)),
    lambda: F.square_spiral(2, 10e-6, 5e-6, 2e-6, 120e-6, F.per_segment_graded([(3, 2, 1.5, 1.0)] * 8)),
    lambda: F.square_spiral(2, 10e-6, 5e-6, 2e-6, 120e-6, F.per_segment([(k % 3 + 1, k % 2 + 1) for k in range(8)])),
]


def ring_deck():
    """A closed square ring plus a tail (one conductor loop), 2 ports."""
    nodes = [(0, 0, 0), (1e-3, 0, 0), (1e-3, 1e-3, 0), (0, 1e-3, 0), (0, 2e-3, 0)]
    segs = [F.segment(0, 1, 1e-4, 2e-5), F.segment(1, 2, 1e-4, 2e-5), F.segment(2, 3, 1e-4, 2e-5),
            F.segment(3, 0, 1e-4, 2e-5), F.segment(3, 4, 1e-4, 2e-5)]
    return F.Deck(nodes, segs, [(0, 2), (4, 1)], F.uniform(2, 2), name="ring")


@pytest.mark.parametrize("make", DECKS + [ring_deck])
def test_discretize_and_mesh_match_oracle_bitwise(fh, oracle, make):
    deck = make()
    g = fh.Geometry.from_deck(deck)
    fil, per = fh.discretize(g, deck.discretization)
    ofil, oper = oracle.discretize(deck)
    assert np.array_equal(fil, ofil)
    assert np.array_equal(per, oper)
    rp, br, sg, ni = fh.mesh_matrix(g, per, deck.ports)
    orp, obr, osg, oni = oracle.mesh(deck, oper)
    assert np.array_equal(rp, orp) and np.array_equal(br, obr) and np.array_equal(sg, osg) and ni == oni


def test_ring_has_one_conductor_loop(fh):
    deck = ring_deck()
    g = fh.Geometry.from_deck(deck)
    fil, per = fh.discretize(g, deck.discretization)
    rp, br, sg, ni = fh.mesh_matrix(g, per, deck.ports)
    assert ni == 5 * 3 + 1  # bundle loops + one link loop
    assert len(rp) - 1 == ni + 2


def test_uniform_grid_tiles_the_cross_section(fh):
    deck = F.Deck([(0, 0, 0), (10e-3, 0, 0)], [F.segment(0, 1, 1e-3, 35e-6)], [(0, 1)], F.uniform(5, 2))
    fil, _ = fh.discretize(fh.Geometry.from_deck(deck), deck.discretization)
    assert len(fil) == 10
    assert abs(np.sum(fil[:, 16] * fil[:, 17]) - 1e-3 * 35e-6) < 1e-12 * 1e-3 * 35e-6
    assert np.allclose(fil[:, 10:13], [0, 1, 0]) and np.allclose(fil[:, 13:16], [0, 0, 1])


def test_graded_grid_follows_the_progression(fh):
    deck = F.Deck([(0, 0, 0), (10e-3, 0, 0)], [F.segment(0, 1, 1e-3, 35e-6)], [(0, 1)], F.graded(1, 4, 3.0))
    fil, _ = fh.discretize(fh.Geometry.from_deck(deck), deck.discretization)
    assert abs(fil[0, 17] - 35e-6 / 8) < 1e-18 and abs(fil[1, 17] - 3 * 35e-6 / 8) < 1e-18


def test_geometry_errors(fh):
    g = fh.Geometry()
    with pytest.raises(fh.GeometryError):
        g.add_node((float("nan"), 0, 0))
    a, b = g.add_node((0, 0, 0)), g.add_node((1e-3, 0, 0))
    with pytest.raises(fh.GeometryError):
        g.add_segment(fh.SegmentDef(a, 5, 1e-4, 1e-5, 5.8e7))
    with pytest.raises(fh.GeometryError):
        g.add_segment(fh.SegmentDef(a, a, 1e-4, 1e-5, 5.8e7))
    with pytest.raises(fh.GeometryError):
        g.add_segment(fh.SegmentDef(a, b, -1e-4, 1e-5, 5.8e7))
    with pytest.raises(fh.GeometryError):
        g.add_segment(fh.SegmentDef(a, b, 1e-4, 1e-5, 0.0))
    with pytest.raises(fh.GeometryError):
        g.add_segment(fh.SegmentDef(a, b, 1e-4, 1e-5, 5.8e7, (1.0, 0.0, 0.0)))  # width dir along the segment
    assert g.add_segment(fh.SegmentDef(a, b, 1e-4, 1e-5, 5.8e7)) == 0


def test_discretize_errors(fh):
    g = fh.Geometry.from_parts([(0, 0, 0), (1e-3, 0, 0)], [fh.SegmentDef(0, 1, 1e-4, 1e-5, 5.8e7)])
    with pytest.raises(fh.DiscretizeError):
        fh.discretize(g, fh.Discretization.uniform(0, 2))
    with pytest.raises(fh.InvalidGrading):
        fh.discretize(g, fh.Discretization.graded(3, 3, 0.5))
    with pytest.raises(fh.InvalidGrading):
        fh.discretize(g, fh.Discretization.skin_depth(-1.0, 1.0, 2.0))
    with pytest.raises(fh.MeshError):
        fh.discretize(g, fh.Discretization.per_segment([(1, 1), (2, 2)]))
    with pytest.raises(fh.DiscretizeError):  # unusable graded grid: cells far too thin
        fh.discretize(g, fh.Discretization.graded(2, 60, 3.0))


def test_mesh_errors(fh):
    g = fh.Geometry.from_parts([(0, 0, 0), (1e-3, 0, 0), (5e-3, 0, 0), (6e-3, 0, 0)],
                               [fh.SegmentDef(0, 1, 1e-4, 1e-5, 5.8e7), fh.SegmentDef(2, 3, 1e-4, 1e-5, 5.8e7)])
    per = [1, 1]
    with pytest.raises(fh.MeshError):
        fh.mesh_matrix(g, per, [])
    with pytest.raises(fh.MeshError):
        fh.mesh_matrix(g, per, [(0, 9)])
    with pytest.raises(fh.MeshError):
        fh.mesh_matrix(g, per, [(1, 1)])
    with pytest.raises(fh.MeshError):
        fh.mesh_matrix(g, per, [(0, 3)])  # not connected
    rp, br, sg, ni = fh.mesh_matrix(g, per, [(0, 1)])
    assert ni == 0 and list(br) == [0] and list(sg) == [1.0]


def test_solver_choice_threshold(fh):
    auto = fh.SolverChoice.AUTO
    assert auto.resolve(0) == "dense"
    assert auto.resolve(fh.DENSE_PATH_MAX_FILAMENTS) == "dense"
    assert auto.resolve(fh.DENSE_PATH_MAX_FILAMENTS + 1) == "iterative"
    for n in [1, 10_000, 100_000]:
        assert fh.SolverChoice.DENSE.resolve(n) == "dense"
        assert fh.SolverChoice.ITERATIVE.resolve(n) == "iterative"


def sample_result(fh):
    z = np.array([[[0.0049 + 0j]], [[0.0051 + 0.0437j]]])
    return fh.SweepResult([fh.Port(0, 1, "trace")], [0.0, 1e6], z,
                          dict(nodes=2, segments=1, filaments=10, meshes=10, internal_meshes=9, ports=1),
                          dict(inductance_s=0.0004, assembly_s=0.0005, solve_s=0.0001, total_s=0.0006))


def test_sweep_json_matches_reference_schema(fh):
    text = sample_result(fh).to_json()
    # The document of result.rs:1-24 (serde_json formatting of f64).
    assert text.startswith('{"schema_version":1,"ports":[{"positive":0,"negative":1,"name":"trace"}],'
                           '"frequencies_hz":[0.0,1000000.0],"impedance_ohm":[[[{"re":0.0049,"im":0.0}]],'
                           '[[{"re":0.0051,"im":0.0437}]]]')
    doc = json.loads(text)
    assert doc["provenance"]["counts"]["internal_meshes"] == 9
    assert doc["provenance"]["timing"]["solve_s"] == 0.0001


@pytest.mark.parametrize("v,s", [(1e-7, "1e-7"), (1.5e21, "1.5e21"), (123456.0, "123456.0"), (0.001234, "0.001234"),
                                 (-2.5e-9, "-2.5e-9"), (1e16, "1e16"), (1e15, "1000000000000000.0")])
def test_json_float_format(fh, v, s):
    r = fh.SweepResult([fh.Port(0, 1)], [v], np.zeros((1, 1, 1), complex),
                       dict(nodes=0, segments=0, filaments=0, meshes=0, internal_meshes=0, ports=1))
    assert ('"frequencies_hz":[%s]' % s) in r.to_json()


def test_zc_mat_reads_back(fh, tmp_path):
    import scipy.io
    z = np.array([[[1 + 2j, 3 + 4j], [5 + 6j, 7 + 8j]], [[9 + 1j, 2 + 3j], [4 + 5j, 6 + 7j]]])
    r = fh.SweepResult([fh.Port(0, 1), fh.Port(2, 3)], [1e6, 1e9], z,
                       dict(nodes=4, segments=2, filaments=2, meshes=2, internal_meshes=0, ports=2))
    path = str(tmp_path / "Zc.mat")
    r.write_zc_mat(path)
    m = scipy.io.loadmat(path)
    assert np.allclose(m["freqs"], [[1e6, 1e9]])
    assert np.array_equal(m["Zc_1"], z[0]) and np.array_equal(m["Zc_2"], z[1])


def test_spice_subckt(fh):
    text = sample_result(fh).spice_subckt(1, "trace")
    lines = text.strip().split("\n")
    assert lines[0] == "* fasterhenry SPICE export: trace at 1.00000000000000000e6 Hz"
    assert lines[2] == ".subckt trace p1 n1"
    assert re.match(r"L1 p1 a0_0 6\.955\d+e-9$", lines[3])
    assert lines[4] == "H1_1 a0_0 a0_1 vsense1 5.10000000000000037e-3"
    assert lines[-1] == ".ends trace"
    dc = sample_result(fh).spice_subckt(0, "trace").split("\n")
    assert dc[3] == "L1 p1 a0_0 0.00000000000000000e0"
