"""The loop basis (mesh.rs:170-361) against what any correct mesh formulation
must satisfy, checked without the oracle: every internal row is a closed
loop (the signed branch incidences cancel at every node: KVL), port row p is
a path from the port's first node to its second, the internal rows are
independent and there are exactly E - V + C of them (the cycle rank of the
filament multigraph: branches, nodes used, connected components), and every
coefficient is +-1.  The bit equality with the oracle's loop rows (in
test_host_model.py) then fixes which basis it is."""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F


def ring_deck():
    nodes = [(0, 0, 0), (1e-3, 0, 0), (1e-3, 1e-3, 0), (0, 1e-3, 0), (0, 2e-3, 0)]
    segs = [F.segment(0, 1, 1e-4, 2e-5), F.segment(1, 2, 1e-4, 2e-5), F.segment(2, 3, 1e-4, 2e-5),
            F.segment(3, 0, 1e-4, 2e-5), F.segment(3, 4, 1e-4, 2e-5)]
    return F.Deck(nodes, segs, [(0, 2), (4, 1)], F.uniform(2, 2), name="ring")


def ladder_deck():
    """Two rails with three rungs (two independent conductor loops) and two
    ports, one filament per segment on the rungs' grid."""
    nodes = [(0, 0, 0), (1e-3, 0, 0), (2e-3, 0, 0), (0, 1e-3, 0), (1e-3, 1e-3, 0), (2e-3, 1e-3, 0)]
    segs = [F.segment(0, 1, 1e-4, 2e-5), F.segment(1, 2, 1e-4, 2e-5), F.segment(3, 4, 1e-4, 2e-5),
            F.segment(4, 5, 1e-4, 2e-5), F.segment(0, 3, 1e-4, 2e-5), F.segment(1, 4, 1e-4, 2e-5),
            F.segment(2, 5, 1e-4, 2e-5)]
    return F.Deck(nodes, segs, [(0, 3), (2, 5)], F.per_segment([(1, 1), (2, 1), (1, 2), (1, 1), (3, 1), (1, 1), (2, 2)]),
                  name="ladder")


def two_bars():
    nodes = [(i * 1e-3, 0, 0) for i in range(4)]
    segs = [F.segment(0, 1, 1e-4, 1e-4), F.segment(2, 3, 1e-4, 1e-4)]
    return F.Deck(nodes, segs, [(0, 1), (2, 3)], F.uniform(3, 2), "two_bars")


DECKS = [
    ring_deck, ladder_deck, two_bars,
    lambda: F.c1_spiral()[0],
    lambda: F.square_spiral(3, 10e-6, 5e-6, 2e-6, 200e-6, F.graded(5, 3, 2.0)),
    lambda: F.square_spiral(2, 10e-6, 5e-6, 2e-6, 120e-6, F.per_segment([(k % 3 + 1, k % 2 + 1) for k in range(8)])),
    lambda: F.meander_legs(3),
]


def components(n_nodes, edges):
    parent = list(range(n_nodes))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in edges:
        parent[find(a)] = find(b)
    used = {v for e in edges for v in e}
    return len({find(v) for v in used}), len(used)


@pytest.mark.parametrize("make", DECKS)
def test_loop_rows_are_kvl_loops_and_port_rows_are_paths(fh, make):
    deck = make()
    g = fh.Geometry.from_deck(deck)
    fil, per = fh.discretize(g, deck.discretization)
    rp, br, sg, ni = fh.mesh_matrix(g, per, deck.ports)
    n_nodes, n_fil = len(deck.nodes), len(fil)
    seg_of = np.repeat(np.arange(len(per)), per)
    ends = [(deck.segments[s]["a"], deck.segments[s]["b"]) for s in seg_of]
    rows = len(rp) - 1
    assert rows == ni + len(deck.ports)
    assert np.all(np.abs(sg) == 1.0)
    M = np.zeros((rows, n_fil))
    for r in range(rows):
        cols = br[rp[r]:rp[r + 1]]
        assert len(set(cols)) == len(cols)  # a branch at most once per row
        M[r, cols] = sg[rp[r]:rp[r + 1]]
    # node balance of each row: current along a filament leaves its first node
    inc = np.zeros((n_fil, n_nodes))
    for j, (a, b) in enumerate(ends):
        inc[j, a] -= 1.0
        inc[j, b] += 1.0
    bal = M @ inc
    assert np.all(bal[:ni] == 0.0)
    for p, (a, b) in enumerate(deck.ports):
        want = np.zeros(n_nodes)
        want[a] -= 1.0
        want[b] += 1.0
        assert np.array_equal(bal[ni + p], want), p
    # the internal rows are a basis of the cycle space
    c, v = components(n_nodes, ends)
    assert ni == n_fil - v + c
    if ni:
        assert np.linalg.matrix_rank(M[:ni]) == ni
