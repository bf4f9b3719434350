"""Coupling truncation (MeshSystem::assemble_with_coupling, solve.rs:703-766;
coupling.rs) at the solve level, on the two-island fixture of the
reference's own tests (fasterhenry/tests/coupling.rs): identities (a declared
coupling and the default reproduce the full assembly bit for bit), bounds the
test computes from the full assembly, warnings, errors, and that truncated
pairs are never evaluated.  The truncated mesh matrices are also checked
against the oracle's L with the dropped entries zeroed."""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu

FREQ = 1e9


def z_of(fh, deck, coupling=None):
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization,
                                coupling=coupling) as s:
        return s.impedance(FREQ), [str(w) for w in s.truncation_warnings()], s.kept_pairs(), fh.fill_stats(s)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(a)


def test_distant_islands_survive_truncation(fh):
    deck, groups = F.two_islands(11.0 * F.ISLAND_EXTENT - F.ISLAND_SIDE)
    full, _, _, _ = z_of(fh, deck)
    trunc, warnings, _, _ = z_of(fh, deck, fh.Coupling.truncated(groups))
    assert warnings == []
    assert rel(full, trunc) < 1e-3
    for i in range(2):
        assert abs(full[i, i] - trunc[i, i]) / abs(full[i, i]) < 1e-3
    assert full[0, 1] != 0
    assert trunc[0, 1] == 0 and trunc[1, 0] == 0
    assert abs(full[0, 1]) / abs(full[0, 0]) < 1e-3


def test_near_islands_warn_and_the_dropped_term_matters(fh):
    deck, groups = F.two_islands(0.5 * F.ISLAND_EXTENT)
    full, _, _, _ = z_of(fh, deck)
    trunc, warnings, _, _ = z_of(fh, deck, fh.Coupling.truncated(groups))
    assert len(warnings) == 1
    for token in ("'a'", "'b'", "truncat"):
        assert token in warnings[0]
    assert abs(full[0, 1]) / abs(full[0, 0]) > 1e-3
    assert rel(full, trunc) > 1e-3


def test_declared_coupling_and_the_default_reproduce_the_full_assembly(fh):
    deck, groups = F.two_islands(0.5 * F.ISLAND_EXTENT)
    ref, _, _, _ = z_of(fh, deck)
    default, w1, _, _ = z_of(fh, deck, fh.Coupling.all_pairs())
    declared, w2, _, _ = z_of(fh, deck, fh.Coupling.truncated(groups).coupled("a", "b"))
    assert np.array_equal(default, ref) and np.array_equal(declared, ref)
    assert w1 == [] and w2 == []


def test_untagged_segments_share_the_default_group(fh):
    deck, groups = F.two_islands(11.0 * F.ISLAND_EXTENT - F.ISLAND_SIDE)
    groups = [""] * 4 + groups[4:]
    full, _, _, _ = z_of(fh, deck)
    trunc, _, _, _ = z_of(fh, deck, fh.Coupling.truncated(groups))
    assert trunc[0, 1] == 0
    assert rel(full, trunc) < 1e-3


def test_truncated_pairs_are_never_evaluated(fh):
    deck, groups = F.two_islands(F.ISLAND_EXTENT)
    _, _, (kept_full, total), st_full = z_of(fh, deck)
    _, _, (kept, total2), st = z_of(fh, deck, fh.Coupling.truncated(groups))
    assert total == total2 == 16 * 17 // 2 and kept_full == total
    assert kept == total - 8 * 8
    assert st["truncated"] == 64 and st_full["truncated"] == 0
    evaluated = st["point_quadrature"] + st["closed_form"] + st["aligned_quadrature"] + st["sampled"]
    assert evaluated + st["orthogonal"] == kept


def test_truncated_mesh_matrices_match_the_masked_oracle(fh, oracle):
    deck, groups = F.two_islands(0.5 * F.ISLAND_EXTENT)
    fil, per = oracle.discretize(deck)
    L = oracle.fill(fil)
    seg = np.repeat(np.arange(len(per)), per)
    g = np.array([groups[s] for s in seg])
    L[g[:, None] != g[None, :]] = 0.0
    row_ptr, cols, signs, _ = oracle.mesh(deck, per)
    M = np.zeros((len(row_ptr) - 1, len(fil)))
    for r in range(len(row_ptr) - 1):
        for k in range(row_ptr[r], row_ptr[r + 1]):
            M[r, cols[k]] += signs[k]
    with fh.MeshSystem.assemble(fh.Geometry.from_deck(deck), deck.ports, deck.discretization,
                                coupling=fh.Coupling.truncated(groups)) as s:
        _, Lm = s.mesh_matrices()
    ref = M @ L @ M.T
    assert np.max(np.abs(Lm - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_coupling_errors(fh):
    deck, groups = F.two_islands(F.ISLAND_EXTENT)
    g = fh.Geometry.from_deck(deck)
    with pytest.raises(fh.CouplingError) as e:
        fh.MeshSystem.assemble(g, deck.ports, deck.discretization, coupling=fh.Coupling.truncated(groups).coupled("a", "typo"))
    assert "typo" in str(e.value) and e.value.kind == "unknown_group"
    with pytest.raises(fh.CouplingError) as e:
        fh.MeshSystem.assemble(g, deck.ports, deck.discretization, coupling=fh.Coupling.truncated(groups + ["c"]))
    assert e.value.kind == "segment_count_mismatch"
    three = ["a", "a", "a", "b", "b", "b", "c", "c"]
    bad = fh.Coupling.truncated(three).coupled("a", "b").coupled("b", "c")
    with pytest.raises(fh.CouplingError) as e:
        fh.MeshSystem.assemble(g, deck.ports, deck.discretization, coupling=bad)
    assert e.value.kind == "non_transitive" and "'a'" in str(e.value) and "'c'" in str(e.value)
    clique = bad.coupled("a", "c")
    with fh.MeshSystem.assemble(g, deck.ports, deck.discretization, coupling=clique) as s:
        assert s.kept_pairs()[0] == s.kept_pairs()[1]
