"""The device near-pair search of the pFFT set-up (fh_near.cu) against the
oracle's restatement of the reference's near_pairs (pfft/near.rs:41-106):
identical rows (j >= i within the radius by the separating-axis gap,
ascending) once the orthogonal pairs, which the set-up does not list, are
dropped from the oracle's rows.  Random clouds (axis-aligned and in general
position, where the bins' candidate sets are wider than the kept pairs), a
meander, radii around and far beyond the filament size, and the edge cases
of one filament and of every pair being near."""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu


def expected(oracle, fil, radius):
    off, cols = oracle.near_pairs(fil, radius)
    rows = []
    for i in range(len(fil)):
        a = fil[i, 7:10]
        keep = []
        for j in cols[off[i]:off[i + 1]]:
            b = fil[j, 7:10]
            c = a[0] * b[0] + a[1] * b[1] + a[2] * b[2]
            if not abs(c) < 1e-14:
                keep.append(int(j))
        rows.append(keep)
    return rows


def device_rows(fh, fil, radius):
    off, cols = fh.near_pairs(fil, radius)
    return [[int(j) for j in cols[off[i]:off[i + 1]]] for i in range(len(fil))]


def filaments_of(fh, deck):
    f, _ = fh.discretize(fh.Geometry.from_deck(deck), deck.discretization)
    return f


@pytest.mark.parametrize("manhattan", [True, False])
@pytest.mark.parametrize("n,seed", [(1, 1), (300, 2), (1500, 3)])
def test_clouds_match_the_reference_search(fh, oracle, n, seed, manhattan):
    fil = filaments_of(fh, F.cloud_deck(n, manhattan, seed))
    span = np.ptp(fil[:, 0:3], axis=0).max() if n > 1 else 1e-3
    for radius in (0.02 * span, 0.1 * span, 3.0 * span):
        assert device_rows(fh, fil, radius) == expected(oracle, fil, radius)


def test_meander_matches_the_reference_search(fh, oracle):
    fil = filaments_of(fh, F.meander_legs(12))
    for radius in (5e-6, 4e-5, 2e-4):
        want = expected(oracle, fil, radius)
        got = device_rows(fh, fil, radius)
        assert got == want
        assert all(row and row[0] == i for i, row in enumerate(got))  # every row holds its diagonal
