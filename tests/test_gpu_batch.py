"""Batched sweeps of independent, unevenly sized systems (fh_batch_sweep):
results equal the systems' own sweeps, and errors name the system."""
import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spirals(fh):
    decks = F.random_spirals(6, seed=7)
    systems = [fh.MeshSystem.assemble(fh.Geometry.from_deck(d), d.ports, d.discretization) for d in decks]
    yield systems
    for s in systems:
        s.close()


def test_batch_equals_the_individual_sweeps(fh, spirals):
    freqs = [F.logspace(7, 10, 4) for _ in spirals]
    alone = [s.sweep(f, fh.Precision.FP64).impedance_ohm for s, f in zip(spirals, freqs)]
    batch = fh.batch_sweep(spirals, freqs, fh.Precision.FP64, concurrency=3)
    sizes = {s.counts()["internal_meshes"] for s in spirals}
    assert len(sizes) > 1  # uneven
    for a, b in zip(alone, batch):
        assert np.array_equal(a, b.impedance_ohm)


def test_batch_mixed_precision_matches_fp64(fh, spirals):
    freqs = [F.logspace(7, 10, 4 + k % 3) for k in range(len(spirals))]
    ref = fh.batch_sweep(spirals, freqs, fh.Precision.FP64, concurrency=2)
    mixed = fh.batch_sweep(spirals, freqs, fh.Precision.MIXED_BF16X3, concurrency=4)
    for r, m in zip(ref, mixed):
        rel = np.max(np.abs(m.impedance_ohm - r.impedance_ohm) / np.abs(r.impedance_ohm))
        assert rel < 1e-9, rel


def test_batch_reports_the_first_failing_system(fh, spirals):
    freqs = [[1e8] for _ in spirals]
    freqs[3] = [1e8, -1.0]
    freqs[5] = [float("nan")]
    with pytest.raises(fh.InvalidFrequency) as e:
        fh.batch_sweep(spirals, freqs, fh.Precision.FP64)
    assert e.value.info.detail == 3
