"""Batched sweeps of independent, unevenly sized systems (fh_batch_sweep):
results equal the systems' own sweeps, and errors name the system.  In the
mixed precisions every (system, frequency) runs in one persistent launch with
tile shapes from the autotuner, whose table lands in a JSON file."""
import json
import os
import tempfile

import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

pytestmark = pytest.mark.gpu

# The autotuner's table for this process goes to a fresh file (read once per
# process, before the first batched call).
CACHE = os.path.join(tempfile.mkdtemp(prefix="fhb_tune_"), "batch_tiles.json")
os.environ.setdefault("FH_AUTOTUNE_CACHE", CACHE)


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


def test_mixed_batch_is_one_launch_and_matches_fp64(fh):
    """Sixteen of the seeded C3 spirals x 6 frequencies: one persistent launch
    for all 96 factorizations and refinements, every Z within 1e-9 of the
    FP64 sweeps, the autotuner's table written."""
    decks = F.random_spirals(16, seed=2026)
    systems = [fh.MeshSystem.assemble(fh.Geometry.from_deck(d), d.ports, d.discretization) for d in decks]
    try:
        freqs = [F.logspace(7, 10, 6) for _ in systems]
        ref = fh.batch_sweep(systems, freqs, fh.Precision.FP64)
        fh.batch_sweep(systems, freqs, fh.Precision.MIXED_BF16X3)  # tunes the buckets it meets
        with fh.Profiler() as prof:
            mixed = fh.batch_sweep(systems, freqs, fh.Precision.MIXED_BF16X3)
            profile = prof.read()
        assert profile["batch"]["launches"] == 1, profile["batch"]
        assert profile["panel"]["launches"] == 0 and profile["gemm_tc"]["launches"] == 0
        for r, m in zip(ref, mixed):
            rel = np.max(np.abs(m.impedance_ohm - r.impedance_ohm) / np.abs(r.impedance_ohm))
            assert rel < 1e-9, rel
        path = os.environ["FH_AUTOTUNE_CACHE"]
        with open(path) as f:
            table = json.load(f)
        assert table["format"] == 1 and "sm_10" in table["device"]
        buckets = {(s.counts()["internal_meshes"] + 127) // 128 for s in systems}
        assert buckets <= {int(b) for b in table["buckets"]}
        assert all(0 <= v < 4 for v in table["buckets"].values())
    finally:
        for s in systems:
            s.close()


def test_mixed_batch_handles_dc_and_a_large_system(fh):
    """DC (real Z, exactly zero imaginary part) in the persistent launch, and a
    system above the batched order limit swept alongside by the per-system
    path."""
    small = F.random_spirals(3, seed=11)
    big = F.meander_legs(20)  # m = 1,160 > the batched limit
    decks = small + [big]
    systems = [fh.MeshSystem.assemble(fh.Geometry.from_deck(d), d.ports, d.discretization) for d in decks]
    try:
        freqs = [[0.0, 1e6, 1e9] for _ in systems]
        ref = fh.batch_sweep(systems, freqs, fh.Precision.FP64)
        mixed = fh.batch_sweep(systems, freqs, fh.Precision.MIXED_BF16X3)
        for r, m in zip(ref, mixed):
            assert np.all(m.impedance_ohm[0].imag == 0.0)
            rel = np.max(np.abs(m.impedance_ohm - r.impedance_ohm) / np.abs(r.impedance_ohm))
            assert rel < 1e-9, rel
    finally:
        for s in systems:
            s.close()
