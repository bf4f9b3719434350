"""Graded and skin-depth discretisation against answers worked out here from
the reference's stated rules and its own test fixtures, not from the
oracle's transliteration (which restates the same functions as the product
path, so a bit-equality test against it cannot catch a shared misreading).

* graded extents are total * w_i / sum(w) with w_i = ratio^min(i, n-1-i)
  (filament.rs:227-276); filament (i, j) sits at j * nw + i (filament.rs:
  288-300);
* the reference's own graded fixtures: the 4-cell 3:1 hand-computed grid
  (filament.rs:1016-1037), the geometric progression and symmetry
  (filament.rs:954-979), centred bundles whose outer faces lie on the
  surfaces (filament.rs:981-1014), the tiling (filament.rs:934-952), the
  surface-extent figures (filament.rs:1067-1076) and rigid motion
  (filament.rs:1039-1065);
* skin depth delta = 1 / sqrt(pi f mu0 sigma) (solve.rs:560-562); the count
  per axis is 1 when the extent is within target = t * delta (or f = 0),
  else the smallest n >= 2 whose surface cell is within the target, capped
  at max_per_axis (solve.rs:384-403); the slab of currents.rs:87-92 has
  delta = t / 4 at its frequency.
"""
import math

import numpy as np
import pytest

from fasterhenry_b200 import fixtures as F

COPPER = 5.8e7
MU0 = 4.0e-7 * math.pi
TOL = 1e-12

START, END, WDIR, HDIR, WIDTH, HEIGHT = slice(0, 3), slice(3, 6), slice(10, 13), slice(13, 16), 16, 17


def weights(n, ratio):
    return [ratio ** min(i, n - 1 - i) for i in range(n)]


def surface_extent(total, n, ratio):
    return total / sum(weights(n, ratio))


def one_segment(fh, a, b, w, h, disc, sigma=COPPER):
    g = fh.Geometry.from_parts([a, b], [fh.SegmentDef(0, 1, w, h, sigma)])
    return fh.discretize(g, disc)


def test_hand_computed_graded_grid(fh):
    """4 cells at 3:1 over a 0.8-wide segment: weights 1, 3, 3, 1 (sum 8),
    extents 0.1, 0.3, 0.3, 0.1 centred at -0.35, -0.15, 0.15, 0.35."""
    fil, per = one_segment(fh, (0, 0, 0), (1, 0, 0), 0.8, 0.2, fh.Discretization.graded(4, 1, 3.0))
    assert list(per) == [4]
    for f, (y, w) in zip(fil, [(-0.35, 0.1), (-0.15, 0.3), (0.15, 0.3), (0.35, 0.1)]):
        assert np.max(np.abs(f[START] - [0.0, y, 0.0])) < TOL
        assert np.max(np.abs(f[END] - [1.0, y, 0.0])) < TOL
        assert abs(f[WIDTH] - w) < TOL and abs(f[HEIGHT] - 0.2) < TOL


def skew():
    # a segment along no axis, with its own default frame
    return (0.1, -0.2, 0.3), (1.3, 0.9, -0.4), 0.7, 0.3


@pytest.mark.parametrize("nw,nh,ratio", [(4, 4, 10.0), (3, 5, 2.0), (1, 8, 1.5), (7, 1, 3.0), (6, 5, 2.5)])
def test_graded_extents_follow_the_progression(fh, nw, nh, ratio):
    a, b, w, h = skew()
    fil, _ = one_segment(fh, a, b, w, h, fh.Discretization.graded(nw, nh, ratio))
    assert len(fil) == nw * nh
    assert abs(np.sum(fil[:, WIDTH] * fil[:, HEIGHT]) - w * h) < TOL * w * h
    widths = fil[:nw, WIDTH]
    heights = fil[::nw, HEIGHT]
    assert np.allclose(widths, [w * x / sum(weights(nw, ratio)) for x in weights(nw, ratio)], rtol=TOL, atol=0)
    assert np.allclose(heights, [h * x / sum(weights(nh, ratio)) for x in weights(nh, ratio)], rtol=TOL, atol=0)
    for k, f in enumerate(fil):  # widths repeat every row, heights every column
        assert abs(f[WIDTH] - fil[k % nw, WIDTH]) < TOL and abs(f[HEIGHT] - fil[(k // nw) * nw, HEIGHT]) < TOL
    assert abs(widths[0] - surface_extent(w, nw, ratio)) < TOL * widths[0]
    assert abs(heights[-1] - surface_extent(h, nh, ratio)) < TOL * heights[-1]


@pytest.mark.parametrize("nw,nh,ratio", [(4, 4, 10.0), (5, 3, 2.0), (2, 6, 1.25)])
def test_graded_bundle_is_centred_and_fills_the_surfaces(fh, nw, nh, ratio):
    fil, _ = one_segment(fh, (0, 0, 0), (2, 0, 0), 0.6, 0.4, fh.Discretization.graded(nw, nh, ratio))
    centres = 0.5 * (fil[:, START] + fil[:, END])
    assert np.max(np.abs(centres.mean(axis=0) - [1.0, 0.0, 0.0])) < TOL
    y, z = centres[:, 1], centres[:, 2]
    assert abs(np.min(y - 0.5 * fil[:, WIDTH]) + 0.3) < TOL and abs(np.max(y + 0.5 * fil[:, WIDTH]) - 0.3) < TOL
    assert abs(np.min(z - 0.5 * fil[:, HEIGHT]) + 0.2) < TOL and abs(np.max(z + 0.5 * fil[:, HEIGHT]) - 0.2) < TOL


def test_graded_surface_extent_figures():
    """16 uniform cells of 1 mm are 62.5 um; 6 cells at 4:1 put 1 mm / 42 on
    each surface (weights 1 4 16 16 4 1), under 0.4 of the uniform cell."""
    assert abs(surface_extent(1e-3, 16, 1.0) - 62.5e-6) < 1e-18
    assert abs(surface_extent(1e-3, 6, 4.0) - 1e-3 / 42.0) < 1e-18
    assert surface_extent(1e-3, 6, 4.0) < 0.4 * 62.5e-6
    assert surface_extent(8.0, 4, 3.0) == 1.0 and abs(surface_extent(8.0, 6, 3.0) - 8.0 / 26.0) < 1e-15


def test_graded_grid_commutes_with_rigid_motion(fh):
    a, b, w, h = skew()
    c, s = math.cos(1.234), math.sin(1.234)
    axis = np.array([0.4, -1.0, 0.7]) / np.linalg.norm([0.4, -1.0, 0.7])
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    rot = np.eye(3) + s * K + (1 - c) * K @ K
    shift = np.array([-2.0, 0.5, 3.0])
    base, _ = one_segment(fh, a, b, w, h, fh.Discretization.graded(4, 3, 2.0))
    # the moved segment keeps its cross-section frame rotated with it
    wdir = tuple(rot @ base[0, WDIR])
    g = fh.Geometry.from_parts([tuple(rot @ np.array(a) + shift), tuple(rot @ np.array(b) + shift)],
                               [fh.SegmentDef(0, 1, w, h, COPPER, wdir)])
    moved, _ = fh.discretize(g, fh.Discretization.graded(4, 3, 2.0))
    assert len(moved) == 12
    for f, m in zip(base, moved):
        assert np.linalg.norm(rot @ f[START] + shift - m[START]) < 1e-12
        assert np.linalg.norm(rot @ f[END] + shift - m[END]) < 1e-12
        assert abs(f[WIDTH] - m[WIDTH]) < TOL and abs(f[HEIGHT] - m[HEIGHT]) < TOL


def count_for(extent, f, sigma, target_depths, ratio, cap=32):
    delta = math.inf if f == 0 else 1.0 / math.sqrt(math.pi * f * MU0 * sigma)
    target = target_depths * delta
    if math.isinf(target) or extent <= target:
        return 1
    for n in range(2, cap + 1):
        if surface_extent(extent, n, ratio) <= target:
            return n
    return cap


def test_skin_depth_formula(fh):
    """The slab of the reference's currents test: t = 200 um, delta = t / 4 at
    f = 1 / (pi mu0 sigma delta^2)."""
    t = 200e-6
    delta = t / 4.0
    f = 1.0 / (math.pi * MU0 * COPPER * delta * delta)
    assert abs(fh.skin_depth(f, COPPER) - delta) < 1e-12


@pytest.mark.parametrize("f,w,h,target,ratio", [
    (1e9, 20e-6, 5e-6, 0.5, 2.0),     # copper at 1 GHz: delta = 2.09 um -> 7 x 4
    (1e8, 1e-3, 35e-6, 0.5, 4.0),     # a PCB trace at 100 MHz: 9 x 5
    (1e6, 1e-3, 35e-6, 0.5, 2.0),     # delta = 66 um: 9 x 2
    (0.0, 1e-3, 35e-6, 0.5, 2.0),     # DC: one filament
    (1e11, 50e-6, 50e-6, 0.25, 1.5),  # 27 x 27
    (1e11, 50e-6, 50e-6, 0.25, 1.0),  # uniform cells: the 32 cap on both axes
])
def test_skin_depth_counts_follow_the_rule(fh, f, w, h, target, ratio):
    fil, per = one_segment(fh, (0, 0, 0), (1e-3, 0, 0), w, h, fh.Discretization.skin_depth(f, target, ratio))
    nw, nh = count_for(w, f, COPPER, target, ratio), count_for(h, f, COPPER, target, ratio)
    assert list(per) == [nw * nh], (nw, nh)
    assert np.allclose(fil[:nw, WIDTH], [w * x / sum(weights(nw, ratio)) for x in weights(nw, ratio)], rtol=TOL, atol=0)
    assert np.allclose(fil[::nw, HEIGHT], [h * x / sum(weights(nh, ratio)) for x in weights(nh, ratio)], rtol=TOL,
                       atol=0)
    if f > 0:
        tgt = target * fh.skin_depth(f, COPPER)
        for extent, n in ((w, nw), (h, nh)):
            if 1 < n < 32:
                # the count is the smallest that resolves the target
                assert surface_extent(extent, n, ratio) <= tgt < surface_extent(extent, n - 1, ratio)


def test_skin_depth_counts_per_segment_material(fh):
    """Each segment takes its own count, from its own extents and sigma: a
    copper trace and a ten-times-less-conductive one side by side."""
    g = fh.Geometry.from_parts([(0, 0, 0), (1e-3, 0, 0), (0, 1e-4, 0), (1e-3, 1e-4, 0)],
                               [fh.SegmentDef(0, 1, 20e-6, 5e-6, COPPER), fh.SegmentDef(2, 3, 20e-6, 5e-6, COPPER / 10)])
    fil, per = fh.discretize(g, fh.Discretization.skin_depth(1e9, 0.5, 2.0))
    want = [count_for(20e-6, 1e9, s, 0.5, 2.0) * count_for(5e-6, 1e9, s, 0.5, 2.0) for s in (COPPER, COPPER / 10)]
    assert list(per) == want and want[0] > want[1]
    assert np.all(fil[:want[0], 18] == COPPER) and np.all(fil[want[0]:, 18] == COPPER / 10)
