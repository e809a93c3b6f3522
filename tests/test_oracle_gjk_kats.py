"""Pins the CPU oracle's GJK distance walk (the core walk that classifies a convex pair as
separated, in the contact band, or overlapping past the margins) against the reference's own
tests in crates/bullet-collision/src/narrowphase/gjk.rs (each test's lines cited), in both
precisions. Shapes the step does not have are left out of the restated inputs.
"""
import numpy as np
import pytest

from oracle_api import OracleWorld, pose

PRECISIONS = ["f32", "f64"]
SEPARATED, BAND, OVERLAP = 0, 1, 2


def contact(w, a, pa, b, pb, thr, seed=None):
    return w.gjk_contact(a, pose(pa), b, pose(pb), thr, seed)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_contact_walk_reports_band_separation(prec):
    # gjk.rs:1106-1124
    w = OracleWorld(prec)
    s = w.sphere(0.5)
    k, d, n, pob, _ = contact(w, s, (0, 0, 0), s, (1.01, 0, 0), 0.0173)
    assert k == BAND
    assert abs(d - 0.01) < 1e-4
    assert np.linalg.norm(n - [1, 0, 0]) < 1e-4
    assert np.linalg.norm(pob - [0.51, 0, 0]) < 1e-4
    assert contact(w, s, (0, 0, 0), s, (1.5, 0, 0), 0.0173)[0] == SEPARATED


@pytest.mark.parametrize("prec", PRECISIONS)
def test_contact_walk_routes_overlap_and_rotated_band(prec):
    # gjk.rs:1131-1191: an overlap inside the margin shell is a band with negative distance; a
    # rotated capsule pair gives the same band distance from any seed.
    w = OracleWorld(prec)
    s, c = w.sphere(0.5), w.capsule(0.5, 1.0)
    k, d, *_ = contact(w, s, (0, 0, 0), s, (0.7, 0, 0), 0.0173)
    assert k == BAND and abs(d + 0.3) < 1e-4
    k, d, *_ = contact(w, c, (0, 0, 0), c, (1.01, 0, 0), 0.5)
    assert k == BAND and abs(d - 0.01) < 1e-4
    qa = (0.0, 0.0, np.sin(0.25), np.cos(0.25))
    pa, pb = pose((0, 0, 0), qa), pose((1.6, 0.2, 0.1))
    k, ref, *_ = w.gjk_contact(c, pa, c, pb, 0.5)
    assert k == BAND
    for seed in ([1, 0, 0], [0, 1, 0], np.array([0.3, -0.5, 0.8]) / np.linalg.norm([0.3, -0.5, 0.8])):
        k, d, *_ = w.gjk_contact(c, pa, c, pb, 0.5, seed)
        assert k == BAND and abs(d - ref) < 2e-3


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_contact_coincident_point_cores_terminate_finitely(prec):
    # gjk.rs:1514-1532: coincident spheres and capsules end with finite output.
    w = OracleWorld(prec)
    for s in (w.sphere(0.5), w.capsule(0.5, 0.5)):
        k, d, n, *_ = contact(w, s, (0, 0, 0), s, (0, 0, 0), 0.0173)
        if k == BAND:
            assert np.isfinite(d) and np.all(np.isfinite(n))


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_contact_touch_gap_overlap_boundary(prec):
    # gjk.rs:1538-1571
    w = OracleWorld(prec)
    s = w.sphere(0.5)
    k, d, n, pob, _ = contact(w, s, (0, 0, 0), s, (1.0, 0, 0), 0.0173)
    assert k == BAND and abs(d) < 1e-6
    assert np.linalg.norm(n - [1, 0, 0]) < 1e-6
    assert np.linalg.norm(pob - [0.5, 0, 0]) < 1e-5
    k, d, *_ = contact(w, s, (0, 0, 0), s, (1.0 + 1e-5, 0, 0), 0.0173)
    assert k == BAND and abs(d - 1e-5) < 1e-6
    k, d, *_ = contact(w, s, (0, 0, 0), s, (1.0 - 1e-5, 0, 0), 0.0173)
    assert k == BAND and abs(d + 1e-5) < 1e-6
    assert contact(w, s, (0, 0, 0), s, (1.05, 0, 0), 0.0173)[0] == SEPARATED


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_contact_band_threshold_routing(prec):
    # gjk.rs:1576-1591
    w = OracleWorld(prec)
    s = w.sphere(0.5)
    k, d, *_ = contact(w, s, (0, 0, 0), s, (1.0199, 0, 0), 0.02)
    assert k == BAND and abs(d - 0.0199) < 1e-5
    assert contact(w, s, (0, 0, 0), s, (1.0201, 0, 0), 0.02)[0] == SEPARATED


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_scale_sweep_sphere_pairs(prec):
    # gjk.rs:1597-1633: the classification and the scaled distance track the unit scale from
    # 1e-3 to 1e3; sphere overlaps stay inside the margin shell (never Overlap).
    for scale in (1e-3, 1e-2, 1.0, 1e2, 1e3):
        w = OracleWorld(prec)
        s = w.sphere(0.5 * scale)
        for centers, band, dist in ((3.0, False, 2.0), (1.0, True, 0.0), (0.9, True, -0.1), (0.5, True, -0.5)):
            k, d, n, *_ = contact(w, s, (0, 0, 0), s, (centers * scale, 0, 0), 0.02 * scale)
            assert k != OVERLAP
            assert (k == BAND) == band, (scale, centers)
            if k == BAND:
                assert np.isfinite(d) and abs(d / scale - dist) < 1e-4, (scale, centers, d)
                assert abs(np.linalg.norm(n) - 1.0) < 1e-5 and abs(n[0]) > 0.999


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_scale_sweep_box_pairs(prec):
    # gjk.rs:1642-1696: face-to-face box pairs at every scale: the walk's distance against the
    # margin model decides band or separated; a deep overlap reaches EPA with a full simplex
    # once the cores exist (scale >= 0.16), else stays in the band.
    margin = 0.04
    for scale in (1e-3, 1e-2, 1.0, 1e2, 1e3):
        w = OracleWorld(prec)
        b = w.box([0.5 * scale] * 3)
        core = max(0.5 * scale - margin, 0.0)
        thr = 0.02 * scale
        for centers in (3.0 * scale, 1.0 * scale):
            expected = centers - 2.0 * core - 2.0 * margin
            k, d, n, *_ = contact(w, b, (0, 0, 0), b, (centers, 0, 0), thr)
            assert k != OVERLAP
            assert (k == BAND) == (expected < thr), (scale, centers)
            if k == BAND:
                assert abs(d - expected) < max(1e-4 * scale, 1e-6), (scale, d, expected)
                assert np.all(np.isfinite(n))
        k, _, _, _, ns = contact(w, b, (0, 0, 0), b, (0.3 * scale, 0, 0), thr)
        if core > 0.0:
            assert k == OVERLAP and ns == 4, scale
        else:
            assert k == BAND, scale


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_seeded_vs_unseeded_stability(prec):
    # gjk.rs:1741-1807: seeds change nothing: the sphere band distance exactly, the box band to
    # 1e-5, the box overlap and separation classes.
    w = OracleWorld(prec)
    s, b = w.sphere(0.5), w.box([0.5, 0.5, 0.5])
    v = np.array([1.0, 7.0, 3.0])
    seeds = (None, [1, 0, 0], [-1, 0, 0], [0, 1, 0], v / np.linalg.norm(v))
    ref = None
    for seed in seeds:
        k, d, n, *_ = contact(w, s, (0, 0, 0), s, (1.01, 0, 0), 0.0173, seed)
        assert k == BAND and abs(n[0] - 1.0) < 1e-6
        ref = d if ref is None else ref
        assert abs(d - ref) < 1e-9
    ref = None
    for seed in seeds:
        k, d, n, *_ = contact(w, b, (0, 0, 0), b, (1.02, 0, 0), 0.05, seed)
        assert k == BAND and abs(n[0]) > 0.999
        ref = d if ref is None else ref
        assert abs(d - ref) < 1e-5
    for seed in seeds:
        k, _, _, _, ns = contact(w, b, (0, 0, 0), b, (0.6, 0, 0), 0.02, seed)
        assert k == OVERLAP and ns == 4
        assert contact(w, b, (0, 0, 0), b, (3.0, 0, 0), 0.02, seed)[0] == SEPARATED


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_elongated_rod_vs_box_stays_finite(prec):
    # gjk.rs:1881-1932: a 2 m rod (hull, no margin) against a box above its tip.
    w = OracleWorld(prec)
    e = 1e-3
    rod = w.hull([[x, y, z] for z in (-e, e) for y in (-1.0, 1.0) for x in (-e, e)])
    b = w.box([0.5, 0.5, 0.5])
    k, d, n, *_ = contact(w, rod, (0, 0, 0), b, (0, 1.51, 0), 0.0173)
    assert k == BAND and abs(d - 0.01) < 1e-4
    assert np.all(np.isfinite(n)) and abs(n[1]) > 0.999
    k, d, *_ = contact(w, rod, (0, 0, 0), b, (0, 1.50, 0), 0.0173)
    assert k == BAND and abs(d) < 1e-5
    k, _, _, _, ns = contact(w, rod, (0, 0, 0), b, (0, 1.45, 0), 0.0173)
    assert k == OVERLAP and ns == 4
    assert contact(w, rod, (0, 0, 0), b, (0, 2.5, 0), 0.0173)[0] == SEPARATED


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_duplicate_support_gate_across_scales(prec):
    # gjk.rs:1703-1734: a cube hull (corner supports repeat) against a sphere with a face gap of
    # 0.01 x scale: a band at that distance from 1e-3 to 1e2.
    for scale in (1e-3, 1e-2, 1.0, 1e2):
        w = OracleWorld(prec)
        e = 0.5 * scale
        hull = w.hull([[x, y, z] for z in (-e, e) for y in (-e, e) for x in (-e, e)])
        s = w.sphere(0.5 * scale)
        k, d, n, *_ = contact(w, hull, (0, 0, 0), s, (1.01 * scale, 0, 0), 0.02 * scale)
        assert k == BAND, scale
        assert abs(d - 0.01 * scale) < max(1e-4 * scale, 1e-9), (scale, d)
        assert np.all(np.isfinite(n)) and abs(n[0]) > 0.999


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gjk_degenerate_segment_hulls_terminate_finitely(prec):
    # gjk.rs:1816-1875 (its contact-walk assertions): crossing segments overlap (a full finite
    # simplex) or touch in the band; parallel segments 2 apart are separated; collinear
    # overlapping segments end with finite output.
    w = OracleWorld(prec)
    sx = w.hull([[-1, 0, 0], [1, 0, 0]])
    sy = w.hull([[0, -1, 0], [0, 1, 0]])
    k, d, n, _, ns = contact(w, sx, (0, 0, 0), sy, (0, 0, 0), 0.0173)
    assert k != SEPARATED
    if k == OVERLAP:
        assert ns == 4
    else:
        assert abs(d) < 1e-3 and np.all(np.isfinite(n))
    assert contact(w, sx, (0, 0, 0), sx, (0, 2, 0), 0.0173)[0] == SEPARATED
    k, d, n, *_ = contact(w, sx, (0, 0, 0), sx, (0.5, 0, 0), 0.0173)
    if k == BAND:
        assert np.isfinite(d) and np.all(np.isfinite(n))
