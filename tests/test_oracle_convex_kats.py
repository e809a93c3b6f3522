"""Pins the CPU oracle's convex narrow phase against more of the reference's own tests.

Each test restates the assertions of one test of crates/bullet-collision/src/narrowphase
(file and lines cited): the GJK/EPA contact's witness geometry, the band-to-EPA transition,
touching and near-touching spheres, separated pairs and the plane and capsule routes of the
dispatcher, in both precisions. Shapes the step does not have (cylinders, cones) are left out
of the restated inputs.
"""
import math

import numpy as np
import pytest

from oracle_api import OracleWorld, pose

PRECISIONS = ["f32", "f64"]
OCTAHEDRON = [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]]


def rot(axis, angle):
    s = math.sin(angle / 2)
    return tuple([s if k == axis else 0.0 for k in range(3)] + [math.cos(angle / 2)])


def rotate(q, v):
    x, y, z, w = q
    b = np.array([x, y, z])
    v = np.asarray(v, dtype=np.float64)
    return v * (w * w - b @ b) + 2 * b * (b @ v) + 2 * w * np.cross(b, v)


def box_support(half, p, q, d):
    # shapes/box_shape.rs:30-37 and shapes/mod.rs:323-332 (world support of the full box)
    qi = (-q[0], -q[1], -q[2], q[3])
    ld = rotate(qi, d)
    local = np.where(ld >= 0.0, half, -np.asarray(half, dtype=np.float64))
    return rotate(q, local) + np.asarray(p, dtype=np.float64)


def sphere_support(r, p, d):
    d = np.asarray(d, dtype=np.float64)
    return np.asarray(p, dtype=np.float64) + r * d / np.linalg.norm(d)


def assert_clean(m, separation):
    # narrowphase/convex_convex.rs:385-391
    n, pos, pen = m[3:6], m[0:3], m[6]
    assert np.all(np.isfinite(n)) and np.isfinite(pen) and np.all(np.isfinite(pos))
    s = np.asarray(separation, dtype=np.float64)
    assert n @ (s / np.linalg.norm(s)) > 0.0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_separated_capsules_do_not_touch(prec):
    # narrowphase/convex_convex.rs:226-230
    w = OracleWorld(prec)
    c = w.capsule(0.5, 1.0)
    assert w.convex_convex(c, pose(), c, pose((2, 0, 0))) is None


@pytest.mark.parametrize("prec", PRECISIONS)
def test_witness_asymmetric_hull_vs_sphere_on_support_plane(prec):
    # narrowphase/convex_convex.rs:455-486: the contact point lies on B's support plane.
    w = OracleWorld(prec)
    h, s = w.hull(OCTAHEDRON), w.sphere(0.5)
    pb = (1.25, 0.3, 0.0)
    m = w.convex_convex(h, pose(), s, pose(pb))
    assert m is not None
    assert_clean(m, pb)
    assert m[6] > 0.0
    n = m[3:6]
    assert n @ m[0:3] == pytest.approx(n @ sphere_support(0.5, pb, -n), abs=2e-2)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_witness_rotated_box_vs_box_on_support_plane(prec):
    # narrowphase/convex_convex.rs:491-503
    w = OracleWorld(prec)
    a, b = w.box([1.0, 0.4, 0.6]), w.box([0.5, 0.5, 0.5])
    qa, qb, pb = rot(2, 0.6), rot(2, -0.35), (1.3, 0.25, 0.1)
    m = w.convex_convex(a, pose((0, 0, 0), qa), b, pose(pb, qb))
    assert m is not None
    assert_clean(m, pb)
    assert m[6] > 0.0
    n = m[3:6]
    assert n @ m[0:3] == pytest.approx(n @ box_support([0.5, 0.5, 0.5], pb, qb, -n), abs=2e-2)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_witness_elongated_hull_vs_hull_stays_clean(prec):
    # narrowphase/convex_convex.rs:509-520
    w = OracleWorld(prec)
    a, b = w.box([1.5, 0.05, 0.05]), w.box([0.3, 0.3, 0.3])
    qa, pb = rot(2, 0.25), (1.7, 0.2, 0.0)
    m = w.convex_convex(a, pose((0, 0, 0), qa), b, pose(pb))
    assert m is not None
    assert_clean(m, pb)
    assert m[6] > 0.0
    n = m[3:6]
    assert n @ m[0:3] == pytest.approx(n @ box_support([0.3, 0.3, 0.3], pb, (0, 0, 0, 1), -n), abs=2e-2)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_witness_unequal_margins_deep_overlap(prec):
    # narrowphase/convex_convex.rs:525-543: the deep-overlap depth is the full-shape overlap.
    w = OracleWorld(prec)
    a, b = w.box([1, 1, 1]), w.sphere(0.25)
    m = w.convex_convex(a, pose(), b, pose((0, 0.9, 0)))
    assert m is not None
    assert_clean(m, (0, 0.9, 0))
    assert m[6] == pytest.approx(0.35, abs=2e-3)
    assert m[1] == pytest.approx(0.65, abs=2e-3)
    assert m[4] == pytest.approx(1.0, abs=1e-3)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_band_to_epa_transition_stays_continuous(prec):
    # narrowphase/convex_convex.rs:550-596: a sphere lowered into a box in 0.01 steps, from the
    # margin band into deep overlap: no normal flip and no jump above 2.5 steps + 2e-3.
    w = OracleWorld(prec)
    a, b = w.box([1, 1, 1]), w.sphere(0.5)
    step, prev = 0.01, None
    for i in range(78):
        py = 1.32 - step * i
        m = w.convex_convex(a, pose(), b, pose((0, py, 0)))
        if m is None:
            prev = None
            continue
        assert abs(m[4] - 1.0) <= 5e-2, py
        assert np.isfinite(m[6]) and np.isfinite(m[1])
        if prev is not None:
            jump = 2.5 * step + 2e-3
            assert abs(m[6] - prev[1]) <= jump, py
            assert abs(m[1] - prev[2]) <= jump, py
            assert m[4] * prev[0] > 0.5, py
        prev = (m[4], m[6], m[1])


@pytest.mark.parametrize("prec", PRECISIONS)
def test_exact_touching_is_clean(prec):
    # narrowphase/convex_convex.rs:601-617
    w = OracleWorld(prec)
    s = w.sphere(0.5)
    m = w.convex_convex(s, pose(), s, pose((1, 0, 0)))
    if m is not None:
        assert np.isfinite(m[6]) and abs(m[6]) <= 1e-3
        assert m[3] == pytest.approx(1.0, abs=1e-2)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_tiny_overlap_and_separation_stay_proportional(prec):
    # narrowphase/convex_convex.rs:622-651
    w = OracleWorld(prec)
    s = w.sphere(0.5)
    m = w.convex_convex(s, pose(), s, pose((1 - 1e-4, 0, 0)))
    if m is not None:
        assert np.isfinite(m[6]) and abs(m[6]) <= 0.1 and np.isfinite(m[3])
    m = w.convex_convex(s, pose(), s, pose((1 + 1e-4, 0, 0)))
    if m is not None:
        assert np.isfinite(m[6]) and abs(m[6]) <= 0.1
        assert m[6] <= 0.0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_separated_boxes(prec):
    # narrowphase/box_box.rs:549-554
    w = OracleWorld(prec)
    b = w.box([1, 1, 1])
    assert len(w.collide(b, pose(), b, pose((3, 0, 0)))) == 0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_plane_vs_box_through_collide(prec):
    # narrowphase/mod.rs:372-381
    w = OracleWorld(prec)
    p, b = w.plane([0, 1, 0], 0.0), w.box([1, 1, 1])
    m = w.collide(p, pose(), b, pose((0, 0.5, 0)))
    assert len(m) >= 1
    assert m[0, 4] == pytest.approx(1.0)
    assert m[0, 6] == pytest.approx(0.5, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_rotated_capsule_on_plane(prec):
    # narrowphase/mod.rs:384-401: a capsule lying along x, its axis 0.4 above the plane.
    w = OracleWorld(prec)
    p, c = w.plane([0, 1, 0], 0.0), w.capsule(0.5, 1.0)
    m = w.collide(p, pose(), c, pose((0, 0.4, 0), rot(2, math.pi / 2)))
    assert len(m) >= 1
    assert m[0, 4] == pytest.approx(1.0)
    assert m[0, 6] == pytest.approx(0.1, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_seeded_collide_matches_unseeded(prec):
    # narrowphase/mod.rs:516-564 (its capsule pair): seeding the search with the found normal,
    # its opposite or an arbitrary direction gives the same contacts to the EPA floor.
    w = OracleWorld(prec)
    c = w.capsule(0.5, 1.0)
    pa, pb = pose((0, 0, 0), rot(1, 0.6)), pose((0.7, 0.2, 0.1))
    u = w.collide(c, pa, c, pb)
    assert len(u) >= 1
    d = np.array([0.3, -0.5, 0.8])
    for seed in (u[0, 3:6], -u[0, 3:6], d / np.linalg.norm(d)):
        s = w.collide(c, pa, c, pb, seed=seed)
        assert len(s) == len(u)
        for a, b in zip(s, u):
            assert a[6] == pytest.approx(b[6], abs=2e-4)
            assert np.linalg.norm(a[3:6] - b[3:6]) < 1e-4 or a[3:6] @ b[3:6] > 0.9999
