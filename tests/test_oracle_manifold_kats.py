"""Pins the CPU oracle's persistent manifold against more of the reference's manifold tests.

Each test restates the assertions that crates/bullet-collision/src/manifold.rs's tests (module
from line 389; each test's lines cited) make about the crate's own manifold: overflow handling,
cache matching, the redetect gate and ContactManifold::reduce. Where a reference test also runs
a model of upstream Bullet's policy to show that the two differ, only the assertions about the
crate's behaviour are restated. Both precisions are checked.
"""
import math

import numpy as np
import pytest

from oracle_api import OracleManifold, manifold_reduce, pose

PRECISIONS = ["f32", "f64"]
THR = 0.02  # manifold.rs:8 CONTACT_BREAKING_THRESHOLD


def pt(x, y, z, pen, n=(0.0, 1.0, 0.0)):
    return [x, y, z, n[0], n[1], n[2], pen]


def spread(a):
    a = np.asarray(a)
    return max((np.linalg.norm(a[i] - a[j]) for i in range(len(a)) for j in range(i + 1, len(a))), default=0.0)


def rot_z(angle):
    return (0.0, 0.0, math.sin(angle / 2), math.cos(angle / 2))


def resting(pen):
    # manifold.rs:399-409: box (A) above a plane (B), one contact at the origin.
    return [pt(0, 0, 0, pen)], pose((0, 0.5 - pen, 0)), pose()


def capture_each(c, points, thr=THR):
    for p in points:
        c.capture([p], pose(), pose(), thr)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capture_overflow_keeps_deepest_four_even_when_clustered(prec):
    # manifold.rs:784-836: overflow keeps the deepest point and then the first shallow points in
    # input order (a clustered patch), not the two far points.
    c = OracleManifold(prec)
    batch = [pt(0, 0, 0, 0.5), pt(0.03, 0, 0, 0.1), pt(0, 0, 0.03, 0.1), pt(0, 0.03, 0, 0.1), pt(1, 0, 0, 0.1),
             pt(0, 1, 0, 0.1)]
    c.capture(batch, pose(), pose(), THR)
    p = c.points()
    assert len(p) == 4
    anchors = p[:, 0:3]
    assert anchors[0, 1] == pytest.approx(0.5, abs=1e-6)
    assert spread(anchors[1:4]) < 0.1
    assert np.all(anchors.max(axis=1) < 0.6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capture_overflow_differs_even_on_spread_inputs(prec):
    # manifold.rs:844-899: a full, spread cache drops a shallow near-duplicate of its deep corner
    # that arrives outside the matching radius.
    c = OracleManifold(prec)
    capture_each(c, [pt(0, 0, 0, 0.4), pt(1, 0, 0, 0.3), pt(0, 0, 1, 0.2), pt(1, 0, 1, 0.1)])
    c.capture([pt(0.015, 0, 0.015, 0.05)], pose(), pose(), THR)
    a = c.points()[:, 0:3]
    assert len(a) == 4
    assert np.any(a[:, 1] > 0.3)
    assert not np.any((np.abs(a[:, 0] - 0.015) < 1e-6) & (np.abs(a[:, 2] - 0.015) < 1e-6))


@pytest.mark.parametrize("prec", PRECISIONS)
def test_overflow_evolution_on_a_planar_patch(prec):
    # manifold.rs:907-959: a deep seed then patch points on a 0.05 grid, one per capture: the
    # cache never exceeds four, the deep anchor is bit-stable, the kept set stays spread and the
    # late patch points never enter.
    c = OracleManifold(prec)
    frames = [pt(0, 0, 0, 0.5)]
    for x in (0.0, 0.05, 0.1):
        for z in (0.0, 0.05, 0.1):
            if x == 0.0 and z == 0.0:
                continue
            frames.append(pt(x, 0, z, 0.1))
    deep = None
    for f in frames:
        c.capture([f], pose(), pose(), THR)
        p = c.points()
        assert len(p) <= 4
        if deep is None:
            deep = p[0, 0:3].copy()
        else:
            np.testing.assert_array_equal(p[0, 0:3], deep)
    a = c.points()[:, 0:3]
    assert len(a) == 4
    assert spread(a) > 0.05
    kept = {(float(np.float32(x)), float(np.float32(z))) for x, z in a[:, [0, 2]]}
    for f in frames[4:]:
        assert (float(np.float32(f[0])), float(np.float32(f[2]))) not in kept


@pytest.mark.parametrize("prec", PRECISIONS)
def test_overflow_evolution_on_a_triangular_patch(prec):
    # manifold.rs:965-1000: after the first four captures the kept anchors never change again,
    # the deep seed survives and the triangle stays spread.
    c = OracleManifold(prec)
    verts = [(0, 0, 0), (0.08, 0, 0), (0, 0, 0.08), (0.06, 0, 0.07), (0.04, 0, 0), (0, 0, 0.04), (0.03, 0, 0.035)]
    seen = []
    for n, v in enumerate(verts):
        c.capture([pt(*v, 0.5 if n == 0 else 0.1)], pose(), pose(), THR)
        p = c.points()
        assert len(p) <= 4
        seen.append(p[:, 0:3].copy())
    for a in seen[4:]:
        np.testing.assert_array_equal(a, seen[3])
    assert c.points()[0, 1] == pytest.approx(0.5, abs=1e-6)
    assert spread(seen[3]) > 0.08


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capture_matches_the_first_cached_point_not_the_nearest(prec):
    # manifold.rs:1007-1053: with two cached points inside the matching radius, the incoming
    # point replaces (and inherits the impulse of) the first one, not the nearest.
    c = OracleManifold(prec)
    capture_each(c, [pt(0, 0, 0, 0.01), pt(0.06, 0, 0, 0.01)])
    c.set_impulse(0, 5.0)
    c.set_impulse(1, 7.0)
    c.capture([pt(0.045, 0, 0, 0.01)], pose(), pose(), 0.1)
    p = c.points()
    assert len(p) == 2
    assert p[0, 0] == pytest.approx(0.045, abs=1e-6)
    assert p[0, 10] == pytest.approx(5.0)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capture_matching_follows_cache_order_deterministically(prec):
    # manifold.rs:1059-1098: the same two seeds in the other order: the first (now near) entry
    # is matched; the other keeps its own impulse.
    c = OracleManifold(prec)
    capture_each(c, [pt(0.06, 0, 0, 0.01), pt(0, 0, 0, 0.01)])
    c.set_impulse(0, 7.0)
    c.set_impulse(1, 5.0)
    c.capture([pt(0.045, 0, 0, 0.01)], pose(), pose(), 0.1)
    p = c.points()
    assert p[0, 10] == pytest.approx(7.0)
    assert p[1, 10] == pytest.approx(5.0)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capture_requires_normal_agreement_to_match(prec):
    # manifold.rs:1103-1166: a point at the cached anchor matches when its normal is 25 degrees
    # off (dot 0.906 >= 0.9) and inherits; at 30 degrees (dot 0.866) it is appended fresh.
    c = OracleManifold(prec)
    c.capture([pt(0, 0, 0, 0.01)], pose(), pose(), THR)
    c.set_impulse(0, 3.0)
    a = 0.4363323
    c.capture([pt(0, 0, 0, 0.01, n=(math.sin(a), math.cos(a), 0.0))], pose(), pose(), THR)
    p = c.points()
    assert len(p) == 1 and p[0, 10] == pytest.approx(3.0)
    c = OracleManifold(prec)
    c.capture([pt(0, 0, 0, 0.01)], pose(), pose(), THR)
    a = math.pi / 6.0
    c.capture([pt(0, 0, 0, 0.01, n=(math.sin(a), math.cos(a), 0.0))], pose(), pose(), THR)
    p = c.points()
    assert len(p) == 2 and p[1, 10] == 0.0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_rotation_gate_boundaries_and_body_sides(prec):
    # manifold.rs:1172-1195: the summed rotation of both bodies against 0.01 rad, strict.
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    c.capture(m, pa, pb, THR)

    def gate(qa, qb):
        a, b = pa.copy(), pb.copy()
        a[3:7], b[3:7] = qa, qb
        return c.needs_redetect(a, b)

    ident = (0.0, 0.0, 0.0, 1.0)
    assert not gate(rot_z(0.008), ident)
    assert not gate(ident, rot_z(0.008))
    assert gate(rot_z(0.012), ident)
    assert gate(ident, rot_z(0.012))
    assert gate(rot_z(0.008), rot_z(-0.008))
    assert not gate(rot_z(0.003), rot_z(-0.003))


@pytest.mark.parametrize("prec", PRECISIONS)
def test_negated_quaternion_only_forces_a_redetect_not_new_geometry(prec):
    # manifold.rs:1228-1255: -q triggers the gate where q does not, but refreshing under either
    # gives the same contact.
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    c.capture(m, pa, pb, THR)
    q = np.array(rot_z(0.008))
    a1, a2 = pa.copy(), pa.copy()
    a1[3:7], a2[3:7] = q, -q
    assert not c.needs_redetect(a1, pb)
    assert c.needs_redetect(a2, pb)
    r1 = c.refresh(a1, pb)
    r2 = c.refresh(a2, pb)
    assert len(r1) == 1 and len(r2) == 1
    np.testing.assert_allclose(r1[0, 0:3], r2[0, 0:3], atol=1e-6)
    assert r1[0, 6] == pytest.approx(r2[0, 6], abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_resting_contact_survives_sub_threshold_perturbations_without_churn(prec):
    # manifold.rs:1264-1312: 20 frames of +-0.002 nudges keep the anchors, the normal and the
    # impulse bit-stable; a 0.006 drift asks for re-detection but the point survives with its
    # penetration; a 0.035 separation kills it.
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    c.capture(m, pa, pb, THR)
    c.set_impulse(0, 3.0)
    p0 = c.points()[0].copy()
    for n in range(20):
        a = pa.copy()
        a[0] += 0.002 if n % 2 == 0 else -0.002
        assert not c.needs_redetect(a, pb)
        out = c.refresh(a, pb)
        assert len(out) == 1, n
        p = c.points()[0]
        np.testing.assert_array_equal(p[0:9], p0[0:9])
        assert out[0, 7] == pytest.approx(3.0)
    a = pa.copy()
    a[0] += 0.006
    assert c.needs_redetect(a, pb)
    out = c.refresh(a, pb)
    assert len(out) == 1 and out[0, 6] == pytest.approx(0.01, abs=1e-6)
    a = pa.copy()
    a[1] -= 0.035
    assert len(c.refresh(a, pb)) == 0 and len(c.points()) == 0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_reduce_keeps_the_deepest_and_spreads_the_rest(prec):
    # manifold.rs:667-684
    r = manifold_reduce([pt(0, 0, 0, 0.5), pt(0.01, 0, 0, 0.4), pt(1, 0, 0, 0.1), pt(0, 1, 0, 0.1), pt(0, 0, 1, 0.1),
                         pt(1, 1, 1, 0.05)], 4, prec)
    assert len(r) == 4
    np.testing.assert_array_equal(r[0, 0:3], [0, 0, 0])
    assert r[0, 6] == 0.5
    assert np.all((r[1:, 0:3] ** 2).sum(axis=1) > 0.5)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_reduce_leaves_small_manifolds_alone(prec):
    # manifold.rs:687-692
    pts = [pt(0, 0, 0, 0.2), pt(1, 0, 0, 0.1), pt(0, 1, 0, 0.1)]
    r = manifold_reduce(pts, 4, prec)
    np.testing.assert_array_equal(r, np.asarray(pts, dtype=np.float32 if prec == "f32" else np.float64))
