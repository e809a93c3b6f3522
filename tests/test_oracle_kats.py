"""Pins the CPU oracle against the reference's own known-answer tests.

Each test restates the assertions of one reference test (file:line cited);
the inputs and expected values come from those tests. Both precisions are
checked where the reference runs its suite under `f32` and `--features f64`.
"""
import math

import numpy as np
import pytest

from oracle_api import (ACTIVE, ISLAND_SLEEPING, OracleManifold, OracleWorld, interpolate_pose, oracle_pairs, pose)

PRECISIONS = ["f32", "f64"]
T_SPHERE = 0.017320508  # sphere.rs:91 / plane.rs:107 — 0.5*sqrt(3)*0.02


def quat_axis_angle(axis, angle):
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    s = math.sin(angle / 2)
    return (a[0] * s, a[1] * s, a[2] * s, math.cos(angle / 2))


# ------------------------------------------------------------------ shapes
@pytest.mark.parametrize("prec", PRECISIONS)
def test_pair_threshold_sphere_box(prec):
    # sphere.rs:89-91: the sphere(r=0.5) threshold is the smaller one vs box(1,1,1).
    w = OracleWorld(prec)
    s, b = w.sphere(0.5), w.box([1, 1, 1])
    assert min(w.threshold(s), w.threshold(b)) == pytest.approx(T_SPHERE, rel=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_box_world_aabb_rotated(prec):
    # box_shape.rs:57-72: corner sweep; a unit cube rotated 45 deg about Y spans sqrt(2)/2 * 2 in x.
    w = OracleWorld(prec)
    b = w.box([0.5, 0.5, 0.5])
    a = w.world_aabb(b, pose((1, 2, 3), quat_axis_angle((0, 1, 0), math.pi / 4)))
    h = math.sqrt(2) / 2
    np.testing.assert_allclose(a, [1 - h, 1.5, 3 - h, 1 + h, 2.5, 3 + h], atol=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capsule_inertia_is_positive_and_symmetric(prec):
    # capsule.rs:84-98
    w = OracleWorld(prec)
    c = w.capsule(0.3, 0.5)
    i = w.inertia(c, 2.0)
    assert i[0] == pytest.approx(i[2]) and i[0] > i[1] > 0


# ------------------------------------------------------------------ sphere.rs:93-141
@pytest.mark.parametrize("prec", PRECISIONS)
def test_spheres_overlap(prec):
    w = OracleWorld(prec)
    a, b = w.sphere(1.0), w.sphere(1.0)
    m = w.collide(a, pose(), b, pose((1.5, 0, 0)))
    assert m[0, 6] == pytest.approx(0.5, rel=1e-6)
    assert m[0, 3] == pytest.approx(1.0)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_spheres_separated(prec):
    w = OracleWorld(prec)
    a, b = w.sphere(1.0), w.sphere(1.0)
    assert len(w.collide(a, pose(), b, pose((3, 0, 0)))) == 0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_sphere_box_contact_and_band(prec):
    w = OracleWorld(prec)
    s, b = w.sphere(0.5), w.box([1, 1, 1])
    # box (A) -> sphere (B): sphere_box's own box->sphere normal, no flip (narrowphase/mod.rs:265-269)
    m = w.collide(b, pose(), s, pose((1.4, 0, 0)))
    assert m[0, 6] == pytest.approx(0.1, rel=1e-5)
    assert m[0, 3] == pytest.approx(1.0)
    m = w.collide(b, pose(), s, pose((1.51, 0, 0)))
    assert m[0, 6] == pytest.approx(-0.01, abs=1e-6)
    assert m[0, 3] == pytest.approx(1.0)
    assert len(w.collide(b, pose(), s, pose((1.6, 0, 0)))) == 0
    # sphere (A) -> box (B) flips (narrowphase/mod.rs:258-264)
    m = w.collide(s, pose((1.4, 0, 0)), b, pose())
    assert m[0, 3] == pytest.approx(-1.0)


# ------------------------------------------------------------------ plane.rs:121-230
@pytest.mark.parametrize("prec", PRECISIONS)
def test_sphere_resting_on_plane(prec):
    w = OracleWorld(prec)
    p, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
    m = w.collide(p, pose(), s, pose((0, 0.4, 0)))
    assert m[0, 4] == pytest.approx(1.0)
    assert m[0, 6] == pytest.approx(0.1, abs=1e-6)
    assert m[0, 1] == pytest.approx(-0.1, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_plane_separated_and_band(prec):
    w = OracleWorld(prec)
    p, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
    assert len(w.collide(p, pose(), s, pose((0, 2, 0)))) == 0
    m = w.collide(p, pose(), s, pose((0, 0.51, 0)))
    assert m[0, 4] == pytest.approx(1.0)
    assert m[0, 6] == pytest.approx(-0.01, abs=1e-6)
    assert len(w.collide(p, pose(), s, pose((0, 0.6, 0)))) == 0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_sphere_below_plane_flips_the_normal(prec):
    w = OracleWorld(prec)
    p, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
    m = w.collide(p, pose(), s, pose((0, -0.3, 0)))
    assert m[0, 4] == pytest.approx(-1.0)
    assert m[0, 6] == pytest.approx(0.2, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_rotated_plane_uses_the_world_normal(prec):
    w = OracleWorld(prec)
    p, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
    q = quat_axis_angle((0, 0, 1), -math.pi / 2)
    m = w.collide(p, pose((0, 0, 0), q), s, pose((0.4, 0, 0)))
    assert m[0, 3] == pytest.approx(1.0, abs=1e-6)
    assert m[0, 6] == pytest.approx(0.1, abs=1e-6)


# ------------------------------------------------------------------ box_box.rs:535-554
@pytest.mark.parametrize("prec", PRECISIONS)
def test_box_box_face_face_along_x(prec):
    w = OracleWorld(prec)
    a, b = w.box([1, 1, 1]), w.box([1, 1, 1])
    m = w.collide(a, pose(), b, pose((1.9, 0, 0)))
    assert len(m) > 0
    for p in m:
        assert p[3] == pytest.approx(1.0, abs=1e-5)
        assert p[6] == pytest.approx(0.1, abs=1e-4)
    assert len(w.collide(a, pose(), b, pose((3, 0, 0)))) == 0


# ------------------------------------------------------------------ convex_convex.rs:215-362
@pytest.mark.parametrize("prec", PRECISIONS)
def test_capsules_along_x_overlap(prec):
    w = OracleWorld(prec)
    a = w.capsule(0.5, 1.0)
    m = w.convex_convex(a, pose(), a, pose((0.7, 0, 0)))
    assert m[3] == pytest.approx(1.0, abs=1e-4)
    assert m[6] == pytest.approx(0.3, abs=1e-3)
    assert w.convex_convex(a, pose(), a, pose((2.0, 0, 0))) is None


OCTAHEDRON = [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]]


@pytest.mark.parametrize("prec", PRECISIONS)
def test_hull_hull_overlap(prec):
    w = OracleWorld(prec)
    h, s = w.hull(OCTAHEDRON), w.sphere(0.5)
    m = w.convex_convex(h, pose(), s, pose((1.25, 0, 0)))
    assert m[3] == pytest.approx(1.0, abs=1e-3)
    assert m[6] == pytest.approx(0.25, abs=1e-3)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_margin_shell_overlap_resolved_by_walk(prec):
    w = OracleWorld(prec)
    b, s = w.box([1, 1, 1]), w.sphere(0.5)
    assert w.gjk_kind(b, pose(), s, pose((0, 1.3, 0))) == 1  # Band route, no EPA
    m = w.convex_convex(b, pose(), s, pose((0, 1.3, 0)))
    assert m[4] == pytest.approx(1.0, abs=1e-3)
    assert m[6] == pytest.approx(0.2, abs=1e-3)
    assert m[1] == pytest.approx(0.8, abs=1e-3)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_deep_overlap_runs_epa_with_margins(prec):
    w = OracleWorld(prec)
    b, s = w.box([1, 1, 1]), w.sphere(0.5)
    assert w.gjk_kind(b, pose(), s, pose((0, 0.6, 0))) == 2  # Overlap route -> EPA
    m = w.convex_convex(b, pose(), s, pose((0, 0.6, 0)))
    assert m[4] == pytest.approx(1.0, abs=1e-3)
    assert m[6] == pytest.approx(0.9, abs=1e-3)
    assert m[1] == pytest.approx(0.1, abs=1e-3)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_margin_shell_separation_reports_band(prec):
    w = OracleWorld(prec)
    c, b = w.capsule(0.5, 1.0), w.box([1, 1, 1])
    m = w.convex_convex(c, pose(), b, pose((1.51, 0, 0)))
    assert m[3] == pytest.approx(1.0, abs=1e-3)
    assert m[6] == pytest.approx(-0.01, abs=1e-3)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capsule_pairs_route_through_gjk(prec):
    # narrowphase/mod.rs:273-284: capsule-* and hull-* pairs use convex_convex.
    w = OracleWorld(prec)
    c, s = w.capsule(0.5, 1.0), w.sphere(0.5)
    via_dispatch = w.collide(c, pose(), s, pose((0.9, 0.2, 0)))
    direct = w.convex_convex(c, pose(), s, pose((0.9, 0.2, 0)))
    np.testing.assert_allclose(via_dispatch[0], direct, atol=1e-12)


# ------------------------------------------------------------------ manifold.rs:411-665
def resting(pen):
    # manifold.rs:399-409: box (A) above a plane (B), one contact at the origin.
    return [[0, 0, 0, 0, 1, 0, pen]], pose((0, 0.5 - pen, 0)), pose()


@pytest.mark.parametrize("prec", PRECISIONS)
def test_refresh_reprojects_separation_and_keeps_band_points(prec):
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    c.capture(m, pa, pb, 0.02)
    pa2 = pa.copy()
    pa2[1] -= 0.015
    r = c.refresh(pa2, pb)
    assert len(r) == 1
    assert r[0, 6] == pytest.approx(-0.005, abs=1e-6)
    np.testing.assert_array_equal(r[0, 0:3], [0, 0, 0])
    np.testing.assert_array_equal(r[0, 3:6], [0, 1, 0])
    assert c.points()[0, 9] == pytest.approx(-0.005, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_refresh_drops_separated_and_sideways_drifted_points(prec):
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    c.capture(m, pa, pb, 0.02)
    pa2 = pa.copy()
    pa2[1] -= 0.05
    assert len(c.refresh(pa2, pb)) == 0 and len(c.points()) == 0
    c.capture(m, pa, pb, 0.02)
    pa3 = pa.copy()
    pa3[0] += 0.03
    assert len(c.refresh(pa3, pb)) == 0 and len(c.points()) == 0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capture_anchors_round_trip(prec):
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    c.capture(m, pa, pb, 0.02)
    p = c.points()[0]
    wa = pa[:3] + p[0:3]
    wb = pb[:3] + p[3:6]
    np.testing.assert_array_equal(wb, [0, 0, 0])
    np.testing.assert_allclose(wa, [0, 0.01, 0], atol=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capture_merges_and_inherits_the_impulse(prec):
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    c.capture(m, pa, pb, 0.02)
    c.set_impulse(0, 5.0)
    c.capture(m, pa, pb, 0.02)
    assert c.points()[0, 10] == pytest.approx(5.0)
    c.capture([[0, 0, 0, 0, -1, 0, 0.01]], pa, pb, 0.02)  # flipped normal: no match
    pts = c.points()
    assert len(pts) == 2
    assert pts[0, 10] == pytest.approx(5.0) and pts[1, 10] == 0.0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_refresh_lifetime_and_capture_reset(prec):
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    c.capture(m, pa, pb, 0.02)
    assert c.points()[0, 11] == 0
    for step in range(1, 6):
        r = c.refresh(pa, pb)
        assert len(r) == 1 and r[0, 8] == step and c.points()[0, 11] == step
    c.capture(m, pa, pb, 0.02)
    assert c.points()[0, 11] == 0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_redetect_triggers_on_relative_drift_only(prec):
    m, pa, pb = resting(0.01)
    c = OracleManifold(prec)
    assert c.needs_redetect(pa, pb)
    c.capture(m, pa, pb, 0.02)
    p = pa.copy(); p[1] += 0.004
    assert not c.needs_redetect(p, pb)
    p = pa.copy(); p[1] += 0.006
    assert c.needs_redetect(p, pb)
    q = pa.copy(); q[3:7] = quat_axis_angle((0, 0, 1), 0.02)
    assert c.needs_redetect(q, pb)
    a2, b2 = pa.copy(), pb.copy()
    a2[0] += 1
    b2[0] += 1
    assert not c.needs_redetect(a2, b2)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capture_overflow_keeps_the_deepest_four(prec):
    # manifold.rs:364-370: overflow sorts deepest-first (stable) and truncates to four.
    c = OracleManifold(prec)
    pts = [[0.1 * k, 0, 0, 0, 1, 0, 0.001 * (k % 3)] for k in range(6)]
    c.capture(pts, pose(), pose(), 0.02)
    p = c.points()
    assert len(p) == 4
    assert list(np.round(p[:, 9], 6)) == [0.002, 0.002, 0.001, 0.001]
    # equal depths keep their order: the 0.002 points are k=2 then k=5
    assert p[0, 0] == pytest.approx(0.2) and p[1, 0] == pytest.approx(0.5)


# ------------------------------------------------------------------ sequential_impulse.rs:1020-1645
def deep_contact_world(pen, prec, **info):
    w = OracleWorld(prec)
    w.set_solver(**info)
    g, c = w.plane([0, 1, 0], 0.0), w.box([0.5, 0.5, 0.5])
    w.add_body(g, [0, 0, 0], mass=0)
    w.add_body(c, [0, 0.5 - pen, 0], mass=1.0)
    contacts = [[0, 1, 0, -pen, 0, 0, 1, 0, pen, 0]]
    return w, contacts


@pytest.mark.parametrize("prec", PRECISIONS)
def test_split_impulse_pushes_deep_penetration_without_touching_velocity(prec):
    w, c = deep_contact_world(0.1, prec)
    rows = w.solve_contacts(c, 60.0)
    assert w.push()[1, 1] > 0
    assert w.state()[1, 8] == pytest.approx(0.0, abs=1e-6)
    assert rows[0, 17] == 1


@pytest.mark.parametrize("prec", PRECISIONS)
def test_split_impulse_ignores_shallow_penetration(prec):
    w, c = deep_contact_world(0.01, prec)
    rows = w.solve_contacts(c, 60.0)
    assert rows[0, 17] == 0
    np.testing.assert_array_equal(w.push()[1, :3], [0, 0, 0])


@pytest.mark.parametrize("prec", PRECISIONS)
def test_split_impulse_converges_and_clamps(prec):
    w, c = deep_contact_world(0.1, prec, num_iterations=5)
    w.solve_contacts(c, 60.0)
    push5 = w.push()[1, 1]
    w2, c2 = deep_contact_world(0.1, prec, num_iterations=20)
    w2.solve_contacts(c2, 60.0)
    assert push5 > 0 and w2.push()[1, 1] >= push5


def sphere_row(prec, sphere_y, cp_y, pen, **info):
    w = OracleWorld(prec)
    w.set_solver(**info)
    g, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
    w.add_body(g, [0, 0, 0], mass=0)
    w.add_body(s, [0, sphere_y, 0], mass=1.0)
    return w.solve_contacts([[0, 1, 0, cp_y, 0, 0, 1, 0, pen, 0]], 60.0)[0], w


@pytest.mark.parametrize("prec", PRECISIONS)
def test_solver_info_erp2_and_slop(prec):
    row, _ = sphere_row(prec, 0.49, -0.01, 0.01)
    assert row[25] == pytest.approx(0.2, abs=1e-7)
    row, _ = sphere_row(prec, 0.49, -0.01, 0.01, erp2=0.4)
    assert row[25] == pytest.approx(0.4, abs=1e-7)
    row, _ = sphere_row(prec, 0.497, -0.003, 0.003)
    assert row[23] == pytest.approx(0.0, abs=1e-12)
    row, _ = sphere_row(prec, 0.497, -0.003, 0.003, linear_slop=0.0)
    assert row[23] == pytest.approx(0.003, abs=1e-7)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_solver_info_restitution_threshold_gates_low_speed_bounces(prec):
    for thr, expected in [(1.0, 0.0), (0.2, 0.5)]:
        w = OracleWorld(prec)
        w.set_solver(num_iterations=1, restitution_threshold=thr)
        g, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
        w.add_body(g, [0, 0, 0], mass=0, restitution=1.0)
        w.add_body(s, [0, 0.5, 0], mass=1.0, restitution=1.0, linvel=(0, -0.5, 0))
        w.solve_contacts([[0, 1, 0, 0, 0, 0, 1, 0, 0.0, 0]], 60.0)
        assert w.state()[1, 8] == pytest.approx(expected, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_solver_info_split_switch_and_threshold(prec):
    w, c = deep_contact_world(0.1, prec, split_impulse=False)
    rows = w.solve_contacts(c, 60.0)
    assert rows[0, 17] == 0 and w.state()[1, 8] > 0
    row, _ = sphere_row(prec, 0.45, -0.05, 0.05)
    assert row[17] == 1
    row, _ = sphere_row(prec, 0.45, -0.05, 0.05, split_threshold=-0.1)
    assert row[17] == 0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_solver_info_global_cfm_and_sor(prec):
    rigid, _ = sphere_row(prec, 0.49, -0.01, 0.01)
    assert rigid[24] == 0.0
    soft, _ = sphere_row(prec, 0.49, -0.01, 0.01, global_cfm=0.1)
    assert soft[24] > 0 and soft[20] < rigid[20]
    relaxed, _ = sphere_row(prec, 0.49, -0.01, 0.01, sor=2.0)
    assert relaxed[20] == pytest.approx(rigid[20] * 2, rel=1e-6)
    assert relaxed[21] == pytest.approx(rigid[21] * 2, rel=1e-6)
    assert relaxed[22] == pytest.approx(rigid[22] * 2, rel=1e-6)


# ------------------------------------------------------------------ body.rs:1405-1487
@pytest.mark.parametrize("prec", PRECISIONS)
def test_integrate_position_matches_the_exact_rotation(prec):
    q = interpolate_pose((0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (0, 0, 0.5), 1.0, prec)[3:]
    expected = np.array([0, 0, math.sin(0.25), math.cos(0.25)])
    assert abs(np.dot(q, expected)) > 1 - 1e-5


@pytest.mark.parametrize("prec", PRECISIONS)
def test_integrate_position_keeps_the_rotation_angle(prec):
    q = interpolate_pose((0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (0, 0.7, 0), 1.0, prec)[3:]
    assert abs(2 * math.acos(q[3]) - 0.7) < 1e-5


def world_angular_momentum(inv_inertia, state):
    x, y, z, w = state[3:7]
    omega = state[10:13]

    def rot(qx, qy, qz, qw, v):
        b = np.array([qx, qy, qz])
        return v * (qw * qw - b @ b) + b * (2 * (v @ b)) + np.cross(b, v) * (2 * qw)

    ob = rot(-x, -y, -z, w, omega)
    return rot(x, y, z, w, (1.0 / inv_inertia) * ob)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gyroscopic_conserves_angular_momentum_of_a_tumbling_body(prec):
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    b = w.box([0.5, 0.25, 0.1])
    q = np.array([0.2, 0.3, 0.4, 0.5])
    q = q / np.linalg.norm(q)
    w.add_body(b, [0, 0, 0], quat=q, angvel=(3, 1, -2), mass=1.0)
    inv = 1.0 / w.inertia(b, 1.0)
    l0 = world_angular_momentum(inv, w.state()[0])
    max_defl, max_drift = 0.0, 0.0
    for _ in range(120):
        w.step(1 / 60)
        l = world_angular_momentum(inv, w.state()[0])
        max_defl = max(max_defl, l0 @ l / (np.linalg.norm(l0) * np.linalg.norm(l)))
        max_drift = max(max_drift, np.linalg.norm(l - l0))
    assert max_defl > math.cos(0.15)
    assert max_drift < 0.3 * np.linalg.norm(l0)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_gyroscopic_is_zero_for_isotropic_inertia(prec):
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    s = w.sphere(0.5)
    q = np.array([0.2, 0.4, 0.6, 0.65])
    w.add_body(s, [0, 0, 0], quat=q / np.linalg.norm(q), angvel=(0.3, -1.0, 2.0), mass=1.0)
    w.step(1 / 60)
    np.testing.assert_allclose(w.state()[0, 10:13], [0.3, -1.0, 2.0], atol=1e-6)


# ------------------------------------------------------------------ broadphase (brute_force.rs:54-68, dbvt.rs:831-905)
class RefRng:
    """The reference tests' LCG (dbvt.rs:831-855), with f32 AABB assembly."""

    def __init__(self, seed):
        self.s = seed & 0xFFFFFFFFFFFFFFFF

    def next(self):
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return self.s

    def aabb(self, spread, size):
        f = np.float32
        base = [f((self.next() >> 32) % spread) / f(10), f((self.next() >> 16) % spread) / f(10),
                f(self.next() % spread) / f(10)]
        ext = [f((self.next() >> 32) % size) / f(100) + f(0.1), f((self.next() >> 16) % size) / f(100) + f(0.1),
               f(self.next() % size) / f(100) + f(0.1)]
        return [base[0], base[1], base[2], base[0] + ext[0], base[1] + ext[1], base[2] + ext[2]]


def ref_scattered_boxes(seed, n, spread, size):
    r = RefRng(seed)
    return np.array([r.aabb(spread, size) for _ in range(n)], dtype=np.float32)


def test_sweep_matches_brute_force_on_scattered_boxes():
    # dbvt.rs:896-905: 64 boxes from Rng(0x9e3779b97f4a7c15).aabb(1000, 100)
    a = ref_scattered_boxes(0x9E3779B97F4A7C15, 64, 1000, 100)
    bf = oracle_pairs(a, 0)
    sw = oracle_pairs(a, 1)
    np.testing.assert_array_equal(bf, sw)


def test_broadphase_contract_closed_bounds_and_order():
    # util.rs:28-38 touching counts; brute_force.rs:54-68 lexicographic (i<j) order.
    a = np.array([[0, 0, 0, 1, 1, 1], [1, 0, 0, 2, 1, 1], [2, 0, 0, 3, 1, 1], [0.5, 0.5, 5, 1.5, 1.5, 6],
                  [-1e30, -1e30, -1e30, 1e30, 1e30, 1e30]], dtype=np.float32)
    bf = oracle_pairs(a, 0)
    assert [tuple(p) for p in bf] == [(0, 1), (0, 4), (1, 2), (1, 4), (2, 4), (3, 4)]
    np.testing.assert_array_equal(bf, oracle_pairs(a, 1))


@pytest.mark.parametrize("seed", range(4))
def test_sweep_and_grid_match_brute_force_dense_sets(seed):
    a = ref_scattered_boxes(0xDB4E7F4A7C150001 ^ ((seed * 0x517CC1B727220A95) & 0xFFFFFFFFFFFFFFFF), 512, 300, 300)
    bf = oracle_pairs(a, 0)
    np.testing.assert_array_equal(bf, oracle_pairs(a, 1))
    np.testing.assert_array_equal(bf, oracle_pairs(a, 2))
    big = np.array([[-1e30, -1e30, -1e30, 1e30, 1e30, 1e30]], dtype=np.float32)
    b = np.concatenate([a[:100], big, a[100:], big], axis=0)
    np.testing.assert_array_equal(oracle_pairs(b, 0), oracle_pairs(b, 2))


# ------------------------------------------------------------------ world-level
@pytest.mark.parametrize("prec", PRECISIONS)
def test_falling_box_settles(prec):
    # examples/falling_box.rs:9-50 (20 iterations, box ground, y ~ 0.5 +- 0.05 after 5 s)
    w = OracleWorld(prec)
    w.set_solver(num_iterations=20)
    g, c = w.box([25, 0.5, 25]), w.box([0.5, 0.5, 0.5])
    w.add_body(g, [0, -0.5, 0], mass=0)
    w.add_body(c, [0, 5, 0], mass=1.0, friction=0.6)
    for _ in range(300):
        w.step(1 / 60)
    assert abs(w.state()[1, 1] - 0.5) < 0.05


@pytest.mark.parametrize("prec", PRECISIONS)
def test_falling_box_ledger_transient(prec):
    # docs/bullet-compare.md:40-80 (falling_box, 10 iterations): free fall is exact
    # (y_n = 5 - g dt^2 n(n+1)/2 through frame 56) and the predicted-pose detection
    # stops the cube at y = 0.650909 on frame 57 — the ledger's 0.155333 peak
    # deviation against Bullet's free-fall 0.495575.
    w = OracleWorld(prec)
    g, c = w.box([25, 0.5, 25]), w.box([0.5, 0.5, 0.5])
    w.add_body(g, [0, -0.5, 0], mass=0)
    w.add_body(c, [0, 5, 0], mass=1.0, friction=0.6)
    ys = []
    for _ in range(57):
        w.step(1 / 60)
        ys.append(w.state()[1, 1])
    gdt2 = 9.81 / 3600
    for n in (10, 30, 55, 56):
        assert ys[n - 1] == pytest.approx(5 - gdt2 * n * (n + 1) / 2, abs=2e-5)
    bullet_free_fall_57 = 5 - gdt2 * 57 * 58 / 2
    assert ys[56] - bullet_free_fall_57 == pytest.approx(0.155333, abs=5e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_step_simulation_persists_contact_impulses(prec):
    # world/step.rs:1941-1967
    w = OracleWorld(prec)
    p, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
    w.add_body(p, [0, 0, 0], mass=0)
    w.add_body(s, [0, 2, 0], mass=1.0)
    for _ in range(90):
        w.step(1 / 60)
    rows = w.rows()
    assert w.num_manifolds() >= 1 and np.any(rows[:, 13] > 0)
    st = w.state()[1]
    assert st[1] == pytest.approx(0.5, abs=0.05)
    assert np.linalg.norm(st[7:10]) < 0.1


@pytest.mark.parametrize("prec", PRECISIONS)
def test_band_contact_survives_brief_separation(prec):
    # world/step.rs:1974-2005 (gravity-free; nudge inside the redetect window)
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    p, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
    w.add_body(p, [0, 0, 0], mass=0)
    w.add_body(s, [0, 0.4999, 0], mass=1.0)
    w.step(1 / 60)
    assert w.num_manifolds() == 1
    st = w.state()
    st[1, 0:3] = [0, 0.5039, 0]
    w.set_state(st)
    w.step(1 / 60)
    rows = w.rows()
    assert np.any(rows[:, 12] < 0)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_band_contact_catches_a_falling_sphere_before_touching(prec):
    # world/step.rs:2012-2032
    w = OracleWorld(prec)
    p, s = w.plane([0, 1, 0], 0.0), w.sphere(0.5)
    w.add_body(p, [0, 0, 0], mass=0)
    w.add_body(s, [0, 0.508, 0], mass=1.0)
    min_y = math.inf
    for _ in range(60):
        w.step(1 / 60)
        min_y = min(min_y, w.state()[1, 1])
    assert min_y > 0.5 - 0.006
    assert w.state()[1, 1] == pytest.approx(0.5, abs=0.006)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_resting_box_goes_to_sleep_and_keeps_its_manifold(prec):
    # body.rs:639-657 (2 s below the thresholds) + world/islands.rs:281-294 (island sleep);
    # a sleeping pair keeps its manifold (step.rs:665-691).
    w = OracleWorld(prec)
    p, c = w.plane([0, 1, 0], 0.0), w.box([0.5, 0.5, 0.5])
    w.add_body(p, [0, 0, 0], mass=0)
    w.add_body(c, [0, 0.5, 0], mass=1.0)
    for _ in range(30):
        w.step(1 / 60)
    assert w.state()[1, 13] == ACTIVE
    for _ in range(200):
        w.step(1 / 60)
    assert w.state()[1, 13] == ISLAND_SLEEPING
    assert w.num_manifolds() == 1
