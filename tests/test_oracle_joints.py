"""Oracle joints pinned by the reference's own joint tests.

Each case restates the scene and the assertions of a test in
crates/bullet-dynamics/src/constraint/tests.rs (point-to-point, hinge and fixed
joints; the line of each test is cited), run through the oracle's full step in
both precisions.
"""
import math

import numpy as np
import pytest

import oracle_api as orc

DT = 1.0 / 60.0
PRECISIONS = ["f32", "f64"]


def quat_z(a):  # Quaternion::from_rotation_z
    return (0.0, 0.0, math.sin(a / 2), math.cos(a / 2))


def rotate(q, v):
    x, y, z, w = q
    b = np.array([x, y, z])
    v = np.asarray(v, dtype=np.float64)
    return v * (w * w - b @ b) + b * (2 * (v @ b)) + np.cross(b, v) * (2 * w)


def quat_angle(q):  # conetwist.rs:546-548
    return 2.0 * math.acos(max(-1.0, min(1.0, q[3])))


def qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return (aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
            aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz)


def world(precision, gravity=(0.0, -9.81, 0.0)):
    w = orc.OracleWorld(precision)
    w.set_gravity(gravity)
    return w


def p2p(w, a, b, pivot_a, pivot_b, **kw):
    return w.add_joint(orc.joint_desc(orc.JOINT_POINT2POINT, a, b, orc.frame(pivot_a), orc.frame(pivot_b), **kw))


def pendulum(precision, bob_offset, anchor_offset):
    w = world(precision)
    anchor_shape = w.add_shape(orc.BOX, [0.2, 0.2, 0.2])
    bob_shape = w.add_shape(orc.SPHERE, [0.1])
    anchor = w.add_body(anchor_shape, (0, 0, 0), mass=0.0)
    bob = w.add_body(bob_shape, tuple(np.subtract(anchor_offset, bob_offset)), mass=1.0)
    p2p(w, bob, anchor, bob_offset, anchor_offset)
    return w, bob


def set_pose(w, i, pos=None, quat=None, linvel=None, angvel=None):
    st = w.state()
    if pos is not None:
        st[i, 0:3] = pos
    if quat is not None:
        st[i, 3:7] = quat
    if linvel is not None:
        st[i, 7:10] = linvel
    if angvel is not None:
        st[i, 10:13] = angvel
    w.set_state(st)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_pendulum_swings_and_keeps_the_pivot(precision):  # tests.rs:46-91
    w, bob = pendulum(precision, (-1.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    a45 = math.pi / 4
    set_pose(w, bob, pos=(math.sin(a45), -math.cos(a45), 0.0), quat=quat_z(-a45))
    max_err, min_x, max_speed, crossings = 0.0, math.inf, 0.0, 0
    prev_x = w.state()[bob, 0]
    for _ in range(600):
        w.step(DT)
        s = w.state()[bob]
        max_err = max(max_err, float(np.linalg.norm(s[0:3] + rotate(s[3:7], (-1.0, 0.0, 0.0)))))
        min_x = min(min_x, s[0])
        max_speed = max(max_speed, float(np.linalg.norm(s[7:10])))
        if prev_x > 0.0 and s[0] <= 0.0:
            crossings += 1
        prev_x = s[0]
    assert max_err < 0.2 and crossings >= 3 and min_x < -0.5 and max_speed > 1.5


@pytest.mark.parametrize("precision", PRECISIONS)
def test_pendulum_hangs_at_equilibrium(precision):  # tests.rs:94-121
    w, bob = pendulum(precision, (0.0, 1.0, 0.0), (0.0, 1.0, 0.0))
    for _ in range(600):
        w.step(DT)
    s = w.state()[bob]
    pivot = s[0:3] + rotate(s[3:7], (0.0, 1.0, 0.0))
    assert np.linalg.norm(pivot - (0.0, 1.0, 0.0)) < 0.01
    assert np.linalg.norm(s[0:3]) < 0.02
    assert np.linalg.norm(s[7:10]) < 0.05


@pytest.mark.parametrize("precision", PRECISIONS)
def test_two_link_chain_keeps_its_lengths(precision):  # tests.rs:124-176
    w = world(precision)
    anchor = w.add_body(w.add_shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    sph = w.add_shape(orc.SPHERE, [0.1])
    upper = w.add_body(sph, (0.0, -1.0, 0.0), mass=1.0)
    lower = w.add_body(sph, (0.0, -3.0, 0.0), mass=1.0)
    p2p(w, upper, anchor, (0.0, 1.0, 0.0), (0.0, 0.0, 0.0))
    p2p(w, lower, upper, (0.0, 1.0, 0.0), (0.0, -1.0, 0.0))
    set_pose(w, lower, linvel=(2.0, 0.0, 0.0))
    max_err = 0.0
    for _ in range(300):
        w.step(DT)
        s = w.state()
        u, l = s[upper], s[lower]
        max_err = max(max_err, float(np.linalg.norm(u[0:3] + rotate(u[3:7], (0, 1, 0)))),
                      float(np.linalg.norm(l[0:3] + rotate(l[3:7], (0, 1, 0)) - (u[0:3] + rotate(u[3:7], (0, -1, 0))))))
    assert max_err < 0.2


def door_world(precision, gravity=(0.0, -9.81, 0.0), door_pos=(0.0, 0.5, 0.0), open_45=True):
    w = world(precision, gravity)
    anchor = w.add_body(w.add_shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    door = w.add_body(w.add_shape(orc.BOX, [0.5, 0.5, 0.2]), door_pos, mass=2.0)
    if open_45:
        a45 = math.pi / 4
        set_pose(w, door, pos=(math.cos(a45) * 0.5, math.sin(a45) * 0.5, 0.0), quat=quat_z(a45))
    fa, fb = orc.hinge_frames((-0.5, 0.0, 0.0), (0, 0, 1), (0, 0, 0), (0, 0, 1), precision)
    return w, door, anchor, fa, fb


@pytest.mark.parametrize("precision", PRECISIONS)
def test_hinge_swings_and_keeps_axis_aligned(precision):  # tests.rs:180-235
    w, door, anchor, fa, fb = door_world(precision)
    w.add_joint(orc.joint_desc(orc.JOINT_HINGE, door, anchor, fa, fb))
    max_pivot, min_align, max_angle, crossings, prev = 0.0, 1.0, 0.0, 0, 0.0
    for step in range(600):
        w.step(DT)
        d = w.state()[door]
        max_pivot = max(max_pivot, float(np.linalg.norm(d[0:3] + rotate(d[3:7], (-0.5, 0.0, 0.0)))))
        min_align = min(min_align, abs(rotate(d[3:7], (0, 0, 1))[2]))
        angle = w.joint_angles(1)[0]
        max_angle = max(max_angle, abs(angle))
        if step > 0 and prev > 0.0 and angle <= 0.0:
            crossings += 1
        prev = angle
    assert max_pivot < 0.2 and min_align > 0.99 and max_angle > 0.5 and crossings >= 3


@pytest.mark.parametrize("precision", PRECISIONS)
def test_hinge_limit_stops_the_door(precision):  # tests.rs:238-281
    w, door, anchor, fa, fb = door_world(precision, door_pos=(0.0, 0.0, 0.0))
    w.add_joint(orc.joint_desc(orc.JOINT_HINGE, door, anchor, fa, fb,
                               flags=orc.JF_DISABLE_COLLISIONS | orc.JF_LIMIT, limit=(-0.3, 0.3)))
    min_angle = 0.0
    for _ in range(600):
        w.step(DT)
        min_angle = min(min_angle, w.joint_angles(1)[0])
    assert min_angle > -0.35
    assert abs(w.joint_angles(1)[0] + 0.3) < 0.05


@pytest.mark.parametrize("precision", PRECISIONS)
def test_hinge_motor_rotates_the_door(precision):  # tests.rs:284-316
    w, door, anchor, fa, fb = door_world(precision, gravity=(0.0, 0.0, 0.0), door_pos=(0.5, 0.0, 0.0), open_45=False)
    w.add_joint(orc.joint_desc(orc.JOINT_HINGE, door, anchor, fa, fb,
                               flags=orc.JF_DISABLE_COLLISIONS | orc.JF_MOTOR, motor=(1.0, 1000.0)))
    for _ in range(180):
        w.step(DT)
    assert abs(w.joint_angles(1)[0] - 3.0) < 1.0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_joint_suppresses_collisions_between_linked_bodies(precision):  # tests.rs:320-360
    def run(with_joint):
        w = world(precision, (0.0, 0.0, 0.0))
        box = w.add_shape(orc.BOX, [0.5, 0.5, 0.5])
        a = w.add_body(box, (0, 0, 0), mass=1.0)
        b = w.add_body(box, (0, 0, 0), mass=1.0)
        if with_joint:
            p2p(w, a, b, (0, 0, 0), (0, 0, 0))
        for _ in range(30):
            w.step(DT)
        s = w.state()
        return s[b, 0:3] - s[a, 0:3]

    assert np.linalg.norm(run(False)) > 0.05
    assert np.linalg.norm(run(True)) < 0.02


@pytest.mark.parametrize("precision", PRECISIONS)
def test_impulse_clamp_limits_the_support_impulse(precision):  # tests.rs:363-400
    def run(clamp):
        w = world(precision)
        anchor = w.add_body(w.add_shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
        bob = w.add_body(w.add_shape(orc.SPHERE, [0.1]), (0, 0, 0), mass=10.0)
        p2p(w, bob, anchor, (0, 0, 0), (0, 0, 0), impulse_clamp=clamp)
        for _ in range(300):
            w.step(DT)
        return w.state()[bob, 1]

    assert run(0.1) < -1.0
    assert abs(run(0.0)) < 0.05


@pytest.mark.parametrize("precision", PRECISIONS)
def test_fixed_joint_locks_a_rigid_assembly(precision):  # tests.rs:403-458
    w = world(precision)
    anchor = w.add_body(w.add_shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    box = w.add_body(w.add_shape(orc.BOX, [0.3, 0.3, 0.3]), (0.0, 1.0, 0.0), mass=1.0)
    w.add_joint(orc.joint_desc(orc.JOINT_FIXED, box, anchor, orc.frame((0.0, 0.5, 0.0)), orc.frame((0.0, 1.5, 0.0))))
    set_pose(w, box, linvel=(2.0, 0.0, 0.0), angvel=(0.0, 0.0, 4.0))
    max_rel = 0.0
    for _ in range(600):
        w.step(DT)
        max_rel = max(max_rel, quat_angle(w.state()[box, 3:7]))
    b = w.state()[box]
    assert max_rel < 0.5
    assert np.linalg.norm(b[0:3] - (0.0, 1.0, 0.0)) < 0.03
    assert np.linalg.norm(b[10:13]) < 0.05
    assert np.linalg.norm(b[0:3] + rotate(b[3:7], (0.0, 0.5, 0.0)) - (0.0, 1.5, 0.0)) < 0.03


@pytest.mark.parametrize("precision", PRECISIONS)
def test_fixed_joint_welds_two_dynamic_bodies(precision):  # tests.rs:461-515
    w = world(precision)
    w.add_body(w.add_shape(orc.PLANE, [0.0, 1.0, 0.0, 0.0]), (0, 0, 0), mass=0.0)
    box = w.add_shape(orc.BOX, [0.4, 0.4, 0.4])
    a = w.add_body(box, (0.0, 1.2, 0.0), mass=1.0)
    b = w.add_body(box, (0.0, 1.6, 0.0), mass=1.0)
    w.add_joint(orc.joint_desc(orc.JOINT_FIXED, a, b, orc.frame((0.0, 0.2, 0.0)), orc.frame((0.0, -0.2, 0.0))))
    set_pose(w, a, angvel=(1.0, 2.0, 0.0))
    set_pose(w, b, angvel=(1.0, 2.0, 0.0))
    max_rel, max_pivot = 0.0, 0.0
    for _ in range(300):
        w.step(DT)
        s = w.state()
        qa, qb = s[a, 3:7], s[b, 3:7]
        rel = qmul((-qb[0], -qb[1], -qb[2], qb[3]), tuple(qa))
        max_rel = max(max_rel, quat_angle(rel))
        pa = s[a, 0:3] + rotate(qa, (0.0, 0.2, 0.0))
        pb = s[b, 0:3] + rotate(qb, (0.0, -0.2, 0.0))
        max_pivot = max(max_pivot, float(np.linalg.norm(pb - pa)))
    assert max_rel < 0.15 and max_pivot < 0.15


def test_hinge_frames_follow_the_pivot_axis_recipe():  # hinge.rs:60-100
    fa, fb = orc.hinge_frames((1.0, 2.0, 3.0), (0.0, 0.0, 2.0), (-1.0, 0.0, 0.5), (0.0, 1.0, 0.0), "f64")
    ba = fa[3:].reshape(3, 3).T
    bb = fb[3:].reshape(3, 3).T
    np.testing.assert_allclose(fa[:3], (1.0, 2.0, 3.0))
    np.testing.assert_allclose(ba[:, 2], (0.0, 0.0, 1.0), atol=1e-12)
    np.testing.assert_allclose(bb[:, 2], (0.0, 1.0, 0.0), atol=1e-12)
    for basis in (ba, bb):  # orthonormal, right-handed
        np.testing.assert_allclose(basis.T @ basis, np.eye(3), atol=1e-12)
        assert np.linalg.det(basis) == pytest.approx(1.0)
    # t1 = axis x (X when |axis.x| < 0.9), normalized; frame B's X is t1 carried by the shortest arc
    np.testing.assert_allclose(ba[:, 0], (0.0, 1.0, 0.0), atol=1e-12)


def gear_world(precision, pos_b, ratio, quat_a=(0, 0, 0, 1)):
    w = world(precision, (0.0, 0.0, 0.0))
    sph = w.add_shape(orc.SPHERE, [0.5])
    a = w.add_body(sph, (0, 0, 0), quat=quat_a, mass=2.0 if ratio == 2.0 else 1.0)
    b = w.add_body(sph, pos_b, mass=2.0 if ratio == 2.0 else 1.0)
    w.add_joint(orc.joint_desc(orc.JOINT_GEAR, a, b, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)), gear_ratio=ratio))
    return w, a, b


@pytest.mark.parametrize("precision", PRECISIONS)
def test_gears_couple_parallel_axes_to_opposite_spins(precision):  # gear.rs:77-101
    w, a, b = gear_world(precision, (3.0, 0.0, 0.0), 2.0)
    set_pose(w, a, angvel=(0.0, 0.0, 6.0))
    for _ in range(10):
        w.step(DT)
    s = w.state()
    wa, wb = s[a, 12], s[b, 12]
    assert abs(wa - 4.8) < 1e-2 and abs(wb + 2.4) < 1e-2 and abs(wb + wa / 2.0) < 1e-3


@pytest.mark.parametrize("precision", PRECISIONS)
def test_gear_offset_bodies_feel_no_position_pull(precision):  # gear.rs:122-157
    w, a, b = gear_world(precision, (5.0, 1.0, -2.0), 1.0)
    set_pose(w, a, angvel=(0.0, 0.0, 6.0))
    before = w.state()
    for _ in range(30):
        w.step(DT)
    s = w.state()
    assert abs(s[a, 0] - before[a, 0]) < 1e-5 and abs(s[a, 1] - before[a, 1]) < 1e-5
    assert abs(s[b, 0] - before[b, 0]) < 1e-5 and abs(s[b, 2] - before[b, 2]) < 1e-5
    assert abs(s[b, 12] + s[a, 12]) < 1e-3


@pytest.mark.parametrize("precision", PRECISIONS)
def test_gear_local_axes_follow_body_rotation(precision):  # gear.rs:159-187
    q = (math.sin(math.pi / 4), 0.0, 0.0, math.cos(math.pi / 4))
    w, a, b = gear_world(precision, (4.0, 0.0, 0.0), 1.0, quat_a=q)
    set_pose(w, a, angvel=(0.0, -6.0, 0.0))
    for _ in range(10):
        w.step(DT)
    s = w.state()
    assert abs(s[a, 11] + 3.0) < 1e-2 and abs(s[b, 12] + 3.0) < 1e-2


def slider_world(precision, box_pos, **kw):
    w = world(precision, (0.0, 0.0, 0.0))
    anchor = w.add_body(w.add_shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    box = w.add_body(w.add_shape(orc.BOX, [0.3, 0.3, 0.3]), box_pos, mass=1.0)
    w.add_joint(orc.joint_desc(orc.JOINT_SLIDER, anchor, box, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)), **kw))
    return w, box


@pytest.mark.parametrize("precision", PRECISIONS)
def test_slider_slides_along_its_axis(precision):  # tests.rs:608-646
    w, box = slider_world(precision, (1.0, 0.0, 0.0))
    set_pose(w, box, linvel=(1.5, 0.5, 0.2), angvel=(0.0, 0.0, 3.0))
    max_off, max_rel = 0.0, 0.0
    for _ in range(180):
        w.step(DT)
        s = w.state()[box]
        max_off = max(max_off, abs(s[1]), abs(s[2]))
        max_rel = max(max_rel, quat_angle(s[3:7]))
    assert w.state()[box, 0] > 1.1 and max_off < 0.05 and max_rel < 0.15


@pytest.mark.parametrize("precision", PRECISIONS)
def test_slider_limit_stops_the_slide(precision):  # tests.rs:651-692
    w, box = slider_world(precision, (0.2, 0.0, 0.0), lin_limits=(-0.3, 0.3))
    set_pose(w, box, linvel=(4.0, 0.0, 0.0))
    max_x, fired = 0.0, False
    for _ in range(180):
        w.step(DT)
        rows = w.joint_rows()
        fired |= bool(np.any((rows[:, 5] == 2) | (rows[:, 5] == 3)))  # a one-sided limit row
        max_x = max(max_x, w.state()[box, 0])
    assert max_x < 0.34 and fired and w.state()[box, 0] < 0.3


@pytest.mark.parametrize("precision", PRECISIONS)
def test_slider_motor_drives_along_the_axis(precision):  # tests.rs:697-735
    w, box = slider_world(precision, (0.0, 0.0, 0.0), flags=orc.JF_DISABLE_COLLISIONS | orc.JF_LIN_MOTOR,
                          lin_motor=(1.5, 100.0))
    for _ in range(150):
        w.step(DT)
    s = w.state()[box]
    assert abs(s[0] - 3.75) < 0.3 and abs(s[7]) < 1.8


@pytest.mark.parametrize("precision", PRECISIONS)
def test_slider_angular_limit_stops_the_twist(precision):  # tests.rs:738-771
    w, box = slider_world(precision, (0.0, 0.0, 0.0), ang_limits=(-0.4, 0.4))
    set_pose(w, box, angvel=(3.0, 0.0, 0.0))
    max_ang = 0.0
    for _ in range(180):
        w.step(DT)
        max_ang = max(max_ang, abs(w.joint_angles(1)[0]))
    assert max_ang < 0.5


def cone_world(precision, spans, angvel, gravity=(0.0, -9.81, 0.0), motor=None):
    """tests.rs:518-600: a 0.1 m bob pinned at a static anchor by a cone twist whose cone axis is X
    on both bodies (identity frames at the origin)."""
    w = world(precision, gravity)
    anchor = w.add_body(w.add_shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    bob = w.add_body(w.add_shape(orc.SPHERE, [0.1]), (0, 0, 0), angvel=angvel, mass=1.0)
    kw = dict(cone=tuple(spans) + (1.0, 0.3, 1.0))
    flags = orc.JF_DISABLE_COLLISIONS
    if motor is not None:
        kw["cone_motor"] = motor
        flags |= JF_CONE_MOTOR
    w.add_joint(orc.joint_desc(orc.JOINT_CONETWIST, bob, anchor, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)),
                               flags=flags, **kw))
    return w, anchor, bob


JF_CONE_MOTOR = 512


def axis_angle_between(st, a, b):
    ax_a, ax_b = rotate(st[a, 3:7], (1, 0, 0)), rotate(st[b, 3:7], (1, 0, 0))
    return math.acos(max(-1.0, min(1.0, float(ax_a @ ax_b))))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_cone_twist_limits_the_swing(precision):  # tests.rs:518-560
    w, anchor, bob = cone_world(precision, (0.44, 0.44, -1.0), (0.0, 0.0, 4.0))
    max_swing = 0.0
    for _ in range(600):
        w.step(DT)
        max_swing = max(max_swing, axis_angle_between(w.state(), anchor, bob))
    assert 0.3 < max_swing < 0.55


@pytest.mark.parametrize("precision", PRECISIONS)
def test_cone_twist_locks_the_twist(precision):  # tests.rs:563-600
    w, anchor, bob = cone_world(precision, (0.9, 0.9, 0.0), (6.0, 0.0, 0.0))
    max_twist = 0.0
    for _ in range(300):
        w.step(DT)
        max_twist = max(max_twist, w.joint_angles(1)[0])
    assert max_twist < 0.1
    assert abs(w.state()[bob, 10]) < 0.1


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("spans, limit", [((0.0, 0.0, 1e30), 0.1), ((0.0, 0.5, 1e30), 0.62), ((0.5, 0.0, 1e30), 0.62)])
def test_cone_twist_fixed_and_hinge_configurations(precision, spans, limit):
    """conetwist.rs:406-461: a span below the fix threshold (0.05) turns the cone into a hinge
    about the other axis (limited by the other span) or, both below, locks the X axes together."""
    w, anchor, bob = cone_world(precision, spans, (0.0, 3.0, 3.0))
    max_swing = 0.0
    for _ in range(240):
        w.step(DT)
        st = w.state()
        assert np.all(np.isfinite(st[:, :13]))
        max_swing = max(max_swing, axis_angle_between(st, anchor, bob))
    assert max_swing < limit


@pytest.mark.parametrize("precision", PRECISIONS)
def test_cone_twist_motor_drives_to_the_target(precision):  # conetwist.rs:138-187, :351-369
    target = (0.0, 0.0, math.sin(0.15), math.cos(0.15))  # 0.3 rad about Z, in constraint space
    w, anchor, bob = cone_world(precision, (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), gravity=(0.0, 0.0, 0.0),
                                motor=(target, 5.0))
    for _ in range(300):
        w.step(DT)
    assert abs(axis_angle_between(w.state(), anchor, bob) - 0.3) < 0.05


def g6dof_world(precision, box_pos, frames, gravity, setup, linvel=(0, 0, 0), angvel=(0, 0, 0)):
    """constraint/tests.rs:770-930: a 0.3 m box tied to a static 0.2 m anchor by a classic 6DOF."""
    import bgpu
    w = world(precision, gravity)
    anchor = w.add_body(w.add_shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    box = w.add_body(w.add_shape(orc.BOX, [0.3, 0.3, 0.3]), box_pos, linvel=linvel, angvel=angvel, mass=1.0)
    j = bgpu.Generic6Dof(box, anchor, orc.frame(frames[0]), orc.frame(frames[1]))
    setup(j)
    w.add_joint(orc.spring2_joint_desc(j))
    return w, box


@pytest.mark.parametrize("precision", PRECISIONS)
def test_generic_6dof_locked_is_rigid(precision):  # tests.rs:773-817
    w, box = g6dof_world(precision, (0, 1, 0), ((0, 0.5, 0), (0, 1.5, 0)), (0, -9.81, 0),
                         lambda j: j.set_angular_limits((0, 0, 0), (0, 0, 0)), linvel=(2, 0, 0), angvel=(0, 0, 4))
    max_rel = 0.0
    for _ in range(600):
        w.step(DT)
        max_rel = max(max_rel, quat_angle(w.state()[box, 3:7]))
    assert max_rel < 0.5
    assert np.linalg.norm(w.state()[box, 0:3] - (0, 1, 0)) < 0.03


@pytest.mark.parametrize("precision", PRECISIONS)
def test_generic_6dof_angular_limit_stops_the_spin(precision):  # tests.rs:820-855
    w, box = g6dof_world(precision, (0, 0, 0), ((0, 0, 0), (0, 0, 0)), (0, 0, 0),
                         lambda j: j.set_angular_limits((-0.4, -1.0, -1.0), (0.4, 1.0, 1.0)), angvel=(4, 0, 0))
    max_angle = 0.0
    for _ in range(300):
        w.step(DT)
        max_angle = max(max_angle, abs(w.spring2_state(1)[0, 0]))
    assert 0.3 < max_angle < 0.5


@pytest.mark.parametrize("precision", PRECISIONS)
def test_generic_6dof_motor_rotates_an_axis(precision):  # tests.rs:858-890
    w, box = g6dof_world(precision, (0, 0, 0), ((0, 0, 0), (0, 0, 0)), (0, 0, 0),
                         lambda j: j.enable_motor(5, 1.0, 100.0))
    for _ in range(180):
        w.step(DT)
    assert abs(abs(w.spring2_state(1)[0, 2]) - 3.0) < 1.0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_generic_6dof_linear_limit_stops_the_slide(precision):  # tests.rs:893-930
    w, box = g6dof_world(precision, (0.2, 0, 0), ((0, 0, 0), (0, 0, 0)), (0, 0, 0),
                         lambda j: j.set_linear_limits((-0.3, 0, 0), (0.3, 0, 0)), linvel=(4, 0, 0))
    max_x = 0.0
    for _ in range(180):
        w.step(DT)
        max_x = max(max_x, w.state()[box, 0])
    assert max_x < 0.34 and w.state()[box, 0] < 0.3


def test_universal_frames_and_limits():  # generic6dof.rs:560-611
    import bgpu
    j = bgpu.Generic6Dof.universal(0, 1, (0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (0, 0, 0, 1), (1.0, 2.0, 3.0), (0, 0, 1),
                                   (1, 0, 0))
    fa = np.array(j.desc.frame_a)
    assert np.array_equal(fa[3:], [0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0])
    assert np.allclose(fa[:3], (1.0, 2.0, 3.0), atol=1e-6)
    for i in range(3):
        assert (j.axis(i).lower_limit, j.axis(i).upper_limit) == (0.0, 0.0)
    assert (j.axis(3).lower_limit, j.axis(3).upper_limit) == (0.0, 0.0)
    assert abs(j.axis(4).lower_limit - (-math.pi / 2 + 0.01)) < 1e-6 and abs(j.axis(4).upper_limit - (math.pi / 2 - 0.01)) < 1e-6
    assert abs(j.axis(5).lower_limit - (-math.pi + 0.01)) < 1e-6 and abs(j.axis(5).upper_limit - (math.pi - 0.01)) < 1e-6


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("spin, free", [((0.0, 0.0, 5.0), True), ((0.0, 5.0, 0.0), False)])
def test_universal_bends_only_about_the_joint_axes(precision, spin, free):  # generic6dof.rs:614-676
    import bgpu
    w = world(precision, (0, 0, 0))
    s = w.add_shape(orc.SPHERE, [0.3])
    a = w.add_body(s, (0, 0, 0), mass=0.0)
    b = w.add_body(s, (1, 0, 0), angvel=spin, mass=1.0)
    j = bgpu.Generic6Dof.universal(a, b, (0, 0, 0), (0, 0, 0, 1), (1, 0, 0), (0, 0, 0, 1), (1, 0, 0), (0, 0, 1),
                                   (1, 0, 0))
    w.add_joint(orc.spring2_joint_desc(j))
    for _ in range(60):
        w.step(DT)
    st = w.state()[b]
    if free:
        assert st[12] > 4.0
    else:
        assert abs(st[11]) < 0.05


@pytest.mark.parametrize("prec", PRECISIONS)
def test_solver_info_damping_scales_the_joint_row_velocity_term(prec):
    # solver/sequential_impulse.rs:1645-1677: one iteration of a point-to-point joint between a
    # moving and a resting sphere; with the solver damping at its default 1.0 the pair ends
    # closer to a common velocity than at 0.5. (Restated through one world step with gravity
    # off and the joint's pair suppressed, so only the joint rows act.)
    def run(damping):
        w = world(prec, gravity=(0.0, 0.0, 0.0))
        w.set_solver(num_iterations=1, damping=damping)
        s = w.add_shape(orc.SPHERE, [0.5])
        a = w.add_body(s, (-0.5, 0, 0), linvel=(1, 0, 0), mass=1.0)
        b = w.add_body(s, (0.5, 0, 0), mass=1.0)
        p2p(w, a, b, (0.5, 0, 0), (-0.5, 0, 0))
        w.step(DT)
        st = w.state()
        return st[a, 7], st[b, 7]

    va1, vb1 = run(1.0)
    va05, vb05 = run(0.5)
    assert abs(vb1 - va1) < abs(vb05 - va05)
