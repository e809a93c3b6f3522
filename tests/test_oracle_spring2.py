"""Oracle spring-2 joints pinned by the reference's own Generic6DofSpring2 tests.

Each case restates the scene and the assertions of a test in
crates/bullet-dynamics/src/constraint/generic6dof_spring2.rs (the line of each test is
cited), run through the oracle's full step in both precisions. The joint parameters are
built with the product's host-side mirror of the reference setters (bgpu.Spring2, pure
host code), so the same descriptors drive the GPU parity tests.
"""
import math

import numpy as np
import pytest

import bgpu
import oracle_api as orc

DT = 1.0 / 60.0
PRECISIONS = ["f32", "f64"]
ORDERS = [bgpu.ROTATE_XYZ, bgpu.ROTATE_XZY, bgpu.ROTATE_YXZ, bgpu.ROTATE_YZX, bgpu.ROTATE_ZXY, bgpu.ROTATE_ZYX]


def quat_axis(axis, a):
    s = math.sin(a / 2)
    v = [0.0, 0.0, 0.0]
    v[axis] = s
    return (v[0], v[1], v[2], math.cos(a / 2))


def rotate(q, v):
    x, y, z, w = q
    b = np.array([x, y, z])
    v = np.asarray(v, dtype=np.float64)
    return v * (w * w - b @ b) + b * (2 * (v @ b)) + np.cross(b, v) * (2 * w)


def rot_matrix(q):
    return np.stack([rotate(q, e) for e in np.eye(3)], axis=1)


def spring2_world(precision, order=bgpu.ROTATE_XYZ, b_quat=(0.0, 0.0, 0.0, 1.0), setup=None):
    """generic6dof_spring2.rs:1590-1630: two 1 kg spheres (r 0.5) at x = -1 and +1, gravity off,
    never sleeping, joined at the origin; B pre-rotated by b_quat with its pivot counter-rotated."""
    w = orc.OracleWorld(precision)
    w.set_gravity((0.0, 0.0, 0.0))
    s = w.add_shape(orc.SPHERE, [0.5])
    a = w.add_body(s, (-1.0, 0.0, 0.0), mass=1.0, activation=orc.DISABLE_DEACTIVATION)
    b = w.add_body(s, (1.0, 0.0, 0.0), quat=b_quat, mass=1.0, activation=orc.DISABLE_DEACTIVATION)
    inv = (-b_quat[0], -b_quat[1], -b_quat[2], b_quat[3])
    j = bgpu.Spring2(a, b, orc.frame((1.0, 0.0, 0.0)), orc.frame(rotate(inv, (-1.0, 0.0, 0.0))), rotate_order=order)
    if setup:
        setup(j)
    w.add_joint(orc.spring2_joint_desc(j))
    return w, a, b


def angle(w, axis):
    return w.spring2_state(1)[0, axis]


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("order", ORDERS)
def test_euler_identity_is_zero_for_all_orders(precision, order):  # :1458-1478
    euler, axes = orc.spring2_angle_info(np.eye(3), np.eye(3), order, precision)
    assert np.all(np.abs(euler) < 1e-6)
    assert np.all(np.abs(np.linalg.norm(axes, axis=1) - 1.0) < 1e-5)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_euler_sign_pins_for_xyz_and_xzy(precision):  # :1481-1495
    theta = 0.4
    euler, _ = orc.spring2_angle_info(np.eye(3), rot_matrix(quat_axis(1, theta)), bgpu.ROTATE_XYZ, precision)
    assert abs(euler[0]) < 1e-5 and abs(euler[2]) < 1e-5
    assert abs(euler[1] + theta) < 1e-5
    euler, _ = orc.spring2_angle_info(np.eye(3), rot_matrix(quat_axis(0, theta)), bgpu.ROTATE_XZY, precision)
    assert abs(euler[1]) < 1e-5 and abs(euler[2]) < 1e-5
    assert abs(euler[0] + theta) < 1e-5


@pytest.mark.parametrize("precision", PRECISIONS)
def test_gimbal_fallback_feeds_the_state(precision):  # :1498-1506
    m = rot_matrix(quat_axis(1, math.pi / 2))
    if precision == "f32":
        m = m.astype(np.float32).astype(np.float64)
    euler, _ = orc.spring2_angle_info(np.eye(3), m, bgpu.ROTATE_XYZ, precision)
    assert abs(euler[1] + math.pi / 2) < 1e-3


@pytest.mark.parametrize("precision", PRECISIONS)
def test_default_joint_is_a_ball_joint(precision):  # :1644-1664
    w, a, b = spring2_world(precision)
    st = w.state()
    st[b, 7:10] = (0.0, 2.0, 0.0)
    st[b, 10:13] = (0.0, 0.0, 3.0)
    w.set_state(st)
    for _ in range(120):
        w.step(DT)
    st = w.state()
    pivot_a = st[a, 0:3] + rotate(st[a, 3:7], (1.0, 0.0, 0.0))
    pivot_b = st[b, 0:3] + rotate(st[b, 3:7], (-1.0, 0.0, 0.0))
    assert np.linalg.norm(pivot_b - pivot_a) < 0.01
    assert st[b, 6] < 0.999


@pytest.mark.parametrize("precision", PRECISIONS)
def test_limited_axis_is_free_inside_and_restores_outside(precision):  # :1668-1706
    w, _, _ = spring2_world(precision, b_quat=quat_axis(0, 0.2), setup=lambda j: j.set_limit(3, -1.0, 1.0))
    for _ in range(120):
        w.step(DT)
    assert abs(angle(w, 0) + 0.2) < 0.02
    w, _, _ = spring2_world(precision, b_quat=quat_axis(0, 1.5), setup=lambda j: j.set_limit(3, -1.0, 1.0))
    for _ in range(60):
        w.step(DT)
    assert angle(w, 0) > -1.3


@pytest.mark.parametrize("precision", PRECISIONS)
def test_locked_axis_pulls_to_the_lock_angle(precision):  # :1709-1727
    w, _, _ = spring2_world(precision, b_quat=quat_axis(0, -0.5), setup=lambda j: j.set_limit(3, 0.3, 0.3))
    for _ in range(180):
        w.step(DT)
    assert abs(angle(w, 0) - 0.3) < 0.02


def _spring_y(stiffness, damping=None):
    def setup(j):
        j.enable_spring(4, True)
        j.set_stiffness(4, stiffness, True)
        if damping is not None:
            j.set_damping(4, damping, True)
    return setup


@pytest.mark.parametrize("precision", PRECISIONS)
def test_angular_spring_oscillates_and_decays(precision):  # :1730-1770
    w, _, _ = spring2_world(precision, b_quat=quat_axis(1, 0.3), setup=_spring_y(40.0, 0.5))
    prev = angle(w, 1)
    max_angle, crossings = abs(prev), 0
    for _ in range(300):
        w.step(DT)
        a = angle(w, 1)
        if math.copysign(1.0, prev) != math.copysign(1.0, a):
            crossings += 1
        max_angle = max(max_angle, abs(a))
        prev = a
    assert crossings >= 2
    assert max_angle < 0.35


@pytest.mark.parametrize("precision", PRECISIONS)
def test_stiffness_clamp_keeps_a_huge_spring_stable(precision):  # :1773-1795
    w, _, _ = spring2_world(precision, b_quat=quat_axis(1, 0.3), setup=_spring_y(1.0e6))
    max_angle = 0.35
    for _ in range(240):
        w.step(DT)
        a = angle(w, 1)
        assert math.isfinite(a)
        max_angle = max(max_angle, abs(a))
    assert max_angle < 0.6


@pytest.mark.parametrize("precision", PRECISIONS)
def test_damping_clamp_overdamps_without_overshoot(precision):  # :1798-1822
    w, _, _ = spring2_world(precision, b_quat=quat_axis(1, 0.3), setup=_spring_y(40.0, 100.0))
    crossed = False
    for _ in range(300):
        w.step(DT)
        a = angle(w, 1)
        assert math.isfinite(a)
        crossed |= a > 0.0
    assert not crossed


@pytest.mark.parametrize("precision", PRECISIONS)
def test_linear_spring_pulls_to_the_equilibrium(precision):  # :1825-1847
    def setup(j):
        j.set_linear_limits((1.0, 1.0, 1.0), (-1.0, -1.0, -1.0))
        j.enable_spring(0, True)
        j.set_stiffness(0, 5.0, True)
        j.set_damping(0, 0.5, True)
        j.set_equilibrium_point(0, 0.5)
    w, _, _ = spring2_world(precision, setup=setup)
    for _ in range(360):
        w.step(DT)
    assert abs(w.spring2_state(1)[0, 3] - 0.5) < 0.05


@pytest.mark.parametrize("precision", PRECISIONS)
def test_servo_drives_to_the_target(precision):  # :1850-1871
    def setup(j):
        j.enable_motor(3, True)
        j.set_servo(3, True)
        j.set_servo_target(3, 0.5)
        j.set_target_velocity(3, 2.0)
        j.set_max_motor_force(3, 10.0)
    w, _, _ = spring2_world(precision, setup=setup)
    for _ in range(300):
        w.step(DT)
    assert abs(angle(w, 0) - 0.5) < 0.05


@pytest.mark.parametrize("precision", PRECISIONS)
def test_global_erp_fallback(precision):  # :1874-1903
    """An axis without its override flag takes the solver's ERP; a set_stop_erp override keeps its
    own. Restated on the rows: the lower-side limit row's bias is inv_dt * stop_erp * error."""
    def limit_row_bias(axis, override):
        def setup(j):
            j.set_limit(axis, -1.0, 1.0)
            if override is not None:
                j.set_stop_erp(axis, override)
        w, _, _ = spring2_world(precision, b_quat=quat_axis(axis - 3, 1.5), setup=setup)
        w.set_solver(erp=0.5)
        w.step(DT)
        rows = w.joint_rows()
        err = w.spring2_state(1)[0, axis - 3] + 1.0  # position - lower
        return rows[0, 4], err
    bias, err = limit_row_bias(3, 0.3)
    assert abs(bias - (1.0 / DT) * 0.3 * err) < 1e-3 * abs(bias) + 1e-4
    bias, err = limit_row_bias(4, None)
    assert abs(bias - (1.0 / DT) * 0.5 * err) < 1e-3 * abs(bias) + 1e-4


@pytest.mark.parametrize("precision", PRECISIONS)
def test_static_body_mass_split(precision):  # :1906-1945
    w = orc.OracleWorld(precision)
    w.set_gravity((0.0, 0.0, 0.0))
    s = w.add_shape(orc.SPHERE, [0.5])
    a = w.add_body(s, (0.0, 0.0, 0.0), mass=0.0)
    b = w.add_body(s, (1.0, 0.0, 0.0), mass=1.0)
    j = bgpu.Spring2(a, b, orc.frame((0.0, 0.0, 0.0)), orc.frame((1.0, 0.0, 0.0)))
    j.set_limit(4, 0.5, 1.0)
    j.set_limit(5, -1.0, -0.5)
    w.add_joint(orc.spring2_joint_desc(j))
    w.step(DT)
    st = w.spring2_state(1)[0]
    assert st[7] == 1.0
    assert abs(st[6] - 1.0) < 1e-6
    assert abs((1.0 - st[6]) - 0.0) < 1e-6


def hinge2_world(precision, gravity, wheel_radius, wheel_pos, angvel=None):
    w = orc.OracleWorld(precision)
    w.set_gravity(gravity)
    chassis = w.add_body(w.add_shape(orc.SPHERE, [0.5]), (0.0, 0.0, 0.0), mass=0.0)
    wheel = w.add_body(w.add_shape(orc.SPHERE, [wheel_radius]), wheel_pos, mass=1.0,
                       angvel=angvel if angvel is not None else (0.0, 0.0, 0.0))
    j = bgpu.Spring2.hinge2(chassis, wheel, (0, 0, 0), (0, 0, 0, 1), wheel_pos, (0, 0, 0, 1), (0, 0, 0), (0, 0, 1),
                            (1, 0, 0))
    w.add_joint(orc.spring2_joint_desc(j))
    return w, wheel


@pytest.mark.parametrize("precision", PRECISIONS)
def test_hinge2_suspension_holds_the_wheel(precision):  # :2027-2058
    w, wheel = hinge2_world(precision, (0.0, 0.0, -9.8), 0.2, (0.0, 0.0, -0.3))
    for _ in range(240):
        w.step(DT)
    st = w.state()[wheel]
    assert -0.45 < st[2] < -0.10
    assert abs(st[9]) < 1.0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_hinge2_axle_spin_is_free(precision):  # :2061-2084
    w, wheel = hinge2_world(precision, (0.0, 0.0, 0.0), 0.2, (0.0, 0.0, 0.0), angvel=(8.0, 0.0, 0.0))
    for _ in range(60):
        w.step(DT)
    st = w.state()[wheel]
    assert st[10] > 7.5
    assert abs(st[2]) < 1e-4


@pytest.mark.parametrize("precision", PRECISIONS)
def test_hinge2_steering_limit_clamps(precision):  # :2087-2111
    w, wheel = hinge2_world(precision, (0.0, 0.0, 0.0), 0.15, (0.9, 0.0, 0.0), angvel=(0.0, 0.0, 6.0))
    limit = math.pi / 4
    for _ in range(120):
        w.step(DT)
        assert abs(w.spring2_state(1)[0, 2]) < limit + 0.15
