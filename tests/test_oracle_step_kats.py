"""Pins the CPU oracle's world step against more of the reference's own world tests.

Each test restates the assertions of one test of crates/bullet-dynamics/src/world/step.rs
(line cited): damping, collision group / mask filtering, a simulation-disabled body, and
kinematic bodies. Both precisions are checked, as the reference runs its suite under `f32`
and `--features f64`.
"""
import numpy as np
import pytest

from oracle_api import ACTIVE, DISABLE_DEACTIVATION, DISABLE_SIMULATION, WANTS_DEACTIVATION, OracleWorld

PRECISIONS = ["f32", "f64"]
DT = 1.0 / 60.0
DEFAULT, STATIC, ALL = 1, 2, 0xFFFF  # body.rs:160-170 filter groups


def is_active(state_row):
    # body.rs:524-532
    return int(state_row[13]) in (ACTIVE, WANTS_DEACTIVATION, DISABLE_DEACTIVATION)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_damping_applied_during_step(prec):
    # world/step.rs:1302-1317: linear damping 0.5 for 1 s halves the speed ((1 - 0.5)^t).
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    s = w.sphere(0.5)
    w.add_body(s, [0, 10, 0], linvel=(10, 0, 0), mass=1.0, lin_damping=0.5)
    for _ in range(60):
        w.step(DT)
    assert w.state()[0, 7] == pytest.approx(5.0, abs=1e-4)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_collision_mask_blocks_pair(prec):
    # world/step.rs:1327-1351: a plate whose mask accepts no group is passed straight through.
    w = OracleWorld(prec)
    plate, ball = w.box([2.0, 0.5, 2.0]), w.sphere(0.5)
    w.add_body(plate, [0, 0, 0], mass=0, group=DEFAULT, mask=0)
    b = w.add_body(ball, [0, 3, 0], mass=1.0)
    for _ in range(90):
        w.step(DT)
    assert w.state()[b, 1] < -1.0
    assert len(w.pairs()) == 0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_collision_group_mask_asymmetric(prec):
    # world/step.rs:1357-1391: the group / mask test needs both directions. A STATIC-group plate
    # that accepts every group is still ignored by a ball whose mask accepts DEFAULT only; once
    # the ball's mask widens to ALL and it is put back above the plate (pose only, its fall
    # velocity kept, as set_body_transform does), it lands and rests on the plate.
    w = OracleWorld(prec)
    plate, ball = w.box([2.0, 0.5, 2.0]), w.sphere(0.5)
    w.add_body(plate, [0, 0, 0], mass=0, group=STATIC, mask=ALL)
    b = w.add_body(ball, [0, 1.01, 0], mass=1.0, group=DEFAULT, mask=DEFAULT)
    for _ in range(60):
        w.step(DT)
    assert w.state()[b, 1] < 0.0
    w.set_filter(b, DEFAULT, ALL)
    st = w.state()
    st[b, 0:3] = [0.0, 1.01, 0.0]
    st[b, 3:7] = [0.0, 0.0, 0.0, 1.0]
    w.set_state(st)
    for _ in range(180):
        w.step(DT)
    assert w.state()[b, 1] == pytest.approx(1.0, abs=0.05)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_disable_simulation_body_takes_solver_impulses_without_integrating(prec):
    # world/step.rs:1729-1759: a DISABLE_SIMULATION body is in the solve (its velocity takes
    # the contact impulse) but its pose is never integrated.
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    s = w.sphere(0.5)
    a = w.add_body(s, [0, 0, 0], linvel=(2, 0, 0), mass=1.0, activation=DISABLE_DEACTIVATION)
    b = w.add_body(s, [0.6, 0, 0], mass=1.0, activation=DISABLE_SIMULATION)
    w.step(DT)
    st = w.state()
    assert st[b, 7] > 0.0
    np.testing.assert_array_equal(st[b, 0:3], np.array([0.6, 0.0, 0.0], dtype=np.float32 if prec == "f32"
                                                        else np.float64).astype(np.float64))
    assert st[a, 7] < 2.0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_kinematic_pushes_dynamic_body(prec):
    # world/step.rs:2591-2619: a kinematic slab moving at 2 m/s shoves a resting box along
    # (its velocity enters the contact rows), and the box stays awake.
    w = OracleWorld(prec)
    w.set_gravity((0, -10, 0))
    ground, slab, small = w.plane([0, 1, 0], 0.0), w.box([1.0, 0.5, 1.0]), w.box([0.25, 0.25, 0.25])
    w.add_body(ground, [0, 0, 0], mass=0)
    w.add_body(slab, [-3.0, 0.5, 0.0], linvel=(2, 0, 0), mass=0, kinematic=1)
    t = w.add_body(small, [0.0, 0.75, 0.0], mass=1.0)
    x0 = w.state()[t, 0]
    for _ in range(120):
        w.step(DT)
    st = w.state()
    assert st[t, 0] > x0 + 0.5
    assert is_active(st[t])


@pytest.mark.parametrize("prec", PRECISIONS)
def test_kinematic_ignores_gravity_forces_and_damping(prec):
    # world/step.rs:2624-2650: gravity, damping and applied forces never change a kinematic
    # body's velocities; its pose integrates from them (x ~ v t after 1 s) and it stays active.
    w = OracleWorld(prec)
    w.set_gravity((0, -10, 0))
    s = w.sphere(0.5)
    k = w.add_body(s, [0, 5, 0], linvel=(1, 0, 0), angvel=(0, 0, 1), mass=0, kinematic=1, lin_damping=0.2,
                   ang_damping=0.2)
    for i in range(60):
        w.apply_force(k, (0, 100, 0))
        w.step(DT)
        st = w.state()[k]
        assert st[1] == pytest.approx(5.0, abs=1e-4), i
        assert tuple(st[7:10]) == (1.0, 0.0, 0.0), i
    st = w.state()[k]
    assert st[0] == pytest.approx(1.0, abs=1e-3)
    assert is_active(st)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_dynamic_body_rests_and_sleeps_on_idle_kinematic_platform(prec):
    # world/step.rs:2655-2675: a box settles on a resting kinematic platform and goes to sleep
    # (idle kinematic contacts do not keep it awake); the platform never moves.
    w = OracleWorld(prec)
    w.set_gravity((0, -10, 0))
    plat, cargo = w.box([2.0, 0.25, 2.0]), w.box([0.25, 0.25, 0.25])
    p = w.add_body(plat, [0, 0.25, 0], mass=0, kinematic=1)
    c = w.add_body(cargo, [0, 2.0, 0], mass=1.0)
    for _ in range(480):
        w.step(DT)
    st = w.state()
    assert st[c, 1] == pytest.approx(0.75, abs=0.05)
    assert not is_active(st[c])
    assert tuple(st[p, 0:3]) == (0.0, 0.25, 0.0)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_kinematic_static_and_kinematic_kinematic_pairs_are_inert(prec):
    # world/step.rs:2681-2711: kinematic-kinematic and kinematic-static overlaps produce no
    # solver rows: both kinematic bodies keep their velocities and stay above the ground.
    w = OracleWorld(prec)
    w.set_gravity((0, -10, 0))
    ground, cube = w.plane([0, 1, 0], 0.0), w.box([0.5, 0.5, 0.5])
    w.add_body(ground, [0, 0, 0], mass=0)
    a = w.add_body(cube, [0.0, 0.5, 0.0], linvel=(0.5, 0, 0), mass=0, kinematic=1)
    b = w.add_body(cube, [0.3, 0.5, 0.0], linvel=(-0.5, 0, 0), mass=0, kinematic=1)
    for _ in range(120):
        w.step(DT)
        assert len(w.rows()) == 0
    st = w.state()
    assert tuple(st[a, 7:10]) == (0.5, 0.0, 0.0)
    assert tuple(st[b, 7:10]) == (-0.5, 0.0, 0.0)
    assert st[a, 1] > 0.0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_interpolate_pose_branches(prec):
    # world/step.rs:3622-3684 (body.rs interpolate_pose): pure translation, the small-angle
    # Taylor branch, the pi/4 clamp of a large turn, an exact moderate turn, a negative span.
    import math

    from oracle_api import interpolate_pose

    r = interpolate_pose((1, 2, 3), (0, 0, 0, 1), (10, 0, 0), (0, 0, 0), 0.5, prec)
    assert r[0] == pytest.approx(6.0, abs=1e-6) and r[6] == pytest.approx(1.0, abs=1e-6)
    w = 5e-4
    r = interpolate_pose((0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (w, 0, 0), 1.0, prec)
    assert r[3] == pytest.approx(0.5 * w, abs=1e-6) and abs(r[6] - 1.0) < 1e-4
    half_pi = float(np.float32(math.pi / 2)) if prec == "f32" else math.pi / 2
    r = interpolate_pose((0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (half_pi, 0, 0), 1.0, prec)
    assert r[3] == pytest.approx(0.6379518, abs=1e-5) and r[6] == pytest.approx(0.7700761, abs=1e-5)
    r = interpolate_pose((0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (0.5, 0, 0), 1.0, prec)
    assert r[3] == pytest.approx(math.sin(0.25), abs=1e-5) and r[6] == pytest.approx(math.cos(0.25), abs=1e-5)
    r = interpolate_pose((0, 1, 0), (0, 0, 0, 1), (2, 0, 0), (0, 0, 0), -1.0 / 128.0, prec)
    assert r[0] == pytest.approx(-2.0 / 128.0, abs=1e-6) and r[1] == pytest.approx(1.0, abs=1e-6)
    assert r[6] == pytest.approx(1.0, abs=1e-6)


def _suppression_world(prec, suppress):
    # world/step.rs:1767-1872's scene: a sphere A that never sleeps, a static sphere B 0.75 away,
    # and a disabled point-to-point joint between them whose only effect is the suppression.
    from oracle_api import JF_DISABLE_COLLISIONS, JF_DISABLED, JOINT_POINT2POINT, frame, joint_desc

    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    s = w.sphere(0.5)
    a = w.add_body(s, [0, 0, 0], mass=1.0, activation=DISABLE_DEACTIVATION)
    b = w.add_body(s, [0.75, 0, 0], mass=0)
    flags = JF_DISABLED | (JF_DISABLE_COLLISIONS if suppress else 0)
    j = w.add_joint(joint_desc(JOINT_POINT2POINT, a, b, frame([0, 0, 0]), frame([0, 0, 0]), flags=flags))
    return w, a, j


def _charge_and_run(w, a):
    st = w.state()
    st[a, 0:3] = [0.0, 0.0, 0.0]
    st[a, 7:10] = [3.0, 0.0, 0.0]
    w.set_state(st)
    for _ in range(90):
        w.step(DT)
    return w.state()[a, 0]


@pytest.mark.parametrize("prec", PRECISIONS)
def test_constraint_suppression_flips_take_effect_next_step(prec):
    # world/step.rs:1767-1838: suppression set at build lets A pass through B; cleared between
    # steps, A is stopped; the other way round likewise.
    from oracle_api import JF_DISABLE_COLLISIONS, JF_DISABLED

    w, a, j = _suppression_world(prec, True)
    assert _charge_and_run(w, a) > 1.5
    w.set_joint_flags(j, JF_DISABLED)
    assert _charge_and_run(w, a) < 1.5
    w, a, j = _suppression_world(prec, False)
    assert _charge_and_run(w, a) < 1.5
    w.set_joint_flags(j, JF_DISABLED | JF_DISABLE_COLLISIONS)
    assert _charge_and_run(w, a) > 1.5


@pytest.mark.parametrize("prec", PRECISIONS)
def test_disabled_constraint_still_suppresses_collisions(prec):
    # world/step.rs:1844-1872
    w, a, _ = _suppression_world(prec, True)
    assert _charge_and_run(w, a) > 1.5
