"""The device step on the scenes of the reference's world tests that the oracle restates in
tests/test_oracle_step_kats.py (world/step.rs: damping, a mask that blocks a pair, a
simulation-disabled body, kinematic bodies). The device world and the oracle take the same
bodies; before every step the oracle takes the device state and after it the device's solve
order, and the states must then agree to 1e-5 relative, activation states and pairs exactly.
The reference's own end assertions are checked on the device trajectory as well.
"""
import numpy as np
import pytest

import oracle_api as orc

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
DEFAULT = 1


def _pairs(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def _lockstep(w, o, steps, forces=None):
    """Steps both worlds `steps` times; forces: {body: (fx, fy, fz)} applied before every step."""
    n = o.num_bodies
    for step in range(steps):
        o.set_state(w.state().astype(np.float64))
        if forces:
            f = np.zeros((n, 3), np.float32)
            for i, v in forces.items():
                f[i] = v
                o.apply_force(i, v)
            w.apply_forces(f)
        w.step(DT)
        o.set_solve_order(w.solve_order())
        o.step(DT)
        st = w.stats()
        assert st["device_status"] == 0, st
        g, r = w.state(), o.state()
        np.testing.assert_array_equal(g[:, 13], r[:, 13], err_msg=f"step {step}")
        np.testing.assert_allclose(g[:, :13], r[:, :13], rtol=1e-5, atol=1e-6, err_msg=f"step {step}")
        np.testing.assert_array_equal(_pairs(w.pairs()), _pairs(o.pairs()))
    return w.state()


def _both(gravity):
    import bgpu

    w = bgpu.World(gravity=gravity)
    o = orc.OracleWorld("f32")
    o.set_gravity(gravity)
    return w, o


def test_damping_applied_during_step(gpu):
    # world/step.rs:1302-1317
    w, o = _both((0.0, 0.0, 0.0))
    for x in (w, o):
        s = x.sphere(0.5)
        x.add_body(s, (0, 10, 0), linvel=(10, 0, 0), mass=1.0, lin_damping=0.5)
    st = _lockstep(w, o, 60)
    assert st[0, 7] == pytest.approx(5.0, abs=1e-4)


def test_collision_mask_blocks_pair(gpu):
    # world/step.rs:1327-1351
    w, o = _both((0.0, -9.81, 0.0))
    for x in (w, o):
        plate, ball = x.box([2.0, 0.5, 2.0]), x.sphere(0.5)
        x.add_body(plate, (0, 0, 0), mass=0, group=DEFAULT, mask=0)
        x.add_body(ball, (0, 3, 0), mass=1.0)
    st = _lockstep(w, o, 90)
    assert st[1, 1] < -1.0


def test_disable_simulation_body_takes_solver_impulses_without_integrating(gpu):
    # world/step.rs:1729-1759
    w, o = _both((0.0, 0.0, 0.0))
    for x in (w, o):
        s = x.sphere(0.5)
        x.add_body(s, (0, 0, 0), linvel=(2, 0, 0), mass=1.0, activation=orc.DISABLE_DEACTIVATION)
        x.add_body(s, (0.6, 0, 0), mass=1.0, activation=orc.DISABLE_SIMULATION)
    st = _lockstep(w, o, 1)
    assert st[1, 7] > 0.0
    np.testing.assert_array_equal(st[1, 0:3], np.float32([0.6, 0.0, 0.0]))


def test_kinematic_pushes_dynamic_body(gpu):
    # world/step.rs:2591-2619
    w, o = _both((0.0, -10.0, 0.0))
    for x in (w, o):
        ground, slab, small = x.plane([0, 1, 0], 0.0), x.box([1.0, 0.5, 1.0]), x.box([0.25, 0.25, 0.25])
        x.add_body(ground, (0, 0, 0), mass=0)
        x.add_body(slab, (-3.0, 0.5, 0.0), linvel=(2, 0, 0), mass=0, kinematic=1)
        x.add_body(small, (0.0, 0.75, 0.0), mass=1.0)
    st = _lockstep(w, o, 120)
    assert st[2, 0] > 0.5
    assert int(st[2, 13]) in (orc.ACTIVE, orc.WANTS_DEACTIVATION, orc.DISABLE_DEACTIVATION)


def test_kinematic_ignores_gravity_forces_and_damping(gpu):
    # world/step.rs:2624-2650
    w, o = _both((0.0, -10.0, 0.0))
    for x in (w, o):
        s = x.sphere(0.5)
        x.add_body(s, (0, 5, 0), linvel=(1, 0, 0), angvel=(0, 0, 1), mass=0, kinematic=1, lin_damping=0.2,
                   ang_damping=0.2)
    st = _lockstep(w, o, 60, forces={0: (0.0, 100.0, 0.0)})
    assert st[0, 1] == pytest.approx(5.0, abs=1e-4)
    assert tuple(st[0, 7:10]) == (1.0, 0.0, 0.0)
    assert st[0, 0] == pytest.approx(1.0, abs=1e-3)


def test_dynamic_body_rests_and_sleeps_on_idle_kinematic_platform(gpu):
    # world/step.rs:2655-2675
    w, o = _both((0.0, -10.0, 0.0))
    for x in (w, o):
        plat, cargo = x.box([2.0, 0.25, 2.0]), x.box([0.25, 0.25, 0.25])
        x.add_body(plat, (0, 0.25, 0), mass=0, kinematic=1)
        x.add_body(cargo, (0, 2.0, 0), mass=1.0)
    st = _lockstep(w, o, 480)
    assert st[1, 1] == pytest.approx(0.75, abs=0.05)
    assert int(st[1, 13]) == orc.ISLAND_SLEEPING
    assert tuple(st[0, 0:3]) == (0.0, 0.25, 0.0)


def test_kinematic_static_and_kinematic_kinematic_pairs_are_inert(gpu):
    # world/step.rs:2681-2711
    w, o = _both((0.0, -10.0, 0.0))
    for x in (w, o):
        ground, cube = x.plane([0, 1, 0], 0.0), x.box([0.5, 0.5, 0.5])
        x.add_body(ground, (0, 0, 0), mass=0)
        x.add_body(cube, (0.0, 0.5, 0.0), linvel=(0.5, 0, 0), mass=0, kinematic=1)
        x.add_body(cube, (0.3, 0.5, 0.0), linvel=(-0.5, 0, 0), mass=0, kinematic=1)
    st = _lockstep(w, o, 120)
    assert tuple(st[1, 7:10]) == (0.5, 0.0, 0.0)
    assert tuple(st[2, 7:10]) == (-0.5, 0.0, 0.0)
    assert st[1, 1] > 0.0


def test_additional_damping_shrinks_low_speeds(gpu):
    # body.rs:1347-1400 (additional damping): the scale block below the thresholds and the
    # 0.005 subtraction under the damping factors, in lockstep with the oracle.
    w, o = _both((0.0, 0.0, 0.0))
    for x in (w, o):
        s = x.sphere(0.5)
        x.add_body(s, (0, 0, 0), linvel=(0.05, 0, 0), angvel=(0, 0.02, 0), mass=1.0, flags=orc.ADDITIONAL_DAMPING)
        x.add_body(s, (5, 0, 0), linvel=(0.04, 0, 0), angvel=(0, 0, 0.15), mass=1.0, flags=orc.ADDITIONAL_DAMPING,
                   lin_damping=0.2, ang_damping=0.2)
    st = _lockstep(w, o, 10)
    assert st[0, 7] < 0.05 * 0.005 + 1e-9


def test_constraint_suppression_flips_take_effect_next_step(gpu):
    # world/step.rs:1767-1838: suppression of a disabled joint's pair set at build and flipped
    # between steps (bgpu_set_joint_flags), in lockstep with the oracle.
    for suppress in (True, False):
        w, o = _both((0.0, 0.0, 0.0))
        flags = orc.JF_DISABLED | (orc.JF_DISABLE_COLLISIONS if suppress else 0)
        s = w.sphere(0.5)
        w.add_body(s, (0, 0, 0), mass=1.0, activation=orc.DISABLE_DEACTIVATION)
        w.add_body(s, (0.75, 0, 0), mass=0.0)
        w.add_joint(orc.JOINT_POINT2POINT, 0, 1, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)), flags=flags)
        so = o.sphere(0.5)
        o.add_body(so, (0, 0, 0), mass=1.0, activation=orc.DISABLE_DEACTIVATION)
        o.add_body(so, (0.75, 0, 0), mass=0.0)
        o.add_joint(orc.joint_desc(orc.JOINT_POINT2POINT, 0, 1, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)),
                                   flags=flags))
        for flip in (False, True):
            if flip:
                flags ^= orc.JF_DISABLE_COLLISIONS
                w.set_joint_flags(0, flags)
                o.set_joint_flags(0, flags)
            st = w.state()
            st[0, 0:3] = (0.0, 0.0, 0.0)
            st[0, 7:10] = (3.0, 0.0, 0.0)
            w.set_state(st)
            x = _lockstep(w, o, 90)[0, 0]
            assert (x > 1.5) == bool(flags & orc.JF_DISABLE_COLLISIONS), (suppress, flip, x)
