"""Pins the oracle's fixed-timestep stepping (step.rs:136-199, PhysicsWorld::step_simulation_fixed)
against the reference's own tests of it (world/step.rs, lines cited), in both precisions: one
substep per call equals the plain step bit for bit, the accumulator's substep rhythm, the clamp
with the unclamped demand returned, forces feeding every substep of a call, and a call without a
substep dropping the applied forces.
"""
import numpy as np
import pytest

from oracle_api import OracleWorld

PRECISIONS = ["f32", "f64"]


def ball(prec, mass=1.0, v=(1.0, 0.0, 0.0)):
    w = OracleWorld(prec)
    w.set_gravity((0, 0, 0))
    b = w.add_body(w.sphere(0.5), [-20.0, 0, 0], linvel=v, mass=mass)
    return w, b


@pytest.mark.parametrize("prec", PRECISIONS)
def test_fixed_degenerates_to_single_step(prec):
    # world/step.rs:3296-3332
    def build():
        w = OracleWorld(prec)
        w.set_gravity((0, -10, 0))
        w.add_body(w.box([4.0, 0.5, 4.0]), [0, 0, 0], mass=0)
        w.add_body(w.sphere(0.5), [0.1, 3.0, 0], mass=1.0, restitution=0.3)
        return w

    single, fixed = build(), build()
    dt = 1.0 / 60.0
    for _ in range(120):
        single.step(dt)
        assert fixed.step_fixed(dt, 1, dt) == 1
    a, b = single.state(), fixed.state()
    np.testing.assert_array_equal(a[1, 0:3], b[1, 0:3])
    np.testing.assert_array_equal(a[1, 7:10], b[1, 7:10])


@pytest.mark.parametrize("prec", PRECISIONS)
def test_accumulator_substep_rhythm(prec):
    # world/step.rs:3339-3362
    w, b = ball(prec)
    dt, fixed_dt = 1.0 / 128.0, 3.0 / 128.0
    moved = 0.0
    for frame, want in enumerate([0, 0, 1, 0, 0, 1]):
        n = w.step_fixed(dt, 4, fixed_dt)
        assert n == want, frame
        moved += n * fixed_dt
        assert w.state()[b, 0] == pytest.approx(-20.0 + moved, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_clamped_substeps(prec):
    # world/step.rs:3368-3384
    w, b = ball(prec)
    x0 = w.state()[b, 0]
    assert w.step_fixed(1.0, 2, 1.0 / 128.0) == 128
    assert w.state()[b, 0] - x0 == pytest.approx(2.0 / 128.0, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_forces_persist_across_substeps(prec):
    # world/step.rs:3488-3504
    w, b = ball(prec, mass=2.0, v=(0.0, 0.0, 0.0))
    w.apply_force(b, (12.0, 0.0, 0.0))
    assert w.step_fixed(1.0, 8, 1.0 / 128.0) == 128
    assert w.state()[b, 7] == pytest.approx(12.0 / 2.0 * (8.0 / 128.0), abs=1e-5)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_no_substep_frame_clears_forces(prec):
    # world/step.rs:3448-3482 (its force assertions)
    w, b = ball(prec)
    fixed_dt = 1.0 / 120.0
    assert w.step_fixed(fixed_dt, 4, fixed_dt) == 1
    w.apply_force(b, (10.0, 0.0, 0.0))
    assert w.step_fixed(0.0, 0, fixed_dt) == 0
    coasting = w.state()[b, 7]
    w.step_fixed(fixed_dt, 4, fixed_dt)
    assert w.state()[b, 7] == pytest.approx(coasting, abs=1e-6)
