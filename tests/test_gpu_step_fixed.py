"""bgpu_step_simulation_fixed (PhysicsWorld::step_simulation_fixed, world/step.rs:136-199) on the
device, restating the reference's fixed-timestep tests (world/step.rs, lines cited): one substep
per call equals the plain step bit for bit, the accumulator's substep rhythm, the clamp with the
unclamped demand returned, forces feeding every substep of a call, and a call without a substep
dropping the applied forces.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ball(gpu, mass=1.0, v=(1.0, 0.0, 0.0)):
    w = gpu.World(gravity=(0.0, 0.0, 0.0))
    s = w.sphere(0.5)
    w.add_body(s, (-20.0, 0.0, 0.0), linvel=v, mass=mass)
    return w


def test_fixed_degenerates_to_single_step(gpu):
    # world/step.rs:3296-3332
    def build():
        w = gpu.World(gravity=(0.0, -10.0, 0.0))
        ground, ball = w.box([4.0, 0.5, 4.0]), w.sphere(0.5)
        w.add_body(ground, (0, 0, 0), mass=0.0)
        w.add_body(ball, (0.1, 3.0, 0.0), mass=1.0, restitution=0.3)
        return w

    single, fixed = build(), build()
    dt = 1.0 / 60.0
    for _ in range(120):
        single.step(dt)
        assert fixed.step_fixed(dt, 1, dt) == 1
    a, b = single.state(), fixed.state()
    np.testing.assert_array_equal(a[1, 0:3], b[1, 0:3])
    np.testing.assert_array_equal(a[1, 7:10], b[1, 7:10])
    single.close()
    fixed.close()


def test_accumulator_substep_rhythm(gpu):
    # world/step.rs:3339-3362
    w = _ball(gpu)
    dt, fixed_dt = 1.0 / 128.0, 3.0 / 128.0
    moved = 0.0
    for frame, want in enumerate([0, 0, 1, 0, 0, 1]):
        n = w.step_fixed(dt, 4, fixed_dt)
        assert n == want, frame
        moved += n * fixed_dt
        assert w.state()[0, 0] == pytest.approx(-20.0 + moved, abs=1e-6)
    w.close()


def test_clamped_substeps(gpu):
    # world/step.rs:3368-3384: the demand (128) is returned unclamped; two substeps run.
    w = _ball(gpu)
    x0 = w.state()[0, 0]
    assert w.step_fixed(1.0, 2, 1.0 / 128.0) == 128
    assert w.state()[0, 0] - x0 == pytest.approx(2.0 / 128.0, abs=1e-6)
    w.close()


def test_forces_persist_across_substeps(gpu):
    # world/step.rs:3488-3504: a force applied before the call acts in each of its 8 substeps.
    w = _ball(gpu, mass=2.0, v=(0.0, 0.0, 0.0))
    w.apply_forces(np.array([[12.0, 0.0, 0.0]], np.float32))
    assert w.step_fixed(1.0, 8, 1.0 / 128.0) == 128
    assert w.state()[0, 7] == pytest.approx(12.0 / 2.0 * (8.0 / 128.0), abs=1e-5)
    w.close()


def test_no_substep_frame_clears_forces(gpu):
    # world/step.rs:3448-3482 (its force assertions): a zero-length frame runs no substep and
    # drops the applied force, so the next substep keeps the coasting velocity.
    w = _ball(gpu)
    fixed_dt = 1.0 / 120.0
    assert w.step_fixed(fixed_dt, 4, fixed_dt) == 1
    w.apply_forces(np.array([[10.0, 0.0, 0.0]], np.float32))
    assert w.step_fixed(0.0, 0, fixed_dt) == 0
    coasting = w.state()[0, 7]
    w.step_fixed(fixed_dt, 4, fixed_dt)
    assert w.state()[0, 7] == pytest.approx(coasting, abs=1e-6)
    w.close()
