"""Drift of the f32 device trajectory against the oracle's f64 build.

The reference's parity harness compares trajectories by position distance and
double-cover-aware orientation angle, with 1e-2 m / 1e-2 rad tolerances
(tools/compare.py:43-47, docs/parity-harness.md "Tolerance"). The device runs
in f32; the f64 oracle is the reference's `--features f64` build restated.
The first 30 steps of the 1,000-box stack are free fall plus first contacts:
there the drift is f32 rounding alone and is pinned tightly.
"""
import numpy as np
import pytest

import drift_f64
import oracle_api as orc


def test_quat_angle_double_cover():
    q = np.array([[0.0, 0.0, 0.0, 1.0]])
    assert drift_f64.quat_angle(q, -q)[0] == 0.0
    h = np.array([[0.0, np.sin(0.05), 0.0, np.cos(0.05)]])
    assert drift_f64.quat_angle(q, h)[0] == pytest.approx(0.1, rel=1e-9)
    assert drift_f64.quat_angle(h, q)[0] == pytest.approx(0.1, rel=1e-9)
    rng = np.random.default_rng(3)
    a = rng.normal(size=(50, 4))
    b = rng.normal(size=(50, 4))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    ref = 2.0 * np.arccos(np.minimum(1.0, np.abs(np.sum(a * b, axis=1))))  # tools/compare.py's form
    np.testing.assert_allclose(drift_f64.quat_angle(a, b), ref, atol=1e-9)
    # an f32-rounded copy of the same rotation: no acos floor
    assert drift_f64.quat_angle(a, a.astype(np.float32)).max() < 1e-6
    assert drift_f64.first_over([0.0, 0.005, 0.02, 0.0], 1e-2) == 3
    assert drift_f64.first_over([0.0, 0.005], 1e-2) is None


def test_oracle_f32_against_f64_free_fall():
    """The oracle's two builds on a lone falling box: f32 rounding alone before contact."""
    import scenes

    s = scenes.Scene("one_box", 1 / 60, 10, 30)
    p = s.add_shape(scenes.PLANE, [0, 1, 0, 0])
    b = s.add_shape(scenes.BOX, [0.5, 0.5, 0.5])
    s.add(p, (0, 0, 0), mass=0.0)
    s.add(b, (0.0, 10.0, 0.0), mass=1.0)
    a, d = s.build_oracle(orc, "f32"), s.build_oracle(orc, "f64")
    for _ in range(30):
        a.step(s.dt)
        d.step(s.dt)
    assert abs(a.state()[1, 1] - d.state()[1, 1]) < 1e-5


@pytest.mark.gpu
def test_drift_f64_first_30_steps_of_the_box_stack(gpu):
    import scenes

    s = scenes.falling_box_stack(10, 10, 10, seed=1, steps=30)
    d = drift_f64.drift_run(gpu, orc, s, 30)
    assert d["device_status"] == 0
    # f32 rounding of the free fall: |y| <= ~13 m, ulp 1e-6, 30 steps
    assert d["max_pos"].max() < 1e-4, d["max_pos"]
    assert d["max_ang"].max() < 1e-4, d["max_ang"]
