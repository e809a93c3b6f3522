"""Oracle CCD swept-sphere clamp pinned by the reference's own CCD tests.

Each case restates a test of crates/bullet-dynamics/src/world/step.rs (line cited), run through
the oracle's full step in both precisions.
"""
import math

import numpy as np
import pytest

import oracle_api as orc

PRECISIONS = ["f32", "f64"]
DT = 1.0 / 60.0


def world(precision):
    w = orc.OracleWorld(precision)
    w.set_gravity((0.0, 0.0, 0.0))
    return w


def wall_and_ball(precision, wall_pos=(0.0, 0.5, 0.0), ball_pos=(0.0, 1.0, 0.0), v=(0.0, -120.0, 0.0),
                  threshold=0.1, radius=0.3, wall_flags=0, angvel=(0.0, 0.0, 0.0)):
    """A thin static wall (half extents 1, 0.1, 1) and a CCD ball of radius 0.3."""
    w = world(precision)
    wall = w.add_body(w.add_shape(orc.BOX, [1.0, 0.1, 1.0]), wall_pos, mass=0.0, flags=wall_flags)
    ball = w.add_body(w.add_shape(orc.SPHERE, [0.3]), ball_pos, linvel=v, angvel=angvel, mass=1.0)
    w.set_ccd(ball, threshold, radius)
    return w, wall, ball


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_clamps_fast_bodies_at_the_impact(precision):  # :2041-2082
    w = world(precision)
    w.add_body(w.add_shape(orc.BOX, [1.0, 0.1, 1.0]), (0.0, 0.5, 0.0), mass=0.0)
    sph = w.add_shape(orc.SPHERE, [0.3])
    ball = w.add_body(sph, (0.0, 1.0, 0.0), linvel=(0.0, -120.0, 0.0), mass=1.0)
    w.set_ccd(ball, 0.1, 0.3)
    control = w.add_body(sph, (2.0, 1.0, 0.0), linvel=(0.0, -120.0, 0.0), mass=1.0)
    w.step(DT)
    st = w.state()
    assert abs(st[ball, 1] - 0.9) <= 0.05
    assert st[control, 1] < -0.5
    assert w.ccd_clamps()[ball] < 1.0 and w.ccd_clamps()[control] == 1.0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_ignores_slow_motion(precision):  # :2085-2111
    w = world(precision)
    w.add_body(w.add_shape(orc.PLANE, [0.0, 1.0, 0.0, 0.0]), (0.0, 0.0, 0.0), mass=0.0)
    ball = w.add_body(w.add_shape(orc.SPHERE, [0.3]), (0.0, 1.0, 0.0), linvel=(0.0, -5.0, 0.0), mass=1.0)
    w.set_ccd(ball, 1.0, 0.3)
    w.step(DT)
    assert abs(w.state()[ball, 1] - (1.0 - 5.0 / 60.0)) <= 1e-5


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_skips_collision_suppressed_pairs(precision):  # :2116-2149
    w, wall, ball = wall_and_ball(precision)
    w.add_joint(orc.joint_desc(orc.JOINT_POINT2POINT, wall, ball, orc.frame((0.0, 0.5, 0.0)),
                               orc.frame((0.0, -0.5, 0.0)), impulse_clamp=0.001))
    w.step(DT)
    assert w.state()[ball, 1] < -0.5


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_ignores_no_contact_response_targets(precision):  # :2152-2182
    w, _, ball = wall_and_ball(precision, wall_flags=orc.NO_CONTACT_RESPONSE)
    w.step(DT)
    assert w.state()[ball, 1] < -0.5


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_threshold_boundary_is_exclusive(precision):  # :2185-2225
    w, _, ball = wall_and_ball(precision, wall_pos=(0.0, 3.0, 0.0), ball_pos=(0.0, 4.0, 0.0), v=(0.0, -6.0, 0.0),
                               threshold=1.5)
    w.step(0.25)
    assert abs(w.state()[ball, 1] - 2.5) <= 1e-5
    w, _, ball = wall_and_ball(precision, wall_pos=(0.0, 3.0, 0.0), ball_pos=(0.0, 4.0, 0.0), v=(0.0, -6.4, 0.0),
                               threshold=1.5)
    w.step(0.25)
    assert abs(w.state()[ball, 1] - 3.4) <= 0.02


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("near_filter", [(1, 0xFFFF), (2, 0)])
def test_ccd_selects_nearest_of_multiple_targets(precision, near_filter):  # :2228-2269
    w = world(precision)
    plate = w.add_shape(orc.BOX, [0.05, 1.0, 1.0])
    w.add_body(plate, (2.0, 0.0, 0.0), mass=0.0, group=near_filter[0], mask=near_filter[1])
    w.add_body(plate, (6.0, 0.0, 0.0), mass=0.0)
    ball = w.add_body(w.add_shape(orc.SPHERE, [0.3]), (0.0, 0.0, 0.0), linvel=(420.0, 0.0, 0.0), mass=1.0)
    w.set_ccd(ball, 0.1, 0.3)
    w.step(DT)
    x = w.state()[ball, 0]
    if near_filter == (1, 0xFFFF):
        assert 1.5 <= x < 1.8
    else:
        assert 5.5 <= x < 5.8


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("k", [1.0, 10.0, 100.0, 1000.0])
def test_ccd_speed_sweep_stays_finite(precision, k):  # :2272-2302
    w, _, ball = wall_and_ball(precision, wall_pos=(10000.0, 0.5, 0.0), ball_pos=(10000.0, 1.0, 0.0),
                               v=(0.0, -120.0 * k, 0.0))
    w.step(DT)
    st = w.state()[ball]
    assert np.all(np.isfinite(st[:13]))
    assert abs(st[1] - 0.9) <= 0.05
    assert abs(st[0] - 10000.0) <= 1.0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_high_spin_stays_finite(precision):  # :2305-2332
    w, _, ball = wall_and_ball(precision, angvel=(0.0, 3000.0, 0.0))
    w.step(DT)
    st = w.state()[ball]
    assert np.all(np.isfinite(st[:13]))
    assert abs(float(np.dot(st[3:7], st[3:7])) - 1.0) <= 1e-3
    assert abs(st[1] - 0.9) <= 0.05


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_starting_inside_is_finite(precision):  # :2335-2357
    w, _, ball = wall_and_ball(precision, ball_pos=(0.0, 0.5, 0.0))
    w.step(DT)
    st = w.state()[ball]
    assert np.all(np.isfinite(st[:13]))
    assert abs(st[1] - 0.5) <= 1e-4


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_respects_collision_filter(precision):  # :1694-1720
    w = world(precision)
    w.add_body(w.add_shape(orc.BOX, [0.5, 2.0, 0.25]), (0.0, 0.0, 0.0), mass=0.0, group=1, mask=0)
    ball = w.add_body(w.add_shape(orc.SPHERE, [0.3]), (0.0, 0.0, -5.0), linvel=(0.0, 0.0, 10.0), mass=1.0)
    w.set_ccd(ball, 0.1, 0.3)
    for _ in range(60):
        w.step(DT)
    assert w.state()[ball, 2] > 4.0


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("shape", ["box", "capsule", "sphere", "hull"])
def test_ccd_clamps_against_every_convex_target(precision, shape):
    """The swept sphere stops at the inflated surface of each convex target kind (the sweep's
    convex branch, convex_sweep.rs:107-125): top face at y = 0.6 for every target here."""
    w = world(precision)
    if shape == "box":
        s = w.add_shape(orc.BOX, [1.0, 0.1, 1.0])
    elif shape == "capsule":
        s = w.add_shape(orc.CAPSULE, [0.1, 1.0])
    elif shape == "sphere":
        s = w.add_shape(orc.SPHERE, [0.1])
    else:
        s = w.hull([[x, y, z] for x in (-1.0, 1.0) for y in (-0.1, 0.1) for z in (-1.0, 1.0)])
    quat = (0.0, 0.0, math.sin(math.pi / 4), math.cos(math.pi / 4)) if shape == "capsule" else (0.0, 0.0, 0.0, 1.0)
    w.add_body(s, (0.0, 0.5, 0.0), quat=quat, mass=0.0)
    ball = w.add_body(w.add_shape(orc.SPHERE, [0.3]), (0.0, 1.5, 0.0), linvel=(0.0, -180.0, 0.0), mass=1.0)
    w.set_ccd(ball, 0.1, 0.3)
    w.step(DT)
    assert abs(w.state()[ball, 1] - 0.9) <= 0.05


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ccd_extreme_timestep_stays_finite(precision):  # :2360-2391
    # dt = 1e-4 moves the ball 0.012, under the 0.1 threshold: plain integration. dt = 0.5 moves
    # it 60: the sweep clamps it at the wall.
    w, _, ball = wall_and_ball(precision)
    w.step(1e-4)
    st = w.state()[ball]
    assert np.all(np.isfinite(st[:13]))
    assert abs(st[1] - (1.0 - 120.0 * 1e-4)) <= 1e-5
    w, _, ball = wall_and_ball(precision)
    w.step(0.5)
    st = w.state()[ball]
    assert np.all(np.isfinite(st[:13]))
    assert abs(st[1] - 0.9) <= 0.05
