"""GPU CCD swept-sphere clamp against the oracle.

Every scene is built on the GPU and in the oracle (f32) through the same calls; before each
compared step the oracle takes the GPU's body state and afterwards the GPU's contact solve
order, so each step is checked on its own: the per-body clamp fractions and the states must
agree. The scenes restate the reference's CCD tests (crates/bullet-dynamics/src/world/step.rs,
line cited), whose own assertions are also checked on the GPU trajectory, plus a many-body rain
of fast CCD spheres onto thin plates.
"""
import math

import numpy as np
import pytest

import oracle_api as orc

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


class Twin:
    def __init__(self, gpu, gravity=(0.0, 0.0, 0.0)):
        self.g = gpu.World(gravity=gravity, num_iterations=10)
        self.o = orc.OracleWorld("f32")
        self.o.set_gravity(gravity)
        self.o.set_solver(num_iterations=10)

    def shape(self, kind, params):
        a, b = self.g.add_shape(kind, params), self.o.add_shape(kind, params)
        assert a == b
        return a

    def hull(self, pts):
        a, b = self.g.hull(pts), self.o.hull(pts)
        assert a == b
        return a

    def body(self, shape, pos, **kw):
        a, b = self.g.add_body(shape, pos, **kw), self.o.add_body(shape, pos, **kw)
        assert a == b
        return a

    def ccd(self, i, threshold, radius):
        self.g.set_ccd(i, threshold, radius)
        self.o.set_ccd(i, threshold, radius)

    def p2p(self, a, b, pivot_a, pivot_b, **kw):
        self.g.add_joint(orc.JOINT_POINT2POINT, a, b, orc.frame(pivot_a), orc.frame(pivot_b), **kw)
        self.o.add_joint(orc.joint_desc(orc.JOINT_POINT2POINT, a, b, orc.frame(pivot_a), orc.frame(pivot_b), **kw))
        self.o.set_joint_order(self.g.joint_order())

    def step(self, dt=DT, tol=1e-4):
        self.o.set_state(self.g.state().astype(np.float64))
        self.g.step(dt)
        self.o.set_solve_order(self.g.solve_order())
        self.o.step(dt)
        assert self.g.stats()["device_status"] == 0
        gc, oc = self.g.ccd_clamps(), self.o.ccd_clamps()
        np.testing.assert_allclose(gc, oc, atol=1e-5, rtol=0, err_msg="clamp fractions")
        g, r = self.g.state(), self.o.state()
        np.testing.assert_array_equal(g[:, 13], r[:, 13])
        err = float(np.abs(g[:, :13] - r[:, :13]).max())
        assert err <= tol * max(1.0, float(np.abs(r[:, :3]).max()) / 100.0), f"max abs state error {err}"
        return g


def wall_and_ball(gpu, wall_pos=(0.0, 0.5, 0.0), ball_pos=(0.0, 1.0, 0.0), v=(0.0, -120.0, 0.0), threshold=0.1,
                  wall_flags=0, angvel=(0.0, 0.0, 0.0)):
    t = Twin(gpu)
    wall = t.body(t.shape(orc.BOX, [1.0, 0.1, 1.0]), wall_pos, mass=0.0, flags=wall_flags)
    ball = t.body(t.shape(orc.SPHERE, [0.3]), ball_pos, linvel=v, angvel=angvel, mass=1.0)
    t.ccd(ball, threshold, 0.3)
    return t, wall, ball


def test_ccd_clamps_fast_bodies_at_the_impact(gpu):  # step.rs:2041-2082
    t = Twin(gpu)
    t.body(t.shape(orc.BOX, [1.0, 0.1, 1.0]), (0.0, 0.5, 0.0), mass=0.0)
    sph = t.shape(orc.SPHERE, [0.3])
    ball = t.body(sph, (0.0, 1.0, 0.0), linvel=(0.0, -120.0, 0.0), mass=1.0)
    t.ccd(ball, 0.1, 0.3)
    control = t.body(sph, (2.0, 1.0, 0.0), linvel=(0.0, -120.0, 0.0), mass=1.0)
    st = t.step()
    assert abs(st[ball, 1] - 0.9) <= 0.05 and st[control, 1] < -0.5
    assert t.g.ccd_clamps()[ball] < 1.0


def test_ccd_ignores_slow_motion(gpu):  # :2085-2111
    t = Twin(gpu)
    t.body(t.shape(orc.PLANE, [0.0, 1.0, 0.0, 0.0]), (0.0, 0.0, 0.0), mass=0.0)
    ball = t.body(t.shape(orc.SPHERE, [0.3]), (0.0, 1.0, 0.0), linvel=(0.0, -5.0, 0.0), mass=1.0)
    t.ccd(ball, 1.0, 0.3)
    st = t.step()
    assert abs(st[ball, 1] - (1.0 - 5.0 / 60.0)) <= 1e-5


def test_ccd_skips_collision_suppressed_pairs(gpu):  # :2116-2149
    t, wall, ball = wall_and_ball(gpu)
    t.p2p(wall, ball, (0.0, 0.5, 0.0), (0.0, -0.5, 0.0), impulse_clamp=0.001)
    assert t.step()[ball, 1] < -0.5


def test_ccd_ignores_no_contact_response_targets(gpu):  # :2152-2182
    t, _, ball = wall_and_ball(gpu, wall_flags=orc.NO_CONTACT_RESPONSE)
    assert t.step()[ball, 1] < -0.5


@pytest.mark.parametrize("v, expect, tol", [(-6.0, 2.5, 1e-5), (-6.4, 3.4, 0.02)])
def test_ccd_threshold_boundary_is_exclusive(gpu, v, expect, tol):  # :2185-2225
    t, _, ball = wall_and_ball(gpu, wall_pos=(0.0, 3.0, 0.0), ball_pos=(0.0, 4.0, 0.0), v=(0.0, v, 0.0), threshold=1.5)
    assert abs(t.step(0.25)[ball, 1] - expect) <= tol


@pytest.mark.parametrize("near_filter, lo, hi", [((1, 0xFFFF), 1.5, 1.8), ((2, 0), 5.5, 5.8)])
def test_ccd_selects_nearest_of_multiple_targets(gpu, near_filter, lo, hi):  # :2228-2269
    t = Twin(gpu)
    plate = t.shape(orc.BOX, [0.05, 1.0, 1.0])
    t.body(plate, (2.0, 0.0, 0.0), mass=0.0, group=near_filter[0], mask=near_filter[1])
    t.body(plate, (6.0, 0.0, 0.0), mass=0.0)
    ball = t.body(t.shape(orc.SPHERE, [0.3]), (0.0, 0.0, 0.0), linvel=(420.0, 0.0, 0.0), mass=1.0)
    t.ccd(ball, 0.1, 0.3)
    assert lo <= t.step()[ball, 0] < hi


@pytest.mark.parametrize("k", [1.0, 10.0, 100.0, 1000.0])
def test_ccd_speed_sweep_stays_finite(gpu, k):  # :2272-2302
    t, _, ball = wall_and_ball(gpu, wall_pos=(10000.0, 0.5, 0.0), ball_pos=(10000.0, 1.0, 0.0),
                               v=(0.0, -120.0 * k, 0.0))
    st = t.step()[ball]
    assert np.all(np.isfinite(st[:13])) and abs(st[1] - 0.9) <= 0.05 and abs(st[0] - 10000.0) <= 1.0


def test_ccd_high_spin_and_starting_inside(gpu):  # :2305-2357
    t, _, ball = wall_and_ball(gpu, angvel=(0.0, 3000.0, 0.0))
    st = t.step()[ball]
    assert abs(float(np.dot(st[3:7], st[3:7])) - 1.0) <= 1e-3 and abs(st[1] - 0.9) <= 0.05
    t, _, ball = wall_and_ball(gpu, ball_pos=(0.0, 0.5, 0.0))
    assert abs(t.step()[ball, 1] - 0.5) <= 1e-4


def test_ccd_respects_collision_filter(gpu):  # :1694-1720
    t = Twin(gpu)
    t.body(t.shape(orc.BOX, [0.5, 2.0, 0.25]), (0.0, 0.0, 0.0), mass=0.0, group=1, mask=0)
    ball = t.body(t.shape(orc.SPHERE, [0.3]), (0.0, 0.0, -5.0), linvel=(0.0, 0.0, 10.0), mass=1.0)
    t.ccd(ball, 0.1, 0.3)
    for _ in range(60):
        st = t.step()
    assert st[ball, 2] > 4.0


@pytest.mark.parametrize("shape", ["box", "capsule", "sphere", "hull"])
def test_ccd_clamps_against_every_convex_target(gpu, shape):
    t = Twin(gpu)
    if shape == "box":
        s = t.shape(orc.BOX, [1.0, 0.1, 1.0])
    elif shape == "capsule":
        s = t.shape(orc.CAPSULE, [0.1, 1.0])
    elif shape == "sphere":
        s = t.shape(orc.SPHERE, [0.1])
    else:
        s = t.hull([[x, y, z] for x in (-1.0, 1.0) for y in (-0.1, 0.1) for z in (-1.0, 1.0)])
    quat = (0.0, 0.0, math.sin(math.pi / 4), math.cos(math.pi / 4)) if shape == "capsule" else (0.0, 0.0, 0.0, 1.0)
    t.body(s, (0.0, 0.5, 0.0), quat=quat, mass=0.0)
    ball = t.body(t.shape(orc.SPHERE, [0.3]), (0.0, 1.5, 0.0), linvel=(0.0, -180.0, 0.0), mass=1.0)
    t.ccd(ball, 0.1, 0.3)
    assert abs(t.step()[ball, 1] - 0.9) <= 0.05


def test_ccd_rain_of_fast_spheres_matches_the_oracle(gpu):
    """400 fast CCD spheres and 200 plain boxes over a grid of thin plates and a ground plane,
    under gravity: many sweeps per step, contacts and clamps in the same steps."""
    rng = np.random.default_rng(7)
    t = Twin(gpu, gravity=(0.0, -9.81, 0.0))
    t.body(t.shape(orc.PLANE, [0.0, 1.0, 0.0, 0.0]), (0.0, 0.0, 0.0), mass=0.0)
    plate = t.shape(orc.BOX, [1.5, 0.05, 1.5])
    for px in range(-3, 4):
        for pz in range(-3, 4):
            t.body(plate, (px * 3.2, 2.0 + 0.3 * ((px + pz) % 3), pz * 3.2), mass=0.0)
    sph = t.shape(orc.SPHERE, [0.2])
    box = t.shape(orc.BOX, [0.2, 0.2, 0.2])
    ids = []
    for k in range(600):
        pos = (float(rng.uniform(-11, 11)), float(rng.uniform(4, 12)), float(rng.uniform(-11, 11)))
        if k % 3 == 2:
            t.body(box, pos, linvel=(0.0, -5.0, 0.0))
        else:
            ids.append(t.body(sph, pos, linvel=(float(rng.uniform(-5, 5)), float(rng.uniform(-400, -60)), 0.0)))
    for i in ids:
        t.ccd(i, 0.05, 0.2)
    clamped = 0
    for _ in range(20):
        t.step(tol=1e-3)
        clamped += int(np.count_nonzero(t.g.ccd_clamps() < 1.0))
    assert clamped > 50


def test_ccd_in_batched_worlds_sweeps_only_its_own_world(gpu):
    """Batched worlds: a CCD ball sweeps only the bodies of its own world. Two worlds hold a ball
    at the same coordinates falling at 120 m/s; only world 0 has a wall under it (world 1's wall is
    50 m aside), so world 0's ball is clamped on its wall and world 1's ball passes through the
    place where world 0's wall is."""
    w = gpu.World(gravity=(0.0, 0.0, 0.0), batch=True)
    wall = w.add_shape(orc.BOX, [1.0, 0.1, 1.0])
    ball = w.add_shape(orc.SPHERE, [0.3])
    shape = np.array([wall, ball, wall, ball], dtype=np.uint32)
    pos = np.array([[0.0, 0.5, 0.0], [0.0, 1.0, 0.0], [50.0, 0.5, 0.0], [0.0, 1.0, 0.0]])
    quat = np.tile([0.0, 0.0, 0.0, 1.0], (4, 1))
    vel = np.array([[0.0, 0.0, 0.0], [0.0, -120.0, 0.0], [0.0, 0.0, 0.0], [0.0, -120.0, 0.0]])
    w.add_worlds_array([2, 2], shape, pos, quat, linvel=vel, mass=np.array([0.0, 1.0, 0.0, 1.0]))
    w.set_ccd(0, np.array([0.0, 0.1, 0.0, 0.1]), np.array([0.0, 0.3, 0.0, 0.3]))
    w.step(DT)
    st, clamps = w.state(), w.ccd_clamps()
    assert abs(st[1, 1] - 0.9) <= 0.05 and clamps[1] < 1.0
    assert st[3, 1] < -0.5 and clamps[3] == 1.0
    assert w.stats()["device_status"] == 0
