"""GPU joint rows (point-to-point, fixed, hinge) against the oracle.

Every scene is built twice from one description, stepped on the GPU and in the
oracle (f32), and the oracle is given the GPU's solve order for the contact
groups and for the joints. Joint rows use atan2/asin (hinge angle, fixed-joint
Euler angles), whose last ulp may differ between CUDA and the host libm, so the
states are compared in windows of 10 steps from a shared state (the oracle takes
the GPU's body state at the start of each window) within 1e-4; activation states
must be equal at every compared step. The reference's own assertions for the
scenes (crates/bullet-dynamics/src/constraint/tests.rs) are also checked on the
GPU trajectory.
"""
import math

import numpy as np
import pytest

import oracle_api as orc

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


class JScene:
    def __init__(self, gravity=(0.0, -9.81, 0.0)):
        self.gravity = gravity
        self.shapes, self.bodies, self.joints = [], [], []
        self.solver = {}

    def shape(self, kind, params):
        self.shapes.append((kind, list(params)))
        return len(self.shapes) - 1

    def body(self, shape, pos, quat=(0, 0, 0, 1), mass=1.0, linvel=(0, 0, 0), angvel=(0, 0, 0), activation=0):
        self.bodies.append(dict(shape=shape, pos=pos, quat=quat, mass=mass, linvel=linvel, angvel=angvel,
                                activation=activation))
        return len(self.bodies) - 1

    def joint(self, kind, a, b, fa, fb, **kw):
        self.joints.append((kind, a, b, np.asarray(fa, dtype=np.float64), np.asarray(fb, dtype=np.float64), kw))

    def spring2(self, joint):
        """A bgpu.Spring2 joint (its descriptor drives both worlds)."""
        self.joints.append(("spring2", joint))

    def build(self, gpu):
        w = gpu.World(gravity=self.gravity, num_iterations=10, **self.solver)
        o = orc.OracleWorld("f32")
        o.set_gravity(self.gravity)
        o.set_solver(num_iterations=10, **self.solver)
        for kind, params in self.shapes:
            w.add_shape(kind, params)
            o.add_shape(kind, params)
        for b in self.bodies:
            w.add_body(b["shape"], b["pos"], b["quat"], b["linvel"], b["angvel"], mass=b["mass"],
                       activation=b["activation"])
            o.add_body(b["shape"], b["pos"], quat=b["quat"], linvel=b["linvel"], angvel=b["angvel"], mass=b["mass"],
                       activation=b["activation"])
        for jt in self.joints:
            if jt[0] == "spring2":
                w.add_spring2(jt[1])
                o.add_joint(orc.spring2_joint_desc(jt[1]))
                continue
            kind, a, b, fa, fb, kw = jt
            w.add_joint(kind, a, b, fa, fb, **kw)
            o.add_joint(orc.joint_desc(kind, a, b, fa, fb, **kw))
        o.set_joint_order(w.joint_order())
        return w, o


def run_pair(scene, gpu, steps, tol=1e-4, window=10, each=None):
    """Steps both worlds; returns the GPU states per step. `each(step, gpu_world)` runs after every step."""
    w, o = scene.build(gpu)
    states = []
    worst = 0.0
    for step in range(steps):
        if step % window == 0:
            o.set_state(w.state().astype(np.float64))
        w.step(DT)
        o.set_solve_order(w.solve_order())
        o.step(DT)
        st = w.stats()
        assert st["device_status"] == 0, st
        g, r = w.state(), o.state()
        np.testing.assert_array_equal(g[:, 13], r[:, 13], err_msg=f"activation, step {step}")
        err = float(np.abs(g[:, :13] - r[:, :13]).max())
        worst = max(worst, err)
        assert err <= tol, f"step {step}: max abs state error {err}"
        if len(scene.joints):
            ga = w.joint_angles()
            ra = o.joint_angles(len(scene.joints))
            assert np.abs(ga - ra).max() <= 10 * tol, (step, ga, ra)
            if any(jt[0] == "spring2" for jt in scene.joints):
                gs, rs = w.spring2_state(), o.spring2_state(len(scene.joints))
                assert np.abs(gs - rs).max() <= 10 * tol, (step, gs, rs)
        states.append(g)
        if each:
            each(step, w)
    return w, o, np.array(states), worst


def quat_z(a):
    return (0.0, 0.0, math.sin(a / 2), math.cos(a / 2))


def rotate(q, v):
    x, y, z, w = q
    b = np.array([x, y, z])
    v = np.asarray(v, dtype=np.float64)
    return v * (w * w - b @ b) + b * (2 * (v @ b)) + np.cross(b, v) * (2 * w)


def test_pendulum_matches_the_oracle_and_keeps_its_pivot(gpu):  # constraint/tests.rs:46-91
    s = JScene()
    anchor = s.body(s.shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    a45 = math.pi / 4
    bob = s.body(s.shape(orc.SPHERE, [0.1]), (math.sin(a45), -math.cos(a45), 0.0), quat=quat_z(-a45))
    s.joint(orc.JOINT_POINT2POINT, bob, anchor, orc.frame((-1.0, 0.0, 0.0)), orc.frame((0.0, 0.0, 0.0)))
    _, _, st, _ = run_pair(s, gpu, 300)
    err = [np.linalg.norm(x[bob, 0:3] + rotate(x[bob, 3:7], (-1.0, 0.0, 0.0))) for x in st]
    assert max(err) < 0.2 and st[:, bob, 0].min() < -0.5


def test_two_link_chain_matches_the_oracle(gpu):  # constraint/tests.rs:124-176
    s = JScene()
    anchor = s.body(s.shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    sph = s.shape(orc.SPHERE, [0.1])
    upper = s.body(sph, (0.0, -1.0, 0.0))
    lower = s.body(sph, (0.0, -3.0, 0.0), linvel=(2.0, 0.0, 0.0))
    s.joint(orc.JOINT_POINT2POINT, upper, anchor, orc.frame((0.0, 1.0, 0.0)), orc.frame((0.0, 0.0, 0.0)))
    s.joint(orc.JOINT_POINT2POINT, lower, upper, orc.frame((0.0, 1.0, 0.0)), orc.frame((0.0, -1.0, 0.0)))
    w, _, st, _ = run_pair(s, gpu, 200)
    assert len(w.joint_order()) == 2


def door(gravity=(0.0, -9.81, 0.0), door_pos=(0.0, 0.5, 0.0), open_45=True, **kw):
    s = JScene(gravity)
    anchor = s.body(s.shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    pos, quat = door_pos, (0, 0, 0, 1)
    if open_45:
        a45 = math.pi / 4
        pos, quat = (math.cos(a45) * 0.5, math.sin(a45) * 0.5, 0.0), quat_z(a45)
    d = s.body(s.shape(orc.BOX, [0.5, 0.5, 0.2]), pos, quat=quat, mass=2.0)
    fa, fb = orc.hinge_frames((-0.5, 0.0, 0.0), (0, 0, 1), (0, 0, 0), (0, 0, 1))
    s.joint(orc.JOINT_HINGE, d, anchor, fa, fb, **kw)
    return s


def test_hinge_door_matches_the_oracle(gpu):  # constraint/tests.rs:180-235
    w, _, st, _ = run_pair(door(), gpu, 300)
    assert abs(w.joint_angles()[0]) <= math.pi


def test_hinge_limit_matches_the_oracle(gpu):  # constraint/tests.rs:238-281
    s = door(door_pos=(0.0, 0.0, 0.0), flags=orc.JF_DISABLE_COLLISIONS | orc.JF_LIMIT, limit=(-0.3, 0.3))
    angles = []
    run_pair(s, gpu, 300, each=lambda step, w: angles.append(float(w.joint_angles()[0])))
    assert min(angles) > -0.35


def test_hinge_motor_matches_the_oracle(gpu):  # constraint/tests.rs:284-316
    s = door(gravity=(0.0, 0.0, 0.0), door_pos=(0.5, 0.0, 0.0), open_45=False,
             flags=orc.JF_DISABLE_COLLISIONS | orc.JF_MOTOR, motor=(1.0, 1000.0))
    w, _, _, _ = run_pair(s, gpu, 180)
    assert abs(w.joint_angles()[0] - 3.0) < 1.0


def test_joint_suppresses_collisions_between_linked_bodies(gpu):  # constraint/tests.rs:320-360
    s = JScene((0.0, 0.0, 0.0))
    box = s.shape(orc.BOX, [0.5, 0.5, 0.5])
    a = s.body(box, (0, 0, 0))
    b = s.body(box, (0, 0, 0))
    s.joint(orc.JOINT_POINT2POINT, a, b, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)))
    w, o, st, _ = run_pair(s, gpu, 30)
    assert w.stats()["num_contacts"] == 0
    assert np.linalg.norm(st[-1, b, 0:3] - st[-1, a, 0:3]) < 0.02


def test_impulse_clamp_matches_the_oracle(gpu):  # constraint/tests.rs:363-400
    s = JScene()
    anchor = s.body(s.shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    bob = s.body(s.shape(orc.SPHERE, [0.1]), (0, 0, 0), mass=10.0)
    s.joint(orc.JOINT_POINT2POINT, bob, anchor, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)), impulse_clamp=0.1)
    _, _, st, _ = run_pair(s, gpu, 120)
    assert st[-1, bob, 1] < -0.5


def test_fixed_joint_matches_the_oracle(gpu):  # constraint/tests.rs:403-458
    s = JScene()
    anchor = s.body(s.shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    box = s.body(s.shape(orc.BOX, [0.3, 0.3, 0.3]), (0.0, 1.0, 0.0), linvel=(2.0, 0.0, 0.0), angvel=(0.0, 0.0, 4.0))
    s.joint(orc.JOINT_FIXED, box, anchor, orc.frame((0.0, 0.5, 0.0)), orc.frame((0.0, 1.5, 0.0)))
    _, _, st, _ = run_pair(s, gpu, 300)
    assert np.linalg.norm(st[-1, box, 0:3] - (0.0, 1.0, 0.0)) < 0.03


def test_welded_pair_lands_on_the_ground_like_the_oracle(gpu):  # constraint/tests.rs:461-515
    """Contacts and joint rows in one solve: the welded boxes tumble onto a plane."""
    s = JScene()
    s.body(s.shape(orc.PLANE, [0.0, 1.0, 0.0, 0.0]), (0, 0, 0), mass=0.0)
    box = s.shape(orc.BOX, [0.4, 0.4, 0.4])
    a = s.body(box, (0.0, 1.2, 0.0), angvel=(1.0, 2.0, 0.0))
    b = s.body(box, (0.0, 1.6, 0.0), angvel=(1.0, 2.0, 0.0))
    s.joint(orc.JOINT_FIXED, a, b, orc.frame((0.0, 0.2, 0.0)), orc.frame((0.0, -0.2, 0.0)))
    w, _, st, _ = run_pair(s, gpu, 150)
    assert w.stats()["num_contacts"] > 0


def chains(kinds, n_chains=80):
    """n_chains eight-link chains of boxes dropped onto a plane, five chains per row, rows 0.6 m
    apart (no two chains touch at the start); link k of chain c is a joint of kind
    kinds[(c + k) % len(kinds)]. 80 chains give two joint colours of 280 joints, more than
    one block, so the grid-wide joint phases run."""
    s = JScene()
    s.body(s.shape(orc.PLANE, [0.0, 1.0, 0.0, 0.0]), (0, 0, 0), mass=0.0)
    box = s.shape(orc.BOX, [0.2, 0.1, 0.1])
    rng = np.random.default_rng(5)
    hfa, hfb = orc.hinge_frames((0.25, 0.0, 0.0), (0, 0, 1), (-0.25, 0.0, 0.0), (0, 0, 1))
    for c in range(n_chains):
        x0, z0 = (c % 5) * 4.5 - 11.0, (c // 5) * 0.6 - 5.0
        y0 = 0.5 + rng.uniform(0.0, 0.4)
        ids = [s.body(box, (x0 + 0.5 * k, y0, z0)) for k in range(8)]
        for k in range(7):
            kind = kinds[(c + k) % len(kinds)]
            if kind == orc.JOINT_HINGE:
                s.joint(kind, ids[k], ids[k + 1], hfa, hfb)
            else:
                s.joint(kind, ids[k], ids[k + 1], orc.frame((0.25, 0.0, 0.0)), orc.frame((-0.25, 0.0, 0.0)))
    return s


def test_many_chains_on_the_ground_match_the_oracle(gpu):
    """80 eight-link chains (point-to-point and hinge links, 560 joints, joint colours larger
    than one block) fall onto a plane: grid-wide joint phases mixed with contacts. The pose
    update's sin/cos and the redetect gate's acos may differ in the last ulp, so the windows
    are 5 steps and the bound 1e-3 (the mixed convex pile's); the rows themselves are
    compared one step from identical states below."""
    w, _, _, _ = run_pair(chains((orc.JOINT_POINT2POINT, orc.JOINT_HINGE)), gpu, 30, tol=1e-3, window=5)
    assert w.num_joints == 560 and w.stats()["num_contacts"] > 0


def test_many_chains_with_fixed_links_match_the_oracle(gpu):
    """The same with a third of the links fixed joints, whose angular rows take their bias
    from atan2/asin of the relative rotation: 5-step windows, 1e-3."""
    w, _, _, _ = run_pair(chains((orc.JOINT_POINT2POINT, orc.JOINT_HINGE, orc.JOINT_FIXED)), gpu, 30, tol=1e-3,
                          window=5)
    assert w.num_joints == 560


def test_chain_joint_rows_match_the_oracle_after_one_step(gpu):
    """One step of the 80 chains from identical states: every joint row (ids, bodies, limit
    kind exact; effective mass, bias and accumulated impulse within 1e-5 relative)."""
    w, o = chains((orc.JOINT_POINT2POINT, orc.JOINT_HINGE, orc.JOINT_FIXED)).build(gpu)
    w.step(DT)
    o.set_solve_order(w.solve_order())
    o.step(DT)
    g, r = w.joint_rows(), o.joint_rows()
    rows_of = {orc.JOINT_POINT2POINT: 3, orc.JOINT_HINGE: 5, orc.JOINT_FIXED: 6}
    kinds = (orc.JOINT_POINT2POINT, orc.JOINT_HINGE, orc.JOINT_FIXED)
    expected = sum(rows_of[kinds[(c + k) % 3]] for c in range(80) for k in range(7))
    assert g.shape == r.shape == (expected, 8)
    np.testing.assert_array_equal(g[:, [0, 1, 2, 5]], r[:, [0, 1, 2, 5]])
    np.testing.assert_allclose(g[:, [3, 4, 6]], r[:, [3, 4, 6]], rtol=1e-5, atol=1e-6)


def test_joint_keeps_its_partner_awake_like_the_oracle(gpu):  # world/islands.rs:539-575
    """Two bodies far apart joined by a point-to-point joint, one that never deactivates:
    the joint links their islands, so the other one never sleeps; an unlinked copy sleeps."""
    s = JScene((0.0, 0.0, 0.0))
    sph = s.shape(orc.SPHERE, [0.5])
    a = s.body(sph, (4.0, 0.0, 0.0), activation=4)  # DISABLE_DEACTIVATION
    b = s.body(sph, (6.0, 0.0, 0.0))
    c = s.body(sph, (20.0, 0.0, 0.0))  # no joint: falls asleep after 2 s
    s.joint(orc.JOINT_POINT2POINT, a, b, orc.frame((1.0, 0.0, 0.0)), orc.frame((-1.0, 0.0, 0.0)))
    _, _, st, _ = run_pair(s, gpu, 200)
    assert st[-1, b, 13] != 2 and st[-1, c, 13] == 2


def test_joint_rows_and_impulses_match_the_oracle(gpu):
    """One step of the door with a motor: the GPU's rows (effective mass, bias, limit kind,
    accumulated impulse) equal the oracle's in solve order."""
    s = door(gravity=(0.0, -9.81, 0.0), flags=orc.JF_DISABLE_COLLISIONS | orc.JF_MOTOR, motor=(0.5, 2.0))
    w, o = s.build(gpu)
    w.step(DT)
    o.set_solve_order(w.solve_order())
    o.step(DT)
    g, r = w.joint_rows(), o.joint_rows()
    assert g.shape == r.shape == (6, 8)
    np.testing.assert_array_equal(g[:, [0, 1, 2, 5]], r[:, [0, 1, 2, 5]])
    np.testing.assert_allclose(g[:, [3, 4, 6]], r[:, [3, 4, 6]], rtol=1e-5, atol=1e-6)


def test_joint_descriptors_are_checked(gpu):
    w = gpu.World()
    sph = w.sphere(0.5)
    a = w.add_body(sph, (0, 0, 0))
    with pytest.raises(gpu.BgpuError):
        w.add_joint(0, a, a, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)))
    with pytest.raises(gpu.BgpuError):
        w.add_joint(0, a, 7, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)))
    with pytest.raises(gpu.BgpuError):
        w.add_joint(9, a, a, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)))
    b = w.add_body(sph, (2, 0, 0))
    w.add_joint(0, a, b, orc.frame((1, 0, 0)), orc.frame((-1, 0, 0)))
    with pytest.raises(gpu.BgpuError):
        gpu.Tape(w, 10)


@pytest.mark.parametrize("ratio,pos_b,quat_a,spin", [
    (2.0, (3.0, 0.0, 0.0), (0, 0, 0, 1), (0.0, 0.0, 6.0)),                                          # gear.rs:77-101
    (1.0, (5.0, 1.0, -2.0), (0, 0, 0, 1), (0.0, 0.0, 6.0)),                                         # gear.rs:122-157
    (1.0, (4.0, 0.0, 0.0), (math.sin(math.pi / 4), 0.0, 0.0, math.cos(math.pi / 4)), (0.0, -6.0, 0.0)),  # :159-187
])
def test_gear_matches_the_oracle(gpu, ratio, pos_b, quat_a, spin):
    s = JScene((0.0, 0.0, 0.0))
    sph = s.shape(orc.SPHERE, [0.5])
    mass = 2.0 if ratio == 2.0 else 1.0
    a = s.body(sph, (0.0, 0.0, 0.0), quat=quat_a, mass=mass, angvel=spin)
    b = s.body(sph, pos_b, mass=mass)
    s.joint(orc.JOINT_GEAR, a, b, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)), gear_ratio=ratio)
    _, _, st, _ = run_pair(s, gpu, 30)
    if ratio == 2.0:
        assert abs(st[9, b, 12] + st[9, a, 12] / 2.0) < 1e-3


def slider_scene(box_pos, linvel=(0, 0, 0), angvel=(0, 0, 0), **kw):
    s = JScene((0.0, 0.0, 0.0))
    anchor = s.body(s.shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    box = s.body(s.shape(orc.BOX, [0.3, 0.3, 0.3]), box_pos, linvel=linvel, angvel=angvel)
    s.joint(orc.JOINT_SLIDER, anchor, box, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)), **kw)
    return s, box


@pytest.mark.parametrize("case", ["slide", "limit", "motor", "angular_limit", "frame_b_motor"])
def test_slider_matches_the_oracle(gpu, case):  # constraint/tests.rs:608-771
    if case == "slide":
        s, box = slider_scene((1.0, 0.0, 0.0), linvel=(1.5, 0.5, 0.2), angvel=(0.0, 0.0, 3.0))
    elif case == "limit":
        s, box = slider_scene((0.2, 0.0, 0.0), linvel=(4.0, 0.0, 0.0), lin_limits=(-0.3, 0.3))
    elif case == "motor":
        s, box = slider_scene((0.0, 0.0, 0.0), flags=orc.JF_DISABLE_COLLISIONS | orc.JF_LIN_MOTOR,
                              lin_motor=(1.5, 100.0))
    elif case == "angular_limit":
        s, box = slider_scene((0.0, 0.0, 0.0), angvel=(3.0, 0.0, 0.0), ang_limits=(-0.4, 0.4))
    else:
        s, box = slider_scene((0.0, 0.0, 0.0), flags=orc.JF_DISABLE_COLLISIONS | orc.JF_LIN_MOTOR | orc.JF_FRAME_B,
                              lin_motor=(-1.0, 50.0), lin_limits=(-1.0, 1.0))
    positions = []

    def each(step, w):
        positions.append(float(w.joint_positions()[0]))

    w, o, st, _ = run_pair(s, gpu, 150, each=each)
    assert abs(positions[-1] - o.joint_positions(1)[0]) < 1e-3
    if case == "limit":
        assert st[:, box, 0].max() < 0.34
    if case == "motor":
        assert abs(st[-1, box, 0] - 3.75) < 0.3


def test_slider_between_two_bodies_on_the_ground_matches_the_oracle(gpu):
    """A slider between two dynamic boxes resting on a plane: contacts and the slider's
    frame-offset rows (both bodies dynamic, so no static-body branch) in one solve."""
    s = JScene()
    s.body(s.shape(orc.PLANE, [0.0, 1.0, 0.0, 0.0]), (0, 0, 0), mass=0.0)
    box = s.shape(orc.BOX, [0.3, 0.3, 0.3])
    a = s.body(box, (0.0, 0.3, 0.0))
    b = s.body(box, (1.0, 0.3, 0.0), linvel=(1.0, 0.0, 0.5))
    s.joint(orc.JOINT_SLIDER, a, b, orc.frame((0.5, 0.0, 0.0)), orc.frame((-0.5, 0.0, 0.0)), lin_limits=(-0.2, 0.4))
    run_pair(s, gpu, 120)


def spring2_pair(b_quat=(0.0, 0.0, 0.0, 1.0), order=0, setup=None, gravity=(0.0, 0.0, 0.0), linvel_b=(0, 0, 0),
                 angvel_b=(0, 0, 0)):
    """generic6dof_spring2.rs:1590-1630: two never-sleeping 1 kg spheres at x = -1 and +1 joined at
    the origin, B pre-rotated by b_quat with its pivot counter-rotated."""
    import bgpu
    s = JScene(gravity)
    sph = s.shape(orc.SPHERE, [0.5])
    a = s.body(sph, (-1.0, 0.0, 0.0), activation=orc.DISABLE_DEACTIVATION)
    b = s.body(sph, (1.0, 0.0, 0.0), quat=b_quat, linvel=linvel_b, angvel=angvel_b,
               activation=orc.DISABLE_DEACTIVATION)
    inv = (-b_quat[0], -b_quat[1], -b_quat[2], b_quat[3])
    j = bgpu.Spring2(a, b, orc.frame((1.0, 0.0, 0.0)), orc.frame(rotate(inv, (-1.0, 0.0, 0.0))), rotate_order=order)
    if setup:
        setup(j)
    s.spring2(j)
    return s, a, b


def quat_axis(axis, a):
    v = [0.0, 0.0, 0.0]
    v[axis] = math.sin(a / 2)
    return (v[0], v[1], v[2], math.cos(a / 2))


def _s2_case(case):
    """The reference's spring-2 world tests (generic6dof_spring2.rs:1644-1903) as scenes."""
    if case == "ball":  # :1644-1664
        return spring2_pair(linvel_b=(0.0, 2.0, 0.0), angvel_b=(0.0, 0.0, 3.0)), 120
    if case == "limit_inside":  # :1668-1706
        return spring2_pair(quat_axis(0, 0.2), setup=lambda j: j.set_limit(3, -1.0, 1.0)), 120
    if case == "limit_outside":
        return spring2_pair(quat_axis(0, 1.5), setup=lambda j: j.set_limit(3, -1.0, 1.0)), 60
    if case == "locked":  # :1709-1727
        return spring2_pair(quat_axis(0, -0.5), setup=lambda j: j.set_limit(3, 0.3, 0.3)), 180

    def spring_y(k, d=None):
        def f(j):
            j.enable_spring(4)
            j.set_stiffness(4, k, True)
            if d is not None:
                j.set_damping(4, d, True)
        return f
    if case == "spring":  # :1730-1770
        return spring2_pair(quat_axis(1, 0.3), setup=spring_y(40.0, 0.5)), 300
    if case == "stiffness_clamp":  # :1773-1795
        return spring2_pair(quat_axis(1, 0.3), setup=spring_y(1.0e6)), 240
    if case == "damping_clamp":  # :1798-1822
        return spring2_pair(quat_axis(1, 0.3), setup=spring_y(40.0, 100.0)), 300
    if case == "linear_spring":  # :1825-1847
        def f(j):
            j.set_linear_limits((1.0, 1.0, 1.0), (-1.0, -1.0, -1.0))
            j.enable_spring(0)
            j.set_stiffness(0, 5.0, True)
            j.set_damping(0, 0.5, True)
            j.set_equilibrium_point(0, 0.5)
        return spring2_pair(setup=f), 360
    if case == "servo":  # :1850-1871
        def f(j):
            j.enable_motor(3)
            j.set_servo(3)
            j.set_servo_target(3, 0.5)
            j.set_target_velocity(3, 2.0)
            j.set_max_motor_force(3, 10.0)
        return spring2_pair(setup=f), 300
    if case == "overrides":  # :1874-1903, plus every override and a bounce
        def f(j):
            j.set_limit(3, -1.0, 1.0)
            j.set_stop_erp(3, 0.3)
            j.set_stop_cfm(3, 0.01)
            j.set_bounce(3, 0.5)
            j.set_limit(4, -0.2, 0.2)
            j.enable_motor(5)
            j.set_target_velocity(5, 1.0)
            j.set_max_motor_force(5, 4.0)
            j.set_motor_erp(5, 0.5)
            j.set_motor_cfm(5, 0.02)
        s = spring2_pair(quat_axis(0, 1.5), setup=f)
        s[0].solver = dict(erp=0.5)
        return s, 120
    raise KeyError(case)


@pytest.mark.parametrize("case", ["ball", "limit_inside", "limit_outside", "locked", "spring", "stiffness_clamp",
                                  "damping_clamp", "linear_spring", "servo", "overrides"])
def test_spring2_matches_the_oracle(gpu, case):
    (s, a, b), steps = _s2_case(case)
    angles = []
    _, _, st, _ = run_pair(s, gpu, steps, each=lambda step, w: angles.append(w.spring2_state()[0].copy()))
    angles = np.array(angles)
    # the reference's own assertions on the GPU trajectory
    if case == "limit_inside":
        assert abs(angles[-1, 0] + 0.2) < 0.02
    if case == "limit_outside":
        assert angles[-1, 0] > -1.3
    if case == "locked":
        assert abs(angles[-1, 0] - 0.3) < 0.02
    if case == "spring":
        assert np.count_nonzero(np.diff(np.sign(angles[:, 1]))) >= 2 and np.abs(angles[:, 1]).max() < 0.35
    if case == "damping_clamp":
        assert angles[:, 1].max() <= 0.0
    if case == "linear_spring":
        assert abs(angles[-1, 3] - 0.5) < 0.05
    if case == "servo":
        assert abs(angles[-1, 0] - 0.5) < 0.05


@pytest.mark.parametrize("order", [0, 1, 2, 3, 4, 5])
def test_spring2_rotate_orders_match_the_oracle(gpu, order):
    """Every Euler order, with a limited, a locked and a sprung angular axis and a linear spring."""
    def f(j):
        j.set_limit(3, -0.3, 0.4)
        j.set_limit(4, 0.1, 0.1)
        j.enable_spring(5)
        j.set_stiffness(5, 20.0, True)
        j.set_damping(5, 0.2, True)
        j.set_limit(2, -0.1, 0.1)
        j.enable_spring(2)
        j.set_stiffness(2, 30.0, True)
    q = (0.1, -0.2, 0.15, math.sqrt(1.0 - 0.01 - 0.04 - 0.0225))
    (s, a, b) = spring2_pair(q, order=order, setup=f, gravity=(0.0, -9.81, 0.0), angvel_b=(1.0, -2.0, 0.5))
    s.bodies[a]["mass"] = 0.0
    s.bodies[a]["activation"] = 0
    run_pair(s, gpu, 90)


def test_spring2_rows_match_the_oracle(gpu):
    """One step's rows (mass, bias, limit kind, impulse, cfm) of a joint with every row shape."""
    def f(j):
        j.set_limit(3, -1.0, 1.0)
        j.set_stop_cfm(3, 0.01)
        j.set_limit(4, 0.2, 0.2)
        j.enable_motor(4)
        j.set_target_velocity(4, 1.0)
        j.enable_motor(5)
        j.set_servo(5)
        j.set_servo_target(5, 0.4)
        j.set_target_velocity(5, 2.0)
        j.enable_spring(5)
        j.set_stiffness(5, 10.0, True)
        j.set_linear_limits((0.0, -0.1, 1.0), (0.0, 0.1, -1.0))
        j.enable_spring(2)
        j.set_stiffness(2, 5.0, False)
        j.set_damping(2, 0.5, False)
    (s, a, b) = spring2_pair(quat_axis(0, 1.5), setup=f, angvel_b=(0.5, 0.2, -0.3))
    w, o = s.build(gpu)
    o.set_state(w.state().astype(np.float64))
    w.step(DT)
    o.step(DT)
    g, r = w.joint_rows(), o.joint_rows()
    assert g.shape == r.shape and len(g) == 2 + 2 + 2 + 1 + 2 + 1, (g.shape, r.shape)
    np.testing.assert_array_equal(g[:, [0, 1, 2, 5]], r[:, [0, 1, 2, 5]])
    np.testing.assert_allclose(g[:, [3, 4, 6, 7]], r[:, [3, 4, 6, 7]], rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("case", ["suspension", "axle_spin", "steering"])
def test_hinge2_matches_the_oracle(gpu, case):  # generic6dof_spring2.rs:2027-2111
    import bgpu
    gravity, radius, pos, angvel, steps = {
        "suspension": ((0.0, 0.0, -9.8), 0.2, (0.0, 0.0, -0.3), (0.0, 0.0, 0.0), 240),
        "axle_spin": ((0.0, 0.0, 0.0), 0.2, (0.0, 0.0, 0.0), (8.0, 0.0, 0.0), 60),
        "steering": ((0.0, 0.0, 0.0), 0.15, (0.9, 0.0, 0.0), (0.0, 0.0, 6.0), 120),
    }[case]
    s = JScene(gravity)
    chassis = s.body(s.shape(orc.SPHERE, [0.5]), (0.0, 0.0, 0.0), mass=0.0)
    wheel = s.body(s.shape(orc.SPHERE, [radius]), pos, angvel=angvel)
    s.spring2(bgpu.Spring2.hinge2(chassis, wheel, (0, 0, 0), (0, 0, 0, 1), pos, (0, 0, 0, 1), (0, 0, 0), (0, 0, 1),
                                  (1, 0, 0)))
    steer = []
    _, _, st, _ = run_pair(s, gpu, steps, each=lambda step, w: steer.append(float(w.spring2_state()[0, 2])))
    if case == "suspension":
        assert -0.45 < st[-1, wheel, 2] < -0.10 and abs(st[-1, wheel, 9]) < 1.0
    if case == "axle_spin":
        assert st[-1, wheel, 10] > 7.5 and abs(st[-1, wheel, 2]) < 1e-4
    if case == "steering":
        assert max(abs(x) for x in steer) < math.pi / 4 + 0.15


def spring2_chains(count=150, cols=15, links=3, spacing=4.0, base_height=4.0, pitch=0.55, half=0.2, mass=1.0,
                   stiffness=5.0, damping=0.3):
    """The reference's spring2_chains perf scene (tools/perf_scenes.json "spring2_chains";
    examples/perf_scenes.rs add_spring2): static anchors with horizontal chains of boxes joined by
    spring-2 joints whose three angular springs are on, never sleeping."""
    import bgpu
    s = JScene()
    box = s.shape(orc.BOX, [half, half, half])
    rows = -(-count // cols)
    for k in range(count):
        col, row = k % cols, k // cols
        x = (col - (cols - 1) / 2.0) * spacing
        z = (row - (rows - 1) / 2.0) * spacing
        prev = s.body(box, (x, base_height, z), mass=0.0)
        for i in range(1, links + 1):
            body = s.body(box, (x + i * pitch, base_height, z), mass=mass, activation=orc.DISABLE_DEACTIVATION)
            j = bgpu.Spring2(prev, body, orc.frame((pitch / 2.0, 0.0, 0.0)), orc.frame((-pitch / 2.0, 0.0, 0.0)))
            for ax in range(3, 6):
                j.enable_spring(ax)
                j.set_stiffness(ax, stiffness, True)
                j.set_damping(ax, damping, True)
            s.spring2(j)
            prev = body
    return s


def test_spring2_chains_match_the_oracle(gpu):
    """The spring2_chains scene (150 chains, 450 joints of 6 rows): hanging under gravity."""
    s = spring2_chains()
    w, _, st, _ = run_pair(s, gpu, 120, tol=1e-3, window=5)
    assert w.joint_rows().shape[0] == 450 * 6
    assert st[-1, :, 1].min() < 3.9  # the chains sag


@pytest.mark.parametrize("case", ["swing_limit", "twist_lock", "fixed", "hinge_y", "hinge_z", "motor"])
def test_cone_twist_matches_the_oracle(gpu, case):  # constraint/tests.rs:518-600; conetwist.rs:222-539
    """A bob pinned at a static anchor by a cone twist (cone axis X on both bodies): the reference's
    two cone-twist tests, the fixed and both hinge configurations, and a motor target."""
    spans, angvel, gravity, steps = {
        "swing_limit": ((0.44, 0.44, -1.0), (0.0, 0.0, 4.0), (0.0, -9.81, 0.0), 300),
        "twist_lock": ((0.9, 0.9, 0.0), (6.0, 0.0, 0.0), (0.0, -9.81, 0.0), 300),
        "fixed": ((0.0, 0.0, 1e30), (0.0, 3.0, 3.0), (0.0, -9.81, 0.0), 120),
        "hinge_y": ((0.0, 0.5, 1e30), (0.0, 3.0, 3.0), (0.0, -9.81, 0.0), 120),
        "hinge_z": ((0.5, 0.0, 1e30), (0.0, 3.0, 3.0), (0.0, -9.81, 0.0), 120),
        "motor": ((1.0, 1.0, 1.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 200),
    }[case]
    s = JScene(gravity)
    anchor = s.body(s.shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    bob = s.body(s.shape(orc.SPHERE, [0.1]), (0, 0, 0), angvel=angvel)
    kw = dict(cone=tuple(spans) + (1.0, 0.3, 1.0))
    flags = orc.JF_DISABLE_COLLISIONS
    if case == "motor":
        kw["cone_motor"] = ((0.0, 0.0, math.sin(0.15), math.cos(0.15)), 5.0)
        flags |= 512
    s.joint(orc.JOINT_CONETWIST, bob, anchor, orc.frame((0, 0, 0)), orc.frame((0, 0, 0)), flags=flags, **kw)
    _, _, st, _ = run_pair(s, gpu, steps)
    ax = lambda x, i: rotate(x[i, 3:7], (1.0, 0.0, 0.0))
    swing = [math.acos(max(-1.0, min(1.0, float(ax(x, anchor) @ ax(x, bob))))) for x in st]
    if case == "swing_limit":
        assert 0.3 < max(swing) < 0.55
    if case == "twist_lock":
        assert abs(st[-1, bob, 10]) < 0.1
    if case == "motor":
        assert abs(swing[-1] - 0.3) < 0.05


@pytest.mark.parametrize("case", ["locked", "angular_limit", "motor", "linear_limit", "universal_free",
                                  "universal_locked"])
def test_generic_6dof_matches_the_oracle(gpu, case):  # constraint/tests.rs:773-930; generic6dof.rs:614-676
    import bgpu
    if case.startswith("universal"):
        s = JScene((0.0, 0.0, 0.0))
        sph = s.shape(orc.SPHERE, [0.3])
        a = s.body(sph, (0, 0, 0), mass=0.0)
        b = s.body(sph, (1, 0, 0), angvel=(0.0, 0.0, 5.0) if case == "universal_free" else (0.0, 5.0, 0.0))
        s.spring2(bgpu.Generic6Dof.universal(a, b, (0, 0, 0), (0, 0, 0, 1), (1, 0, 0), (0, 0, 0, 1), (1, 0, 0),
                                             (0, 0, 1), (1, 0, 0)))
        _, _, st, _ = run_pair(s, gpu, 60)
        if case == "universal_free":
            assert st[-1, b, 12] > 4.0
        else:
            assert abs(st[-1, b, 11]) < 0.05
        return
    box_pos, frames, gravity, setup, linvel, angvel, steps = {
        "locked": ((0, 1, 0), ((0, 0.5, 0), (0, 1.5, 0)), (0, -9.81, 0),
                   lambda j: j.set_angular_limits((0, 0, 0), (0, 0, 0)), (2, 0, 0), (0, 0, 4), 300),
        "angular_limit": ((0, 0, 0), ((0, 0, 0), (0, 0, 0)), (0, 0, 0),
                          lambda j: j.set_angular_limits((-0.4, -1.0, -1.0), (0.4, 1.0, 1.0)), (0, 0, 0), (4, 0, 0), 300),
        "motor": ((0, 0, 0), ((0, 0, 0), (0, 0, 0)), (0, 0, 0), lambda j: j.enable_motor(5, 1.0, 100.0), (0, 0, 0),
                  (0, 0, 0), 180),
        "linear_limit": ((0.2, 0, 0), ((0, 0, 0), (0, 0, 0)), (0, 0, 0),
                         lambda j: j.set_linear_limits((-0.3, 0, 0), (0.3, 0, 0)), (4, 0, 0), (0, 0, 0), 180),
    }[case]
    s = JScene(gravity)
    anchor = s.body(s.shape(orc.BOX, [0.2, 0.2, 0.2]), (0, 0, 0), mass=0.0)
    box = s.body(s.shape(orc.BOX, [0.3, 0.3, 0.3]), box_pos, linvel=linvel, angvel=angvel)
    j = bgpu.Generic6Dof(box, anchor, orc.frame(frames[0]), orc.frame(frames[1]))
    setup(j)
    s.spring2(j)
    angles = []
    _, _, st, _ = run_pair(s, gpu, steps, each=lambda step, w: angles.append(w.spring2_state()[0].copy()))
    angles = np.array(angles)
    if case == "angular_limit":
        assert 0.3 < np.abs(angles[:, 0]).max() < 0.5
    if case == "motor":
        assert abs(abs(angles[-1, 2]) - 3.0) < 1.0
    if case == "linear_limit":
        assert st[:, box, 0].max() < 0.34 and st[-1, box, 0] < 0.3
