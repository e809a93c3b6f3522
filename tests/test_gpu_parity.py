"""GPU parity: every stage of the device step against the CPU oracle.

Tolerances (f32 compute):
  broad phase   bit-exact pair lists (the reference's brute-force contract)
  narrow phase  identical point counts; positions / normals / depths within 1e-5
  solver        the oracle solves the same rows in the GPU's colour order; body
                velocities within 1e-5 relative (atol 1e-6)
  world step    rollouts from a shared start within 1e-4 .. 2e-3 (last-ulp
                differences of sin/cos/acos compound over many steps); the
                per-step 1e-5 contract is in test_gpu_lockstep.py
"""
import math

import numpy as np
import pytest

import oracle_api as orc
from test_oracle_kats import ref_scattered_boxes

pytestmark = pytest.mark.gpu


def _pairs_equal(a, b):
    a = np.asarray(a, dtype=np.uint32).reshape(-1, 2)
    b = np.asarray(b, dtype=np.uint32).reshape(-1, 2)
    assert a.shape == b.shape, f"{a.shape} vs {b.shape}"
    np.testing.assert_array_equal(a, b)


# ------------------------------------------------------------------ broad phase
def test_broadphase_reference_recipe(gpu):
    a = ref_scattered_boxes(0x9E3779B97F4A7C15, 64, 1000, 100)
    _pairs_equal(gpu.broadphase_pairs(a), orc.oracle_pairs(a, 0))


@pytest.mark.parametrize("seed", range(4))
def test_broadphase_dense_sets(gpu, seed):
    a = ref_scattered_boxes(0xDB4E7F4A7C150001 ^ ((seed * 0x517CC1B727220A95) & 0xFFFFFFFFFFFFFFFF), 2048, 300, 300)
    _pairs_equal(gpu.broadphase_pairs(a), orc.oracle_pairs(a, 0))


def test_broadphase_with_unbounded_proxies(gpu):
    a = ref_scattered_boxes(12345, 1000, 500, 200)
    big = np.array([[-1e30, -1e30, -1e30, 1e30, 1e30, 1e30]], dtype=np.float32)
    a = np.concatenate([big, a[:400], big, a[400:]], axis=0)
    _pairs_equal(gpu.broadphase_pairs(a), orc.oracle_pairs(a, 1))


def test_broadphase_edge_cases(gpu):
    assert len(gpu.broadphase_pairs(np.zeros((0, 6), dtype=np.float32))) == 0
    assert len(gpu.broadphase_pairs([[0, 0, 0, 1, 1, 1]])) == 0
    touching = np.array([[0, 0, 0, 1, 1, 1], [1, 0, 0, 2, 1, 1], [2, 1, 1, 3, 2, 2], [5, 5, 5, 6, 6, 6]], np.float32)
    _pairs_equal(gpu.broadphase_pairs(touching), orc.oracle_pairs(touching, 0))
    same = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (300, 1))  # every pair overlaps
    p = gpu.broadphase_pairs(same)
    assert len(p) == 300 * 299 // 2
    _pairs_equal(p, orc.oracle_pairs(same, 1))


def test_broadphase_pile_scale(gpu):
    import scenes

    _, pos, _ = scenes.large_pile_arrays(64, 64, 32, seed=3)
    h = 0.5 * math.sqrt(3) + 0.02
    a = np.concatenate([pos - h, pos + h], axis=1).astype(np.float32)
    _pairs_equal(gpu.broadphase_pairs(a), orc.oracle_pairs(a, 1))


# ------------------------------------------------------------------ narrow phase
def _rand_quat(rng):
    q = rng.normal(size=4)
    return q / np.linalg.norm(q)


def _narrow_case(gpu_world, oracle_world, shapes, rng, n, spread):
    sa = rng.integers(0, len(shapes), size=n)
    sb = rng.integers(0, len(shapes), size=n)
    pa = np.zeros((n, 7))
    pb = np.zeros((n, 7))
    for t in range(n):
        pa[t, :3] = rng.uniform(-0.2, 0.2, 3)
        pa[t, 3:] = _rand_quat(rng)
        pb[t, :3] = pa[t, :3] + rng.normal(size=3) * spread
        pb[t, 3:] = _rand_quat(rng)
    pa = pa.astype(np.float32).astype(np.float64)
    pb = pb.astype(np.float32).astype(np.float64)
    out, cnt = gpu_world.collide([shapes[i] for i in sa], pa, [shapes[i] for i in sb], pb)
    mismatches = []
    max_err = 0.0
    for t in range(n):
        ref = oracle_world.collide(shapes[sa[t]], pa[t], shapes[sb[t]], pb[t])
        if len(ref) != cnt[t]:
            mismatches.append((t, len(ref), int(cnt[t])))
            continue
        if len(ref):
            err = np.abs(out[t, :cnt[t]] - ref).max()
            max_err = max(max_err, float(err))
    return mismatches, max_err


@pytest.mark.parametrize("kind", ["analytic", "convex"])
def test_narrowphase_matches_oracle(gpu, kind):
    rng = np.random.default_rng(7 if kind == "analytic" else 8)
    w = gpu.World()
    o = orc.OracleWorld("f32")
    shapes = []

    def both(method, *args):
        a = getattr(w, method)(*args)
        b = getattr(o, method)(*args)
        assert a == b
        shapes.append(a)

    if kind == "analytic":
        both("box", [0.5, 0.5, 0.5])
        both("box", [0.3, 0.6, 0.2])
        both("sphere", 0.5)
        both("sphere", 0.25)
        both("plane", [0, 1, 0], 0.0)
    else:
        both("capsule", 0.3, 0.5)
        both("capsule", 0.1, 0.6)
        pts = rng.normal(size=(24, 3))
        pts = 0.45 * pts / np.linalg.norm(pts, axis=1, keepdims=True)
        both("hull", pts.astype(np.float32))
        both("box", [0.4, 0.4, 0.4])
        both("sphere", 0.35)
    mism, err = _narrow_case(w, o, shapes, rng, 3000, 0.45)
    assert not mism, f"point-count mismatches (idx, oracle, gpu): {mism[:10]} of {len(mism)}"
    assert err <= 1e-5, f"max abs error {err}"


def test_narrowphase_forced_convex_path(gpu):
    """Box / sphere pairs through GJK/EPA (convex_convex.rs KATs' route)."""
    w = gpu.World()
    o = orc.OracleWorld("f32")
    b1 = w.box([1, 1, 1]); o.box([1, 1, 1])
    s1 = w.sphere(0.5); o.sphere(0.5)
    c1 = w.capsule(0.5, 1.0); o.capsule(0.5, 1.0)
    cases = [(b1, (0, 0, 0), s1, (0, 1.3, 0)), (b1, (0, 0, 0), s1, (0, 0.6, 0)), (c1, (0, 0, 0), b1, (1.51, 0, 0)),
             (c1, (0, 0, 0), c1, (0.7, 0, 0))]
    sa = [c[0] for c in cases]
    sb = [c[2] for c in cases]
    pa = [list(c[1]) + [0, 0, 0, 1] for c in cases]
    pb = [list(c[3]) + [0, 0, 0, 1] for c in cases]
    out, cnt = w.collide(sa, pa, sb, pb, force_convex=True)
    for t in range(len(cases)):
        ref = o.convex_convex(sa[t], pa[t], sb[t], pb[t])
        assert cnt[t] == 1
        np.testing.assert_allclose(out[t, 0], ref, atol=1e-5)
    # convex_convex.rs:305-333: the deep case reports depth 0.9 at y = 0.1
    assert out[1, 0, 6] == pytest.approx(0.9, abs=1e-3) and out[1, 0, 1] == pytest.approx(0.1, abs=1e-3)


# ------------------------------------------------------------------ solver
def _solver_scene(rng, nbodies=120, ngroups=400):
    bodies = []
    for i in range(nbodies):
        static = i < 3
        bodies.append(dict(kind=("box" if i % 3 else "sphere"), pos=rng.uniform(-3, 3, 3), quat=_rand_quat(rng),
                           v=rng.normal(size=3), w=rng.normal(size=3), mass=0.0 if static else rng.uniform(0.5, 3.0),
                           mu=rng.uniform(0.2, 0.9), e=rng.uniform(0.0, 0.5)))
    contacts = []
    used = set()
    for g in range(ngroups):
        a, b = rng.choice(nbodies, size=2, replace=False)
        while (int(a), int(b)) in used:  # unique (body_a, body_b) keys: one row group each
            a, b = rng.choice(nbodies, size=2, replace=False)
        used.add((int(a), int(b)))
        n = np.array([0.0, 1.0, 0.0]) + rng.normal(size=3) * 0.3
        n /= np.linalg.norm(n)
        for k in range(int(rng.integers(1, 5))):
            p = 0.5 * (bodies[a]["pos"] + bodies[b]["pos"]) + rng.normal(size=3) * 0.2
            pen = rng.uniform(-0.01, 0.08)
            imp = rng.uniform(0.0, 0.3)
            contacts.append([a, b, *p, *n, pen, imp])
    return bodies, np.array(contacts)


def _populate(world, bodies, oracle=False):
    box = world.box([0.5, 0.4, 0.3])
    sph = world.sphere(0.45)
    for b in bodies:
        world.add_body(box if b["kind"] == "box" else sph, b["pos"].astype(np.float32).astype(np.float64),
                       quat=b["quat"].astype(np.float32).astype(np.float64),
                       linvel=b["v"].astype(np.float32).astype(np.float64),
                       angvel=b["w"].astype(np.float32).astype(np.float64), mass=b["mass"], friction=b["mu"],
                       restitution=b["e"])


@pytest.mark.parametrize("seed", [11, 12])
def test_solver_matches_oracle_in_colour_order(gpu, seed):
    rng = np.random.default_rng(seed)
    bodies, contacts = _solver_scene(rng)
    contacts = contacts.astype(np.float32).astype(np.float64)
    w = gpu.World(num_iterations=10)
    _populate(w, bodies)
    rows, keys = w.solve_contacts(contacts, 60.0)
    gpu_state = w.state()
    # Reorder the caller's row groups into the GPU's solve order for the oracle.
    groups = []
    i = 0
    while i < len(contacts):
        j = i
        while j < len(contacts) and contacts[j, 0] == contacts[i, 0] and contacts[j, 1] == contacts[i, 1] and j - i < 4:
            j += 1
        groups.append(contacts[i:j])
        i = j
    key_of = [(int(g[0, 0]) << 32) | int(g[0, 1]) for g in groups]
    rank = {}
    for r, k in enumerate(keys[:len(groups)]):
        rank.setdefault(int(k), []).append(r)
    order = sorted(range(len(groups)), key=lambda gi: rank[key_of[gi]].pop(0))
    ordered = np.concatenate([groups[gi] for gi in order], axis=0)
    o = orc.OracleWorld("f32")
    o.set_solver(num_iterations=10)
    _populate(o, bodies)
    ref_rows = o.solve_contacts(ordered, 60.0)
    ref_state = o.state()
    np.testing.assert_allclose(gpu_state[:, 7:13], ref_state[:, 7:13], rtol=1e-5, atol=1e-6)
    # impulses row by row (GPU rows come back in the same order)
    np.testing.assert_allclose(rows[:, 13:16], ref_rows[:, 13:16], rtol=1e-5, atol=1e-6)
    push = w.push()
    np.testing.assert_allclose(push, o.push(), rtol=1e-5, atol=1e-6)
    # every colour batch is conflict-free: recorded by bit-identical results above


# ------------------------------------------------------------------ world step
def _run_pair(scene, steps, tol, check_every=1):
    import bgpu
    import scenes

    w = scene.build_gpu(bgpu)
    o = scene.build_oracle(orc)
    worst = 0.0
    for s in range(steps):
        w.step(scene.dt)
        order = w.solve_order()
        o.set_solve_order(order)
        o.step(scene.dt)
        st = w.stats()
        assert st["device_status"] == 0, st
        if s % check_every == 0 or s == steps - 1:
            g = w.state()
            r = o.state()
            np.testing.assert_array_equal(g[:, 13], r[:, 13])  # activation states
            err = np.abs(g[:, :13] - r[:, :13]).max()
            worst = max(worst, float(err))
            assert err <= tol, f"step {s}: max abs state error {err}"
            _pairs_equal(w.pairs(), o.pairs())
    return worst


def test_world_falling_box_matches_oracle(gpu):
    import scenes

    s = scenes.Scene("one_box", 1 / 60, 10, 150)
    p = s.add_shape(scenes.PLANE, [0, 1, 0, 0])
    b = s.add_shape(scenes.BOX, [0.5, 0.5, 0.5])
    s.add(p, (0, 0, 0), mass=0.0)
    s.add(b, (0.0, 2.0, 0.0), (0.05, 0.02, 0.01, 0.998), mass=1.0)
    _run_pair(s, 150, 1e-4)


def test_world_small_stack_matches_oracle(gpu):
    import scenes

    s = scenes.falling_box_stack(3, 3, 3, seed=5, steps=90)
    _run_pair(s, 90, 2e-3, check_every=10)


def test_world_mixed_convex_pile_matches_oracle(gpu):
    """Config 2 recipe at small scale (boxes, spheres, capsules, 24-point hulls): the world step
    with GJK/EPA manifolds against the oracle, the oracle taking the device state before every
    step; state within 1e-5 relative and pairs bit-exact after every step. (Windows of several
    steps without that copy are not comparable here: a last-ulp sin/cos difference can flip a
    contact decision of a tumbling hull and the trajectories part.)"""
    import bgpu
    import scenes

    s = scenes.mixed_convex_pile(n=96, seed=21, steps=90, extent=6.0)
    w = s.build_gpu(bgpu)
    o = s.build_oracle(orc)
    convex_pairs = 0
    for step in range(90):
        o.set_state(w.state().astype(np.float64))
        w.step(s.dt)
        o.set_solve_order(w.solve_order())
        o.step(s.dt)
        st = w.stats()
        assert st["device_status"] == 0, st
        convex_pairs = max(convex_pairs, st["num_detect"])
        g = w.state()
        r = o.state()
        np.testing.assert_array_equal(g[:, 13], r[:, 13])
        np.testing.assert_allclose(g[:, :13], r[:, :13], rtol=1e-5, atol=1e-6, err_msg=f"step {step}")
        _pairs_equal(w.pairs(), o.pairs())
    assert convex_pairs > 0


def test_world_sleeping_chain_wakes_like_the_oracle(gpu):
    """Islands: a chain of touching boxes settles and falls asleep as one island, a lone box
    sleeps on its own, and a box dropped onto the chain's end (landing after the chain slept)
    wakes the whole chain but not the lone box. Activation states equal the oracle's at every
    step; the rest of the state within 1e-3."""
    import bgpu
    import scenes

    s = scenes.Scene("sleeping_chain", 1 / 120, 10, 420)
    p = s.add_shape(scenes.PLANE, [0, 1, 0, 0])
    b = s.add_shape(scenes.BOX, [0.5, 0.5, 0.5])
    s.add(p, (0, 0, 0), mass=0.0)
    chain = list(range(1, 6))
    for k in range(5):
        s.add(b, (1.0 * k, 0.5, 0.0))
    lone = 6
    s.add(b, (10.0, 0.5, 0.0))
    drop = 7
    s.add(b, (4.0, 40.0, 0.0))
    w = s.build_gpu(bgpu)
    o = s.build_oracle(orc)
    history = []
    for step in range(s.steps):
        w.step(s.dt)
        o.set_solve_order(w.solve_order())
        o.step(s.dt)
        assert w.stats()["device_status"] == 0
        g, r = w.state(), o.state()
        np.testing.assert_array_equal(g[:, 13], r[:, 13], err_msg=f"step {step}")
        err = float(np.abs(g[:, :13] - r[:, :13]).max())
        assert err <= 1e-3, f"step {step}: max abs state error {err}"
        history.append(g[:, 13].copy())
    h = np.array(history)
    asleep = h[:, chain] == 2
    slept = np.flatnonzero(asleep.all(axis=1))
    assert len(slept) > 0, "the chain never slept"
    assert not asleep[-1].any(), "the dropped box did not wake the chain"
    assert h[-1, lone] == 2 and h[slept[0]:, lone].min() == 2
    assert h[slept[0], drop] != 2  # still falling while the chain slept


def test_colour_batches_cover_every_row_group(gpu):
    import bgpu
    import scenes

    s = scenes.falling_box_stack(4, 4, 4, seed=6, steps=40)
    w = s.build_gpu(bgpu)
    w.step(s.dt, 40)
    st = w.stats()
    groups, split = w.colour_batches()
    assert len(groups) == st["num_colours"] > 0
    assert int(groups.sum()) == st["num_contact_pairs"]
    assert int(split.sum()) == st["num_split_pairs"]
    assert np.all(groups > 0) and np.all(split <= groups)


def test_device_wait_gives_up_with_an_error_status(gpu):
    """A solver team barrier that nothing completes ends after its time limit with
    BGPU_DEVSTAT_BARRIER_TIMEOUT (0x4) in the status word, and the context stays usable."""
    import scenes

    status, ms = gpu.selftest_wait_timeout(50)
    assert status & 0x4, status
    assert 45.0 <= ms < 2000.0, ms
    s = scenes.falling_box_stack(2, 2, 2, seed=1, steps=5)
    w = s.build_gpu(gpu)
    w.step(s.dt, 5)
    assert w.stats()["device_status"] == 0
    with pytest.raises(gpu.BgpuError):
        gpu.selftest_wait_timeout(0)
