"""Batched worlds against the oracle, world by world.

A batch steps many independent worlds through one sequence of launches. Each
world of the batch must evolve exactly like that world stepped alone: the
oracle steps every world on its own, fed the batch's solve order restricted to
that world's pairs (the colouring of the batch is global, so its order inside
one world differs from a world coloured alone, and the oracle's sequential
solve has to take the same order to match).
"""
import numpy as np
import pytest

import oracle_api as orc

gpu_only = pytest.mark.gpu


def _world_order(order, lo, hi):
    a = (order >> np.uint64(32)).astype(np.int64)
    b = (order & np.uint64(0xFFFFFFFF)).astype(np.int64)
    sel = (a >= lo) & (a < hi)
    return ((a[sel] - lo).astype(np.uint64) << np.uint64(32)) | (b[sel] - lo).astype(np.uint64)


def _world_pairs(pairs, lo, hi):
    sel = (pairs[:, 0] >= lo) & (pairs[:, 0] < hi)
    return pairs[sel] - lo


def _mixed_batch():
    import scenes

    b = scenes.batched_worlds(n_worlds=10, seed=11, steps=150, min_bodies=8, max_bodies=40)
    plane, box = 0, 1
    # A box at rest on the ground (it falls asleep after 2 s) and one dropped from 25 m
    # (still falling then): their worlds' simulate / prune flags must stay apart.
    b.add_world([plane, box], [[0, 0, 0], [0, 0.5, 0]], [[0, 0, 0, 1], [0, 0, 0, 1]], [0.0, 1.0])
    b.add_world([plane, box], [[0, 0, 0], [0, 25.0, 0]], [[0, 0, 0, 1], [0, 0, 0, 1]], [0.0, 1.0])
    return b


@gpu_only
def test_batch_worlds_match_the_oracle_world_by_world(gpu):
    """Windows of 10 steps from a shared state: every world stays within 1e-3 of its
    oracle (the oracle takes the batch's body state at the start of each window, so
    last-ulp differences of sin/cos/pow cannot compound chaotically over the run)."""
    b = _mixed_batch()
    w = b.build_gpu(gpu)
    off = w.world_offsets()
    assert list(np.diff(off)) == list(b.bodies_per_world)
    oracles = [b.world_scene(k).build_oracle(orc) for k in range(len(b.worlds))]
    for step in range(150):
        if step % 10 == 0:
            g = w.state()
            for k, o in enumerate(oracles):
                o.set_state(g[int(off[k]):int(off[k + 1])].astype(np.float64))
        w.step(b.dt)
        st = w.stats()
        assert st["device_status"] == 0, st
        order = w.solve_order()
        for k, o in enumerate(oracles):
            o.set_solve_order(_world_order(order, int(off[k]), int(off[k + 1])))
            o.step(b.dt)
        if step % 10 == 9:
            g = w.state()
            pairs = w.pairs()
            for k, o in enumerate(oracles):
                lo, hi = int(off[k]), int(off[k + 1])
                r = o.state()
                np.testing.assert_array_equal(g[lo:hi, 13], r[:, 13])
                err = float(np.abs(g[lo:hi, :13] - r[:, :13]).max())
                assert err <= 1e-3, f"step {step} world {k}: {err}"
                np.testing.assert_array_equal(_world_pairs(pairs, lo, hi), o.pairs())
    # the resting box sleeps, the dropped one does not
    g = w.state()
    rest, drop = int(off[10]) + 1, int(off[11]) + 1
    assert g[rest, 13] == 2 and g[drop, 13] != 2


@gpu_only
def test_batch_pairs_never_cross_worlds(gpu):
    """Worlds share one origin, so every body overlaps bodies of other worlds in space."""
    import scenes

    b = scenes.batched_worlds(n_worlds=64, seed=5, steps=1, min_bodies=8, max_bodies=64)
    w = b.build_gpu(gpu)
    off = w.world_offsets().astype(np.int64)
    w.step(b.dt)
    pairs = w.pairs().astype(np.int64)
    world_a = np.searchsorted(off, pairs[:, 0], side="right") - 1
    world_b = np.searchsorted(off, pairs[:, 1], side="right") - 1
    assert len(pairs) > 0
    np.testing.assert_array_equal(world_a, world_b)
    key = pairs[:, 0] * (1 << 32) + pairs[:, 1]
    assert np.all(np.diff(key) > 0)
    # each world's pair set equals the oracle brute force on that world's AABBs
    for k in range(len(b.worlds)):
        o = b.world_scene(k).build_oracle(orc)
        o.set_brute_force(True)
        o.step(b.dt)
        np.testing.assert_array_equal(pairs[(world_a == k)] - off[k], o.pairs())


@gpu_only
def test_batch_pairs_of_crowded_proxies(gpu):
    """Proxies with more than 32 partners j > i (the ground plane and large static boxes among
    small spheres) take the broad phase's second, ballot-ranked write pass. The large boxes sit
    at several positions of a world, two of them in one 64-proxy tile and one in the next, so
    a tile holds several such proxies. Every world's pairs must equal the oracle's brute force
    on that world, in ascending order."""
    import scenes

    rng = np.random.default_rng(21)
    b = scenes.BatchScene("crowded_proxies", 1.0 / 60.0, 10, 1)
    plane = b.add_shape(scenes.PLANE, [0.0, 1.0, 0.0, 0.0])
    big = b.add_shape(scenes.BOX, [2.0, 2.0, 2.0])
    ball = b.add_shape(scenes.SPHERE, [0.2])
    for k in range(6):
        ns = 110 + 10 * k  # at least 40 spheres after the last big box
        at = sorted({3 + k, 20 + 2 * k, 66 + k})  # the big boxes' indices in the world
        n = 1 + ns + len(at)
        shape = np.full(n, ball)
        shape[0] = plane
        shape[at] = big
        pos = rng.uniform(-2.0, 2.0, size=(n, 3)) + np.array([0.0, 3.0, 0.0])
        pos[0] = 0.0
        pos[at] = rng.uniform(-0.3, 0.3, size=(len(at), 3)) + np.array([0.0, 3.0, 0.0])
        mass = np.ones(n)
        mass[0] = 0.0
        mass[at] = 0.0
        b.add_world(shape, pos, np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1)), mass)
    w = b.build_gpu(gpu)
    off = w.world_offsets().astype(np.int64)
    w.step(b.dt)
    assert w.stats()["device_status"] == 0
    pairs = w.pairs().astype(np.int64)
    key = pairs[:, 0] * (1 << 32) + pairs[:, 1]
    assert np.all(np.diff(key) > 0)
    for k in range(len(b.worlds)):
        lo = off[k]
        mine = pairs[(pairs[:, 0] >= lo) & (pairs[:, 0] < off[k + 1])] - lo
        crowded = np.bincount(mine[:, 0], minlength=int(off[k + 1] - lo))
        assert (crowded > 32).sum() >= 4  # the plane and the three boxes
        o = b.world_scene(k).build_oracle(orc)
        o.set_brute_force(True)
        o.step(b.dt)
        np.testing.assert_array_equal(mine, o.pairs())


@gpu_only
def test_batch_rejects_plain_body_insertion(gpu):
    import bgpu

    w = bgpu.World(batch=True)
    box = w.box([0.5, 0.5, 0.5])
    with pytest.raises(bgpu.BgpuError):
        w.add_body(box, (0, 1, 0))
    plain = bgpu.World()
    with pytest.raises(bgpu.BgpuError):
        plain.add_worlds_array([1], [box], [[0, 1, 0]], [[0, 0, 0, 1]], mass=[1.0])


def test_batched_worlds_recipe():
    import scenes

    b = scenes.batched_worlds(n_worlds=256, seed=4)
    n = b.bodies_per_world - 1
    assert n.min() >= 8 and n.max() <= 255
    assert all(w["mass"][0] == 0.0 and w["shape"][0] == 0 for w in b.worlds)
    assert b.num_dynamic == int(n.sum())
    s = b.world_scene(7)
    assert s.num_bodies == int(b.bodies_per_world[7])


def _lockstep_batch(w, b, steps, oracles=None):
    """Per-step parity of every world against its own oracle (state copied in before each step;
    the oracles must have stepped alongside the device world from the start, so that both hold
    the same manifold caches). Returns the oracles."""
    off = w.world_offsets().astype(np.int64)
    if oracles is None:
        oracles = [b.world_scene(k).build_oracle(orc) for k in range(len(b.worlds))]
    for step in range(steps):
        g0 = w.state()
        for k, o in enumerate(oracles):
            o.set_state(g0[off[k]:off[k + 1]].astype(np.float64))
        w.step(b.dt)
        st = w.stats()
        assert st["device_status"] == 0, st
        order = w.solve_order()
        g = w.state()
        pairs = w.pairs().astype(np.int64)
        for k, o in enumerate(oracles):
            lo, hi = int(off[k]), int(off[k + 1])
            o.set_solve_order(_world_order(order, lo, hi))
            o.step(b.dt)
            r = o.state()
            np.testing.assert_array_equal(g[lo:hi, 13], r[:, 13])
            np.testing.assert_allclose(g[lo:hi, :13], r[:, :13], rtol=1e-5, atol=1e-6,
                                       err_msg=f"step {step} world {k}")
            sel = (pairs[:, 0] >= lo) & (pairs[:, 0] < hi)
            np.testing.assert_array_equal(pairs[sel] - lo, o.pairs())
    return oracles


@gpu_only
@pytest.mark.parametrize("threads,warp_max", [(0, 0), (32, 1 << 30), (64, 32), (128, 64), (256, 0)])
def test_batch_solver_launch_shapes_match_the_oracle(gpu, threads, warp_max):
    """Every launch shape of the batch solver (the global solver; one world per warp; worlds
    split between warps and whole CTAs; one world per CTA) solves each world in an order the
    oracle replays to 1e-5 after every step."""
    import scenes

    b = scenes.batched_worlds(n_worlds=24, seed=13, steps=40, min_bodies=8, max_bodies=160)
    w = b.build_gpu(gpu)
    w.set_tuning(threads, warp_max)
    t = w.tuning()
    assert t["threads_per_cta"] == threads
    assert (t["ctas"] > 0) == (threads > 0)
    _lockstep_batch(w, b, 40)


@gpu_only
def test_batch_autotune_keeps_the_state_and_the_parity(gpu):
    """The autotuner times every launch shape from one checkpoint and puts the batch back:
    the state after tuning equals the state before, and stepping goes on in parity."""
    import scenes

    b = scenes.batched_worlds(n_worlds=48, seed=17, steps=30, min_bodies=8, max_bodies=200)
    w = b.build_gpu(gpu)
    oracles = _lockstep_batch(w, b, 20)
    before = w.state()
    t = w.autotune(b.dt, 2)
    np.testing.assert_array_equal(w.state(), before)
    assert t["candidates"] >= 2 and t["ms_per_step"] > 0.0 and t["global_ms_per_step"] > 0.0
    assert t["threads_per_cta"] in (0, 32, 64, 128, 256)
    assert t["ms_per_step"] <= t["global_ms_per_step"] * 1.0001
    _lockstep_batch(w, b, 10, oracles)  # the manifold caches came back with the state


@gpu_only
def test_batch_set_tuning_rejects_bad_shapes(gpu):
    import bgpu
    import scenes

    b = scenes.batched_worlds(n_worlds=4, seed=1, steps=1)
    w = b.build_gpu(gpu)
    for bad in (16, 48, 512):
        with pytest.raises(bgpu.BgpuError):
            w.set_tuning(bad, 64)
    plain = bgpu.World()
    with pytest.raises(bgpu.BgpuError):
        plain.set_tuning(128, 64)
