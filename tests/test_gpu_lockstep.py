"""Per-step world parity at the benchmark configurations' sizes.

The device world and the oracle step side by side. Before every step the
oracle takes the device's body state (pose, velocities, activation state,
deactivation timer) and, for the step's solve, the device's colour order of
the row groups. Each step therefore starts from an identical state, and the
manifold caches stay identical too: a cache is built from the predicted poses
of the step's start, before the pose integration that carries the only
non-bit-exact arithmetic of the step (sinf / cosf of the exponential-map
rotation, interpolate_pose body.rs:92-137, where the device's and the host
libm's results may differ in the last ulp; the redetect rotation gate's acosf,
manifold.rs:158-160, and damping's powf, body.rs:1066-1111, have the same
allowance but see no damping in these scenes).

After every step:
  pairs             bit-exact (the broad-phase contract)
  activation state  equal
  velocities        within 1e-5 relative (atol 1e-6) of the reference solver
                    run in the same colour order (sequential_impulse.rs:692-735)
  pose              within 1e-5 relative (atol 1e-6): one step's sin/cos ulps
Scenes: the 1,000-box stack at full size (300 steps), a 8,192-body slice of
the 131,072-body pile (settle and measure, 300 steps), 256 worlds of the
4,096-world batch and a 1,024-body slice of the mixed convex pile.
"""
import numpy as np
import pytest

import oracle_api as orc

pytestmark = pytest.mark.gpu

RTOL = 1e-5
ATOL = 1e-6


def _check(g, r, step, tag=""):
    np.testing.assert_array_equal(g[:, 13], r[:, 13], err_msg=f"{tag} step {step}: activation states")
    np.testing.assert_allclose(g[:, 7:13], r[:, 7:13], rtol=RTOL, atol=ATOL,
                               err_msg=f"{tag} step {step}: velocities")
    np.testing.assert_allclose(g[:, 0:7], r[:, 0:7], rtol=RTOL, atol=ATOL, err_msg=f"{tag} step {step}: poses")
    np.testing.assert_allclose(g[:, 14], r[:, 14], rtol=RTOL, atol=ATOL,
                               err_msg=f"{tag} step {step}: deactivation timers")


def _vel_stats(g, r):
    d = np.abs(g[:, 7:13].astype(np.float64) - r[:, 7:13])
    exact = int(np.count_nonzero(d == 0.0))
    return float(d.max()) if d.size else 0.0, exact, d.size


def lockstep(w, o, dt, steps, tag=""):
    """Step the device world and the oracle from the same state every step; returns the
    largest velocity difference seen and the share of bit-identical velocity components."""
    worst, exact, total = 0.0, 0, 0
    for s in range(steps):
        o.set_state(w.state().astype(np.float64))
        w.step(dt)
        o.set_solve_order(w.solve_order())
        o.step(dt)
        st = w.stats()
        assert st["device_status"] == 0, st
        g, r = w.state(), o.state()
        _check(g, r, s, tag)
        np.testing.assert_array_equal(w.pairs(), o.pairs(), err_msg=f"{tag} step {s}: pairs")
        m, e, t = _vel_stats(g, r)
        worst, exact, total = max(worst, m), exact + e, total + t
    return worst, exact / max(total, 1)


def test_world_single_step_from_identical_state(gpu):
    """A 4x4x4 pile settles for 40 steps in lockstep (the oracle takes the device state before
    each step, so both hold the same manifold cache), then one more step starts from a state
    copied from the device: the whole post-step state within 1e-5 relative, pairs and
    contacts identical."""
    import scenes

    s = scenes.large_pile_fast(4, 4, 4, seed=9, steps=41)
    w = s.build_gpu(gpu)
    o = s.build_oracle(orc)
    lockstep(w, o, s.dt, 40, "settle")
    o.set_state(w.state().astype(np.float64))
    w.step(s.dt)
    o.set_solve_order(w.solve_order())
    o.step(s.dt)
    g, r = w.state(), o.state()
    _check(g, r, 40, "single")
    np.testing.assert_array_equal(w.pairs(), o.pairs())
    rows = w.contacts()
    ref = o.rows()
    assert rows.shape[0] == ref.shape[0] > 0
    assert w.stats()["device_status"] == 0


def test_lockstep_falling_box_stack_full_size(gpu):
    """The 1,000-box stack at full size, every one of its 300 steps."""
    import scenes

    s = scenes.falling_box_stack(10, 10, 10, seed=1, steps=300)
    w = s.build_gpu(gpu)
    o = s.build_oracle(orc)
    worst, exact = lockstep(w, o, s.dt, s.steps, "C1")
    assert w.stats()["num_contacts"] > 1000
    print(f"C1 lockstep: max |dv| {worst:.3e}, bit-identical velocity components {exact:.4f}")


def test_lockstep_large_pile_slice(gpu):
    """An 8,192-body slice of the large pile (16x16 columns of the full pile's 32 layers, same
    recipe): 240 settle steps then 60 more, all in lockstep and all checked."""
    import scenes

    s = scenes.large_pile_fast(16, 16, 32, seed=3, steps=300)
    w = s.build_gpu(gpu)
    o = s.build_oracle(orc)
    worst, exact = lockstep(w, o, s.dt, s.steps, "C3 slice")
    st = w.stats()
    assert st["num_contacts"] > 2 * s.num_dynamic  # a dense settled pile
    print(f"C3 slice lockstep: max |dv| {worst:.3e}, bit-identical {exact:.4f}, contacts {st['num_contacts']}")


def test_lockstep_mixed_convex_slice(gpu):
    """1,024 bodies of the mixed convex recipe (boxes, spheres, capsules, 24-point hulls; the
    GJK/EPA path) in a 13 m cube, 150 steps."""
    import scenes

    s = scenes.mixed_convex_pile(n=1024, seed=2, steps=150, extent=13.0)
    w = s.build_gpu(gpu)
    o = s.build_oracle(orc)
    worst, exact = lockstep(w, o, s.dt, s.steps, "C2 slice")
    assert w.stats()["num_detect"] > 0
    print(f"C2 slice lockstep: max |dv| {worst:.3e}, bit-identical {exact:.4f}")


def _world_order(order, lo, hi):
    a = (order >> np.uint64(32)).astype(np.int64)
    b = (order & np.uint64(0xFFFFFFFF)).astype(np.int64)
    sel = (a >= lo) & (a < hi)
    return ((a[sel] - lo).astype(np.uint64) << np.uint64(32)) | (b[sel] - lo).astype(np.uint64)


def test_lockstep_batched_worlds_slice(gpu):
    """256 worlds of the batched-worlds recipe (8-255 bodies each), 120 steps: every world
    against its own oracle fed the batch's order restricted to that world."""
    import scenes

    b = scenes.batched_worlds(n_worlds=256, seed=4, steps=120)
    w = b.build_gpu(gpu)
    off = w.world_offsets().astype(np.int64)
    oracles = [b.world_scene(k).build_oracle(orc) for k in range(len(b.worlds))]
    for step in range(b.steps):
        g0 = w.state()
        for k, o in enumerate(oracles):
            o.set_state(g0[off[k]:off[k + 1]].astype(np.float64))
        w.step(b.dt)
        st = w.stats()
        assert st["device_status"] == 0, st
        order = w.solve_order()
        pairs = w.pairs().astype(np.int64)
        g = w.state()
        for k, o in enumerate(oracles):
            lo, hi = int(off[k]), int(off[k + 1])
            o.set_solve_order(_world_order(order, lo, hi))
            o.step(b.dt)
            _check(g[lo:hi], o.state(), step, f"world {k}")
            sel = (pairs[:, 0] >= lo) & (pairs[:, 0] < hi)
            np.testing.assert_array_equal(pairs[sel] - lo, o.pairs(), err_msg=f"world {k} step {step}")
