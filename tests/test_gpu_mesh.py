"""GPU parity for static triangle meshes and heightfields.

  narrow phase  convex (box, sphere, capsule, 24-point hull) against a wavy
                mesh and against heightfields with every diagonal / winding /
                up-axis option, in both pair orders: identical point counts,
                positions / normals / depths within 1e-5 of the oracle
                (narrowphase/convex_mesh.rs:26-153, manifold.rs:80-108)
  world step    the reference's rain_500 perf scene (mixed convex raining
                onto a wavy terrain mesh) in lockstep with the oracle: pairs
                bit-exact, the state within 1e-5 relative after every step
  CCD           fast CCD spheres onto a heightfield: the clamp fractions of
                every step equal the oracle's (convex_sweep.rs:305-345)
"""
import numpy as np
import pytest

import oracle_api as orc

pytestmark = pytest.mark.gpu


def _rand_quat(rng):
    q = rng.normal(size=4)
    return q / np.linalg.norm(q)


def _shapes(w, o, rng):
    """The same shape list in both worlds; returns (convex ids, mesh ids)."""
    import scenes

    ids = []

    def both(method, *args):
        a = getattr(w, method)(*args)
        b = getattr(o, method)(*args)
        assert a == b
        ids.append(a)
        return a

    convex = [both("box", [0.4, 0.3, 0.5]), both("sphere", 0.35), both("capsule", 0.3, 0.5)]
    pts = rng.normal(size=(24, 3))
    pts = (0.45 * pts / np.linalg.norm(pts, axis=1, keepdims=True)).astype(np.float32)
    convex.append(both("hull", pts))
    v, idx = scenes.wavy_grid_mesh(12, 12, (-5.5, -5.5), (1.0, 1.0), 0.4, 0.7, 0.6)
    meshes = [both("mesh", v, idx)]
    x, z = np.meshgrid(np.arange(9), np.arange(9))
    h = (0.5 * np.sin(0.9 * x) * np.cos(0.8 * z)).astype(np.float32).ravel()
    for opt in (0, 1, 2, 4, 8, 16, 32):
        meshes.append(both("heightfield", h, 9, 9, (0.8, 1.0, 0.7), opt))
    return convex, meshes


def test_mesh_narrowphase_matches_oracle(gpu):
    rng = np.random.default_rng(31)
    w = gpu.World()
    o = orc.OracleWorld("f32")
    convex, meshes = _shapes(w, o, rng)
    n = 3000
    sa, sb, pa, pb = [], [], np.zeros((n, 7)), np.zeros((n, 7))
    for t in range(n):
        c = convex[rng.integers(len(convex))]
        m = meshes[rng.integers(len(meshes))]
        mpose = np.concatenate([rng.uniform(-0.3, 0.3, 3), _rand_quat(rng) if rng.random() < 0.3 else [0, 0, 0, 1]])
        cpose = np.concatenate([mpose[:3] + [rng.uniform(-3, 3), rng.uniform(-0.9, 0.9), rng.uniform(-3, 3)],
                                _rand_quat(rng)])
        if rng.random() < 0.5:
            sa.append(c), sb.append(m)
            pa[t], pb[t] = cpose, mpose
        else:
            sa.append(m), sb.append(c)
            pa[t], pb[t] = mpose, cpose
    pa = pa.astype(np.float32).astype(np.float64)
    pb = pb.astype(np.float32).astype(np.float64)
    out, cnt = w.collide(sa, pa, sb, pb)
    mism, worst, touching = [], 0.0, 0
    for t in range(n):
        ref = o.collide(sa[t], pa[t], sb[t], pb[t])
        if len(ref) != cnt[t]:
            mism.append((t, len(ref), int(cnt[t])))
            continue
        if len(ref):
            touching += 1
            worst = max(worst, float(np.abs(out[t, :cnt[t]] - ref).max()))
    assert not mism, f"point-count mismatches (idx, oracle, gpu): {mism[:10]} of {len(mism)}"
    assert touching > n // 5
    assert worst <= 1e-5, worst
    assert w.stats()["device_status"] == 0


def test_mesh_rain_lockstep(gpu):
    """The rain_500 perf scene (500 boxes, spheres and capsules onto a 20 x 20 terrain mesh), 180
    steps: the oracle takes the device state before every step and the device's colour order."""
    import scenes

    s = scenes.mesh_rain(steps=180)
    w = s.build_gpu(gpu)
    o = s.build_oracle(orc)
    for step in range(s.steps):
        o.set_state(w.state().astype(np.float64))
        w.step(s.dt)
        o.set_solve_order(w.solve_order())
        o.step(s.dt)
        st = w.stats()
        assert st["device_status"] == 0, st
        g, r = w.state(), o.state()
        np.testing.assert_array_equal(g[:, 13], r[:, 13])
        np.testing.assert_allclose(g[:, :13], r[:, :13], rtol=1e-5, atol=1e-6, err_msg=f"step {step}")
        np.testing.assert_array_equal(w.pairs(), o.pairs())
    assert st["num_contacts"] > 500


def test_ccd_spheres_onto_a_heightfield(gpu):
    """Fast spheres with CCD settings dropped onto a heightfield: per-step clamp fractions equal
    the oracle's sweep_mesh (one BVH walk per CCD body and target mesh)."""
    import scenes

    s = scenes.Scene("ccd_terrain", 1.0 / 60.0, 10, 40)
    x, z = np.meshgrid(np.arange(10), np.arange(10))
    h = (0.3 * np.sin(0.8 * x) * np.cos(0.7 * z)).ravel()
    hf = s.add_heightfield(h, 10, 10, (1.0, 1.0, 1.0))
    sph = s.add_shape(scenes.SPHERE, [0.2])
    s.add(hf, (0.0, 0.0, 0.0), mass=0.0)
    rng = np.random.default_rng(3)
    for k in range(24):
        p = (rng.uniform(-3.5, 3.5), rng.uniform(2.0, 6.0), rng.uniform(-3.5, 3.5))
        s.add(sph, p, mass=1.0, linvel=(rng.uniform(-5, 5), -rng.uniform(80, 200), rng.uniform(-5, 5)))
    w = s.build_gpu(gpu)
    o = s.build_oracle(orc)
    ids = list(range(1, s.num_bodies))
    w.set_ccd(1, np.full(len(ids), 0.05), np.full(len(ids), 0.2))
    for i in ids:
        o.set_ccd(i, 0.05, 0.2)
    clamped = 0
    for step in range(s.steps):
        o.set_state(w.state().astype(np.float64))
        w.step(s.dt)
        o.set_solve_order(w.solve_order())
        o.step(s.dt)
        assert w.stats()["device_status"] == 0
        gc, rc = w.ccd_clamps()[ids], o.ccd_clamps()[ids]
        np.testing.assert_allclose(gc, rc, rtol=1e-5, atol=1e-6, err_msg=f"step {step}")
        clamped += int(np.count_nonzero(gc < 1.0))
        g, r = w.state(), o.state()
        np.testing.assert_allclose(g[:, :13], r[:, :13], rtol=1e-5, atol=1e-6, err_msg=f"step {step}")
    assert clamped > 0


def test_mesh_bodies_must_be_static(gpu):
    w = gpu.World()
    m = w.heightfield(np.zeros(16), 4, 4)
    with pytest.raises(gpu.BgpuError):
        w.add_body(m, (0, 0, 0), mass=1.0)
    w.add_body(m, (0, 0, 0), mass=0.0)
    with pytest.raises(gpu.BgpuError):
        w.mesh(np.zeros((3, 3)), [[0, 1, 5]])
