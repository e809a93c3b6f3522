"""Oracle pins for static triangle meshes and heightfields.

Restates the assertions of the reference's own inline tests, in both
precisions: shapes/triangle_mesh.rs (local AABB, BVH candidate query),
shapes/heightfield.rs (centring, midpoint offset, up axes, the four quad
diagonal rules, winding flip, vertex layout) and narrowphase/convex_mesh.rs
(sphere resting on a mesh, the sphere detector against GJK/EPA on the
triangle hull, edge / vertex / band / back-face semantics, separation, a box
on a heightfield, reduction to four points). The internal-edge seam test
(convex_mesh.rs seam_contact_normal_snaps_with_edge_info) needs the
triangle-info map, which this build does not restate (the map is off unless a
caller generates it), and the ray-cast tests belong to ray queries, which are
not on the step.
"""
import numpy as np
import pytest

import oracle_api as orc

PREC = ["f32", "f64"]
IDENT = [0, 0, 0, 1]


def pose(p, q=IDENT):
    return list(p) + list(q)


def flat_ground(o):
    return o.mesh([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1]], [[0, 1, 2], [0, 2, 3]])


def local_aabb(o, s):
    return o.world_aabb(s, pose([0, 0, 0]))


@pytest.mark.parametrize("prec", PREC)
def test_mesh_local_aabb_and_candidate_query(prec):
    """triangle_mesh.rs local_aabb_covers_the_vertices, aabb_query_finds_touching_triangles."""
    o = orc.OracleWorld(prec)
    m = flat_ground(o)
    a = local_aabb(o, m)
    assert a[0] == pytest.approx(0.0) and a[4] == pytest.approx(0.0) and a[5] == pytest.approx(1.0)
    hits = o.mesh_query(m, [0.8, -1.0, 0.8, 1.2, 1.0, 1.2])
    assert 1 in hits and len(hits) == 2


@pytest.mark.parametrize("prec", PREC)
def test_mesh_bvh_query_equals_brute_force(prec):
    """The BVH walk returns exactly the triangles whose leaf boxes it reaches; every
    triangle whose own box overlaps the query is among them (bvh.rs:45-66)."""
    rng = np.random.default_rng(5)
    o = orc.OracleWorld(prec)
    n = 24
    x, z = np.meshgrid(np.arange(n), np.arange(n))
    heights = 0.3 * np.sin(0.7 * x) * np.cos(0.6 * z)
    hf = o.heightfield(heights.ravel(), n, n, (1.0, 1.0, 1.0))
    v, idx = o.mesh_data(hf)
    tri = v[idx]
    tmin, tmax = tri.min(axis=1), tri.max(axis=1)
    for _ in range(50):
        c = rng.uniform(-12, 12, 3)
        e = rng.uniform(0.1, 3.0, 3)
        q = np.concatenate([c - e, c + e])
        hits = set(o.mesh_query(hf, q).tolist())
        truth = set(np.flatnonzero(np.all(tmin <= q[3:], axis=1) & np.all(q[:3] <= tmax, axis=1)).tolist())
        assert truth <= hits


@pytest.mark.parametrize("prec", PREC)
def test_heightfield_layout(prec):
    """heightfield.rs local_aabb_spans_the_centered_grid, heights_are_offset_by_the_midpoint,
    x_and_z_up_grids_lay_the_grid_along_the_axis, vertex_layout_matches_upstream_centering."""
    o = orc.OracleWorld(prec)
    a = local_aabb(o, o.heightfield([0, 0, 0, 0], 2, 2))
    np.testing.assert_allclose(a, [-0.5, 0, -0.5, 0.5, 0, 0.5], atol=1e-7)
    a = local_aabb(o, o.heightfield([-1, 1, -1, 1], 2, 2))
    assert a[1] == pytest.approx(-1.0) and a[4] == pytest.approx(1.0)
    ax = local_aabb(o, o.heightfield([0, 0, 1, 1], 2, 2, options=1 << 4))
    np.testing.assert_allclose(ax[[0, 3, 1, 4, 2]], [-0.5, 0.5, -0.5, 0.5, -0.5], atol=1e-7)
    az = local_aabb(o, o.heightfield([0, 0, 1, 1], 2, 2, options=2 << 4))
    np.testing.assert_allclose(az[[2, 5, 3]], [-0.5, 0.5, 0.5], atol=1e-7)
    v, idx = o.mesh_data(o.heightfield(np.arange(9.0), 3, 3))
    np.testing.assert_allclose(v[idx[0, 0]], [-1, -4, -1], atol=1e-7)
    centre = v[np.flatnonzero(v[:, 1] == 0.0)[0]]
    assert centre[0] == 0.0 and centre[2] == 0.0


def _tri_ids(o, s, t):
    v, idx = o.mesh_data(s)
    return [int(round(v[k, 1] + 4.0)) for k in idx[t]]


@pytest.mark.parametrize("prec", PREC)
def test_heightfield_diagonals_and_winding(prec):
    """heightfield.rs diagonal_options_pick_the_upstream_splits and
    flip_triangle_winding_reverses_every_triangle."""
    o = orc.OracleWorld(prec)
    h = np.arange(9.0)
    d = o.heightfield(h, 3, 3)
    assert _tri_ids(o, d, 0) == [0, 3, 1] and _tri_ids(o, d, 1) == [1, 3, 4]
    f = o.heightfield(h, 3, 3, options=1)
    assert _tri_ids(o, f, 0) == [0, 3, 4] and _tri_ids(o, f, 1) == [0, 4, 1]
    z = o.heightfield(h, 3, 3, options=4)
    assert _tri_ids(o, z, 0) == [0, 3, 4] and _tri_ids(o, z, 2) == [1, 4, 5] and _tri_ids(o, z, 4) == [3, 6, 4]
    m = o.heightfield(h, 3, 3, options=2)
    assert _tri_ids(o, m, 0) == [0, 3, 4] and _tri_ids(o, m, 2) == [1, 4, 2]
    assert _tri_ids(o, m, 5) == [4, 6, 7] and _tri_ids(o, m, 7) == [4, 8, 5]
    plain = o.heightfield(h, 3, 3)
    flipped = o.heightfield(h, 3, 3, options=8)
    vp, ip = o.mesh_data(plain)
    vf, i_f = o.mesh_data(flipped)
    for t in range(8):
        np.testing.assert_array_equal(vp[ip[t, 0]], vf[i_f[t, 2]])
        np.testing.assert_array_equal(vp[ip[t, 1]], vf[i_f[t, 1]])
        np.testing.assert_array_equal(vp[ip[t, 2]], vf[i_f[t, 0]])


@pytest.mark.parametrize("prec", PREC)
def test_sphere_resting_on_mesh(prec):
    """convex_mesh.rs sphere_resting_on_mesh: penetration 0.1, normal -Y (sphere to mesh)."""
    o = orc.OracleWorld(prec)
    m = flat_ground(o)
    s = o.sphere(0.5)
    c = o.collide(s, pose([0.5, 0.4, 0.5]), m, pose([0, 0, 0]))
    assert len(c) >= 1
    assert c[0, 4] == pytest.approx(-1.0, abs=1e-3) and c[0, 6] == pytest.approx(0.1, abs=1e-3)
    # the same pair with the mesh first: flipped normal (mod.rs:200-213)
    c2 = o.collide(m, pose([0, 0, 0]), s, pose([0.5, 0.4, 0.5]))
    np.testing.assert_allclose(c2[:, 3:6], -c[:, 3:6])
    np.testing.assert_allclose(c2[:, [0, 1, 2, 6]], c[:, [0, 1, 2, 6]])


@pytest.mark.parametrize("prec", PREC)
def test_sphere_fast_path_matches_gjk(prec):
    """convex_mesh.rs sphere_fast_path_matches_gjk: the analytic detector against convex_convex on
    the triangle's three-vertex hull, over face, vertex, off-vertex, band and deep poses."""
    o = orc.OracleWorld(prec)
    tri = [[0, 0, 0], [1, 0, 0], [0.3, 0.2, 0.9]]
    m = o.mesh(tri, [[0, 1, 2]])
    hull = o.hull(np.array(tri, dtype=np.float64))
    s = o.sphere(0.5)
    for center in ([0.4, 0.3, 0.4], [0.95, 0.15, 0.1], [-0.3, 0.3, 0.2], [0.3, 0.55, 0.3], [0.6, 0.05, 0.4]):
        fast = o.collide(s, pose(center), m, pose([0, 0, 0]))
        slow = o.convex_convex(s, pose(center), hull, pose([0, 0, 0]))
        if slow is None:
            assert len(fast) == 0, center
            continue
        assert len(fast) == 1, center
        fp = fast[0]
        assert fp[6] == pytest.approx(slow[6], abs=5e-3)
        assert float(np.dot(fp[3:6], slow[3:6])) > 0.999
        np.testing.assert_allclose(fp[0:3], slow[0:3], atol=1e-2)


@pytest.mark.parametrize("prec", PREC)
def test_sphere_triangle_edge_vertex_band_backface(prec):
    """convex_mesh.rs sphere_triangle_edge_vertex_band_backface."""
    o = orc.OracleWorld(prec)
    a, b, c = [0, 0, 0], [1, 0, 0], [0, 0, 1]
    m = o.mesh([a, b, c], [[0, 1, 2]])
    s = o.sphere(0.5)
    th = o.threshold(s)
    p = o.collide(s, pose([0, 0.4, 0]), m, pose([0, 0, 0]))[0]
    assert p[6] == pytest.approx(0.1, abs=1e-4) and p[4] == pytest.approx(-1.0, abs=1e-3)
    assert float(np.dot(p[0:3], p[0:3])) == pytest.approx(0.0, abs=1e-6)
    p = o.collide(s, pose([0.5, 0.4, 0]), m, pose([0, 0, 0]))[0]
    assert p[6] == pytest.approx(0.1, abs=1e-4) and p[4] == pytest.approx(-1.0, abs=1e-3)
    assert p[0] == pytest.approx(0.5, abs=1e-6) and p[1] == pytest.approx(0.0, abs=1e-6)
    pt, n, pen = orc.sphere_triangle([0.3, 0.51, 0.3], 0.5, th, a, b, c, prec)
    assert pen == pytest.approx(-0.01, abs=1e-4) and n[1] == pytest.approx(1.0, abs=1e-3)
    assert pt[1] == pytest.approx(0.0, abs=1e-6)
    assert orc.sphere_triangle([0.3, 0.6, 0.3], 0.5, th, a, b, c, prec) is None
    p = o.collide(s, pose([0.3, -0.4, 0.3]), m, pose([0, 0, 0]))[0]
    assert p[6] == pytest.approx(0.1, abs=1e-4) and p[4] == pytest.approx(1.0, abs=1e-3)
    assert p[1] == pytest.approx(0.0, abs=1e-6)


@pytest.mark.parametrize("prec", PREC)
def test_separated_sphere_and_box_on_heightfield(prec):
    """convex_mesh.rs separated_sphere_does_not_touch_mesh, box_on_heightfield,
    box_over_many_triangles_reduces_contacts."""
    o = orc.OracleWorld(prec)
    m = flat_ground(o)
    s = o.sphere(0.5)
    assert len(o.collide(s, pose([0.5, 5.0, 0.5]), m, pose([0, 0, 0]))) == 0
    hf = o.heightfield(np.zeros(9), 3, 3)
    bx = o.box([0.5, 0.5, 0.5])
    c = o.collide(bx, pose([0.5, 0.4, 0.5]), hf, pose([0, 0, 0]))
    assert c[0, 4] == pytest.approx(-1.0, abs=1e-3) and c[0, 6] == pytest.approx(0.1, abs=1e-3)
    hf5 = o.heightfield(np.zeros(25), 5, 5)
    c = o.collide(bx, pose([0.0, 0.4, 0.0]), hf5, pose([0, 0, 0]))
    assert 1 <= len(c) <= 4
    assert c[0, 4] == pytest.approx(-1.0, abs=1e-3) and c[0, 6] == pytest.approx(0.1, abs=1e-3)


@pytest.mark.parametrize("prec", PREC)
def test_box_falls_onto_a_heightfield_and_rests(prec):
    """A world step with a static heightfield body: a box dropped on a flat 6x6 terrain comes to
    rest on it (y = half extent within the slop), through the pair pass, the manifold and the
    solver, as example scenes of the reference do with their terrains."""
    o = orc.OracleWorld(prec)
    o.set_gravity([0, -9.81, 0])
    hf = o.heightfield(np.zeros(36), 6, 6, (1.0, 1.0, 1.0))
    bx = o.box([0.5, 0.5, 0.5])
    o.add_body(hf, [0, 0, 0], mass=0.0)
    o.add_body(bx, [0.2, 2.0, 0.1], mass=1.0)
    for _ in range(240):
        o.step(1 / 60)
    st = o.state()
    assert st[1, 1] == pytest.approx(0.5, abs=0.02)
    assert np.abs(st[1, 7:13]).max() < 1e-2


def test_mesh_rain_recipe():
    """rain_500 / dbvt_rain_2000 (tools/perf_scenes.json): lattice sizes, the kind cycling
    (i + nz j + layer) % 3 (box, sphere, capsule), the terrain's grid and wave heights."""
    import scenes

    s = scenes.mesh_rain()
    a = s.arrays()
    assert s.num_bodies == 501 and s.num_dynamic == 500 and a["mass"][0] == 0.0
    kind, params, _ = s.shapes[0]
    assert kind == scenes.MESH
    v, idx = params["vertices"], params["indices"]
    assert v.shape == (400, 3) and idx.shape == (2 * 19 * 19, 3)
    np.testing.assert_allclose(v[0], [-9.5, 0.0, -9.5])
    np.testing.assert_allclose(v[21], [-8.5, 0.2 * np.sin(0.7) * np.cos(0.6), -8.5], rtol=1e-6)
    assert list(idx[0]) == [0, 21, 1] and list(idx[1]) == [0, 20, 21]
    # body 1 + (layer * 100 + j * 10 + i): kind (i + 10 j + layer) % 3 -> shape ids 1 (box), 2, 3
    for layer, j, i in ((0, 0, 0), (0, 0, 1), (0, 1, 0), (4, 9, 9)):
        b = 1 + layer * 100 + j * 10 + i
        assert a["shape"][b] == 1 + (i + 10 * j + layer) % 3
        np.testing.assert_allclose(a["pos"][b], [-6.3 + 1.4 * i, 4.0 + 2.0 * layer, -6.3 + 1.4 * j], rtol=1e-6)
    big = scenes.mesh_rain(nx=20, nz=20, layers=5, grid=40)
    assert big.num_dynamic == 2000
    np.testing.assert_allclose(big.shapes[0][1]["vertices"][0], [-19.5, 0.0, -19.5])
    np.testing.assert_allclose(big.arrays()["pos"][1], [-13.3, 4.0, -13.3], rtol=1e-6)
