"""Pins the oracle's shape bounds and inertias against the reference's shape tests
(crates/bullet-collision/src/shapes, file and lines cited), in both precisions.
"""
import math

import pytest

from oracle_api import OracleWorld, pose

PRECISIONS = ["f32", "f64"]
OCTAHEDRON = [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]]


@pytest.mark.parametrize("prec", PRECISIONS)
def test_box_inertia_matches_analytical(prec):
    # shapes/box_shape.rs:102-109
    w = OracleWorld(prec)
    i = w.inertia(w.box([1.0, 2.0, 3.0]), 12.0)
    assert i[0] == pytest.approx(4.0 * 13.0) and i[1] == pytest.approx(4.0 * 10.0) and i[2] == pytest.approx(4.0 * 5.0)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_sphere_inertia_matches_analytical(prec):
    # shapes/sphere.rs:71-77
    w = OracleWorld(prec)
    i = w.inertia(w.sphere(1.0), 5.0)
    assert list(i) == pytest.approx([2.0, 2.0, 2.0])


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capsule_inertia_matches_analytical(prec):
    # shapes/capsule.rs:116-123: mass split 0.6 / 0.4 between the cylinder and the two caps.
    w = OracleWorld(prec)
    i = w.inertia(w.capsule(1.0, 1.0), 1.0)
    assert i[0] == pytest.approx(0.6 * 7.0 / 12.0 + 0.4 * (0.4 + 1.0), rel=1e-6)
    assert i[1] == pytest.approx(0.6 * 0.5 + 0.4 * 0.4, rel=1e-6)
    assert i[2] == pytest.approx(i[0])


@pytest.mark.parametrize("prec", PRECISIONS)
def test_capsule_rotated_aabb_swings_the_axis(prec):
    # shapes/capsule.rs:126-135: turned 90 degrees about z, the segment lies along x.
    w = OracleWorld(prec)
    q = (0.0, 0.0, math.sin(math.pi / 4), math.cos(math.pi / 4))
    a = w.world_aabb(w.capsule(0.5, 1.0), pose((0, 0, 0), q))
    assert a[0] == pytest.approx(-1.5, abs=1e-6) and a[3] == pytest.approx(1.5, abs=1e-6)
    assert a[1] == pytest.approx(-0.5, abs=1e-6) and a[4] == pytest.approx(0.5, abs=1e-6)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_hull_aabb_covers_the_vertices(prec):
    # shapes/convex_hull.rs:117-123 (the local box, seen at the identity pose)
    w = OracleWorld(prec)
    a = w.world_aabb(w.hull(OCTAHEDRON), pose())
    assert a[0] == pytest.approx(-1.0) and a[4] == pytest.approx(1.0) and a[5] == pytest.approx(1.0)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_hull_inertia_uses_the_bounding_box(prec):
    # shapes/convex_hull.rs:126-133: a 2 x 2 x 2 bounding box, like a unit-half-extent box.
    w = OracleWorld(prec)
    i = w.inertia(w.hull(OCTAHEDRON), 3.0)
    assert list(i) == pytest.approx([2.0, 2.0, 2.0])


@pytest.mark.parametrize("prec", PRECISIONS)
def test_plane_aabb_is_unbounded(prec):
    # shapes/plane.rs:61-66
    w = OracleWorld(prec)
    a = w.world_aabb(w.plane([0, 1, 0], 0.0), pose())
    assert a[0] < -1e9 and a[3] > 1e9
