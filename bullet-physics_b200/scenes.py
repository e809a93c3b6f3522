"""Seeded synthetic scenes of the five benchmark configurations.

Each builder returns a plain description (shape list + per-body numpy arrays)
that both the device world (bgpu.World) and the CPU oracle can ingest, so a
parity check and a benchmark run start from bit-identical inputs.

  falling_box_stack  1,000 boxes (half 0.5, 1 kg) on a 10x10x10 grid, 1.1 m
                     spacing, 2 m above a ground plane, jitter U(-0.05,0.05) m
                     and +-5 deg about a random axis; 10 iterations; 300 steps.
  mixed_convex_pile  16,384 bodies: 40% boxes (half U(0.2,0.6)^3), 30% spheres
                     (r U(0.2,0.5)), 15% capsules (r U(0.1,0.3), hh U(0.2,0.6)),
                     15% hulls of 24 points on a sphere of R U(0.3,0.6);
                     rho 1000; uniform in a 40 m cube above the ground, random
                     orientation; 10 iterations; 300 steps.
  large_pile         131,072 bodies (50% unit boxes half 0.5, 50% spheres
                     r 0.5) on a jittered 64x64x32 grid, 1.05 m spacing;
                     20 iterations; 600 steps.
  batched_worlds     4,096 independent worlds of n = floor(exp(U(ln 8, ln 256)))
                     dynamic bodies each, half of them columns of 1-16 unit
                     boxes, half jittered sphere piles (r 0.5), every world on
                     its own ground plane; 10 iterations; 500 steps.
  adjoint_worlds     1,024 worlds of 64 unit boxes (4x4x4, 1.2 m apart) thrown
                     with v0 U(-2,2)^3, friction U(0.2,0.9), restitution
                     U(0,0.3); ground plane with friction and restitution 1 (so
                     a ground contact's coefficients are the box's); dt 1/120;
                     10 iterations; 120 steps; loss sum_w |com_w - target_w|^2.
Scaled-down variants (`scale`) keep the recipe and shrink the grid.
"""
import math

import numpy as np

SPHERE, BOX, CAPSULE, HULL, PLANE, MESH = 0, 1, 2, 3, 4, 5


ACT_DISABLE_DEACTIVATION = 4  # ActivationState::DisableDeactivation (body.rs:140-153)


class Scene:
    def __init__(self, name, dt, iterations, steps):
        self.name = name
        self.dt = dt
        self.iterations = iterations
        self.steps = steps
        self.gravity = (0.0, -9.81, 0.0)
        self.shapes = []  # (type, params list, points or None)
        self.shape_of = []
        self.pos = []
        self.quat = []
        self.linvel = []
        self.angvel = []
        self.mass = []
        self.friction = []
        self.restitution = []

    def add_shape(self, kind, params=(), points=None):
        self.shapes.append((kind, list(params), None if points is None else np.asarray(points, dtype=np.float32)))
        return len(self.shapes) - 1

    def add_mesh(self, vertices, indices):
        """A static triangle mesh shape (vertices n x 3, triangles m x 3)."""
        self.shapes.append((MESH, {"vertices": np.asarray(vertices, dtype=np.float32).reshape(-1, 3),
                                   "indices": np.asarray(indices, dtype=np.uint32).reshape(-1, 3)}, None))
        return len(self.shapes) - 1

    def add_heightfield(self, heights, width, depth, cell=(1.0, 1.0, 1.0), options=0):
        """A static heightfield shape (width x depth row-major heights)."""
        self.shapes.append((MESH, {"heights": np.asarray(heights, dtype=np.float32).reshape(-1), "width": width,
                                   "depth": depth, "cell": tuple(cell), "options": options}, None))
        return len(self.shapes) - 1

    def add(self, shape, pos, quat=(0, 0, 0, 1), mass=1.0, linvel=(0, 0, 0), angvel=(0, 0, 0), friction=0.5,
            restitution=0.0):
        self.shape_of.append(shape)
        self.pos.append(pos)
        self.quat.append(quat)
        self.linvel.append(linvel)
        self.angvel.append(angvel)
        self.mass.append(mass)
        self.friction.append(friction)
        self.restitution.append(restitution)

    def arrays(self):
        return dict(shape=np.asarray(self.shape_of, dtype=np.uint32), pos=np.asarray(self.pos, dtype=np.float32),
                    quat=np.asarray(self.quat, dtype=np.float32), linvel=np.asarray(self.linvel, dtype=np.float32),
                    angvel=np.asarray(self.angvel, dtype=np.float32), mass=np.asarray(self.mass, dtype=np.float32),
                    friction=np.asarray(self.friction, dtype=np.float32),
                    restitution=np.asarray(self.restitution, dtype=np.float32))

    @property
    def num_bodies(self):
        return len(self.shape_of)

    @property
    def num_dynamic(self):
        return int(np.count_nonzero(np.asarray(self.mass) > 0))

    def build_gpu(self, bgpu_module, **solver):
        w = bgpu_module.World(gravity=self.gravity, num_iterations=self.iterations, **solver)
        add_shapes(w, self.shapes)
        a = self.arrays()
        w.add_bodies_array(a["shape"], a["pos"], a["quat"], a["linvel"], a["angvel"], a["mass"], a["friction"],
                           a["restitution"])
        return w

    def build_oracle(self, oracle_module, precision="f32", **solver):
        w = oracle_module.OracleWorld(precision)
        w.set_gravity(self.gravity)
        w.set_solver(num_iterations=self.iterations, **solver)
        add_shapes(w, self.shapes)
        a = self.arrays()
        for i in range(self.num_bodies):
            w.add_body(int(a["shape"][i]), a["pos"][i].astype(np.float64), quat=a["quat"][i].astype(np.float64),
                       linvel=a["linvel"][i].astype(np.float64), angvel=a["angvel"][i].astype(np.float64),
                       mass=float(a["mass"][i]), friction=float(a["friction"][i]),
                       restitution=float(a["restitution"][i]))
        return w


def add_shapes(w, shapes):
    """Register a scene's shape list with a device world or an oracle world (same calls)."""
    for kind, params, pts in shapes:
        if kind == MESH and "heights" in params:
            w.heightfield(params["heights"], params["width"], params["depth"], params["cell"], params["options"])
        elif kind == MESH:
            w.mesh(params["vertices"], params["indices"])
        else:
            w.add_shape(kind, params, pts)


def wavy_grid_mesh(nx, nz, origin, cell, amp, ax, az):
    """The perf scenes' terrain (tools/perf_scenes.json "mesh" shapes: heights
    amp * sin(ax * x) * cos(az * z) on an nx x nz grid, vertices z-major at
    origin + (x, z) * cell, two triangles per cell wound (v00, v11, v10),
    (v00, v01, v11) for +Y faces)."""
    z, x = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    h = amp * np.sin(x * ax) * np.cos(z * az)
    v = np.stack([origin[0] + x * cell[0], h, origin[1] + z * cell[1]], axis=-1).reshape(-1, 3)
    idx = []
    for zz in range(nz - 1):
        for xx in range(nx - 1):
            v00 = zz * nx + xx
            v10, v01 = v00 + 1, v00 + nx
            v11 = v01 + 1
            idx += [[v00, v11, v10], [v00, v01, v11]]
    return v.astype(np.float32), np.asarray(idx, dtype=np.uint32)


def mesh_rain(nx=10, nz=10, layers=5, grid=20, steps=300):
    """The reference's rain_500 / dbvt_rain_2000 perf scenes (tools/perf_scenes.json): a lattice of
    boxes (half 0.35), spheres (r 0.35) and capsules (r 0.3, half height 0.5), the kind cycling
    with (i + nz j + layer) % 3, spaced 1.4 x 2.0 x 1.4 m from 4 m up, raining onto a wavy
    grid x grid terrain mesh (amp 0.2, ax 0.7, az 0.6, 1 m cells, centred); mass 1, friction
    0.6, restitution 0; dt 1/60, 10 iterations. nx = nz = 10, grid 20 is rain_500; 20 x 20 with
    grid 40 is dbvt_rain_2000."""
    s = Scene(f"mesh_rain_{nx * nz * layers}", 1.0 / 60.0, 10, steps)
    half = (grid - 1) / 2.0
    v, idx = wavy_grid_mesh(grid, grid, (-half, -half), (1.0, 1.0), 0.2, 0.7, 0.6)
    terrain = s.add_mesh(v, idx)
    box = s.add_shape(BOX, [0.35, 0.35, 0.35])
    sph = s.add_shape(SPHERE, [0.35])
    cap = s.add_shape(CAPSULE, [0.3, 0.5])
    s.add(terrain, (0.0, 0.0, 0.0), mass=0.0, friction=0.6)
    bx = -0.7 * (nx - 1)
    bz = -0.7 * (nz - 1)
    for layer in range(layers):
        for j in range(nz):
            for i in range(nx):
                kind = (box, sph, cap)[(i + nz * j + layer) % 3]
                s.add(kind, (bx + i * 1.4, 4.0 + layer * 2.0, bz + j * 1.4), mass=1.0, friction=0.6)
    return s


def random_quat_small(rng, max_deg):
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    ang = math.radians(rng.uniform(-max_deg, max_deg))
    s = math.sin(ang / 2)
    q = np.array([axis[0] * s, axis[1] * s, axis[2] * s, math.cos(ang / 2)], dtype=np.float32)
    return q / np.linalg.norm(q)


def random_quat(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    if q[3] < 0:
        q = -q
    return q.astype(np.float32)


def falling_box_stack(nx=10, ny=10, nz=10, seed=1, steps=300):
    """Config 1: box grid over a ground plane (10 iterations, dt 1/60)."""
    rng = np.random.default_rng(seed)
    s = Scene(f"falling_box_stack_{nx}x{ny}x{nz}", 1.0 / 60.0, 10, steps)
    plane = s.add_shape(PLANE, [0.0, 1.0, 0.0, 0.0])
    box = s.add_shape(BOX, [0.5, 0.5, 0.5])
    s.add(plane, (0.0, 0.0, 0.0), mass=0.0)
    sp = 1.1
    for j in range(ny):
        for i in range(nx):
            for k in range(nz):
                p = np.array([(i - (nx - 1) / 2) * sp, 2.0 + j * sp, (k - (nz - 1) / 2) * sp])
                p = p + rng.uniform(-0.05, 0.05, size=3)
                s.add(box, tuple(p.astype(np.float32)), random_quat_small(rng, 5.0), mass=1.0, friction=0.5)
    return s


def fibonacci_free_points(rng, n, radius):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (v * radius).astype(np.float32)


def hull_volume(points):
    from scipy.spatial import ConvexHull  # scene generation only

    return float(ConvexHull(points).volume)


def mixed_convex_pile(n=16384, seed=2, steps=300, extent=40.0):
    """Config 2: boxes/spheres/capsules/hulls at rho 1000, uniform in a cube above the ground."""
    rng = np.random.default_rng(seed)
    s = Scene(f"mixed_convex_pile_{n}", 1.0 / 60.0, 10, steps)
    plane = s.add_shape(PLANE, [0.0, 1.0, 0.0, 0.0])
    s.add(plane, (0.0, 0.0, 0.0), mass=0.0)
    rho = 1000.0
    kinds = rng.choice(4, size=n, p=[0.4, 0.3, 0.15, 0.15])
    for t in range(n):
        kind = kinds[t]
        if kind == 0:
            h = rng.uniform(0.2, 0.6, size=3)
            sh = s.add_shape(BOX, list(h))
            mass = rho * 8.0 * h[0] * h[1] * h[2]
        elif kind == 1:
            r = rng.uniform(0.2, 0.5)
            sh = s.add_shape(SPHERE, [r])
            mass = rho * 4.0 / 3.0 * math.pi * r ** 3
        elif kind == 2:
            r = rng.uniform(0.1, 0.3)
            hh = rng.uniform(0.2, 0.6)
            sh = s.add_shape(CAPSULE, [r, hh])
            mass = rho * (math.pi * r * r * 2.0 * hh + 4.0 / 3.0 * math.pi * r ** 3)
        else:
            R = rng.uniform(0.3, 0.6)
            pts = fibonacci_free_points(rng, 24, R)
            sh = s.add_shape(HULL, [], pts)
            mass = rho * hull_volume(pts)
        p = (rng.uniform(-extent / 2, extent / 2), rng.uniform(1.0, 1.0 + extent), rng.uniform(-extent / 2, extent / 2))
        s.add(sh, p, random_quat(rng), mass=float(mass))
    return s


def large_pile(nx=64, nz=64, ny=32, seed=3, steps=600, spacing=1.05):
    """Config 3: 50% unit boxes / 50% r-0.5 spheres on a jittered grid (20 iterations)."""
    rng = np.random.default_rng(seed)
    s = Scene(f"large_pile_{nx}x{nz}x{ny}", 1.0 / 60.0, 20, steps)
    plane = s.add_shape(PLANE, [0.0, 1.0, 0.0, 0.0])
    box = s.add_shape(BOX, [0.5, 0.5, 0.5])
    sph = s.add_shape(SPHERE, [0.5])
    s.add(plane, (0.0, 0.0, 0.0), mass=0.0)
    n = nx * ny * nz
    is_box = rng.random(n) < 0.5
    jit = rng.uniform(-0.02, 0.02, size=(n, 3))
    t = 0
    for j in range(ny):
        for i in range(nx):
            for k in range(nz):
                p = np.array([(i - (nx - 1) / 2) * spacing, 0.6 + j * spacing, (k - (nz - 1) / 2) * spacing]) + jit[t]
                if is_box[t]:
                    s.add(box, tuple(p.astype(np.float32)), random_quat_small(rng, 5.0), mass=1.0)
                else:
                    s.add(sph, tuple(p.astype(np.float32)), mass=1.0)
                t += 1
    return s


def large_pile_arrays(nx=64, nz=64, ny=32, seed=3, spacing=1.05):
    """Vectorised builder of the same recipe as large_pile (fast for 131k bodies)."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    is_box = rng.random(n) < 0.5
    jit = rng.uniform(-0.02, 0.02, size=(n, 3))
    j, i, k = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz), indexing="ij")
    base = np.stack([(i.ravel() - (nx - 1) / 2) * spacing, 0.6 + j.ravel() * spacing,
                     (k.ravel() - (nz - 1) / 2) * spacing], axis=1)
    pos = (base + jit).astype(np.float32)
    axis = rng.normal(size=(n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    ang = np.radians(rng.uniform(-5.0, 5.0, size=n))
    quat = np.concatenate([axis * np.sin(ang / 2)[:, None], np.cos(ang / 2)[:, None]], axis=1).astype(np.float32)
    quat[~is_box] = [0, 0, 0, 1]
    quat /= np.linalg.norm(quat, axis=1, keepdims=True)
    return is_box, pos, quat


def large_pile_fast(nx=64, nz=64, ny=32, seed=3, steps=600, spacing=1.05):
    s = Scene(f"large_pile_{nx}x{nz}x{ny}", 1.0 / 60.0, 20, steps)
    plane = s.add_shape(PLANE, [0.0, 1.0, 0.0, 0.0])
    box = s.add_shape(BOX, [0.5, 0.5, 0.5])
    sph = s.add_shape(SPHERE, [0.5])
    is_box, pos, quat = large_pile_arrays(nx, nz, ny, seed, spacing)
    n = len(pos)
    s.shape_of = [plane] + list(np.where(is_box, box, sph))
    s.pos = [(0.0, 0.0, 0.0)] + list(map(tuple, pos))
    s.quat = [(0, 0, 0, 1)] + list(map(tuple, quat))
    s.linvel = [(0, 0, 0)] * (n + 1)
    s.angvel = [(0, 0, 0)] * (n + 1)
    s.mass = [0.0] + [1.0] * n
    s.friction = [0.5] * (n + 1)
    s.restitution = [0.0] * (n + 1)
    return s


class BatchScene:
    """Independent worlds sharing one shape list (batched-worlds configuration)."""

    FIELDS = ("shape", "pos", "quat", "linvel", "angvel", "mass", "friction", "restitution")

    def __init__(self, name, dt, iterations, steps):
        self.name = name
        self.dt = dt
        self.iterations = iterations
        self.steps = steps
        self.gravity = (0.0, -9.81, 0.0)
        self.shapes = []
        self.worlds = []  # per world: dict of the FIELDS arrays

    def add_shape(self, kind, params=(), points=None):
        self.shapes.append((kind, list(params), None if points is None else np.asarray(points, dtype=np.float32)))
        return len(self.shapes) - 1

    def add_world(self, shape, pos, quat, mass, linvel=None, friction=None, restitution=None):
        n = len(shape)
        self.worlds.append(dict(shape=np.asarray(shape, dtype=np.uint32), pos=np.asarray(pos, dtype=np.float32),
                                quat=np.asarray(quat, dtype=np.float32),
                                linvel=(np.zeros((n, 3), np.float32) if linvel is None
                                        else np.asarray(linvel, dtype=np.float32).reshape(n, 3)),
                                angvel=np.zeros((n, 3), np.float32), mass=np.asarray(mass, dtype=np.float32),
                                friction=(np.full(n, 0.5, np.float32) if friction is None
                                          else np.asarray(friction, dtype=np.float32)),
                                restitution=(np.zeros(n, np.float32) if restitution is None
                                             else np.asarray(restitution, dtype=np.float32))))

    @property
    def bodies_per_world(self):
        return np.array([len(w["shape"]) for w in self.worlds], dtype=np.uint32)

    @property
    def num_bodies(self):
        return int(self.bodies_per_world.sum())

    @property
    def num_dynamic(self):
        return int(sum(np.count_nonzero(w["mass"] > 0) for w in self.worlds))

    def arrays(self):
        return {f: np.concatenate([w[f] for w in self.worlds]) for f in self.FIELDS}

    def build_gpu(self, bgpu_module, **solver):
        w = bgpu_module.World(gravity=self.gravity, batch=True, num_iterations=self.iterations, **solver)
        add_shapes(w, self.shapes)
        a = self.arrays()
        w.add_worlds_array(self.bodies_per_world, a["shape"], a["pos"], a["quat"], a["linvel"], a["angvel"],
                           a["mass"], a["friction"], a["restitution"])
        return w

    def world_scene(self, k):
        """World k alone, as a Scene with the same shape list (for the oracle or a plain GPU world)."""
        s = Scene(f"{self.name}_world{k}", self.dt, self.iterations, self.steps)
        s.gravity = self.gravity
        s.shapes = list(self.shapes)
        w = self.worlds[k]
        s.shape_of = [int(x) for x in w["shape"]]
        s.pos = list(map(tuple, w["pos"]))
        s.quat = list(map(tuple, w["quat"]))
        s.linvel = list(map(tuple, w["linvel"]))
        s.angvel = list(map(tuple, w["angvel"]))
        s.mass = [float(x) for x in w["mass"]]
        s.friction = [float(x) for x in w["friction"]]
        s.restitution = [float(x) for x in w["restitution"]]
        return s


def _small_rotations(rng, n, max_deg):
    axis = rng.normal(size=(n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    ang = np.radians(rng.uniform(-max_deg, max_deg, size=n))
    q = np.concatenate([axis * np.sin(ang / 2)[:, None], np.cos(ang / 2)[:, None]], axis=1)
    return (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)


def batched_worlds(n_worlds=4096, seed=4, steps=500, min_bodies=8, max_bodies=256):
    """Batched-worlds configuration: n = floor(exp(U(ln 8, ln 256))) dynamic bodies per world,
    box columns (heights U{1..16}, 1.5 m apart) or a jittered sphere pile, each on its own plane."""
    rng = np.random.default_rng(seed)
    s = BatchScene(f"batched_worlds_{n_worlds}", 1.0 / 60.0, 10, steps)
    plane = s.add_shape(PLANE, [0.0, 1.0, 0.0, 0.0])
    box = s.add_shape(BOX, [0.5, 0.5, 0.5])
    sph = s.add_shape(SPHERE, [0.5])
    for _ in range(n_worlds):
        nb = int(math.floor(math.exp(rng.uniform(math.log(min_bodies), math.log(max_bodies)))))
        if rng.random() < 0.5:  # columns of boxes
            heights = []
            left = nb
            while left > 0:
                h = min(int(rng.integers(1, 17)), left)
                heights.append(h)
                left -= h
            side = int(math.ceil(math.sqrt(len(heights))))
            col = np.repeat(np.arange(len(heights)), heights)
            lvl = np.concatenate([np.arange(h) for h in heights])
            x = (col % side - (side - 1) / 2) * 1.5
            z = (col // side - (side - 1) / 2) * 1.5
            y = 0.55 + lvl * 1.05
            pos = np.stack([x, y, z], axis=1) + np.concatenate(
                [rng.uniform(-0.02, 0.02, size=(nb, 1)), np.zeros((nb, 1)), rng.uniform(-0.02, 0.02, size=(nb, 1))],
                axis=1)
            quat = _small_rotations(rng, nb, 2.0)
            kind = box
        else:  # sphere pile
            side = int(math.ceil(nb ** (1.0 / 3.0)))
            t = np.arange(nb)
            gx, gz, gy = t % side, (t // side) % side, t // (side * side)
            pos = np.stack([(gx - (side - 1) / 2) * 1.05, 0.6 + gy * 1.05, (gz - (side - 1) / 2) * 1.05], axis=1)
            pos = pos + rng.uniform(-0.05, 0.05, size=(nb, 3))
            quat = np.tile(np.array([0, 0, 0, 1], np.float32), (nb, 1))
            kind = sph
        shape = np.concatenate([[plane], np.full(nb, kind)])
        pos = np.concatenate([np.zeros((1, 3)), pos]).astype(np.float32)
        quat = np.concatenate([np.array([[0, 0, 0, 1]], np.float32), quat])
        mass = np.concatenate([[0.0], np.ones(nb)])
        s.add_world(shape, pos, quat, mass)
    return s


def adjoint_worlds(n_worlds=1024, seed=5, steps=120, side=4):
    """Adjoint configuration: boxes thrown in independent worlds; world targets for the loss."""
    rng = np.random.default_rng(seed)
    s = BatchScene(f"adjoint_worlds_{n_worlds}", 1.0 / 120.0, 10, steps)
    plane = s.add_shape(PLANE, [0.0, 1.0, 0.0, 0.0])
    box = s.add_shape(BOX, [0.5, 0.5, 0.5])
    nb = side ** 3
    t = np.arange(nb)
    gx, gz, gy = t % side, (t // side) % side, t // (side * side)
    base = np.stack([(gx - (side - 1) / 2) * 1.2, 0.6 + gy * 1.2, (gz - (side - 1) / 2) * 1.2], axis=1)
    s.targets = []
    for _ in range(n_worlds):
        pos = base + rng.uniform(-0.05, 0.05, size=(nb, 3))
        v0 = rng.uniform(-2.0, 2.0, size=(nb, 3))
        mu = rng.uniform(0.2, 0.9, size=nb)
        e = rng.uniform(0.0, 0.3, size=nb)
        s.add_world(np.concatenate([[plane], np.full(nb, box)]),
                    np.concatenate([np.zeros((1, 3)), pos]).astype(np.float32),
                    np.tile(np.array([0, 0, 0, 1], np.float32), (nb + 1, 1)),
                    np.concatenate([[0.0], np.ones(nb)]),
                    linvel=np.concatenate([np.zeros((1, 3)), v0]),
                    friction=np.concatenate([[1.0], mu]), restitution=np.concatenate([[1.0], e]))
        s.targets.append(pos.mean(axis=0) + np.array([1.0, 0.0, 0.5]))
    s.targets = np.asarray(s.targets, dtype=np.float64)
    return s


def com_loss(positions, masses, offsets, targets):
    """sum_w |com_w - target_w|^2 over the dynamic bodies of each world, and dL/dx per body."""
    x = np.asarray(positions, dtype=np.float64)
    m = np.asarray(masses, dtype=np.float64)
    g = np.zeros_like(x)
    loss = 0.0
    for k in range(len(offsets) - 1):
        lo, hi = int(offsets[k]), int(offsets[k + 1])
        mk = m[lo:hi]
        M = mk.sum()
        com = (mk[:, None] * x[lo:hi]).sum(axis=0) / M
        d = com - targets[k]
        loss += float(d @ d)
        g[lo:hi] = 2.0 * d[None, :] * (mk / M)[:, None]
    return loss, g


def spring2_chains_world(bgpu, count=150, cols=15, links=3, spacing=4.0, base_height=4.0, pitch=0.55, half=0.2,
                         mass=1.0, stiffness=5.0, damping=0.3, iterations=10):
    """The spring2_chains perf scene (tools/perf_scenes.json "spring2_chains",
    examples/perf_scenes.rs add_spring2): `count` static anchor boxes in a grid of `cols` columns,
    each with a horizontal chain of `links` 1 kg boxes joined by spring-2 joints whose three angular
    springs are on (linear axes locked), never sleeping. The reference's scene is count=150 (600
    bodies, 450 joints); larger counts extend the grid. Returns the GPU world."""
    w = bgpu.World(gravity=(0.0, -9.81, 0.0), num_iterations=iterations)
    box = w.add_shape(bgpu.BOX, [half, half, half])
    rows = -(-count // cols)
    k = np.arange(count)
    x = (k % cols - (cols - 1) / 2.0) * spacing
    z = (k // cols - (rows - 1) / 2.0) * spacing
    per = links + 1
    n = count * per
    pos = np.zeros((n, 3), dtype=np.float32)
    pos[:, 0] = np.repeat(x, per) + np.tile(np.arange(per), count) * pitch
    pos[:, 1] = base_height
    pos[:, 2] = np.repeat(z, per)
    quat = np.tile(np.array([0.0, 0.0, 0.0, 1.0], dtype=np.float32), (n, 1))
    m = np.tile(np.array([0.0] + [mass] * links, dtype=np.float32), count)
    d = bgpu.desc_array(np.full(n, box), pos, quat, mass=m)
    d["activation"] = np.where(m > 0, ACT_DISABLE_DEACTIVATION, 0).astype(np.uint32)
    first = bgpu.ctypes.c_uint32()
    bgpu.check(w.L.bgpu_add_bodies(w.h, n, d.ctypes.data_as(bgpu.ctypes.POINTER(bgpu.BodyDesc)),
                                   bgpu.ctypes.byref(first)), "add_bodies")
    frame = lambda ox: [ox, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
    descs = (bgpu.Spring2Desc * (count * links))()
    t = 0
    for c in range(count):
        for i in range(1, links + 1):
            j = bgpu.Spring2(c * per + i - 1, c * per + i, frame(pitch / 2.0), frame(-pitch / 2.0))
            for ax in range(3, 6):
                j.enable_spring(ax)
                j.set_stiffness(ax, stiffness, True)
                j.set_damping(ax, damping, True)
            descs[t] = j.desc
            t += 1
    bgpu.check(w.L.bgpu_add_spring2_joints(w.h, t, descs, bgpu.ctypes.byref(first)), "add_spring2_joints")
    return w


def ccd_rain_world(bgpu, n_ccd=2048, n_boxes=1024, plates=16, seed=7, iterations=10):
    """Fast CCD spheres (r 0.2, falling at 60-400 m/s, motion threshold 0.05, swept radius 0.2)
    and plain boxes raining onto a `plates` x `plates` grid of thin static plates (0.1 m thick) over
    a ground plane: each step sweeps every CCD sphere against the bodies of the world, as the
    reference's CCD stage does (world/step.rs:1068-1155). Returns (world, CCD body ids)."""
    rng = np.random.default_rng(seed)
    w = bgpu.World(gravity=(0.0, -9.81, 0.0), num_iterations=iterations)
    w.add_body(w.add_shape(bgpu.PLANE, [0.0, 1.0, 0.0, 0.0]), (0.0, 0.0, 0.0), mass=0.0)
    plate = w.add_shape(bgpu.BOX, [1.5, 0.05, 1.5])
    ext = plates * 3.2 / 2.0
    for px in range(plates):
        for pz in range(plates):
            w.add_body(plate, (px * 3.2 - ext + 1.6, 2.0 + 0.3 * ((px + pz) % 3), pz * 3.2 - ext + 1.6), mass=0.0)
    sph = w.add_shape(bgpu.SPHERE, [0.2])
    box = w.add_shape(bgpu.BOX, [0.2, 0.2, 0.2])
    n = n_ccd + n_boxes
    kind = np.zeros(n, dtype=bool)
    kind[rng.permutation(n)[:n_ccd]] = True
    pos = np.stack([rng.uniform(-ext, ext, n), rng.uniform(4.0, 12.0, n), rng.uniform(-ext, ext, n)], axis=1)
    vel = np.zeros((n, 3))
    vel[:, 0] = np.where(kind, rng.uniform(-5.0, 5.0, n), 0.0)
    vel[:, 1] = np.where(kind, rng.uniform(-400.0, -60.0, n), -5.0)
    quat = np.tile(np.array([0.0, 0.0, 0.0, 1.0]), (n, 1))
    d = bgpu.desc_array(np.where(kind, sph, box), pos, quat, linvel=vel, mass=np.ones(n))
    first = bgpu.ctypes.c_uint32()
    bgpu.check(w.L.bgpu_add_bodies(w.h, n, d.ctypes.data_as(bgpu.ctypes.POINTER(bgpu.BodyDesc)),
                                   bgpu.ctypes.byref(first)), "add_bodies")
    ids = first.value + np.flatnonzero(kind)
    thr = np.zeros(n, dtype=np.float32)
    rad = np.zeros(n, dtype=np.float32)
    thr[kind], rad[kind] = 0.05, 0.2
    w.set_ccd(first.value, thr, rad)
    return w, ids
