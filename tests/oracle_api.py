"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) — test infrastructure.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module; the product library never does.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "liboracle.so")

SPHERE, BOX, CAPSULE, HULL, PLANE, MESH = 0, 1, 2, 3, 4, 5
ACTIVE, ISLAND_SLEEPING, WANTS_DEACTIVATION, DISABLE_DEACTIVATION, DISABLE_SIMULATION = 1, 2, 3, 4, 5
NO_CONTACT_RESPONSE, DISABLE_WORLD_GRAVITY, KINEMATIC = 0x1, 0x2, 0x4
ADDITIONAL_DAMPING = 0x10  # the additional_damping(true) builder (the library's body flag of that name)

DESC = 24   # body descriptor doubles (oracle_capi.cpp)
STATE = 15  # body state doubles
ROW = 26    # contact row doubles

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle/liboracle.so is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        U32 = ctypes.c_uint32
        sig = {
            "orc_world_new": (P, [ctypes.c_int]),
            "orc_world_free": (None, [P]),
            "orc_world_set_gravity": (None, [P, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
            "orc_world_set_solver": (None, [P, D]),
            "orc_world_set_brute_force": (None, [P, ctypes.c_int]),
            "orc_world_add_shape": (U32, [P, U32, D, D, U32]),
            "orc_shape_threshold": (ctypes.c_double, [P, U32]),
            "orc_shape_world_aabb": (None, [P, U32, D, D]),
            "orc_shape_inertia": (None, [P, U32, ctypes.c_double, D]),
            "orc_world_add_body": (U32, [P, D]),
            "orc_world_num_bodies": (U32, [P]),
            "orc_world_step": (None, [P, ctypes.c_double]),
            "orc_world_get_state": (None, [P, D]),
            "orc_world_set_state": (None, [P, D]),
            "orc_world_get_push": (None, [P, D]),
            "orc_world_apply_force": (None, [P, ctypes.c_uint32, D, D]),
            "orc_world_step_fixed": (ctypes.c_uint32, [P, ctypes.c_double, ctypes.c_uint32, ctypes.c_double]),
            "orc_world_set_filter": (None, [P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
            "orc_world_num_pairs": (U32, [P]),
            "orc_world_get_pairs": (None, [P, ctypes.POINTER(U32)]),
            "orc_world_num_rows": (U32, [P]),
            "orc_world_get_rows": (None, [P, ctypes.c_int, D]),
            "orc_world_narrowphase_calls": (U32, [P]),
            "orc_world_num_manifolds": (U32, [P]),
            "orc_world_set_solve_order": (None, [P, ctypes.POINTER(ctypes.c_uint64), U32]),
            "orc_world_stage_seconds": (None, [P, D]),
            "orc_collide": (ctypes.c_int, [P, U32, D, U32, D, D, D]),
            "orc_gjk_kind": (ctypes.c_int, [P, U32, D, U32, D]),
            "orc_gjk_contact": (ctypes.c_int, [P, U32, D, U32, D, D, ctypes.c_double, D]),
            "orc_convex_convex": (ctypes.c_int, [P, U32, D, U32, D, D]),
            "orc_solve_contacts": (None, [P, D, U32, ctypes.c_double, D]),
            "orc_pairs": (ctypes.c_uint64, [ctypes.c_int, D, U32, ctypes.c_int, ctypes.POINTER(U32), ctypes.c_uint64]),
            "orc_pm_new": (P, [ctypes.c_int]),
            "orc_pm_free": (None, [P]),
            "orc_pm_capture": (None, [P, D, U32, D, D, ctypes.c_double]),
            "orc_pm_refresh": (U32, [P, D, D, D]),
            "orc_pm_needs_redetect": (ctypes.c_int, [P, D, D]),
            "orc_pm_set_impulse": (None, [P, U32, ctypes.c_double]),
            "orc_pm_points": (U32, [P, D]),
            "orc_manifold_reduce": (U32, [ctypes.c_int, D, ctypes.c_uint32, ctypes.c_uint32, D]),
            "orc_interpolate_pose": (None, [ctypes.c_int, D, ctypes.c_double, D]),
            "orc_world_add_joint": (U32, [P, D]),
            "orc_world_set_joint_order": (None, [P, ctypes.POINTER(U32), U32]),
            "orc_world_set_joint_flags": (None, [P, U32, U32]),
            "orc_world_joint_angles": (None, [P, D]),
            "orc_world_joint_positions": (None, [P, D]),
            "orc_world_num_joint_rows": (U32, [P]),
            "orc_world_joint_rows": (None, [P, D]),
            "orc_hinge_frames": (None, [ctypes.c_int, D, D, D, D, D]),
            "orc_world_joint_spring2_state": (None, [P, D]),
            "orc_world_set_ccd": (None, [P, U32, ctypes.c_double, ctypes.c_double]),
            "orc_world_ccd_clamps": (None, [P, D]),
            "orc_spring2_angle_info": (None, [ctypes.c_int, D, D, U32, D]),
            "orc_world_add_mesh": (U32, [P, D, U32, ctypes.POINTER(U32), U32]),
            "orc_world_add_heightfield": (U32, [P, D, U32, U32, D, U32]),
            "orc_mesh_counts": (U32, [P, U32, ctypes.POINTER(U32)]),
            "orc_mesh_data": (None, [P, U32, D, ctypes.POINTER(U32)]),
            "orc_mesh_query": (U32, [P, U32, D, ctypes.POINTER(U32), U32]),
            "orc_sphere_triangle": (ctypes.c_int, [ctypes.c_int, D, ctypes.c_double, ctypes.c_double, D, D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def pose(p=(0, 0, 0), q=(0, 0, 0, 1)):
    return f64(list(p) + list(q))


def body_desc(shape, pos, quat=(0, 0, 0, 1), linvel=(0, 0, 0), angvel=(0, 0, 0), mass=1.0, friction=0.5,
              restitution=0.0, flags=0, group=1, mask=0xFFFF, lin_damping=0.0, ang_damping=0.0, activation=0,
              kinematic=0):
    d = np.zeros(DESC)
    d[0] = shape
    d[1:4] = pos
    d[4:8] = quat
    d[8:11] = linvel
    d[11:14] = angvel
    d[14] = mass
    d[15] = friction
    d[16] = restitution
    d[17] = flags
    d[18] = group
    d[19] = mask
    d[20] = lin_damping
    d[21] = ang_damping
    d[22] = activation
    d[23] = kinematic
    return d


JDESC = 148   # joint descriptor doubles (orc_world_add_joint)
JOINT_POINT2POINT, JOINT_FIXED, JOINT_HINGE, JOINT_GEAR, JOINT_SLIDER, JOINT_CONETWIST = 0, 1, 2, 3, 4, 6
JF_DISABLE_COLLISIONS, JF_DISABLED, JF_ANGULAR_ONLY, JF_LIMIT, JF_MOTOR, JF_ERP = 1, 2, 4, 8, 16, 32
JF_LIN_MOTOR, JF_ANG_MOTOR, JF_FRAME_B = 64, 128, 256


def joint_desc(kind, body_a, body_b, frame_a, frame_b, flags=JF_DISABLE_COLLISIONS, erp=0.0, impulse_clamp=0.0,
               limit=(1.0, -1.0), softness=0.9, bias_factor=0.3, relaxation=1.0, motor=(0.0, 0.0), gear_ratio=1.0,
               lin_limits=(1.0, -1.0), ang_limits=(0.0, 0.0), slider_softness=(1.0, 1.0, 1.0, 1.0, 1.0, 1.0),
               lin_motor=(0.0, 0.0), ang_motor=(0.0, 0.0), rotate_order=0, s2_axes=None,
               cone=(1e30, 1e30, 1e30, 1.0, 0.3, 1.0), cone_motor=((0.0, 0.0, 0.0, 1.0), -1.0)):
    """frame_*: 12 numbers (origin xyz, basis columns x, y, z) in the body's frame; s2_axes: the
    (6, 14) spring-2 axis table (parameters in bgpu_spring2_axis field order, then the flags)."""
    d = np.zeros(JDESC)
    d[0], d[1], d[2], d[3] = kind, body_a, body_b, flags
    d[4:16] = frame_a
    d[16:28] = frame_b
    d[28], d[29] = erp, impulse_clamp
    d[30], d[31] = limit
    d[32], d[33], d[34] = softness, bias_factor, relaxation
    d[35], d[36] = motor
    d[37] = gear_ratio
    d[38], d[39] = lin_limits
    d[40], d[41] = ang_limits
    d[42:48] = slider_softness  # softness lim lin, lim ang, damping lim lin, lim ang, ortho lin, ortho ang
    d[48], d[49] = lin_motor
    d[50], d[51] = ang_motor
    d[52] = rotate_order
    d[137:143] = cone  # swing span 1, swing span 2, twist span, softness, bias factor, relaxation
    d[143:147] = cone_motor[0]
    d[147] = cone_motor[1]
    if s2_axes is not None:
        d[53:53 + 84] = np.asarray(s2_axes, dtype=np.float64).reshape(84)
    return d


def spring2_joint_desc(joint):
    """The oracle descriptor of a bgpu.Spring2 (kind 5) or bgpu.Generic6Dof (kind 7) joint: same
    bodies, frames, order and axes."""
    d = joint.desc
    return joint_desc(getattr(joint, "KIND", 5), d.body_a, d.body_b, list(d.frame_a), list(d.frame_b), flags=d.flags,
                      rotate_order=d.rotate_order, s2_axes=joint.axis_table())


def spring2_angle_info(tr_a, tr_b, order, precision="f32"):
    """generic6dof_spring2.rs:1164-1233: (Euler angles, 3 axes) of two 3x3 frames (numpy, row-major)."""
    out = np.zeros(12)
    a = np.ascontiguousarray(np.asarray(tr_a, dtype=np.float64).T.reshape(9))
    b = np.ascontiguousarray(np.asarray(tr_b, dtype=np.float64).T.reshape(9))
    lib().orc_spring2_angle_info(1 if precision == "f64" else 0, dptr(a), dptr(b), order, dptr(out))
    return out[:3], out[3:].reshape(3, 3)


def frame(origin, basis=np.eye(3)):
    """origin + basis (columns) as the 12 numbers of a joint descriptor frame."""
    b = np.asarray(basis, dtype=np.float64)
    return np.concatenate([np.asarray(origin, dtype=np.float64), b[:, 0], b[:, 1], b[:, 2]])


def hinge_frames(pivot_a, axis_a, pivot_b, axis_b, precision="f32"):
    """hinge.rs:60-100: the two hinge frames (12 numbers each) from pivots and axes."""
    out = np.zeros(24)
    lib().orc_hinge_frames(1 if precision == "f64" else 0, dptr(f64(pivot_a)), dptr(f64(axis_a)), dptr(f64(pivot_b)),
                           dptr(f64(axis_b)), dptr(out))
    return out[:12], out[12:]


class OracleWorld:
    """One oracle world (precision 'f32' or 'f64')."""

    def __init__(self, precision="f32"):
        self.L = lib()
        self.h = self.L.orc_world_new(1 if precision == "f64" else 0)
        self.precision = precision

    def __del__(self):
        try:
            if self.h:
                self.L.orc_world_free(self.h)
                self.h = None
        except Exception:
            pass

    def set_gravity(self, g):
        self.L.orc_world_set_gravity(self.h, *map(float, g))

    def set_solver(self, erp2=0.2, linear_slop=0.005, restitution_threshold=1.0, split_impulse=True,
                   split_threshold=-0.04, split_turn_erp=0.1, warmstarting_factor=0.85, global_cfm=0.0, sor=1.0,
                   num_iterations=10, erp=0.2, damping=1.0):
        s = f64([erp2, linear_slop, restitution_threshold, 1.0 if split_impulse else 0.0, split_threshold,
                 split_turn_erp, warmstarting_factor, global_cfm, sor, num_iterations, erp, damping])
        self.L.orc_world_set_solver(self.h, dptr(s))

    def set_brute_force(self, on=True):
        self.L.orc_world_set_brute_force(self.h, 1 if on else 0)

    def add_shape(self, kind, params=(), points=None):
        p = f64(list(params) + [0.0] * (4 - len(params)))
        if points is not None:
            pts = f64(np.asarray(points).reshape(-1, 3))
            return self.L.orc_world_add_shape(self.h, kind, dptr(p), dptr(pts), len(pts))
        return self.L.orc_world_add_shape(self.h, kind, dptr(p), None, 0)

    def sphere(self, r):
        return self.add_shape(SPHERE, [r])

    def box(self, h):
        return self.add_shape(BOX, list(h))

    def capsule(self, r, hh):
        return self.add_shape(CAPSULE, [r, hh])

    def plane(self, n, c):
        return self.add_shape(PLANE, list(n) + [c])

    def hull(self, pts):
        return self.add_shape(HULL, [], pts)

    def mesh(self, vertices, indices):
        """Static triangle mesh (triangle_mesh.rs:59-123): vertices n x 3, triangles m x 3."""
        v = f64(np.asarray(vertices).reshape(-1, 3))
        i = np.ascontiguousarray(np.asarray(indices).reshape(-1, 3), dtype=np.uint32)
        return self.L.orc_world_add_mesh(self.h, dptr(v), len(v), i.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                         len(i))

    def heightfield(self, heights, width, depth, cell=(1.0, 1.0, 1.0), options=0):
        """Heightfield (heightfield.rs:84-140); options: 1 flip quad edges, 2 diamond, 4 zigzag,
        8 flip winding, up axis << 4 (0 Y, the default; 1 X; 2 Z)."""
        h = f64(np.asarray(heights).reshape(-1))
        return self.L.orc_world_add_heightfield(self.h, dptr(h), width, depth, dptr(f64(cell)), options)

    def mesh_data(self, s):
        nv = ctypes.c_uint32(0)
        nt = self.L.orc_mesh_counts(self.h, s, ctypes.byref(nv))
        v = np.zeros((nv.value, 3))
        i = np.zeros((nt, 3), dtype=np.uint32)
        self.L.orc_mesh_data(self.h, s, dptr(v), i.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        return v, i

    def mesh_query(self, s, box6):
        out = np.zeros(4096, dtype=np.uint32)
        n = self.L.orc_mesh_query(self.h, s, dptr(f64(box6)), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                  len(out))
        return out[:n]

    def threshold(self, s):
        return self.L.orc_shape_threshold(self.h, s)

    def world_aabb(self, s, p):
        out = np.zeros(6)
        self.L.orc_shape_world_aabb(self.h, s, dptr(f64(p)), dptr(out))
        return out

    def inertia(self, s, mass):
        out = np.zeros(3)
        self.L.orc_shape_inertia(self.h, s, mass, dptr(out))
        return out

    def add_body(self, *args, **kw):
        d = f64(body_desc(*args, **kw))
        return self.L.orc_world_add_body(self.h, dptr(d))

    def add_desc(self, d):
        return self.L.orc_world_add_body(self.h, dptr(f64(d)))

    @property
    def num_bodies(self):
        return self.L.orc_world_num_bodies(self.h)

    def step(self, dt):
        self.L.orc_world_step(self.h, dt)

    def step_fixed(self, dt, max_sub_steps, fixed_dt):
        """step.rs:136-199; returns the unclamped substep demand."""
        return self.L.orc_world_step_fixed(self.h, dt, max_sub_steps, fixed_dt)

    def state(self):
        out = np.zeros((self.num_bodies, STATE))
        self.L.orc_world_get_state(self.h, dptr(out))
        return out

    def set_state(self, s):
        s = f64(s)
        self.L.orc_world_set_state(self.h, dptr(s))

    def apply_force(self, i, force, torque=(0.0, 0.0, 0.0)):
        f, t = f64(force), f64(torque)
        self.L.orc_world_apply_force(self.h, int(i), dptr(f), dptr(t))

    def set_filter(self, i, group, mask):
        self.L.orc_world_set_filter(self.h, int(i), int(group), int(mask))

    def push(self):
        out = np.zeros((self.num_bodies, 6))
        self.L.orc_world_get_push(self.h, dptr(out))
        return out

    def pairs(self):
        n = self.L.orc_world_num_pairs(self.h)
        out = np.zeros((n, 2), dtype=np.uint32)
        if n:
            self.L.orc_world_get_pairs(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        return out

    def rows(self, pre=False):
        n = self.L.orc_world_num_rows(self.h)
        out = np.zeros((n, ROW))
        if n:
            self.L.orc_world_get_rows(self.h, 1 if pre else 0, dptr(out))
        return out

    def narrowphase_calls(self):
        return self.L.orc_world_narrowphase_calls(self.h)

    def num_manifolds(self):
        return self.L.orc_world_num_manifolds(self.h)

    def stage_seconds(self):
        out = np.zeros(7)
        self.L.orc_world_stage_seconds(self.h, dptr(out))
        return out

    def add_joint(self, desc):
        return self.L.orc_world_add_joint(self.h, dptr(f64(desc)))

    def set_joint_flags(self, j, flags):
        """JF_DISABLE_COLLISIONS / JF_DISABLED of joint j, between steps."""
        self.L.orc_world_set_joint_flags(self.h, int(j), int(flags))

    def set_joint_order(self, ids):
        a = np.ascontiguousarray(ids, dtype=np.uint32)
        self.L.orc_world_set_joint_order(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(a))

    def joint_angles(self, n):
        out = np.zeros(n)
        self.L.orc_world_joint_angles(self.h, dptr(out))
        return out

    def joint_positions(self, n):
        out = np.zeros(n)
        self.L.orc_world_joint_positions(self.h, dptr(out))
        return out

    def set_ccd(self, i, threshold, radius):
        self.L.orc_world_set_ccd(self.h, i, threshold, radius)

    def ccd_clamps(self):
        out = np.ones(self.num_bodies)
        self.L.orc_world_ccd_clamps(self.h, dptr(out))
        return out

    def spring2_state(self, n):
        out = np.zeros((n, 8))
        if n:
            self.L.orc_world_joint_spring2_state(self.h, dptr(out))
        return out

    def joint_rows(self):
        n = self.L.orc_world_num_joint_rows(self.h)
        out = np.zeros((n, 8))
        if n:
            self.L.orc_world_joint_rows(self.h, dptr(out))
        return out

    def set_solve_order(self, keys):
        k = np.ascontiguousarray(keys, dtype=np.uint64)
        self.L.orc_world_set_solve_order(self.h, k.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(k))

    def collide(self, sa, pa, sb, pb, seed=None):
        out = np.zeros((8, 7))
        sd = dptr(f64(seed)) if seed is not None else None
        n = self.L.orc_collide(self.h, sa, dptr(f64(pa)), sb, dptr(f64(pb)), sd, dptr(out))
        return out[:n]

    def convex_convex(self, sa, pa, sb, pb):
        out = np.zeros(7)
        n = self.L.orc_convex_convex(self.h, sa, dptr(f64(pa)), sb, dptr(f64(pb)), dptr(out))
        return out if n else None

    def gjk_kind(self, sa, pa, sb, pb):
        return self.L.orc_gjk_kind(self.h, sa, dptr(f64(pa)), sb, dptr(f64(pb)))

    def gjk_contact(self, sa, pa, sb, pb, threshold, seed=None):
        """gjk.rs:171-288: (kind 0 separated / 1 band / 2 overlap, distance, normal, point_on_b,
        overlap simplex point count)."""
        out = np.zeros(8)
        sd = dptr(f64(seed)) if seed is not None else None
        k = self.L.orc_gjk_contact(self.h, sa, dptr(f64(pa)), sb, dptr(f64(pb)), sd, float(threshold), dptr(out))
        return k, out[0], out[1:4], out[4:7], int(out[7])

    def solve_contacts(self, contacts, inv_dt):
        c = f64(np.asarray(contacts).reshape(-1, 10))
        out = np.zeros((len(c), ROW))
        self.L.orc_solve_contacts(self.h, dptr(c), len(c), inv_dt, dptr(out))
        return out


def oracle_pairs(aabbs, method=0, precision="f32"):
    """Pairs of an (n, 6) AABB array: method 0 brute force, 1 sweep."""
    a = f64(np.asarray(aabbs).reshape(-1, 6))
    L = lib()
    n = L.orc_pairs(1 if precision == "f64" else 0, dptr(a), len(a), method, None, 0)
    out = np.zeros((n, 2), dtype=np.uint32)
    if n:
        L.orc_pairs(1 if precision == "f64" else 0, dptr(a), len(a), method,
                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n)
    return out


def manifold_reduce(points, keep, precision="f32"):
    """manifold.rs:80-108 ContactManifold::reduce on rows (pos3, normal3, penetration)."""
    p = f64(np.asarray(points).reshape(-1, 7))
    out = np.zeros((max(len(p), 1), 7))
    n = lib().orc_manifold_reduce(1 if precision == "f64" else 0, dptr(p), len(p), keep, dptr(out))
    return out[:n]


class OracleManifold:
    def __init__(self, precision="f32"):
        self.L = lib()
        self.h = self.L.orc_pm_new(1 if precision == "f64" else 0)

    def __del__(self):
        try:
            if self.h:
                self.L.orc_pm_free(self.h)
                self.h = None
        except Exception:
            pass

    def capture(self, points, pa, pb, thr):
        p = f64(np.asarray(points).reshape(-1, 7))
        self.L.orc_pm_capture(self.h, dptr(p), len(p), dptr(f64(pa)), dptr(f64(pb)), thr)

    def refresh(self, pa, pb):
        out = np.zeros((16, 9))
        n = self.L.orc_pm_refresh(self.h, dptr(f64(pa)), dptr(f64(pb)), dptr(out))
        return out[:n]

    def needs_redetect(self, pa, pb):
        return bool(self.L.orc_pm_needs_redetect(self.h, dptr(f64(pa)), dptr(f64(pb))))

    def set_impulse(self, k, v):
        self.L.orc_pm_set_impulse(self.h, k, v)

    def points(self):
        out = np.zeros((16, 12))
        n = self.L.orc_pm_points(self.h, dptr(out))
        return out[:n]


def interpolate_pose(pos, quat, linvel, angvel, dt, precision="f32"):
    inp = f64(list(pos) + list(quat) + list(linvel) + list(angvel))
    out = np.zeros(7)
    lib().orc_interpolate_pose(1 if precision == "f64" else 0, dptr(inp), dt, dptr(out))
    return out


def sphere_triangle(center, radius, threshold, a, b, c, precision="f32"):
    """convex_mesh.rs:160-232: (point, normal toward the centre, penetration) or None."""
    out = np.zeros(7)
    tri = f64(np.concatenate([a, b, c]))
    n = lib().orc_sphere_triangle(1 if precision == "f64" else 0, dptr(f64(center)), radius, threshold, dptr(tri),
                                  dptr(out))
    return (out[0:3], out[3:6], out[6]) if n else None
