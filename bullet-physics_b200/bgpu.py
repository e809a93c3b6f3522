"""ctypes binding of libbgpu.so (the C ABI in include/bgpu.h).

The product is the C ABI; this module is a thin caller used by the tests,
the benchmark and the smoke entry. It refuses to run without the compiled
library: there is no fallback implementation.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbgpu.so")

SPHERE, BOX, CAPSULE, HULL, PLANE, MESH = 0, 1, 2, 3, 4, 5
HF_FLIP_QUAD_EDGES, HF_DIAMOND, HF_ZIGZAG, HF_FLIP_WINDING = 1, 2, 4, 8
HF_UP_Y, HF_UP_X, HF_UP_Z = 0, 16, 32
JOINT_POINT2POINT, JOINT_FIXED, JOINT_HINGE, JOINT_GEAR, JOINT_SLIDER = 0, 1, 2, 3, 4
JOINT_DISABLE_COLLISIONS, JOINT_DISABLED, JOINT_ANGULAR_ONLY, JOINT_LIMIT, JOINT_MOTOR, JOINT_ERP = 1, 2, 4, 8, 16, 32
JOINT_LIN_MOTOR, JOINT_ANG_MOTOR, JOINT_FRAME_B = 64, 128, 256
JOINT_SPRING2, JOINT_CONETWIST, JOINT_CONE_MOTOR, JOINT_GENERIC6DOF = 5, 6, 512, 7
ROTATE_XYZ, ROTATE_XZY, ROTATE_YXZ, ROTATE_YZX, ROTATE_ZXY, ROTATE_ZYX = range(6)
(S2_MOTOR, S2_SERVO, S2_SPRING, S2_STIFFNESS_LIMITED, S2_DAMPING_LIMITED, S2_STOP_ERP, S2_STOP_CFM, S2_MOTOR_ERP,
 S2_MOTOR_CFM) = (1, 2, 4, 8, 16, 32, 64, 128, 256)
NO_CONTACT_RESPONSE, DISABLE_WORLD_GRAVITY, KINEMATIC, ADDITIONAL_DAMPING = 0x1, 0x2, 0x4, 0x10
STATE = 15
CONTACT = 18


class SolverInfo(ctypes.Structure):
    _fields_ = [("erp2", ctypes.c_float), ("linear_slop", ctypes.c_float),
                ("restitution_velocity_threshold", ctypes.c_float), ("split_impulse", ctypes.c_uint32),
                ("split_impulse_penetration_threshold", ctypes.c_float), ("split_impulse_turn_erp", ctypes.c_float),
                ("warmstarting_factor", ctypes.c_float), ("global_cfm", ctypes.c_float), ("sor", ctypes.c_float),
                ("num_iterations", ctypes.c_uint32), ("erp", ctypes.c_float), ("damping", ctypes.c_float)]


class JointDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("body_a", ctypes.c_uint32), ("body_b", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("frame_a", ctypes.c_float * 12), ("frame_b", ctypes.c_float * 12),
                ("erp", ctypes.c_float), ("impulse_clamp", ctypes.c_float), ("limit_low", ctypes.c_float),
                ("limit_high", ctypes.c_float), ("limit_softness", ctypes.c_float),
                ("limit_bias_factor", ctypes.c_float), ("limit_relaxation", ctypes.c_float),
                ("motor_target_velocity", ctypes.c_float), ("motor_max_impulse", ctypes.c_float),
                ("gear_ratio", ctypes.c_float), ("lin_limit_low", ctypes.c_float), ("lin_limit_high", ctypes.c_float),
                ("ang_limit_low", ctypes.c_float), ("ang_limit_high", ctypes.c_float),
                ("softness_lim_lin", ctypes.c_float), ("softness_lim_ang", ctypes.c_float),
                ("damping_lim_lin", ctypes.c_float), ("damping_lim_ang", ctypes.c_float),
                ("softness_ortho_lin", ctypes.c_float), ("softness_ortho_ang", ctypes.c_float),
                ("lin_motor_target_velocity", ctypes.c_float), ("lin_motor_max_force", ctypes.c_float),
                ("ang_motor_target_velocity", ctypes.c_float), ("ang_motor_max_force", ctypes.c_float),
                ("swing_span1", ctypes.c_float), ("swing_span2", ctypes.c_float), ("twist_span", ctypes.c_float),
                ("cone_softness", ctypes.c_float), ("cone_bias_factor", ctypes.c_float),
                ("cone_relaxation", ctypes.c_float), ("cone_motor_target", ctypes.c_float * 4),
                ("cone_motor_max_impulse", ctypes.c_float)]


class Spring2Axis(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("lower_limit", "upper_limit", "bounce", "stop_erp", "stop_cfm",
                                              "motor_erp", "motor_cfm", "target_velocity", "max_motor_force",
                                              "servo_target", "stiffness", "damping", "equilibrium_point")] + \
        [("flags", ctypes.c_uint32)]


class Spring2Desc(ctypes.Structure):
    _fields_ = [("body_a", ctypes.c_uint32), ("body_b", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("rotate_order", ctypes.c_uint32), ("frame_a", ctypes.c_float * 12), ("frame_b", ctypes.c_float * 12),
                ("axis", Spring2Axis * 6)]


_PI = np.float32(np.pi)
_TWO_PI = np.float32(2.0) * _PI


def _normalize_angle(angle):
    """shared.rs:17-27 (normalize_angle) in f32."""
    a = np.fmod(np.float32(angle), _TWO_PI)
    if a < -_PI:
        a = np.float32(a + _TWO_PI)
    elif a > _PI:
        a = np.float32(a - _TWO_PI)
    return float(a)


class Spring2:
    """One generic 6DOF spring-2 joint (Generic6DofSpring2Constraint, generic6dof_spring2.rs:259-650)
    with the reference's setters: axes 0-2 linear, 3-5 angular. Starts from Bullet's defaults
    (linear locked, angular free), so a fresh joint is a ball joint."""

    def __init__(self, body_a, body_b, frame_a=None, frame_b=None, rotate_order=ROTATE_XYZ,
                 flags=JOINT_DISABLE_COLLISIONS):
        self.desc = Spring2Desc()
        lib().bgpu_spring2_desc_default(ctypes.byref(self.desc))
        d = self.desc
        d.body_a, d.body_b, d.flags, d.rotate_order = body_a, body_b, flags, rotate_order
        if frame_a is not None:
            d.frame_a[:] = [float(x) for x in frame_a]
        if frame_b is not None:
            d.frame_b[:] = [float(x) for x in frame_b]

    @classmethod
    def hinge2(cls, body_a, body_b, pos_a, quat_a, pos_b, quat_b, anchor, axis1, axis2):
        """Generic6DofSpring2Constraint::hinge2 (PhysicsWorld::add_hinge2) from the bodies' poses."""
        j = cls.__new__(cls)
        j.desc = Spring2Desc()
        args = [f32(v) for v in (pos_a, quat_a, pos_b, quat_b, anchor, axis1, axis2)]
        check(lib().bgpu_spring2_hinge2(*[fptr(a) for a in args], body_a, body_b, ctypes.byref(j.desc)), "hinge2")
        return j

    def axis(self, i):
        return self.desc.axis[i]

    def set_linear_limits(self, lower, upper):
        for i in range(3):
            self.desc.axis[i].lower_limit, self.desc.axis[i].upper_limit = lower[i], upper[i]

    def set_angular_limits(self, lower, upper):
        for i in range(3):
            a = self.desc.axis[3 + i]
            a.lower_limit, a.upper_limit = _normalize_angle(lower[i]), _normalize_angle(upper[i])

    def set_limit(self, axis, lo, hi):
        a = self.desc.axis[axis]
        if axis < 3:
            a.lower_limit, a.upper_limit = lo, hi
        else:
            a.lower_limit, a.upper_limit = _normalize_angle(lo), _normalize_angle(hi)

    def set_limit_reversed(self, axis, lo, hi):
        a = self.desc.axis[axis]
        if axis < 3:
            a.lower_limit, a.upper_limit = lo, hi
        else:
            a.upper_limit, a.lower_limit = _normalize_angle(-lo), _normalize_angle(-hi)

    def set_rotation_order(self, order):
        self.desc.rotate_order = order

    def set_bounce(self, axis, bounce):
        self.desc.axis[axis].bounce = bounce

    def _flag(self, axis, bit, on):
        a = self.desc.axis[axis]
        a.flags = (a.flags | bit) if on else (a.flags & ~bit)

    def enable_motor(self, axis, on=True):
        self._flag(axis, S2_MOTOR, on)

    def set_servo(self, axis, on=True):
        self._flag(axis, S2_SERVO, on)

    def set_target_velocity(self, axis, velocity):
        self.desc.axis[axis].target_velocity = velocity

    def set_servo_target(self, axis, target):
        """Angular targets wrap into [-pi, pi] (generic6dof_spring2.rs:489-514), in f32."""
        if axis < 3:
            self.desc.axis[axis].servo_target = target
            return
        t = np.float32(np.float32(target) + _PI)
        m = np.fmod(t, _TWO_PI)
        if m >= _TWO_PI:
            t = np.float32(0.0)
        elif m < 0:
            t = np.float32(0.0) if np.float32(_TWO_PI + m) == _TWO_PI else np.float32(_TWO_PI + m)
        else:
            t = m
        self.desc.axis[axis].servo_target = float(np.float32(t - _PI))

    def set_max_motor_force(self, axis, force):
        self.desc.axis[axis].max_motor_force = force

    def enable_spring(self, axis, on=True):
        self._flag(axis, S2_SPRING, on)

    def set_stiffness(self, axis, stiffness, limit_needed=True):
        self.desc.axis[axis].stiffness = stiffness
        self._flag(axis, S2_STIFFNESS_LIMITED, limit_needed)

    def set_damping(self, axis, damping, limit_needed=True):
        self.desc.axis[axis].damping = damping
        self._flag(axis, S2_DAMPING_LIMITED, limit_needed)

    def set_equilibrium_point(self, axis, value):
        self.desc.axis[axis].equilibrium_point = value

    def set_stop_erp(self, axis, value):
        self.desc.axis[axis].stop_erp = value
        self._flag(axis, S2_STOP_ERP, True)

    def set_stop_cfm(self, axis, value):
        self.desc.axis[axis].stop_cfm = value
        self._flag(axis, S2_STOP_CFM, True)

    def set_motor_erp(self, axis, value):
        self.desc.axis[axis].motor_erp = value
        self._flag(axis, S2_MOTOR_ERP, True)

    def set_motor_cfm(self, axis, value):
        self.desc.axis[axis].motor_cfm = value
        self._flag(axis, S2_MOTOR_CFM, True)

    def axis_table(self):
        """(6, 14) array: per axis the 13 parameters in field order, then the flags."""
        return np.array([[getattr(a, f) for f, _ in Spring2Axis._fields_] for a in self.desc.axis], dtype=np.float64)


class Generic6Dof(Spring2):
    """One classic generic 6DOF joint (Generic6DofConstraint, generic6dof.rs:131-262) with the
    reference's setters; defaults are Bullet's (linear locked at 0, angular free)."""
    KIND = JOINT_GENERIC6DOF

    def __init__(self, body_a, body_b, frame_a=None, frame_b=None, flags=JOINT_DISABLE_COLLISIONS):
        super().__init__(body_a, body_b, frame_a, frame_b, ROTATE_XYZ, flags)

    @classmethod
    def universal(cls, body_a, body_b, pos_a, quat_a, pos_b, quat_b, anchor, axis1, axis2):
        """Generic6DofConstraint::universal (PhysicsWorld::add_universal) from the bodies' poses."""
        j = cls.__new__(cls)
        j.desc = Spring2Desc()
        args = [f32(v) for v in (pos_a, quat_a, pos_b, quat_b, anchor, axis1, axis2)]
        check(lib().bgpu_generic6dof_universal(*[fptr(a) for a in args], body_a, body_b, ctypes.byref(j.desc)),
              "universal")
        return j

    def enable_motor(self, axis, target_velocity, max_force):
        a = self.desc.axis[axis]
        a.target_velocity, a.max_motor_force = target_velocity, max_force
        self._flag(axis, S2_MOTOR, True)

    def disable_motor(self, axis):
        self._flag(axis, S2_MOTOR, False)


class BodyDesc(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_uint32), ("position", ctypes.c_float * 3), ("orientation", ctypes.c_float * 4),
                ("linear_velocity", ctypes.c_float * 3), ("angular_velocity", ctypes.c_float * 3),
                ("mass", ctypes.c_float), ("friction", ctypes.c_float), ("restitution", ctypes.c_float),
                ("linear_damping", ctypes.c_float), ("angular_damping", ctypes.c_float), ("flags", ctypes.c_uint32),
                ("group", ctypes.c_uint16), ("mask", ctypes.c_uint16), ("activation", ctypes.c_uint32),
                ("linear_sleeping_threshold", ctypes.c_float), ("angular_sleeping_threshold", ctypes.c_float)]


class StepStats(ctypes.Structure):
    _fields_ = [("num_bodies", ctypes.c_uint32), ("num_pairs", ctypes.c_uint32),
                ("num_contact_pairs", ctypes.c_uint32), ("num_contacts", ctypes.c_uint32),
                ("num_colours", ctypes.c_uint32), ("num_detect", ctypes.c_uint32), ("num_manifolds", ctypes.c_uint32),
                ("device_status", ctypes.c_uint32), ("num_split_pairs", ctypes.c_uint32),
                ("timed_steps", ctypes.c_uint32), ("stage_ms", ctypes.c_float * 7), ("solve_kernel_ms", ctypes.c_float),
                ("step_ms", ctypes.c_float), ("num_split_contacts", ctypes.c_uint32)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("threads_per_cta", ctypes.c_uint32), ("warp_world_max_bodies", ctypes.c_uint32),
                ("ctas", ctypes.c_uint32), ("candidates", ctypes.c_uint32), ("ms_per_step", ctypes.c_float),
                ("global_ms_per_step", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


# numpy view of bgpu_body_desc (96 bytes), for building many descriptors at once
DESC_DTYPE = np.dtype([("shape", "<u4"), ("position", "<f4", 3), ("orientation", "<f4", 4),
                       ("linear_velocity", "<f4", 3), ("angular_velocity", "<f4", 3), ("mass", "<f4"),
                       ("friction", "<f4"), ("restitution", "<f4"), ("linear_damping", "<f4"),
                       ("angular_damping", "<f4"), ("flags", "<u4"), ("group", "<u2"), ("mask", "<u2"),
                       ("activation", "<u4"), ("linear_sleeping_threshold", "<f4"),
                       ("angular_sleeping_threshold", "<f4")])
assert DESC_DTYPE.itemsize == ctypes.sizeof(BodyDesc)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        F = ctypes.POINTER(ctypes.c_float)
        U32 = ctypes.c_uint32
        U32P = ctypes.POINTER(ctypes.c_uint32)
        U64P = ctypes.POINTER(ctypes.c_uint64)
        S = ctypes.c_int32
        sig = {
            "bgpu_version": (ctypes.c_char_p, []),
            "bgpu_device_count": (ctypes.c_int, []),
            "bgpu_set_device": (S, [ctypes.c_int]),
            "bgpu_last_error": (ctypes.c_size_t, [ctypes.c_char_p, ctypes.c_size_t]),
            "bgpu_solver_info_default": (None, [ctypes.POINTER(SolverInfo)]),
            "bgpu_body_desc_default": (None, [ctypes.POINTER(BodyDesc)]),
            "bgpu_world_create": (S, [ctypes.POINTER(SolverInfo), F, ctypes.POINTER(P)]),
            "bgpu_world_destroy": (None, [P]),
            "bgpu_world_set_gravity": (S, [P, F]),
            "bgpu_world_set_solver_info": (S, [P, ctypes.POINTER(SolverInfo)]),
            "bgpu_add_shape": (S, [P, U32, F, F, U32, U32P]),
            "bgpu_add_bodies": (S, [P, U32, ctypes.POINTER(BodyDesc), U32P]),
            "bgpu_add_mesh_shape": (S, [P, F, U32, U32P, U32, U32P]),
            "bgpu_add_heightfield_shape": (S, [P, F, U32, U32, F, U32, U32P]),
            "bgpu_num_bodies": (U32, [P]),
            "bgpu_step": (S, [P, ctypes.c_float, U32]),
            "bgpu_step_simulation_fixed": (S, [P, ctypes.c_float, U32, ctypes.c_float, U32P]),
            "bgpu_step_timed": (S, [P, ctypes.c_float, U32, F]),
            "bgpu_read_state": (S, [P, F]),
            "bgpu_write_state": (S, [P, F]),
            "bgpu_read_poses": (S, [P, F]),
            "bgpu_apply_forces": (S, [P, F, F]),
            "bgpu_read_pairs": (S, [P, U32P, ctypes.c_uint64, U64P]),
            "bgpu_read_contacts": (S, [P, F, ctypes.c_uint64, U64P]),
            "bgpu_read_solve_order": (S, [P, U64P, ctypes.c_uint64, U64P]),
            "bgpu_read_colour_batches": (S, [P, U32P, U32P, U32, U32P]),
            "bgpu_selftest_wait_timeout": (S, [U32, U32P, F]),
            "bgpu_joint_desc_default": (None, [ctypes.POINTER(JointDesc)]),
            "bgpu_add_joints": (S, [P, U32, ctypes.POINTER(JointDesc), U32P]),
            "bgpu_spring2_desc_default": (None, [ctypes.POINTER(Spring2Desc)]),
            "bgpu_spring2_hinge2": (S, [F, F, F, F, F, F, F, U32, U32, ctypes.POINTER(Spring2Desc)]),
            "bgpu_add_spring2_joints": (S, [P, U32, ctypes.POINTER(Spring2Desc), U32P]),
            "bgpu_read_joint_spring2_state": (S, [P, F]),
            "bgpu_add_generic6dof_joints": (S, [P, U32, ctypes.POINTER(Spring2Desc), U32P]),
            "bgpu_generic6dof_universal": (S, [F, F, F, F, F, F, F, U32, U32, ctypes.POINTER(Spring2Desc)]),
            "bgpu_set_ccd": (S, [P, U32, U32, F, F]),
            "bgpu_read_ccd_clamps": (S, [P, F]),
            "bgpu_num_joints": (U32, [P]),
            "bgpu_set_joint_flags": (S, [P, U32, U32]),
            "bgpu_read_joint_angles": (S, [P, F]),
            "bgpu_read_joint_positions": (S, [P, F]),
            "bgpu_read_joint_order": (S, [P, U32P, U32, U32P]),
            "bgpu_read_joint_rows": (S, [P, F, U32, U32P]),
            "bgpu_get_stats": (S, [P, ctypes.POINTER(StepStats)]),
            "bgpu_enable_step_timing": (S, [P, ctypes.c_int]),
            "bgpu_broadphase_pairs": (S, [F, U32, U32P, ctypes.c_uint64, U64P]),
            "bgpu_collide": (S, [P, U32, U32P, F, U32P, F, F, ctypes.c_int, F, U32P]),
            "bgpu_solve_contacts": (S, [P, U32, F, ctypes.c_float, F, U64P]),
            "bgpu_read_push": (S, [P, F]),
            "bgpu_batch_create": (S, [ctypes.POINTER(SolverInfo), F, ctypes.POINTER(P)]),
            "bgpu_batch_add_worlds": (S, [P, U32, U32P, ctypes.c_void_p, U32P]),
            "bgpu_batch_num_worlds": (U32, [P]),
            "bgpu_batch_world_offsets": (S, [P, U32P]),
            "bgpu_batch_step": (S, [P, ctypes.c_float, U32]),
            "bgpu_batch_autotune": (S, [P, ctypes.c_float, U32, ctypes.POINTER(BatchTuning)]),
            "bgpu_batch_set_tuning": (S, [P, U32, U32]),
            "bgpu_batch_get_tuning": (S, [P, ctypes.POINTER(BatchTuning)]),
            "bgpu_tape_create": (S, [P, U32, ctypes.POINTER(P)]),
            "bgpu_tape_destroy": (None, [P]),
            "bgpu_tape_forward": (S, [P, ctypes.c_float, U32]),
            "bgpu_tape_backward": (S, [P, F, F, F, F, F]),
            "bgpu_tape_timing": (S, [P, F, F]),
            "bgpu_tape_rewind": (S, [P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class BgpuError(RuntimeError):
    pass


def last_error():
    buf = ctypes.create_string_buffer(512)
    lib().bgpu_last_error(buf, 512)
    return buf.value.decode()


def check(status, what=""):
    if status != 0:
        raise BgpuError(f"{what}: status {status}: {last_error()}")


def fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def u32ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def u64ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def device_count():
    return lib().bgpu_device_count()


def set_device(device):
    """Makes `device` the calling thread's device for the library (bgpu_set_device)."""
    check(lib().bgpu_set_device(int(device)), "set_device")


def selftest_wait_timeout(limit_ms):
    """Runs a device wait that nothing completes; returns (device status bits, device ms)."""
    st = ctypes.c_uint32()
    ms = ctypes.c_float()
    check(lib().bgpu_selftest_wait_timeout(int(limit_ms), ctypes.byref(st), ctypes.byref(ms)), "selftest_wait_timeout")
    return st.value, ms.value


def solver_info(**kw):
    s = SolverInfo()
    lib().bgpu_solver_info_default(ctypes.byref(s))
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def body_descs(n):
    arr = (BodyDesc * n)()
    for i in range(n):
        lib().bgpu_body_desc_default(ctypes.byref(arr[i]))
    return arr


def desc_array(shape, pos, quat, linvel=None, angvel=None, mass=None, friction=None, restitution=None):
    """bgpu_body_desc records for n bodies from numpy arrays (n,), (n,3), (n,4); other fields default."""
    n = len(shape)
    base = body_descs(1)
    d = np.repeat(np.frombuffer(bytes(base), dtype=DESC_DTYPE), n)
    d["shape"] = np.asarray(shape, dtype=np.uint32)
    d["position"] = np.asarray(pos, dtype=np.float32).reshape(n, 3)
    d["orientation"] = np.asarray(quat, dtype=np.float32).reshape(n, 4)
    if linvel is not None:
        d["linear_velocity"] = np.asarray(linvel, dtype=np.float32).reshape(n, 3)
    if angvel is not None:
        d["angular_velocity"] = np.asarray(angvel, dtype=np.float32).reshape(n, 3)
    if mass is not None:
        d["mass"] = np.asarray(mass, dtype=np.float32)
    if friction is not None:
        d["friction"] = np.asarray(friction, dtype=np.float32)
    if restitution is not None:
        d["restitution"] = np.asarray(restitution, dtype=np.float32)
    return d


class World:
    """One world, or with batch=True a batch of independent worlds (bgpu_batch_*)."""

    def __init__(self, gravity=(0.0, -9.81, 0.0), batch=False, **info):
        self.L = lib()
        self.h = ctypes.c_void_p()
        g = f32(gravity)
        s = solver_info(**info)
        create = self.L.bgpu_batch_create if batch else self.L.bgpu_world_create
        check(create(ctypes.byref(s), fptr(g), ctypes.byref(self.h)), "bgpu_world_create")
        self.batch = batch

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.bgpu_world_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_solver(self, **info):
        s = solver_info(**info)
        check(self.L.bgpu_world_set_solver_info(self.h, ctypes.byref(s)), "set_solver_info")

    def set_gravity(self, g):
        check(self.L.bgpu_world_set_gravity(self.h, fptr(f32(g))), "set_gravity")

    def add_shape(self, kind, params=(), points=None):
        p = f32(list(params) + [0.0] * (4 - len(params)))
        out = ctypes.c_uint32()
        if points is not None:
            pts = f32(np.asarray(points).reshape(-1, 3))
            check(self.L.bgpu_add_shape(self.h, kind, fptr(p), fptr(pts), len(pts), ctypes.byref(out)), "add_shape")
        else:
            check(self.L.bgpu_add_shape(self.h, kind, fptr(p), None, 0, ctypes.byref(out)), "add_shape")
        return out.value

    def mesh(self, vertices, indices):
        """Static triangle mesh: vertices n x 3, triangles m x 3 vertex indices."""
        v = f32(np.asarray(vertices).reshape(-1, 3))
        i = np.ascontiguousarray(np.asarray(indices).reshape(-1, 3), dtype=np.uint32)
        out = ctypes.c_uint32()
        check(self.L.bgpu_add_mesh_shape(self.h, fptr(v), len(v), u32ptr(i), len(i), ctypes.byref(out)), "add_mesh")
        return out.value

    def heightfield(self, heights, width, depth, cell=(1.0, 1.0, 1.0), options=0):
        """Static heightfield (width x depth row-major heights) built into a triangle mesh."""
        h = f32(np.asarray(heights).reshape(-1))
        out = ctypes.c_uint32()
        check(self.L.bgpu_add_heightfield_shape(self.h, fptr(h), width, depth, fptr(f32(cell)), options,
                                                ctypes.byref(out)), "add_heightfield")
        return out.value

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

    def add_descs(self, descs):
        out = ctypes.c_uint32()
        check(self.L.bgpu_add_bodies(self.h, len(descs), descs, ctypes.byref(out)), "add_bodies")
        return out.value

    def add_body(self, shape, pos, quat=(0, 0, 0, 1), linvel=(0, 0, 0), angvel=(0, 0, 0), mass=1.0, friction=0.5,
                 restitution=0.0, flags=0, group=1, mask=0xFFFF, lin_damping=0.0, ang_damping=0.0, activation=0,
                 kinematic=0):
        d = body_descs(1)
        b = d[0]
        b.shape = shape
        b.position[:] = list(map(float, pos))
        b.orientation[:] = list(map(float, quat))
        b.linear_velocity[:] = list(map(float, linvel))
        b.angular_velocity[:] = list(map(float, angvel))
        b.mass = mass
        b.friction = friction
        b.restitution = restitution
        b.flags = flags | (KINEMATIC if kinematic else 0)
        b.group = group
        b.mask = mask
        b.linear_damping = lin_damping
        b.angular_damping = ang_damping
        b.activation = activation
        return self.add_descs(d)

    def add_bodies_array(self, shape, pos, quat, linvel=None, angvel=None, mass=None, friction=None,
                         restitution=None):
        """Vectorised insertion from numpy arrays (n,), (n,3), (n,4)."""
        d = desc_array(shape, pos, quat, linvel, angvel, mass, friction, restitution)
        out = ctypes.c_uint32()
        check(self.L.bgpu_add_bodies(self.h, len(d), d.ctypes.data_as(ctypes.POINTER(BodyDesc)), ctypes.byref(out)),
              "add_bodies")
        return out.value

    def add_worlds_array(self, bodies_per_world, shape, pos, quat, linvel=None, angvel=None, mass=None,
                         friction=None, restitution=None):
        """Batched worlds: append worlds whose bodies follow each other in the arrays."""
        counts = np.ascontiguousarray(bodies_per_world, dtype=np.uint32)
        d = desc_array(shape, pos, quat, linvel, angvel, mass, friction, restitution)
        assert len(d) == int(counts.sum())
        out = ctypes.c_uint32()
        check(self.L.bgpu_batch_add_worlds(self.h, len(counts), u32ptr(counts), d.ctypes.data, ctypes.byref(out)),
              "batch_add_worlds")
        return out.value

    def autotune(self, dt, steps_per_candidate=3):
        """Batched worlds: time the solver's launch shapes from the current state, keep the fastest."""
        t = BatchTuning()
        check(self.L.bgpu_batch_autotune(self.h, dt, steps_per_candidate, ctypes.byref(t)), "batch_autotune")
        return t.as_dict()

    def set_tuning(self, threads_per_cta, warp_world_max_bodies=64):
        check(self.L.bgpu_batch_set_tuning(self.h, threads_per_cta, warp_world_max_bodies), "batch_set_tuning")

    def tuning(self):
        t = BatchTuning()
        check(self.L.bgpu_batch_get_tuning(self.h, ctypes.byref(t)), "batch_get_tuning")
        return t.as_dict()

    @property
    def num_worlds(self):
        return self.L.bgpu_batch_num_worlds(self.h)

    def world_offsets(self):
        out = np.zeros(self.num_worlds + 1, dtype=np.uint32)
        check(self.L.bgpu_batch_world_offsets(self.h, u32ptr(out)), "batch_world_offsets")
        return out

    @property
    def num_bodies(self):
        return self.L.bgpu_num_bodies(self.h)

    def step(self, dt, n=1):
        check(self.L.bgpu_step(self.h, dt, n), "bgpu_step")

    def step_timed(self, dt, n):
        """Runs n steps; returns the device time (ms) measured on the world's stream."""
        ms = ctypes.c_float()
        check(self.L.bgpu_step_timed(self.h, dt, n, ctypes.byref(ms)), "bgpu_step_timed")
        return ms.value

    def step_fixed(self, dt, max_sub_steps, fixed_dt):
        out = ctypes.c_uint32()
        check(self.L.bgpu_step_simulation_fixed(self.h, dt, max_sub_steps, fixed_dt, ctypes.byref(out)), "step_fixed")
        return out.value

    def state(self):
        out = np.zeros((self.num_bodies, STATE), dtype=np.float32)
        check(self.L.bgpu_read_state(self.h, fptr(out)), "read_state")
        return out

    def set_state(self, s):
        s = f32(s)
        check(self.L.bgpu_write_state(self.h, fptr(s)), "write_state")

    def poses(self, out=None):
        if out is None:
            out = np.zeros((self.num_bodies, 7), dtype=np.float32)
        check(self.L.bgpu_read_poses(self.h, fptr(out)), "read_poses")
        return out

    def apply_forces(self, force=None, torque=None):
        f = fptr(f32(force)) if force is not None else None
        t = fptr(f32(torque)) if torque is not None else None
        check(self.L.bgpu_apply_forces(self.h, f, t), "apply_forces")

    def pairs(self):
        n = ctypes.c_uint64()
        check(self.L.bgpu_read_pairs(self.h, None, 0, ctypes.byref(n)), "read_pairs")
        out = np.zeros((n.value, 2), dtype=np.uint32)
        if n.value:
            check(self.L.bgpu_read_pairs(self.h, u32ptr(out), n.value, ctypes.byref(n)), "read_pairs")
        return out

    def contacts(self):
        n = ctypes.c_uint64()
        check(self.L.bgpu_read_contacts(self.h, None, 0, ctypes.byref(n)), "read_contacts")
        out = np.zeros((n.value, CONTACT), dtype=np.float32)
        if n.value:
            check(self.L.bgpu_read_contacts(self.h, fptr(out), n.value, ctypes.byref(n)), "read_contacts")
        return out

    def solve_order(self):
        n = ctypes.c_uint64()
        check(self.L.bgpu_read_solve_order(self.h, None, 0, ctypes.byref(n)), "read_solve_order")
        out = np.zeros(n.value, dtype=np.uint64)
        if n.value:
            check(self.L.bgpu_read_solve_order(self.h, u64ptr(out), n.value, ctypes.byref(n)), "read_solve_order")
        return out

    def add_joint(self, kind, body_a, body_b, frame_a, frame_b, flags=JOINT_DISABLE_COLLISIONS, erp=0.0,
                  impulse_clamp=0.0, limit=(1.0, -1.0), softness=0.9, bias_factor=0.3, relaxation=1.0,
                  motor=(0.0, 0.0), gear_ratio=1.0, lin_limits=(1.0, -1.0), ang_limits=(0.0, 0.0),
                  slider_softness=(1.0, 1.0, 1.0, 1.0, 1.0, 1.0), lin_motor=(0.0, 0.0), ang_motor=(0.0, 0.0),
                  cone=None, cone_motor=None):
        """frame_*: 12 numbers (pivot xyz, basis columns x, y, z) in the body's frame."""
        d = JointDesc()
        self.L.bgpu_joint_desc_default(ctypes.byref(d))
        d.kind, d.body_a, d.body_b, d.flags = kind, body_a, body_b, flags
        d.frame_a[:] = [float(x) for x in frame_a]
        d.frame_b[:] = [float(x) for x in frame_b]
        d.erp, d.impulse_clamp = erp, impulse_clamp
        d.limit_low, d.limit_high = limit
        d.limit_softness, d.limit_bias_factor, d.limit_relaxation = softness, bias_factor, relaxation
        d.motor_target_velocity, d.motor_max_impulse = motor
        d.gear_ratio = gear_ratio
        d.lin_limit_low, d.lin_limit_high = lin_limits
        d.ang_limit_low, d.ang_limit_high = ang_limits
        (d.softness_lim_lin, d.softness_lim_ang, d.damping_lim_lin, d.damping_lim_ang, d.softness_ortho_lin,
         d.softness_ortho_ang) = slider_softness
        d.lin_motor_target_velocity, d.lin_motor_max_force = lin_motor
        d.ang_motor_target_velocity, d.ang_motor_max_force = ang_motor
        if cone is not None:  # swing span 1, swing span 2, twist span, softness, bias factor, relaxation
            (d.swing_span1, d.swing_span2, d.twist_span, d.cone_softness, d.cone_bias_factor,
             d.cone_relaxation) = cone
        if cone_motor is not None:  # (target quaternion in constraint space, max impulse)
            d.cone_motor_target[:] = [float(x) for x in cone_motor[0]]
            d.cone_motor_max_impulse = cone_motor[1]
        first = ctypes.c_uint32()
        check(self.L.bgpu_add_joints(self.h, 1, ctypes.byref(d), ctypes.byref(first)), "add_joints")
        return first.value

    def set_ccd(self, first, motion_threshold, swept_sphere_radius):
        """RigidBody::ccd for bodies first, first + 1, ... (arrays or scalars for one body)."""
        thr = np.atleast_1d(f32(motion_threshold))
        rad = np.atleast_1d(f32(swept_sphere_radius))
        check(self.L.bgpu_set_ccd(self.h, first, len(thr), fptr(thr), fptr(rad)), "set_ccd")

    def ccd_clamps(self):
        out = np.ones(self.num_bodies, dtype=np.float32)
        if len(out):
            check(self.L.bgpu_read_ccd_clamps(self.h, fptr(out)), "read_ccd_clamps")
        return out

    def add_spring2(self, joint):
        """Adds a Spring2 joint (Constraint::generic_6dof_spring2) or a Generic6Dof joint
        (Constraint::generic_6dof); returns its joint id."""
        first = ctypes.c_uint32()
        add = self.L.bgpu_add_generic6dof_joints if getattr(joint, "KIND", 5) == JOINT_GENERIC6DOF \
            else self.L.bgpu_add_spring2_joints
        check(add(self.h, 1, ctypes.byref(joint.desc), ctypes.byref(first)), "add_joints")
        return first.value

    @property
    def num_joints(self):
        return self.L.bgpu_num_joints(self.h)

    def set_joint_flags(self, joint, flags):
        """Joint `joint`'s JOINT_DISABLE_COLLISIONS / JOINT_DISABLED bits, from the next step on."""
        check(self.L.bgpu_set_joint_flags(self.h, int(joint), int(flags)), "set_joint_flags")

    def spring2_state(self):
        """Per joint: Euler angles (3), pivot offset in frame A (3), fact_a, has_static_body."""
        out = np.zeros((self.num_joints, 8), dtype=np.float32)
        if len(out):
            check(self.L.bgpu_read_joint_spring2_state(self.h, fptr(out)), "read_joint_spring2_state")
        return out

    def joint_angles(self):
        out = np.zeros(self.num_joints, dtype=np.float32)
        if len(out):
            check(self.L.bgpu_read_joint_angles(self.h, fptr(out)), "read_joint_angles")
        return out

    def joint_positions(self):
        out = np.zeros(self.num_joints, dtype=np.float32)
        if len(out):
            check(self.L.bgpu_read_joint_positions(self.h, fptr(out)), "read_joint_positions")
        return out

    def joint_order(self):
        n = ctypes.c_uint32()
        check(self.L.bgpu_read_joint_order(self.h, None, 0, ctypes.byref(n)), "read_joint_order")
        out = np.zeros(n.value, dtype=np.uint32)
        if n.value:
            check(self.L.bgpu_read_joint_order(self.h, u32ptr(out), n.value, ctypes.byref(n)), "read_joint_order")
        return out

    def joint_rows(self):
        """Rows of the last step in solve order: joint, body_a, body_b, mass, bias, limit kind, impulse, cfm."""
        n = ctypes.c_uint32()
        check(self.L.bgpu_read_joint_rows(self.h, None, 0, ctypes.byref(n)), "read_joint_rows")
        out = np.zeros((n.value, 8), dtype=np.float32)
        if n.value:
            check(self.L.bgpu_read_joint_rows(self.h, fptr(out), n.value, ctypes.byref(n)), "read_joint_rows")
        return out

    def colour_batches(self):
        """Per colour of the last step's PGS: (row groups, row groups with split-impulse rows)."""
        n = ctypes.c_uint32()
        check(self.L.bgpu_read_colour_batches(self.h, None, None, 0, ctypes.byref(n)), "read_colour_batches")
        g = np.zeros(n.value, dtype=np.uint32)
        sg = np.zeros(n.value, dtype=np.uint32)
        if n.value:
            check(self.L.bgpu_read_colour_batches(self.h, u32ptr(g), u32ptr(sg), n.value, ctypes.byref(n)),
                  "read_colour_batches")
        return g, sg

    def stats(self):
        s = StepStats()
        check(self.L.bgpu_get_stats(self.h, ctypes.byref(s)), "get_stats")
        return {f: (list(getattr(s, f)) if f == "stage_ms" else getattr(s, f)) for f, _ in StepStats._fields_}

    def enable_timing(self, on=True):
        check(self.L.bgpu_enable_step_timing(self.h, 1 if on else 0), "timing")

    def collide(self, sa, pa, sb, pb, seeds=None, force_convex=False):
        sa = np.ascontiguousarray(sa, dtype=np.uint32)
        sb = np.ascontiguousarray(sb, dtype=np.uint32)
        n = len(sa)
        pa = f32(np.asarray(pa).reshape(n, 7))
        pb = f32(np.asarray(pb).reshape(n, 7))
        out = np.zeros((n, 4, 7), dtype=np.float32)
        cnt = np.zeros(n, dtype=np.uint32)
        sd = fptr(f32(np.asarray(seeds).reshape(n, 3))) if seeds is not None else None
        check(self.L.bgpu_collide(self.h, n, u32ptr(sa), fptr(pa), u32ptr(sb), fptr(pb), sd, 1 if force_convex else 0,
                                  fptr(out), u32ptr(cnt)), "collide")
        return out, cnt

    def solve_contacts(self, contacts, inv_dt):
        c = f32(np.asarray(contacts).reshape(-1, 10))
        rows = np.zeros((len(c), CONTACT), dtype=np.float32)
        keys = np.zeros(len(c), dtype=np.uint64)
        check(self.L.bgpu_solve_contacts(self.h, len(c), fptr(c), inv_dt, fptr(rows), u64ptr(keys)), "solve_contacts")
        return rows, keys

    def push(self):
        out = np.zeros((self.num_bodies, 6), dtype=np.float32)
        check(self.L.bgpu_read_push(self.h, fptr(out)), "read_push")
        return out


class Tape:
    """Adjoint of a world's steps (bgpu_tape_*): forward with checkpoints, then gradients
    of a loss of the final state w.r.t. initial velocities, friction and restitution."""

    def __init__(self, world, checkpoint_every=20):
        self.L = lib()
        self.world = world  # the world must outlive the tape
        self.h = ctypes.c_void_p()
        check(self.L.bgpu_tape_create(world.h, checkpoint_every, ctypes.byref(self.h)), "bgpu_tape_create")

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.bgpu_tape_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, dt, nsteps):
        check(self.L.bgpu_tape_forward(self.h, dt, nsteps), "bgpu_tape_forward")

    def backward(self, grad_x, grad_v=None, grad_w=None):
        """grad_x, grad_v, grad_w: (n, 3) dL/d(final position, linear, angular velocity).
        Returns dict of gradients: v0 (n,3), w0 (n,3), friction (n,), restitution (n,)."""
        n = self.world.num_bodies
        g = np.zeros((n, 9), dtype=np.float32)
        g[:, 0:3] = grad_x
        if grad_v is not None:
            g[:, 3:6] = grad_v
        if grad_w is not None:
            g[:, 6:9] = grad_w
        out = {"v0": np.zeros((n, 3), np.float32), "w0": np.zeros((n, 3), np.float32),
               "friction": np.zeros(n, np.float32), "restitution": np.zeros(n, np.float32)}
        check(self.L.bgpu_tape_backward(self.h, fptr(g), fptr(out["v0"]), fptr(out["w0"]), fptr(out["friction"]),
                                        fptr(out["restitution"])), "bgpu_tape_backward")
        return out

    def rewind(self):
        check(self.L.bgpu_tape_rewind(self.h), "bgpu_tape_rewind")

    def timing(self):
        f = ctypes.c_float()
        b = ctypes.c_float()
        check(self.L.bgpu_tape_timing(self.h, ctypes.byref(f), ctypes.byref(b)), "bgpu_tape_timing")
        return f.value, b.value


def broadphase_pairs(aabbs):
    a = f32(np.asarray(aabbs).reshape(-1, 6))
    n = ctypes.c_uint64()
    check(lib().bgpu_broadphase_pairs(fptr(a), len(a), None, 0, ctypes.byref(n)), "broadphase_pairs")
    out = np.zeros((n.value, 2), dtype=np.uint32)
    if n.value:
        check(lib().bgpu_broadphase_pairs(fptr(a), len(a), u32ptr(out), n.value, ctypes.byref(n)), "broadphase_pairs")
    return out
