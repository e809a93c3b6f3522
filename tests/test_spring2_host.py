"""Host side of the spring-2 joint: the C ABI defaults, the Hinge-2 constructor and the
reference setters mirrored by bgpu.Spring2. No device work: these run on the CPU.

Each case restates a test of crates/bullet-dynamics/src/constraint/generic6dof_spring2.rs
(line cited)."""
import math

import numpy as np

import bgpu

PI = float(np.float32(math.pi))


def test_defaults_match_bullet():  # :1437-1455
    j = bgpu.Spring2(0, 1)
    for i in range(3):
        lin, ang = j.axis(i), j.axis(3 + i)
        assert (ang.lower_limit, ang.upper_limit) == (1.0, -1.0)
        assert ang.stop_erp == np.float32(0.2) and ang.motor_erp == np.float32(0.9)
        assert ang.max_motor_force == 6.0
        assert ang.flags == 0
        assert (lin.lower_limit, lin.upper_limit, lin.max_motor_force) == (0.0, 0.0, 0.0)
        assert lin.stop_erp == np.float32(0.2) and lin.motor_erp == np.float32(0.9)
    assert j.desc.rotate_order == bgpu.ROTATE_XYZ
    assert j.desc.flags == bgpu.JOINT_DISABLE_COLLISIONS


def test_servo_target_wraps_into_pi_range():  # :1554-1564
    j = bgpu.Spring2(0, 1)
    j.set_servo_target(3, 7.0)
    assert abs(j.axis(3).servo_target - (7.0 - 2.0 * PI)) < 1e-5
    j.set_servo_target(3, -7.0)
    assert abs(j.axis(3).servo_target + (7.0 - 2.0 * PI)) < 1e-5
    j.set_servo_target(3, 0.3)
    assert abs(j.axis(3).servo_target - 0.3) < 1e-6
    j.set_servo_target(0, 12.0)
    assert j.axis(0).servo_target == 12.0


def test_reversed_limit_setters_mirror_the_convention():  # :1567-1587
    j = bgpu.Spring2(0, 1)
    j.set_limit_reversed(4, 0.3, 0.7)
    assert j.axis(4).upper_limit == np.float32(-0.3)
    assert j.axis(4).lower_limit == np.float32(-0.7)
    j.set_limit_reversed(3, PI + 0.1, PI + 0.2)
    assert abs(j.axis(3).upper_limit - (PI - 0.1)) < 1e-5


def test_override_setters_raise_their_flags():  # :579-625 (setParam flags)
    j = bgpu.Spring2(0, 1)
    j.set_stop_erp(3, 0.3)
    j.set_stop_cfm(0, 0.01)
    j.set_motor_erp(5, 0.7)
    j.set_motor_cfm(2, 0.02)
    assert j.axis(3).flags == bgpu.S2_STOP_ERP and j.axis(3).stop_erp == np.float32(0.3)
    assert j.axis(0).flags == bgpu.S2_STOP_CFM
    assert j.axis(5).flags == bgpu.S2_MOTOR_ERP
    assert j.axis(2).flags == bgpu.S2_MOTOR_CFM
    j.enable_spring(4)
    j.set_stiffness(4, 5.0, True)
    j.set_damping(4, 0.3, False)
    assert j.axis(4).flags == bgpu.S2_SPRING | bgpu.S2_STIFFNESS_LIMITED


def test_hinge2_config_hand_computed():  # :1949-1999
    j = bgpu.Spring2.hinge2(0, 1, (0, 0, 0), (0, 0, 0, 1), (0, 0, 0), (0, 0, 0, 1), (1.0, 2.0, 3.0), (0, 0, 1),
                            (1, 0, 0))
    fa, fb = np.array(j.desc.frame_a), np.array(j.desc.frame_b)
    assert np.allclose(fa[:3], (1.0, 2.0, 3.0), atol=1e-6)
    assert np.array_equal(fa, fb)
    assert np.array_equal(fa[3:], np.eye(3).reshape(9))
    for i in range(2):
        assert (j.axis(i).lower_limit, j.axis(i).upper_limit) == (0.0, 0.0)
    assert (j.axis(2).lower_limit, j.axis(2).upper_limit) == (-1.0, 1.0)
    steer = math.pi / 4
    assert (j.axis(3).lower_limit, j.axis(3).upper_limit) == (1.0, -1.0)
    assert (j.axis(4).lower_limit, j.axis(4).upper_limit) == (0.0, 0.0)
    assert abs(j.axis(5).lower_limit + steer) < 1e-6 and abs(j.axis(5).upper_limit - steer) < 1e-6
    assert j.axis(2).flags & bgpu.S2_SPRING
    assert abs(j.axis(2).stiffness - PI * PI * 4.0) < 1e-5
    assert abs(j.axis(2).damping - 0.01) < 1e-9


def test_hinge2_equilibrium_is_the_construction_pose():  # :2002-2024
    qa = (0.0, 0.0, math.sin(math.pi / 4), math.cos(math.pi / 4))
    qb = (0.0, 0.0, math.sin(0.25), math.cos(0.25))
    j = bgpu.Spring2.hinge2(0, 1, (0, 0, 0), qa, (1.0, 0.0, 0.5), qb, (1.0, 0.0, 0.0), (0, 0, 1), (1, 0, 0))
    for i in range(6):
        assert abs(j.axis(i).equilibrium_point) < 1e-5
