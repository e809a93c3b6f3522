"""CPU checks of the C ABI library: it loads, exports every entry point that
include/bgpu.h declares, and fails loudly (no fallback) without a device."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bgpu.h")
LIB = os.path.join(ROOT, "bullet-physics_b200", "libbgpu.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bgpu_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ["bgpu_world_create", "bgpu_world_destroy", "bgpu_add_shape", "bgpu_add_bodies", "bgpu_step",
                     "bgpu_read_state", "bgpu_read_pairs", "bgpu_read_contacts", "bgpu_broadphase_pairs",
                     "bgpu_collide", "bgpu_solve_contacts", "bgpu_last_error"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "libbgpu.so not built"
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (bgpu_[a-z0-9_]+)$", out, flags=re.M))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, f"not exported: {missing}"


def test_library_loads_and_reports_defaults(bgpu_mod):
    s = bgpu_mod.solver_info()
    # solver/info.rs:88-107 defaults
    assert s.erp2 == pytest.approx(0.2) and s.linear_slop == pytest.approx(0.005)
    assert s.restitution_velocity_threshold == 1.0 and s.split_impulse == 1
    assert s.split_impulse_penetration_threshold == pytest.approx(-0.04)
    assert s.split_impulse_turn_erp == pytest.approx(0.1) and s.warmstarting_factor == pytest.approx(0.85)
    assert s.global_cfm == 0.0 and s.sor == 1.0 and s.num_iterations == 10
    d = bgpu_mod.body_descs(1)[0]
    assert d.friction == pytest.approx(0.5) and d.group == 1 and d.mask == 0xFFFF and d.orientation[3] == 1.0


def test_no_device_fails_loudly(bgpu_mod):
    if bgpu_mod.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(bgpu_mod.BgpuError, match="no CUDA device"):
        bgpu_mod.World()
    with pytest.raises(bgpu_mod.BgpuError):
        bgpu_mod.broadphase_pairs([[0, 0, 0, 1, 1, 1]])
    with pytest.raises(bgpu_mod.BgpuError, match="no CUDA device"):
        bgpu_mod.set_device(0)


def test_struct_layouts_match_the_header(bgpu_mod):
    # bgpu_body_desc: 4 + 12 + 16 + 12 + 12 + 5*4 + 4 + 2 + 2 + 4 + 8 = 96 bytes
    assert ctypes.sizeof(bgpu_mod.BodyDesc) == 96
    assert ctypes.sizeof(bgpu_mod.SolverInfo) == 48
    assert ctypes.sizeof(bgpu_mod.JointDesc) == 4 * 4 + 24 * 4 + 35 * 4
    assert ctypes.sizeof(bgpu_mod.StepStats) == 10 * 4 + 7 * 4 + 2 * 4 + 4


@pytest.mark.gpu
def test_set_device_takes_a_visible_ordinal(gpu):
    """bgpu_set_device selects among the devices the process sees and rejects any other
    ordinal with an error (no CUDA call is made for it); a world created after it steps."""
    n = gpu.device_count()
    assert n >= 1
    gpu.set_device(0)
    for bad in (-1, n):
        with pytest.raises(gpu.BgpuError, match="no device with that ordinal"):
            gpu.set_device(bad)
    w = gpu.World()
    box = w.box([0.5, 0.5, 0.5])
    w.add_body(box, (0, 2, 0))
    w.step(1.0 / 60.0)
    assert w.stats()["device_status"] == 0
    w.close()


def test_rejected_arguments_say_why(bgpu_mod):
    """A NULL world or buffer is rejected before any CUDA call, with a message naming the call
    (no stale message from an earlier failure)."""
    L = bgpu_mod.lib()
    assert L.bgpu_world_set_gravity(None, None) == 1
    assert "bgpu_world_set_gravity" in bgpu_mod.last_error()
    assert L.bgpu_read_state(None, None) == 1
    assert "bgpu_read_state" in bgpu_mod.last_error()
