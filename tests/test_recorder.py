"""Scene loader and trajectory recorder in the reference's parity formats
(docs/parity-harness.md: scenes.json contract, `t px py pz qx qy qz qw` CSV lines)."""
import os

import numpy as np
import pytest

import oracle_api as orc

HERE = os.path.dirname(os.path.abspath(__file__))
SCENES = os.path.join(HERE, "golden", "parity_scenes.json")


def test_scene_fields_are_read():
    import recorder

    sc = recorder.load_scenes(SCENES)
    assert set(sc) >= {"dropped_cube", "capsule_and_ball", "three_stack_substeps"}
    assert recorder.scene_dt(sc["dropped_cube"]) == pytest.approx(1.0 / 60.0)
    kind, params = recorder.shape_params(sc["capsule_and_ball"]["bodies"][1]["shape"])
    assert params == [0.3, 0.6]
    with pytest.raises(ValueError):
        recorder.shape_params(sc["unsupported_cylinder"]["bodies"][0]["shape"])


def oracle_record(scene, out_path_of):
    """The same recording through the oracle's full step (f32)."""
    import recorder

    o = orc.OracleWorld("f32")
    o.set_gravity(scene["gravity"])
    o.set_solver(num_iterations=scene["iterations"])
    index = {}
    for b in scene["bodies"]:
        kind, params = recorder.shape_params(b["shape"])
        s = o.add_shape(kind, params)
        index[b["name"]] = o.add_body(s, b["position"], linvel=b.get("velocity", (0, 0, 0)),
                                      angvel=b.get("angular_velocity", (0, 0, 0)), mass=b["mass"],
                                      friction=b.get("friction", 0.5), restitution=b.get("restitution", 0.0),
                                      lin_damping=b.get("linear_damping", 0.0))
        if "ccd" in b:
            o.set_ccd(index[b["name"]], b["ccd"]["motion_threshold"], b["ccd"]["swept_sphere_radius"])
    dt = recorder.scene_dt(scene)
    out = {n: [] for n in scene["record"]}
    for frame in range(1, scene["frames"] + 1):
        o.step(dt)
        st = o.state()
        for n in scene["record"]:
            out[n].append([np.float32(frame) * np.float32(dt)] + list(st[index[n], 0:7]))
    return {n: np.array(v) for n, v in out.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["dropped_cube", "capsule_and_ball", "ccd_wall"])
def test_recorded_trajectories_match_the_oracle(gpu, tmp_path, name):
    import recorder

    scene = recorder.load_scenes(SCENES)[name]
    paths = recorder.record(name, scene, str(tmp_path), suffix="gpu")
    ref = oracle_record(scene, None)
    for path, body in zip(paths, scene["record"]):
        assert os.path.basename(path) == f"{name}_{body}_gpu.csv"
        lines = open(path).read().splitlines()
        assert len(lines) == scene["frames"] and all(len(l.split()) == 8 for l in lines)
        got = recorder.read_csv(path)
        # %.6f output; the harness tolerance is 1e-2, the GPU holds 1e-4 here
        np.testing.assert_allclose(got[:, 0], ref[body][:, 0], atol=1e-6)
        np.testing.assert_allclose(got[:, 1:], ref[body][:, 1:], atol=1e-4)


@pytest.mark.gpu
def test_substep_scene_records_every_frame(gpu, tmp_path):
    import recorder

    scene = recorder.load_scenes(SCENES)["three_stack_substeps"]
    paths = recorder.record("three_stack_substeps", scene, str(tmp_path))
    top = recorder.read_csv(paths[2])
    assert top.shape == (90, 8)
    assert top[-1, 2] > 2.3  # the stack stands
    with pytest.raises(ValueError):
        recorder.build_world(recorder.load_scenes(SCENES)["unsupported_cylinder"])
