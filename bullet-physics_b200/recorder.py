"""Parity-scene loader and trajectory recorder in the reference's formats.

Scene format: the reference's parity-scene contract (docs/parity-harness.md, "Scene
protocol"; tools/scenes.json): a JSON object {"scenes": {name: scene}} where a scene has
"dt" as a fraction [num, den], "frames", "iterations", "gravity", "bodies" (each with
"name", "shape" {"type": box | sphere | capsule | plane, ...}, "position", "mass" (0 =
static), optional "friction", "restitution", "velocity", "angular_velocity",
"linear_damping", "angular_damping", "additional_damping", "no_contact_response",
"group", "mask" (-1 = all), "ccd" {"motion_threshold", "swept_sphere_radius"}), "record" (body
names) and optional "substeps"
{"max_sub_steps", "fixed_dt"}.

Output format (docs/parity-harness.md, "Output format"; tools/bullet_record.cpp:352-383):
one file <scene>_<body>_<suffix>.csv per recorded body, one line per frame
"t px py pz qx qy qz qw" with %.6f, t = frame * dt in f32.

Shape types the GPU step has no narrow phase for (cylinder, cone, mesh, mesh_parts),
per-body gravity vectors and ray probes are rejected with ValueError.
"""
import json
import os

import numpy as np

import bgpu

_SHAPES = {"box": bgpu.BOX, "sphere": bgpu.SPHERE, "capsule": bgpu.CAPSULE, "plane": bgpu.PLANE}


def load_scenes(path_or_dict):
    """All scenes of a scenes.json file (or an already parsed dict), by name."""
    if isinstance(path_or_dict, dict):
        data = path_or_dict
    else:
        with open(path_or_dict) as f:
            data = json.load(f)
    return data["scenes"]


def shape_params(shape):
    kind = shape["type"]
    if kind not in _SHAPES:
        raise ValueError(f"shape type '{kind}' has no narrow phase in the GPU step")
    if kind == "box":
        return _SHAPES[kind], list(shape["half_extents"])
    if kind == "sphere":
        return _SHAPES[kind], [shape["radius"]]
    if kind == "capsule":
        return _SHAPES[kind], [shape["radius"], shape["half_height"]]
    return _SHAPES[kind], list(shape["normal"]) + [shape.get("constant", 0.0)]


def scene_dt(scene):
    num, den = scene["dt"]
    return float(np.float32(num) / np.float32(den))


def build_world(scene, lib=bgpu):
    """A GPU world holding the scene's bodies (in file order); returns (world, {name: index})."""
    for key in ("rays", "pair_filter"):
        if key in scene:
            raise ValueError(f"scene field '{key}' is not supported by the GPU step")
    w = lib.World(gravity=tuple(scene.get("gravity", (0.0, -9.81, 0.0))), num_iterations=int(scene["iterations"]))
    shape_ids = {}
    index = {}
    for body in scene["bodies"]:
        if "gravity" in body:
            raise ValueError(f"body '{body['name']}': per-body gravity is not supported by the GPU step")
        kind, params = shape_params(body["shape"])
        key = (kind, tuple(params))
        if key not in shape_ids:
            shape_ids[key] = w.add_shape(kind, params)
        flags = 0
        if body.get("no_contact_response"):
            flags |= bgpu.NO_CONTACT_RESPONSE
        if body.get("additional_damping"):
            flags |= bgpu.ADDITIONAL_DAMPING
        group = body.get("group", 1)
        mask = body.get("mask", -1)
        index[body["name"]] = w.add_body(
            shape_ids[key], body["position"], quat=tuple(body.get("orientation", (0.0, 0.0, 0.0, 1.0))),
            linvel=tuple(body.get("velocity", (0.0, 0.0, 0.0))),
            angvel=tuple(body.get("angular_velocity", (0.0, 0.0, 0.0))), mass=float(body["mass"]),
            friction=float(body.get("friction", 0.5)), restitution=float(body.get("restitution", 0.0)), flags=flags,
            group=0xFFFF if group == -1 else group, mask=0xFFFF if mask == -1 else mask,
            lin_damping=float(body.get("linear_damping", 0.0)), ang_damping=float(body.get("angular_damping", 0.0)))
        if "ccd" in body:
            w.set_ccd(index[body["name"]], float(body["ccd"]["motion_threshold"]),
                      float(body["ccd"]["swept_sphere_radius"]))
    return w, index


def record(scene_name, scene, out_dir, suffix="gpu", lib=bgpu):
    """Steps the scene for its frames and writes one CSV per recorded body; returns the paths."""
    w, index = build_world(scene, lib)
    dt = scene_dt(scene)
    sub = scene.get("substeps")
    names = list(scene["record"])
    rows = {n: [] for n in names}
    for frame in range(1, int(scene["frames"]) + 1):
        if sub:
            w.step_fixed(dt, int(sub["max_sub_steps"]), float(sub["fixed_dt"]))
        else:
            w.step(dt)
        st = w.state()
        t = np.float32(frame) * np.float32(dt)
        for n in names:
            rows[n].append((float(t),) + tuple(float(x) for x in st[index[n], 0:7]))
    w.close()
    paths = []
    os.makedirs(out_dir, exist_ok=True)
    for n in names:
        path = os.path.join(out_dir, f"{scene_name}_{n}_{suffix}.csv")
        with open(path, "w") as f:
            for r in rows[n]:
                f.write(" ".join("%.6f" % v for v in r) + "\n")
        paths.append(path)
    return paths


def read_csv(path):
    """A recorded trajectory as an (frames, 8) array: t, position, quaternion."""
    return np.loadtxt(path, ndmin=2)
