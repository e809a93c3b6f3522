"""Trajectory drift of the f32 device step against the oracle's f64 build.

Test infrastructure (it runs the CPU oracle): used by tests/test_drift_f64.py
and by bench.py's CPU-baseline leg, never by the library.

Both sides start from the same scene inputs. The f64 oracle is fed the
device's colour order every step (the rows of a pair missing from that order,
once the two trajectories hold different pairs, go last in pair order), so
the figure is the precision drift of the same algorithm, not an order effect.
Per step and over the dynamic bodies: the position distance and the
orientation angle 2 acos(|q1 . q2|) (double-cover aware, in a stable form), the two measures of
the reference's parity harness (tools/compare.py:43-47, tolerances 1e-2 m and
1e-2 rad from docs/parity-harness.md "Tolerance").
"""
import numpy as np

LEDGER_TOL_POS = 1e-2
LEDGER_TOL_ANG = 1e-2


def quat_angle(qa, qb):
    """Row-wise angle between two quaternion arrays (x y z w): tools/compare.py:43-47's
    2 acos(|qa . qb|) for unit quaternions, computed as 2 atan2(|v|, |w|) of the relative
    rotation conj(qa) qb after normalising both in f64. (acos near 1 turns the ~1e-7 norm
    error of an f32 quaternion into a ~5e-4 rad floor; the atan2 form has none.)"""
    a = np.asarray(qa, np.float64)
    b = np.asarray(qb, np.float64)
    a = a / np.linalg.norm(a, axis=1, keepdims=True)
    b = b / np.linalg.norm(b, axis=1, keepdims=True)
    w = np.sum(a * b, axis=1)
    v = a[:, 3:4] * b[:, 0:3] - b[:, 3:4] * a[:, 0:3] - np.cross(a[:, 0:3], b[:, 0:3])
    return 2.0 * np.arctan2(np.linalg.norm(v, axis=1), np.abs(w))


def drift_run(bgpu, orc, scene, steps=None):
    """Step `scene` on the device (f32) and in the f64 oracle side by side; per-step
    max / median drift of position (m) and orientation (rad) over the dynamic bodies."""
    steps = scene.steps if steps is None else steps
    w = scene.build_gpu(bgpu)
    o = scene.build_oracle(orc, precision="f64")
    dyn = np.asarray(scene.mass) > 0
    out = {k: np.zeros(steps) for k in ("max_pos", "median_pos", "max_ang", "median_ang")}
    try:
        for s in range(steps):
            w.step(scene.dt)
            o.set_solve_order(w.solve_order())
            o.step(scene.dt)
            g = w.state().astype(np.float64)[dyn]
            r = o.state()[dyn]
            dp = np.linalg.norm(g[:, 0:3] - r[:, 0:3], axis=1)
            da = quat_angle(g[:, 3:7], r[:, 3:7])
            out["max_pos"][s], out["median_pos"][s] = dp.max(), np.median(dp)
            out["max_ang"][s], out["median_ang"][s] = da.max(), np.median(da)
        out["final_pos"] = dp
        status = int(w.stats()["device_status"])
    finally:
        w.close()
    out["device_status"] = status
    return out


def first_over(series, tol):
    """1-based step at which `series` first exceeds `tol` (None if never)."""
    idx = np.flatnonzero(np.asarray(series) > tol)
    return int(idx[0]) + 1 if len(idx) else None


def summary(name, scene, d, marks=(30, 60, 150, 300)):
    """Compact report of one drift run (the bench's drift_f64 entries)."""
    n = len(d["max_pos"])
    at = {str(m): {"max_pos": float(d["max_pos"][m - 1]), "median_pos": float(d["median_pos"][m - 1]),
                   "max_ang": float(d["max_ang"][m - 1]), "median_ang": float(d["median_ang"][m - 1])}
          for m in marks if m <= n}
    return {"workload": name, "bodies": int(scene.num_dynamic), "steps": n,
            "at_step": at,
            "max_pos_over_run": float(d["max_pos"].max()), "max_ang_over_run": float(d["max_ang"].max()),
            "first_step_pos_over_1e-2": first_over(d["max_pos"], LEDGER_TOL_POS),
            "first_step_ang_over_1e-2": first_over(d["max_ang"], LEDGER_TOL_ANG),
            "bodies_over_1e-2_at_end_fraction": float(np.mean(d["final_pos"] > LEDGER_TOL_POS)),
            "device_status": d["device_status"]}
