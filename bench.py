#!/usr/bin/env python
"""Benchmark: body-steps/s of the rigid-body step on the 131,072-body pile.

Workload (config 3 of the benchmark set): 65,536 unit boxes (half 0.5) and
65,536 spheres (r 0.5) on a jittered 64x64x32 grid with 1.05 m spacing over a
ground plane; f32; dt 1/60; 20 PGS iterations; 600 steps. The pile first
settles for --preroll untimed steps, then --warmup untimed steps, then --steps
timed steps; by default the preroll is 600 - warmup - steps, so the timed
window is the last steps of the configuration's 600 (the settled pile).

Arms:
  default            the sm_100a library through its C ABI; `value` is device
                     time on the world's stream; `e2e` repeats the steps through
                     the public API with host buffers (force upload + step +
                     pose read-back every step) on the wall clock.
  --impl reference   the CPU implementation of the same step on the host
                     cores (the C++ restatement in oracle/: the Rust reference
                     has no toolchain on this machine), on a bounded sample of
                     the same pile recipe.
Multi-GPU (torchrun): one independent replica per rank (no collective on the
data path); value = all ranks' body-steps / max rank time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "bullet-physics_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "body-steps/s (128k-body pile; 4096 batched worlds) and adjoint steps/s vs plain"
UNIT = "body-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=60)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--preroll", type=int, default=None,
                   help="untimed settle steps (default: 600 - warmup - steps, so the window ends at step 600)")
    p.add_argument("--impl", default="bgpu", choices=["bgpu", "reference"])
    p.add_argument("--grid", default="64,64,32", help="pile grid nx,nz,ny (default: the full 131,072-body pile)")
    p.add_argument("--cpu-sample-grid", default="16,16,32")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--batch-worlds", type=int, default=4096, help="batched-worlds leg: number of worlds (0: skip)")
    p.add_argument("--batch-steps", type=int, default=30)
    p.add_argument("--adjoint-worlds", type=int, default=1024, help="adjoint leg: number of worlds (0: skip)")
    p.add_argument("--ccd-spheres", type=int, default=2048, help="CCD leg: fast CCD spheres (0: skip)")
    p.add_argument("--spring2-counts", default="150,15000",
                   help="joint leg: chain counts of the spring2_chains scene, comma separated (empty: skip)")
    p.add_argument("--stack-steps", type=int, default=300, help="1,000-box stack leg: steps (0: skip)")
    p.add_argument("--mixed-steps", type=int, default=300, help="16,384-body mixed convex leg: steps (0: skip)")
    p.add_argument("--drift-steps", type=int, default=300, help="f64 drift report: steps (0: skip)")
    p.add_argument("--mesh-frames", type=int, default=300, help="terrain-mesh legs: frames (0: skip)")
    a = p.parse_args()
    if a.preroll is None:
        a.preroll = max(0, 600 - a.warmup - a.steps)
    return a


def smi_gpu_id(local_rank):
    """nvidia-smi's id of this rank's GPU. nvidia-smi ignores CUDA_VISIBLE_DEVICES, so the rank's
    entry there (an index or a UUID) is used when nvidia-smi knows it; otherwise (unset, or a
    container that shows nvidia-smi only its own GPUs) the local rank."""
    vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    if local_rank < len(vis):
        try:
            r = subprocess.run(["nvidia-smi", "-i", vis[local_rank], "--query-gpu=index", "--format=csv,noheader"],
                               capture_output=True, text=True, timeout=20)
            if r.returncode == 0 and r.stdout.strip():
                return vis[local_rank]
        except (OSError, subprocess.TimeoutExpired):
            pass
    return str(local_rank)


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region: the sampler is running
    (its first sample seen, then dropped) before the region starts, samples every 20 ms, and
    takes one more sample after the region ends."""

    INTERVAL_MS = 20

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5.0:
                time.sleep(0.005)
            self.samples.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            time.sleep(1.5 * self.INTERVAL_MS / 1000.0)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def grid_of(s):
    nx, nz, ny = (int(x) for x in s.split(","))
    return nx, nz, ny


def cpu_baseline(grid, preroll, steps):
    """The CPU step (oracle restatement, single thread) on a bounded sample of the pile recipe."""
    import oracle_api
    import scenes

    nx, nz, ny = grid
    sc = scenes.large_pile_fast(nx, nz, ny, seed=3)
    w = sc.build_oracle(oracle_api)
    for _ in range(preroll):
        w.step(sc.dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        w.step(sc.dt)
    dt = time.perf_counter() - t0
    n = sc.num_dynamic
    return {"value": n * steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"large-pile recipe {nx}x{nz}x{ny} ({n} bodies), {preroll} untimed steps, then steps "
                      f"{preroll + 1}-{preroll + steps} timed, single thread, {dt:.2f} s",
            "contacts_per_body": len(w.rows()) / n}


def algorithmic_pgs_bytes(st, iters):
    """Per-launch algorithmic bytes of the PGS kernel: per contact and iteration 300 B
    (180 B row + 24 B impulse r/w + 96 B velocity gather/scatter), 120 B per contact of
    warm start, 100 B per split-active contact and iteration."""
    c = st["num_contacts"]
    split_c = st.get("num_split_contacts", 0)
    return c * (300 * iters + 120) + 100 * split_c * iters


def max_over_ranks(dist, x, device=None):
    """The largest of every rank's x (the job's time is its slowest replica's); x itself on one rank."""
    if not dist:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device or ("cuda" if torch.cuda.is_available() else "cpu"))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, steps, world_size, seconds):
    """Whole-job throughput of independent replicas: all ranks' units x steps over the slowest rank's time."""
    return units_per_rank * steps * world_size / seconds


def pinned_array(shape):
    """A float32 host array in page-locked memory (falls back to pageable if torch cannot pin)."""
    try:
        import torch

        return torch.zeros(shape, dtype=torch.float32, pin_memory=True).numpy()
    except Exception:
        return np.zeros(shape, dtype=np.float32)


def count_launches(w, dt, nsteps=2):
    """Kernels the library launches per step, counted by CUPTI (torch.profiler) over
    `nsteps` untimed steps run after the timed region; memcpy/memset are not counted."""
    try:
        import torch
        from torch.autograd import DeviceType
        from torch.profiler import ProfilerActivity, profile

        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            w.step(dt, nsteps)
            torch.cuda.synchronize()
        names = {}
        for e in prof.events():
            if e.device_type != DeviceType.CUDA or e.name.startswith(("Memcpy", "Memset")):
                continue
            names[e.name] = names.get(e.name, 0) + 1
        total = sum(names.values())
        return (total / nsteps if total else None), len(names)
    except Exception:  # profiler unavailable: report no count rather than a guess
        return None, 0


def solve_traffic(contacts):
    """DRAM bytes of the PGS launches of one step, from the committed ncu capture of the same
    kernels (profiles/k_solve_chunks_large_pile_131072.md, a shorter-settled pile), scaled to
    this step by its contact count (the kernels' traffic grows with the rows they sweep)."""
    import re

    path = os.path.join(ROOT, "profiles", "k_solve_chunks_large_pile_131072.md")
    try:
        text = open(path).read()
        dram = float(re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", text).group(1))
        cap_contacts = float(re.search(r"capture_contacts:\s*([0-9]+)", text).group(1))
    except (OSError, AttributeError, ValueError):
        return None, None
    return dram * contacts / cap_contacts, {"captured_bytes": dram, "captured_contacts": int(cap_contacts)}


def bench_batched(bgpu, scenes, n_worlds, steps, warmup, sample_worlds=128, sample_steps=20):
    """Batched-worlds leg: body-steps/s of n_worlds independent worlds stepped as one batch,
    against the same worlds stepped one world at a time as plain worlds (a sample of the
    worlds, scaled to the whole batch by its body count)."""
    sc = scenes.batched_worlds(n_worlds=n_worlds, seed=4)
    w = sc.build_gpu(bgpu)
    n_dyn = sc.num_dynamic
    w.step_timed(sc.dt, 60)  # settle
    tuning = w.autotune(sc.dt, 3)  # the solver's launch shape, timed from this state
    w.step_timed(sc.dt, warmup)
    w.enable_timing(True)
    ms = w.step_timed(sc.dt, steps)
    st = w.stats()
    w.enable_timing(False)
    w.close()
    batched = n_dyn * steps / (ms / 1000.0)
    # one plain world per world, stepped one after another (a sample of the worlds)
    idx = np.linspace(0, n_worlds - 1, min(sample_worlds, n_worlds)).astype(int)
    total_ms, sample_dyn = 0.0, 0
    for k in idx:
        ws = sc.world_scene(int(k))
        pw = ws.build_gpu(bgpu)
        pw.step_timed(ws.dt, 60)
        total_ms += pw.step_timed(ws.dt, sample_steps)
        sample_dyn += ws.num_dynamic
        pw.close()
    per_world = sample_dyn * sample_steps / (total_ms / 1000.0)
    return {"workload": f"batched_worlds_{n_worlds} (config 4): {n_dyn} dynamic bodies, "
                        f"{sc.num_bodies} bodies, 8-255 per world, 10 iterations",
            "value": batched, "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "pairs": st["num_pairs"], "contacts": st["num_contacts"], "colours": st["num_colours"],
            "stage_ms_per_step": [x / max(st["timed_steps"], 1) for x in st["stage_ms"]],
            "one_world_per_launch": {"value": per_world, "unit": UNIT,
                                     "sample": f"{len(idx)} of the worlds as plain worlds, {sample_steps} steps each, "
                                               f"device time summed"},
            "speedup_vs_one_world_per_launch": batched / per_world if per_world else None,
            "autotune": {"threads_per_cta": tuning["threads_per_cta"],
                         "warp_world_max_bodies": tuning["warp_world_max_bodies"], "ctas": tuning["ctas"],
                         "candidates": tuning["candidates"], "ms_per_step": tuning["ms_per_step"],
                         "global_solver_ms_per_step": tuning["global_ms_per_step"],
                         "note": "threads_per_cta 0 = the global solver; worlds of at most warp_world_max_bodies "
                                 "bodies are solved one per warp, larger ones one per CTA"},
            "device_status": st["device_status"]}


def bench_adjoint(bgpu, scenes, n_worlds, steps=120, every=20):
    """Adjoint leg: 1,024 worlds x 64 thrown boxes, 120 steps at dt 1/120. Times the plain
    forward (bgpu_step), the taped forward (with checkpoints) and the backward pass (replay of
    every segment with recording, then the reverse sweeps), all device time."""
    sc = scenes.adjoint_worlds(n_worlds=n_worlds, seed=5, steps=steps)
    w = sc.build_gpu(bgpu)
    tuning = w.autotune(sc.dt, 3)  # from the initial state, which it restores
    tape = bgpu.Tape(w, every)
    tape.forward(sc.dt, steps)  # first pass: grows the world's buffers
    tape.rewind()
    plain_ms = w.step_timed(sc.dt, steps)  # the same rollout, plain steps
    tape.rewind()
    tape.forward(sc.dt, steps)
    st = w.state()
    loss, gx = scenes.com_loss(st[:, 0:3], sc.arrays()["mass"], w.world_offsets(), sc.targets)
    g = tape.backward(gx.astype(np.float32))  # first call: allocates the segment records
    fwd_ms, cold_bwd_ms = tape.timing()
    g = tape.backward(gx.astype(np.float32))
    _, bwd_ms = tape.timing()
    tape.close()
    w.close()
    n_dyn = sc.num_dynamic
    grad_ms = fwd_ms + bwd_ms
    return {"workload": f"adjoint_worlds_{n_worlds} (config 5): {n_dyn} boxes, {steps} steps, dt 1/120, "
                        f"10 iterations, checkpoint every {every} steps",
            "value": steps / (grad_ms / 1000.0), "unit": "adjoint steps/s",
            "value_basis": "rollout steps / (taped forward + backward) device time",
            "adjoint_over_forward": grad_ms / plain_ms if plain_ms > 0 else None,
            "adjoint_over_forward_target": 3.0,
            "plain_forward_ms": plain_ms, "taped_forward_ms": fwd_ms, "backward_ms": bwd_ms,
            "backward_first_call_ms": cold_bwd_ms,
            "backward_over_plain_forward": bwd_ms / plain_ms if plain_ms > 0 else None,
            "plain_steps_per_s": steps / (plain_ms / 1000.0), "loss": loss,
            "solver_launch_shape": {k: tuning[k] for k in ("threads_per_cta", "warp_world_max_bodies", "ctas")},
            "grad_norms": {k: float(np.linalg.norm(v)) for k, v in g.items()}}


def bench_spring2(bgpu, scenes, count, frames=300, warmup=5):
    """Joint leg: the spring2_chains perf scene (spring-2 joint rows in the PGS) at `count`
    chains of 3 boxes (150 is the reference's scene: 600 bodies, 450 joints), `frames` steps at
    dt 1/60 after `warmup`, device time. The reference publishes its own CPU times for the
    150-chain scene (docs/perf/speed.md, spring2_chains); they are quoted beside ours."""
    w = scenes.spring2_chains_world(bgpu, count=count)
    dt = 1.0 / 60.0
    w.step_timed(dt, warmup)
    ms = w.step_timed(dt, frames)
    rows = int(w.joint_rows().shape[0])
    n = int(w.num_bodies)
    status = int(w.stats()["device_status"])
    w.close()
    out = {"workload": f"spring2_chains_{count}: {n} bodies, {3 * count} spring-2 joints, {rows} joint rows per "
                       f"step, 10 iterations, dt 1/60, {frames} steps",
           "value": n * frames / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / frames,
           "joint_rows_per_step": rows, "device_status": status}
    if count == 150:
        out["reference_published_ms_per_frame"] = {"rust": 0.709, "bullet": 1.318,
                                                   "source": "docs/perf/speed.md spring2_chains, f32, their CPU"}
    return out


def bench_ccd(bgpu, scenes, n_ccd, steps=60, warmup=5):
    """CCD leg: `n_ccd` fast CCD spheres and half as many boxes raining onto thin plates
    (scenes.ccd_rain_world); device time of `steps` steps after `warmup`, and the clamps of the
    last step."""
    w, ids = scenes.ccd_rain_world(bgpu, n_ccd=n_ccd, n_boxes=n_ccd // 2)
    dt = 1.0 / 60.0
    w.step_timed(dt, warmup)
    ms = w.step_timed(dt, steps)
    clamped = int(np.count_nonzero(w.ccd_clamps()[ids] < 1.0))
    n = int(w.num_bodies)
    status = int(w.stats()["device_status"])
    w.close()
    return {"workload": f"ccd_rain_{n_ccd}: {n} bodies, {n_ccd} CCD spheres (60-400 m/s) and {n_ccd // 2} boxes "
                        f"over 256 thin plates, 10 iterations, dt 1/60, {steps} steps",
            "value": n * steps / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / steps,
            "ccd_bodies_clamped_last_step": clamped, "device_status": status}


def bench_scene(bgpu, sc, name, steps, warmup=5):
    """Device time of `steps` steps of a plain-world scene from its initial state (the
    configuration's own step window), with the per-stage split of the step."""
    w = sc.build_gpu(bgpu)
    w.step_timed(sc.dt, 1)  # sizes the world's buffers; the window below starts at step 2
    w.enable_timing(True)
    ms = w.step_timed(sc.dt, steps)
    st = w.stats()
    w.enable_timing(False)
    w.close()
    n = sc.num_dynamic
    return {"workload": name, "value": n * steps / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "last_step": {"pairs": st["num_pairs"], "contacts": st["num_contacts"],
                                          "narrow_phase_detections": st["num_detect"], "colours": st["num_colours"]},
            "stage_ms_per_step": [x / max(st["timed_steps"], 1) for x in st["stage_ms"]],
            "device_status": st["device_status"]}


def bench_stack(bgpu, scenes, steps):
    """Config 1: the 1,000-box stack, steps 2..steps+1 of the recipe. The reference publishes
    its own single-thread CPU frame time for its closest scene (stack_1000: 1,000 boxes on a box
    ground, 10 iterations, 600 frames)."""
    sc = scenes.falling_box_stack(10, 10, 10, seed=1, steps=steps)
    out = bench_scene(bgpu, sc, f"falling_box_stack_1000 (config 1): 10x10x10 boxes, 10 iterations, dt 1/60, "
                                f"{steps} steps", steps)
    out["reference_published_ms_per_frame"] = {"rust": 1.211, "bullet": 1.208, "scene": "stack_1000",
                                               "source": "docs/perf/speed.md stack_1000 per-frame median, f32, "
                                                         "their CPU, 1 thread"}
    return out


def bench_mixed(bgpu, scenes, steps):
    """Config 2: 16,384 mixed convex bodies (boxes, spheres, capsules, 24-point hulls; the
    GJK/EPA path) dropped in a 40 m cube, steps 2..steps+1 of the recipe."""
    sc = scenes.mixed_convex_pile(n=16384, seed=2, steps=steps)
    return bench_scene(bgpu, sc, f"mixed_convex_pile_16384 (config 2): 40% boxes, 30% spheres, 15% capsules, "
                                 f"15% hulls, 10 iterations, dt 1/60, {steps} steps", steps)


def bench_mesh_rain(bgpu, scenes, frames=300):
    """Triangle-mesh legs: the reference's rain_500 and dbvt_rain_2000 perf scenes (mixed convex
    raining onto a wavy terrain mesh, tools/perf_scenes.json), all `frames` frames from the
    start, device time; the reference's own published CPU frame times quoted beside."""
    out = []
    for nx, grid, name, rust, bullet in ((10, 20, "rain_500", 1.253, 3.470), (20, 40, "dbvt_rain_2000", 5.988, 17.893)):
        sc = scenes.mesh_rain(nx=nx, nz=nx, layers=5, grid=grid, steps=frames)
        r = bench_scene(bgpu, sc, f"{name}: {sc.num_dynamic} boxes / spheres / capsules onto a {grid}x{grid} terrain "
                                  f"mesh, 10 iterations, dt 1/60, {frames} frames", frames)
        r["reference_published_ms_per_frame"] = {"rust": rust, "bullet": bullet,
                                                 "source": f"docs/perf/speed.md {name} per-frame median, f32, their "
                                                           f"CPU, 1 thread"}
        out.append(r)
    return out


def drift_report(bgpu, scenes, steps):
    """Drift of the f32 device trajectory against the oracle's f64 build (the reference's
    `--features f64` restated), on the 1,000-box stack and a 1,024-body slice of the mixed
    convex recipe; the oracle runs as the checker, the device step is what is measured."""
    import drift_f64
    import oracle_api

    out = {"tolerance": {"pos_m": drift_f64.LEDGER_TOL_POS, "ang_rad": drift_f64.LEDGER_TOL_ANG,
                         "source": "docs/parity-harness.md Tolerance; tools/compare.py quat_angle"},
           "solve_order": "the f64 oracle is fed the device's colour order every step"}
    for key, sc in (("stack_1000", scenes.falling_box_stack(10, 10, 10, seed=1, steps=steps)),
                    ("mixed_convex_1024", scenes.mixed_convex_pile(n=1024, seed=2, steps=steps, extent=13.0))):
        d = drift_f64.drift_run(bgpu, oracle_api, sc, steps)
        out[key] = drift_f64.summary(sc.name, sc, d)
    return out


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world_size > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta

        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist
    if args.impl == "reference":
        if rank == 0:
            base = cpu_baseline(grid_of(args.cpu_sample_grid), args.preroll + args.warmup, args.steps)
            line = {"metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                    "config": {"workload": "large_pile_131072 (config 3): CPU sample of the same recipe",
                               "sample_grid": args.cpu_sample_grid, "sample_bodies": int(np.prod(grid_of(args.cpu_sample_grid))),
                               "timed_window": f"steps {args.preroll + args.warmup + 1}-"
                                               f"{args.preroll + args.warmup + args.steps} of 600",
                               "iterations": 20, "dt": 1 / 60},
                    "cpu_baseline": base,
                    "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import bgpu
    import scenes

    if world_size > 1:
        # The library has its own CUDA runtime: make this rank's GPU its current device too.
        bgpu.set_device(local_rank)

    nx, nz, ny = grid_of(args.grid)
    sc = scenes.large_pile_fast(nx, nz, ny, seed=3 + rank)
    w = sc.build_gpu(bgpu)
    n_dyn = sc.num_dynamic
    w.step_timed(sc.dt, args.preroll)
    w.step_timed(sc.dt, args.warmup)
    w.enable_timing(True)
    if dist:
        import torch

        dist.barrier()
        torch.cuda.synchronize()
    with ClockSampler(smi_gpu_id(local_rank)) as clocks:
        ms = w.step_timed(sc.dt, args.steps)
    st = w.stats()
    w.enable_timing(False)
    act = w.state()[:, 13]
    dyn = np.asarray(sc.mass) > 0
    awake_fraction = float(np.count_nonzero(act[dyn] != 2)) / max(n_dyn, 1)  # 2 = island sleeping
    region_ms = max_over_ranks(dist, ms)
    if dist:
        dist.barrier()
    value = replica_throughput(n_dyn, args.steps, world_size, region_ms / 1000.0)

    # End to end through the public API with pinned host buffers (force upload, step, pose read-back).
    forces = pinned_array((w.num_bodies, 3))
    poses = pinned_array((w.num_bodies, 7))
    e2e_steps = max(1, min(args.steps, 30))

    def e2e_round(nsteps):
        t0 = time.perf_counter()
        for _ in range(nsteps):
            w.apply_forces(forces)
            w.step(sc.dt)
            w.poses(poses)
        return time.perf_counter() - t0

    e2e_round(max(1, min(args.warmup, 3)))  # the first calls size the staging buffers
    # Wall-clock time of three rounds, the median kept (a host-side stall in one round,
    # e.g. another process on the host, would otherwise decide the figure).
    e2e_s = max_over_ranks(dist, sorted(e2e_round(e2e_steps) for _ in range(3))[1])
    e2e_value = replica_throughput(n_dyn, e2e_steps, world_size, e2e_s)

    launches_per_step, kernel_kinds = count_launches(w, sc.dt) if rank == 0 else (None, 0)

    if rank == 0:
        hbm, peak_kind = peaks()
        launches = max(st["timed_steps"], 1)
        solve_ms = st["solve_kernel_ms"] / launches
        alg = algorithmic_pgs_bytes(st, sc.iterations)
        achieved = alg / (solve_ms / 1000.0) / 1e9 if solve_ms > 0 else None
        traffic, traffic_src = solve_traffic(st["num_contacts"])
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": region_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"large_pile_{n_dyn} (config 3): {nx}x{nz}x{ny} grid, 50% unit boxes / 50% r0.5 "
                                   f"spheres, 1.05 m spacing, ground plane",
                       "iterations": sc.iterations, "dt": sc.dt, "preroll_steps": args.preroll,
                       "timed_window": f"steps {args.preroll + args.warmup + 1}-{args.preroll + args.warmup + args.steps}"
                                       f" of the recipe's 600",
                       "awake_fraction": awake_fraction, "contacts_per_body": st["num_contacts"] / max(n_dyn, 1),
                       "parallelism": f"replicas x{world_size}",
                       "l2": "inputs larger than L2 (rows + manifolds + bodies > 126 MB)",
                       "pairs": st["num_pairs"], "contacts": st["num_contacts"],
                       "contact_pairs": st["num_contact_pairs"], "colours": st["num_colours"],
                       "stage_ms_per_step": [x / launches for x in st["stage_ms"]]},
            "roofline": {"kernel": "k_solve_chunks (chunked colour-batched PGS)", "bound": "hbm",
                         "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                         "traffic_source": traffic_src, "peak_kind": peak_kind,
                         "kernel_ms_per_launch": solve_ms, "algorithmic_bytes_per_launch": alg,
                         "split_contacts": st["num_split_contacts"]},
            "contacts_per_s": st["num_contacts"] * args.steps / (region_ms / 1000.0) * world_size,
            "contacts_per_s_note": "contacts of the last timed step x timed steps / device time",
            "clocks": clocks.summary(),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(forces.nbytes),
                    "d2h_bytes_per_step": int(poses.nbytes)},
            "gpu_launches": int(round(launches_per_step * args.steps)) if launches_per_step else None,
            "gpu_launches_note": f"CUPTI count of one step x steps ({kernel_kinds} kernel kinds)",
            "device_status": st["device_status"],
        }
        # The other configurations are single-GPU legs: they run at n_gpus 1 only, so that the
        # other ranks of a multi-GPU run do not sit in the closing barrier for minutes.
        if world_size > 1:
            line["other_legs"] = "measured at n_gpus 1 only; each rank of this run steps a pile replica"
        if world_size == 1 and args.batch_worlds > 0:
            line["batched_worlds"] = bench_batched(bgpu, scenes, args.batch_worlds, args.batch_steps, args.warmup)
        if world_size == 1 and args.adjoint_worlds > 0:
            line["adjoint"] = bench_adjoint(bgpu, scenes, args.adjoint_worlds)
        if world_size == 1 and args.ccd_spheres > 0:
            line["ccd_rain"] = bench_ccd(bgpu, scenes, args.ccd_spheres)
        if world_size == 1 and args.spring2_counts:
            line["spring2_chains"] = [bench_spring2(bgpu, scenes, int(c)) for c in args.spring2_counts.split(",")]
        if world_size == 1 and args.stack_steps > 0:
            line["stack_1000"] = bench_stack(bgpu, scenes, args.stack_steps)
        if world_size == 1 and args.mixed_steps > 0:
            line["mixed_convex_16384"] = bench_mixed(bgpu, scenes, args.mixed_steps)
        if world_size == 1 and args.mesh_frames > 0:
            line["mesh_rain"] = bench_mesh_rain(bgpu, scenes, args.mesh_frames)
        if world_size == 1 and not args.no_cpu_baseline:
            # CPU leg: the oracle timed on the host (the baseline) and run as the f64 checker.
            line["cpu_baseline"] = cpu_baseline(grid_of(args.cpu_sample_grid), args.preroll + args.warmup, args.steps)
            if args.drift_steps > 0:
                line["drift_f64"] = drift_report(bgpu, scenes, args.drift_steps)
        print(json.dumps(line), flush=True)
    w.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
