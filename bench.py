#!/usr/bin/env python
"""Throughput benchmark of the B200 particle pipeline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload: the large single-scene double dam break, DFSPH, 1,000,000
fluid + 409,599 Akinci boundary particles (r = 0.005 m, 4 x 2 x 2 m tank,
sphere obstacle R = 0.2 m), seeded synthetic lattice. One "step" is one
DFSPH time step of the whole scene. `value` is fluid particle-steps/s with
the state resident in HBM, timed with CUDA events recorded by the library on
the stream its kernels run on; `e2e` is the same metric through the public C
ABI with host buffers over the same window (the state entering it uploaded
from pinned host memory, statistics read back by every step, the final
state read back). The line also carries, under "secondary", the
differentiable WCSPH workload (32,768 particles, 500 steps, forward +
backward) and the 256-scene batches (WCSPH and DFSPH) against the plain
per-scene GPU loop.

With N > 1 (torchrun) every rank runs an independent replica of the scene
(the single-scene path does not shard): weak scaling, value = all ranks'
particle-steps / max-over-ranks device time.

--impl reference times SPH2O's own OpenMP CPU path (the reference sources
built by oracle/Makefile, fast-math + OpenMP variant) on the host cores for
the same scene; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s (DFSPH 1M, batched 256 scenes, WCSPH adjoint) at ≤0.1% ρ err"
UNIT = "particle-steps/s"
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "sph2o_ref_fast")
FALLBACK_HBM_GBS = 6650.0

# Algorithmic HBM bytes per fluid particle for each timed phase (FP32, vec3 =
# 12 B, each quantity read/written once per unavoidable global dependency).
# Boundary traffic is counted per pass as 16 B per boundary particle that has
# a fluid neighbour; it is added by bytes_per_launch().
BYTES = {
    "sort": 52,            # read pos+vel 24, write reordered 24, cell offset 4
    "lists": 52 + 4,       # read pos 12 (+ 4 B count), neighbour indices written: counted separately
    "density": 20,         # read pos 12, write rho + alpha 8
    "normals": 28,         # read pos, rho -> n
    "forces": 52,          # read pos, v, rho, n -> a (viscosity + surface tension)
    "predict": 36,         # read v, a; write v
    "warm_start": 76,      # residual 36 + correction 40
    "iteration": 84,       # residual + k 44, correction 40
    "positions": 36,       # read x, v; write x
}


# Measured DRAM traffic (ncu dram__bytes_read.sum + dram__bytes_write.sum) of
# a kernel on a workload, per neighbour pass, recorded together with a hash of
# the CUDA sources the kernel is compiled from. A record is used only while
# those sources are unchanged; otherwise the line reports no traffic.
TRAFFIC_RECORDS = os.path.join(ROOT, "profiles", "density_solver_dfsph_1m_dram_traffic.json")
SOLVER_SOURCES = ("sph2o_b200/csrc/sph_solvers.cu", "sph2o_b200/csrc/sph_device.cuh",
                  "sph2o_b200/csrc/sph_internal.h")


def solver_source_key():
    """sha256 (16 hex digits) of the sources of the solver kernels."""
    h = hashlib.sha256()
    for rel in SOLVER_SOURCES:
        with open(os.path.join(ROOT, rel), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def traffic_record(kernel, workload):
    """The measured-traffic record of `kernel` on `workload` for the current
    sources, or None."""
    try:
        with open(TRAFFIC_RECORDS) as f:
            recs = json.load(f).get("records", [])
    except (OSError, ValueError):
        return None
    key = solver_source_key()
    for r in recs:
        if r.get("kernel") == kernel and r.get("workload") == workload and r.get("source_key") == key:
            return r
    return None


def workloads():
    from sph2o_b200 import scenes as S
    return {
        "double_dam_break_dfsph_1m": ("double dam break DFSPH, 1,000,000 fluid + 409,599 boundary particles, "
                                      "r=0.005 m, 4x2x2 m tank, sphere R=0.2 m", lambda: S.double_dam_break_1m()),
        "double_dam_break_pcisph_1m": ("double dam break PCISPH, 1,000,000 fluid + 409,599 boundary particles",
                                       lambda: S.double_dam_break_1m(method=S.PCISPH)),
        "dam_break_dfsph_125k": ("DFSPH dam break + Akinci surface tension, 125,000 fluid, r=0.01 m",
                                 lambda: S.dam_break_dfsph_125k()),
        "dam_break_wcsph_8k": ("WCSPH dam break, 8,000 fluid, r=0.025 m", lambda: S.dam_break_wcsph_8k()),
        "wcsph_32k": ("WCSPH block, 32,768 fluid, r=0.02 m", lambda: S.adjoint_wcsph_32k()),
    }


def batched_run(steps, warmup, method=0, count=256, loop_steps=None, indices=None):
    """Batched scenes vs the plain per-scene GPU loop on the same scenes
    (`indices`: this rank's shard of the `count` scenes, default all).
    Returns particle-steps/s of both (device events for the batch, wall clock
    for both in the ratio) and the scene statistics."""
    import time as _t

    import torch

    from sph2o_b200 import scenes as S
    from sph2o_b200.api import Batch, Scene, Simulation

    dicts = S.batched_scenes(count, method=method)
    if indices is not None:
        dicts = [dicts[s] for s in indices]
    scs = [Scene.from_dict(d) for d in dicts]
    batch = Batch(scs)
    total = batch.nf
    # launch shape and cell order picked by the library's autotuner (trial
    # steps from a snapshot that is restored), cached per GPU and workload
    tuned = batch.autotune(trial_steps=3, cache_path=os.path.join(tempfile.gettempdir(), "sph2o_autotune.json"))
    batch.step(warmup)
    torch.cuda.synchronize()
    t0 = _t.perf_counter()
    st = batch.step(steps)
    wall_batch = _t.perf_counter() - t0
    dev_ms = st["device_ms"]
    batch.close()
    loop_steps = loop_steps or steps  # the same window as the batch
    sims = [Simulation.from_scene(sc) for sc in scs]
    for sim in sims:
        sim.step(warmup)
    torch.cuda.synchronize()
    t0 = _t.perf_counter()
    for sim in sims:
        sim.step(loop_steps)
    torch.cuda.synchronize()
    wall_loop = _t.perf_counter() - t0
    for sim in sims:
        sim.close()
    for sc in scs:
        sc.close()
    batched = total * steps / (dev_ms / 1e3)
    batched_wall = total * steps / wall_batch
    loop = total * loop_steps / wall_loop
    return {"scenes": len(scs), "fluid_particles": total, "steps": steps, "value": batched,
            "value_wall": batched_wall, "per_scene_loop": loop, "speedup_vs_loop": batched_wall / loop,
            "ms_per_step": dev_ms / steps, "mean_iterations": st["total_iterations"] / max(1, steps) / count,
            "method": "WCSPH" if method == 0 else "DFSPH", "loop_steps": loop_steps, "autotuned": tuned,
            "timing": f"batch: {steps} steps after {warmup} warm-up steps; per-scene loop: {loop_steps} steps after "
                      f"the same warm-up, every scene in turn; wall clock for both in speedup_vs_loop"}


def adjoint_run(steps=500, every=50, repeats=3):
    """Differentiable WCSPH workload: 32,768 particles, 500 steps, checkpoint
    every 50; one forward + backward pair per repeat from the same initial
    state, device time from the library's events. Rate = particles x steps
    / (forward + backward) time."""
    import numpy as np

    from sph2o_b200 import scenes as S
    from sph2o_b200.api import Scene, Simulation

    sc = Scene.from_dict(S.adjoint_wcsph_32k())
    x0, _ = sc.fluid()
    v0, t = S.adjoint_problem(x0)
    sim = Simulation(sc.desc(), x0, sc.boundary(), vel=v0)
    t_0, dt_0 = sim.time()
    nf = sim.nf
    best = None
    for r in range(repeats + 1):
        sim.set_state(x0, v0)
        sim.set_time(t_0, dt_0)
        loss = sim.wcsph_forward(steps, t, ckpt_every=every)
        g = sim.wcsph_backward()
        f_ms, b_ms = sim.wcsph_timing()
        if r > 0 and (best is None or f_ms + b_ms < best[0] + best[1]):  # r == 0 warms up (graph capture)
            best = (f_ms, b_ms, loss, g)
    sim.close()
    sc.close()
    f_ms, b_ms, loss, g = best
    algo = 480.0 * nf * steps  # forward 120 B + backward ~3 x forward per particle-step
    peak, kind = hbm_peak()
    return {"workload": "differentiable WCSPH, 32,768 fluid particles (32^3, r=0.02), 500 steps at dt=2e-4, "
                        "checkpoint every 50, gradient w.r.t. v0 (32,768 x 3), viscosity and stiffness",
            "value": nf * steps / ((f_ms + b_ms) / 1e3), "unit": "particle-steps/s (forward + backward)",
            "forward_ms": f_ms, "backward_ms": b_ms, "forward_rate": nf * steps / (f_ms / 1e3),
            "loss": loss, "grad_v0_norm": float(np.linalg.norm(g["v0"].astype(np.float64))),
            "dL_dviscosity": g["viscosity"], "dL_dstiffness": g["stiffness"],
            "roofline": {"bound": "hbm", "algorithmic_bytes_per_particle_step": 480,
                         "achieved": algo / ((f_ms + b_ms) / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": algo / ((f_ms + b_ms) / 1e3) / 1e9 / peak, "peak_kind": f"of {kind}"},
            "timing": f"best of {repeats} pairs after one warm-up pair, CUDA events on the library stream"}


def l2_note(nf, nb):
    """How the timed steps stand to the 126 MB L2: the working set is the
    particle state (~7 float4 arrays + scalars, ~140 B per fluid particle),
    the neighbour lists (64 + 64 entries of 4 B per fluid particle) and the
    boundary particles (32 B each)."""
    ws = nf * (140 + 512) + nb * 32
    if ws > 126e6:
        return f"working set (~{ws / 1e6:.0f} MB: particle state + neighbour lists) larger than the 126 MB L2"
    return (f"working set (~{ws / 1e6:.1f} MB) fits in the 126 MB L2 and is not flushed between steps: "
            "a secondary workload, timed warm")


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
               "-i", str(self.gpu_id)]
        self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[0]) for r in self.rows if num(r[0]) is not None]
        mx = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[4 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def physical_cores():
    """Physical cores this process may run on (SMT siblings counted once)."""
    try:
        cpus = sorted(os.sched_getaffinity(0))
    except AttributeError:
        cpus = list(range(os.cpu_count() or 1))
    cores = set()
    for c in cpus:
        try:
            with open(f"/sys/devices/system/cpu/cpu{c}/topology/core_id") as f:
                core = f.read().strip()
            with open(f"/sys/devices/system/cpu/cpu{c}/topology/physical_package_id") as f:
                pkg = f.read().strip()
            cores.add((pkg, core))
        except OSError:
            cores.add(("cpu", c))
    return max(1, len(cores))


def reference_run(scene_dict, steps, warmup, threads=None, state=None, dt=None):
    """Time SPH2O's OpenMP CPU path on this host for the given scene: one
    OpenMP thread per physical core (OMP_PLACES=cores, OMP_PROC_BIND=close).
    `state` = (positions, velocities) replaces the scene's initial fluid
    state (caller order); `dt` the initial time step."""
    if not os.path.exists(REF_BIN):
        return None, "reference build missing (oracle/_ref/sph2o_ref_fast; run make -C oracle)"
    threads = threads or physical_cores()
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "scene.json")
        with open(path, "w") as f:
            json.dump(scene_dict, f)
        cmd = [REF_BIN, "-c", path, "--mode", "time", "--steps", str(steps), "--warmup", str(warmup),
               "--threads", str(threads)]
        if state is not None:
            from oracle import sphd
            sp = os.path.join(td, "state.sphd")
            sphd.write(sp, {"pos": np.asarray(state[0], np.float32), "vel": np.asarray(state[1], np.float32)})
            cmd += ["--state-in", sp]
        if dt is not None:
            cmd += ["--dt-in", repr(float(dt))]
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    if r.returncode != 0:
        return None, f"reference run failed: {r.stderr.strip()[-200:]}"
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    out = json.loads(line)
    out["threads"] = threads
    return out, None


def cpu_baseline_entry(res, err, sample):
    """The cpu_baseline object of a line from a reference_run result."""
    if res is None:
        return {"value": None, "unit": UNIT, "cores": physical_cores(), "kind": "reference", "sample": err}
    return {"value": res["particle_steps_per_s"], "unit": UNIT, "cores": res["threads"], "kind": "reference",
            "sample": f"{sample}; {res['steps']} timed steps after {res['warmup']} warm-up steps, SPH2O sources "
                      f"built -O3 -ffast-math -fopenmp, {res['threads']} OpenMP threads (one per physical core) "
                      f"on {cpu_model()}; mean iterations {res['mean_iterations']:.2f} + "
                      f"{res['mean_iterations_v']:.2f}"}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def bytes_per_launch(phase, nf, nb_active, its):
    if phase == "density_solve":
        per = BYTES["predict"] + BYTES["warm_start"] + its * BYTES["iteration"] + BYTES["positions"]
        passes = 2 + 2 * its
    elif phase == "divergence_solve":
        per = BYTES["warm_start"] + its * BYTES["iteration"]
        passes = 2 + 2 * its
    else:
        per = BYTES.get(phase, 0)
        passes = 1
    return nf * per + 16 * nb_active * passes


def reference_window(steps, warmup):
    """Steps of the CPU reference sample for a GPU window of `steps` timed
    steps after `warmup`: the same window when it is short (at most 40 steps,
    about 40 s on 16 cores for the 1M scene), else its first 20 steps after
    at most 5 warm-up steps."""
    if steps + warmup <= 40:
        return steps, warmup
    return min(steps, 20), min(warmup, 5)


def run_reference_arm(args, name, desc, scene_dict, world, rank):
    if rank != 0:
        return 0
    steps, warm = reference_window(args.steps, args.warmup)
    res, err = reference_run(scene_dict, steps, warm)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    v = res["particle_steps_per_s"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": warm, "ms_per_step": 1e3 * res["seconds"] / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "fluid_particles": res["fluid_particles"],
                   "boundary_particles": res["boundary_particles"], "mean_iterations": res["mean_iterations"],
                   "mean_iterations_v": res["mean_iterations_v"]},
        "cpu_baseline": cpu_baseline_entry(res, None, "the same scene and step window as the GPU arm"),
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---- across ranks (one process per GPU; gloo on CPU in the tests) -------------------------------------------

def max_over_ranks(x, world, device="cpu"):
    """The largest of a per-rank number over all ranks (all_reduce MAX)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world, device="cpu"):
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_value(particles, steps, device_ms, world, device="cpu"):
    """Whole-job particle-steps/s of `world` replicas of one scene: all ranks'
    particle-steps over the slowest rank's device time."""
    max_ms = max_over_ranks(device_ms, world, device)
    return world * particles * steps / (max_ms / 1e3), max_ms


def batch_shard(count, world, rank):
    """This rank's scenes of the batched workload (greedy longest-processing-
    time on fluid particles; every rank computes the same partition)."""
    from sph2o_b200 import scenes as S
    from sph2o_b200.sharding import scene_cost, shard_for_rank
    costs = [scene_cost(p["dims"][0] * p["dims"][1] * p["dims"][2]) for p in S.batched_scene_params(count)]
    return shard_for_rank(costs, world, rank)


def combine_batch_results(res, world, device="cpu"):
    """Whole-job batched rate: all ranks' fluid particles over the slowest
    rank's step time (no collective touches particle data)."""
    if world <= 1:
        return res
    tmax = max_over_ranks(res["ms_per_step"], world, device)
    tot = sum_over_ranks(res["fluid_particles"], world, device)
    res = dict(res)
    res["value"] = tot / (tmax / 1e3)
    res["fluid_particles_all_ranks"] = int(tot)
    res["ms_per_step_max_rank"] = tmax
    return res


# ---- secondary workloads --------------------------------------------------------------------------------------

def config_run(name, steps, warmup, cpu=True, cpu_window=None, tune=True):
    """One named workload on this GPU (device-timed window of `steps` after
    `warmup`) and, when cpu, the reference's OpenMP path on the host cores over
    `cpu_window` = (steps, warmup) (default: the same window). With tune, the
    library's autotuner picks cell order, solver occupancy, pass block and
    solver lanes first (trial steps from a restored snapshot, cached per GPU
    and workload)."""
    from sph2o_b200.api import Scene, Simulation
    desc, make = workloads()[name]
    d = make()
    scene = Scene.from_dict(d)
    sim = Simulation.from_scene(scene)
    nf, nb = sim.nf, sim.nb
    tuned = None
    if tune:
        tuned = sim.autotune(trial_steps=3, cache_path=os.path.join(tempfile.gettempdir(), "sph2o_autotune.json"))
    if warmup:
        sim.step(warmup)
    st = sim.step(steps)
    sim.close()
    scene.close()
    out = {"workload": desc, "fluid_particles": nf, "boundary_particles": nb, "steps": steps, "warmup": warmup,
           "value": nf * steps / (st["device_ms"] / 1e3), "unit": UNIT, "ms_per_step": st["device_ms"] / steps,
           "mean_iterations": st["total_iterations"] / steps, "mean_iterations_v": st["total_iterations_v"] / steps,
           "last_avg_density_error": st["avg_density_error"], "l2": l2_note(nf, nb), "autotuned": tuned,
           "timing": "CUDA events on the library stream around the window"}
    if cpu:
        cs, cw = cpu_window or (steps, warmup)
        res, err = reference_run(d, cs, cw)
        out["cpu_baseline"] = cpu_baseline_entry(
            res, err, "the same scene and step window" if (cs, cw) == (steps, warmup) else "the same scene")
        if res is not None:
            out["vs_cpu_baseline"] = out["value"] / res["particle_steps_per_s"]
    return out


def later_window_run(scene_dict, desc, start, steps, cpu=True, cpu_steps=5, cpu_warmup=3):
    """The same scene later in the run: steps start + 1 .. start + steps (the
    first `start` steps untimed). The CPU reference starts from the GPU's
    state after step `start` (positions, velocities and time step; its
    solver warm start begins empty), takes a few warm-up steps, then a
    bounded sample."""
    from sph2o_b200.api import Scene, Simulation
    scene = Scene.from_dict(scene_dict)
    sim = Simulation.from_scene(scene)
    nf = sim.nf
    sim.step(start)
    x, v, _ = sim.state()
    _, dt_start = sim.time()
    st = sim.step(steps)
    sim.close()
    scene.close()
    out = {"workload": desc + f", steps {start + 1}-{start + steps}", "fluid_particles": nf, "steps": steps,
           "warmup": start, "value": nf * steps / (st["device_ms"] / 1e3), "unit": UNIT,
           "ms_per_step": st["device_ms"] / steps, "mean_iterations": st["total_iterations"] / steps,
           "mean_iterations_v": st["total_iterations_v"] / steps, "last_avg_density_error": st["avg_density_error"],
           "density_error_gate": bool(st["avg_density_error"] <= 1e-3), "simulated_time_s": st["time"]}
    if cpu:
        res, err = reference_run(scene_dict, cpu_steps, cpu_warmup, state=(x, v), dt=dt_start)
        out["cpu_baseline"] = cpu_baseline_entry(res, err, f"the same scene from the GPU state after step {start}")
        if res is not None:
            out["vs_cpu_baseline"] = out["value"] / res["particle_steps_per_s"]
    return out


def neighbor_search_roofline(nf, entries, prof, steps, peak, peak_kind):
    """Sort + list build against HBM: algorithmic bytes per fluid particle =
    52 (sort: read position and velocity 24, write them reordered 24, cell
    offset 4) + 20 (list build: read position 12, write two list lengths 8)
    + 4 per neighbour-list entry written, over their event time per step."""
    ms = (prof["sort"]["ms"] + prof["lists"]["ms"]) / steps
    algo = nf * (52 + 20) + 4 * entries
    achieved = algo / (ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": f"of {peak_kind}", "algorithmic_bytes_per_step": algo, "ms_per_step": ms,
            "list_entries_per_particle": entries / nf,
            "kernels": "k_ns_count, scan, k_ns_scatter, k_ns_rank_gather (sort); k_ns_build_lists (lists)"}


def pair_evaluations(entries, its, itsv, prof, steps, window_ms, surface_tension=False):
    """Neighbour-pair evaluations of a DFSPH step (the pair-bound side of the
    roofline): every list entry (fluid and boundary) is evaluated once per
    neighbour pass. Passes per step: density + alpha + divergence error,
    surface-tension normals when on, non-pressure forces, the density solver's
    warm start (2) and 2 per iteration, the divergence solver's warm-start
    correction (its residual comes from the density pass) and 2 per
    iteration."""
    passes = 2 + (1 if surface_tension else 0) + (2 + 2 * its) + (1 + 2 * itsv)
    solver_passes = 2 + 2 * its
    return {"list_entries": entries, "passes_per_step": passes,
            "per_step": entries * passes, "per_s": entries * passes * steps / (window_ms / 1e3),
            "density_solver_per_s": entries * solver_passes * steps / (prof["density_solve"]["ms"] / 1e3),
            "unit": "neighbour-pair evaluations"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="double_dam_break_dfsph_1m")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-only", action="store_true", help="time only the batched-scenes workload")
    ap.add_argument("--batch-method", type=int, default=0)
    ap.add_argument("--batch-scenes", type=int, default=256)
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the secondary workloads (other configurations, later window, adjoint, batches)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    name = args.workload
    desc, make = workloads()[name]
    scene_dict = make()

    if args.impl == "reference":
        return run_reference_arm(args, name, desc, scene_dict, world, rank)
    if args.batch_only:
        import torch
        torch.cuda.set_device(local)
        res = batched_run(args.steps, args.warmup, method=args.batch_method, count=args.batch_scenes)
        print(json.dumps(res))
        return 0

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    from sph2o_b200.api import Scene, Simulation, select_device

    select_device(local)
    scene = Scene.from_dict(scene_dict)
    sim = Simulation.from_scene(scene)
    nf, nb = sim.nf, sim.nb
    if args.warmup > 0:
        sim.step(args.warmup)
    # the state entering the timed window, kept in pinned host memory so the
    # end-to-end run below replays the same window through the public API
    px = torch.empty((nf, 3), dtype=torch.float32, pin_memory=True).numpy()
    pv = torch.empty((nf, 3), dtype=torch.float32, pin_memory=True).numpy()
    # the window's results go to their own pinned buffers, so the inputs stay
    # as they are and no host copy restores them between runs of the window
    ox = torch.empty((nf, 3), dtype=torch.float32, pin_memory=True).numpy()
    ov = torch.empty((nf, 3), dtype=torch.float32, pin_memory=True).numpy()
    pr = torch.empty(nf, dtype=torch.float32, pin_memory=True).numpy()
    x_w, v_w, _ = sim.state()
    px[:] = x_w
    pv[:] = v_w
    t_w, dt_w = sim.time()

    gpu_uuid = torch.cuda.get_device_properties(local).uuid
    sampler = ClockSampler(f"GPU-{gpu_uuid}" if gpu_uuid else local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    sim.profile(True)
    t0 = time.perf_counter()
    stats = sim.step(args.steps)
    wall = time.perf_counter() - t0
    prof = sim.profile_read()
    sim.profile(False)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()

    value, max_ms = replica_value(nf, args.steps, stats["device_ms"], world, dev)
    its = stats["total_iterations"] / max(args.steps, 1)
    itsv = stats["total_iterations_v"] / max(args.steps, 1)

    # roofline of the dominant kernel (largest device time in the timed region)
    peak, peak_kind = hbm_peak()
    dom = max((k for k in prof if prof[k]["launches"]), key=lambda k: prof[k]["ms"])
    launches = prof[dom]["launches"]
    avg_ms = prof[dom]["ms"] / launches
    it_for = its if dom == "density_solve" else itsv
    # (the boundary term, boundary particles with a fluid neighbour, is
    # counted from the lists after the end-to-end run below)
    algo = bytes_per_launch(dom, nf, 0, it_for)
    achieved = algo / (avg_ms / 1e3) / 1e9
    traffic, traffic_note = None, "no DRAM capture recorded for this build of the kernel"
    rec = traffic_record("k_dfsph_solve(density)", name) if dom == "density_solve" else None
    if rec is not None:
        traffic = rec["dram_bytes_per_pass"] * (2 + 2 * it_for)
        traffic_note = (f"ncu DRAM bytes per neighbour pass of this kernel on this workload, captured for this "
                        f"build of the solver sources (key {rec['source_key']}), x the window's mean passes per "
                        f"launch")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_note": traffic_note, "kernel": dom, "peak_kind": f"of {peak_kind}",
                "algorithmic_bytes_per_launch": algo, "avg_launch_ms": avg_ms}

    # End to end through the C ABI with host buffers, over the same window:
    # the state entering it is uploaded from pinned host memory, every step
    # is one sph_step call that returns its statistics (density error,
    # iterations) to the host, and the final state is read back.
    from sph2o_b200.api import StepStats, _fptr, lib
    L = lib()
    ke = args.steps

    def api_window():
        """The caller's sequence: upload, ke single steps with their
        statistics, read back. Returns (status, iterations)."""
        rc = L.sph_set_state(sim._h, _fptr(px), _fptr(pv))
        rc = rc or L.sph_set_time(sim._h, t_w, dt_w)
        its_sum = 0
        st1 = StepStats()
        for _ in range(ke):
            if rc:
                break
            rc = L.sph_step(sim._h, 1, st1)
            its_sum += st1.total_iterations
        rc = rc or L.sph_get_state(sim._h, _fptr(ox), _fptr(ov), _fptr(pr))
        return rc, its_sum

    # untimed once: the library captures its one-step CUDA graphs (one per
    # buffer assignment the single steps pass through) on first use
    api_window()
    # the window is timed three times and the median reported: its host part
    # (PCIe copies, one host round trip per step) varies with the load of the
    # shared host more than the device part does
    windows = []
    rc, e2e_its = 0, 0
    for _ in range(3):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc, e2e_its = api_window()
        windows.append(max_over_ranks(time.perf_counter() - t0, world, dev))
        if rc:
            break
    e2e_s = statistics.median(windows)
    e2e = None
    if rc == 0:
        e2e = {"value": world * nf * ke / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": (nf * 24) // ke,
               "d2h_bytes_per_step": ctypes.sizeof(StepStats) + (nf * 28) // ke,
               "steps": ke, "mean_iterations": e2e_its / ke,
               "windows_ms": [round(w * 1e3, 3) for w in windows],
               "note": "state uploaded once from pinned host memory, per-step statistics read back by every "
                       "sph_step call, final state (x, v, rho) read back; same window as value; median of three "
                       "timed runs of the window after one untimed run of the same calls (one-step graph "
                       "capture)"}
    # boundary particles with a fluid neighbour (the boundary is static; the
    # fluid's reach changes little over a window), read from the lists after
    # the timed runs: reading the lists back before the end-to-end window
    # slowed that window by ~25 %
    fo, fi, bo, bi = sim.neighbors()
    nb_active = int(np.unique(bi).size)
    list_entries = int(fi.size) + int(bi.size)
    del fo, fi, bo, bi
    algo = bytes_per_launch(dom, nf, nb_active, it_for)
    achieved = algo / (avg_ms / 1e3) / 1e9
    roofline.update({"achieved": achieved, "frac": achieved / peak, "algorithmic_bytes_per_launch": algo,
                     "boundary_particles_with_fluid_neighbour": nb_active})
    roofline["neighbor_search"] = neighbor_search_roofline(nf, list_entries, prof, args.steps, peak, peak_kind)
    if scene_dict["Configuration"].get("simulationMethod") == 2:
        roofline["pair_evaluations"] = pair_evaluations(list_entries, its, itsv, prof, args.steps, max_ms,
                                                        surface_tension=any(
                                                            fm.get("surfaceTension", 0.0) != 0.0
                                                            for fm in scene_dict["Fluid"]["FluidModel"]))
    sim.close()
    scene.close()

    cpu = None
    on_cpu = rank == 0 and world == 1 and not args.no_cpu_baseline
    if on_cpu:
        cs, cw = reference_window(args.steps, args.warmup)
        res, err = reference_run(scene_dict, cs, cw)
        cpu = cpu_baseline_entry(res, err, "the same scene" + (" and step window as value"
                                                               if (cs, cw) == (args.steps, args.warmup) else ""))

    secondary = None
    if not args.no_secondary:
        secondary = {}
        if name == "double_dam_break_dfsph_1m":
            secondary["double_dam_break_dfsph_1m_later"] = later_window_run(scene_dict, desc, 200, 100, cpu=on_cpu)
        secondary["double_dam_break_pcisph_1m"] = config_run("double_dam_break_pcisph_1m", 20, 5, cpu=on_cpu,
                                                             cpu_window=(5, 2))
        secondary["dam_break_wcsph_8k"] = config_run("dam_break_wcsph_8k", 2000, 20, cpu=on_cpu)
        secondary["dam_break_dfsph_125k"] = config_run("dam_break_dfsph_125k", 50, 20, cpu=on_cpu,
                                                       cpu_window=(30, 20))
        secondary["adjoint_wcsph_32k"] = adjoint_run()
        # independent scenes shard across ranks: each steps its own subset as
        # one batch; only the timing and particle totals are reduced
        shard = batch_shard(args.batch_scenes, world, rank)
        for m, bname in ((0, "batched_wcsph_256"), (2, "batched_dfsph_256")):
            res = batched_run(50, 3, method=m, count=args.batch_scenes, indices=shard)
            res = combine_batch_results(res, world, dev)
            res["sharding"] = {"ranks": world, "scenes_this_rank": len(shard),
                               "rule": "greedy longest-processing-time on fluid particles, no collective on particle data"}
            secondary[bname] = res

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "fluid_particles": nf, "boundary_particles": nb,
                   "parallelism": "replicas" if world > 1 else "single",
                   "mean_iterations": its, "mean_iterations_v": itsv,
                   "last_avg_density_error": stats["avg_density_error"],
                   "density_error_gate": bool(stats["avg_density_error"] <= 1e-3),
                   "simulated_time_s": stats["time"], "dt": stats["dt"],
                   "l2": l2_note(nf, nb),
                   "wall_s": wall},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": stats["kernel_launches"],
        "clocks": clocks,
        "phases_ms_per_step": {k: prof[k]["ms"] / args.steps for k in prof if prof[k]["launches"]},
        "secondary": secondary,
    }
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
