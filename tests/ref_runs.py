"""Runs of the SPH2O reference harness for the GPU tests (test
infrastructure): oracle/_ref/sph2o_ref_f32 (FP32, strict IEEE) and
sph2o_ref_f64 (Real = double), both the unmodified reference sources built
by oracle/Makefile and driven by oracle/ref_harness.cpp, plus the bars the
trace comparisons use."""
import json
import os
import subprocess
import time

import numpy as np

from conftest import ROOT, rel_err
from oracle import sphd

REF32 = os.path.join(ROOT, "oracle", "_ref", "sph2o_ref_f32")
REF64 = os.path.join(ROOT, "oracle", "_ref", "sph2o_ref_f64")


def have_reference():
    return os.path.exists(REF32) and os.path.exists(REF64)


class Reference:
    """Runs the reference harness on one scene in a scratch directory."""

    def __init__(self, scene, workdir):
        self.dir = str(workdir)
        os.makedirs(self.dir, exist_ok=True)
        self.scene = os.path.join(self.dir, "scene.json")
        with open(self.scene, "w") as f:
            json.dump(scene, f)
        self.seconds = {}

    def run(self, binary, mode, steps=1, name=None, state=None, boundary=None):
        name = name or f"{os.path.basename(binary)}_{mode}_{steps}"
        out = os.path.join(self.dir, name + ".sphd")
        cmd = [binary, "-c", self.scene, "--mode", mode, "--steps", str(steps), "--out", out]
        if state is not None:
            p = os.path.join(self.dir, name + "_state.sphd")
            sphd.write(p, {"pos": np.asarray(state, np.float64)})
            cmd += ["--state-in", p]
        if boundary is not None:
            p = os.path.join(self.dir, name + "_boundary.sphd")
            sphd.write(p, {"bpos": np.asarray(boundary, np.float64)})
            cmd += ["--boundary-in", p]
        t0 = time.perf_counter()
        subprocess.run(cmd, check=True, capture_output=True)
        self.seconds[name] = round(time.perf_counter() - t0, 2)
        return sphd.read(out)

    def f64_from_f32_inputs(self, ref32, mode, steps):
        """The FP64 build started from the FP32 build's float particles (its
        own box sampler yields a different boundary count)."""
        return self.run(REF64, mode, steps, state=ref32["init_pos"].astype(np.float64),
                        boundary=ref32["bpos"].astype(np.float64))


def aggregates(x, v, rho, rho0, mass):
    x64, v64 = x.astype(np.float64), v.astype(np.float64)
    return (x64.mean(axis=0), 0.5 * mass * float((v64 * v64).sum()),
            float(np.mean(np.maximum(rho.astype(np.float64) - rho0, 0.0) / rho0)))


def check_aggregates(x, v, rho, rho0, mass, row64, row32):
    """Centroid within 1e-6 m, kinetic energy within 2e-3 relative, mean
    density error within 1e-6 of the FP64 reference -- or within twice the
    FP32 reference's own distance from it where that is larger.
    row*: one step_stats row [time, dt, its, itsV, avg, avgV, cx, cy, cz, ke, derr]."""
    c, ke, de = aggregates(x, v, rho, rho0, mass)
    spread = np.abs(np.asarray(row32) - np.asarray(row64))
    assert np.max(np.abs(c - row64[6:9])) <= max(1e-6, 2 * float(np.max(spread[6:9]))), (c, row64[6:9])
    assert abs(ke - row64[9]) <= max(2e-3 * abs(row64[9]), 2 * float(spread[9])), (ke, row64[9])
    assert abs(de - row64[10]) <= max(1e-6, 2 * float(spread[10])), (de, row64[10])


def check_trace(stats, row32, s):
    """Iteration counts equal to the FP32 reference's; time and dt within 1e-5."""
    assert stats["iterations"] == int(row32[2]), f"step {s}: iterations {stats['iterations']} vs {row32[2]}"
    assert stats["iterations_v"] == int(row32[3]), f"step {s}: iterations_v {stats['iterations_v']} vs {row32[3]}"
    assert abs(stats["time"] - row32[0]) <= 1e-5 * row32[0], f"step {s}: time"
    assert abs(stats["dt"] - row32[1]) <= 1e-5 * row32[1], f"step {s}: dt"


def check_state_vs_f64(x, v, r32, r64):
    """State after several steps: no further from the FP64 reference than
    1.5x the FP32 reference's own distance from it (or 1e-5), positions and
    velocities norm-wise. After one step the FP32 bars hold; over several
    steps the solvers' FP32 round-off (residuals of a difference of two
    ~1000 densities) grows in both FP32 implementations alike."""
    ex, ev = rel_err(r32["pos"], r64["pos"]), rel_err(r32["vel"], r64["vel"])
    gx, gv = rel_err(x, r64["pos"]), rel_err(v, r64["vel"])
    print(f"positions: GPU-FP64 {gx:.3g}, FP32 ref-FP64 {ex:.3g}; velocities: GPU-FP64 {gv:.3g}, FP32 ref-FP64 {ev:.3g}")
    assert gx <= max(1e-5, 1.5 * ex), (gx, ex)
    assert gv <= max(1e-5, 1.5 * ev), (gv, ev)
