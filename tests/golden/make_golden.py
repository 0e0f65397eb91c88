"""Generates the golden fixtures in this directory by running the SPH2O
reference itself (oracle/_ref/sph2o_ref_f32 and _f64, built by
`make -C oracle` from the reference sources).

    python tests/golden/make_golden.py

For every small scene below it stores, in <name>.npz:
  scene            the scene JSON text
  init_pos, bpos   particles as the reference builds them (lattice + jitter,
                   Akinci box/sphere sampling), f32
  bvol             Akinci boundary volumes after init, f32
  density, alpha   SPHSolver::computeDensities / DFSPHSolver::computeAlpha at
                   the initial positions (phase mode), f32
  a_np             SPHSimulation::computeNonPressureForces, f32
  pressure, a_pressure   WCSPH computePressures / computePressureForce, f32
  nbr_*            neighbour sets N(i) = {j in 27 cells : |xi - xj| <= h}
                   in the reference's candidate order (CSR), u32
  step1_pos/vel/density  state after one SPHSimulation::step(), f32
  step1_*_f64      the same from the FP64 build (same float inputs)
  trace_f32, trace_f64   per-step [time, dt, iterations, iterationsV,
                   avg density residual, avg divergence residual,
                   centroid x y z, kinetic energy, mean density error] over
                   NSTEPS steps (STEPS for the emitter scenes), from the FP32-strict and FP64 builds (the FP64
                   run starts from the same float inputs)
  final_pos_f64, final_vel_f64   FP64 state after NSTEPS steps
  active_f32, active_f64   active fluid particles after every step (emitter
                   scenes; emitted particles take the slots after the active ones)

The OBJ meshes of the geometry scenes (sph2o_b200.scenes.GEOMETRY_MESHES)
are written beside the fixtures as <name>.obj; the stored scene refers to
them by bare file name, the reference is run on a copy with absolute paths.

    python tests/golden/make_golden.py [name ...]    # default: every scene

Test infrastructure only.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import sphd  # noqa: E402
from sph2o_b200 import scenes as S  # noqa: E402

NSTEPS = 20
# emitter scenes run long enough for several emissions
STEPS = {"emitter_wcsph_square": 120, "emitter_dfsph_circle": 120, "cube_dfsph_floor": 120,
         "pcib_wcsph_sphere": 120, "pcib_pcisph": 60, "pcib_dfsph_sphere": 60, "pcib_wcsph_farwall": 400,
         "pcib_wcsph_wallslide": 400}
REF32 = os.path.join(ROOT, "oracle", "_ref", "sph2o_ref_f32")
REF64 = os.path.join(ROOT, "oracle", "_ref", "sph2o_ref_f64")


def golden_scenes():
    return {
        **S.emitter_scenes(),
        **S.cube_scenes(),
        **S.geometry_scenes(),
        **S.pcisph_boundary_scenes(),
        "dfsph_st_sphere": S.small(method=S.DFSPH, surface_tension=0.05, sphere=True),
        "wcsph_artificial": S.small(method=S.WCSPH, n=(12, 10, 10)),
        "pcisph_artificial": S.small(method=S.PCISPH, n=(10, 10, 12), eta=0.01, time_step=5e-4),
        "dfsph_standard_adhesion": S.small(method=S.DFSPH, viscosity_method=S.VISC_STANDARD, viscosity=0.05,
                                           boundary_viscosity=0.01, adhesion=0.5),
        "wcsph_xsph_st_adhesion": S.small(method=S.WCSPH, viscosity_method=S.VISC_XSPH, viscosity=0.1,
                                          boundary_viscosity=0.05, surface_tension=0.05, adhesion=0.5),
    }


def run(binary, scene_path, mode, out, *extra):
    r = subprocess.run([binary, "-c", scene_path, "--mode", mode, "--out", out, *extra], capture_output=True,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{binary} {mode} failed: {r.stderr}")
    return sphd.read(out)


def write_meshes():
    for fname, text in S.GEOMETRY_MESHES.items():
        with open(os.path.join(HERE, fname), "w", newline="") as f:
            f.write(text())


def make(name, scene, td):
    path = os.path.join(td, name + ".json")
    with open(path, "w") as f:
        json.dump(S.resolve_geometry_paths(scene, HERE), f)
    g = {"scene": np.array(json.dumps(scene))}
    nb = run(REF32, path, "neighbors", os.path.join(td, "nb.sphd"))
    for k in ("init_pos", "bpos", "nbr_f_offsets", "nbr_f", "nbr_b_offsets", "nbr_b"):
        g[k] = nb[k]
    ph = run(REF32, path, "phases", os.path.join(td, "ph.sphd"))
    g["bvol"] = ph.get("bvol", np.zeros(0, np.float32))  # absent without Akinci boundary particles
    for k in ("bnormal", "bdensity", "bpressure"):  # PCISPH boundary particles
        if k in ph:
            g[k] = ph[k]
    g["density"] = ph["density"]
    g["a_np"] = ph["a_nonpressure"]
    for k in ("alpha", "pressure", "a_pressure"):
        if k in ph:
            g[k] = ph[k]
    s1 = run(REF32, path, "step", os.path.join(td, "s1.sphd"), "--steps", "1")
    g["step1_pos"], g["step1_vel"], g["step1_density"] = s1["pos"], s1["vel"], s1["density"]
    nsteps = STEPS.get(name, NSTEPS)
    sn = run(REF32, path, "step", os.path.join(td, "sn.sphd"), "--steps", str(nsteps))
    g["trace_f32"] = sn["step_stats"]
    g["active_f32"] = sn["active"]
    g["final_pos_f32"], g["final_vel_f32"] = sn["pos"], sn["vel"]
    state = os.path.join(td, "state.sphd")
    sphd.write(state, {"pos": nb["init_pos"].astype(np.float64)})
    bnd = os.path.join(td, "bnd.sphd")
    sphd.write(bnd, {"bpos": nb["bpos"].astype(np.float64)})
    s1d = run(REF64, path, "step", os.path.join(td, "s1d.sphd"), "--steps", "1", "--state-in", state,
              "--boundary-in", bnd)
    g["step1_pos_f64"], g["step1_vel_f64"], g["step1_density_f64"] = s1d["pos"], s1d["vel"], s1d["density"]
    s64 = run(REF64, path, "step", os.path.join(td, "s64.sphd"), "--steps", str(nsteps), "--state-in", state,
              "--boundary-in", bnd)
    g["trace_f64"] = s64["step_stats"]
    g["active_f64"] = s64["active"]
    g["final_pos_f64"], g["final_vel_f64"] = s64["pos"], s64["vel"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **g)
    return g


def main():
    for b in (REF32, REF64):
        if not os.path.exists(b):
            raise SystemExit(f"{b} missing: run make -C oracle first")
    want = set(sys.argv[1:])
    write_meshes()
    with tempfile.TemporaryDirectory() as td:
        for name, scene in golden_scenes().items():
            if want and name not in want:
                continue
            g = make(name, scene, td)
            print(name, g["init_pos"].shape[0], "fluid", g["bpos"].shape[0], "boundary")


if __name__ == "__main__":
    main()
