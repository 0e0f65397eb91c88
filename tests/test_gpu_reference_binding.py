"""The reference-side binding (include/sph2o_gpu_solver.hpp) compiled against
SPH2O's own headers and objects, and the frame output, against SPH2O.

oracle/_ref/sph2o_ref_gpu is the unmodified SPH2O sources (FP32 build) plus
the harness, with the scene's CPU solver handed to a GPUSolver after import,
as a maintainer would do in SPHSimulation::init(); SPHSimulation::init,
SPHSimulation::step and SceneLoader::writeFluid then run unchanged around
the GPU step. Checks:
  * stepping a golden scene through SPHSimulation::step() with the binding
    gives the ABI run's state bit for bit, with the same iteration counts;
  * frames: the reference's own run (TimeHelper::hasToSave +
    SceneLoader::writeFluid), the binding inside SPH2O, and this
    repository's driver (sph2o -o true) write the same frame files (names
    and count); the binding's and the driver's frames are identical (the
    binding run reports that SPH2O stepped with the GPU solver); against the
    reference's frames: WCSPH time and time step equal, positions and
    velocities within 1e-5 (norm-wise); DFSPH time and time step within
    1e-5, positions within 1e-5, velocities within 2e-4 -- the bars of
    test_gpu_parity (the force pass is held to a relative tolerance, not to
    the bit, so near-cancelling velocity components differ in their last
    bits).
"""
import glob
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden, rel_err
from oracle import sphd
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation

pytestmark = pytest.mark.gpu
REF32 = os.path.join(ROOT, "oracle", "_ref", "sph2o_ref_f32")
REFGPU = os.path.join(ROOT, "oracle", "_ref", "sph2o_ref_gpu")
DRIVER = os.path.join(ROOT, "sph2o_b200", "bin", "sph2o")
need = pytest.mark.skipif(not (os.path.exists(REF32) and os.path.exists(REFGPU) and os.path.exists(DRIVER)),
                          reason="reference builds missing (make -C oracle ref gpu-binding)")


def write_scene(d, directory, name="scene.json"):
    os.makedirs(directory, exist_ok=True)
    p = os.path.join(str(directory), name)
    with open(p, "w") as f:
        json.dump(d, f)
    return p


@need
@pytest.mark.parametrize("name", ["wcsph_artificial", "dfsph_st_sphere", "pcisph_artificial"])
def test_binding_steps_like_the_abi(name, tmp_path):
    g = load_golden(name)
    scene = write_scene(g["scene"], tmp_path)
    out = os.path.join(str(tmp_path), "o.sphd")
    steps = 10
    subprocess.run([REFGPU, "-c", scene, "--mode", "step", "--steps", str(steps), "--out", out, "--gpu"], check=True,
                   capture_output=True)
    ref = sphd.read(out)
    sim = Simulation.from_scene(Scene.from_dict(g["scene"]))
    for s in range(steps):
        st = sim.step(1)
        assert st["iterations"] == int(ref["step_stats"][s, 2]), s
        assert np.float32(st["time"]) == np.float32(ref["step_stats"][s, 0]), s
    x, v, rho = sim.state()
    sim.close()
    assert np.array_equal(x, ref["pos"]) and np.array_equal(v, ref["vel"]) and np.array_equal(rho, ref["density"])


def read_frames(directory):
    out = {}
    for p in sorted(glob.glob(os.path.join(str(directory), "scene_*.json"))):
        with open(p) as f:
            d = json.load(f)
        out[os.path.basename(p)] = {"time": np.float32(d["time"]), "timeStep": np.float32(d["timeStep"]),
                                    "n": (d["numParticles"], d["numActiveParticles"]),
                                    "x": np.asarray(d["positions"], np.float32),
                                    "v": np.asarray(d["velocities"], np.float32)}
    return out


@need
@pytest.mark.parametrize("method", [S.WCSPH, S.DFSPH], ids=["wcsph", "dfsph"])
def test_frames_match_the_reference(method, tmp_path):
    d = S.small(method=method, n=(8, 8, 8), seed=3, fps=2000.0, time_step=1e-4)
    steps = 23  # 2.3 ms at dt = 1e-4 (WCSPH): four frames at 1/fps = 0.5 ms
    dirs = {k: tmp_path / k for k in ("reference", "binding", "driver")}
    s_ref = write_scene(d, dirs["reference"])
    s_bind = write_scene(d, dirs["binding"])
    s_drv = write_scene(d, dirs["driver"])
    subprocess.run([REF32, "-c", s_ref, "--mode", "frames", "--steps", str(steps)], check=True, capture_output=True)
    r = subprocess.run([REFGPU, "-c", s_bind, "--mode", "frames", "--steps", str(steps), "--gpu"], check=True,
                       capture_output=True, text=True)
    info = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert info["gpu_solver"] is True
    subprocess.run([DRIVER, "-c", s_drv, "-o", "true", "--steps", str(steps), "--quiet"], check=True,
                   capture_output=True)
    ref, bind, drv = (read_frames(dirs[k]) for k in ("reference", "binding", "driver"))
    assert len(ref) >= 2
    assert sorted(ref) == sorted(bind) == sorted(drv)
    for name in ref:
        a, b, c = ref[name], bind[name], drv[name]
        assert b["n"] == c["n"] == a["n"], name
        for key in ("time", "timeStep"):
            assert b[key] == c[key], (name, key)
        assert np.array_equal(b["x"], c["x"]) and np.array_equal(b["v"], c["v"]), name
        if method == S.WCSPH:
            assert a["time"] == b["time"] and a["timeStep"] == b["timeStep"], name
            assert rel_err(b["x"], a["x"]) <= 1e-5, name
            assert rel_err(b["v"], a["v"]) <= 1e-5, name
        else:
            assert abs(float(a["time"]) - float(b["time"])) <= 1e-5 * float(a["time"]), name
            assert abs(float(a["timeStep"]) - float(b["timeStep"])) <= 1e-5 * float(a["timeStep"]), name
            assert rel_err(b["x"], a["x"]) <= 1e-5, name
            assert rel_err(b["v"], a["v"]) <= 2e-4, name
