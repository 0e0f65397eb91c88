"""The sph2o driver (host/sph2o_main.cpp): SPH2O's -c/-g/-o/-f command line
on the GPU path. Frames are SceneLoader::writeFluid's JSON; a run resumed
from a frame reproduces the straight run (WCSPH carries no other state)."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation

pytestmark = pytest.mark.gpu
DRIVER = os.path.join(ROOT, "sph2o_b200", "bin", "sph2o")


def scene_file(tmp_path, **kw):
    sc = S.small(method=S.WCSPH, n=(8, 8, 8), end_time=0.003, fps=2000.0, **kw)
    p = tmp_path / "tank.json"
    p.write_text(json.dumps(sc))
    return p, sc


def run(*args):
    r = subprocess.run([DRIVER, *map(str, args), "--quiet"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout, json.loads(r.stdout.strip().splitlines()[-1])


def test_frames_match_api_run(tmp_path):
    p, sc = scene_file(tmp_path)
    out, summary = run("-c", p, "-g", "false", "-o", "true")
    frames = sorted(f for f in os.listdir(tmp_path) if f.startswith("tank_") and f.endswith(".json"))
    assert len(frames) == summary["frames"] >= 5
    assert frames[0] == "tank_0001.json"
    last = json.loads((tmp_path / frames[-1]).read_text())
    assert set(last) == {"numActiveParticles", "numParticles", "positions", "time", "timeStep", "velocities"}
    steps = summary["steps"]
    # every step: dt = 1e-4, frames every 5e-4 s -> the last frame is written after the last multiple of 5 steps
    sim = Simulation.from_scene(Scene.from_dict(sc))
    t = np.float32(0.0)
    n_at_last = None
    for k in range(steps):
        sim.step(1)
        t = np.float32(t + np.float32(sc["Configuration"]["timeStep"]))
        if abs(float(t) - last["time"]) < 1e-12:
            n_at_last = k + 1
            x, v, _ = sim.state()
            break
    assert n_at_last is not None
    assert np.array_equal(np.asarray(last["positions"], np.float32), x)
    assert np.array_equal(np.asarray(last["velocities"], np.float32), v)


def test_resume_reproduces_straight_run(tmp_path):
    p, _ = scene_file(tmp_path)
    run("-c", p, "-o", "true")
    frames = sorted(f for f in os.listdir(tmp_path) if f.startswith("tank_"))
    final = json.loads((tmp_path / frames[-1]).read_text())
    for f in frames[2:]:
        os.remove(tmp_path / f)
    run("-c", p, "-o", "true", "-f", 2)
    resumed = json.loads((tmp_path / frames[-1]).read_text())
    assert resumed["time"] == final["time"]
    assert resumed["positions"] == final["positions"]
    assert resumed["velocities"] == final["velocities"]


def test_graphics_flag_runs_headless(tmp_path):
    p, _ = scene_file(tmp_path)
    out, summary = run("-c", p, "-g", "true", "--steps", 3)
    assert "graphics unavailable" in out
    assert summary["steps"] == 3


def test_bad_scene_fails_cleanly(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text('{"Configuration": {}}')
    r = subprocess.run([DRIVER, "-c", str(p), "-g", "false"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Cannot import scene" in r.stderr


def last_frame_matches_api(tmp_path, scene_dict, api_scene):
    """Runs the driver on scene_dict (written beside its OBJ meshes) and
    checks its last frame against the API stepped to the same time."""
    out, summary = run("-c", tmp_path / "scene.json", "-g", "false", "-o", "true")
    frames = sorted(f for f in os.listdir(tmp_path) if f.startswith("scene_") and f.endswith(".json"))
    assert len(frames) == summary["frames"] >= 2
    last = json.loads((tmp_path / frames[-1]).read_text())
    sim = Simulation.from_scene(Scene.from_dict(api_scene))
    for _ in range(summary["steps"]):
        sim.step(1)
        t, _ = sim.time()
        if abs(t - last["time"]) < 1e-12:
            break
    assert abs(t - last["time"]) < 1e-12
    x, v, _ = sim.state()
    sim.close()
    assert np.array_equal(np.asarray(last["positions"], np.float32), x)
    assert np.array_equal(np.asarray(last["velocities"], np.float32), v)


def test_driver_geometry_scene_relative_mesh_path(tmp_path):
    """An OBJ geometry given by a path relative to the scene file."""
    import shutil

    from conftest import GOLDEN, load_golden

    g = load_golden("geometry_dfsph_cup")
    sc = json.loads(json.dumps(g["scene"]))
    sc["Configuration"]["endTime"] = 0.004
    sc["Configuration"]["fps"] = 1000.0
    api_scene = json.loads(json.dumps(sc))
    sc["Boundary"][0]["geometry"][0]["path"] = "cup.obj"
    shutil.copy(os.path.join(GOLDEN, "cup.obj"), tmp_path / "cup.obj")
    (tmp_path / "scene.json").write_text(json.dumps(sc))
    last_frame_matches_api(tmp_path, sc, api_scene)


def test_driver_pcisph_boundary_scene(tmp_path):
    sc = S.pcisph_boundary_scenes()["pcib_wcsph_sphere"]
    sc["Configuration"]["endTime"] = 0.004
    sc["Configuration"]["fps"] = 1000.0
    (tmp_path / "scene.json").write_text(json.dumps(sc))
    last_frame_matches_api(tmp_path, sc, sc)
