"""Host scene loader (C ABI, no GPU): the particles it generates are
bit-identical to the reference's FluidObject::build + jitter and
AkinciBoundaryObject::sampleCube / sampleSphere, and malformed scenes fail
with status codes instead of exceptions or asserts."""
import copy
import json

import numpy as np
import pytest

from conftest import golden_names, load_golden
from sph2o_b200 import scenes as S
from sph2o_b200.api import SPH_OK, Scene, SphError, lib


@pytest.mark.parametrize("name", [n for n in golden_names() if not n.startswith("geometry_")])
def test_particles_bit_exact(name):
    """(The OBJ geometry scenes are sampled on the GPU: test_gpu_geometry.py.)"""
    g = load_golden(name)
    sc = Scene.from_dict(g["scene"])
    x, v = sc.fluid()
    assert np.array_equal(x, g["init_pos"])
    assert np.array_equal(sc.boundary(), g["bpos"])
    assert not v.any()


@pytest.mark.parametrize("name", [n for n in golden_names() if n.startswith("pcib_")])
def test_pcisph_boundary_normals_bit_exact(name):
    """PCISPHBoundaryObject::sampleCube / sampleSphere: positions and normals
    bit for bit, and the object's velocity factors."""
    g = load_golden(name)
    sc = Scene.from_dict(g["scene"])
    nrm, nf, tf = sc.boundary_normals()
    assert np.array_equal(nrm.view(np.uint32), g["bnormal"].view(np.uint32))
    b = g["scene"]["Boundary"][0]
    assert nf == np.float32(b["normalFct"]) and tf == np.float32(b["tangFct"])


@pytest.mark.parametrize("mutate,code", [
    # SPH2O truncates PCISPH box sides to whole numbers: a 0.6 side would be 0
    (lambda d: d["Boundary"][0]["box"][0].__setitem__("max", [1.0, 0.6, 1.0]), -1),
    (lambda d: d["Boundary"].append(copy.deepcopy(d["Boundary"][0])), -1),
    (lambda d: d["Boundary"][0]["box"][0].pop("inverted"), -8),
    (lambda d: d["Boundary"][0].pop("tangFct"), -8),
])
def test_bad_pcisph_boundary_scenes_rejected(mutate, code):
    d = S.pcisph_boundary_scenes()["pcib_pcisph"]
    mutate(d)
    with pytest.raises(SphError) as e:
        Scene.from_dict(d)
    assert e.value.code == code


def test_pcisph_boundary_ignores_geometry_entries():
    """importScene's PCISPH branch adds boxes and spheres only
    (SPHSimulation.cpp:428-453): geometry entries are not even opened."""
    d = S.pcisph_boundary_scenes()["pcib_pcisph"]
    n = Scene.from_dict(d).boundary().shape[0]
    d["Boundary"][0]["geometry"] = [{"path": "missing.obj", "spacing": 1.0}]
    assert Scene.from_dict(d).boundary().shape[0] == n


def test_desc_fields():
    sc = Scene.from_dict(S.dam_break_dfsph_125k())
    d = sc.desc()
    assert d.simulation_method == S.DFSPH and d.boundary_method == 2
    assert d.surface_tension_method == 3 and abs(d.surface_tension - 0.05) < 1e-7
    assert d.min_iterations == 2 and d.max_iterations == 100
    assert abs(d.particle_radius - 0.01) < 1e-9


def test_missing_sphere_geometry_keys_tolerated():
    sc = S.small()
    for b in sc["Boundary"]:
        del b["sphere"]
        del b["geometry"]
    s2 = Scene.from_dict(sc)
    assert s2.boundary().shape[0] > 0


@pytest.mark.parametrize("mutate,code", [
    (lambda d: d["Configuration"].pop("timeStep"), -8),
    (lambda d: d["Fluid"]["FluidModel"].append(copy.deepcopy(d["Fluid"]["FluidModel"][0])), -1),
    (lambda d: d["Configuration"].__setitem__("boundaryMethod", 3), -1),
    (lambda d: d["Fluid"]["FluidModel"][0].__setitem__("emitters", [{"type": 0}]), -8),
    (lambda d: d["Boundary"][0].__setitem__("geometry", [{"path": "missing.obj", "spacing": 1.0}]), -8),
    (lambda d: d["Boundary"][0].__setitem__("geometry", [{"spacing": 1.0}]), -8),
    (lambda d: d["Configuration"].__setitem__("simulationMethod", 7), -8),
])
def test_bad_scenes_rejected(mutate, code):
    d = S.small()
    mutate(d)
    with pytest.raises(SphError) as e:
        Scene.from_dict(d)
    assert e.value.code == code


def test_emitters_parsed():
    """The "emitters" keys of SceneLoader.cpp:128-143; rotation is (w, x, y, z)."""
    d = S.small()
    d["Fluid"]["FluidModel"][0]["emitters"] = [
        {"position": [0.5, 0.25, 0.75], "rotation": [0.5, 0.5, -0.5, 0.5], "velocity": 2.0, "numParticles": 300,
         "startTime": 0.01, "type": 1, "width": 0.1, "height": 0.0, "spacing": 1.5},
        {"position": [0.1, 0.2, 0.3], "rotation": [1.0, 0.0, 0.0, 0.0], "velocity": 1.0, "numParticles": 64,
         "startTime": 0.0, "type": 0, "width": 0.2, "height": 0.2, "spacing": 1.0}]
    sc = Scene.from_dict(d)
    em = sc.emitters()
    assert len(em) == 2
    e = em[0]
    assert e.type == 1 and e.num_particles == 300 and list(e.position) == [0.5, 0.25, 0.75]
    assert list(e.rotation) == [0.5, 0.5, -0.5, 0.5] and e.velocity == 2.0 and e.spacing == 1.5
    assert e.start_time == float(np.float32(0.01)) and e.width == float(np.float32(0.1))
    assert em[1].type == 0 and em[1].num_particles == 64


def test_malformed_json():
    import ctypes as C
    h = C.c_void_p()
    rc = lib().sph_scene_parse(b'{"Configuration": [1, 2', C.byref(h))
    assert rc == -8
    assert b"parse error" in lib().sph_scene_error()


def test_workload_counts():
    """Fluid counts of the benchmark scenes (boundary counts from the reference sampler)."""
    for make, nf in [(S.dam_break_wcsph_8k, 8000), (S.dam_break_dfsph_125k, 125000), (S.adjoint_wcsph_32k, 32768)]:
        sc = Scene.from_dict(make())
        assert sc.fluid()[0].shape[0] == nf
