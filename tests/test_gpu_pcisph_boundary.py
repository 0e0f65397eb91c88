"""PCISPH boundary method (boundaryMethod 1) on the GPU, beyond the generic
golden-scene parity of test_gpu_parity.py: boundary densities and WCSPH
boundary pressures bit for bit against the reference, the collision
correction's invariants, and the options that are closed for this method."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from sph2o_b200 import api
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation, SphError

pytestmark = pytest.mark.gpu
PCIB = [n for n in golden_names() if n.startswith("pcib_")]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name", PCIB)
def test_boundary_density_bit_exact(name):
    """SPHSolver::computeBoundaryDensities at the initial positions (the
    reference's computeDensities covers the boundary particles too)."""
    g = load_golden(name)
    sim = Simulation.from_scene(Scene.from_dict(g["scene"]))
    assert np.array_equal(bits(sim.phase(api.PHASE_DENSITY)), bits(g["density"]))
    rho_b, _ = sim.boundary_state()
    assert np.array_equal(bits(rho_b), bits(g["bdensity"]))
    if "bpressure" in g:  # WCSPH: computeBoundaryPressures
        sim.phase(api.PHASE_PRESSURE)
        _, p_b = sim.boundary_state()
        assert np.array_equal(bits(p_b), bits(g["bpressure"]))
    sim.close()


def test_fluid_stays_inside_the_tank():
    """A WCSPH block dropped in the 1 m tank: the collision correction keeps
    every particle inside the boundary box for 400 steps."""
    sc = S.pcisph_boundary_scenes()["pcib_wcsph_sphere"]
    sim = Simulation.from_scene(Scene.from_dict(sc))
    sim.step(400)
    x, v, _ = sim.state()
    sim.close()
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(v))
    assert x.min() > -0.05 and x.max() < 1.05


def test_deterministic_and_graph_replay_equal_eager():
    sc = S.pcisph_boundary_scenes()["pcib_dfsph_sphere"]
    runs = []
    for graphs in (1, 1, 0):
        sim = Simulation.from_scene(Scene.from_dict(sc))
        sim.set_option(api.OPT_CUDA_GRAPHS, graphs)
        for _ in range(6):
            sim.step(2)
        runs.append(sim.state())
        sim.close()
    for r in runs[1:]:
        for a, b in zip(runs[0], r):
            assert np.array_equal(a, b)


def test_closed_options():
    sim = Simulation.from_scene(Scene.from_dict(S.pcisph_boundary_scenes()["pcib_pcisph"]))
    with pytest.raises(SphError):
        sim.autotune(trial_steps=1)
    other = 1 - sim.get_option(api.OPT_CELL_ORDER)
    with pytest.raises(SphError):
        sim.set_option(api.OPT_CELL_ORDER, other)
    sim.close()


def test_adhesion_rejected():
    d = S.pcisph_boundary_scenes()["pcib_wcsph_sphere"]
    d["Fluid"]["adhesionMethod"] = S.ADHESION_AKINCI
    d["Fluid"]["FluidModel"][0]["adhesion"] = 0.5
    with pytest.raises(SphError) as e:
        Simulation.from_scene(Scene.from_dict(d))
    assert e.value.code == -1


def test_unlisted_cells_skip_the_collision_pass():
    """Two lone particles slide along the far x wall into cells no particle
    has visited (pcib_wcsph_wallslide). SPH2O's hash table holds no candidate
    lists for such a cell until the next search, so the collision pass skips
    them for that step. The GPU run ends where the FP32 reference ends
    (measured: identical); a run that treats every cell as listed ends
    7.2e-7 m away."""
    g = load_golden("pcib_wcsph_wallslide")
    sim = Simulation.from_scene(Scene.from_dict(g["scene"]))
    for _ in range(g["trace_f32"].shape[0]):
        sim.step(1)
    x, _, _ = sim.state()
    sim.close()
    assert np.max(np.abs(x.astype(np.float64) - g["final_pos_f32"])) <= 1e-7
