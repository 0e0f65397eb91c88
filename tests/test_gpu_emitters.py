"""Particle emitters (Emitter.cpp, FluidObject::addEmitter) on the GPU
against the SPH2O reference run on the same scenes (tests/golden/emitter_*,
generated by tests/golden/make_golden.py from its FP32 and FP64 builds).

Bars: the active particle count after every step equals the reference's;
the particles a group adds land bit-exactly where the reference puts them
(glm's FP32 quaternion rotation and the emission offset, restated
operation by operation); iteration counts, time and dt follow the FP32
reference step by step; final aggregates over the active particles meet the
trajectory bars of test_gpu_parity against the FP64 build."""
import ctypes as C

import numpy as np
import pytest

from conftest import emitter_golden_names, load_golden, rel_err
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation, SphError, lib

pytestmark = pytest.mark.gpu
NAMES = emitter_golden_names()


def make_sim(g):
    return Simulation.from_scene(Scene.from_dict(g["scene"]))


@pytest.mark.parametrize("name", NAMES)
def test_capacity_and_first_emission(name):
    g = load_golden(name)
    sim = make_sim(g)
    n = g["init_pos"].shape[0]
    assert sim.nf == n
    a0 = sim.num_active()
    x0, v0, _ = sim.state()
    # inactive particles read as zero until emitted
    assert np.all(x0[a0:] == 0.0) and np.all(v0[a0:] == 0.0)
    assert np.array_equal(x0[:a0], g["init_pos"][:a0])
    sim.step(1)
    a1 = sim.num_active()
    assert a1 == int(g["active_f32"][0]) and a1 > a0
    x, v, rho = sim.state()
    sim.close()
    # the emitted group: positions bit-exact (no solver moves them within the
    # step they appear in: WCSPH emits after integrating, DFSPH after updating
    # positions); velocities bit-exact for WCSPH, through the divergence
    # solver for DFSPH
    assert np.array_equal(x[a0:a1], g["step1_pos"][a0:a1])
    if g["scene"]["Configuration"]["simulationMethod"] == S.WCSPH:
        assert np.array_equal(v[a0:a1], g["step1_vel"][a0:a1])
        assert np.array_equal(x[:a0], g["step1_pos"][:a0])
    else:
        assert rel_err(v[:a1], g["step1_vel"][:a1]) <= 2e-4
        assert rel_err(x[:a1], g["step1_pos"][:a1]) <= 1e-5
    assert np.all(x[a1:] == 0.0)


@pytest.mark.parametrize("name", NAMES)
def test_trajectory_with_emissions(name):
    """WCSPH (fixed dt): active counts, iterations and time equal the FP32
    reference at every step. DFSPH: its dt follows the CFL speed, which the
    emitted jet makes chaotic -- the reference's own FP32 and FP64 builds
    drift apart after a few dozen steps -- so steps are compared one by one
    while those two agree within 1e-5, emission events by the simulated time
    they happen at (within one step), and the final aggregates against the
    FP64 build within twice the FP32 build's own distance from it."""
    g = load_golden(name)
    ref32, ref64 = g["trace_f32"], g["trace_f64"]
    act32 = g["active_f32"].astype(int)
    sim = make_sim(g)
    rho0 = g["scene"]["Fluid"]["FluidModel"][0]["density0"]
    mass = rho0 * (2 * g["scene"]["Configuration"]["particleRadius"]) ** 3
    wcsph = g["scene"]["Configuration"]["simulationMethod"] == S.WCSPH
    drift = np.abs(ref32[:, 1] - ref64[:, 1]) > 1e-5 * ref64[:, 1]
    window = ref32.shape[0] if wcsph or not drift.any() else int(np.argmax(drift))
    active, times = [], []
    for s in range(ref32.shape[0]):
        st = sim.step(1)
        active.append(sim.num_active())
        times.append(st["time"])
        if wcsph:
            assert active[-1] == act32[s], f"step {s}"
            assert st["time"] == ref32[s, 0], f"step {s}"  # float time, fixed dt: bit-exact
        if s < window:
            assert active[-1] == act32[s], f"step {s}"
            assert st["iterations"] == int(ref32[s, 2]), f"step {s}"
            assert st["iterations_v"] == int(ref32[s, 3]), f"step {s}"
            assert abs(st["time"] - ref32[s, 0]) <= 1e-5 * ref32[s, 0], f"step {s}"
            assert abs(st["dt"] - ref32[s, 1]) <= 1e-5 * ref32[s, 1], f"step {s}"
    active = np.array(active)
    times = np.array(times)
    # emission events: same count, at the same simulated time within one step
    ev_ours = np.nonzero(np.diff(np.concatenate([[0], active])))[0]
    ev_ref = np.nonzero(np.diff(np.concatenate([[0], act32])))[0]
    assert len(ev_ours) == len(ev_ref) and active[-1] == act32[-1]
    for a, b in zip(ev_ours, ev_ref):
        assert abs(times[a] - ref32[b, 0]) <= 1.01 * max(ref32[b, 1], times[a] - (times[a - 1] if a else 0.0))
    na = active[-1]
    x, v, rho = sim.state()
    sim.close()
    x64 = x[:na].astype(np.float64)
    v64 = v[:na].astype(np.float64)
    centroid = x64.mean(axis=0)
    ke = 0.5 * mass * float((v64 * v64).sum())
    derr = float(np.mean(np.maximum(rho[:na].astype(np.float64) - rho0, 0.0) / rho0))
    last32, last64 = ref32[-1], ref64[-1]
    spread = np.abs(last32 - last64)
    assert np.max(np.abs(centroid - last64[6:9])) <= max(1e-5, 2 * float(np.max(spread[6:9])))
    assert abs(ke - last64[9]) <= max(2e-3 * abs(last64[9]), 2 * float(spread[9]))
    assert abs(derr - last64[10]) <= max(1e-5, 2 * float(spread[10]))


def test_graph_replay_with_emitters_matches_eager():
    """Emission runs on the device (the active count is device state), so
    graph replay and eager steps agree bit for bit."""
    d = S.emitter_scenes()["emitter_wcsph_square"]
    out = []
    for graphs in (1, 0):
        sim = Simulation.from_scene(Scene.from_dict(d))
        sim.set_option(0, graphs)
        sim.step(60)
        out.append((sim.num_active(),) + sim.state())
        sim.close()
    assert out[0][0] == out[1][0]
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.array_equal(a, b)


def test_emitter_api_errors():
    d = S.emitter_scenes()["emitter_dfsph_circle"]
    sc = Scene.from_dict(d)
    sim = Simulation.from_scene(sc)
    e = sc.emitters()[0]
    assert lib().sph_add_emitter(sim._h, C.byref(e)) == -6          # after init
    with pytest.raises(SphError) as err:                              # WCSPH adjoint only, no emitters
        sim.wcsph_forward(2, np.zeros((sim.nf, 3), np.float32))
    assert err.value.code == -1
    sim.close()
    wc = Scene.from_dict(S.emitter_scenes()["emitter_wcsph_square"])
    sim = Simulation.from_scene(wc)
    with pytest.raises(SphError) as err:
        sim.wcsph_forward(2, np.zeros((sim.nf, 3), np.float32))
    assert err.value.code == -1
    sim.close()
    bad = wc.emitters()[0]
    bad.velocity = 0.0
    with pytest.raises(SphError):
        Simulation(wc.desc(), *wc.fluid()[:1], wc.boundary(), emitters=[bad])
