"""CUDA path vs the SPH2O reference itself on the named workloads, at their
own sizes:

  C3  double dam break, 1,000,000 fluid + 409,599 boundary particles
      (r = 0.005 m, 4 x 2 x 2 m tank, sphere obstacle), DFSPH and PCISPH --
      the configuration the headline throughput is measured on;
  C1  WCSPH dam break, 8,000 fluid particles, all 2,000 steps at dt = 1e-4;
  C2  DFSPH dam break with Akinci surface tension, 125,000 fluid particles,
      25 steps.

The reference runs here are the unmodified SPH2O sources built by
oracle/Makefile (oracle/_ref/sph2o_ref_f32: FP32 with strict IEEE
arithmetic; sph2o_ref_f64: the same sources with Real = double), driven by
oracle/ref_harness.cpp on the same scene JSON.

Bars (the ones of test_gpu_parity, which holds them on the small goldens):
  * neighbour sets: bit-exact, in the reference's candidate order (the full
    CSR of all 1,000,000 particles: ~45 M fluid + boundary entries);
  * boundary volumes and initial densities: bit-exact;
  * alpha and non-pressure accelerations: norm-wise relative <= 1e-5;
  * state after one step: positions and densities <= 1e-5 of the FP32
    reference; velocities <= 1e-5 (PCISPH), or for DFSPH no further from
    the FP64 reference than 1.5x the FP32 reference's own distance and
    <= 2e-4 of the FP32 reference (the density solver divides by
    rho* - rho0, a difference known only to an FP32 ulp);
  * traces: iteration counts equal to the FP32 reference's at every step,
    time and dt within 1e-5 relative; the 1M state after 5 steps no further
    from the FP64 reference than 1.5x the FP32 reference's own distance;
    aggregates (centroid, kinetic energy,
    mean density error) against the FP64 reference within 1e-6 m,
    2e-3 relative and 1e-6 -- or twice the FP32 reference's own distance
    from FP64 where that is larger.
"""
import json

import numpy as np
import pytest

from conftest import rel_err
from ref_runs import REF32, REF64, Reference, check_aggregates, check_state_vs_f64, check_trace, have_reference
from sph2o_b200 import api
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation

pytestmark = pytest.mark.gpu
need_ref = pytest.mark.skipif(not have_reference(), reason="reference build missing (make -C oracle)")


# ---- C3: 1,000,000 particles, DFSPH --------------------------------------------------------------------------

C3_TRACE = 5


@pytest.fixture(scope="module")
def c3_dfsph(tmp_path_factory):
    if not have_reference():
        pytest.skip("reference build missing (make -C oracle)")
    scene = S.double_dam_break_1m()
    ref = Reference(scene, tmp_path_factory.mktemp("c3_dfsph"))
    out = {"neighbors": ref.run(REF32, "neighbors"), "phases": ref.run(REF32, "phases"),
           "step1": ref.run(REF32, "step", 1), "trace": ref.run(REF32, "step", C3_TRACE)}
    out["step1_f64"] = ref.f64_from_f32_inputs(out["step1"], "step", 1)
    out["trace_f64"] = ref.f64_from_f32_inputs(out["step1"], "step", C3_TRACE)
    print("reference seconds (1M DFSPH):", json.dumps(ref.seconds))
    sim = Simulation.from_scene(Scene.from_dict(scene))
    yield scene, out, sim
    sim.close()


def test_c3_dfsph_inputs_identical(c3_dfsph):
    """The scene loader builds the reference's particles bit for bit (lattice,
    seeded jitter, box and sphere sampling)."""
    scene, ref, _ = c3_dfsph
    sc = Scene.from_dict(scene)
    x, _ = sc.fluid()
    b = sc.boundary()
    sc.close()
    assert x.shape == (1_000_000, 3) and b.shape == (409_599, 3)
    assert np.array_equal(x, ref["step1"]["init_pos"])
    assert np.array_equal(b, ref["step1"]["bpos"])


def test_c3_dfsph_neighbor_sets_bit_exact(c3_dfsph):
    _, ref, sim = c3_dfsph
    n = ref["neighbors"]
    fo, fi, bo, bi = sim.neighbors()
    assert fi.size > 25_000_000  # ~29 fluid neighbours per particle in the initial lattice
    assert np.array_equal(fo, n["nbr_f_offsets"]) and np.array_equal(fi, n["nbr_f"])
    assert np.array_equal(bo, n["nbr_b_offsets"]) and np.array_equal(bi, n["nbr_b"])


def test_c3_dfsph_init_phases(c3_dfsph):
    _, ref, sim = c3_dfsph
    ph = ref["phases"]
    assert np.array_equal(sim.boundary_volume(), ph["bvol"])
    assert np.array_equal(sim.phase(api.PHASE_DENSITY), ph["density"])
    assert np.array_equal(sim.phase(api.PHASE_DENSITY), ref["step1"]["init_density"])
    assert rel_err(sim.phase(api.PHASE_ALPHA), ph["alpha"]) <= 1e-5
    assert rel_err(sim.phase(api.PHASE_NONPRESSURE_ACC), ph["a_nonpressure"]) <= 1e-5


def test_c3_dfsph_one_step(c3_dfsph):
    scene, ref, _ = c3_dfsph
    r32, r64 = ref["step1"], ref["step1_f64"]
    sim = Simulation.from_scene(Scene.from_dict(scene))
    st = sim.step(1)
    x, v, rho = sim.state()
    sim.close()
    check_trace(st, r32["step_stats"][0], 0)
    assert rel_err(x, r32["pos"]) <= 1e-5
    assert rel_err(rho, r32["density"]) <= 1e-5
    assert rel_err(v, r64["vel"]) <= max(1e-5, 1.5 * rel_err(r32["vel"], r64["vel"]))
    assert rel_err(v, r32["vel"]) <= 2e-4


def test_c3_dfsph_trace(c3_dfsph):
    scene, ref, _ = c3_dfsph
    tr = ref["trace"]["step_stats"]
    sim = Simulation.from_scene(Scene.from_dict(scene))
    for s in range(C3_TRACE):
        check_trace(sim.step(1), tr[s], s)
    x, v, rho = sim.state()
    sim.close()
    check_state_vs_f64(x, v, ref["trace"], ref["trace_f64"])


# ---- C3: 1,000,000 particles, PCISPH -------------------------------------------------------------------------

@pytest.fixture(scope="module")
def c3_pcisph(tmp_path_factory):
    if not have_reference():
        pytest.skip("reference build missing (make -C oracle)")
    scene = S.double_dam_break_1m(method=S.PCISPH)
    ref = Reference(scene, tmp_path_factory.mktemp("c3_pcisph"))
    out = {"phases": ref.run(REF32, "phases"), "step1": ref.run(REF32, "step", 1),
           "trace": ref.run(REF32, "step", C3_TRACE)}
    out["trace_f64"] = ref.f64_from_f32_inputs(out["step1"], "step", C3_TRACE)
    print("reference seconds (1M PCISPH):", json.dumps(ref.seconds))
    yield scene, out


def test_c3_pcisph_init_phases(c3_pcisph):
    scene, ref = c3_pcisph
    sim = Simulation.from_scene(Scene.from_dict(scene))
    ph = ref["phases"]
    assert np.array_equal(sim.boundary_volume(), ph["bvol"])
    assert np.array_equal(sim.phase(api.PHASE_DENSITY), ph["density"])
    assert rel_err(sim.phase(api.PHASE_NONPRESSURE_ACC), ph["a_nonpressure"]) <= 1e-5
    sim.close()


def test_c3_pcisph_one_step_and_trace(c3_pcisph):
    scene, ref = c3_pcisph
    r32, tr = ref["step1"], ref["trace"]
    sim = Simulation.from_scene(Scene.from_dict(scene))
    st = sim.step(1)
    check_trace(st, r32["step_stats"][0], 0)
    x, v, rho = sim.state()
    assert rel_err(x, r32["pos"]) <= 1e-5
    assert rel_err(v, r32["vel"]) <= 1e-5
    assert rel_err(rho, r32["density"]) <= 1e-5
    for s in range(1, C3_TRACE):
        check_trace(sim.step(1), tr["step_stats"][s], s)
    x, v, rho = sim.state()
    sim.close()
    check_state_vs_f64(x, v, tr, ref["trace_f64"])


# ---- C1: WCSPH 8k, all 2,000 steps ---------------------------------------------------------------------------

C1_STEPS = 2000
C1_CHECK_EVERY = 500


@need_ref
def test_c1_wcsph_8k_2000_steps(tmp_path):
    scene = S.dam_break_wcsph_8k()
    ref = Reference(scene, tmp_path)
    r32 = ref.run(REF32, "step", C1_STEPS)
    r64 = ref.f64_from_f32_inputs(r32, "step", C1_STEPS)
    print("reference seconds (C1):", json.dumps(ref.seconds))
    rho0 = scene["Fluid"]["FluidModel"][0]["density0"]
    mass = rho0 * (2 * scene["Configuration"]["particleRadius"]) ** 3
    sim = Simulation.from_scene(Scene.from_dict(scene))
    done = 0
    while done < C1_STEPS:
        st = sim.step(C1_CHECK_EVERY)
        done += C1_CHECK_EVERY
        row32, row64 = r32["step_stats"][done - 1], r64["step_stats"][done - 1]
        assert abs(st["time"] - row32[0]) <= 1e-5 * row32[0]
        x, v, rho = sim.state()
        check_aggregates(x, v, rho, rho0, mass, row64, row32)
    sim.close()


# ---- C2: DFSPH + surface tension 125k, 25 steps --------------------------------------------------------------

C2_STEPS = 25


@need_ref
def test_c2_dfsph_surface_tension_125k_25_steps(tmp_path):
    scene = S.dam_break_dfsph_125k()
    ref = Reference(scene, tmp_path)
    r32 = ref.run(REF32, "step", C2_STEPS)
    r64 = ref.f64_from_f32_inputs(r32, "step", C2_STEPS)
    print("reference seconds (C2):", json.dumps(ref.seconds))
    rho0 = scene["Fluid"]["FluidModel"][0]["density0"]
    mass = rho0 * (2 * scene["Configuration"]["particleRadius"]) ** 3
    sim = Simulation.from_scene(Scene.from_dict(scene))
    for s in range(C2_STEPS):
        check_trace(sim.step(1), r32["step_stats"][s], s)
    x, v, rho = sim.state()
    sim.close()
    check_aggregates(x, v, rho, rho0, mass, r64["step_stats"][-1], r32["step_stats"][-1])
