"""Batches of independent scenes (sph_batch_*): each scene of a batch must
evolve exactly as it does alone. WCSPH: bit-identical states (batch and
scenes here are all below 2^16 particles, so both take the same lanes per
particle in the force pass). DFSPH: the same iteration counts per scene and
step, states equal to 1e-6 (norm-wise; the per-scene FP64 residual sums are
reduced in a different order)."""
import numpy as np
import pytest

from conftest import rel_err
from sph2o_b200 import scenes as S
from sph2o_b200.api import Batch, Scene, Simulation

pytestmark = pytest.mark.gpu


def batch_scenes(method):
    dims = [(6, 5, 7), (9, 8, 6), (5, 5, 5), (10, 7, 8)]
    visc = [0.005, 0.02, 0.05, 0.0]
    out = []
    for k, (n, v) in enumerate(zip(dims, visc)):
        out.append(S.small(method=method, n=n, radius=0.02 + 0.0 * k, viscosity=v, seed=40 + k,
                           time_step=1e-4 * (1 + 0.25 * k) if method == S.DFSPH else 1e-4))
    return out


def test_wcsph_batch_bit_identical_to_single_runs():
    scs = [Scene.from_dict(d) for d in batch_scenes(S.WCSPH)]
    b = Batch(scs)
    b.step(6)
    for k, sc in enumerate(scs):
        sim = Simulation.from_scene(sc)
        sim.step(6)
        x, v, r = sim.state()
        bx, bv, br = b.scene_state(k)
        assert np.array_equal(x, bx) and np.array_equal(v, bv) and np.array_equal(r, br), f"scene {k}"
        st = b.scene_stats(k)
        t = np.float32(0.0)
        for _ in range(6):  # simulated time is a float sum, as the reference keeps it
            t = np.float32(t + np.float32(1e-4))
        assert st["steps"] == 6 and st["time"] == float(t)
        sim.close()
    b.close()


def test_dfsph_batch_matches_single_runs():
    scs = [Scene.from_dict(d) for d in batch_scenes(S.DFSPH)]
    b = Batch(scs)
    singles = [Simulation.from_scene(sc) for sc in scs]
    for step in range(5):
        b.step(1)
        for k, sim in enumerate(singles):
            st = sim.step(1)
            bs = b.scene_stats(k)
            assert bs["iterations"] == st["iterations"] and bs["iterations_v"] == st["iterations_v"], (step, k)
            assert abs(bs["dt"] - st["dt"]) <= 1e-7 * st["dt"]
    for k, sim in enumerate(singles):
        x, v, r = sim.state()
        bx, bv, br = b.scene_state(k)
        assert rel_err(bx, x) <= 1e-6 and rel_err(bv, v) <= 1e-6 and rel_err(br, r) <= 1e-6, k
        sim.close()
    b.close()


def test_batch_rejects_mixed_shared_parameters():
    a = Scene.from_dict(S.small(method=S.DFSPH))
    c = Scene.from_dict(S.small(method=S.DFSPH, radius=0.03))
    with pytest.raises(Exception):
        Batch([a, c])


# ---- batches against the reference itself ----------------------------------------------------------------------

BATCH_REF_STEPS = 20
def _c4_subset(method):
    dicts = S.batched_scenes(256, method=method)
    sizes = [p["dims"][0] * p["dims"][1] * p["dims"][2] for p in S.batched_scene_params(256)]
    order = sorted(range(256), key=lambda k: sizes[k])
    picks = [order[0], order[-1]] + [order[k] for k in (51, 102, 153, 204)]
    return [dicts[k] for k in picks], [sizes[k] for k in picks]


@pytest.mark.parametrize("method", [S.WCSPH, S.DFSPH], ids=["wcsph", "dfsph"])
def test_c4_batch_scenes_against_reference(method, tmp_path):
    """Six scenes of the 256-scene batched workload -- the smallest, the
    largest and four quantiles of its log-uniform sizes, each with its own
    viscosity -- stepped as one batch; every scene against the reference run
    alone on it: iteration counts, time and dt at every step equal to the
    FP32 reference's, final aggregates against the FP64 reference within the
    trace bars of test_gpu_parity, and final positions and velocities no
    further from the FP64 reference than 1.5x the FP32 reference's own
    distance."""
    from ref_runs import REF32, Reference, check_aggregates, check_state_vs_f64, check_trace, have_reference

    if not have_reference():
        pytest.skip("reference build missing (make -C oracle)")
    dicts, sizes = _c4_subset(method)
    assert min(sizes) < 3000 and max(sizes) > 35000
    refs = []
    for k, d in enumerate(dicts):
        ref = Reference(d, tmp_path / f"s{k}")
        r32 = ref.run(REF32, "step", BATCH_REF_STEPS)
        refs.append((r32, ref.f64_from_f32_inputs(r32, "step", BATCH_REF_STEPS)))
    scs = [Scene.from_dict(d) for d in dicts]
    b = Batch(scs)
    for s in range(BATCH_REF_STEPS):
        b.step(1)
        for k in range(len(scs)):
            check_trace(b.scene_stats(k), refs[k][0]["step_stats"][s], f"{s} (scene {k})")
    for k, d in enumerate(dicts):
        x, v, r = b.scene_state(k)
        rho0 = d["Fluid"]["FluidModel"][0]["density0"]
        mass = rho0 * (2 * d["Configuration"]["particleRadius"]) ** 3
        r32, r64 = refs[k]
        check_aggregates(x, v, r, rho0, mass, r64["step_stats"][-1], r32["step_stats"][-1])
        check_state_vs_f64(x, v, r32, r64)
    b.close()


def test_wcsph_golden_batch_against_reference_traces():
    """The two WCSPH goldens that share every batch-wide parameter (plain
    Akinci box tank, and OBJ-mesh boundary objects; different time steps) as
    one batch: each scene's time at every step and its final state against
    its golden traces from the reference's FP32 and FP64 builds."""
    from conftest import load_golden
    from ref_runs import check_aggregates

    names = ["wcsph_artificial", "geometry_wcsph_quirks"]
    gs = [load_golden(n) for n in names]
    scs = [Scene.from_dict(g["scene"]) for g in gs]
    b = Batch(scs)
    steps = min(g["trace_f32"].shape[0] for g in gs)
    for s in range(steps):
        b.step(1)
        for k, g in enumerate(gs):
            st = b.scene_stats(k)
            assert abs(st["time"] - g["trace_f32"][s, 0]) <= 1e-5 * g["trace_f32"][s, 0], (names[k], s)
    for k, g in enumerate(gs):
        x, v, r = b.scene_state(k)
        rho0 = g["scene"]["Fluid"]["FluidModel"][0]["density0"]
        mass = rho0 * (2 * g["scene"]["Configuration"]["particleRadius"]) ** 3
        check_aggregates(x, v, r, rho0, mass, g["trace_f64"][steps - 1], g["trace_f32"][steps - 1])
    b.close()
