"""DFSPH with minimum iteration counts of zero.

SPH2O's solver loops run while (error > tolerance or iterations < minimum)
and iterations < maximum, with the error set to 0 before the loop
(DFSPHSolver.cpp:427-429, 744-746): a minimum of 0 runs no iteration at all,
and the warm-start values, zeroed after the warm start (:1052-1059), are
left at zero times the time step. The persistent GPU solvers then zero and
scale those values with no grid barrier between the two passes, so both
must map particles to threads alike. Checked against the reference's FP32
and FP64 builds over 30 steps (iteration counts, time and dt each step,
final aggregates and state), and for bit-identical repeat runs."""
import numpy as np
import pytest

from ref_runs import REF32, Reference, check_aggregates, check_state_vs_f64, check_trace, have_reference
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation

pytestmark = pytest.mark.gpu
need_ref = pytest.mark.skipif(not have_reference(), reason="reference build missing (make -C oracle)")

STEPS = 30


@need_ref
@pytest.mark.parametrize("mins", [(2, 0), (0, 0)], ids=["divergence-0", "both-0"])
def test_zero_minimum_iterations_against_reference(mins, tmp_path):
    scene = S.small(method=S.DFSPH, n=(16, 16, 16), seed=21, min_iterations=mins[0], min_iterations_v=mins[1])
    ref = Reference(scene, tmp_path)
    r32 = ref.run(REF32, "step", STEPS)
    r64 = ref.f64_from_f32_inputs(r32, "step", STEPS)
    assert all(int(row[3]) == 0 for row in r32["step_stats"]), "the reference runs no divergence iteration"
    rho0 = scene["Fluid"]["FluidModel"][0]["density0"]
    mass = rho0 * (2 * scene["Configuration"]["particleRadius"]) ** 3
    runs = []
    for _ in range(2):
        sim = Simulation.from_scene(Scene.from_dict(scene))
        for s in range(STEPS):
            check_trace(sim.step(1), r32["step_stats"][s], s)
        runs.append(sim.state())
        sim.close()
    x, v, rho = runs[0]
    check_aggregates(x, v, rho, rho0, mass, r64["step_stats"][-1], r32["step_stats"][-1])
    check_state_vs_f64(x, v, r32, r64)
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(a, b), "repeat runs differ"
