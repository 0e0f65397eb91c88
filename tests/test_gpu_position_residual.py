"""Position residuals (SPH_OPT_POSITION_RESIDUAL): every position carries
the rounding residual of its integration, so long runs of small steps keep
about twice float precision. With the option off the trajectory is the
reference's FP32 one (test_gpu_parity.py); on, the WCSPH trajectories end
much closer to the reference's FP64 build than its own FP32 build does
(measured: 13x on the 20-step scenes, 38x on the 120-step one)."""
import numpy as np
import pytest

from conftest import load_golden
from sph2o_b200 import api
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation, SphError

pytestmark = pytest.mark.gpu


def final_positions(g, residual):
    sim = Simulation.from_scene(Scene.from_dict(g["scene"]), options={api.OPT_POSITION_RESIDUAL: residual})
    for _ in range(g["trace_f32"].shape[0]):
        sim.step(1)
    x, _, _ = sim.state()
    sim.close()
    return x.astype(np.float64)


@pytest.mark.parametrize("name", ["wcsph_artificial", "wcsph_xsph_st_adhesion", "pcib_wcsph_sphere",
                                  "pcib_wcsph_farwall"])
def test_residual_brings_wcsph_closer_to_fp64(name):
    g = load_golden(name)
    ref32 = float(np.abs(g["final_pos_f32"] - g["final_pos_f64"]).max())
    plain = float(np.abs(final_positions(g, 0) - g["final_pos_f64"]).max())
    resid = float(np.abs(final_positions(g, 1) - g["final_pos_f64"]).max())
    assert plain <= 1.5 * ref32          # the FP32 trajectory: as far as the reference's FP32 build
    assert resid <= 0.5 * ref32          # with residuals: at least twice as close to FP64


@pytest.mark.parametrize("name", ["pcisph_artificial", "dfsph_st_sphere", "cube_dfsph_floor"])
def test_residual_stays_within_the_fp32_spread(name):
    """PCISPH and DFSPH: the residual changes the rounding of the position
    update only; the solvers' own FP32 conditioning dominates there, and the
    result stays within the reference's FP32-to-FP64 spread."""
    g = load_golden(name)
    ref32 = float(np.abs(g["final_pos_f32"] - g["final_pos_f64"]).max())
    resid = float(np.abs(final_positions(g, 1) - g["final_pos_f64"]).max())
    assert resid <= 1.5 * ref32


def test_option_is_set_before_init_and_for_single_scenes():
    sim = Simulation.from_scene(Scene.from_dict(S.small(method=S.WCSPH)))
    with pytest.raises(SphError):
        sim.set_option(api.OPT_POSITION_RESIDUAL, 1)
    assert sim.get_option(api.OPT_POSITION_RESIDUAL) == 0
    sim.close()
    sim = Simulation.from_scene(Scene.from_dict(S.small(method=S.WCSPH)), options={api.OPT_POSITION_RESIDUAL: 1})
    assert sim.get_option(api.OPT_POSITION_RESIDUAL) == 1
    x, v, _ = sim.state()
    with pytest.raises(SphError):  # the adjoint differentiates FP32 positions
        sim.wcsph_forward(2, x)
    sim.close()


@pytest.mark.parametrize("name", ["emitter_wcsph_square", "emitter_dfsph_circle", "cube_wcsph_outside",
                                  "pcib_dfsph_sphere"])
def test_residual_with_emitters_cubes_and_pcisph_boundaries(name):
    """Emitted particles start without a residual, cube clamps zero the
    clamped coordinates', PCISPH-boundary pushes leave it: the runs stay
    finite, emit the same particles and end within the reference's own
    FP32-to-FP64 spread of the plain run."""
    g = load_golden(name)
    runs = []
    for residual in (0, 1):
        sim = Simulation.from_scene(Scene.from_dict(g["scene"]), options={api.OPT_POSITION_RESIDUAL: residual})
        sim.step(g["trace_f32"].shape[0])
        runs.append((sim.state(), sim.num_active()))
        sim.close()
    (x0, v0, _), n0 = runs[0]
    (x1, v1, _), n1 = runs[1]
    assert n0 == n1 and np.all(np.isfinite(x1[:n1])) and np.all(np.isfinite(v1[:n1]))
    spread = float(np.abs(g["final_pos_f32"] - g["final_pos_f64"]).max())
    assert float(np.abs(x1[:n1] - x0[:n0]).max()) <= 2.0 * spread + 1e-6
