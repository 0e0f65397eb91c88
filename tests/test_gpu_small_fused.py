"""Small WCSPH scenes stepped as one cooperative launch per sph_step call
(SPH_OPT_FUSED_SMALL_STEPS, k_wcsph_small_steps) against one launch per
phase: the fused kernel runs the same per-particle bodies (counting sort,
warp list build, 4-lane density and force passes), so states, neighbour
lists, times and adjoint gradients must be equal bit for bit. The golden
WCSPH parity tests (test_gpu_parity) run through the fused path by default
and hold it to the reference."""
import numpy as np
import pytest

from conftest import load_golden
from sph2o_b200 import api
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation

pytestmark = pytest.mark.gpu

CHUNKS = (1, 1, 5, 13)  # single steps, an odd and a longer multi-step launch


def scenes():
    return {
        "wcsph_artificial": load_golden("wcsph_artificial")["scene"],
        "geometry_wcsph_quirks": load_golden("geometry_wcsph_quirks")["scene"],
        "wcsph_standard_sphere": S.small(method=S.WCSPH, n=(12, 9, 9), viscosity_method=S.VISC_STANDARD,
                                         viscosity=0.02, boundary_viscosity=0.01, sphere=True, seed=21),
        "dam_break_wcsph_8k": S.dam_break_wcsph_8k(),
        "adjoint_wcsph_32k": S.adjoint_wcsph_32k(),
    }


def run(d, fused):
    sim = Simulation.from_scene(Scene.from_dict(d), options={api.OPT_FUSED_SMALL_STEPS: fused})
    out = []
    for n in CHUNKS:
        st = sim.step(n)
        out.append((st, sim.state()))
    lists = sim.neighbors()
    sim.close()
    return out, lists


@pytest.mark.parametrize("name", sorted(scenes()))
def test_fused_steps_equal_separate_kernels(name):
    d = scenes()[name]
    fused, lf = run(d, 1)
    plain, lp = run(d, 0)
    for k, ((sf, (xf, vf, rf)), (sp, (xp, vp, rp))) in enumerate(zip(fused, plain)):
        assert sf["time"] == sp["time"] and sf["steps"] == sp["steps"], k
        assert np.array_equal(xf, xp) and np.array_equal(vf, vp) and np.array_equal(rf, rp), k
    for a, b in zip(lf, lp):
        assert np.array_equal(a, b)


def test_fused_path_is_one_launch_per_call():
    d = scenes()["dam_break_wcsph_8k"]
    sim = Simulation.from_scene(Scene.from_dict(d))
    assert sim.get_option(api.OPT_FUSED_SMALL_STEPS) == 1
    st = sim.step(20)
    assert st["kernel_launches"] == 1
    sim.set_option(api.OPT_FUSED_SMALL_STEPS, 0)
    st = sim.step(20)
    assert st["kernel_launches"] >= 20 * 8
    sim.close()


def test_fused_adjoint_gradients_identical():
    """The differentiable run's forward and its recomputed segments go
    through the same step: gradients are bit-identical either way."""
    d = S.small(method=S.WCSPH, n=(10, 9, 8), radius=0.02, time_step=2e-4, seed=5, viscosity=0.01)
    sc = Scene.from_dict(d)
    x0, _ = sc.fluid()
    v0, t = S.adjoint_problem(x0)
    out = []
    for fused in (1, 0):
        sim = Simulation(sc.desc(), x0, sc.boundary(), vel=v0, options={api.OPT_FUSED_SMALL_STEPS: fused})
        loss = sim.wcsph_forward(40, t, ckpt_every=8)
        out.append((loss, sim.wcsph_backward(want_x0=True)))
        sim.close()
    (l1, g1), (l0, g0) = out
    assert l1 == l0
    for key in ("v0", "x0"):
        assert np.array_equal(g1[key], g0[key]), key
    assert g1["viscosity"] == g0["viscosity"] and g1["stiffness"] == g0["stiffness"]
