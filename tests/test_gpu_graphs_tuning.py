"""CUDA-graph replay, launch options and the autotuner.

Graph replay must not change a single bit of the trajectory; the cell order
changes only the storage order of the particles (each particle's neighbours
are visited in the same order either way), the solver occupancy and pass
block size only the launch shape. The autotuner runs trials from a snapshot
and must leave the simulation exactly where it found it."""
import json

import numpy as np
import pytest

from sph2o_b200 import api
from sph2o_b200 import scenes as S
from sph2o_b200.api import Batch, Scene, Simulation, SphError

pytestmark = pytest.mark.gpu

METHODS = [S.WCSPH, S.PCISPH, S.DFSPH]


def small_sim(method, **kw):
    return Simulation.from_scene(Scene.from_dict(S.small(method=method, surface_tension=0.05, **kw)))


def run(method, steps, options=(), chunk=None):
    sim = small_sim(method)
    for opt, val in options:
        sim.set_option(opt, val)
    st = None
    if chunk:
        for _ in range(steps // chunk):
            st = sim.step(chunk)
    else:
        st = sim.step(steps)
    out = sim.state(), sim.time(), st
    sim.close()
    return out


@pytest.mark.parametrize("method", METHODS)
def test_graph_replay_matches_eager_bitwise(method):
    (xg, vg, rg), tg, sg = run(method, 10)
    (xe, ve, re), te, se = run(method, 10, [(api.OPT_CUDA_GRAPHS, 0)])
    assert np.array_equal(xg, xe) and np.array_equal(vg, ve) and np.array_equal(rg, re)
    assert tg == te
    assert sg["total_iterations"] == se["total_iterations"]
    assert sg["total_iterations_v"] == se["total_iterations_v"]
    assert sg["kernel_launches"] == se["kernel_launches"]


@pytest.mark.parametrize("method", METHODS)
def test_graph_replay_odd_chunks(method):
    """Odd step counts mix a single-step graph with graph pairs; the buffer
    assignment alternates, so every graph key is exercised."""
    a, ta, _ = run(method, 9, chunk=3)
    b, tb, _ = run(method, 9, [(api.OPT_CUDA_GRAPHS, 0)])
    for u, w in zip(a, b):
        assert np.array_equal(u, w)
    assert ta == tb


def test_options_round_trip_and_reject_bad_values():
    sim = small_sim(S.DFSPH)
    defaults = {api.OPT_CUDA_GRAPHS: 1, api.OPT_CELL_ORDER: 0, api.OPT_SOLVER_OCCUPANCY: 8, api.OPT_PASS_BLOCK: 256,
                api.OPT_SOLVER_LANES: 2}
    for k, v in defaults.items():
        assert sim.get_option(k) == v
    for opt, bad in [(api.OPT_CELL_ORDER, 2), (api.OPT_SOLVER_OCCUPANCY, 6), (api.OPT_PASS_BLOCK, 64),
                     (api.OPT_SOLVER_LANES, 3), (99, 0)]:
        with pytest.raises(SphError):
            sim.set_option(opt, bad)
    sim.set_option(api.OPT_SOLVER_OCCUPANCY, 4)
    sim.set_option(api.OPT_PASS_BLOCK, 128)
    sim.set_option(api.OPT_SOLVER_LANES, 4)
    assert sim.get_option(api.OPT_SOLVER_OCCUPANCY) == 4 and sim.get_option(api.OPT_PASS_BLOCK) == 128
    assert sim.get_option(api.OPT_SOLVER_LANES) == 4
    sim.step(4)
    sim.close()


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("lanes", [1, 2, 4])
def test_launch_shape_does_not_change_results(method, lanes):
    """Launch shape changes no WCSPH/PCISPH bit; in DFSPH the FP64 residual
    order and, with several lanes per particle, the FP32 summation order of
    the solver passes change, within rounding."""
    (x0, v0, r0), t0, s0 = run(method, 8)
    (x1, v1, r1), t1, s1 = run(method, 8, [(api.OPT_SOLVER_OCCUPANCY, 4), (api.OPT_PASS_BLOCK, 128),
                                           (api.OPT_SOLVER_LANES, lanes)])
    assert t0 == t1
    assert s0["total_iterations"] == s1["total_iterations"]
    if method == S.WCSPH:
        assert np.array_equal(x0, x1) and np.array_equal(v0, v1)
    else:
        # residual sums are fp64 atomics whose order depends on the launch shape
        np.testing.assert_allclose(x1, x0, rtol=0, atol=1e-6)
        np.testing.assert_allclose(v1, v0, rtol=0, atol=1e-4)


@pytest.mark.parametrize("method", METHODS)
def test_cell_order_changes_storage_not_physics(method):
    (x0, v0, r0), t0, _ = run(method, 8)
    (x1, v1, r1), t1, _ = run(method, 8, [(api.OPT_CELL_ORDER, 1)])
    assert t0 == t1
    if method == S.WCSPH:
        assert np.array_equal(x0, x1) and np.array_equal(v0, v1) and np.array_equal(r0, r1)
    else:
        np.testing.assert_allclose(x1, x0, rtol=0, atol=1e-6)
        np.testing.assert_allclose(v1, v0, rtol=0, atol=1e-4)


def test_cell_order_switch_mid_run():
    """Switching the order after init re-sorts boundary and fluid; the next
    steps continue the same trajectory."""
    a = small_sim(S.WCSPH)
    a.step(4)
    a.set_option(api.OPT_CELL_ORDER, 1)
    a.step(4)
    b = small_sim(S.WCSPH)
    b.step(8)
    for u, w in zip(a.state(), b.state()):
        assert np.array_equal(u, w)
    np.testing.assert_array_equal(a.boundary_volume(), b.boundary_volume())
    a.close(); b.close()


@pytest.mark.parametrize("method", METHODS)
def test_autotune_leaves_state_untouched(method, tmp_path):
    sim = small_sim(method)
    sim.step(3)
    before, tb = sim.state(), sim.time()
    cache = tmp_path / "tune.json"
    cfg = sim.autotune(trial_steps=2, cache_path=str(cache))
    assert cfg["cell_order"] in (0, 1) and cfg["solver_occupancy"] in (4, 8) and cfg["pass_block"] in (128, 256)
    assert cfg["solver_lanes"] in (1, 2, 4)
    assert sim.get_option(api.OPT_SOLVER_LANES) == cfg["solver_lanes"]
    assert sim.get_option(api.OPT_CELL_ORDER) == cfg["cell_order"]
    assert sim.get_option(api.OPT_SOLVER_OCCUPANCY) == cfg["solver_occupancy"]
    assert sim.get_option(api.OPT_PASS_BLOCK) == cfg["pass_block"]
    after, ta = sim.state(), sim.time()
    for u, w in zip(before, after):
        assert np.array_equal(u, w)
    assert ta == tb
    st = sim.step(3)
    assert st["steps"] == 3
    # the continued run follows the untuned one
    ref = small_sim(method)
    ref.step(6)
    x_ref = ref.state()[0]
    atol = 0 if method == S.WCSPH else 1e-6
    np.testing.assert_allclose(sim.state()[0], x_ref, rtol=0, atol=atol)
    # the cache now holds the choice, and a second context reuses it
    table = json.loads(cache.read_text())
    assert len(table) == 1 and list(table.values())[0] == [cfg["cell_order"], cfg["solver_occupancy"],
                                                            cfg["pass_block"], cfg["solver_lanes"]]
    other = small_sim(method)
    assert other.autotune(trial_steps=2, cache_path=str(cache)) == cfg
    assert len(json.loads(cache.read_text())) == 1
    sim.close(); ref.close(); other.close()


def test_autotune_batch_restores_scene_states():
    dims = [(6, 5, 7), (9, 8, 6), (5, 5, 5)]
    b = Batch([Scene.from_dict(S.small(method=S.DFSPH, n=n, radius=0.02, seed=40 + k)) for k, n in enumerate(dims)])
    b.step(2)
    before = [b.scene_state(s) for s in range(3)]
    b.autotune(trial_steps=1)
    after = [b.scene_state(s) for s in range(3)]
    for sa, sb in zip(before, after):
        for u, w in zip(sa, sb):
            assert np.array_equal(u, w)
    st = b.step(2)
    assert st["steps"] == 2
    b.close()
