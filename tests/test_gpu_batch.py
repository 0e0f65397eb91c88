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
