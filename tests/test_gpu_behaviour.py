"""GPU behaviour beyond reference parity: determinism, bounded waits,
error statuses, state round trips and accounting. Failures are produced on
the host (bad inputs) or with the bounded-wait probe; nothing here faults or
hangs the device."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from sph2o_b200 import scenes as S
from sph2o_b200.api import SPH_OK, Scene, SceneDesc, Simulation, SphError, lib

pytestmark = pytest.mark.gpu


def small_sim(method=S.DFSPH, **kw):
    return Simulation.from_scene(Scene.from_dict(S.small(method=method, **kw)))


@pytest.mark.parametrize("method", [S.WCSPH, S.PCISPH, S.DFSPH])
def test_deterministic(method):
    runs = []
    for _ in range(2):
        sim = small_sim(method, surface_tension=0.05)
        sim.step(10)
        runs.append(sim.state())
        sim.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


def test_step_in_chunks_equals_one_call():
    a = small_sim()
    a.step(6)
    b = small_sim()
    for _ in range(3):
        b.step(2)
    for u, w in zip(a.state(), b.state()):
        assert np.array_equal(u, w)
    a.close(); b.close()


def test_async_and_sync():
    sim = small_sim()
    sim.step_async(3)
    sim.step_async(2)
    st = sim.sync()
    assert st["steps"] == 5 and st["kernel_launches"] > 0 and st["device_ms"] > 0
    sim.close()


def test_barrier_wait_runs_out_and_context_survives():
    sim = small_sim()
    rc = lib().sph_debug_barrier_timeout(sim._h)
    assert rc == -5  # SPH_ERR_TIMEOUT
    st = sim.step(2)  # the context is still usable
    assert st["steps"] == 2
    sim.close()


def test_nan_detected():
    sim = small_sim(method=S.WCSPH)
    x, v, _ = sim.state()
    x[7, 1] = np.nan
    sim.set_state(x, v)
    with pytest.raises(SphError) as e:
        sim.step(1)
    assert e.value.code == -3
    sim.close()


def test_set_get_state_roundtrip():
    sim = small_sim()
    sim.step(2)
    x, v, _ = sim.state()
    x2 = x + np.float32(1e-4)
    v2 = v * np.float32(0.5)
    sim.set_state(x2, v2)
    x3, v3, _ = sim.state()
    assert np.array_equal(x3, x2) and np.array_equal(v3, v2)
    sim.close()


def test_call_order_errors():
    L = lib()
    d = Scene.from_dict(S.small()).desc()
    h = C.c_void_p()
    assert L.sph_create(C.byref(d), C.byref(h)) == SPH_OK
    assert L.sph_step(h, 1, None) == -6                   # before init
    assert L.sph_init(h) == -1                             # no fluid
    L.sph_destroy(h)
    bad = SceneDesc()
    C.memmove(C.byref(bad), C.byref(d), C.sizeof(d))
    bad.boundary_method = 3  # no such method
    assert L.sph_create(C.byref(bad), C.byref(h)) == -1
    bad.boundary_method = 1  # PCISPH boundary particles need their normals before init
    assert L.sph_create(C.byref(bad), C.byref(h)) == SPH_OK
    x = np.zeros((8, 3), np.float32)
    x[:, 0] = np.arange(8) * 0.05
    assert L.sph_set_fluid(h, 8, x.ctypes.data_as(C.POINTER(C.c_float)), None) == SPH_OK
    assert L.sph_set_boundary(h, 8, (x + np.float32(1.0)).ctypes.data_as(C.POINTER(C.c_float))) == SPH_OK
    assert L.sph_init(h) == -1
    L.sph_destroy(h)


def test_outside_grid_particles_still_found():
    """A particle far outside the initial bounding box lands in a clamped edge
    cell; its neighbour search must still find every particle within h."""
    g = load_golden("wcsph_artificial")
    sim = Simulation.from_scene(Scene.from_dict(g["scene"]))
    x, v, _ = sim.state()
    x[0] = (-3.0, -3.0, -3.0)
    x[1] = (-3.05, -3.0, -3.0)
    sim.set_state(x, v)
    fo, fi, bo, bi = sim.neighbors()
    assert set(fi[fo[0]:fo[1]].tolist()) == {0, 1}
    sim.close()
