"""sph_density_noalloc: the allocation-free density entry point.

It serves callers that must not allocate GPU memory (host callbacks,
allocator hooks, framework-pooled memory, real-time paths that cannot take
the allocator's locks); its scratch is a fixed device array inside the
library. This file is named to be collected last, so a run that stops at
the first failure has already run every other test; it also passes alone in
a fresh process.

The check: two calls in a row on different particle sets, each compared
with the context path's densities (sph_compute_phase) for the same
particles -- equal bit for bit, the tolerance the density tests use; a
fluid-only call (no boundary array) against the context path without
boundary particles, bit for bit; particles outside the given domain,
which are clamped into edge cells and summed in another order, within 1e-6
relative; oversize input rejected with SPH_ERR_CAPACITY and non-finite
bounds with SPH_ERR_ARG before any work is queued.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from sph2o_b200 import api
from sph2o_b200.api import Scene, Simulation, lib

pytestmark = pytest.mark.gpu


def _bind():
    L = lib()
    L.sph_density_noalloc.restype = C.c_int
    L.sph_density_noalloc.argtypes = [C.c_float, C.c_float, C.c_void_p, C.c_uint, C.c_void_p, C.c_uint,
                                      C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p, C.c_void_p]
    L.sph_noalloc_error.restype = C.c_char_p
    return L


def _context_density(desc, fluid, boundary):
    sim = Simulation(desc, fluid, boundary)
    rho = sim.phase(api.PHASE_DENSITY)
    vol = sim.boundary_volume()
    sim.close()
    return rho, vol


def test_noalloc_density_equals_context_path_twice():
    import torch

    L = _bind()
    g = load_golden("dfsph_st_sphere")
    sc = Scene.from_dict(g["scene"])
    desc = sc.desc()
    x, _ = sc.fluid()
    b = sc.boundary()
    r, rho0 = desc.particle_radius, desc.density0
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    lo = np.minimum(x.min(0), b.min(0)).astype(np.float32)
    hi = np.maximum(x.max(0), b.max(0)).astype(np.float32)
    lo_c = (C.c_float * 3)(*lo)
    hi_c = (C.c_float * 3)(*hi)
    shifts = [np.float32(0.0), np.float32(0.5 * r)]
    for call, shift in enumerate(shifts):
        xs = (x + shift).astype(np.float32)
        ref, vol = _context_density(desc, xs, b)
        psi = (np.float32(rho0) * vol).astype(np.float32)
        bx = np.ascontiguousarray(np.concatenate([b, psi[:, None]], axis=1), np.float32)
        xt = torch.from_numpy(np.ascontiguousarray(xs)).to(dev)
        bt = torch.from_numpy(bx).to(dev)
        out = torch.full((xs.shape[0],), -1.0, dtype=torch.float32, device=dev)
        rc = L.sph_density_noalloc(r, rho0, xt.data_ptr(), xs.shape[0], bt.data_ptr(), b.shape[0], lo_c, hi_c,
                                   out.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.sph_noalloc_error()
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        assert np.array_equal(got, ref), f"call {call}: max |diff| {np.max(np.abs(got - ref))}"


def test_noalloc_rejects_oversize():
    import torch

    L = _bind()
    dev = torch.device("cuda", 0)
    n = 65537
    xt = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    out = torch.zeros(n, dtype=torch.float32, device=dev)
    lo = (C.c_float * 3)(0, 0, 0)
    hi = (C.c_float * 3)(1, 1, 1)
    rc = L.sph_density_noalloc(0.01, 1000.0, xt.data_ptr(), n, None, 0, lo, hi, out.data_ptr(), None)
    assert rc == -9
    assert b"SPH_NOALLOC_MAX_FLUID" in L.sph_noalloc_error()
    big_hi = (C.c_float * 3)(100, 100, 100)
    rc = L.sph_density_noalloc(0.01, 1000.0, xt.data_ptr(), 10, None, 0, lo, big_hi, out.data_ptr(), None)
    assert rc == -9
    assert b"SPH_NOALLOC_MAX_CELLS" in L.sph_noalloc_error() or b"too large" in L.sph_noalloc_error()


def _call(L, r, rho0, xs, bx, lo, hi):
    """One allocation-free call on cuda:0's current stream; returns the densities."""
    import torch

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    xt = torch.from_numpy(np.ascontiguousarray(xs, np.float32)).to(dev)
    bt = None if bx is None else torch.from_numpy(np.ascontiguousarray(bx, np.float32)).to(dev)
    out = torch.full((xs.shape[0],), -1.0, dtype=torch.float32, device=dev)
    lo_c = (C.c_float * 3)(*[float(v) for v in lo])
    hi_c = (C.c_float * 3)(*[float(v) for v in hi])
    rc = L.sph_density_noalloc(r, rho0, xt.data_ptr(), xs.shape[0], None if bt is None else bt.data_ptr(),
                               0 if bx is None else bx.shape[0], lo_c, hi_c, out.data_ptr(),
                               C.c_void_p(stream.cuda_stream))
    assert rc == 0, L.sph_noalloc_error()
    torch.cuda.synchronize(dev)
    return out.cpu().numpy()


def test_noalloc_fluid_only_equals_context_path():
    """nb = 0 (no boundary array): the boundary cell table is cleared instead
    of sorted; the densities equal the context path's for the same fluid
    with no boundary particles, twice in a row."""
    L = _bind()
    g = load_golden("dfsph_st_sphere")
    sc = Scene.from_dict(g["scene"])
    desc = sc.desc()
    x, _ = sc.fluid()
    r, rho0 = desc.particle_radius, desc.density0
    none = np.zeros((0, 3), np.float32)
    for call in range(2):
        xs = (x + np.float32(call * 0.3 * r)).astype(np.float32)
        ref, _ = _context_density(desc, xs, none)
        got = _call(L, r, rho0, xs, None, xs.min(0), xs.max(0))
        assert np.array_equal(got, ref), f"call {call}: max |diff| {np.max(np.abs(got - ref))}"


def test_noalloc_particles_outside_domain():
    """A domain that leaves a slab of the fluid (several cells deep) outside:
    those particles are clamped into edge cells and still find every
    neighbour; densities within 1e-6 relative of the context path, and the
    particles well inside the domain still bit for bit."""
    L = _bind()
    g = load_golden("dfsph_st_sphere")
    sc = Scene.from_dict(g["scene"])
    desc = sc.desc()
    x, _ = sc.fluid()
    b = sc.boundary()
    r, rho0 = desc.particle_radius, desc.density0
    h = 4.0 * r
    ref, vol = _context_density(desc, x, b)
    psi = (np.float32(rho0) * vol).astype(np.float32)
    bx = np.concatenate([b, psi[:, None]], axis=1)
    lo = np.minimum(x.min(0), b.min(0)).astype(np.float32)
    hi = np.maximum(x.max(0), b.max(0)).astype(np.float32)
    lo_cut = lo.copy()
    lo_cut[0] = np.float32(x.min(0)[0] + 3.5 * h)  # the first ~3.5 cells of fluid in x lie outside
    outside = x[:, 0] < lo_cut[0] - 2 * h
    assert outside.sum() > 0
    got = _call(L, r, rho0, x, bx, lo_cut, hi)
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got.astype(np.float64) - ref) / np.abs(ref)) <= 1e-6
    inside = x[:, 0] > lo_cut[0] + 2 * h
    assert np.array_equal(got[inside], ref[inside])


def test_noalloc_rejects_non_finite_bounds():
    import torch

    L = _bind()
    dev = torch.device("cuda", 0)
    xt = torch.zeros((4, 3), dtype=torch.float32, device=dev)
    out = torch.zeros(4, dtype=torch.float32, device=dev)
    inf = float("inf")
    for lo, hi in (((0, 0, 0), (inf, 1, 1)), ((inf, 0, 0), (inf, 1, 1)), ((0, 0, 0), (1, float("nan"), 1)),
                   ((1e30, 0, 0), (1e30, 1, 1))):
        rc = L.sph_density_noalloc(0.01, 1000.0, xt.data_ptr(), 4, None, 0, (C.c_float * 3)(*lo),
                                   (C.c_float * 3)(*hi), out.data_ptr(), None)
        assert rc == -1, (lo, hi, rc)
