"""The FP64 WCSPH adjoint of the oracle (oracle/wcsph_adjoint.cpp), on the CPU.

Pinning: its forward run equals the FP64 restatement of the reference
(oracle/sph_oracle.cpp, itself pinned to the reference's FP64 build by
test_oracle.py) after the same steps, and its gradients equal FP64 central
differences of that forward run. The GPU adjoint is then checked against it
(test_gpu_adjoint.py)."""
import numpy as np
import pytest

from oracle.oracle import Oracle, wcsph_adjoint
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene

NSTEPS = 20


@pytest.fixture(scope="module")
def problem():
    d = S.small(method=S.WCSPH, n=(8, 8, 8), radius=0.02, time_step=2e-4, viscosity=0.01,
                boundary_viscosity=0.005, seed=5)
    sc = Scene.from_dict(d)
    desc = sc.desc()
    x0, _ = sc.fluid()
    b = sc.boundary()
    v0, t = S.adjoint_problem(x0)
    g = wcsph_adjoint(desc, x0, v0, b, NSTEPS, t)
    return desc, x0, v0, b, t, g


def test_forward_equals_fp64_restatement(problem):
    desc, x0, v0, b, t, g = problem
    o = Oracle(desc, x0, b, vel=v0, fp64=True)
    o.step(NSTEPS)
    ox, _, _ = o.state()
    err = np.max(np.abs(ox - g["x"])) / np.max(np.abs(ox))
    assert err <= 1e-12, err
    assert g["loss"] == pytest.approx(float(np.mean(np.sum((ox - t) ** 2, axis=1))), rel=1e-10)


def central(desc, x0, v0, b, t, eps, dx=None, dv=None, nu=None, k=None):
    def loss(sign):
        xx = x0 if dx is None else x0.astype(np.float64) + sign * eps * dx
        vv = v0 if dv is None else v0.astype(np.float64) + sign * eps * dv
        kw = {}
        if nu is not None:
            kw["nu"] = nu + sign * eps
        if k is not None:
            kw["k"] = k + sign * eps
        return wcsph_adjoint(desc, xx, vv, b, NSTEPS, t, grad=False, **kw)["loss"]
    return (loss(1) - loss(-1)) / (2 * eps)


@pytest.mark.parametrize("seed", [100, 101, 102])
def test_v0_gradient_vs_central_differences(problem, seed):
    """Directional derivative along a seeded direction, eps = 1e-4 (FP64)."""
    desc, x0, v0, b, t, g = problem
    d = np.random.default_rng(seed).normal(size=x0.shape)
    fd = central(desc, x0, v0, b, t, 1e-4, dv=d)
    ad = float(np.sum(g["v0"] * d))
    assert abs(ad - fd) <= 1e-5 * abs(fd), (ad, fd)


def test_x0_gradient_vs_central_differences(problem):
    """Positions start on a lattice of spacing h / 2, where the spline's
    second derivative jumps (q = 1/2): central differences converge to the
    adjoint only linearly there, so the step is small (1e-7 m)."""
    desc, x0, v0, b, t, g = problem
    d = np.random.default_rng(7).normal(size=x0.shape)
    fd = central(desc, x0, v0, b, t, 1e-7, dx=d)
    ad = float(np.sum(g["x0"] * d))
    assert abs(ad - fd) <= 1e-5 * abs(fd), (ad, fd)


def test_parameter_gradients_vs_central_differences(problem):
    desc, x0, v0, b, t, g = problem
    nu, k = float(desc.viscosity), float(desc.stiffness)
    fd_nu = central(desc, x0, v0, b, t, 1e-6, nu=nu)
    fd_k = central(desc, x0, v0, b, t, 1e-2, k=k)
    assert abs(g["viscosity"] - fd_nu) <= 1e-5 * abs(fd_nu), (g["viscosity"], fd_nu)
    assert abs(g["stiffness"] - fd_k) <= 1e-5 * abs(fd_k), (g["stiffness"], fd_k)


def test_zero_steps_is_the_loss_gradient(problem):
    desc, x0, v0, b, t, _ = problem
    g = wcsph_adjoint(desc, x0, v0, b, 0, t)
    n = x0.shape[0]
    assert np.allclose(g["x0"], 2.0 * (x0.astype(np.float64) - t) / n, rtol=1e-12, atol=0)
    assert np.all(g["v0"] == 0.0) and g["viscosity"] == 0.0 and g["stiffness"] == 0.0
