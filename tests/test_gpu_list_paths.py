"""Both neighbour-list builds against an exact CPU neighbour search.

Scenes below 2^16 fluid particles take the warp-per-particle build, larger
ones the one-lane-per-particle build. Around that threshold each build's
fluid and boundary sets must equal { j : sqrt_rn((dx dx + dy dy) + dz dz) <= h }
in FP32 (the golden fixtures' filter), found here with a k-d tree and the
reference's float test, and each list must follow the reference's candidate
order: the 27 cells in x-major offset order, ascending slot inside a cell."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation

pytestmark = pytest.mark.gpu


def exact_sets(points, others, h):
    tree = cKDTree(others.astype(np.float64))
    cand = tree.query_ball_point(points.astype(np.float64), r=float(h) * (1 + 1e-5))
    out = []
    for i, c in enumerate(cand):
        c = np.asarray(sorted(c), np.int64)
        if c.size:
            d = points[i][None, :] - others[c]
            s = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
            c = c[np.sqrt(s) <= h]
        out.append(c)
    return out


def cell_rank(points, idx, xi, h):
    """(cell offset index in x-major order, position within the cell) of each
    candidate: the reference's candidate order for particle position xi."""
    ci = np.floor(xi / h).astype(np.int64)
    cj = np.floor(points[idx] / h).astype(np.int64)
    off = cj - ci
    return (off[:, 0] + 1) * 9 + (off[:, 1] + 1) * 3 + (off[:, 2] + 1)


@pytest.mark.parametrize("n", [(40, 40, 38), (42, 42, 40)])  # 60,800 (warp build) and 70,560 (one lane)
def test_list_build_matches_exact_search(n):
    sc = Scene.from_dict(S.small(method=S.WCSPH, n=n, seed=9))
    x, _ = sc.fluid()
    b = sc.boundary()
    desc = sc.desc()
    h = np.float32(np.float32(4.0) * np.float32(desc.particle_radius))
    sim = Simulation.from_scene(sc)
    fo, fi, bo, bi = sim.neighbors()
    sim.close()
    nf = x.shape[0]
    assert nf == n[0] * n[1] * n[2]
    want_f = exact_sets(x, x, h)
    want_b = exact_sets(x, b, h)
    for i in range(0, nf, 7):
        got = fi[fo[i]:fo[i + 1]].astype(np.int64)
        assert np.array_equal(np.sort(got), want_f[i]), f"fluid set of particle {i}"
        # candidate order: cell offset index non-decreasing, caller index rising inside a cell
        k = cell_rank(x, got, x[i], h)
        dk, dj = np.diff(k), np.diff(got)
        assert np.all((dk > 0) | ((dk == 0) & (dj > 0))), f"candidate order of particle {i}"
        got_b = bi[bo[i]:bo[i + 1]].astype(np.int64)
        assert np.array_equal(np.sort(got_b), want_b[i]), f"boundary set of particle {i}"


@pytest.mark.parametrize("make,steps", [
    (lambda: S.small(method=S.WCSPH, n=(42, 42, 40), seed=9), 60),   # 70,560: full cells, tank walls
    (lambda: S.dam_break_dfsph_125k(), 25),                          # surface tension, splashing cells
    (lambda: S.double_dam_break_1m(), 2),                            # 1M, sphere obstacle
])
def test_staged_build_equals_one_lane_build(make, steps):
    """OPT_LIST_STAGED = 1 builds the lists of large single scenes one brick
    per block from the brick's 6x6x6 cells staged in shared memory; it must
    write the one-lane build's lists entry for entry, and so give the same
    trajectory bit for bit: at the start and after `steps` steps."""
    from sph2o_b200.api import OPT_LIST_STAGED
    d = make()
    out = {}
    for staged in (1, 0):
        sim = Simulation.from_scene(Scene.from_dict(d), options={OPT_LIST_STAGED: staged})
        first = sim.neighbors()
        sim.step(steps)
        out[staged] = first + sim.neighbors() + sim.state()
        sim.close()
    for k, (a, b) in enumerate(zip(out[1], out[0])):
        assert a.dtype == b.dtype and np.array_equal(a, b), f"array {k} differs"
