"""Neighbour sets at the edge of the support radius.

A pair is in the set when glm::length(x_i - x_j) <= h in FP32, i.e.
sqrt_rn((dx dx + dy dy) + dz dz) <= h (the filter the golden fixtures were
written with, applied to the reference's 27-cell candidates, HashTable.cpp:23-86).
The list build decides it without the square root, against the largest FP32
sum whose rounded square root is still <= h. These pairs are placed within a
few ulps of h along axes, face and body diagonals and random directions, for
fluid and boundary partners, so both sides of the bound are hit."""
import numpy as np
import pytest

from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, Simulation

pytestmark = pytest.mark.gpu


def ref_within(a, b, h):
    """The reference's test in FP32 (numpy rounds each operation, no FMA)."""
    d = np.asarray(a, np.float32) - np.asarray(b, np.float32)
    s = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    return np.sqrt(s) <= np.float32(h)


def edge_pairs(h, n_centres, rng, origin):
    """Centres on a lattice of spacing 3h; each has one partner at h * (1 + k eps)."""
    dirs = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (-1, 0, 0), (1, 1, 0), (0, 1, -1), (1, 1, 1), (-1, 1, -1)]
    dirs = [np.array(d, np.float64) / np.linalg.norm(d) for d in dirs]
    side = int(np.ceil(n_centres ** (1 / 3)))
    centres, partners = [], []
    for m in range(n_centres):
        ix, iy, iz = m % side, (m // side) % side, m // (side * side)
        c = origin + 3.0 * h * np.array([ix, iy, iz], np.float64) + rng.uniform(0, 0.5 * h, 3)
        d = dirs[m % len(dirs)] if m % 3 else rng.normal(size=3)
        d = d / np.linalg.norm(d)
        k = int(rng.integers(-6, 7))
        dist = float(h) * (1.0 + k * float(np.finfo(np.float32).eps))
        centres.append(c)
        partners.append(c + dist * d)
    return np.asarray(centres, np.float32), np.asarray(partners, np.float32)


def test_neighbor_sets_at_h_to_the_ulp():
    sc = Scene.from_dict(S.small(method=S.WCSPH))
    desc = sc.desc()
    h = np.float32(np.float32(4.0) * np.float32(desc.particle_radius))
    rng = np.random.default_rng(5)
    origin = np.array([0.3, 0.3, 0.3])
    cf, pf = edge_pairs(h, 600, rng, origin)                 # fluid-fluid pairs
    cb, pb = edge_pairs(h, 600, rng, origin + [0.0, 0.0, 30 * h])   # fluid-boundary pairs
    fluid = np.concatenate([cf, pf, cb])
    boundary = pb
    sim = Simulation(desc, fluid, boundary)
    fo, fi, bo, bi = sim.neighbors()
    sim.close()

    nf = fluid.shape[0]
    want_f = ref_within(fluid[:, None, :], fluid[None, :, :], h)
    want_b = ref_within(fluid[:, None, :], boundary[None, :, :], h)
    # the placement puts both outcomes in play
    pair_f = ref_within(cf, pf, h)
    pair_b = ref_within(cb, pb, h)
    assert 0 < pair_f.sum() < pair_f.size and 0 < pair_b.sum() < pair_b.size
    for i in range(nf):
        got = np.sort(fi[fo[i]:fo[i + 1]])
        assert np.array_equal(got, np.flatnonzero(want_f[i])), f"fluid set of particle {i}"
        got = np.sort(bi[bo[i]:bo[i + 1]])
        assert np.array_equal(got, np.flatnonzero(want_b[i])), f"boundary set of particle {i}"
