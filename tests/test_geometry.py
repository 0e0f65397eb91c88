"""OBJ "geometry" boundaries without a GPU: the host OBJ loader, and the CPU
oracle of the regular triangle sampler pinned bit for bit against the
boundary particles the SPH2O reference itself generated (golden fixtures
from its FP32 build); properties that hold for any mesh (every sample on
the surface, the surface covered at the stated spacing); and the product
sampler refusing to run without a device. The GPU sampler is checked
against the same fixtures and the oracle in test_gpu_geometry.py."""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oracle import oracle as O
from sph2o_b200.api import Scene, SphError, load_obj, sample_mesh

GEOMETRY_GOLDEN = ["geometry_dfsph_cup", "geometry_wcsph_quirks"]
MESHES = ["cup.obj", "quirks.obj", "shards.obj"]
ROT = (np.float32(math.pi * 0.5), 0.0, 0.0)


def read_obj(path):
    """Plain reader for the test meshes: vertices and 0-based faces."""
    v, f = [], []
    with open(path) as fh:
        for line in fh:
            t = line.split()
            if t and t[0] == "v":
                v.append([float(x) for x in t[1:4]])
            elif t and t[0] == "f":
                f.append([int(x.split("/")[0]) - 1 for x in t[1:4]])
    return np.array(v, np.float32), np.array(f, np.uint32)


def spacing_of(scene, spacing):
    """spacing * particleRadius * 2 in float (SPHSimulation.cpp:423)."""
    r = np.float32(scene["Configuration"]["particleRadius"])
    return np.float32(np.float32(np.float32(spacing) * r) * np.float32(2.0))


def scene_geometries(scene):
    for b in scene["Boundary"]:
        for g in b.get("geometry", []):
            yield g["path"], spacing_of(scene, g["spacing"])


@pytest.mark.parametrize("obj", MESHES)
def test_obj_loader(obj):
    v, f = load_obj(os.path.join(GOLDEN, obj))
    rv, rf = read_obj(os.path.join(GOLDEN, obj))
    assert np.array_equal(v, rv) and np.array_equal(f, rf)
    vs, _ = load_obj(os.path.join(GOLDEN, obj), scale=(2.0, 0.5, 1.0))
    assert np.array_equal(vs, rv * np.float32([2.0, 0.5, 1.0]))


@pytest.mark.parametrize("name", GEOMETRY_GOLDEN)
def test_oracle_matches_reference_samples(name):
    """The oracle's samples with addGeometry's placement are the mesh part
    of the reference's boundary object (boxes and spheres come first)."""
    g = load_golden(name)
    geo = np.concatenate([O.sample_mesh(*load_obj(p), d, rotate=ROT) for p, d in scene_geometries(g["scene"])])
    assert len(geo) > 100
    assert np.array_equal(geo.view(np.uint32), g["bpos"][-len(geo):].view(np.uint32))


def point_triangle_distance(p, a, b, c):
    """Distance from p to triangle abc (closest point by region tests)."""
    ab, ac, ap = b - a, c - a, p - a
    n = np.cross(ab, ac)
    nn = float(n @ n)
    if nn > 0:
        q = p - (float(ap @ n) / nn) * n
        w1 = float(np.cross(q - a, ac) @ n) / nn
        w2 = float(np.cross(ab, q - a) @ n) / nn
        if w1 >= -1e-7 and w2 >= -1e-7 and w1 + w2 <= 1 + 1e-7:
            return float(np.linalg.norm(p - q))
    best = math.inf
    for u, w in ((a, b), (b, c), (c, a)):
        e = w - u
        t = 0.0 if float(e @ e) == 0 else min(1.0, max(0.0, float((p - u) @ e) / float(e @ e)))
        best = min(best, float(np.linalg.norm(p - (u + t * e))))
    return best


@pytest.mark.parametrize("obj", MESHES)
def test_samples_lie_on_the_surface(obj):
    v, f = read_obj(os.path.join(GOLDEN, obj))
    v64 = v.astype(np.float64)
    s = O.sample_mesh(v, f, 0.05).astype(np.float64)
    assert np.array_equal(s[:len(v)], v64)  # the vertices come first, in file order
    tri = [(v64[a], v64[b], v64[c]) for a, b, c in f]
    for p in s[len(v):]:
        assert min(point_triangle_distance(p, *t) for t in tri) < 1e-5


def test_surface_covered_at_spacing():
    """Random points of each cup face have a sample within the spacing d
    (the lines and stops are at most d apart)."""
    v, f = read_obj(os.path.join(GOLDEN, "cup.obj"))
    d = 0.05
    s = O.sample_mesh(v, f, d).astype(np.float64)
    rng = np.random.default_rng(3)
    for a, b, c in f:
        w = rng.dirichlet((1, 1, 1), size=40)
        pts = w @ np.stack([v[a], v[b], v[c]]).astype(np.float64)
        dist = np.sqrt(((pts[:, None, :] - s[None, :, :]) ** 2).sum(-1)).min(1)
        assert dist.max() <= d


def test_coincident_face_adds_no_face_samples():
    """A face whose three vertices coincide: its (zero-length) edge is
    sampled as its first vertex once more, the face adds nothing."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    base = O.sample_mesh(v, [[0, 1, 2]], 0.1)
    withdeg = O.sample_mesh(v, [[0, 1, 2], [1, 1, 1]], 0.1)
    expect = np.concatenate([base, v[1:2]])
    assert len(withdeg) == len(expect)
    key = [("", np.float32)] * 3
    assert np.array_equal(np.sort(withdeg.view(key), axis=0), np.sort(expect.view(key), axis=0))


def test_loader_errors(tmp_path):
    with pytest.raises(SphError) as e:
        load_obj(str(tmp_path / "none.obj"))
    assert e.value.code == -8
    p = tmp_path / "bad.obj"
    for text in ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n", "v 0 0 nan\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
                 "v 0 0\n", "v 0 0 0\nf 1 1\n"):
        p.write_text(text)
        with pytest.raises(SphError) as e:
            load_obj(str(p))
        assert e.value.code == -1


def test_missing_geometry_file_is_an_io_error():
    g = load_golden("geometry_dfsph_cup")
    g["scene"]["Boundary"][0]["geometry"][0]["path"] = os.path.join(GOLDEN, "missing.obj")
    with pytest.raises(SphError) as e:
        Scene.from_dict(g["scene"])
    assert e.value.code == -8


def test_sampler_needs_a_device():
    """The product sampler runs on the GPU only: without a device it fails
    with SPH_ERR_NO_DEVICE instead of computing on the host."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    v, f = read_obj(os.path.join(GOLDEN, "cup.obj"))
    with pytest.raises(SphError) as e:
        sample_mesh(v, f, 0.05)
    assert e.value.code == -7
    with pytest.raises(SphError) as e:
        Scene.from_dict(load_golden("geometry_dfsph_cup")["scene"])
    assert e.value.code == -7
