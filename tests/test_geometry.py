"""OBJ "geometry" boundaries on the host (no GPU): the loader and the
regular triangle sampler against the SPH2O reference's own boundary
particles (golden fixtures from its FP32 build, bit-exact), the C ABI's
two-call convention and errors, and properties that hold for any mesh
(every sample on the surface; the surface covered at the stated spacing)."""
import json
import math
import os
import shutil

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from sph2o_b200 import scenes as S
from sph2o_b200.api import Scene, SphError, sample_geometry, sample_mesh

GEOMETRY_GOLDEN = ["geometry_dfsph_cup", "geometry_wcsph_quirks"]
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
    return np.array(v, np.float32), np.array(f, np.int64)


def spacing_of(scene, spacing):
    r = np.float32(scene["Configuration"]["particleRadius"])
    return np.float32(np.float32(np.float32(spacing) * r) * np.float32(2.0))


def geometry_samples(scene):
    """The scene's geometry samples, in load order, from the C ABI."""
    out = []
    for b in scene["Boundary"]:
        for g in b.get("geometry", []):
            out.append(sample_geometry(g["path"], spacing_of(scene, g["spacing"]), rotate=ROT))
    return np.concatenate(out)


@pytest.mark.parametrize("name", GEOMETRY_GOLDEN)
def test_scene_boundary_bit_exact(name):
    g = load_golden(name)
    b = Scene.from_dict(g["scene"]).boundary()
    assert b.shape == g["bpos"].shape
    assert np.array_equal(b.view(np.uint32), g["bpos"].view(np.uint32))


@pytest.mark.parametrize("name", GEOMETRY_GOLDEN)
def test_geometry_entry_point_matches_scene_tail(name):
    """sph_sample_geometry with addGeometry's placement gives the mesh part
    of the reference's boundary object (boxes and spheres come first)."""
    g = load_golden(name)
    geo = geometry_samples(g["scene"])
    assert len(geo) > 100
    assert np.array_equal(geo.view(np.uint32), g["bpos"][-len(geo):].view(np.uint32))


def test_mesh_entry_point_equals_unrotated_geometry():
    v, f = read_obj(os.path.join(GOLDEN, "shards.obj"))
    d = np.float32(0.05)
    a = sample_mesh(v, f, d)
    b = sample_geometry(os.path.join(GOLDEN, "shards.obj"), d)
    assert np.array_equal(a, b)
    # the vertices come first, in file order
    assert np.array_equal(a[:len(v)], v)


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


@pytest.mark.parametrize("obj", ["cup.obj", "quirks.obj", "shards.obj"])
def test_samples_lie_on_the_surface(obj):
    v, f = read_obj(os.path.join(GOLDEN, obj))
    v64 = v.astype(np.float64)
    s = sample_mesh(v, f, 0.05).astype(np.float64)
    tri = [(v64[a], v64[b], v64[c]) for a, b, c in f]
    for p in s[len(v):]:
        assert min(point_triangle_distance(p, *t) for t in tri) < 1e-5


def test_surface_covered_at_spacing():
    """Random points of each cup face have a sample within the spacing d
    (the lines and stops are at most d apart)."""
    v, f = read_obj(os.path.join(GOLDEN, "cup.obj"))
    d = 0.05
    s = sample_mesh(v, f, d).astype(np.float64)
    rng = np.random.default_rng(3)
    for a, b, c in f:
        w = rng.dirichlet((1, 1, 1), size=40)
        pts = w @ np.stack([v[a], v[b], v[c]]).astype(np.float64)
        dist = np.sqrt(((pts[:, None, :] - s[None, :, :]) ** 2).sum(-1)).min(1)
        assert dist.max() <= d


def test_two_call_convention_and_errors(tmp_path):
    from sph2o_b200.api import lib
    import ctypes as C

    v, f = read_obj(os.path.join(GOLDEN, "cup.obj"))
    v = np.ascontiguousarray(v)
    fu = np.ascontiguousarray(f, np.uint32)
    n = C.c_size_t()
    L = lib()
    fp = v.ctypes.data_as(C.POINTER(C.c_float))
    up = fu.ctypes.data_as(C.POINTER(C.c_uint))
    assert L.sph_sample_mesh(fp, len(v), up, len(fu), 0.05, None, 0, C.byref(n)) == 0
    small = np.zeros((n.value - 1, 3), np.float32)
    assert L.sph_sample_mesh(fp, len(v), up, len(fu), 0.05, small.ctypes.data_as(C.POINTER(C.c_float)),
                             len(small), C.byref(n)) == -9
    assert n.value == len(small) + 1
    with pytest.raises(SphError) as e:
        sample_mesh(v, f, 0.0)
    assert e.value.code == -1
    bad = f.copy()
    bad[3, 1] = len(v)
    with pytest.raises(SphError) as e:
        sample_mesh(v, bad, 0.05)
    assert e.value.code == -1
    with pytest.raises(SphError) as e:
        sample_geometry(str(tmp_path / "none.obj"), 0.05)
    assert e.value.code == -8
    p = tmp_path / "badidx.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n")
    with pytest.raises(SphError) as e:
        sample_geometry(str(p), 0.05)
    assert e.value.code == -1
    p.write_text("v 0 0 nan\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    with pytest.raises(SphError) as e:
        sample_geometry(str(p), 0.05)
    assert e.value.code == -1


def test_coincident_face_adds_no_face_samples():
    """A face whose three vertices coincide: its vertices and (zero-length)
    edges are sampled, the face itself adds nothing."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    base = sample_mesh(v, [[0, 1, 2]], 0.1)
    withdeg = sample_mesh(v, [[0, 1, 2], [1, 1, 1]], 0.1)
    # the degenerate face contributes one zero-length edge (1, 1): vertex 1
    # once more, in its sorted-edge slot after the edges of vertex 0
    expect = np.concatenate([base, v[1:2]])
    assert len(withdeg) == len(expect)
    assert np.array_equal(np.sort(withdeg.view([("", np.float32)] * 3), axis=0),
                          np.sort(expect.view([("", np.float32)] * 3), axis=0))


def test_scene_file_relative_path(tmp_path, monkeypatch):
    """A relative geometry path that does not open from the working
    directory is taken from the scene file's directory."""
    g = load_golden("geometry_dfsph_cup")
    raw = json.loads(json.dumps(g["scene"]))
    raw["Boundary"][0]["geometry"][0]["path"] = "cup.obj"
    scene_dir = tmp_path / "scene"
    scene_dir.mkdir()
    shutil.copy(os.path.join(GOLDEN, "cup.obj"), scene_dir / "cup.obj")
    (scene_dir / "s.json").write_text(json.dumps(raw))
    elsewhere = tmp_path / "cwd"
    elsewhere.mkdir()
    monkeypatch.chdir(elsewhere)
    b = Scene.load(str(scene_dir / "s.json")).boundary()
    assert np.array_equal(b, g["bpos"])
    with pytest.raises(SphError) as e:  # text has no file to resolve against
        Scene.from_dict(raw)
    assert e.value.code == -8
