"""OBJ "geometry" boundaries on the GPU: the device sampler and the scene
loader against the boundary particles the SPH2O reference generated
(golden fixtures, bit for bit), and against the CPU oracle on larger
random meshes; relative paths, the two-call convention and its errors."""
import ctypes as C
import json
import math
import os
import shutil

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oracle import oracle as O
from sph2o_b200.api import Scene, SphError, lib, load_obj, sample_geometry, sample_mesh
from test_geometry import GEOMETRY_GOLDEN, ROT, read_obj, scene_geometries

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name", GEOMETRY_GOLDEN)
def test_scene_boundary_bit_exact(name):
    g = load_golden(name)
    b = Scene.from_dict(g["scene"]).boundary()
    assert b.shape == g["bpos"].shape
    assert np.array_equal(bits(b), bits(g["bpos"]))


@pytest.mark.parametrize("name", GEOMETRY_GOLDEN)
def test_geometry_entry_point_matches_reference(name):
    g = load_golden(name)
    geo = np.concatenate([sample_geometry(p, d, rotate=ROT) for p, d in scene_geometries(g["scene"])])
    assert np.array_equal(bits(geo), bits(g["bpos"][-len(geo):]))


def random_mesh(seed, nv, nf, extent=1.0):
    rng = np.random.default_rng(seed)
    v = (rng.random((nv, 3)) * extent).astype(np.float32)
    f = np.stack([rng.choice(nv, 3, replace=False) for _ in range(nf)]).astype(np.uint32)
    return v, f


def sphere_mesh(n_lat=60, n_lon=120, radius=0.5):
    """UV sphere: many small, unequal triangles and shared edges."""
    v = [(0.0, 0.0, radius)]
    for i in range(1, n_lat):
        t = math.pi * i / n_lat
        for j in range(n_lon):
            p = 2 * math.pi * j / n_lon
            v.append((radius * math.sin(t) * math.cos(p), radius * math.sin(t) * math.sin(p), radius * math.cos(t)))
    v.append((0.0, 0.0, -radius))
    ring = lambda i, j: 1 + (i - 1) * n_lon + j % n_lon
    f = [(0, ring(1, j), ring(1, j + 1)) for j in range(n_lon)]
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            f.append((ring(i, j), ring(i + 1, j), ring(i + 1, j + 1)))
            f.append((ring(i, j), ring(i + 1, j + 1), ring(i, j + 1)))
    last = len(v) - 1
    f += [(ring(n_lat - 1, j + 1), ring(n_lat - 1, j), last) for j in range(n_lon)]
    return np.array(v, np.float32), np.array(f, np.uint32)


@pytest.mark.parametrize("case", ["random_small", "random_large", "sphere", "sphere_placed"])
def test_device_sampler_equals_oracle(case):
    if case == "random_small":
        v, f = random_mesh(1, 40, 60)
        d, rot, tr = 0.03, None, None
    elif case == "random_large":
        v, f = random_mesh(2, 3000, 6000, extent=2.0)
        d, rot, tr = 0.07, None, None
    else:
        v, f = sphere_mesh()
        d = 0.004
        rot, tr = ((0.3, -1.1, 2.0), (0.5, -0.25, 1.0)) if case == "sphere_placed" else (None, None)
    ref = O.sample_mesh(v, f, d, rotate=rot, translate=tr)
    if rot is None:
        got = sample_mesh(v, f, d)
    else:
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"sph2o_sphere_{os.getpid()}.obj")
        with open(path, "w") as fh:
            fh.writelines("v %.9g %.9g %.9g\n" % tuple(float(c) for c in p) for p in v)
            fh.writelines("f %d %d %d\n" % tuple(int(i) + 1 for i in t) for t in f)
        try:
            vv, ff = load_obj(path)
            assert np.array_equal(vv, v) and np.array_equal(ff, f)
            got = sample_geometry(path, d, rotate=rot, translate=tr)
        finally:
            os.remove(path)
    assert len(ref) > len(v)
    assert got.shape == ref.shape
    assert np.array_equal(bits(got), bits(ref))


def test_two_call_convention_and_errors(tmp_path):
    v, f = read_obj(os.path.join(GOLDEN, "cup.obj"))
    v = np.ascontiguousarray(v)
    n = C.c_size_t()
    L = lib()
    fp = v.ctypes.data_as(C.POINTER(C.c_float))
    up = f.ctypes.data_as(C.POINTER(C.c_uint))
    assert L.sph_sample_mesh(fp, len(v), up, len(f), 0.05, None, 0, C.byref(n)) == 0
    small = np.zeros((n.value - 1, 3), np.float32)
    assert L.sph_sample_mesh(fp, len(v), up, len(f), 0.05, small.ctypes.data_as(C.POINTER(C.c_float)),
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
    with pytest.raises(SphError) as e:  # about 4e10 samples: refused before any is written
        sample_mesh(v * np.float32(1000.0), f, 0.01)
    assert e.value.code == -9
    assert sample_mesh(v, np.zeros((0, 3), np.uint32), 0.05).shape == v.shape


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
    assert np.array_equal(bits(b), bits(g["bpos"]))
    with pytest.raises(SphError) as e:  # text has no file to resolve against
        Scene.from_dict(raw)
    assert e.value.code == -8
