"""Test configuration.

Markers:
  gpu  -- needs a CUDA device (run with `pytest -m gpu` on a B200)
Everything unmarked runs on a CPU-only machine: the oracle against the golden
fixtures, the host scene loader, the C ABI symbol table and the multi-process
host logic (gloo).
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


@pytest.fixture(scope="session", autouse=True)
def built_library():
    """Build the in-tree CUDA library if it is missing or stale (nvcc
    cross-compiles without a GPU). On a box without nvcc the prebuilt .so
    that travels with the tree is used as is."""
    from sph2o_b200 import build

    try:
        build.nvcc_path()
    except RuntimeError:
        return build.LIB
    return build.build()


def golden_names():
    """Fixed-particle golden scenes (the emitter scenes have their own tests)."""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and not f.startswith("emitter_"))


def emitter_golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("emitter_"))


def load_golden(name):
    """Fixture arrays; the scene's relative OBJ geometry paths point into
    the golden directory."""
    from sph2o_b200.scenes import resolve_geometry_paths

    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    g["scene"] = resolve_geometry_paths(json.loads(str(g["scene"])), GOLDEN)
    return g


def rel_err(a, b):
    """max |a - b| / max |b| (norm-wise relative error)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = max(float(np.max(np.abs(b))), 1e-30)
    return float(np.max(np.abs(a - b))) / den


def csr_rows(off, idx):
    return [idx[off[i]:off[i + 1]] for i in range(len(off) - 1)]
