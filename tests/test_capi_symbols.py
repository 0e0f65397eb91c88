"""The shared library loads without a GPU and exports every function that
include/*.h declares."""
import ctypes
import os
import re

from conftest import ROOT
from sph2o_b200.api import LIB_PATH


def declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(inc, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(sph_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_exported():
    lib = ctypes.CDLL(LIB_PATH)
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_error_is_reported():
    """Without a GPU, sph_create fails with SPH_ERR_NO_DEVICE (never a crash)."""
    import torch
    if torch.cuda.is_available():
        return
    from sph2o_b200 import scenes as S
    from sph2o_b200.api import Scene, Simulation, SphError
    sc = Scene.from_dict(S.small())
    try:
        Simulation.from_scene(sc)
    except SphError as e:
        assert e.code == -7
    else:
        raise AssertionError("expected SPH_ERR_NO_DEVICE")
