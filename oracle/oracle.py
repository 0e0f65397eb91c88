"""ctypes binding of the CPU oracle (oracle/sph_oracle.cpp). Test
infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it, as the checker."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libsph2o_oracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} missing: run make -C oracle oracle")
        L = C.CDLL(LIB)
        P, D, F, U = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_uint)
        L.sph_oracle_create.restype = P
        L.sph_oracle_create.argtypes = [C.c_void_p, C.c_int]
        L.sph_oracle_set_fluid.argtypes = [P, C.c_uint, F, F]
        L.sph_oracle_set_boundary.argtypes = [P, C.c_uint, F]
        L.sph_oracle_init.argtypes = [P]
        L.sph_oracle_add_cube.argtypes = [P, F, F, C.c_float, C.c_float]
        L.sph_oracle_step.argtypes = [P, C.c_int, D]
        L.sph_oracle_get_state.argtypes = [P, D, D, D]
        L.sph_oracle_get_boundary_volume.argtypes = [P, D]
        L.sph_oracle_phase.argtypes = [P, C.c_int, D]
        L.sph_oracle_neighbors.argtypes = [P, U, U, C.c_size_t, U, U, C.c_size_t, C.POINTER(C.c_size_t),
                                           C.POINTER(C.c_size_t)]
        L.sph_oracle_destroy.argtypes = [P]
        L.sph_oracle_wcsph_adjoint.argtypes = [P, C.c_double, C.c_double, C.c_uint, D, D, C.c_uint, D, C.c_int, D,
                                               D, D, D, D, D, D]
        L.sph_oracle_set_boundary_normals.argtypes = [P, C.c_uint, F, C.c_float, C.c_float]
        L.sph_oracle_boundary_state.argtypes = [P, D, D]
        L.sph_oracle_sample_mesh.argtypes = [F, C.c_uint, U, C.c_uint, C.c_float, F, F, F, C.c_size_t,
                                             C.POINTER(C.c_size_t)]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _u(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint))


class Oracle:
    """CPU restatement of the reference; fp64=False reproduces its FP32 build."""

    def __init__(self, desc, fluid, boundary, vel=None, fp64=False, cubes=(), boundary_normals=None):
        L = lib()
        self.h = L.sph_oracle_create(C.addressof(desc), 1 if fp64 else 0)
        x = np.ascontiguousarray(fluid, np.float32)
        b = np.ascontiguousarray(boundary, np.float32).reshape(-1, 3)
        v = None if vel is None else np.ascontiguousarray(vel, np.float32)
        self.nf, self.nb = x.shape[0], b.shape[0]
        L.sph_oracle_set_fluid(self.h, self.nf, _f(x), _f(v))
        L.sph_oracle_set_boundary(self.h, self.nb, _f(b))
        if boundary_normals is not None:
            nrm, nfct, tfct = boundary_normals
            nrm = np.ascontiguousarray(nrm, np.float32).reshape(-1, 3)
            L.sph_oracle_set_boundary_normals(self.h, nrm.shape[0], _f(nrm), float(nfct), float(tfct))
        for mn, mx, nfct, tfct in cubes:
            L.sph_oracle_add_cube(self.h, _f(np.ascontiguousarray(mn, np.float32)),
                                  _f(np.ascontiguousarray(mx, np.float32)), float(nfct), float(tfct))
        L.sph_oracle_init(self.h)

    def step(self, n=1):
        st = np.zeros((n, 6), np.float64)
        lib().sph_oracle_step(self.h, n, _d(st))
        return st

    def state(self):
        x = np.zeros((self.nf, 3))
        v = np.zeros((self.nf, 3))
        r = np.zeros(self.nf)
        lib().sph_oracle_get_state(self.h, _d(x), _d(v), _d(r))
        return x, v, r

    def boundary_volume(self):
        out = np.zeros(self.nb)
        lib().sph_oracle_get_boundary_volume(self.h, _d(out))
        return out

    def boundary_state(self):
        """(densities, pressures) of PCISPH boundary particles, last computed."""
        d = np.zeros(self.nb)
        p = np.zeros(self.nb)
        lib().sph_oracle_boundary_state(self.h, _d(d), _d(p))
        return d, p

    def phase(self, phase):
        vec = phase in (2, 4)
        out = np.zeros((self.nf, 3) if vec else self.nf)
        lib().sph_oracle_phase(self.h, phase, _d(out))
        return out

    def neighbors(self):
        L = lib()
        tf, tb = C.c_size_t(), C.c_size_t()
        L.sph_oracle_neighbors(self.h, None, None, 0, None, None, 0, C.byref(tf), C.byref(tb))
        fo = np.zeros(self.nf + 1, np.uint32)
        bo = np.zeros(self.nf + 1, np.uint32)
        fi = np.zeros(max(1, tf.value), np.uint32)
        bi = np.zeros(max(1, tb.value), np.uint32)
        L.sph_oracle_neighbors(self.h, _u(fo), _u(fi), fi.size, _u(bo), _u(bi), bi.size, C.byref(tf), C.byref(tb))
        return fo, fi[: tf.value], bo, bi[: tb.value]

    def close(self):
        if self.h:
            lib().sph_oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sample_mesh(vertices, faces, max_distance, rotate=None, translate=None):
    """Regular triangle sampling of a mesh on the CPU (mesh_sampling.cpp);
    rotate / translate place the samples as sampleGeometry does."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
    r = None if rotate is None else np.ascontiguousarray(rotate, np.float32).reshape(3)
    t = None if translate is None else np.ascontiguousarray(translate, np.float32).reshape(3)
    n = C.c_size_t()
    L = lib()
    rc = L.sph_oracle_sample_mesh(_f(v), len(v), _u(f), len(f), float(max_distance), _f(r), _f(t), None, 0,
                                  C.byref(n))
    if rc != 0:
        raise ValueError(f"mesh sampling failed ({rc})")
    out = np.zeros((n.value, 3), np.float32)
    rc = L.sph_oracle_sample_mesh(_f(v), len(v), _u(f), len(f), float(max_distance), _f(r), _f(t), _f(out),
                                  n.value, C.byref(n))
    if rc != 0:
        raise ValueError(f"mesh sampling failed ({rc})")
    return out


def wcsph_adjoint(desc, x0, v0, boundary, nsteps, target, nu=None, k=None, grad=True):
    """FP64 WCSPH run + adjoint (oracle/wcsph_adjoint.cpp). nu / k default to
    the description's viscosity / stiffness. Returns a dict with the loss,
    the final positions and, when grad, dL/dx0, dL/dv0, dL/dnu, dL/dk."""
    L = lib()
    x0 = np.ascontiguousarray(x0, np.float64).reshape(-1, 3)
    v0 = np.ascontiguousarray(v0, np.float64).reshape(-1, 3)
    b = np.ascontiguousarray(boundary, np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(target, np.float64).reshape(-1, 3)
    n = x0.shape[0]
    loss = C.c_double()
    xo = np.zeros((n, 3))
    gx = np.zeros((n, 3)) if grad else None
    gv = np.zeros((n, 3)) if grad else None
    gnu, gk = C.c_double(), C.c_double()
    nu = float(desc.viscosity) if nu is None else float(nu)
    k = float(desc.stiffness) if k is None else float(k)
    rc = L.sph_oracle_wcsph_adjoint(C.addressof(desc), nu, k, n, _d(x0), _d(v0), b.shape[0], _d(b), int(nsteps),
                                    _d(t), C.byref(loss), _d(xo), _d(gx) if grad else None,
                                    _d(gv) if grad else None, C.byref(gnu), C.byref(gk))
    if rc != 0:
        raise RuntimeError(f"sph_oracle_wcsph_adjoint failed: {rc}")
    out = {"loss": loss.value, "x": xo}
    if grad:
        out.update(x0=gx, v0=gv, viscosity=gnu.value, stiffness=gk.value)
    return out
