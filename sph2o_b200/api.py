"""ctypes binding of the C ABI in include/sph2o_cuda.h.

This is the binding a Python caller (tests, bench.py) uses; it adds no
computation of its own. The CUDA library must have been built in-tree
(`python -m sph2o_b200.build`); loading fails loudly if it is missing.

    from sph2o_b200.api import Scene, Simulation
    sim = Simulation.from_scene(Scene.load("scene.json"))
    stats = sim.step(10)
    pos, vel, rho = sim.state()
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SPH2O_LIBRARY") or os.path.join(HERE, "libsph2o_cuda.so")

SPH_OK = 0
STATUS = {
    0: "SPH_OK", -1: "SPH_ERR_ARG", -2: "SPH_ERR_CUDA", -3: "SPH_ERR_NAN",
    -4: "SPH_ERR_NEIGHBOR_OVERFLOW", -5: "SPH_ERR_TIMEOUT", -6: "SPH_ERR_STATE",
    -7: "SPH_ERR_NO_DEVICE", -8: "SPH_ERR_IO", -9: "SPH_ERR_CAPACITY",
}
PHASE_DENSITY, PHASE_ALPHA, PHASE_NONPRESSURE_ACC, PHASE_PRESSURE, PHASE_PRESSURE_ACC = range(5)
(OPT_CUDA_GRAPHS, OPT_CELL_ORDER, OPT_SOLVER_OCCUPANCY, OPT_PASS_BLOCK, OPT_SOLVER_LANES, OPT_POSITION_RESIDUAL,
 OPT_LIST_STAGED) = range(7)
TUNE_COUNT = 4
PROF_NAMES = ["sort", "lists", "density", "normals", "forces", "density_solve", "divergence_solve",
              "pressure_solve"]
PROF_COUNT = len(PROF_NAMES)


class SceneDesc(C.Structure):
    _fields_ = [
        ("simulation_method", C.c_int), ("boundary_method", C.c_int), ("viscosity_method", C.c_int),
        ("surface_tension_method", C.c_int), ("adhesion_method", C.c_int),
        ("particle_radius", C.c_float), ("density0", C.c_float), ("gravity", C.c_float * 3),
        ("time_step", C.c_float), ("min_time_step", C.c_float), ("max_time_step", C.c_float),
        ("fps", C.c_float), ("start_time", C.c_float), ("end_time", C.c_float),
        ("stiffness", C.c_float), ("gamma", C.c_float),
        ("eta", C.c_float), ("eta_v", C.c_float), ("cfl_factor", C.c_float),
        ("min_iterations", C.c_uint), ("max_iterations", C.c_uint),
        ("min_iterations_v", C.c_uint), ("max_iterations_v", C.c_uint),
        ("viscosity", C.c_float), ("boundary_viscosity", C.c_float),
        ("surface_tension", C.c_float), ("adhesion", C.c_float),
        ("domain_min", C.c_float * 3), ("domain_max", C.c_float * 3), ("flags", C.c_uint),
    ]


class EmitterDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int), ("num_particles", C.c_uint), ("position", C.c_float * 3), ("rotation", C.c_float * 4),
        ("velocity", C.c_float), ("start_time", C.c_float), ("width", C.c_float), ("height", C.c_float),
        ("spacing", C.c_float),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("avg_density_error", C.c_double), ("avg_divergence_error", C.c_double),
        ("dt", C.c_float), ("max_velocity", C.c_float), ("iterations", C.c_uint), ("iterations_v", C.c_uint),
        ("total_iterations", C.c_ulonglong), ("total_iterations_v", C.c_ulonglong),
        ("steps", C.c_uint), ("neighbor_overflows", C.c_uint),
        ("device_ms", C.c_double), ("kernel_launches", C.c_ulonglong),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class SphError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m sph2o_b200.build`")
    L = C.CDLL(LIB_PATH)
    P, U, I, F = C.c_void_p, C.c_uint, C.c_int, C.POINTER(C.c_float)
    sigs = {
        "sph_select_device": (I, [I]),
        "sph_create": (I, [C.POINTER(SceneDesc), C.POINTER(P)]),
        "sph_set_fluid": (I, [P, U, F, F]),
        "sph_set_boundary": (I, [P, U, F]),
        "sph_init": (I, [P]),
        "sph_step": (I, [P, I, C.POINTER(StepStats)]),
        "sph_step_async": (I, [P, I]),
        "sph_sync": (I, [P, C.POINTER(StepStats)]),
        "sph_get_state": (I, [P, F, F, F]),
        "sph_set_state": (I, [P, F, F]),
        "sph_get_boundary_volume": (I, [P, F]),
        "sph_get_time": (I, [P, C.POINTER(C.c_double), F]),
        "sph_set_time": (I, [P, C.c_double, C.c_float]),
        "sph_num_fluid": (U, [P]),
        "sph_num_boundary": (U, [P]),
        "sph_last_error": (C.c_char_p, [P]),
        "sph_global_error": (C.c_char_p, []),
        "sph_destroy": (I, [P]),
        "sph_compute_phase": (I, [P, I, F]),
        "sph_debug_neighbors": (I, [P, C.POINTER(U), C.POINTER(U), C.c_size_t, C.POINTER(U), C.POINTER(U),
                                    C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
        "sph_debug_barrier_timeout": (I, [P]),
        "sph_set_option": (I, [P, I, I]),
        "sph_get_option": (I, [P, I, C.POINTER(I)]),
        "sph_autotune": (I, [P, I, C.c_char_p, C.POINTER(I)]),
        "sph_profile_enable": (I, [P, I]),
        "sph_profile_read": (I, [P, C.POINTER(C.c_double), C.POINTER(C.c_ulonglong)]),
        "sph_batch_create": (I, [C.POINTER(SceneDesc), U, C.POINTER(P)]),
        "sph_batch_set_scene": (I, [P, U, U, F, F, U, F]),
        "sph_batch_num_scenes": (U, [P]),
        "sph_batch_scene_range": (I, [P, U, C.POINTER(U), C.POINTER(U)]),
        "sph_batch_scene_stats": (I, [P, U, C.POINTER(StepStats)]),
        "sph_scene_load": (I, [C.c_char_p, C.POINTER(P)]),
        "sph_scene_parse": (I, [C.c_char_p, C.POINTER(P)]),
        "sph_scene_get_desc": (I, [P, C.POINTER(SceneDesc)]),
        "sph_scene_num_fluid": (U, [P]),
        "sph_scene_num_boundary": (U, [P]),
        "sph_scene_get_fluid": (I, [P, F, F]),
        "sph_scene_get_boundary": (I, [P, F]),
        "sph_scene_error": (C.c_char_p, []),
        "sph_scene_free": (None, [P]),
        "sph_create_from_scene": (I, [P, C.POINTER(P)]),
        "sph_add_emitter": (I, [P, C.POINTER(EmitterDesc)]),
        "sph_add_cube_boundary": (I, [P, F, F, C.c_float, C.c_float]),
        "sph_scene_num_cube_boundaries": (U, [P]),
        "sph_scene_get_cube_boundary": (I, [P, U, F, F, F, F]),
        "sph_get_num_active": (I, [P, C.POINTER(U)]),
        "sph_scene_num_emitters": (U, [P]),
        "sph_scene_get_emitter": (I, [P, U, C.POINTER(EmitterDesc)]),
        "sph_wcsph_forward": (I, [P, I, I, F, C.POINTER(C.c_double)]),
        "sph_wcsph_backward": (I, [P, F, F, F]),
        "sph_wcsph_grad_x0": (I, [P, F]),
        "sph_wcsph_timing": (I, [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "sph_load_obj": (I, [C.c_char_p, F, F, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(U), C.c_size_t,
                             C.POINTER(C.c_size_t)]),
        "sph_sample_mesh": (I, [F, U, C.POINTER(U), U, C.c_float, F, C.c_size_t, C.POINTER(C.c_size_t)]),
        "sph_set_boundary_normals": (I, [P, U, F, C.c_float, C.c_float]),
        "sph_get_boundary_state": (I, [P, F, F]),
        "sph_scene_get_boundary_normals": (I, [P, F, F, F]),
        "sph_sample_geometry": (I, [C.c_char_p, C.c_float, F, F, F, F, C.c_size_t, C.POINTER(C.c_size_t)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


def _uptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint)) if a is not None else None


def select_device(device: int):
    rc = lib().sph_select_device(int(device))
    if rc != SPH_OK:
        raise SphError(rc, lib().sph_global_error().decode())


def _two_call(call):
    """Runs a sampler entry point twice: once for the count, once to fill."""
    n = C.c_size_t()
    rc = call(None, 0, C.byref(n))
    if rc != SPH_OK:
        raise SphError(rc, lib().sph_scene_error().decode())
    out = np.zeros((n.value, 3), np.float32)
    rc = call(_fptr(out), n.value, C.byref(n))
    if rc != SPH_OK:
        raise SphError(rc, lib().sph_scene_error().decode())
    return out


def load_obj(path, scale=None):
    """Triangulated OBJ file -> (vertices (V, 3) float32, faces (F, 3) uint32, 0-based)."""
    s = None if scale is None else np.ascontiguousarray(scale, np.float32).reshape(3)
    nv, nf = C.c_size_t(), C.c_size_t()
    rc = lib().sph_load_obj(os.fsencode(path), _fptr(s), None, 0, C.byref(nv), None, 0, C.byref(nf))
    if rc != SPH_OK:
        raise SphError(rc, lib().sph_scene_error().decode())
    v = np.zeros((nv.value, 3), np.float32)
    f = np.zeros((nf.value, 3), np.uint32)
    rc = lib().sph_load_obj(os.fsencode(path), _fptr(s), _fptr(v), nv.value, C.byref(nv), _uptr(f), nf.value,
                            C.byref(nf))
    if rc != SPH_OK:
        raise SphError(rc, lib().sph_scene_error().decode())
    return v, f


def sample_mesh(vertices, faces, max_distance):
    """Regular triangle sampling of a mesh on the current GPU
    (RegularTriangleSampling::sampleMesh): vertices (V, 3) float, faces
    (F, 3) 0-based indices -> samples (S, 3)."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
    return _two_call(lambda out, cap, n: lib().sph_sample_mesh(_fptr(v), len(v), _uptr(f), len(f),
                                                                float(max_distance), out, cap, n))


def sample_geometry(path, max_distance, scale=None, translate=None, rotate=None):
    """OBJ file -> boundary samples on the current GPU
    (AkinciBoundaryObject::sampleGeometry): scaled, sampled, turned by
    glm::rotate about x, y, z (radians), translated."""
    vec = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).reshape(3)
    s, t, r = vec(scale), vec(translate), vec(rotate)
    return _two_call(lambda out, cap, n: lib().sph_sample_geometry(os.fsencode(path), float(max_distance), _fptr(s),
                                                                    _fptr(t), _fptr(r), out, cap, n))


class Scene:
    """Host-side scene: SPH2O JSON schema -> parameters + particles."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    @classmethod
    def load(cls, path):
        h = C.c_void_p()
        rc = lib().sph_scene_load(os.fsencode(path), C.byref(h))
        if rc != SPH_OK:
            raise SphError(rc, lib().sph_scene_error().decode())
        return cls(h.value)

    @classmethod
    def from_dict(cls, d):
        h = C.c_void_p()
        rc = lib().sph_scene_parse(json.dumps(d).encode(), C.byref(h))
        if rc != SPH_OK:
            raise SphError(rc, lib().sph_scene_error().decode())
        return cls(h.value)

    def desc(self):
        d = SceneDesc()
        lib().sph_scene_get_desc(self._h, C.byref(d))
        return d

    def fluid(self):
        n = lib().sph_scene_num_fluid(self._h)
        x = np.zeros((n, 3), np.float32)
        v = np.zeros((n, 3), np.float32)
        lib().sph_scene_get_fluid(self._h, _fptr(x), _fptr(v))
        return x, v

    def cube_boundaries(self):
        """[(min, max, normal_fct, tangential_fct)] of a boundaryMethod-0 scene."""
        out = []
        for k in range(lib().sph_scene_num_cube_boundaries(self._h)):
            mn = np.zeros(3, np.float32)
            mx = np.zeros(3, np.float32)
            nf, tf = C.c_float(), C.c_float()
            lib().sph_scene_get_cube_boundary(self._h, k, _fptr(mn), _fptr(mx), C.byref(nf), C.byref(tf))
            out.append((mn, mx, nf.value, tf.value))
        return out

    def emitters(self):
        out = []
        for k in range(lib().sph_scene_num_emitters(self._h)):
            e = EmitterDesc()
            lib().sph_scene_get_emitter(self._h, k, C.byref(e))
            out.append(e)
        return out

    def boundary_normals(self):
        """(normals (nb, 3), normal_fct, tangential_fct) of a boundaryMethod-1
        scene, else None."""
        if self.desc().boundary_method != 1:
            return None
        n = lib().sph_scene_num_boundary(self._h)
        nrm = np.zeros((n, 3), np.float32)
        nf, tf = C.c_float(), C.c_float()
        lib().sph_scene_get_boundary_normals(self._h, _fptr(nrm), C.byref(nf), C.byref(tf))
        return nrm, nf.value, tf.value

    def boundary(self):
        n = lib().sph_scene_num_boundary(self._h)
        b = np.zeros((n, 3), np.float32)
        lib().sph_scene_get_boundary(self._h, _fptr(b))
        return b

    def close(self):
        if self._h:
            lib().sph_scene_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Simulation:
    """One GPU simulation context (sph_ctx)."""

    def __init__(self, desc: SceneDesc, fluid, boundary, vel=None, emitters=(), cubes=(), boundary_normals=None,
                 options=None):
        """boundary_normals: (normals (nb, 3), normal_fct, tangential_fct) for
        the PCISPH boundary method (boundary_method 1); options: {option:
        value} set before sph_init (e.g. OPT_POSITION_RESIDUAL)."""
        L = lib()
        h = C.c_void_p()
        rc = L.sph_create(C.byref(desc), C.byref(h))
        if rc != SPH_OK:
            raise SphError(rc, L.sph_global_error().decode())
        self._h = h
        self.desc = desc
        x = np.ascontiguousarray(fluid, np.float32).reshape(-1, 3)
        v = None if vel is None else np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        b = np.ascontiguousarray(boundary, np.float32).reshape(-1, 3)
        self._check(L.sph_set_fluid(h, x.shape[0], _fptr(x), _fptr(v)))
        self._check(L.sph_set_boundary(h, b.shape[0], _fptr(b)))
        if boundary_normals is not None:
            nrm, nfct, tfct = boundary_normals
            nrm = np.ascontiguousarray(nrm, np.float32).reshape(-1, 3)
            self._check(L.sph_set_boundary_normals(h, nrm.shape[0], _fptr(nrm), float(nfct), float(tfct)))
        for mn, mx, nfct, tfct in cubes:
            mn = np.ascontiguousarray(mn, np.float32)
            mx = np.ascontiguousarray(mx, np.float32)
            self._check(L.sph_add_cube_boundary(h, _fptr(mn), _fptr(mx), float(nfct), float(tfct)))
        for e in emitters:
            self._check(L.sph_add_emitter(h, C.byref(e)))
        for opt, val in (options or {}).items():
            self._check(L.sph_set_option(h, int(opt), int(val)))
        self._check(L.sph_init(h))
        self.nf, self.nb = L.sph_num_fluid(h), b.shape[0]

    @classmethod
    def from_scene(cls, scene: Scene, vel=None, options=None):
        x, v = scene.fluid()
        return cls(scene.desc(), x, scene.boundary(), v if vel is None else vel, emitters=scene.emitters(),
                   cubes=scene.cube_boundaries(), boundary_normals=scene.boundary_normals(), options=options)

    def num_active(self):
        n = C.c_uint()
        self._check(lib().sph_get_num_active(self._h, C.byref(n)))
        return n.value

    def _check(self, rc):
        if rc != SPH_OK:
            raise SphError(rc, lib().sph_last_error(self._h).decode())

    def step(self, n=1):
        s = StepStats()
        self._check(lib().sph_step(self._h, int(n), C.byref(s)))
        return s.as_dict()

    def step_async(self, n=1):
        self._check(lib().sph_step_async(self._h, int(n)))

    def sync(self):
        s = StepStats()
        self._check(lib().sph_sync(self._h, C.byref(s)))
        return s.as_dict()

    def boundary_state(self):
        """(densities, pressures) of PCISPH boundary particles, caller order."""
        d = np.zeros(self.nb, np.float32)
        p = np.zeros(self.nb, np.float32)
        self._check(lib().sph_get_boundary_state(self._h, _fptr(d), _fptr(p)))
        return d, p

    def state(self):
        x = np.zeros((self.nf, 3), np.float32)
        v = np.zeros((self.nf, 3), np.float32)
        r = np.zeros(self.nf, np.float32)
        self._check(lib().sph_get_state(self._h, _fptr(x), _fptr(v), _fptr(r)))
        return x, v, r

    def set_state(self, x=None, v=None):
        x = None if x is None else np.ascontiguousarray(x, np.float32)
        v = None if v is None else np.ascontiguousarray(v, np.float32)
        self._check(lib().sph_set_state(self._h, _fptr(x), _fptr(v)))

    def boundary_volume(self):
        out = np.zeros(self.nb, np.float32)
        self._check(lib().sph_get_boundary_volume(self._h, _fptr(out)))
        return out

    def time(self):
        t = C.c_double()
        dt = C.c_float()
        self._check(lib().sph_get_time(self._h, C.byref(t), C.byref(dt)))
        return t.value, dt.value

    def set_time(self, time, dt):
        self._check(lib().sph_set_time(self._h, float(time), float(dt)))

    def phase(self, phase):
        vec = phase in (PHASE_NONPRESSURE_ACC, PHASE_PRESSURE_ACC)
        out = np.zeros((self.nf, 3) if vec else self.nf, np.float32)
        self._check(lib().sph_compute_phase(self._h, int(phase), _fptr(out)))
        return out

    def set_option(self, option, value):
        self._check(lib().sph_set_option(self._h, int(option), int(value)))

    def get_option(self, option):
        v = C.c_int()
        self._check(lib().sph_get_option(self._h, int(option), C.byref(v)))
        return v.value

    def autotune(self, trial_steps=3, cache_path=None):
        cfg = (C.c_int * TUNE_COUNT)()
        path = os.fsencode(cache_path) if cache_path else None
        self._check(lib().sph_autotune(self._h, int(trial_steps), path, cfg))
        return {"cell_order": cfg[0], "solver_occupancy": cfg[1], "pass_block": cfg[2], "solver_lanes": cfg[3]}

    def profile(self, enable=True):
        self._check(lib().sph_profile_enable(self._h, 1 if enable else 0))

    def profile_read(self):
        ms = (C.c_double * PROF_COUNT)()
        n = (C.c_ulonglong * PROF_COUNT)()
        self._check(lib().sph_profile_read(self._h, ms, n))
        return {PROF_NAMES[i]: {"ms": ms[i], "launches": n[i]} for i in range(PROF_COUNT)}

    def wcsph_forward(self, nsteps, target, ckpt_every=50):
        """Differentiable WCSPH run from the current state; returns the loss
        (1/N) sum |x_i(T) - target_i|^2."""
        t = np.ascontiguousarray(target, np.float32).reshape(-1, 3)
        loss = C.c_double()
        self._check(lib().sph_wcsph_forward(self._h, int(nsteps), int(ckpt_every), _fptr(t), C.byref(loss)))
        return loss.value

    def wcsph_backward(self, want_x0=False):
        """Gradients of the last wcsph_forward's loss: dL/dv0 (n x 3), dL/dviscosity,
        dL/dstiffness (and dL/dx0 when want_x0)."""
        gv = np.zeros((self.nf, 3), np.float32)
        dvisc = C.c_float()
        dk = C.c_float()
        self._check(lib().sph_wcsph_backward(self._h, _fptr(gv), C.byref(dvisc), C.byref(dk)))
        out = {"v0": gv, "viscosity": dvisc.value, "stiffness": dk.value}
        if want_x0:
            gx = np.zeros((self.nf, 3), np.float32)
            self._check(lib().sph_wcsph_grad_x0(self._h, _fptr(gx)))
            out["x0"] = gx
        return out

    def wcsph_timing(self):
        f, b = C.c_double(), C.c_double()
        self._check(lib().sph_wcsph_timing(self._h, C.byref(f), C.byref(b)))
        return f.value, b.value

    def neighbors(self):
        """CSR neighbour sets (caller order): (f_off, f_idx, b_off, b_idx)."""
        L = lib()
        tf, tb = C.c_size_t(), C.c_size_t()
        self._check(L.sph_debug_neighbors(self._h, None, None, 0, None, None, 0, C.byref(tf), C.byref(tb)))
        f_off = np.zeros(self.nf + 1, np.uint32)
        b_off = np.zeros(self.nf + 1, np.uint32)
        f_idx = np.zeros(max(tf.value, 1), np.uint32)
        b_idx = np.zeros(max(tb.value, 1), np.uint32)
        self._check(L.sph_debug_neighbors(self._h, _uptr(f_off), _uptr(f_idx), f_idx.size, _uptr(b_off),
                                          _uptr(b_idx), b_idx.size, C.byref(tf), C.byref(tb)))
        return f_off, f_idx[: tf.value], b_off, b_idx[: tb.value]

    def close(self):
        if getattr(self, "_h", None):
            lib().sph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch(Simulation):
    """Many independent scenes stepped together (sph_batch_*)."""

    def __init__(self, scenes, vels=None):
        L = lib()
        descs = (SceneDesc * len(scenes))(*[sc.desc() for sc in scenes])
        h = C.c_void_p()
        rc = L.sph_batch_create(descs, len(scenes), C.byref(h))
        if rc != SPH_OK:
            raise SphError(rc, L.sph_global_error().decode())
        self._h = h
        self.desc = descs[0]
        self.nscenes = len(scenes)
        for s, sc in enumerate(scenes):
            x, v = sc.fluid()
            if vels is not None and vels[s] is not None:
                v = np.ascontiguousarray(vels[s], np.float32)
            b = sc.boundary()
            self._check(L.sph_batch_set_scene(h, s, x.shape[0], _fptr(x), _fptr(v), b.shape[0], _fptr(b)))
        self._check(L.sph_init(h))
        self.nf = L.sph_num_fluid(h)
        self.nb = L.sph_num_boundary(h)
        self.ranges = []
        for s in range(self.nscenes):
            b0, e0 = C.c_uint(), C.c_uint()
            L.sph_batch_scene_range(h, s, C.byref(b0), C.byref(e0))
            self.ranges.append((b0.value, e0.value))

    def scene_stats(self, scene):
        st = StepStats()
        self._check(lib().sph_batch_scene_stats(self._h, int(scene), C.byref(st)))
        return st.as_dict()

    def scene_state(self, scene):
        x, v, r = self.state()
        b0, e0 = self.ranges[scene]
        return x[b0:e0], v[b0:e0], r[b0:e0]
