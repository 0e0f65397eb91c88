"""Seeded synthetic scenes in SPH2O's scene-JSON schema.

The schema is the one SPH2O's loader reads (src/SPH2O/SceneLoader.cpp:40-209):
"Configuration", "Fluid" {"viscosityMethod", "surfaceTensionMethod",
"adhesionMethod", "FluidModel": [...]}, "Boundary": [{"box", "sphere",
"geometry"}]. Every boundary carries "sphere" and "geometry" lists even when
empty, because the reference indexes both keys unconditionally
(SceneLoader.cpp:161-162). Two extra "Configuration" keys, "jitter" and
"jitterSeed", describe the seeded lattice perturbation (host/scene_rng.h);
the reference loader ignores them.

All real values are rounded to float32 before they are written, so the FP32
and FP64 builds of the reference read the same numbers.

Workloads (fluid kept at the stated particle counts; tanks enlarged where the
fluid would otherwise touch or cross the walls, fluid placed 4r from walls):
  dam_break_wcsph_8k     WCSPH, 20^3 lattice, r=0.025, Tait k=400 gamma=7,
                         artificial viscosity 0.01, dt=1e-4 fixed
  dam_break_dfsph_125k   DFSPH + Akinci surface tension 0.05, 50^3, r=0.01
  double_dam_break_1m    DFSPH or PCISPH, 2 x 100x100x50 blocks, r=0.005,
                         4x2x2 m tank with a sphere obstacle R=0.2
  adjoint_wcsph_32k      WCSPH, 32^3, r=0.02 (with adjoint_problem: seeded
                         initial velocities and target block)
"""
from __future__ import annotations

import json
import math

import numpy as np

WCSPH, PCISPH, DFSPH = 0, 1, 2
BOUNDARY_CUBE, BOUNDARY_PCISPH, BOUNDARY_AKINCI = 0, 1, 2
VISC_STANDARD, VISC_ARTIFICIAL, VISC_XSPH = 0, 1, 2
SURFACE_TENSION_AKINCI = 3
ADHESION_AKINCI = 4


def f32(x):
    """Round to float32 and return a Python float holding that exact value."""
    if isinstance(x, (list, tuple)):
        return [f32(v) for v in x]
    return float(np.float32(x))


def scene(
    *,
    method: int,
    radius: float,
    blocks,
    tank,
    spheres=(),
    gravity=(0.0, 0.0, -9.81),
    time_step=1e-4,
    min_time_step=1e-6,
    max_time_step=1e-3,
    fps=60.0,
    end_time=1000.0,
    stiffness=400.0,
    gamma=7.0,
    eta=1e-3,
    eta_v=1e-3,
    min_iterations=2,
    max_iterations=100,
    min_iterations_v=1,
    max_iterations_v=100,
    cfl=1.0,
    viscosity_method=VISC_ARTIFICIAL,
    viscosity=0.01,
    boundary_viscosity=0.0,
    surface_tension_method=-1,
    surface_tension=0.0,
    adhesion_method=-1,
    adhesion=0.0,
    density0=1000.0,
    jitter=0.01,
    seed=1,
    boundary_method=BOUNDARY_AKINCI,
):
    """Build one scene dict. `blocks` are (min, max) pairs; `tank` is (min, max)."""
    cfg = {
        "startTime": 0.0,
        "endTime": f32(end_time),
        "timeStep": f32(time_step),
        "fps": f32(fps),
        "minTimeStep": f32(min_time_step),
        "maxTimeStep": f32(max_time_step),
        "gravity": f32(list(gravity)),
        "particleRadius": f32(radius),
        "simulationMethod": int(method),
        "boundaryMethod": int(boundary_method),
        "cflFactor": f32(cfl),
        "jitter": f32(jitter),
        "jitterSeed": int(seed),
    }
    if method == WCSPH:
        cfg.update(stiffness=f32(stiffness), gamma=f32(gamma))
    elif method == PCISPH:
        cfg.update(eta=f32(eta), minIterations=int(min_iterations), maxIterations=int(max_iterations))
    else:
        cfg.update(
            eta=f32(eta),
            etaV=f32(eta_v),
            minIterations=int(min_iterations),
            maxIterations=int(max_iterations),
            minIterationsV=int(min_iterations_v),
            maxIterationsV=int(max_iterations_v),
        )
    fluid_model = {
        "density0": f32(density0),
        "viscosity": f32(viscosity),
        "boundaryViscosity": f32(boundary_viscosity),
        "surfaceTension": f32(surface_tension),
        "adhesion": f32(adhesion),
        "fluidBlocks": [{"min": f32(list(lo)), "max": f32(list(hi))} for lo, hi in blocks],
    }
    return {
        "Configuration": cfg,
        "Fluid": {
            "viscosityMethod": int(viscosity_method),
            "surfaceTensionMethod": int(surface_tension_method),
            "adhesionMethod": int(adhesion_method),
            "FluidModel": [fluid_model],
        },
        "Boundary": [
            {
                "box": [{"min": f32(list(tank[0])), "max": f32(list(tank[1]))}],
                "sphere": [{"pos": f32(list(c)), "radius": f32(rad)} for c, rad in spheres],
                "geometry": [],
            }
        ],
    }


def block(n, radius, lo):
    """Lattice block of n = (nx, ny, nz) particles at spacing 2r starting at lo.
    The max corner sits half a spacing beyond the last particle so that the
    reference's count floor((max - min) / 2r + 1e-5) (FluidObject.cpp:38) is n
    without depending on float rounding."""
    d = 2.0 * radius
    lo = [float(np.float32(v)) for v in lo]
    return (lo, [lo[k] + (n[k] + 0.5) * d for k in range(3)])


def dam_break_wcsph_8k(seed=1):
    r = 0.025
    return scene(
        method=WCSPH, radius=r, blocks=[block((20, 20, 20), r, (4 * r,) * 3)],
        tank=((0, 0, 0), (2.0, 1.2, 1.2)), time_step=1e-4, stiffness=400.0, gamma=7.0,
        viscosity=0.01, seed=seed,
    )


def dam_break_dfsph_125k(seed=2):
    r = 0.01
    return scene(
        method=DFSPH, radius=r, blocks=[block((50, 50, 50), r, (4 * r,) * 3)],
        tank=((0, 0, 0), (2.0, 1.08, 1.08)), time_step=1e-4, min_time_step=1e-6,
        max_time_step=1e-3, eta=1e-4, eta_v=1e-3, viscosity=0.01,
        surface_tension_method=SURFACE_TENSION_AKINCI, surface_tension=0.05, seed=seed,
    )


def double_dam_break_1m(method=DFSPH, seed=3):
    r = 0.005
    a = block((100, 100, 50), r, (4 * r, 4 * r, 4 * r))
    b = block((100, 100, 50), r, (4.0 - 4 * r - 1.0, 2.0 - 4 * r - 1.0, 4 * r))
    return scene(
        method=method, radius=r, blocks=[a, b], tank=((0, 0, 0), (4.0, 2.0, 2.0)),
        spheres=[((2.0, 1.0, 0.3), 0.2)], time_step=1e-4 if method == DFSPH else 5e-4,
        min_time_step=1e-6, max_time_step=1e-3,
        eta=1e-4 if method == DFSPH else 0.01, eta_v=1e-3, viscosity=0.01, seed=seed,
    )


def adjoint_wcsph_32k(seed=5):
    r = 0.02
    return scene(
        method=WCSPH, radius=r, blocks=[block((32, 32, 32), r, (4 * r,) * 3)],
        tank=((0, 0, 0), (2.5, 1.28 + 8 * r, 1.28 + 8 * r)), time_step=2e-4,
        stiffness=400.0, gamma=7.0, viscosity=0.01, seed=seed,
    )


def adjoint_problem(x0, seed_v=5, seed_t=6, sigma=0.1):
    """Initial velocities and target of the differentiable WCSPH workload:
    v0 ~ N(0, sigma^2) per component (seed_v) and the target = the initial
    block shifted by a seeded offset (seed_t) of 0.05-0.15 m in x and
    -0.05-0.05 m in y, z unchanged. Returns float32 arrays (n, 3)."""
    x0 = np.asarray(x0, np.float32)
    v0 = np.random.default_rng(seed_v).normal(0.0, sigma, x0.shape).astype(np.float32)
    rng = np.random.default_rng(seed_t)
    shift = np.array([rng.uniform(0.05, 0.15), rng.uniform(-0.05, 0.05), 0.0], np.float32)
    return v0, (x0 + shift).astype(np.float32)


def small(method=DFSPH, n=(10, 10, 10), radius=0.025, surface_tension=0.0,
          viscosity_method=VISC_ARTIFICIAL, viscosity=0.01, boundary_viscosity=0.0,
          adhesion=0.0, sphere=False, seed=11, **kw):
    """Small tank scene for parity tests: n lattice block at 4r inset in a tank
    2 x the block plus margins along x."""
    r = radius
    blk = block(n, r, (4 * r,) * 3)
    ext = [n[k] * 2 * r for k in range(3)]
    tank = ((0, 0, 0), (2 * ext[0] + 8 * r, ext[1] + 8 * r, ext[2] + 8 * r))
    spheres = [((ext[0] + 8 * r, 0.5 * tank[1][1], 4 * r + 0.25 * ext[2]), 0.15 * ext[2])] if sphere else []
    return scene(
        method=method, radius=r, blocks=[blk], tank=tank, spheres=spheres,
        viscosity_method=viscosity_method, viscosity=viscosity,
        boundary_viscosity=boundary_viscosity,
        surface_tension_method=SURFACE_TENSION_AKINCI if surface_tension else -1,
        surface_tension=surface_tension,
        adhesion_method=ADHESION_AKINCI if adhesion else -1, adhesion=adhesion,
        seed=seed, **kw,
    )


def with_emitter(scene_dict, *, etype=0, position, rotation=(1.0, 0.0, 0.0, 0.0), velocity=1.0, num_particles=100,
                 start_time=0.0, width=0.1, height=0.1, spacing=1.0):
    """Adds an emitter to the scene's fluid model (SceneLoader.cpp:128-143
    keys; rotation is the quaternion w, x, y, z)."""
    scene_dict["Fluid"]["FluidModel"][0].setdefault("emitters", []).append({
        "type": int(etype), "position": f32(list(position)), "rotation": f32(list(rotation)),
        "velocity": f32(velocity), "numParticles": int(num_particles), "startTime": f32(start_time),
        "width": f32(width), "height": f32(height), "spacing": f32(spacing)})
    return scene_dict


def emitter_scenes():
    """Small scenes with an emitter shooting along +x (local z turned by 90
    degrees about y) from the middle of the tank, emitting from t = 0."""
    q = (math.cos(math.pi / 4), 0.0, math.sin(math.pi / 4), 0.0)
    wc = small(method=WCSPH, n=(6, 6, 6), time_step=2e-4, seed=31)
    tank = wc["Boundary"][0]["box"][0]["max"]
    with_emitter(wc, etype=0, position=(0.35 * tank[0], 0.5 * tank[1], 0.5 * tank[2]), rotation=q, velocity=5.0,
                 num_particles=4 * 16, width=0.2, height=0.2, spacing=1.0)
    df = small(method=DFSPH, n=(6, 6, 6), time_step=5e-4, seed=32)
    tank = df["Boundary"][0]["box"][0]["max"]
    with_emitter(df, etype=1, position=(0.35 * tank[0], 0.5 * tank[1], 0.5 * tank[2]), rotation=q, velocity=4.0,
                 num_particles=3 * 19, width=0.11, spacing=1.2)
    return {"emitter_wcsph_square": wc, "emitter_dfsph_circle": df}


def cube_scenes():
    """Cube-boundary scenes (boundaryMethod 0: no boundary particles, the
    fluid is clamped into the box after every step). WCSPH: the block's last
    x layers start outside the box, so the first step clamps them. DFSPH: the
    block's bottom layer starts below the floor and the rest falls onto it."""
    r = 0.025
    wc = scene(method=WCSPH, radius=r, blocks=[block((8, 6, 6), r, (4 * r,) * 3)],
               tank=((0, 0, 0), (0.4, 1.0, 1.0)), time_step=2e-4, seed=41, boundary_method=BOUNDARY_CUBE)
    df = scene(method=DFSPH, radius=r, blocks=[block((6, 6, 6), r, (4 * r, 4 * r, -2 * r))],
               tank=((0, 0, 0), (1.0, 1.0, 1.0)), time_step=5e-4, seed=42, boundary_method=BOUNDARY_CUBE)
    return {"cube_wcsph_outside": wc, "cube_dfsph_floor": df}


def cup_obj(*, segments=12, r_bottom=0.3, r_top=0.4, height=0.45):
    """OBJ text of a flared open cup in y-up coordinates (a scene geometry is
    turned by pi/2 about x, so y becomes z): a fan floor at y = 0 and a ring
    of wall quads split in two triangles, written with vertex normals
    ("f v//n"), comment, object and smoothing lines."""
    lines = ["# flared cup, y up", "o cup"]
    ring = [2 * math.pi * k / segments for k in range(segments)]
    lines.append("v 0 0 0")
    for rad, y in ((r_bottom, 0.0), (r_top, height)):
        for t in ring:
            lines.append("v %.9g %.9g %.9g" % (f32(rad * math.cos(t)), f32(y), f32(rad * math.sin(t))))
    lines += ["vn 0 1 0", "s off"]
    b = lambda k: 2 + k % segments              # bottom ring, 1-based
    t = lambda k: 2 + segments + k % segments   # top ring
    for k in range(segments):
        lines.append("f 1//1 %d//1 %d//1" % (b(k + 1), b(k)))
        lines.append("f %d//1 %d//1 %d//1" % (b(k), b(k + 1), t(k + 1)))
        lines.append("f %d//1 %d//1 %d//1" % (b(k), t(k + 1), t(k)))
    return "\n".join(lines) + "\n"


def quirks_obj():
    """OBJ text that exercises the loader's and the sampler's corner cases:
    "v/vt/vn" faces, a face with a repeated vertex (a zero-length edge), a
    face whose vertices are (nearly) collinear, a long thin face, a
    four-entry face (only its first three entries count), CRLF line ends."""
    lines = [
        "# corner cases", "o quirks", "g part",
        "v 0 0 0", "v 0.37 0.01 -0.02", "v 0.05 0.29 0.11", "v 0.4 0.33 0.2",
        "v 0.2 0.165 0.1", "v 1.3 -0.2 0.05", "v 1.31 -0.18 0.06",
        "vt 0 0", "vt 1 0", "vt 0 1", "vn 0 0 1",
        "f 1/1/1 2/2/1 3/3/1", "f 2/1/1 4/2/1 3/3/1", "f 1/1/1 5/2/1 4/3/1",
        "f 2/1/1 2/2/1 6/3/1", "f 2/1/1 6/2/1 7/3/1", "f 7/1/1 6/2/1 2/3/1 4/1/1",
    ]
    return "\r\n".join(lines) + "\r\n"


def shards_obj(seed=7, vertices=12, faces=16):
    """OBJ text of a seeded soup of random triangles (plain "f a b c"
    faces): irregular float coordinates, so the sampler's rounding order
    shows in the last bits of the samples."""
    rng = np.random.default_rng(seed)
    lo, hi = np.array([0.6, -0.1, -0.3]), np.array([1.4, 0.3, 0.2])
    v = (lo + rng.random((vertices, 3)) * (hi - lo)).astype(np.float32)
    lines = ["v %.9g %.9g %.9g" % tuple(float(c) for c in p) for p in v]
    for _ in range(faces):
        a, b, c = rng.choice(vertices, 3, replace=False) + 1
        lines.append("f %d %d %d" % (a, b, c))
    return "\n".join(lines) + "\n"


GEOMETRY_MESHES = {"cup.obj": cup_obj, "quirks.obj": quirks_obj, "shards.obj": shards_obj}


def geometry_scenes():
    """Akinci scenes whose boundary includes OBJ geometries (the files of
    GEOMETRY_MESHES, referenced by bare file name). DFSPH: a block resting
    just above the floor of the cup, with an outer tank box in the same
    boundary object (box samples first, then the mesh). WCSPH: a
    second boundary object of two meshes, the corner-case mesh sampled at
    0.8 x 2r and a random triangle soup, beside a tank, a block above them."""
    r = 0.025
    df = scene(method=DFSPH, radius=r, blocks=[block((6, 6, 6), r, (-0.15, -0.15, 0.0))],
               tank=((-0.6, -0.6, -0.3), (0.6, 0.6, 0.8)), time_step=5e-4, seed=51)
    df["Boundary"][0]["geometry"] = [{"path": "cup.obj", "spacing": 1.0}]
    wc = scene(method=WCSPH, radius=r, blocks=[block((6, 4, 4), r, (0.1, -0.3, 0.3))],
               tank=((-0.2, -0.5, -0.3), (1.5, 0.4, 0.7)), time_step=2e-4, seed=52)
    wc["Boundary"].append({"box": [], "sphere": [], "geometry": [{"path": "quirks.obj", "spacing": f32(0.8)},
                                                                 {"path": "shards.obj", "spacing": 1.0}]})
    return {"geometry_dfsph_cup": df, "geometry_wcsph_quirks": wc}


def with_pcisph_boundary(scene_dict, normal_fct=0.5, tangential_fct=0.9):
    """The scene with the PCISPH boundary method (boundaryMethod 1): every
    boundary object gets "normalFct"/"tangFct" and every box and sphere an
    "inverted" flag (SceneLoader.cpp:168-195): boxes are containers (True),
    spheres obstacles (False)."""
    scene_dict["Configuration"]["boundaryMethod"] = BOUNDARY_PCISPH
    for b in scene_dict["Boundary"]:
        b["normalFct"] = f32(normal_fct)
        b["tangFct"] = f32(tangential_fct)
        for box in b.get("box", []):
            box["inverted"] = True
        for sph in b.get("sphere", []):
            sph["inverted"] = False
    return scene_dict


def pcisph_boundary_scenes():
    """Small scenes with PCISPH boundary particles (mass particles sampled at
    0.45 h with per-particle normals, densities and pressures, and collision
    correction of positions and velocities), one per solver, in a 1 m tank
    (SPH2O's sampler for this method truncates box lengths to whole numbers),
    with a sphere obstacle in the WCSPH and DFSPH scenes."""
    r = 0.025
    tank = ((0, 0, 0), (1, 1, 1))
    blk = lambda n: block(n, r, (4 * r,) * 3)
    sphere = [((0.8, 0.3, 0.15), 0.12)]  # clear of the blocks by more than h
    wc = with_pcisph_boundary(scene(method=WCSPH, radius=r, blocks=[blk((10, 8, 8))], tank=tank, spheres=sphere,
                                    time_step=2e-4, seed=61), 0.5, 0.9)
    pc = with_pcisph_boundary(scene(method=PCISPH, radius=r, blocks=[blk((8, 8, 10))], tank=tank, eta=0.01,
                                    time_step=5e-4, seed=62), 0.3, 1.0)
    df = with_pcisph_boundary(scene(method=DFSPH, radius=r, blocks=[blk((8, 8, 8))], tank=tank, spheres=sphere,
                                    seed=63), 0.5, 0.8)
    # a block against the far x wall (whose particles sit in the next cell
    # row, x = 1.0): the fluid spreads along the wall into cells no particle
    # has visited, which hold no candidate lists until the next search
    fw = with_pcisph_boundary(scene(method=WCSPH, radius=r, blocks=[block((5, 4, 8), r, (0.72, 0.4, 0.03))], tank=tank,
                                    time_step=2e-4, seed=64), 0.4, 0.95)
    # two lone particles pressed against the far x wall and driven along it
    # (gravity 20 along x, 40 along y), at the heights of wall particle rows
    # (z = 16 and 9 spacings of 1/23): when they cross y = 0.6 they enter
    # cells no particle has visited, which hold no candidate lists until the
    # next search, so that step goes uncorrected though they touch the wall
    ws = with_pcisph_boundary(scene(method=WCSPH, radius=r,
                                    blocks=[block((1, 1, 1), r, (0.94, 0.52, 16 / 23 - r)),
                                            block((1, 1, 1), r, (0.94, 0.52, 9 / 23 - r))], tank=tank,
                                    gravity=(20.0, 40.0, 0.0), time_step=2e-4, seed=65), 0.4, 1.0)
    return {"pcib_wcsph_sphere": wc, "pcib_pcisph": pc, "pcib_dfsph_sphere": df, "pcib_wcsph_farwall": fw,
            "pcib_wcsph_wallslide": ws}


def resolve_geometry_paths(scene_dict, directory):
    """Copy of the scene with every relative geometry path joined to `directory`."""
    import copy
    import os

    out = copy.deepcopy(scene_dict)
    for b in out.get("Boundary", []):
        for g in b.get("geometry", []):
            if not os.path.isabs(g["path"]):
                g["path"] = os.path.join(directory, g["path"])
    return out


def batched_scene_params(count=256, seed=4):
    """Per-scene parameters of the batched workload: N_f log-uniform in
    [2000, 40000], block aspect ratios uniform in [0.5, 2] (normalised so the
    lattice holds about N_f particles), viscosity uniform in [0.005, 0.05],
    r = 0.01, each in its own tank sized to the block."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nf = math.exp(rng.uniform(math.log(2000), math.log(40000)))
        ax, ay = rng.uniform(0.5, 2.0, size=2)
        visc = float(rng.uniform(0.005, 0.05))
        # nx : ny : nz = ax : ay : 1 with nx*ny*nz ~= nf
        nz = (nf / (ax * ay)) ** (1.0 / 3.0)
        dims = (max(2, int(round(ax * nz))), max(2, int(round(ay * nz))), max(2, int(round(nz))))
        out.append({"dims": dims, "viscosity": visc})
    return out


def batched_scenes(count=256, method=WCSPH, seed=4):
    r = 0.01
    scenes = []
    for i, p in enumerate(batched_scene_params(count, seed)):
        nx, ny, nz = p["dims"]
        ext = (nx * 2 * r, ny * 2 * r, nz * 2 * r)
        tank = ((0, 0, 0), (max(1.0, 2 * ext[0] + 8 * r), max(1.0, ext[1] + 8 * r), max(1.0, ext[2] + 8 * r)))
        scenes.append(scene(
            method=method, radius=r, blocks=[block((nx, ny, nz), r, (4 * r,) * 3)], tank=tank,
            time_step=1e-4, viscosity=p["viscosity"], eta=1e-3, eta_v=1e-3, seed=1000 + i,
        ))
    return scenes


def write(scene_dict, path):
    with open(path, "w") as f:
        json.dump(scene_dict, f, indent=1)
    return path
