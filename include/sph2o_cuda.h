/*
 * sph2o_cuda.h -- C ABI of the B200 (sm_100a) SPH particle pipeline.
 *
 * This is the drop-in boundary for SPH2O's per-step particle path. SPH2O has
 * no plugin or FFI layer: its boundary is the C++ virtual class
 *   SPHSolver { init(); step(); resize(); computeDensities(); integrate();
 *               insertFluidParticles(); neighborhoodSearch(); }
 * (inc/SPH2O/SPHSolver/SPHSolver.h:22-37), created by
 * SPHSimulation::setSimulationMethod (src/SPH2O/SPHSimulation.cpp:216-239)
 * and stepped by SPHSimulation::step (src/SPH2O/SPHSimulation.cpp:168).
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions: every function returns an int status (SPH_OK = 0, negative =
 * error; see sph_status). No C++ exception crosses this ABI. Arrays are plain
 * host pointers; xyz arrays hold n*3 floats (x0 y0 z0 x1 ...). A context owns
 * all of its device memory and one CUDA stream; the caller keeps ownership of
 * every array it passes. One host thread drives a context at a time.
 * Particle order at this boundary is always the caller's (reference) order;
 * the internal cell-sorted order never leaks out.
 */
#ifndef SPH2O_CUDA_H
#define SPH2O_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPH2O_ABI_VERSION 1

/* Method ids, identical to SPHSimulation's constants
   (src/SPH2O/SPHSimulation.cpp:21-33). */
enum sph_method { SPH_WCSPH = 0, SPH_PCISPH = 1, SPH_DFSPH = 2 };
enum sph_boundary_method { SPH_BOUNDARY_CUBE = 0, SPH_BOUNDARY_PCISPH = 1, SPH_BOUNDARY_AKINCI = 2 };
enum sph_force_method {
    SPH_VISCOSITY_STANDARD = 0,
    SPH_VISCOSITY_ARTIFICIAL = 1,
    SPH_VISCOSITY_XSPH = 2,
    SPH_SURFACE_TENSION_AKINCI = 3,
    SPH_ADHESION_AKINCI = 4
};

enum sph_status {
    SPH_OK = 0,
    SPH_ERR_ARG = -1,              /* bad argument or unsupported option      */
    SPH_ERR_CUDA = -2,             /* CUDA runtime error (text in last_error) */
    SPH_ERR_NAN = -3,              /* non-finite particle state detected      */
    SPH_ERR_NEIGHBOR_OVERFLOW = -4,/* a particle exceeded the neighbour capacity */
    SPH_ERR_TIMEOUT = -5,          /* a bounded device-side wait gave up      */
    SPH_ERR_STATE = -6,            /* call out of order (e.g. step before init) */
    SPH_ERR_NO_DEVICE = -7,        /* no CUDA device / extension unusable     */
    SPH_ERR_IO = -8,               /* file or JSON error                      */
    SPH_ERR_CAPACITY = -9          /* size above a fixed, documented maximum  */
};

/* Scene parameters: the fields of SceneInfo + Fluid (inc/SPH2O/SPHStructs.h:11-67)
   that the particle path reads. */
typedef struct sph_scene_desc {
    int simulation_method;          /* sph_method */
    int boundary_method;            /* SPH_BOUNDARY_AKINCI, SPH_BOUNDARY_PCISPH or SPH_BOUNDARY_CUBE */
    int viscosity_method;           /* -1 none, 0 standard, 1 artificial, 2 XSPH */
    int surface_tension_method;     /* -1 none, 3 Akinci */
    int adhesion_method;            /* -1 none, 4 Akinci */
    float particle_radius;          /* r; support radius h = 4r (SPHSimulation.cpp:201-208) */
    float density0;                 /* rest density */
    float gravity[3];
    float time_step;                /* initial (DFSPH) or fixed (WCSPH/PCISPH) dt */
    float min_time_step, max_time_step, fps;
    float start_time, end_time;
    float stiffness, gamma;         /* WCSPH Tait EOS */
    float eta, eta_v, cfl_factor;   /* PCISPH/DFSPH tolerances, DFSPH CFL factor */
    unsigned min_iterations, max_iterations, min_iterations_v, max_iterations_v;
    float viscosity, boundary_viscosity, surface_tension, adhesion;
    float domain_min[3], domain_max[3]; /* grid bounds hint; all zero = derive from particles */
    unsigned flags;                 /* reserved, must be 0 */
} sph_scene_desc;

/* Per-call statistics (the values SPH2O prints only under DEBUG). */
typedef struct sph_step_stats {
    double time;                    /* simulated time after the last step */
    double avg_density_error;       /* last density-solver residual (FP64 reduction) */
    double avg_divergence_error;    /* last divergence-solver residual (FP64 reduction) */
    float dt;                       /* time step used by the last step */
    float max_velocity;             /* CFL speed of the last DFSPH step, else 0 */
    unsigned iterations;            /* density / pressure iterations of the last step */
    unsigned iterations_v;          /* divergence iterations of the last step (DFSPH) */
    unsigned long long total_iterations;   /* summed over the steps of this call */
    unsigned long long total_iterations_v;
    unsigned steps;                 /* steps taken by this call */
    unsigned neighbor_overflows;    /* particles whose neighbour list was truncated */
    double device_ms;               /* device time of the steps of this call (CUDA
                                       events on the context stream) */
    unsigned long long kernel_launches; /* kernels this call launched */
} sph_step_stats;

/* Per-phase device timing (CUDA events around each phase on the context
   stream). Phases of one step, in launch order: */
enum sph_profile_phase {
    SPH_PROF_SORT = 0,        /* cell keys, counting sort, reorder        */
    SPH_PROF_LISTS = 1,       /* neighbour-list build                      */
    SPH_PROF_DENSITY = 2,     /* density (+alpha, +EOS)                    */
    SPH_PROF_NORMALS = 3,     /* surface-tension normals                   */
    SPH_PROF_FORCES = 4,      /* non-pressure forces (+WCSPH pressure, integrate) */
    SPH_PROF_DENSITY_SOLVE = 5,  /* DFSPH density solver (persistent kernel) */
    SPH_PROF_DIVERGENCE_SOLVE = 6,/* DFSPH divergence solver (persistent kernel) */
    SPH_PROF_PRESSURE_SOLVE = 7, /* PCISPH pressure solver (persistent kernel) */
    SPH_PROF_COUNT = 8
};

typedef struct sph_ctx sph_ctx;

/* ---- context lifecycle ------------------------------------------------ */

/* Make `device` the current CUDA device of the calling thread for this
   library (contexts created afterwards live on it). No reference counterpart:
   SPH2O is CPU-only. */
int sph_select_device(int device);

/* Replaces SPHSimulation::setSimulationMethod + the solver constructors
   (SPHSimulation.cpp:216-239, 316-350). Selects the device with
   cudaGetDevice at the time of the call. */
int sph_create(const sph_scene_desc* desc, sph_ctx** out);

/* Fluid particles (FluidObject::r / v, inc/SPH2O/FluidObject/FluidObject.h:17-24).
   v may be NULL (zero velocities). Must precede sph_init. */
int sph_set_fluid(sph_ctx* ctx, unsigned n, const float* xyz, const float* v);

/* Akinci boundary particles of all boundary objects, concatenated in object
   order (AkinciBoundaryObject::r, AkinciBoundaryObject.cpp:36-95). */
int sph_set_boundary(sph_ctx* ctx, unsigned n, const float* xyz);

/* Cube boundary (boundary_method SPH_BOUNDARY_CUBE; CubeBoundaryObject,
   CubeBoundaryObject.cpp:10-88): no boundary particles; after each step's
   integration every fluid particle outside [min, max] is put back on the
   violated face, the velocity component pointing out scaled by
   -normal_fct and the other two by tangential_fct, axis by axis (x, y, z),
   cube by cube in the order added. SPH2O's loader never reads the factors
   for this method, so scenes loaded by sph_scene_load carry 0 and 0 (a
   particle that hits a wall stops there), as in the reference. Before
   sph_init; single scenes only. */
/* Replaces the per-particle normals n[] and setNormalFct / setTangentialFct
   of PCISPHBoundaryObject (PCISPHBoundaryObject.h:8-26) for boundary_method
   SPH_BOUNDARY_PCISPH: one normal per boundary particle of sph_set_boundary
   (same order), before sph_init. The boundary particles then carry the mass
   rho0 (2r)^3 and their own densities and pressures, and fluid particles
   closer than h/2 are pushed out along the weighted boundary normal with
   their velocity split into normal_fct and tangential_fct parts
   (PCISPHBoundaryObject.cpp:218-447). One boundary object: SPH2O indexes a
   boundary object's arrays with the candidates of all objects
   (PCISPHBoundaryObject.cpp:242), which is well defined for one. */
int sph_set_boundary_normals(sph_ctx* ctx, unsigned n, const float* normals, float normal_fct,
                             float tangential_fct);
/* Boundary densities and pressures of the PCISPH boundary method (the last
   computed: by a step or sph_compute_phase), caller order; either pointer
   may be NULL. */
int sph_get_boundary_state(sph_ctx* ctx, float* density, float* pressure);
int sph_add_cube_boundary(sph_ctx* ctx, const float min[3], const float max[3], float normal_fct,
                          float tangential_fct);

/* Particle emitter of the fluid model (Emitter.h:10-33; scene keys of
   SceneLoader.cpp:128-143). An emitter holds num_particles inactive
   particles; every time the simulated time reaches its next emission time
   (start_time, then + spacing * 1.105 * 2r / velocity after each emission)
   it activates one group -- a square lattice of width x height at spacing 2r
   or concentric rings out to radius width -- moving at `velocity` along the
   emitter's local z, rotated by `rotation` and placed at `position`
   (Emitter.cpp:25-128). */
enum sph_emitter_type { SPH_EMITTER_SQUARE = 0, SPH_EMITTER_CIRCLE = 1 };
typedef struct sph_emitter_desc {
    int type;                       /* sph_emitter_type */
    unsigned num_particles;         /* particles it emits in total */
    float position[3];
    float rotation[4];              /* quaternion w, x, y, z (glm::quat order) */
    float velocity;                 /* emission speed (> 0) */
    float start_time;
    float width, height;            /* square: width x height; circle: radius width */
    float spacing;                  /* emission period factor */
} sph_emitter_desc;

/* Replaces FluidObject::addEmitter (FluidObject.cpp:177-194): adds an
   emitter before sph_init; the context's fluid grows by num_particles
   inactive particles (sph_num_fluid counts them, as FluidObject::getSize
   does). Single scenes only. */
int sph_add_emitter(sph_ctx* ctx, const sph_emitter_desc* emitter);

/* Active fluid particles (FluidObject::getNumActiveParticles): the first n
   of the caller order; emitted particles take the next caller ids in
   emission order, as in the reference. Waits for queued work. */
int sph_get_num_active(sph_ctx* ctx, unsigned* n);

/* Replaces SPHSimulation::init (SPHSimulation.cpp:117-126): kernel constants,
   masses m = rho0 (2r)^3, boundary volumes (AkinciBoundaryObject::computeVolume,
   AkinciBoundaryObject.cpp:10-34) and the solver's init (DFSPHSolver::init,
   DFSPHSolver.cpp:22-31: neighbour search, densities, alpha;
   PCISPHSolver::init: scaling factor, PCISPHSolver.cpp:403-436). */
int sph_init(sph_ctx* ctx);

/* Replaces nsteps calls of SPHSolver::step (WCSPHSolver.cpp:14-78,
   PCISPHSolver.cpp:20-80, DFSPHSolver.cpp:33-107). Kernels are queued on the
   context stream; the call returns after the last step completes and `out`
   (may be NULL) is filled. Steps are taken unconditionally: the start/end
   time window of SPHSimulation::step is the driver's business. */
int sph_step(sph_ctx* ctx, int nsteps, sph_step_stats* out);

/* Queue nsteps steps without waiting (no stats); sph_sync waits and returns
   the status of everything queued since the last wait. */
int sph_step_async(sph_ctx* ctx, int nsteps);
int sph_sync(sph_ctx* ctx, sph_step_stats* out);

/* Enable (1) or disable (0) per-phase event timing; enabling clears the totals. */
int sph_profile_enable(sph_ctx* ctx, int enable);
/* Accumulated per-phase device milliseconds and launch counts since enabling
   (arrays of SPH_PROF_COUNT; either may be NULL). Waits for queued work. */
int sph_profile_read(sph_ctx* ctx, double* ms, unsigned long long* launches);

/* ---- launch options and autotuning (no reference counterpart) -------- */
enum sph_option {
    SPH_OPT_CUDA_GRAPHS = 0,      /* 1 (default): steps replay captured CUDA graphs of two steps (one
                                     for an odd remainder), keyed by the buffer assignment */
    SPH_OPT_CELL_ORDER = 1,       /* 0 (default): 4x4x4 cell bricks, Morton inside; 1: linear, x fastest */
    SPH_OPT_SOLVER_OCCUPANCY = 2, /* DFSPH persistent solver blocks per SM: 8 (default) or 4 */
    SPH_OPT_PASS_BLOCK = 3,       /* threads per block of the particle-pass kernels: 256 (default) or 128 */
    SPH_OPT_SOLVER_LANES = 4,     /* lanes sharing one particle's neighbour list in the persistent DFSPH
                                     solver: 1, 2 (default) or 4 */
    SPH_OPT_POSITION_RESIDUAL = 5,/* 1: every position keeps the rounding residual of its integration
                                     (float pair, error-free sums), so long runs of small steps keep about
                                     twice float precision; 0 (default): FP32 positions rounded as the
                                     reference rounds them. Single scenes, set before sph_init. */
    SPH_OPT_LIST_STAGED = 6       /* neighbour-list build of single scenes of 2^16 fluid particles and more
                                     in brick cell order: 1 one block per 4x4x4-cell brick with the
                                     positions of the 6x6x6 cells around it staged in shared memory;
                                     0 (default) one thread per particle reading the cells from global
                                     memory. Both write the same lists. */
};
/* Number of values sph_autotune chooses (options 1..4 in order). */
#define SPH_TUNE_COUNT 4
int sph_set_option(sph_ctx* ctx, int option, int value);
int sph_get_option(const sph_ctx* ctx, int option, int* value);

/* Chooses SPH_OPT_CELL_ORDER, SPH_OPT_SOLVER_OCCUPANCY, SPH_OPT_PASS_BLOCK and
   SPH_OPT_SOLVER_LANES by timing trial_steps steps (CUDA events) of every
   combination, each from a snapshot of the current state that is restored
   afterwards: the simulation is left exactly where it was. cache_path (may
   be NULL) names a JSON file keyed by GPU name, method and particle counts;
   a hit skips the trials and a miss appends the result. config (may be NULL)
   receives the SPH_TUNE_COUNT chosen values in option order 1..4. */
int sph_autotune(sph_ctx* ctx, int trial_steps, const char* cache_path, int* config);

/* Fluid state in the caller's particle order. Any pointer may be NULL.
   rho is FluidObject::density as SPH2O leaves it after a step. Arrays hold
   sph_num_fluid particles; with emitters the inactive ones read as zero. */
int sph_get_state(sph_ctx* ctx, float* xyz, float* v, float* rho);

/* Replace positions/velocities (same order as sph_set_fluid) between steps;
   replaces writes through FluidObject::getPosition/getVelocity. With
   emitters only the active particles are taken from the arrays. */
int sph_set_state(sph_ctx* ctx, const float* xyz, const float* v);

/* Akinci boundary volumes V_b in the sph_set_boundary order. */
int sph_get_boundary_volume(sph_ctx* ctx, float* vol);

/* Simulated time and current dt (TimeHelper::getTime/getTimeStep). */
int sph_get_time(sph_ctx* ctx, double* time, float* dt);

/* Set simulated time and the current dt (TimeHelper::setTime / setTimeStep,
   inc/SPH2O/TimeHelper.h:51-54), e.g. when resuming from a frame file. */
int sph_set_time(sph_ctx* ctx, double time, float dt);

unsigned sph_num_fluid(const sph_ctx* ctx);
unsigned sph_num_boundary(const sph_ctx* ctx);

/* Text of the last error on this context (never NULL). */
const char* sph_last_error(const sph_ctx* ctx);
/* Text of the last error of a call that had no context (sph_create). */
const char* sph_global_error(void);

int sph_destroy(sph_ctx* ctx);

/* ---- batches of independent scenes --------------------------------------
   No reference counterpart (SPH2O runs one scene per process). A batch
   steps many independent scenes in one launch per phase: scenes keep their
   own coordinates, cell grids, boundaries, time steps, viscosity and DFSPH
   convergence (a converged scene stops iterating while others continue).
   All scenes share the method (WCSPH or DFSPH), particle radius, rest
   density, gravity, force methods and solver tolerances; viscosity,
   boundary viscosity and the initial time step may differ per scene.
   A batch is a context: sph_init, sph_step, sph_sync, sph_get_state
   (all scenes concatenated in scene order), sph_profile_* and
   sph_compute_phase apply to it; sph_set_fluid/sph_set_boundary do not. */

int sph_batch_create(const sph_scene_desc* descs, unsigned nscenes, sph_ctx** out);
/* Particles of one scene (before sph_init); v and bxyz may be NULL. */
int sph_batch_set_scene(sph_ctx* ctx, unsigned scene, unsigned nf, const float* xyz, const float* v, unsigned nb,
                        const float* bxyz);
unsigned sph_batch_num_scenes(const sph_ctx* ctx);
/* The scene's fluid particles occupy [begin, end) of the concatenated order. */
int sph_batch_scene_range(const sph_ctx* ctx, unsigned scene, unsigned* begin, unsigned* end);
/* Per-scene time, dt, iterations and residuals (cumulative iteration totals). */
int sph_batch_scene_stats(sph_ctx* ctx, unsigned scene, sph_step_stats* out);

/* ---- differentiable WCSPH (no reference counterpart) -------------------
   SPH2O has no adjoint; these entry points differentiate its WCSPH step
   (WCSPHSolver::step, WCSPHSolver.cpp:14-78: densities, Tait EOS, pressure
   force, artificial viscosity, symplectic Euler; Akinci boundaries) with the
   neighbour lists of each step held fixed. Loss:
       L = (1/N) sum_i |x_i(T) - target_i|^2
   over the N fluid particles after nsteps steps. Single-scene WCSPH
   contexts with artificial viscosity (or none) and neither surface tension
   nor adhesion; anything else returns SPH_ERR_ARG. */

/* Steps the context nsteps WCSPH steps from its current state (which
   becomes x(0), v(0)), keeping a checkpoint of the state entering every
   ckpt_every-th step, and returns the loss against `target` (n*3 floats,
   caller order). The context is left in the final state, as sph_step
   leaves it. Device memory: (nsteps / ckpt_every + ckpt_every) states of
   36 bytes per particle. */
int sph_wcsph_forward(sph_ctx* ctx, int nsteps, int ckpt_every, const float* target, double* loss);

/* Gradients of the last sph_wcsph_forward's loss with respect to the
   initial velocities (dL_dv0: n*3 floats, caller order), the artificial
   viscosity coefficient and the EOS stiffness (any pointer may be NULL).
   Segments are recomputed from their checkpoints (bit-identical to the
   forward run); the context is returned to the state the forward run left. */
int sph_wcsph_backward(sph_ctx* ctx, float* dL_dv0, float* dL_dvisc, float* dL_dk);

/* Gradient with respect to the initial positions from the last
   sph_wcsph_backward (n*3 floats, caller order). */
int sph_wcsph_grad_x0(sph_ctx* ctx, float* dL_dx0);

/* Device milliseconds of the last sph_wcsph_forward / sph_wcsph_backward
   (CUDA events on the context stream). */
int sph_wcsph_timing(const sph_ctx* ctx, double* forward_ms, double* backward_ms);

/* ---- phase access for parity checks ------------------------------------- */

enum sph_phase {
    SPH_PHASE_DENSITY = 0,          /* SPHSolver::computeDensities (SPHSolver.cpp:42-89), n floats */
    SPH_PHASE_ALPHA = 1,            /* DFSPHSolver::computeAlpha (DFSPHSolver.cpp:109-178), n floats */
    SPH_PHASE_NONPRESSURE_ACC = 2,  /* SPHSimulation::computeNonPressureForces, n*3 floats */
    SPH_PHASE_PRESSURE = 3,         /* WCSPHSolver::computePressures (WCSPHSolver.cpp:80-129), n floats */
    SPH_PHASE_PRESSURE_ACC = 4      /* WCSPHSolver::computePressureForce (WCSPHSolver.cpp:132-188), n*3 */
};

/* Runs the neighbour search at the current positions, then the named phase
   (and the phases it depends on: densities before alpha/forces/pressure),
   and copies its per-particle result out in caller order. State used by the
   next sph_step is not changed except densities and neighbour lists, which
   the next step recomputes anyway. */
int sph_compute_phase(sph_ctx* ctx, int phase, float* out);

/* Neighbour sets of every fluid particle at the current positions, in CSR
   form and caller order: N(i) = { j in the 27 cells around floor(x_i / h) :
   |x_i - x_j| <= h } with |.| evaluated as sqrt((dx*dx + dy*dy) + dz*dz) in
   IEEE single precision, the test of DFSPHSolver.cpp:575,589,603.
   With NULL index arrays only the totals are returned in *nf_total/*nb_total.
   Offsets arrays hold n+1 entries. Indices are caller-order fluid / boundary ids. */
int sph_debug_neighbors(sph_ctx* ctx, unsigned* f_offsets, unsigned* f_index, size_t f_cap,
                        unsigned* b_offsets, unsigned* b_index, size_t b_cap,
                        size_t* nf_total, size_t* nb_total);

/* Test hook for the bounded device-side waits (no reference counterpart):
   launches a two-block cooperative kernel in which one block never reaches
   the grid barrier. The waiting block gives up after its spin limit (about
   a second), records the timeout and returns; the call then reports
   SPH_ERR_TIMEOUT and clears the flag, leaving the context usable. */
int sph_debug_barrier_timeout(sph_ctx* ctx);

/* ---- allocation-free density evaluation ------------------------------- */

/* Fixed capacity of sph_density_noalloc's scratch. */
#define SPH_NOALLOC_MAX_FLUID 65536u
#define SPH_NOALLOC_MAX_BOUNDARY 65536u
#define SPH_NOALLOC_MAX_CELLS 262144u

/* Densities of nf fluid particles, for callers that must not allocate GPU
   memory: code running inside a host callback or an allocator hook, or in a
   process whose device memory is pooled by a framework, or on a real-time
   path that may not take the allocator's locks or its implicit
   synchronisation. No counterpart in the reference (SPH2O is CPU-only); the
   density is SPHSolver::computeFluidDensities' sum.
   Inputs and output are device pointers owned by the caller:
     xyz      nf * 3 floats, fluid positions
     bxyzpsi  nb * 4 floats, boundary x, y, z and psi = rho0 * V_b
              (may be NULL when nb = 0)
     rho_out  nf floats, written in the order of xyz
   domain_min/max (host, 3 finite floats each) bound the particles. For
   particles inside them the densities equal
   sph_compute_phase(SPH_PHASE_DENSITY) bit for bit; a particle outside is
   clamped into an edge cell of the grid, still finds all its neighbours but
   sums them in another order, so its density agrees only to rounding (and
   takes longer). Work is queued on `stream`
   (a cudaStream_t; NULL = the legacy default stream) and the call returns
   without waiting. Nothing is allocated: the neighbour-search scratch is a
   fixed file-scope device array of about 9.5 MiB that every GPU loading this
   library keeps until exit. Sizes above SPH_NOALLOC_MAX_FLUID,
   SPH_NOALLOC_MAX_BOUNDARY or SPH_NOALLOC_MAX_CELLS (cells of edge 4r over
   the domain, padded) return SPH_ERR_CAPACITY with the reason in
   sph_noalloc_error(). All calls on a device share that array: calls whose
   work overlaps on the GPU race and must be serialised by the caller. The
   first call on each device looks up the array's address
   (cudaGetSymbolAddress) with that device current; make it before any stream
   capture on that device. The address is kept per device and CUDA context:
   after cudaDeviceReset the next call looks it up again, so that call also
   belongs outside a stream capture. Non-finite bounds, or bounds whose cell
   indices do not fit in an int, return SPH_ERR_ARG. */
int sph_density_noalloc(float particle_radius, float density0, const float* xyz, unsigned nf,
                        const float* bxyzpsi, unsigned nb, const float domain_min[3],
                        const float domain_max[3], float* rho_out, void* stream);
const char* sph_noalloc_error(void);

/* ---- host scene loading (SceneLoader + object builders) --------------- */

typedef struct sph_scene sph_scene;

/* Replaces SceneLoader::readConfiguration (SceneLoader.cpp:11-209) and the
   object construction of SPHSimulation::importScene (SPHSimulation.cpp:299-481):
   FluidObject::build lattice (FluidObject.cpp:30-61), seeded jitter,
   AkinciBoundaryObject::sampleCube/sampleSphere (AkinciBoundaryObject.cpp:97-153)
   and addGeometry (:74-95) for OBJ "geometry" entries (see sph_sample_geometry).
   Missing "sphere"/"geometry" keys are tolerated. A relative geometry path
   is opened as given, else relative to the scene file's directory.
   Returns SPH_ERR_IO for unreadable files or malformed JSON, SPH_ERR_ARG for
   unsupported options or malformed meshes, SPH_ERR_CAPACITY for a mesh
   sampled into more than 2^30 points. Scenes with geometry entries are
   sampled on the current CUDA device (SPH_ERR_NO_DEVICE without one). */
int sph_scene_load(const char* json_path, sph_scene** out);
int sph_scene_parse(const char* json_text, sph_scene** out);
int sph_scene_get_desc(const sph_scene* s, sph_scene_desc* out);
unsigned sph_scene_num_fluid(const sph_scene* s);
unsigned sph_scene_num_boundary(const sph_scene* s);
/* Cube boundaries of a scene with boundaryMethod 0 (the first "box" of each
   boundary object, SPHSimulation.cpp:459-477). */
unsigned sph_scene_num_cube_boundaries(const sph_scene* s);
int sph_scene_get_cube_boundary(const sph_scene* s, unsigned k, float min[3], float max[3], float* normal_fct,
                                float* tangential_fct);
/* Boundary normals (nb x 3, the order of sph_scene_get_boundary) and the
   object's normalFct / tangFct of a scene with boundaryMethod 1, sampled by
   PCISPHBoundaryObject::sampleCube / sampleSphere
   (PCISPHBoundaryObject.cpp:6-213); SPH_ERR_ARG for other methods. */
int sph_scene_get_boundary_normals(const sph_scene* s, float* xyz, float* normal_fct, float* tangential_fct);
/* Emitters of the scene's fluid model ("emitters" key, SceneLoader.cpp:109-143). */
unsigned sph_scene_num_emitters(const sph_scene* s);
int sph_scene_get_emitter(const sph_scene* s, unsigned k, sph_emitter_desc* out);
int sph_scene_get_fluid(const sph_scene* s, float* xyz, float* v);
int sph_scene_get_boundary(const sph_scene* s, float* xyz);
const char* sph_scene_error(void);
void sph_scene_free(sph_scene* s);

/* ---- triangle meshes as boundary particles --------------------------- */

/* Replaces Utilities::OBJLoader::loadObj (extern/OBJLoader/OBJLoader.h:31-158)
   for triangulated meshes, on the host: vertex coordinates times `scale`
   (NULL: 1) and 0-based triangle indices. *num_vertices / *num_faces
   receive the counts; the arrays (NULL to query) receive the data when
   their capacities suffice, else SPH_ERR_CAPACITY. SPH_ERR_IO for an
   unreadable file, SPH_ERR_ARG for a malformed mesh. */
int sph_load_obj(const char* obj_path, const float scale[3], float* vertices, size_t vertex_capacity,
                 size_t* num_vertices, unsigned* faces, size_t face_capacity, size_t* num_faces);

/* Replaces SPH::RegularTriangleSampling::sampleMesh
   (extern/RegularTriangleSampling/RegularTriangleSampling.cpp:12-20), run
   on the current CUDA device (sph_select_device): `vertices` holds
   num_vertices xyz triples, `faces` num_faces 0-based index triples. The
   samples are every vertex, then the interior stops of each unique edge,
   then the interior stops of each face's lines parallel to its longest
   edge, at most max_distance apart, bit-identical to the reference's FP32
   build. Two-call convention: *count receives the number of xyz samples;
   `samples` (NULL to query) receives them when `capacity` (in points)
   suffices, else SPH_ERR_CAPACITY. SPH_ERR_ARG for a bad index, a
   non-finite vertex or max_distance <= 0; SPH_ERR_NO_DEVICE without a GPU;
   text in sph_scene_error(). */
int sph_sample_mesh(const float* vertices, unsigned num_vertices, const unsigned* faces, unsigned num_faces,
                    float max_distance, float* samples, size_t capacity, size_t* count);

/* Replaces AkinciBoundaryObject::sampleGeometry
   (src/SPH2O/BoundaryObject/AkinciBoundaryObject.cpp:155-214): reads a
   triangulated OBJ file (OBJLoader::loadObj, extern/OBJLoader/OBJLoader.h:31-158;
   coordinates times `scale`), samples it as sph_sample_mesh does, then maps
   each sample p to R (p, 1) + translate with R = glm::rotate(I, rotate[0], x)
   -> (.., rotate[1], y) -> (.., rotate[2], z). NULL scale/translate/rotate
   mean 1, 0, 0. Scene geometries use scale 1, translate 0, rotate (pi/2, 0, 0)
   (AkinciBoundaryObject::addGeometry, :74-80). SPH_ERR_IO for an unreadable
   file; otherwise as sph_sample_mesh. */
int sph_sample_geometry(const char* obj_path, float max_distance, const float scale[3], const float translate[3],
                        const float rotate[3], float* samples, size_t capacity, size_t* count);

/* create + set_fluid + set_boundary (+ set_boundary_normals) +
   add_cube_boundary + add_emitter + init from a loaded scene. */
int sph_create_from_scene(const sph_scene* s, sph_ctx** out);

#ifdef __cplusplus
}
#endif
#endif
