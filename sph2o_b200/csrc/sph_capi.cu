/*
 * Context management and the extern "C" entry points of include/sph2o_cuda.h.
 *
 * A context owns one CUDA stream and every device buffer of one scene. The
 * step sequences mirror the reference solvers' step() order:
 *   WCSPH  (WCSPHSolver.cpp:14-78):  neighbour search -> density + Tait EOS ->
 *          [surface-tension normals] -> pressure + non-pressure forces +
 *          symplectic Euler (one kernel, writes the spare buffers)
 *   PCISPH (PCISPHSolver.cpp:20-80): neighbour search -> density ->
 *          [normals] -> non-pressure forces -> persistent pressure solver
 *          (predict / density / pressure / pressure force loop + integrate)
 *   DFSPH  (DFSPHSolver.cpp:33-107): [normals] -> non-pressure forces + CFL
 *          speed -> persistent density solver (dt update, predict v, warm
 *          start, loop, update x) -> neighbour search -> density + alpha ->
 *          persistent divergence solver (warm start, loop, t += dt)
 * No step makes a host round trip; sph_step waits once at the end.
 */
#include "../../include/sph2o_cuda.h"
#include "../host/json_lite.h"
#include "sph_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <vector>

using namespace sph;

namespace {

thread_local std::string g_global_error;

/* The host-side buffer assignment (which of each swapped pair is current). */
struct Buffers {
    float4 *pos, *pos2, *vel, *vel2;
    unsigned *orig, *orig2;
    float *kws, *kws2, *kvws, *kvws2;
    float4 *normal, *normal2;
    float4 *plo, *plo2;
    bool lists_valid;
};

} // namespace

struct sph_ctx {
    sph_scene_desc desc{};
    SimParams P{};
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    bool initialized = false;
    unsigned nf = 0, nb = 0;
    std::vector<float> h_fluid, h_vel, h_bound;
    std::vector<void*> allocations;

    /* current / spare buffers (swapped by the neighbour-search sort) */
    float4 *pos = nullptr, *vel = nullptr, *pos2 = nullptr, *vel2 = nullptr;
    unsigned *orig = nullptr, *orig2 = nullptr;
    float *kws = nullptr, *kws2 = nullptr, *kvws = nullptr, *kvws2 = nullptr;
    float4 *acc = nullptr, *normal = nullptr, *predr = nullptr, *pacc = nullptr;
    float *rho = nullptr, *alpha = nullptr, *k = nullptr, *press = nullptr;
    unsigned *cell_of = nullptr, *slot = nullptr, *tmp_key = nullptr, *tmp_src = nullptr, *cell_sorted = nullptr;
    unsigned *cell_count = nullptr, *cell_start = nullptr, *bcell_start = nullptr, *block_sums = nullptr;
    float4* bpos = nullptr;
    float* bvol = nullptr;
    unsigned* borig = nullptr;
    unsigned *nbr_f = nullptr, *cnt_f = nullptr, *nbr_b = nullptr, *cnt_b = nullptr;
    DevState* st = nullptr;
    DevState* st_host = nullptr; /* pinned mirror */
    double* accum = nullptr;
    size_t accum_len = 0;
    int grid_pcisph = 0;
    int grid_solve[2][2][3] = {};  /* DFSPH solver grid by [divergence][occupancy 8, 4][lanes 1, 2, 4] */
    DevState last{};
    bool lists_valid = false;
    /* timing: batch events + per-phase profiling */
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    bool batch_open = false;
    unsigned long long launches = 0, launches_at_open = 0;
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Pending { int phase; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    double prof_ms[SPH_PROF_COUNT] = {};
    unsigned long long prof_launch[SPH_PROF_COUNT] = {};
    /* batch of independent scenes (nscenes > 0) */
    unsigned nscenes = 0;
    std::vector<sph_scene_desc> descs;
    std::vector<std::vector<float>> sc_fluid, sc_vel, sc_bound;
    std::vector<unsigned> fsplit, bsplit;
    std::vector<SceneInfo> h_scenes;
    SceneInfo* d_scenes = nullptr;
    unsigned *d_scene_of = nullptr, *d_bscene_of = nullptr, *d_any = nullptr;
    SceneState* d_sst = nullptr;
    unsigned accum_stride = 0;
    int grid_batch_density = 0, grid_batch_div = 0;
    std::vector<SceneState> last_sst;
    /* CUDA graphs of two steps, keyed by the buffer assignment they start
       from (the sort swaps buffers, two steps may return to the start) */
    bool use_graphs = true;
    /* tunables (sph_set_option / sph_autotune) */
    int pass_block = 256;
    int solver_occ = 8;
    bool staged_lists = false; /* SPH_OPT_LIST_STAGED */
    int solver_tpp = 2;  /* measured best on B200 for the 1M-particle scene (1, 2, 4: 1.03, 0.84, 0.92 ms) */
    float4* braw = nullptr;      /* boundary in caller order (re-sorted when the cell order changes) */
    unsigned* bid = nullptr;
    /* PCISPH boundary method: boundary normals (caller order on the host,
       sorted on the device), boundary densities / pressures / p over rho^2,
       predicted velocities, the spare normal buffer of the DFSPH sort and
       the per-cell search that first listed each cell */
    std::vector<float> h_bnormal;
    float pcib_nf = 0.0f, pcib_tf = 0.0f;
    float4 *bnormal = nullptr, *normal2 = nullptr, *predv = nullptr;
    float *bdens = nullptr, *bpress = nullptr, *bdp = nullptr;
    unsigned* cell_entry = nullptr;
    /* position residuals (SPH_OPT_POSITION_RESIDUAL): current / spare */
    int pos_lo = 0;
    float4 *plo = nullptr, *plo2 = nullptr;
    float4* snap_plo = nullptr;
    float* divres = nullptr;  /* DFSPH: divergence error of the density pass */
    /* autotune snapshot */
    float4 *snap_pos = nullptr, *snap_vel = nullptr;
    unsigned* snap_orig = nullptr;
    float *snap_kws = nullptr, *snap_kvws = nullptr, *snap_rho = nullptr;
    SceneState* snap_sst = nullptr;
    DevState* snap_st = nullptr;
    struct Graph { unsigned key; cudaGraphExec_t exec; unsigned long long launches; Buffers end; };
    std::vector<Graph> graphs;
    float4* pos_base = nullptr;
    unsigned* orig_base = nullptr;
    float* kws_base = nullptr;
    /* emitters of a single scene (sph_add_emitter): descriptions, the fluid
       particles active at init, the device table and group offsets */
    std::vector<sph_emitter_desc> emitters;
    std::vector<CubeBox> cubes;      /* cube boundaries (boundary method 0) */
    CubeBox* d_cubes = nullptr;
    unsigned n_init = 0;
    EmitterState* d_emit = nullptr;
    float4* d_group = nullptr;
    EmitterState* snap_emit = nullptr;
    /* WCSPH adjoint (sph_wcsph_forward / sph_wcsph_backward) */
    struct Adjoint {
        int nsteps = 0, every = 0, nseg = 0;
        int cap_seg = 0, cap_every = 0;
        float4 *ck_pos = nullptr, *ck_vel = nullptr;   /* checkpoints: state entering each segment */
        unsigned* ck_orig = nullptr;
        float4 *sl_pos = nullptr, *sl_vel = nullptr;   /* per step of one segment: its input state, or */
        unsigned* sl_orig = nullptr;                   /* its sorted state when lists are kept       */
        /* per step of one segment, when they fit kAdjointListBudget: neighbour
           lists, densities and pressures of the recomputed step */
        bool keep_lists = false;
        unsigned sl_capF = 0, sl_capB = 0;
        unsigned *sl_nbr_f = nullptr, *sl_cnt_f = nullptr, *sl_nbr_b = nullptr, *sl_cnt_b = nullptr;
        float *sl_rho = nullptr, *sl_press = nullptr;
        float4 *fin_pos = nullptr, *fin_vel = nullptr; /* state after the forward run */
        unsigned* fin_orig = nullptr;
        DevState *st0 = nullptr, *st1 = nullptr;       /* solver state at the start / end of the run */
        float* target = nullptr;
        float4 *xbar = nullptr, *vbar = nullptr, *abar = nullptr, *xacc = nullptr, *vacc = nullptr;
        float *Ap = nullptr, *rhobar = nullptr;
        double *part = nullptr, *red = nullptr;  /* per-block partial sums, their totals */
        bool ready = false, have_grad = false;
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
        double fwd_ms = 0.0, bwd_ms = 0.0;
        struct Graph { int len; cudaGraphExec_t exec; unsigned long long launches; Buffers end; };
        std::vector<Graph> graphs;
        bool use_graphs = true;
    } adj;
};

namespace {

void drop_graphs(sph_ctx* c);

int fail(sph_ctx* c, int code, const std::string& msg)
{
    if (c) c->err = msg;
    else g_global_error = msg;
    return code;
}

#define CUDA_TRY(ctx, expr)                                                                          \
    do {                                                                                             \
        cudaError_t e_ = (expr);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return fail(ctx, SPH_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));      \
    } while (0)

template <typename T> int dalloc(sph_ctx* c, T** p, size_t count)
{
    void* v = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&v, bytes);
    if (e != cudaSuccess) return fail(c, SPH_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    e = cudaMemsetAsync(v, 0, bytes, c->stream);
    if (e != cudaSuccess) return fail(c, SPH_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    c->allocations.push_back(v);
    *p = static_cast<T*>(v);
    return SPH_OK;
}

void free_all(sph_ctx* c)
{
    for (void* p : c->allocations) cudaFree(p);
    c->allocations.clear();
    if (c->st_host) { cudaFreeHost(c->st_host); c->st_host = nullptr; }
}

/* CubicSpline::gradW on the host, operation for operation (CubicSpline.h:52-74) */
void host_gradW(float x, float y, float z, float h, float l, float* out)
{
    out[0] = out[1] = out[2] = 0.0f;
    const float rl = std::sqrt((x * x + y * y) + z * z);
    const float q = rl / h;
    if (((double)rl > 1.0e-9) && (q <= 1.0f)) {
        float gx = x / rl, gy = y / rl, gz = z / rl;
        gx /= h; gy /= h; gz /= h;
        float c;
        if (q <= 0.5f) c = l * q * (3.0f * q - 2.0f);
        else {
            const float factor = 1.0f - q;
            c = l * (-factor * factor);
        }
        out[0] = c * gx; out[1] = c * gy; out[2] = c * gz;
    }
}

/* Kernel constants and solver parameters (SPHSimulation::initKernels / initMasses,
   SPHSimulation.cpp:133-155; the kernels' setSupportRadius). */
void derive_params(sph_ctx* c)
{
    const sph_scene_desc& d = c->desc;
    SimParams& P = c->P;
    const float pi = (float)M_PI;
    P.r = d.particle_radius;
    P.h = 4.0f * d.particle_radius;
    const float h = P.h;
    P.h2 = h * h;
    P.inv_h = 1.0f / h;
    P.rho0 = d.density0;
    const float diameter = 2.0f * d.particle_radius;
    const float volume = (float)std::pow((double)diameter, 3.0);
    P.mass = d.density0 * volume;
    const float h3 = h * h * h;
    P.cs_k = 8.0f / (pi * h3);
    P.cs_l = 48.0f / (pi * h3);
    P.cs_l_h2 = P.cs_l / (h * h);
    P.cs_l_h = P.cs_l / h;
    const float h6 = h * h * h * h * h * h;
    const float h9 = h * h * h * h * h * h * h * h * h;
    P.coh_c1 = (float)(32.0 / M_PI) / h9;
    P.coh_c2 = h6 / 64.0f;
    P.lapl_c = 45.0f / (pi * h6);
    P.gx = d.gravity[0]; P.gy = d.gravity[1]; P.gz = d.gravity[2];
    P.stiffness = d.stiffness;
    P.gamma = d.gamma;
    P.kr_g = d.gamma != 0.0f ? d.stiffness * d.density0 / d.gamma : 0.0f;
    P.h2_guard = (float)((double)h * (double)h * (1.0 + 1.0e-5));
    P.h2_exact = sqrt_le_bound(h);
    P.eta = d.eta;
    P.eta_v = d.eta_v;
    P.cfl = d.cfl_factor;
    const float min_fps_ts = 1.0f / d.fps;
    P.min_ts = min_fps_ts < d.min_time_step ? min_fps_ts : d.min_time_step; /* TimeHelper.h:57 */
    P.max_ts = d.max_time_step;
    P.min_it = d.min_iterations;
    P.max_it = d.max_iterations;
    P.min_it_v = d.min_iterations_v;
    P.max_it_v = d.max_iterations_v;
    P.eps = 1.0e-5f;
    /* forces exist only when the method is set and the coefficient non-zero
       (SPHSimulation.cpp:380-387) */
    P.visc_method = (d.viscosity_method > -1 && d.viscosity_method <= 2 && d.viscosity != 0.0f) ? d.viscosity_method : -1;
    P.visc = d.viscosity;
    P.bvisc = d.boundary_viscosity;
    P.st_on = (d.surface_tension_method == SPH_SURFACE_TENSION_AKINCI && d.surface_tension != 0.0f) ? 1 : 0;
    P.st = d.surface_tension;
    P.adh_on = (d.adhesion_method == SPH_ADHESION_AKINCI && d.adhesion != 0.0f) ? 1 : 0;
    P.adh = d.adhesion;
    /* PCISPH boundary method: boundary viscosity is an Akinci-only term
       (ArtificialViscosity.cpp:39 and the other viscosity forces) */
    P.pcib = d.boundary_method == SPH_BOUNDARY_PCISPH ? 1 : 0;
    if (P.pcib) P.bvisc = 0.0f;
    P.rest_r = 0.5f * h;
    P.poly6_c = 315.0f / ((float)(64.0 * M_PI) * h9);
    P.spiky_g = 45.0f / ((float)M_PI * h6);
    /* PCISPHSolver::computeScalingFactor (PCISPHSolver.cpp:403-436) at the initial dt */
    float sg[3] = {0, 0, 0}, ssq = 0.0f;
    for (int i = -1; i <= 1; i++)
        for (int j = -1; j <= 1; j++)
            for (int k = -1; k <= 1; k++) {
                const float rx = (float)(-i) * diameter, ry = (float)(-j) * diameter, rz = (float)(-k) * diameter;
                float g[3];
                host_gradW(rx, ry, rz, h, P.cs_l, g);
                sg[0] += g[0]; sg[1] += g[1]; sg[2] += g[2];
                ssq += (g[0] * g[0] + g[1] * g[1]) + g[2] * g[2];
            }
    const float x = P.mass * d.time_step / d.density0;
    const float beta = (float)(2.0 * std::pow((double)x, 2.0));
    const float dot_sg = (sg[0] * sg[0] + sg[1] * sg[1]) + sg[2] * sg[2];
    P.pcisph_delta = -1.0f / (beta * (-dot_sg - ssq));
}

/* Emitter::buildCircleGroup / buildSquareGroup (Emitter.cpp:25-80) with the
   reference's types: float arithmetic, with sin, cos and floor in double
   (the overloads its translation unit resolves to for float arguments) and
   the result rounded to float. Appends x, y, z triples to out. */
void emitter_group(const sph_emitter_desc& e, float radius, std::vector<float>& out)
{
    const float dist = 2.0f * radius;
    if (e.type == SPH_EMITTER_CIRCLE) {
        const unsigned levels = (unsigned)std::floor((double)((e.width - 0.5f * dist) / dist));
        out.insert(out.end(), {0.0f, 0.0f, 0.0f});
        for (unsigned i = 0; i < levels; ++i) {
            const float rad = (float)(i + 1) * dist;
            const float l = (float)(2.0 * M_PI) * rad;
            const unsigned parts = (unsigned)std::floor((double)(l / dist));
            const float inc = (float)(2.0 * M_PI) / (float)parts;
            for (unsigned k = 0; k < parts; ++k) {
                const float angle = (float)k * inc;
                out.push_back((float)((double)rad * std::sin((double)angle)));
                out.push_back((float)((double)rad * std::cos((double)angle)));
                out.push_back(0.0f);
            }
        }
    } else {
        const unsigned nx = (unsigned)std::floor((double)(e.width / dist));
        const unsigned ny = (unsigned)(e.height / dist);
        const float rw = (float)(nx - 1) * dist, rh = (float)(ny - 1) * dist;
        for (unsigned i = 0; i < nx; ++i)
            for (unsigned j = 0; j < ny; ++j) {
                out.push_back((float)((double)rw * 0.5 - (double)((float)i * dist)));
                out.push_back((float)((double)rh * 0.5 - (double)((float)j * dist)));
                out.push_back(0.0f);
            }
    }
}

DeviceArrays arrays(sph_ctx* c)
{
    DeviceArrays A{};
    A.pos = c->pos; A.vel = c->vel; A.pos_alt = c->pos2; A.vel_alt = c->vel2;
    A.acc = c->acc; A.normal = c->normal; A.predr = c->predr; A.pacc = c->pacc;
    A.rho = c->rho; A.alpha = c->alpha; A.k = c->k; A.kws = c->kws; A.kvws = c->kvws; A.press = c->press;
    A.orig_w = c->orig;
    A.cell_start = c->cell_start; A.cell_sorted = c->cell_sorted;
    A.bpos = c->bpos; A.bcell_start = c->bcell_start;
    A.nbr_f = c->nbr_f; A.cnt_f = c->cnt_f; A.nbr_b = c->nbr_b; A.cnt_b = c->cnt_b;
    A.accum = c->accum; A.st = c->st;
    A.bnormal = c->bnormal; A.bdens = c->bdens; A.bpress = c->bpress; A.bdp = c->bdp;
    A.predv = c->predv; A.cell_entry = c->cell_entry;
    A.plo = c->P.pos_lo ? c->plo : nullptr;
    A.divres = c->divres;
    A.plo_alt = c->P.pos_lo ? c->plo2 : nullptr;
    if (c->nscenes) {
        A.sref.scenes = c->d_scenes;
        A.sref.scene_of = c->d_scene_of;
        A.sst = c->d_sst;
        A.any_active = c->d_any;
        A.nscenes = (int)c->nscenes;
        A.accum_stride = c->accum_stride;
    }
    return A;
}

int check_launch(sph_ctx* c, const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(c, SPH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return SPH_OK;
}

cudaEvent_t take_event(sph_ctx* c)
{
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

/* Brackets one phase with events when profiling; counts its kernel launches. */
struct Phase {
    sph_ctx* c;
    int phase;
    int kernels;
    cudaEvent_t a = nullptr;
    Phase(sph_ctx* ctx, int ph, int nk) : c(ctx), phase(ph), kernels(nk)
    {
        if (c->prof) {
            a = take_event(c);
            cudaEventRecord(a, c->stream);
        }
    }
    ~Phase()
    {
        c->launches += (unsigned long long)kernels;
        if (c->prof) {
            cudaEvent_t b = take_event(c);
            cudaEventRecord(b, c->stream);
            c->pending.push_back({phase, a, b});
            c->prof_launch[phase] += (unsigned long long)kernels;
        }
    }
};

void drain_profile(sph_ctx* c)
{
    for (auto& p : c->pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) c->prof_ms[p.phase] += ms;
        c->ev_pool.push_back(p.a);
        c->ev_pool.push_back(p.b);
    }
    c->pending.clear();
}

int alloc_lists(sph_ctx* c)
{
    int rc;
    if ((rc = dalloc(c, &c->nbr_f, (size_t)c->P.capF * c->nf)) != SPH_OK) return rc;
    if ((rc = dalloc(c, &c->nbr_b, (size_t)c->P.capB * c->nf)) != SPH_OK) return rc;
    return SPH_OK;
}

/* Sort the fluid into cells and rebuild the neighbour lists. */
int neighbor_search(sph_ctx* c)
{
    GatherSet g{};
    if (c->P.dynamic) g.n_dev = &c->st->n_active;
    g.orig_out = c->orig2;
    g.cell_out = c->cell_sorted;
    g.v4_in[0] = c->pos; g.v4_out[0] = c->pos2;
    g.v4_in[1] = c->vel; g.v4_out[1] = c->vel2;
    if (c->P.pos_lo) { g.v4_in[3] = c->plo; g.v4_out[3] = c->plo2; }
    if (c->desc.simulation_method == SPH_DFSPH) {
        g.f_in[0] = c->kws; g.f_out[0] = c->kws2;
        g.f_in[1] = c->kvws; g.f_out[1] = c->kvws2;
        /* PCISPH boundary method: the collision normals of this step feed the
           next step's velocity correction */
        if (c->P.pcib) { g.v4_in[2] = c->normal; g.v4_out[2] = c->normal2; }
    }
    {
        Phase ph(c, SPH_PROF_SORT, 5);
        launch_sort(c->P, SceneRef{c->d_scenes, c->d_scene_of}, (int)c->nf, c->pos, c->cell_count, c->cell_start, c->block_sums, c->cell_of, c->slot,
                    c->tmp_key, c->tmp_src, c->orig, g, c->stream);
    }
    std::swap(c->pos, c->pos2);
    std::swap(c->vel, c->vel2);
    std::swap(c->orig, c->orig2);
    if (c->P.pos_lo) std::swap(c->plo, c->plo2);
    if (c->desc.simulation_method == SPH_DFSPH) {
        std::swap(c->kws, c->kws2);
        std::swap(c->kvws, c->kvws2);
        if (c->P.pcib) std::swap(c->normal, c->normal2);
    }
    {
        Phase ph(c, SPH_PROF_LISTS, 1);
        launch_build_lists(c->P, SceneRef{c->d_scenes, c->d_scene_of}, c->pos, c->cell_start, c->bpos, c->bcell_start, c->nbr_f, c->cnt_f, c->nbr_b,
                           c->cnt_b, c->st, c->stream, c->staged_lists);
    }
    if (c->P.pcib) {
        /* the fluid's cells get candidate lists at this search */
        Phase ph(c, SPH_PROF_LISTS, 2);
        launch_mark_entries(c->P, c->pos, (int)c->nf, c->P.dynamic ? &c->st->n_active : nullptr, c->cell_entry, c->st,
                            true, c->stream);
    }
    c->lists_valid = true;
    return check_launch(c, "neighbour search");
}

/* Cube boundaries after integration (a no-op without them). */
void cube_correct(sph_ctx* c)
{
    if (c->cubes.empty()) return;
    launch_cube_correct(c->P, arrays(c), c->d_cubes, (int)c->cubes.size(), c->stream);
    c->launches += 1;
    c->lists_valid = false;
}

/* Emission of the due emitter groups (a no-op without emitters). */
void emit(sph_ctx* c, bool advance_time)
{
    if (!c->P.dynamic) return;
    launch_emit(c->P, arrays(c), c->d_emit, c->d_group, (int)c->emitters.size(), advance_time, c->stream);
    c->launches += 1;
}

int zero_accum(sph_ctx* c)
{
    CUDA_TRY(c, cudaMemsetAsync(c->accum, 0, c->accum_len * sizeof(double), c->stream));
    if (c->d_any) CUDA_TRY(c, cudaMemsetAsync(c->d_any, 0, 2 * ((size_t)c->P.max_it + 2) * sizeof(unsigned), c->stream));
    return SPH_OK;
}

int step_wcsph(sph_ctx* c)
{
    int rc;
    if ((rc = neighbor_search(c)) != SPH_OK) return rc;
    DeviceArrays A = arrays(c);
    { Phase ph(c, SPH_PROF_DENSITY, 1); launch_density(c->P, A, false, true, c->pass_block, c->stream); }
    if (c->P.pcib) { Phase ph(c, SPH_PROF_DENSITY, 1); launch_boundary_density(c->P, A, c->stream); }
    if (c->P.st_on) { Phase ph(c, SPH_PROF_NORMALS, 1); launch_normals(c->P, A, c->pass_block, c->stream); }
    { Phase ph(c, SPH_PROF_FORCES, 1); launch_forces(c->P, A, FORCE_WCSPH, c->pass_block, c->stream); }
    std::swap(c->pos, c->pos2);
    std::swap(c->vel, c->vel2);
    if (c->P.pos_lo) std::swap(c->plo, c->plo2);
    c->lists_valid = false;
    cube_correct(c); /* WCSPHSolver.cpp:51-60 */
    if (c->P.pcib) { /* WCSPHSolver.cpp:62-72 */
        Phase ph(c, SPH_PROF_FORCES, 1);
        launch_pcib_correct(c->P, arrays(c), true, c->stream);
    }
    emit(c, true); /* WCSPHSolver.cpp:75: emission, then t += dt */
    return check_launch(c, "wcsph step");
}

int step_pcisph(sph_ctx* c)
{
    int rc;
    if ((rc = neighbor_search(c)) != SPH_OK) return rc;
    DeviceArrays A = arrays(c);
    { Phase ph(c, SPH_PROF_DENSITY, 1); launch_density(c->P, A, false, false, c->pass_block, c->stream); }
    if (c->P.st_on) { Phase ph(c, SPH_PROF_NORMALS, 1); launch_normals(c->P, A, c->pass_block, c->stream); }
    { Phase ph(c, SPH_PROF_FORCES, 1); launch_forces(c->P, A, FORCE_NP, c->pass_block, c->stream); }
    if ((rc = zero_accum(c)) != SPH_OK) return rc;
    int e;
    { Phase ph(c, SPH_PROF_PRESSURE_SOLVE, 1); e = launch_pcisph_solve(c->P, A, c->grid_pcisph, c->stream); }
    if (e != 0) return fail(c, SPH_ERR_CUDA, std::string("pcisph solver launch: ") + cudaGetErrorString((cudaError_t)e));
    c->lists_valid = !c->P.dynamic && c->cubes.empty();
    cube_correct(c); /* PCISPHSolver.cpp:53-62 */
    emit(c, true); /* PCISPHSolver.cpp:77: emission, then t += dt */
    return check_launch(c, "pcisph step");
}

int tpp_index(int tpp) { return tpp == 4 ? 2 : tpp == 2 ? 1 : 0; }

int solve_grid(const sph_ctx* c, bool divergence)
{
    return c->grid_solve[divergence ? 1 : 0][c->solver_occ == 4 ? 1 : 0][tpp_index(c->solver_tpp)];
}

int step_dfsph(sph_ctx* c)
{
    int rc;
    DeviceArrays A = arrays(c);
    if (c->P.st_on) { Phase ph(c, SPH_PROF_NORMALS, 1); launch_normals(c->P, A, c->pass_block, c->stream); }
    { Phase ph(c, SPH_PROF_FORCES, 1); launch_forces(c->P, A, FORCE_NP_CFL, c->pass_block, c->stream); }
    if ((rc = zero_accum(c)) != SPH_OK) return rc;
    int e;
    {
        Phase ph(c, SPH_PROF_DENSITY_SOLVE, 1);
        e = c->nscenes ? launch_dfsph_solve_batch(c->P, A, false, c->grid_batch_density, c->stream)
                       : launch_dfsph_solve(c->P, A, false, solve_grid(c, false), c->solver_occ, c->solver_tpp, c->stream);
    }
    if (e != 0) return fail(c, SPH_ERR_CUDA, std::string("dfsph density solver launch: ") + cudaGetErrorString((cudaError_t)e));
    if (c->P.pcib) { /* DFSPHSolver.cpp:60-70 */
        Phase ph(c, SPH_PROF_DENSITY_SOLVE, 1);
        launch_pcib_correct(c->P, A, false, c->stream);
    }
    emit(c, false); /* DFSPHSolver.cpp:72: after the position update, before the neighbour search */
    if ((rc = neighbor_search(c)) != SPH_OK) return rc;
    A = arrays(c);
    { Phase ph(c, SPH_PROF_DENSITY, 1); launch_density(c->P, A, true, false, c->pass_block, c->stream); }
    A.accum = c->accum + c->accum_len / 2;
    if (c->d_any) A.any_active = c->d_any + ((size_t)c->P.max_it + 2);
    {
        Phase ph(c, SPH_PROF_DIVERGENCE_SOLVE, 1);
        e = c->nscenes ? launch_dfsph_solve_batch(c->P, A, true, c->grid_batch_div, c->stream)
                       : launch_dfsph_solve(c->P, A, true, solve_grid(c, true), c->solver_occ, c->solver_tpp, c->stream);
    }
    if (e != 0) return fail(c, SPH_ERR_CUDA, std::string("dfsph divergence solver launch: ") + cudaGetErrorString((cudaError_t)e));
    cube_correct(c); /* DFSPHSolver.cpp:94-103 */
    if (!c->cubes.empty()) {
        /* The next step's force and solver passes run on this step's lists,
           but the cube correction has moved particles since they were built.
           SPH2O's loops take the candidates of the cells around each
           particle's current position, with the cell contents of the last
           insertion, and evaluate distances at current positions: rebuild
           the lists from the current positions against the same cell table. */
        Phase ph(c, SPH_PROF_LISTS, 1);
        launch_build_lists(c->P, SceneRef{c->d_scenes, c->d_scene_of}, c->pos, c->cell_start, c->bpos, c->bcell_start,
                           c->nbr_f, c->cnt_f, c->nbr_b, c->cnt_b, c->st, c->stream);
    }
    return check_launch(c, "dfsph step");
}

int read_state(sph_ctx* c, DevState* out)
{
    CUDA_TRY(c, cudaMemcpyAsync(c->st_host, c->st, sizeof(DevState), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    *out = *c->st_host;
    return SPH_OK;
}

/* Active fluid particles (reads the device state; waits for queued work). */
int active_count(sph_ctx* c, unsigned* n)
{
    if (!c->P.dynamic) { *n = c->nf; return SPH_OK; }
    DevState s{};
    const int rc = read_state(c, &s);
    if (rc != SPH_OK) return rc;
    *n = s.n_active;
    return SPH_OK;
}

int status_from_state(sph_ctx* c, const DevState& s)
{
    if (s.err & ERRBIT_TIMEOUT) return fail(c, SPH_ERR_TIMEOUT, "a bounded device-side barrier gave up");
    if (s.err & ERRBIT_NAN) return fail(c, SPH_ERR_NAN, "non-finite particle position");
    if (s.err & ERRBIT_OVERFLOW) return fail(c, SPH_ERR_NEIGHBOR_OVERFLOW, "neighbour list capacity exceeded");
    return SPH_OK;
}

/* After an overflow: clear the flag and grow the lists for later steps. */
int recover_overflow(sph_ctx* c)
{
    int zero = 0;
    unsigned uzero = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&c->st->err, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(&c->st->overflow, &uzero, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    auto drop = [&](unsigned* p) {
        auto it = std::find(c->allocations.begin(), c->allocations.end(), (void*)p);
        if (it != c->allocations.end()) { cudaFree(p); c->allocations.erase(it); }
    };
    drop_graphs(c);
    drop(c->nbr_f);
    drop(c->nbr_b);
    c->P.capF = c->P.capF + c->P.capF / 2;
    c->P.capB = c->P.capB + c->P.capB / 2;
    c->lists_valid = false;
    return alloc_lists(c);
}

int fill_stats(sph_ctx* c, const DevState& before, const DevState& now, sph_step_stats* out)
{
    if (!out) return SPH_OK;
    std::memset(out, 0, sizeof *out);
    out->time = now.time;
    out->dt = now.dt;
    out->avg_density_error = now.avg_dens;
    out->avg_divergence_error = now.avg_div;
    out->max_velocity = now.last_vmax;
    out->iterations = now.its;
    out->iterations_v = now.its_v;
    out->total_iterations = now.sum_its - before.sum_its;
    out->total_iterations_v = now.sum_its_v - before.sum_its_v;
    out->steps = now.steps - before.steps;
    out->neighbor_overflows = now.overflow;
    (void)c;
    return SPH_OK;
}

unsigned buffer_key(const sph_ctx* c)
{
    return (c->pos == c->pos_base ? 1u : 0u) | (c->orig == c->orig_base ? 2u : 0u) | (c->kws == c->kws_base ? 4u : 0u);
}

void drop_graphs(sph_ctx* c)
{
    for (auto& g : c->graphs) cudaGraphExecDestroy(g.exec);
    c->graphs.clear();
    for (auto& g : c->adj.graphs) cudaGraphExecDestroy(g.exec);
    c->adj.graphs.clear();
}

int eager_step(sph_ctx* c)
{
    switch (c->desc.simulation_method) {
    case SPH_WCSPH: return step_wcsph(c);
    case SPH_PCISPH: return step_pcisph(c);
    default: return step_dfsph(c);
    }
}

Buffers get_buffers(const sph_ctx* c)
{
    return {c->pos, c->pos2, c->vel, c->vel2, c->orig, c->orig2, c->kws, c->kws2, c->kvws, c->kvws2, c->normal,
            c->normal2, c->plo, c->plo2, c->lists_valid};
}

void set_buffers(sph_ctx* c, const Buffers& b)
{
    c->pos = b.pos; c->pos2 = b.pos2; c->vel = b.vel; c->vel2 = b.vel2; c->orig = b.orig; c->orig2 = b.orig2;
    c->kws = b.kws; c->kws2 = b.kws2; c->kvws = b.kvws; c->kvws2 = b.kvws2; c->lists_valid = b.lists_valid;
    c->normal = b.normal; c->normal2 = b.normal2;
    c->plo = b.plo; c->plo2 = b.plo2;
}

/* nsteps (1 or 2) steps as one CUDA graph, captured on first use for the
   current buffer assignment (which the key determines) and replayed
   afterwards; a replay leaves the host-side assignment where the captured
   steps left it. Returns false when capture is not possible (the caller
   then steps eagerly and stops trying). */
bool graph_steps(sph_ctx* c, int nsteps, int* rc)
{
    const unsigned key = buffer_key(c) | ((unsigned)nsteps << 8);
    for (auto& g : c->graphs)
        if (g.key == key) {
            const cudaError_t e = cudaGraphLaunch(g.exec, c->stream);
            if (e != cudaSuccess) { *rc = fail(c, SPH_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e)); return true; }
            set_buffers(c, g.end);
            c->launches += g.launches;
            *rc = SPH_OK;
            return true;
        }
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    /* captured work never runs during capture: the swaps it makes on the host
       are undone afterwards and applied by the replay */
    const Buffers start = get_buffers(c);
    const unsigned long long l0 = c->launches;
    int r = SPH_OK;
    for (int n = 0; n < nsteps && r == SPH_OK; ++n) r = eager_step(c);
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &graph);
    const unsigned long long nl = c->launches - l0;
    c->launches = l0;
    const Buffers end = get_buffers(c);
    set_buffers(c, start);
    cudaGraphExec_t exec = nullptr;
    const bool ok = r == SPH_OK && ec == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
        cudaGetLastError();
        c->err.clear();
        return false;
    }
    c->graphs.push_back({key, exec, nl, end});
    return graph_steps(c, nsteps, rc);
}

/* Queue nsteps steps: pairs (and a remaining single step) replay captured
   graphs; while profiling every step runs eagerly. */
int run_steps(sph_ctx* c, int nsteps)
{
    int left = nsteps;
    while (left > 0) {
        int rc = SPH_OK;
        if (c->use_graphs && !c->prof) {
            const int n = left >= 2 ? 2 : 1;
            if (graph_steps(c, n, &rc)) {
                if (rc != SPH_OK) return rc;
                left -= n;
                continue;
            }
            c->use_graphs = false;  /* capture unsupported: stay eager */
            drop_graphs(c);
        }
        rc = eager_step(c);
        if (rc != SPH_OK) return rc;
        --left;
    }
    return SPH_OK;
}

} // namespace

extern "C" {

int sph_select_device(int device)
{
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, SPH_ERR_NO_DEVICE, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return SPH_OK;
}

int sph_create(const sph_scene_desc* desc, sph_ctx** out)
{
    if (!desc || !out) return fail(nullptr, SPH_ERR_ARG, "null argument");
    *out = nullptr;
    if (desc->simulation_method < SPH_WCSPH || desc->simulation_method > SPH_DFSPH)
        return fail(nullptr, SPH_ERR_ARG, "simulation_method must be 0, 1 or 2");
    if (desc->boundary_method < SPH_BOUNDARY_CUBE || desc->boundary_method > SPH_BOUNDARY_AKINCI)
        return fail(nullptr, SPH_ERR_ARG, "boundary_method must be 0 (cube), 1 (PCISPH) or 2 (Akinci)");
    if (desc->boundary_method == SPH_BOUNDARY_PCISPH && desc->adhesion_method == SPH_ADHESION_AKINCI &&
        desc->adhesion != 0.0f)
        /* AdhesionForce reads Akinci volumes (AdhesionForce.cpp:22-29) */
        return fail(nullptr, SPH_ERR_ARG, "adhesion needs Akinci boundary particles (boundary method 2)");
    if (!(desc->particle_radius > 0.0f) || !(desc->density0 > 0.0f) || !(desc->time_step > 0.0f) || !(desc->fps > 0.0f))
        return fail(nullptr, SPH_ERR_ARG, "particle_radius, density0, time_step and fps must be positive");
    if (desc->simulation_method == SPH_WCSPH && !(desc->gamma != 0.0f))
        return fail(nullptr, SPH_ERR_ARG, "WCSPH needs a non-zero gamma");
    if (desc->simulation_method != SPH_WCSPH && desc->max_iterations > 100000)
        return fail(nullptr, SPH_ERR_ARG, "max_iterations above 100000");
    if (desc->flags != 0) return fail(nullptr, SPH_ERR_ARG, "flags must be 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, SPH_ERR_NO_DEVICE, "no CUDA device available");
    sph_ctx* c = new (std::nothrow) sph_ctx();
    if (!c) return fail(nullptr, SPH_ERR_ARG, "out of host memory");
    c->desc = *desc;
    cudaGetDevice(&c->device);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return fail(nullptr, SPH_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    derive_params(c);
    *out = c;
    return SPH_OK;
}

int sph_set_fluid(sph_ctx* c, unsigned n, const float* xyz, const float* v)
{
    if (!c) return SPH_ERR_ARG;
    if (c->nscenes) return fail(c, SPH_ERR_STATE, "batch contexts take particles through sph_batch_set_scene");
    if (c->initialized) return fail(c, SPH_ERR_STATE, "sph_set_fluid after sph_init; use sph_set_state");
    if (n > 0 && !xyz) return fail(c, SPH_ERR_ARG, "null positions");
    c->nf = n;
    c->h_fluid.assign(xyz, xyz + 3ull * n);
    if (v) c->h_vel.assign(v, v + 3ull * n);
    else c->h_vel.assign(3ull * n, 0.0f);
    return SPH_OK;
}

int sph_set_boundary(sph_ctx* c, unsigned n, const float* xyz)
{
    if (!c) return SPH_ERR_ARG;
    if (c->nscenes) return fail(c, SPH_ERR_STATE, "batch contexts take particles through sph_batch_set_scene");
    if (c->initialized) return fail(c, SPH_ERR_STATE, "sph_set_boundary after sph_init");
    if (n > 0 && !xyz) return fail(c, SPH_ERR_ARG, "null positions");
    c->nb = n;
    c->h_bound.assign(xyz, xyz + 3ull * n);
    return SPH_OK;
}

int sph_set_boundary_normals(sph_ctx* c, unsigned n, const float* normals, float normal_fct, float tangential_fct)
{
    if (!c) return SPH_ERR_ARG;
    if (c->initialized) return fail(c, SPH_ERR_STATE, "sph_set_boundary_normals after sph_init");
    if (c->desc.boundary_method != SPH_BOUNDARY_PCISPH)
        return fail(c, SPH_ERR_ARG, "boundary normals need boundary_method SPH_BOUNDARY_PCISPH");
    if (n != c->nb) return fail(c, SPH_ERR_ARG, "one normal per boundary particle (call sph_set_boundary first)");
    if (n > 0 && !normals) return fail(c, SPH_ERR_ARG, "null normals");
    c->h_bnormal.assign(normals, normals + 3ull * n);
    c->pcib_nf = normal_fct;
    c->pcib_tf = tangential_fct;
    return SPH_OK;
}

int sph_add_cube_boundary(sph_ctx* c, const float mn[3], const float mx[3], float normal_fct, float tangential_fct)
{
    if (!c || !mn || !mx) return SPH_ERR_ARG;
    if (c->nscenes) return fail(c, SPH_ERR_ARG, "cube boundaries apply to single scenes, not to batches");
    if (c->initialized) return fail(c, SPH_ERR_STATE, "sph_add_cube_boundary after sph_init");
    if (c->desc.boundary_method != SPH_BOUNDARY_CUBE)
        return fail(c, SPH_ERR_ARG, "cube boundaries need boundary_method SPH_BOUNDARY_CUBE");
    c->cubes.push_back({mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], normal_fct, tangential_fct});
    return SPH_OK;
}

int sph_add_emitter(sph_ctx* c, const sph_emitter_desc* e)
{
    if (!c || !e) return SPH_ERR_ARG;
    if (c->nscenes) return fail(c, SPH_ERR_ARG, "emitters apply to single scenes, not to batches");
    if (c->initialized) return fail(c, SPH_ERR_STATE, "sph_add_emitter after sph_init");
    if (e->type != SPH_EMITTER_SQUARE && e->type != SPH_EMITTER_CIRCLE)
        return fail(c, SPH_ERR_ARG, "emitter type must be 0 (square) or 1 (circle)");
    if (!(e->velocity > 0.0f) || !(e->spacing > 0.0f)) return fail(c, SPH_ERR_ARG, "emitter velocity and spacing must be > 0");
    if ((unsigned long long)c->nf + e->num_particles > (1ull << 31)) return fail(c, SPH_ERR_CAPACITY, "too many particles");
    c->emitters.push_back(*e);
    return SPH_OK;
}

int sph_get_num_active(sph_ctx* c, unsigned* n)
{
    if (!c || !n) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_get_num_active before sph_init");
    return active_count(c, n);
}

int sph_init(sph_ctx* c)
{
    if (!c) return SPH_ERR_ARG;
    if (c->initialized) return fail(c, SPH_ERR_STATE, "sph_init called twice");
    if (c->nf == 0 && c->nscenes == 0) return fail(c, SPH_ERR_ARG, "no fluid particles");
    CUDA_TRY(c, cudaSetDevice(c->device));
    SimParams& P = c->P;
    if (c->nscenes) {
        /* concatenate the scenes in scene order */
        c->fsplit.assign(1, 0u);
        c->bsplit.assign(1, 0u);
        c->h_fluid.clear(); c->h_vel.clear(); c->h_bound.clear();
        for (unsigned s = 0; s < c->nscenes; ++s) {
            if (c->sc_fluid[s].empty()) return fail(c, SPH_ERR_ARG, "scene " + std::to_string(s) + " has no fluid");
            c->h_fluid.insert(c->h_fluid.end(), c->sc_fluid[s].begin(), c->sc_fluid[s].end());
            c->h_vel.insert(c->h_vel.end(), c->sc_vel[s].begin(), c->sc_vel[s].end());
            c->h_bound.insert(c->h_bound.end(), c->sc_bound[s].begin(), c->sc_bound[s].end());
            c->fsplit.push_back((unsigned)(c->h_fluid.size() / 3));
            c->bsplit.push_back((unsigned)(c->h_bound.size() / 3));
        }
        c->nf = c->fsplit.back();
        c->nb = c->bsplit.back();
    }
    if (c->desc.boundary_method == SPH_BOUNDARY_CUBE && c->nb > 0)
        return fail(c, SPH_ERR_ARG, "the cube boundary method has no boundary particles");
    if (c->P.pcib) {
        if (c->nscenes) return fail(c, SPH_ERR_ARG, "the PCISPH boundary method applies to single scenes");
        if (c->h_bnormal.size() != 3ull * c->nb)
            return fail(c, SPH_ERR_ARG, "PCISPH boundary particles need their normals (sph_set_boundary_normals)");
        P.pcib_nf = c->pcib_nf;
        P.pcib_tf = c->pcib_tf;
    }
    /* emitters: their particles are allocated inactive after the blocks */
    c->n_init = c->nf;
    std::vector<float> groups;
    std::vector<EmitterState> etab;
    if (!c->emitters.empty()) {
        unsigned extra = 0;
        for (const sph_emitter_desc& e : c->emitters) {
            EmitterState es{};
            es.px = e.position[0]; es.py = e.position[1]; es.pz = e.position[2];
            es.qw = e.rotation[0]; es.qx = e.rotation[1]; es.qy = e.rotation[2]; es.qz = e.rotation[3];
            es.v = e.velocity;
            es.next = e.start_time;
            /* nextTimeEmit += spacing * 1.105 * dist / v (Emitter.cpp:124) */
            es.period = e.spacing * 1.105f * (2.0f * c->desc.particle_radius) / e.velocity;
            es.remaining = e.num_particles;
            es.group_begin = (unsigned)(groups.size() / 3);
            emitter_group(e, c->desc.particle_radius, groups);
            es.group_count = (unsigned)(groups.size() / 3) - es.group_begin;
            etab.push_back(es);
            extra += e.num_particles;
        }
        c->nf += extra;
        c->h_fluid.resize(3ull * c->nf, 0.0f);
        c->h_vel.resize(3ull * c->nf, 0.0f);
        P.dynamic = 1;
    }
    P.nf = (int)c->nf;
    P.nb = (int)c->nb;

    if (c->nscenes) {
        /* one grid per scene, each owning a disjoint range of the cell table */
        unsigned long long base = 0;
        c->h_scenes.resize(c->nscenes);
        for (unsigned s = 0; s < c->nscenes; ++s) {
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (const std::vector<float>* a : {&c->sc_fluid[s], &c->sc_bound[s]})
                for (size_t i = 0; i + 2 < a->size(); i += 3)
                    for (int k = 0; k < 3; ++k) {
                        const float v = (*a)[i + k];
                        if (!std::isfinite(v)) continue;
                        lo[k] = std::min(lo[k], (double)v);
                        hi[k] = std::max(hi[k], (double)v);
                    }
            SceneInfo& si = c->h_scenes[s];
            int dim[3], cmin[3];
            for (int k = 0; k < 3; ++k) {
                cmin[k] = (int)std::floor(lo[k] / P.h) - 2;
                const int b = (int)std::floor(hi[k] / P.h) + 2;
                dim[k] = ((b - cmin[k] + 1) + 3) / 4 * 4;
            }
            si.grid.cminx = cmin[0]; si.grid.cminy = cmin[1]; si.grid.cminz = cmin[2];
            si.grid.dimx = dim[0]; si.grid.dimy = dim[1]; si.grid.dimz = dim[2];
            si.grid.nbx = dim[0] / 4; si.grid.nby = dim[1] / 4;
            si.grid.base = (unsigned)base;
            si.grid.order = P.cell_order;
            base += (unsigned long long)dim[0] * dim[1] * dim[2];
            if (base > (1ull << 28)) return fail(c, SPH_ERR_CAPACITY, "batch too large: more than 2^28 grid cells");
            const sph_scene_desc& ds = c->descs[s];
            si.visc = ds.viscosity;
            si.bvisc = ds.boundary_viscosity;
            si.fbegin = c->fsplit[s]; si.fend = c->fsplit[s + 1];
            si.bbegin = c->bsplit[s]; si.bend = c->bsplit[s + 1];
        }
        const SceneInfo& s0 = c->h_scenes[0];
        P.cminx = s0.grid.cminx; P.cminy = s0.grid.cminy; P.cminz = s0.grid.cminz;
        P.dimx = s0.grid.dimx; P.dimy = s0.grid.dimy; P.dimz = s0.grid.dimz;
        P.nbx = s0.grid.nbx; P.nby = s0.grid.nby;
        P.ncells = (unsigned)((base + 4095) / 4096 * 4096);
        P.capF = 64;
        P.capB = 64;
    } else {
    /* grid over the particle bounding box (+ hint), 2 cells of margin */
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    auto grow = [&](const std::vector<float>& a) {
        for (size_t i = 0; i + 2 < a.size(); i += 3)
            for (int k = 0; k < 3; ++k) {
                if (!std::isfinite(a[i + k])) continue;
                lo[k] = std::min(lo[k], (double)a[i + k]);
                hi[k] = std::max(hi[k], (double)a[i + k]);
            }
    };
    grow(std::vector<float>(c->h_fluid.begin(), c->h_fluid.begin() + 3ull * c->n_init));
    grow(c->h_bound);
    /* cube boundaries keep the fluid inside their boxes */
    for (const CubeBox& b : c->cubes) grow({b.minx, b.miny, b.minz, b.maxx, b.maxy, b.maxz});
    /* emitted particles start around their emitter */
    for (const sph_emitter_desc& e : c->emitters) {
        const float ext = std::max(e.width, e.height) + 4.0f * P.h;
        grow({e.position[0] - ext, e.position[1] - ext, e.position[2] - ext, e.position[0] + ext, e.position[1] + ext,
              e.position[2] + ext});
    }
    const sph_scene_desc& d = c->desc;
    if (d.domain_min[0] != 0 || d.domain_min[1] != 0 || d.domain_min[2] != 0 || d.domain_max[0] != 0 ||
        d.domain_max[1] != 0 || d.domain_max[2] != 0)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], (double)d.domain_min[k]);
            hi[k] = std::max(hi[k], (double)d.domain_max[k]);
        }
    int cmin[3], dim[3];
    for (int k = 0; k < 3; ++k) {
        const int a = (int)std::floor(lo[k] / P.h) - 2;
        const int b = (int)std::floor(hi[k] / P.h) + 2;
        cmin[k] = a;
        dim[k] = ((b - a + 1) + 3) / 4 * 4;
    }
    const unsigned long long ncells = (unsigned long long)dim[0] * dim[1] * dim[2];
    if (ncells > (1ull << 27))
        return fail(c, SPH_ERR_CAPACITY, "domain too large: more than 2^27 grid cells of size h");
    P.cminx = cmin[0]; P.cminy = cmin[1]; P.cminz = cmin[2];
    P.dimx = dim[0]; P.dimy = dim[1]; P.dimz = dim[2];
    P.nbx = dim[0] / 4; P.nby = dim[1] / 4;
    P.ncells = (unsigned)((ncells + 4095) / 4096 * 4096);
    P.capF = 64;
    P.capB = 64;
    }

    const size_t nf = c->nf, nb = c->nb, nmax = std::max(nf, nb);
    int rc = SPH_OK;
#define ALLOC(ptr, count) if ((rc = dalloc(c, &c->ptr, (count))) != SPH_OK) return rc
    ALLOC(pos, nf); ALLOC(vel, nf); ALLOC(pos2, nf); ALLOC(vel2, nf);
    ALLOC(orig, nf); ALLOC(orig2, nf);
    ALLOC(kws, nf); ALLOC(kws2, nf); ALLOC(kvws, nf); ALLOC(kvws2, nf);
    ALLOC(acc, nf); ALLOC(rho, nf); ALLOC(alpha, nf); ALLOC(k, nf); ALLOC(press, nf);
    ALLOC(normal, nf); ALLOC(predr, nf); ALLOC(pacc, nf);
    ALLOC(cell_of, nmax); ALLOC(slot, nmax); ALLOC(tmp_key, nmax); ALLOC(tmp_src, nmax); ALLOC(cell_sorted, nmax);
    ALLOC(cell_count, (size_t)P.ncells); ALLOC(cell_start, (size_t)P.ncells + 1);
    ALLOC(bcell_start, (size_t)P.ncells + 1); ALLOC(block_sums, (size_t)P.ncells / 4096 + 1);
    ALLOC(bpos, nb); ALLOC(bvol, nb); ALLOC(borig, nb);
    ALLOC(cnt_f, nf); ALLOC(cnt_b, nf);
    ALLOC(st, 1);
    if (P.pcib) {
        ALLOC(bnormal, nb); ALLOC(bdens, nb); ALLOC(bpress, nb); ALLOC(bdp, nb);
        ALLOC(predv, nf); ALLOC(normal2, nf);
        ALLOC(cell_entry, (size_t)P.ncells);
    }
#undef ALLOC
    c->pos_base = c->pos;
    c->orig_base = c->orig;
    c->kws_base = c->kws;
    if ((rc = alloc_lists(c)) != SPH_OK) return rc;
    if (c->desc.simulation_method == SPH_DFSPH && (rc = dalloc(c, &c->divres, nf)) != SPH_OK) return rc;
    if (c->pos_lo) {
        if (c->nscenes) return fail(c, SPH_ERR_ARG, "position residuals apply to single scenes, not to batches");
        if ((rc = dalloc(c, &c->plo, nf)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->plo2, nf)) != SPH_OK) return rc;
        P.pos_lo = 1;
    }
    c->accum_len = 2 * ((size_t)P.max_it + 2) * std::max(1u, c->nscenes);
    if ((rc = dalloc(c, &c->accum, c->accum_len)) != SPH_OK) return rc;
    if (c->nscenes) {
        const unsigned ns = c->nscenes;
        c->accum_stride = P.max_it + 2;
        if ((rc = dalloc(c, &c->d_scenes, ns)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->d_sst, ns)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->d_scene_of, nf)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->d_bscene_of, std::max<size_t>(nb, 1))) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->d_any, 2 * ((size_t)P.max_it + 2))) != SPH_OK) return rc;
        std::vector<unsigned> so(nf), bso(nb);
        std::vector<SceneState> sst(ns);
        for (unsigned s = 0; s < ns; ++s) {
            for (unsigned i = c->fsplit[s]; i < c->fsplit[s + 1]; ++i) so[i] = s;
            for (unsigned i = c->bsplit[s]; i < c->bsplit[s + 1]; ++i) bso[i] = s;
            sst[s] = SceneState{};
            sst[s].dt = c->descs[s].time_step;
        }
        CUDA_TRY(c, cudaMemcpyAsync(c->d_scenes, c->h_scenes.data(), ns * sizeof(SceneInfo), cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(c->d_sst, sst.data(), ns * sizeof(SceneState), cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(c->d_scene_of, so.data(), nf * 4, cudaMemcpyHostToDevice, c->stream));
        if (nb) CUDA_TRY(c, cudaMemcpyAsync(c->d_bscene_of, bso.data(), nb * 4, cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        c->grid_batch_density = persistent_grid(false, false, true);
        c->grid_batch_div = persistent_grid(false, true, true);
        if (c->grid_batch_density <= 0 || c->grid_batch_div <= 0)
            return fail(c, SPH_ERR_CUDA, "cannot size the persistent batch solver grid");
    }
    CUDA_TRY(c, cudaMallocHost((void**)&c->st_host, sizeof(DevState)));
    CUDA_TRY(c, cudaEventCreate(&c->ev_begin));
    CUDA_TRY(c, cudaEventCreate(&c->ev_end));

    c->grid_pcisph = persistent_grid(true, false);
    if (c->grid_pcisph <= 0) return fail(c, SPH_ERR_CUDA, "cannot size the persistent solver grid");
    for (int dv = 0; dv < 2; ++dv)
        for (int o = 0; o < 2; ++o)
            for (int t = 0; t < 3; ++t) {
                c->grid_solve[dv][o][t] = persistent_grid(false, dv == 1, false, o ? 4 : 8, 1 << t);
                if (c->grid_solve[dv][o][t] <= 0) return fail(c, SPH_ERR_CUDA, "cannot size the persistent solver grid");
            }

    /* upload: fluid in caller order becomes the first "unsorted" state */
    float* stage = nullptr;
    const size_t stage_n = 3 * std::max<size_t>(nmax, 1);
    CUDA_TRY(c, cudaMalloc(&stage, stage_n * sizeof(float)));
    c->allocations.push_back(stage);
    CUDA_TRY(c, cudaMemcpyAsync(stage, c->h_fluid.data(), 3 * nf * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    launch_pack_v3((int)nf, stage, c->pos, 0.0f, c->stream);
    CUDA_TRY(c, cudaMemcpyAsync(stage, c->h_vel.data(), 3 * nf * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    launch_pack_v3((int)nf, stage, c->vel, 0.0f, c->stream);
    launch_iota((int)nf, c->orig, c->stream);

    /* boundary: sort once, volumes (SPHSolver::init, SPHSolver.cpp:21-38) */
    if (nb > 0) {
        if ((rc = dalloc(c, &c->braw, nb)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->bid, nb)) != SPH_OK) return rc;
        float4* braw = c->braw;
        unsigned* bid = c->bid;
        CUDA_TRY(c, cudaMemcpyAsync(stage, c->h_bound.data(), 3 * nb * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        /* w: the particle's density weight, rho0 V_b once the volumes are
           known (Akinci) or the boundary mass m_b = rho0 (2r)^3 (PCISPH,
           SPHSimulation.cpp:435-437), which equals the fluid mass */
        launch_pack_v3((int)nb, stage, braw, P.pcib ? P.mass : 0.0f, c->stream);
        launch_iota((int)nb, bid, c->stream);
        GatherSet g{};
        g.orig_out = c->borig;
        g.v4_in[0] = braw;
        g.v4_out[0] = c->bpos;
        float4* nraw = nullptr;
        if (P.pcib) {
            if ((rc = dalloc(c, &nraw, nb)) != SPH_OK) return rc;
            CUDA_TRY(c, cudaStreamSynchronize(c->stream)); /* the stage buffer is reused */
            CUDA_TRY(c, cudaMemcpyAsync(stage, c->h_bnormal.data(), 3 * nb * sizeof(float), cudaMemcpyHostToDevice,
                                        c->stream));
            launch_pack_v3((int)nb, stage, nraw, 0.0f, c->stream);
            g.v4_in[1] = nraw;
            g.v4_out[1] = c->bnormal;
        }
        const SceneRef bref{c->d_scenes, c->d_bscene_of};
        launch_sort(P, bref, (int)nb, braw, c->cell_count, c->bcell_start, c->block_sums, c->cell_of, c->slot,
                    c->tmp_key, c->tmp_src, bid, g, c->stream);
        if (!P.pcib) launch_boundary_volume(P, bref, c->bpos, c->bcell_start, c->bvol, c->stream);
    } else {
        CUDA_TRY(c, cudaMemsetAsync(c->bcell_start, 0, ((size_t)P.ncells + 1) * sizeof(unsigned), c->stream));
    }

    if (!c->cubes.empty()) {
        if ((rc = dalloc(c, &c->d_cubes, c->cubes.size())) != SPH_OK) return rc;
        CUDA_TRY(c, cudaMemcpyAsync(c->d_cubes, c->cubes.data(), c->cubes.size() * sizeof(CubeBox), cudaMemcpyHostToDevice,
                                    c->stream));
    }
    if (!etab.empty()) {
        if ((rc = dalloc(c, &c->d_emit, etab.size())) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->snap_emit, etab.size())) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->d_group, std::max<size_t>(groups.size() / 3, 1))) != SPH_OK) return rc;
        std::vector<float4> g4(groups.size() / 3);
        for (size_t k = 0; k < g4.size(); ++k) g4[k] = make_float4(groups[3 * k], groups[3 * k + 1], groups[3 * k + 2], 0.0f);
        CUDA_TRY(c, cudaMemcpyAsync(c->d_emit, etab.data(), etab.size() * sizeof(EmitterState), cudaMemcpyHostToDevice,
                                    c->stream));
        if (!g4.empty())
            CUDA_TRY(c, cudaMemcpyAsync(c->d_group, g4.data(), g4.size() * sizeof(float4), cudaMemcpyHostToDevice,
                                        c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }

    /* solver state */
    DevState s0{};
    s0.dt = c->desc.time_step;
    s0.n_active = c->n_init;
    CUDA_TRY(c, cudaMemcpyAsync(c->st, &s0, sizeof s0, cudaMemcpyHostToDevice, c->stream));
    /* PCISPH boundary method: the boundary's cells hold lists from the first
       search on (SPHSolver::init inserts the boundary first) */
    if (P.pcib) launch_mark_entries(P, c->bpos, (int)nb, nullptr, c->cell_entry, c->st, false, c->stream);
    if ((rc = neighbor_search(c)) != SPH_OK) return rc;
    if (c->desc.simulation_method == SPH_DFSPH) {
        /* DFSPHSolver::init: densities and alpha at the initial positions */
        launch_density(P, arrays(c), true, false, c->pass_block, c->stream);
    }
    if ((rc = check_launch(c, "init")) != SPH_OK) return rc;
    DevState now{};
    if ((rc = read_state(c, &now)) != SPH_OK) return rc;
    c->last = now;
    c->initialized = true;
    if ((rc = status_from_state(c, now)) != SPH_OK) return rc;
    return SPH_OK;
}

int sph_step_async(sph_ctx* c, int nsteps)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_step before sph_init");
    if (nsteps < 0) return fail(c, SPH_ERR_ARG, "negative step count");
    if (!c->batch_open) {
        CUDA_TRY(c, cudaEventRecord(c->ev_begin, c->stream));
        c->batch_open = true;
        c->launches_at_open = c->launches;
    }
    const int rc = run_steps(c, nsteps);
    if (rc != SPH_OK) return rc;
    CUDA_TRY(c, cudaEventRecord(c->ev_end, c->stream));
    return SPH_OK;
}

int sph_sync(sph_ctx* c, sph_step_stats* out)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_sync before sph_init");
    DevState now{};
    int rc = read_state(c, &now);
    if (rc != SPH_OK) return rc;
    fill_stats(c, c->last, now, out);
    if (c->nscenes) {
        /* batch: time/dt of the slowest scene, iterations summed over scenes */
        std::vector<SceneState> sst(c->nscenes);
        CUDA_TRY(c, cudaMemcpy(sst.data(), c->d_sst, c->nscenes * sizeof(SceneState), cudaMemcpyDeviceToHost));
        if (out) {
            if (c->last_sst.size() != sst.size()) c->last_sst.assign(sst.size(), SceneState{});
            double tmin = 1e300;
            float dtmin = 3e38f;
            unsigned long long its = 0, itsv = 0;
            unsigned mx = 0, mxv = 0;
            double avg = 0.0, avgv = 0.0;
            for (unsigned s = 0; s < c->nscenes; ++s) {
                tmin = std::min(tmin, sst[s].time);
                dtmin = std::min(dtmin, sst[s].dt);
                its += sst[s].sum_its - c->last_sst[s].sum_its;
                itsv += sst[s].sum_its_v - c->last_sst[s].sum_its_v;
                mx = std::max(mx, sst[s].its);
                mxv = std::max(mxv, sst[s].its_v);
                avg = std::max(avg, sst[s].avg_dens);
                avgv = std::max(avgv, sst[s].avg_div);
            }
            out->time = tmin;
            out->dt = dtmin;
            out->iterations = mx;
            out->iterations_v = mxv;
            out->total_iterations = its;
            out->total_iterations_v = itsv;
            out->avg_density_error = avg;
            out->avg_divergence_error = avgv;
            out->steps = sst[0].steps - c->last_sst[0].steps;
        }
        c->last_sst = sst;
    }
    if (c->batch_open) {
        float ms = 0.0f;
        if (out && cudaEventElapsedTime(&ms, c->ev_begin, c->ev_end) == cudaSuccess) out->device_ms = ms;
        if (out) out->kernel_launches = c->launches - c->launches_at_open;
        c->batch_open = false;
    }
    drain_profile(c);
    c->last = now;
    rc = status_from_state(c, now);
    if (rc == SPH_ERR_NEIGHBOR_OVERFLOW) {
        const int r2 = recover_overflow(c);
        if (r2 != SPH_OK) return r2;
        c->last.err = 0;
        c->last.overflow = 0;
        c->err = "neighbour list capacity exceeded; capacity grown for later steps";
    }
    return rc;
}

int sph_step(sph_ctx* c, int nsteps, sph_step_stats* out)
{
    const int rc = sph_step_async(c, nsteps);
    if (rc != SPH_OK) return rc;
    return sph_sync(c, out);
}

int sph_get_state(sph_ctx* c, float* xyz, float* v, float* rho)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_get_state before sph_init");
    const size_t nf = c->nf;
    unsigned na = 0;
    int rc = active_count(c, &na);
    if (rc != SPH_OK) return rc;
    float* tmp = nullptr;
    CUDA_TRY(c, cudaMallocAsync((void**)&tmp, 3 * nf * sizeof(float), c->stream));
    if (na < nf) CUDA_TRY(c, cudaMemsetAsync(tmp, 0, 3 * nf * sizeof(float), c->stream)); /* inactive: 0 */
    auto copy_out = [&](float* dst, size_t count) -> int {
        CUDA_TRY(c, cudaMemcpyAsync(dst, tmp, count * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        return SPH_OK;
    };
    if (xyz) { launch_unsort_v4((int)na, c->orig, c->pos, tmp, c->stream); rc = copy_out(xyz, 3 * nf); }
    if (rc == SPH_OK && v) { launch_unsort_v4((int)na, c->orig, c->vel, tmp, c->stream); rc = copy_out(v, 3 * nf); }
    if (rc == SPH_OK && rho) {
        if (na < nf) CUDA_TRY(c, cudaMemsetAsync(tmp, 0, nf * sizeof(float), c->stream));
        launch_unsort_f((int)na, c->orig, c->rho, tmp, c->stream);
        rc = copy_out(rho, nf);
    }
    cudaFreeAsync(tmp, c->stream);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (rc != SPH_OK) return rc;
    return check_launch(c, "get_state");
}

int sph_set_state(sph_ctx* c, const float* xyz, const float* v)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_set_state before sph_init");
    const size_t nf = c->nf;
    unsigned na = 0;
    int rc0 = active_count(c, &na);
    if (rc0 != SPH_OK) return rc0;
    float* tmp = nullptr;
    CUDA_TRY(c, cudaMallocAsync((void**)&tmp, 3 * nf * sizeof(float), c->stream));
    if (xyz) {
        CUDA_TRY(c, cudaMemcpyAsync(tmp, xyz, 3 * nf * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        launch_sort_v3((int)na, c->orig, tmp, c->pos, c->stream);
        /* the given positions are exact: no residual */
        if (c->P.pos_lo) CUDA_TRY(c, cudaMemsetAsync(c->plo, 0, nf * sizeof(float4), c->stream));
    }
    if (v) {
        CUDA_TRY(c, cudaMemcpyAsync(tmp, v, 3 * nf * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        launch_sort_v3((int)na, c->orig, tmp, c->vel, c->stream);
    }
    cudaFreeAsync(tmp, c->stream);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->lists_valid = false;
    if (xyz && c->desc.simulation_method == SPH_DFSPH) {
        /* DFSPH keeps densities/alpha of the current positions between steps */
        int rc = neighbor_search(c);
        if (rc != SPH_OK) return rc;
        launch_density(c->P, arrays(c), true, false, c->pass_block, c->stream);
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }
    return check_launch(c, "set_state");
}

int sph_get_boundary_state(sph_ctx* c, float* density, float* pressure)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_get_boundary_state before sph_init");
    if (!c->P.pcib) return fail(c, SPH_ERR_ARG, "boundary densities exist for the PCISPH boundary method only");
    if (c->nb == 0) return SPH_OK;
    float* tmp = nullptr;
    CUDA_TRY(c, cudaMallocAsync((void**)&tmp, c->nb * sizeof(float), c->stream));
    for (int k = 0; k < 2; ++k) {
        float* out = k == 0 ? density : pressure;
        if (!out) continue;
        launch_unsort_f((int)c->nb, c->borig, k == 0 ? c->bdens : c->bpress, tmp, c->stream);
        CUDA_TRY(c, cudaMemcpyAsync(out, tmp, c->nb * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }
    cudaFreeAsync(tmp, c->stream);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_launch(c, "get_boundary_state");
}

int sph_get_boundary_volume(sph_ctx* c, float* vol)
{
    if (!c || !vol) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_get_boundary_volume before sph_init");
    if (c->P.pcib) return fail(c, SPH_ERR_ARG, "boundary volumes exist for the Akinci boundary method only");
    if (c->nb == 0) return SPH_OK;
    float* tmp = nullptr;
    CUDA_TRY(c, cudaMallocAsync((void**)&tmp, c->nb * sizeof(float), c->stream));
    launch_unsort_f((int)c->nb, c->borig, c->bvol, tmp, c->stream);
    CUDA_TRY(c, cudaMemcpyAsync(vol, tmp, c->nb * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    cudaFreeAsync(tmp, c->stream);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_launch(c, "get_boundary_volume");
}

int sph_get_time(sph_ctx* c, double* time, float* dt)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_get_time before sph_init");
    DevState s{};
    const int rc = read_state(c, &s);
    if (rc != SPH_OK) return rc;
    if (time) *time = s.time;
    if (dt) *dt = s.dt;
    return SPH_OK;
}

int sph_profile_enable(sph_ctx* c, int enable)
{
    if (!c) return SPH_ERR_ARG;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    drain_profile(c);
    c->prof = enable != 0;
    for (int i = 0; i < SPH_PROF_COUNT; ++i) { c->prof_ms[i] = 0.0; c->prof_launch[i] = 0; }
    return SPH_OK;
}

int sph_profile_read(sph_ctx* c, double* ms, unsigned long long* launches)
{
    if (!c) return SPH_ERR_ARG;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    drain_profile(c);
    for (int i = 0; i < SPH_PROF_COUNT; ++i) {
        if (ms) ms[i] = c->prof_ms[i];
        if (launches) launches[i] = c->prof_launch[i];
    }
    return SPH_OK;
}

int sph_set_time(sph_ctx* c, double time, float dt)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_set_time before sph_init");
    if (!(dt > 0.0f)) return fail(c, SPH_ERR_ARG, "dt must be positive");
    DevState s{};
    int rc = read_state(c, &s);
    if (rc != SPH_OK) return rc;
    s.time = time;
    s.dt = dt;
    CUDA_TRY(c, cudaMemcpyAsync(c->st, &s, sizeof s, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->last.time = time;
    c->last.dt = dt;
    return SPH_OK;
}

unsigned sph_num_fluid(const sph_ctx* c) { return c ? c->nf : 0u; }
unsigned sph_num_boundary(const sph_ctx* c) { return c ? c->nb : 0u; }
const char* sph_last_error(const sph_ctx* c) { return c ? c->err.c_str() : "null context"; }
const char* sph_global_error(void) { return g_global_error.c_str(); }

int sph_destroy(sph_ctx* c)
{
    if (!c) return SPH_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    drain_profile(c);
    drop_graphs(c);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    if (c->ev_begin) cudaEventDestroy(c->ev_begin);
    if (c->ev_end) cudaEventDestroy(c->ev_end);
    for (cudaEvent_t e : c->adj.ev)
        if (e) cudaEventDestroy(e);
    free_all(c);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return SPH_OK;
}

int sph_compute_phase(sph_ctx* c, int phase, float* out)
{
    if (!c || !out) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_compute_phase before sph_init");
    if (phase < SPH_PHASE_DENSITY || phase > SPH_PHASE_PRESSURE_ACC) return fail(c, SPH_ERR_ARG, "unknown phase");
    if ((phase == SPH_PHASE_PRESSURE || phase == SPH_PHASE_PRESSURE_ACC) && c->desc.simulation_method != SPH_WCSPH)
        return fail(c, SPH_ERR_ARG, "pressure phases exist for WCSPH only");
    unsigned na = 0;
    int rc = active_count(c, &na);
    if (rc != SPH_OK) return rc;
    if ((rc = neighbor_search(c)) != SPH_OK) return rc;
    DeviceArrays A = arrays(c);
    const bool eos = phase == SPH_PHASE_PRESSURE || phase == SPH_PHASE_PRESSURE_ACC;
    launch_density(c->P, A, phase == SPH_PHASE_ALPHA || c->desc.simulation_method == SPH_DFSPH, eos, c->pass_block, c->stream);
    /* PCISPH boundary method: SPHSolver::computeDensities covers the
       boundary particles too (SPHSolver.cpp:126-137), WCSPH their pressures */
    if (c->P.pcib) launch_boundary_density(c->P, A, c->stream);
    const size_t nf = c->nf;
    float* tmp = nullptr;
    CUDA_TRY(c, cudaMallocAsync((void**)&tmp, 3 * nf * sizeof(float), c->stream));
    CUDA_TRY(c, cudaMemsetAsync(tmp, 0, 3 * nf * sizeof(float), c->stream)); /* inactive particles read 0 */
    size_t count = nf;
    switch (phase) {
    case SPH_PHASE_DENSITY: launch_unsort_f((int)na, c->orig, c->rho, tmp, c->stream); break;
    case SPH_PHASE_ALPHA: launch_unsort_f((int)na, c->orig, c->alpha, tmp, c->stream); break;
    case SPH_PHASE_PRESSURE: launch_unsort_f((int)na, c->orig, c->press, tmp, c->stream); break;
    case SPH_PHASE_NONPRESSURE_ACC:
        if (c->P.st_on) launch_normals(c->P, A, c->pass_block, c->stream);
        launch_forces(c->P, A, FORCE_NP, c->pass_block, c->stream);
        launch_unsort_v4((int)na, c->orig, c->acc, tmp, c->stream);
        count = 3 * nf;
        break;
    default:
        launch_forces(c->P, A, FORCE_PRESSURE, c->pass_block, c->stream);
        launch_unsort_v4((int)na, c->orig, c->acc, tmp, c->stream);
        count = 3 * nf;
        break;
    }
    CUDA_TRY(c, cudaMemcpyAsync(out, tmp, count * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    if (phase == SPH_PHASE_NONPRESSURE_ACC || phase == SPH_PHASE_PRESSURE_ACC)
        CUDA_TRY(c, cudaMemsetAsync(c->acc, 0, nf * sizeof(float4), c->stream));
    cudaFreeAsync(tmp, c->stream);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_launch(c, "compute_phase");
}

} // extern "C"

namespace {

/* Re-sort the static boundary and recompute its volumes (cell order change). */
int resort_boundary(sph_ctx* c)
{
    if (c->nb == 0) return SPH_OK;
    GatherSet g{};
    g.orig_out = c->borig;
    g.v4_in[0] = c->braw;
    g.v4_out[0] = c->bpos;
    const SceneRef bref{c->d_scenes, c->d_bscene_of};
    launch_sort(c->P, bref, (int)c->nb, c->braw, c->cell_count, c->bcell_start, c->block_sums, c->cell_of, c->slot,
                c->tmp_key, c->tmp_src, c->bid, g, c->stream);
    launch_boundary_volume(c->P, bref, c->bpos, c->bcell_start, c->bvol, c->stream);
    return check_launch(c, "boundary re-sort");
}

/* Make the between-steps data consistent with the current cell order. WCSPH
   and PCISPH search at the start of every step and need nothing; DFSPH
   carries lists, densities and alpha from the end of a step, so it searches
   again (at unchanged positions the sort is the identity up to the cell
   order) and recomputes them, which reproduces them bit for bit. */
int refresh(sph_ctx* c)
{
    if (c->desc.simulation_method != SPH_DFSPH) {
        c->lists_valid = false;
        return SPH_OK;
    }
    int rc = neighbor_search(c);
    if (rc != SPH_OK) return rc;
    launch_density(c->P, arrays(c), true, false, c->pass_block, c->stream);
    return check_launch(c, "refresh");
}

int apply_cell_order(sph_ctx* c, int order)
{
    c->P.cell_order = order;
    if (c->nscenes) {
        for (auto& si : c->h_scenes) si.grid.order = order;
        CUDA_TRY(c, cudaMemcpyAsync(c->d_scenes, c->h_scenes.data(), c->nscenes * sizeof(SceneInfo),
                                    cudaMemcpyHostToDevice, c->stream));
    }
    drop_graphs(c);
    int rc = resort_boundary(c);
    if (rc != SPH_OK) return rc;
    return refresh(c);
}

int snapshot(sph_ctx* c, bool save)
{
    const size_t nf = c->nf;
    int rc;
    if (!c->snap_pos) {
        if ((rc = dalloc(c, &c->snap_pos, nf)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->snap_vel, nf)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->snap_orig, nf)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->snap_kws, nf)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->snap_kvws, nf)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->snap_rho, nf)) != SPH_OK) return rc;
        if ((rc = dalloc(c, &c->snap_st, 1)) != SPH_OK) return rc;
        if (c->nscenes && (rc = dalloc(c, &c->snap_sst, c->nscenes)) != SPH_OK) return rc;
    }
    auto cp = [&](void* a, void* b, size_t bytes) -> int {
        CUDA_TRY(c, cudaMemcpyAsync(save ? b : a, save ? a : b, bytes, cudaMemcpyDeviceToDevice, c->stream));
        return SPH_OK;
    };
    if ((rc = cp(c->pos, c->snap_pos, nf * sizeof(float4))) != SPH_OK) return rc;
    if ((rc = cp(c->vel, c->snap_vel, nf * sizeof(float4))) != SPH_OK) return rc;
    if ((rc = cp(c->orig, c->snap_orig, nf * sizeof(unsigned))) != SPH_OK) return rc;
    if ((rc = cp(c->kws, c->snap_kws, nf * sizeof(float))) != SPH_OK) return rc;
    if ((rc = cp(c->kvws, c->snap_kvws, nf * sizeof(float))) != SPH_OK) return rc;
    if ((rc = cp(c->rho, c->snap_rho, nf * sizeof(float))) != SPH_OK) return rc;
    if ((rc = cp(c->st, c->snap_st, sizeof(DevState))) != SPH_OK) return rc;
    if (c->nscenes && (rc = cp(c->d_sst, c->snap_sst, c->nscenes * sizeof(SceneState))) != SPH_OK) return rc;
    if (c->d_emit && (rc = cp(c->d_emit, c->snap_emit, c->emitters.size() * sizeof(EmitterState))) != SPH_OK) return rc;
    if (c->P.pos_lo) {
        if (!c->snap_plo && (rc = dalloc(c, &c->snap_plo, nf)) != SPH_OK) return rc;
        if ((rc = cp(c->plo, c->snap_plo, nf * sizeof(float4))) != SPH_OK) return rc;
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SPH_OK;
}

std::string tune_key(sph_ctx* c)
{
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, c->device);
    std::ostringstream k;
    k << prop.name << "|m" << c->desc.simulation_method << "|n" << c->nf << "|b" << c->nb << "|s" << c->nscenes;
    return k.str();
}

bool tune_lookup(const char* path, const std::string& key, int* cfg)
{
    if (!path) return false;
    std::ifstream f(path);
    if (!f) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    try {
        const sphjson::Value root = sphjson::parse(ss.str());
        const sphjson::Value* v = root.find(key);
        if (!v || v->size() != SPH_TUNE_COUNT) return false;
        for (int i = 0; i < SPH_TUNE_COUNT; ++i) cfg[i] = (int)v->at(i).as_number();
        return true;
    } catch (const std::exception&) {
        return false;
    }
}

void tune_store(const char* path, const std::string& key, const int* cfg)
{
    if (!path) return;
    std::vector<std::pair<std::string, std::vector<int>>> entries;
    {
        std::ifstream f(path);
        if (f) {
            std::stringstream ss;
            ss << f.rdbuf();
            try {
                const sphjson::Value root = sphjson::parse(ss.str());
                for (const auto& kv : root.items()) {
                    if (kv.first == key || kv.second.size() != SPH_TUNE_COUNT) continue;
                    std::vector<int> v;
                    for (int i = 0; i < SPH_TUNE_COUNT; ++i) v.push_back((int)kv.second.at(i).as_number());
                    entries.push_back({kv.first, v});
                }
            } catch (const std::exception&) {
            }
        }
    }
    entries.push_back({key, std::vector<int>(cfg, cfg + SPH_TUNE_COUNT)});
    std::ofstream o(path);
    o << "{\n";
    for (size_t i = 0; i < entries.size(); ++i) {
        std::string k;
        for (char ch : entries[i].first) k += (ch == '"' || ch == '\\') ? std::string("\\") + ch : std::string(1, ch);
        o << "  \"" << k << "\": [";
        for (int q = 0; q < SPH_TUNE_COUNT; ++q) o << (q ? ", " : "") << entries[i].second[q];
        o << "]" << (i + 1 < entries.size() ? "," : "") << "\n";
    }
    o << "}\n";
}

int apply_config(sph_ctx* c, const int* cfg)
{
    c->solver_occ = cfg[1] == 4 ? 4 : 8;
    c->pass_block = cfg[2] == 128 ? 128 : 256;
    c->solver_tpp = (cfg[3] == 2 || cfg[3] == 4) ? cfg[3] : 1;
    drop_graphs(c);
    if (cfg[0] != c->P.cell_order) return apply_cell_order(c, cfg[0] == 1 ? 1 : 0);
    return SPH_OK;
}

} // namespace

extern "C" {

int sph_set_option(sph_ctx* c, int option, int value)
{
    if (!c) return SPH_ERR_ARG;
    switch (option) {
    case SPH_OPT_CUDA_GRAPHS:
        c->use_graphs = value != 0;
        if (!c->use_graphs) drop_graphs(c);
        return SPH_OK;
    case SPH_OPT_CELL_ORDER:
        if (value != 0 && value != 1) return fail(c, SPH_ERR_ARG, "cell order is 0 or 1");
        if (!c->initialized) { c->P.cell_order = value; return SPH_OK; }
        if (value == c->P.cell_order) return SPH_OK;
        if (c->P.pcib)
            /* the per-cell search record is indexed by the cell order */
            return fail(c, SPH_ERR_ARG, "with the PCISPH boundary method the cell order is set before sph_init");
        return apply_cell_order(c, value);
    case SPH_OPT_SOLVER_OCCUPANCY:
        if (value != 4 && value != 8) return fail(c, SPH_ERR_ARG, "solver occupancy is 4 or 8");
        c->solver_occ = value;
        drop_graphs(c);
        return SPH_OK;
    case SPH_OPT_PASS_BLOCK:
        if (value != 128 && value != 256) return fail(c, SPH_ERR_ARG, "pass block is 128 or 256");
        c->pass_block = value;
        drop_graphs(c);
        return SPH_OK;
    case SPH_OPT_SOLVER_LANES:
        if (value != 1 && value != 2 && value != 4) return fail(c, SPH_ERR_ARG, "solver lanes per particle is 1, 2 or 4");
        c->solver_tpp = value;
        drop_graphs(c);
        return SPH_OK;
    case SPH_OPT_POSITION_RESIDUAL:
        if (value != 0 && value != 1) return fail(c, SPH_ERR_ARG, "the position residual option is 0 or 1");
        if (c->initialized) return fail(c, SPH_ERR_STATE, "position residuals are chosen before sph_init");
        c->pos_lo = value;
        return SPH_OK;
    case SPH_OPT_LIST_STAGED:
        if (value != 0 && value != 1) return fail(c, SPH_ERR_ARG, "the staged-list option is 0 or 1");
        c->staged_lists = value == 1;
        drop_graphs(c);
        return SPH_OK;
    default:
        return fail(c, SPH_ERR_ARG, "unknown option");
    }
}

int sph_get_option(const sph_ctx* c, int option, int* value)
{
    if (!c || !value) return SPH_ERR_ARG;
    switch (option) {
    case SPH_OPT_CUDA_GRAPHS: *value = c->use_graphs ? 1 : 0; return SPH_OK;
    case SPH_OPT_CELL_ORDER: *value = c->P.cell_order; return SPH_OK;
    case SPH_OPT_SOLVER_OCCUPANCY: *value = c->solver_occ; return SPH_OK;
    case SPH_OPT_PASS_BLOCK: *value = c->pass_block; return SPH_OK;
    case SPH_OPT_SOLVER_LANES: *value = c->solver_tpp; return SPH_OK;
    case SPH_OPT_POSITION_RESIDUAL: *value = c->pos_lo; return SPH_OK;
    case SPH_OPT_LIST_STAGED: *value = c->staged_lists ? 1 : 0; return SPH_OK;
    default: return SPH_ERR_ARG;
    }
}

int sph_autotune(sph_ctx* c, int trial_steps, const char* cache_path, int* config)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_autotune before sph_init");
    if (trial_steps < 1) return fail(c, SPH_ERR_ARG, "trial_steps must be positive");
    if (c->P.pcib)
        /* trial steps would advance the carried normals and the per-cell search record */
        return fail(c, SPH_ERR_ARG, "sph_autotune is not available with the PCISPH boundary method");
    const std::string key = tune_key(c);
    int best[SPH_TUNE_COUNT] = {c->P.cell_order, c->solver_occ, c->pass_block, c->solver_tpp};
    int rc;
    if (tune_lookup(cache_path, key, best)) {
        if ((rc = apply_config(c, best)) != SPH_OK) return rc;
        if (config) for (int i = 0; i < SPH_TUNE_COUNT; ++i) config[i] = best[i];
        return SPH_OK;
    }
    if ((rc = snapshot(c, true)) != SPH_OK) return rc;
    const DevState last = c->last;
    const std::vector<SceneState> last_sst = c->last_sst;
    const bool graphs = c->use_graphs;
    c->use_graphs = false;
    double best_ms = 1e300;
    const bool dfsph = c->desc.simulation_method == SPH_DFSPH;
    for (int order = 0; order < 2; ++order)
        for (int occ : {8, 4})
            for (int tpp : {1, 2, 4}) {
            /* only the single-scene DFSPH solver has these variants */
            if ((!dfsph || c->nscenes) && (occ == 4 || tpp != 1)) continue;
            for (int blk : {256, 128}) {
                const int cfg[SPH_TUNE_COUNT] = {order, occ, blk, tpp};
                if ((rc = snapshot(c, false)) != SPH_OK) return rc;
                c->solver_occ = occ;
                c->solver_tpp = tpp;
                c->pass_block = blk;
                rc = order != c->P.cell_order ? apply_cell_order(c, order) : refresh(c);
                if (rc != SPH_OK) return rc;
                if ((rc = sph_step_async(c, 1)) != SPH_OK) return rc;  /* warm-up */
                CUDA_TRY(c, cudaStreamSynchronize(c->stream));
                c->batch_open = false;
                CUDA_TRY(c, cudaEventRecord(c->ev_begin, c->stream));
                for (int s = 0; s < trial_steps; ++s)
                    if ((rc = eager_step(c)) != SPH_OK) return rc;
                CUDA_TRY(c, cudaEventRecord(c->ev_end, c->stream));
                CUDA_TRY(c, cudaStreamSynchronize(c->stream));
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, c->ev_begin, c->ev_end);
                if (ms < best_ms) {
                    best_ms = ms;
                    for (int i = 0; i < SPH_TUNE_COUNT; ++i) best[i] = cfg[i];
                }
            }
            }
    /* back to the snapshot with the chosen configuration */
    if ((rc = snapshot(c, false)) != SPH_OK) return rc;
    c->solver_occ = best[1];
    c->pass_block = best[2];
    c->solver_tpp = best[3];
    rc = best[0] != c->P.cell_order ? apply_cell_order(c, best[0]) : refresh(c);
    if (rc != SPH_OK) return rc;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->last = last;
    c->last_sst = last_sst;
    c->use_graphs = graphs;
    c->batch_open = false;
    tune_store(cache_path, key, best);
    if (config) for (int i = 0; i < SPH_TUNE_COUNT; ++i) config[i] = best[i];
    return SPH_OK;
}

int sph_batch_create(const sph_scene_desc* descs, unsigned nscenes, sph_ctx** out)
{
    if (!descs || !out || nscenes == 0) return fail(nullptr, SPH_ERR_ARG, "descs, nscenes > 0 and out are required");
    const sph_scene_desc& d0 = descs[0];
    if (d0.simulation_method != SPH_WCSPH && d0.simulation_method != SPH_DFSPH)
        return fail(nullptr, SPH_ERR_ARG, "batches run WCSPH or DFSPH scenes");
    for (unsigned s = 1; s < nscenes; ++s) {
        const sph_scene_desc& d = descs[s];
        const bool same = d.simulation_method == d0.simulation_method && d.boundary_method == d0.boundary_method &&
                          d.viscosity_method == d0.viscosity_method &&
                          d.surface_tension_method == d0.surface_tension_method &&
                          d.adhesion_method == d0.adhesion_method && d.particle_radius == d0.particle_radius &&
                          d.density0 == d0.density0 && d.gravity[0] == d0.gravity[0] &&
                          d.gravity[1] == d0.gravity[1] && d.gravity[2] == d0.gravity[2] &&
                          d.stiffness == d0.stiffness && d.gamma == d0.gamma && d.eta == d0.eta &&
                          d.eta_v == d0.eta_v && d.cfl_factor == d0.cfl_factor &&
                          d.min_iterations == d0.min_iterations && d.max_iterations == d0.max_iterations &&
                          d.min_iterations_v == d0.min_iterations_v && d.max_iterations_v == d0.max_iterations_v &&
                          d.surface_tension == d0.surface_tension && d.adhesion == d0.adhesion &&
                          d.min_time_step == d0.min_time_step && d.max_time_step == d0.max_time_step &&
                          d.fps == d0.fps;
        if (!same)
            return fail(nullptr, SPH_ERR_ARG, "scene " + std::to_string(s) + " differs from scene 0 in a shared "
                                              "parameter (only viscosity, boundary viscosity and time step may differ)");
    }
    sph_scene_desc shared = d0;
    /* the viscosity force exists for the batch if its method is set; scenes
       with a zero coefficient add exact zeros */
    int rc = sph_create(&shared, out);
    if (rc != SPH_OK) return rc;
    sph_ctx* c = *out;
    if (c->P.visc_method < 0 && d0.viscosity_method > -1 && d0.viscosity_method <= 2)
        c->P.visc_method = d0.viscosity_method;
    c->nscenes = nscenes;
    c->descs.assign(descs, descs + nscenes);
    c->sc_fluid.resize(nscenes);
    c->sc_vel.resize(nscenes);
    c->sc_bound.resize(nscenes);
    return SPH_OK;
}

int sph_batch_set_scene(sph_ctx* c, unsigned scene, unsigned nf, const float* xyz, const float* v, unsigned nb,
                        const float* bxyz)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->nscenes) return fail(c, SPH_ERR_STATE, "not a batch context");
    if (c->initialized) return fail(c, SPH_ERR_STATE, "sph_batch_set_scene after sph_init");
    if (scene >= c->nscenes) return fail(c, SPH_ERR_ARG, "scene index out of range");
    if ((nf && !xyz) || (nb && !bxyz)) return fail(c, SPH_ERR_ARG, "null positions");
    c->sc_fluid[scene].assign(xyz, xyz + 3ull * nf);
    if (v) c->sc_vel[scene].assign(v, v + 3ull * nf);
    else c->sc_vel[scene].assign(3ull * nf, 0.0f);
    c->sc_bound[scene].assign(bxyz, bxyz + 3ull * nb);
    return SPH_OK;
}

unsigned sph_batch_num_scenes(const sph_ctx* c) { return c ? c->nscenes : 0u; }

int sph_batch_scene_range(const sph_ctx* c, unsigned scene, unsigned* begin, unsigned* end)
{
    if (!c || !c->nscenes || scene >= c->nscenes || !c->initialized) return SPH_ERR_ARG;
    if (begin) *begin = c->fsplit[scene];
    if (end) *end = c->fsplit[scene + 1];
    return SPH_OK;
}

int sph_batch_scene_stats(sph_ctx* c, unsigned scene, sph_step_stats* out)
{
    if (!c || !out) return SPH_ERR_ARG;
    if (!c->nscenes || !c->initialized) return fail(c, SPH_ERR_STATE, "not an initialised batch");
    if (scene >= c->nscenes) return fail(c, SPH_ERR_ARG, "scene index out of range");
    SceneState s{};
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    CUDA_TRY(c, cudaMemcpy(&s, c->d_sst + scene, sizeof s, cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof *out);
    out->time = s.time;
    out->dt = s.dt;
    out->iterations = s.its;
    out->iterations_v = s.its_v;
    out->total_iterations = s.sum_its;
    out->total_iterations_v = s.sum_its_v;
    out->avg_density_error = s.avg_dens;
    out->avg_divergence_error = s.avg_div;
    out->max_velocity = s.last_vmax;
    out->steps = s.steps;
    return SPH_OK;
}

int sph_debug_barrier_timeout(sph_ctx* c)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_debug_barrier_timeout before sph_init");
    const int e = launch_barrier_timeout_probe(c->st, c->stream);
    if (e != 0) return fail(c, SPH_ERR_CUDA, std::string("probe launch: ") + cudaGetErrorString((cudaError_t)e));
    DevState s{};
    int rc = read_state(c, &s);
    if (rc != SPH_OK) return rc;
    /* reset the barrier and the flag so the context stays usable */
    DevState fix = s;
    fix.err &= ~ERRBIT_TIMEOUT;
    fix.bar_count = 0;
    CUDA_TRY(c, cudaMemcpyAsync(c->st, &fix, sizeof fix, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->last = fix;
    if (s.err & ERRBIT_TIMEOUT) return fail(c, SPH_ERR_TIMEOUT, "grid barrier wait ran out (probe)");
    return SPH_OK;
}

int sph_debug_neighbors(sph_ctx* c, unsigned* f_offsets, unsigned* f_index, size_t f_cap, unsigned* b_offsets,
                        unsigned* b_index, size_t b_cap, size_t* nf_total, size_t* nb_total)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_debug_neighbors before sph_init");
    int rc = neighbor_search(c);
    if (rc != SPH_OK) return rc;
    const size_t nf = c->nf, nb = c->nb;
    std::vector<unsigned> cntf(nf), cntb(nf), orig(nf), borig(nb);
    std::vector<unsigned> nbrf((size_t)c->P.capF * nf), nbrb((size_t)c->P.capB * nf);
    CUDA_TRY(c, cudaMemcpyAsync(cntf.data(), c->cnt_f, nf * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(cntb.data(), c->cnt_b, nf * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(orig.data(), c->orig, nf * 4, cudaMemcpyDeviceToHost, c->stream));
    if (nb) CUDA_TRY(c, cudaMemcpyAsync(borig.data(), c->borig, nb * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(nbrf.data(), c->nbr_f, nbrf.size() * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(nbrb.data(), c->nbr_b, nbrb.size() * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    DevState s{};
    if ((rc = read_state(c, &s)) != SPH_OK) return rc;
    if (s.err & ERRBIT_OVERFLOW) return fail(c, SPH_ERR_NEIGHBOR_OVERFLOW, "neighbour list capacity exceeded");
    const size_t na = c->P.dynamic ? s.n_active : nf;
    std::vector<size_t> slot_of(nf, (size_t)-1);
    for (size_t i = 0; i < na; ++i) slot_of[orig[i]] = i;
    size_t tf = 0, tb = 0;
    for (size_t o = 0; o < nf; ++o) {
        const size_t i = slot_of[o];
        if (f_offsets) f_offsets[o] = (unsigned)tf;
        if (b_offsets) b_offsets[o] = (unsigned)tb;
        if (i == (size_t)-1) continue; /* inactive (emitter) particle: no neighbours */
        for (unsigned k = 0; k < cntf[i]; ++k, ++tf)
            if (f_index && tf < f_cap) f_index[tf] = orig[nbrf[(size_t)k * nf + i]];
        for (unsigned k = 0; k < cntb[i]; ++k, ++tb)
            if (b_index && tb < b_cap) b_index[tb] = borig[nbrb[(size_t)k * nf + i]];
    }
    if (f_offsets) f_offsets[nf] = (unsigned)tf;
    if (b_offsets) b_offsets[nf] = (unsigned)tb;
    if (nf_total) *nf_total = tf;
    if (nb_total) *nb_total = tb;
    if ((f_index && tf > f_cap) || (b_index && tb > b_cap)) return fail(c, SPH_ERR_ARG, "index arrays too small");
    return SPH_OK;
}

} // extern "C"

/* ---- WCSPH adjoint ----------------------------------------------------
   Forward: nsteps ordinary WCSPH steps from the current state, the state
   entering every ckpt_every-th step kept as a checkpoint (positions,
   velocities and the sorted-slot ids, 36 B per particle). Backward: per
   segment, last first, the segment is recomputed from its checkpoint with
   the state entering each step kept (the recomputation is bit-identical:
   the sort ranks particles inside a cell by id and every pass is a
   gather), then each step's adjoint kernels run, newest step first. While
   the recomputation keeps every step's neighbour lists, densities and
   pressures (when K steps of them fit kAdjointListBudget) the backward step
   is the three adjoint kernels alone; otherwise each step's neighbour search
   and densities are redone from its kept input state. Memory: (nsteps / K +
   K) states of 36 B per particle for K = ckpt_every, plus K x (capacity x 8
   + 16) B per particle of lists and densities when they are kept. */
namespace {

constexpr size_t kAdjointListBudget = size_t(8) << 30;

void dfree(sph_ctx* c, void* p)
{
    if (!p) return;
    auto it = std::find(c->allocations.begin(), c->allocations.end(), p);
    if (it != c->allocations.end()) {
        cudaFree(p);
        c->allocations.erase(it);
    }
}

int adj_supported(sph_ctx* c)
{
    if (c->nscenes) return fail(c, SPH_ERR_ARG, "the WCSPH adjoint applies to a single scene, not to a batch");
    if (c->desc.simulation_method != SPH_WCSPH) return fail(c, SPH_ERR_ARG, "the adjoint differentiates the WCSPH step only");
    if (c->P.dynamic) return fail(c, SPH_ERR_ARG, "the WCSPH adjoint does not cover emitters");
    if (c->desc.boundary_method != SPH_BOUNDARY_AKINCI)
        return fail(c, SPH_ERR_ARG, "the WCSPH adjoint covers Akinci boundaries (boundary method 2) only");
    if (c->P.pos_lo) return fail(c, SPH_ERR_ARG, "the WCSPH adjoint differentiates FP32 positions (no residuals)");
    if (c->P.st_on || c->P.adh_on)
        return fail(c, SPH_ERR_ARG, "the WCSPH adjoint covers neither surface tension nor adhesion");
    if (c->P.visc_method != -1 && c->P.visc_method != SPH_VISCOSITY_ARTIFICIAL)
        return fail(c, SPH_ERR_ARG, "the WCSPH adjoint covers artificial viscosity (or none) only");
    return SPH_OK;
}

int adj_reserve(sph_ctx* c, int nseg, int every)
{
    auto& a = c->adj;
    const size_t nf = c->nf;
    int rc;
#define AALLOC(ptr, count) if ((rc = dalloc(c, &a.ptr, (count))) != SPH_OK) return rc
    if (!a.xbar) {
        AALLOC(fin_pos, nf); AALLOC(fin_vel, nf); AALLOC(fin_orig, nf);
        AALLOC(st0, 1); AALLOC(st1, 1); AALLOC(target, 3 * nf);
        AALLOC(xbar, nf); AALLOC(vbar, nf); AALLOC(abar, nf); AALLOC(xacc, nf); AALLOC(vacc, nf);
        AALLOC(Ap, nf); AALLOC(rhobar, nf); AALLOC(red, 4);
        AALLOC(part, 3 * (size_t)adjoint_blocks((int)nf));
        for (auto& e : a.ev) CUDA_TRY(c, cudaEventCreate(&e));
    }
    if (nseg > a.cap_seg) {
        dfree(c, a.ck_pos); dfree(c, a.ck_vel); dfree(c, a.ck_orig);
        a.ck_pos = a.ck_vel = nullptr; a.ck_orig = nullptr; a.cap_seg = 0;
        AALLOC(ck_pos, (size_t)nseg * nf); AALLOC(ck_vel, (size_t)nseg * nf); AALLOC(ck_orig, (size_t)nseg * nf);
        a.cap_seg = nseg;
    }
    const size_t list_bytes = (size_t)every * nf * ((size_t)(c->P.capF + c->P.capB) * 4 + 16);
    const bool keep = list_bytes <= kAdjointListBudget;
    if (every > a.cap_every || keep != a.keep_lists ||
        (keep && (a.sl_capF != c->P.capF || a.sl_capB != c->P.capB))) {
        drop_graphs(c);
        for (void* p : {(void*)a.sl_pos, (void*)a.sl_vel, (void*)a.sl_orig, (void*)a.sl_nbr_f, (void*)a.sl_cnt_f,
                        (void*)a.sl_nbr_b, (void*)a.sl_cnt_b, (void*)a.sl_rho, (void*)a.sl_press})
            dfree(c, p);
        a.sl_pos = a.sl_vel = nullptr; a.sl_orig = a.sl_nbr_f = a.sl_cnt_f = a.sl_nbr_b = a.sl_cnt_b = nullptr;
        a.sl_rho = a.sl_press = nullptr;
        const int cap = std::max(every, a.cap_every);
        a.cap_every = 0;
        AALLOC(sl_pos, (size_t)cap * nf); AALLOC(sl_vel, (size_t)cap * nf); AALLOC(sl_orig, (size_t)cap * nf);
        if (keep) {
            AALLOC(sl_nbr_f, (size_t)cap * c->P.capF * nf); AALLOC(sl_nbr_b, (size_t)cap * c->P.capB * nf);
            AALLOC(sl_cnt_f, (size_t)cap * nf); AALLOC(sl_cnt_b, (size_t)cap * nf);
            AALLOC(sl_rho, (size_t)cap * nf); AALLOC(sl_press, (size_t)cap * nf);
            a.sl_capF = c->P.capF;
            a.sl_capB = c->P.capB;
        }
        a.keep_lists = keep;
        a.cap_every = cap;
    }
#undef AALLOC
    return SPH_OK;
}

int copy_state(sph_ctx* c, float4* dp, float4* dv, unsigned* dorig, const float4* sp, const float4* sv,
               const unsigned* sorig)
{
    const size_t nf = c->nf;
    CUDA_TRY(c, cudaMemcpyAsync(dp, sp, nf * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(dv, sv, nf * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(dorig, sorig, nf * sizeof(unsigned), cudaMemcpyDeviceToDevice, c->stream));
    return SPH_OK;
}

/* Name the first-allocated buffers "current" (contents are about to be
   overwritten by a restore), so that a segment always starts from the same
   buffer assignment and its captured graph can be replayed. */
void canonical_buffers(sph_ctx* c)
{
    if (c->pos != c->pos_base) { std::swap(c->pos, c->pos2); std::swap(c->vel, c->vel2); }
    if (c->orig != c->orig_base) std::swap(c->orig, c->orig2);
}

AdjointArrays adj_arrays(sph_ctx* c)
{
    auto& a = c->adj;
    AdjointArrays J{};
    J.pos = c->pos; J.vel = c->vel; J.rho = c->rho; J.press = c->press; J.orig = c->orig;
    J.bpos = c->bpos; J.nbr_f = c->nbr_f; J.cnt_f = c->cnt_f; J.nbr_b = c->nbr_b; J.cnt_b = c->cnt_b;
    J.st = c->st;
    J.xbar = a.xbar; J.vbar = a.vbar; J.abar = a.abar; J.xacc = a.xacc; J.vacc = a.vacc;
    J.Ap = a.Ap; J.rhobar = a.rhobar; J.part = a.part;
    return J;
}

/* Adjoint arrays of step n of the segment from the kept lists and state. */
AdjointArrays adj_arrays_kept(sph_ctx* c, int n)
{
    auto& a = c->adj;
    const size_t nf = c->nf;
    AdjointArrays J = adj_arrays(c);
    J.pos = a.sl_pos + n * nf; J.vel = a.sl_vel + n * nf; J.orig = a.sl_orig + n * nf;
    J.rho = a.sl_rho + n * nf; J.press = a.sl_press + n * nf;
    J.nbr_f = a.sl_nbr_f + (size_t)n * a.sl_capF * nf; J.nbr_b = a.sl_nbr_b + (size_t)n * a.sl_capB * nf;
    J.cnt_f = a.sl_cnt_f + n * nf; J.cnt_b = a.sl_cnt_b + n * nf;
    return J;
}

/* Recompute a segment of len steps from the state in the current buffers,
   keeping what each step's adjoint needs, then run the adjoint of its
   steps, last first. */
int adj_segment_body(sph_ctx* c, int len)
{
    auto& a = c->adj;
    const size_t nf = c->nf;
    int rc;
    if (a.keep_lists) {
        for (int n = 0; n < len; ++n) {
            /* the step builds its lists and densities straight into slot n */
            unsigned *lf = c->nbr_f, *cf = c->cnt_f, *lb = c->nbr_b, *cb = c->cnt_b;
            float *rho = c->rho, *press = c->press;
            c->nbr_f = a.sl_nbr_f + (size_t)n * a.sl_capF * nf; c->nbr_b = a.sl_nbr_b + (size_t)n * a.sl_capB * nf;
            c->cnt_f = a.sl_cnt_f + n * nf; c->cnt_b = a.sl_cnt_b + n * nf;
            c->rho = a.sl_rho + n * nf; c->press = a.sl_press + n * nf;
            rc = step_wcsph(c);
            c->nbr_f = lf; c->cnt_f = cf; c->nbr_b = lb; c->cnt_b = cb; c->rho = rho; c->press = press;
            if (rc != SPH_OK) return rc;
            /* the sorted state the step's forces read (integrated into the spare buffers) */
            if ((rc = copy_state(c, a.sl_pos + n * nf, a.sl_vel + n * nf, a.sl_orig + n * nf, c->pos2, c->vel2, c->orig)) != SPH_OK)
                return rc;
        }
        for (int n = len - 1; n >= 0; --n) {
            launch_adjoint_step(c->P, adj_arrays_kept(c, n), c->stream);
            c->launches += 3;
        }
        c->lists_valid = false;
        return check_launch(c, "adjoint segment");
    }
    for (int n = 0; n < len; ++n) {
        if ((rc = copy_state(c, a.sl_pos + n * nf, a.sl_vel + n * nf, a.sl_orig + n * nf, c->pos, c->vel, c->orig)) != SPH_OK)
            return rc;
        if ((rc = step_wcsph(c)) != SPH_OK) return rc;
    }
    for (int n = len - 1; n >= 0; --n) {
        if ((rc = copy_state(c, c->pos, c->vel, c->orig, a.sl_pos + n * nf, a.sl_vel + n * nf, a.sl_orig + n * nf)) != SPH_OK)
            return rc;
        if ((rc = neighbor_search(c)) != SPH_OK) return rc;
        { Phase ph(c, SPH_PROF_DENSITY, 1); launch_density(c->P, arrays(c), false, true, c->pass_block, c->stream); }
        launch_adjoint_step(c->P, adj_arrays(c), c->stream);
        c->launches += 3;
    }
    c->lists_valid = false;
    return check_launch(c, "adjoint segment");
}

/* One segment, from a graph captured on the first segment of this length
   (segments start from the canonical buffer assignment, so the captured
   launch sequence is the same for every segment of that length). */
int adj_segment(sph_ctx* c, int len)
{
    auto& a = c->adj;
    if (a.use_graphs && !c->prof) {
        for (auto& g : a.graphs)
            if (g.len == len) {
                const cudaError_t e = cudaGraphLaunch(g.exec, c->stream);
                if (e != cudaSuccess) return fail(c, SPH_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
                set_buffers(c, g.end);
                c->launches += g.launches;
                return SPH_OK;
            }
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const Buffers start = get_buffers(c);
            const unsigned long long l0 = c->launches;
            const int r = adj_segment_body(c, len);
            cudaGraph_t graph = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(c->stream, &graph);
            const unsigned long long nl = c->launches - l0;
            c->launches = l0;
            cudaGraphExec_t exec = nullptr;
            const bool ok = r == SPH_OK && ec == cudaSuccess && graph &&
                            cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
            if (graph) cudaGraphDestroy(graph);
            const Buffers end = get_buffers(c);
            set_buffers(c, start);
            if (ok) {
                a.graphs.push_back({len, exec, nl, end});
                return adj_segment(c, len);
            }
            cudaGetLastError();
            c->err.clear();
        } else {
            cudaGetLastError();
        }
        a.use_graphs = false;  /* capture unsupported: stay eager */
        drop_graphs(c);
    }
    return adj_segment_body(c, len);
}

} // namespace

extern "C" {

int sph_wcsph_forward(sph_ctx* c, int nsteps, int ckpt_every, const float* target, double* loss)
{
    if (!c) return SPH_ERR_ARG;
    if (!c->initialized) return fail(c, SPH_ERR_STATE, "sph_wcsph_forward before sph_init");
    if (nsteps <= 0 || ckpt_every <= 0) return fail(c, SPH_ERR_ARG, "nsteps and ckpt_every must be positive");
    if (!target || !loss) return fail(c, SPH_ERR_ARG, "target and loss must not be NULL");
    int rc = adj_supported(c);
    if (rc != SPH_OK) return rc;
    auto& a = c->adj;
    a.ready = false;
    a.have_grad = false;
    const int every = std::min(ckpt_every, nsteps);
    const int nseg = (nsteps + every - 1) / every;
    if ((rc = adj_reserve(c, nseg, every)) != SPH_OK) return rc;
    const size_t nf = c->nf;
    CUDA_TRY(c, cudaMemcpyAsync(a.target, target, 3 * nf * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaEventRecord(a.ev[0], c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(a.st0, c->st, sizeof(DevState), cudaMemcpyDeviceToDevice, c->stream));
    for (int s = 0; s < nseg; ++s) {
        if ((rc = copy_state(c, a.ck_pos + s * nf, a.ck_vel + s * nf, a.ck_orig + s * nf, c->pos, c->vel, c->orig)) != SPH_OK)
            return rc;
        if ((rc = run_steps(c, std::min(every, nsteps - s * every))) != SPH_OK) return rc;
    }
    if ((rc = copy_state(c, a.fin_pos, a.fin_vel, a.fin_orig, c->pos, c->vel, c->orig)) != SPH_OK) return rc;
    CUDA_TRY(c, cudaMemcpyAsync(a.st1, c->st, sizeof(DevState), cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaMemsetAsync(a.part, 0, 3 * (size_t)adjoint_blocks((int)nf) * sizeof(double), c->stream));
    launch_adjoint_seed((int)nf, a.fin_pos, a.fin_orig, a.target, a.xbar, a.vbar, a.part, c->stream);
    launch_adjoint_finish((int)nf, a.part, a.red, c->stream);
    c->launches += 2;
    CUDA_TRY(c, cudaEventRecord(a.ev[1], c->stream));
    double red[4] = {0, 0, 0, 0};
    CUDA_TRY(c, cudaMemcpyAsync(red, a.red, sizeof red, cudaMemcpyDeviceToHost, c->stream));
    DevState now{};
    if ((rc = read_state(c, &now)) != SPH_OK) return rc;
    if ((rc = check_launch(c, "wcsph forward")) != SPH_OK) return rc;
    float ms = 0.0f;
    a.fwd_ms = cudaEventElapsedTime(&ms, a.ev[0], a.ev[1]) == cudaSuccess ? ms : 0.0;
    c->last = now;
    if ((rc = status_from_state(c, now)) != SPH_OK) {
        if (rc == SPH_ERR_NEIGHBOR_OVERFLOW) {
            const int r2 = recover_overflow(c);
            if (r2 != SPH_OK) return r2;
            c->err = "neighbour list capacity exceeded during the forward run; capacity grown, run it again";
        }
        return rc;
    }
    *loss = red[2] / (double)nf;
    a.nsteps = nsteps;
    a.every = every;
    a.nseg = nseg;
    a.ready = true;
    return SPH_OK;
}

int sph_wcsph_backward(sph_ctx* c, float* dL_dv0, float* dL_dvisc, float* dL_dk)
{
    if (!c) return SPH_ERR_ARG;
    auto& a = c->adj;
    if (!c->initialized || !a.ready) return fail(c, SPH_ERR_STATE, "sph_wcsph_backward before sph_wcsph_forward");
    int rc = adj_supported(c);
    if (rc != SPH_OK) return rc;
    const size_t nf = c->nf;
    CUDA_TRY(c, cudaEventRecord(a.ev[2], c->stream));
    CUDA_TRY(c, cudaMemsetAsync(a.part, 0, 3 * (size_t)adjoint_blocks((int)nf) * sizeof(double), c->stream));
    launch_adjoint_seed((int)nf, a.fin_pos, a.fin_orig, a.target, a.xbar, a.vbar, a.part, c->stream);
    c->launches += 1;
    CUDA_TRY(c, cudaMemcpyAsync(c->st, a.st0, sizeof(DevState), cudaMemcpyDeviceToDevice, c->stream));
    for (int s = a.nseg - 1; s >= 0; --s) {
        canonical_buffers(c);
        if ((rc = copy_state(c, c->pos, c->vel, c->orig, a.ck_pos + s * nf, a.ck_vel + s * nf, a.ck_orig + s * nf)) != SPH_OK)
            return rc;
        if ((rc = adj_segment(c, std::min(a.every, a.nsteps - s * a.every))) != SPH_OK) return rc;
    }
    launch_adjoint_finish((int)nf, a.part, a.red, c->stream);
    c->launches += 1;
    CUDA_TRY(c, cudaEventRecord(a.ev[3], c->stream));
    if (dL_dv0) {
        float* tmp = reinterpret_cast<float*>(a.xacc); /* 4 nf floats of scratch */
        launch_adjoint_unpack((int)nf, a.vbar, tmp, c->stream);
        CUDA_TRY(c, cudaMemcpyAsync(dL_dv0, tmp, 3 * nf * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    }
    double red[4] = {0, 0, 0, 0};
    CUDA_TRY(c, cudaMemcpyAsync(red, a.red, sizeof red, cudaMemcpyDeviceToHost, c->stream));
    DevState seen{};
    if ((rc = read_state(c, &seen)) != SPH_OK) return rc;
    if ((rc = check_launch(c, "wcsph backward")) != SPH_OK) return rc;
    float ms = 0.0f;
    a.bwd_ms = cudaEventElapsedTime(&ms, a.ev[2], a.ev[3]) == cudaSuccess ? ms : 0.0;
    /* back to the state the forward run ended in */
    canonical_buffers(c);
    if ((rc = copy_state(c, c->pos, c->vel, c->orig, a.fin_pos, a.fin_vel, a.fin_orig)) != SPH_OK) return rc;
    CUDA_TRY(c, cudaMemcpyAsync(c->st, a.st1, sizeof(DevState), cudaMemcpyDeviceToDevice, c->stream));
    c->lists_valid = false;
    DevState now{};
    if ((rc = read_state(c, &now)) != SPH_OK) return rc;
    c->last = now;
    if ((rc = status_from_state(c, seen)) != SPH_OK) return rc;
    if (dL_dvisc) *dL_dvisc = (float)red[1];
    if (dL_dk) *dL_dk = (float)red[0];
    a.have_grad = true;
    return SPH_OK;
}

int sph_wcsph_grad_x0(sph_ctx* c, float* dL_dx0)
{
    if (!c || !dL_dx0) return SPH_ERR_ARG;
    auto& a = c->adj;
    if (!a.have_grad) return fail(c, SPH_ERR_STATE, "sph_wcsph_grad_x0 before sph_wcsph_backward");
    float* tmp = reinterpret_cast<float*>(a.xacc);
    launch_adjoint_unpack((int)c->nf, a.xbar, tmp, c->stream);
    CUDA_TRY(c, cudaMemcpyAsync(dL_dx0, tmp, 3 * (size_t)c->nf * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_launch(c, "grad_x0");
}

int sph_wcsph_timing(const sph_ctx* c, double* forward_ms, double* backward_ms)
{
    if (!c) return SPH_ERR_ARG;
    if (forward_ms) *forward_ms = c->adj.fwd_ms;
    if (backward_ms) *backward_ms = c->adj.bwd_ms;
    return SPH_OK;
}

} // extern "C"
