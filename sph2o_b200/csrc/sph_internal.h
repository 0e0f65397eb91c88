/*
 * Host-side declarations of the kernel launchers (one CUDA stream each).
 * Kernels live in sph_grid.cu (neighbour search, sort, boundary volumes),
 * sph_solvers.cu (density, forces, WCSPH / PCISPH / DFSPH steps),
 * sph_adjoint.cu (reverse-mode WCSPH step); sph_mesh.h declares the mesh
 * sampler of sph_mesh.cu.
 */
#ifndef SPH2O_INTERNAL_H
#define SPH2O_INTERNAL_H

#include <cuda_runtime.h>

#include "sph_device.cuh"
#include "sph_grid_body.cuh"

namespace sph {


/* Device pointers of one scene, handed to the solver launchers. */
struct DeviceArrays {
    float4* pos;
    float4* vel;
    float4* pos_alt;      /* WCSPH integrate target */
    float4* vel_alt;
    float4* acc;
    float4* normal;
    float4* predr;        /* PCISPH predicted position */
    float4* pacc;         /* PCISPH pressure acceleration */
    float* rho;
    float* alpha;
    float* k;
    float* kws;
    float* kvws;
    float* press;
    const unsigned* cell_start;
    const unsigned* cell_sorted;   /* cell index of each sorted slot */
    const float4* bpos;
    const unsigned* bcell_start;
    const unsigned* nbr_f;
    const unsigned* cnt_f;
    const unsigned* nbr_b;
    const unsigned* cnt_b;
    unsigned* orig_w;     /* caller-order ids of the sorted slots (emitters write new ones) */
    double* accum;        /* per-iteration residual accumulators, zeroed per solve */
    DevState* st;
    SceneRef sref;        /* batch scene table (empty for a single scene) */
    SceneState* sst;      /* per-scene state of a batch (NULL for a single scene) */
    unsigned* any_active; /* batch: per-iteration "some scene still iterates" flags */
    int nscenes;
    unsigned accum_stride;/* batch: doubles per scene in accum */
    /* PCISPH boundary method (SimParams::pcib): boundary normals, densities,
       pressures and p / rho^2 in boundary sorted order, predicted velocities,
       and the per-cell search that first listed each cell */
    const float4* bnormal;
    float* bdens;
    float* bpress;
    float* bdp;
    float4* predv;
    unsigned* cell_entry;
    /* position residuals (SimParams::pos_lo; NULL when off) and the WCSPH
       integration target */
    float4* plo;
    float4* plo_alt;
    /* DFSPH: divergence error of the density pass (NULL: the divergence
       solver computes its warm-start residual itself) */
    float* divres;
};

/* sph_grid.cu */
void launch_sort(const SimParams& P, const SceneRef& S, int n, const float4* pos_for_keys, unsigned* cell_count,
                 unsigned* cell_start,
                 unsigned* block_sums, unsigned* cell_of, unsigned* slot, unsigned* tmp_key, unsigned* tmp_src,
                 const unsigned* orig_in, const GatherSet& g, cudaStream_t s);
void launch_build_lists(const SimParams& P, const SceneRef& S, const float4* pos, const unsigned* cell_start,
                        const float4* bpos,
                        const unsigned* bcell_start, unsigned* nbr_f, unsigned* cnt_f, unsigned* nbr_b,
                        unsigned* cnt_b, DevState* st, cudaStream_t s, bool staged = false);
void launch_boundary_volume(const SimParams& P, const SceneRef& S, float4* bpos, const unsigned* bcell_start,
                            float* bvol, cudaStream_t s);
void launch_unsort_v4(int n, const unsigned* orig, const float4* in, float* out3, cudaStream_t s);
void launch_unsort_f(int n, const unsigned* orig, const float* in, float* out, cudaStream_t s);
void launch_sort_v3(int n, const unsigned* orig, const float* in3, float4* out, cudaStream_t s);
void launch_pack_v3(int n, const float* in3, float4* out, float w, cudaStream_t s);
void launch_iota(int n, unsigned* out, cudaStream_t s);

/* sph_solvers.cu */
enum ForceMode : int {
    FORCE_NP = 0,          /* non-pressure forces -> acc                      */
    FORCE_NP_CFL = 1,      /* + DFSPH CFL speed |v + (a + g) dt| -> st->vmax   */
    FORCE_WCSPH = 2,       /* pressure + non-pressure + symplectic Euler       */
    FORCE_PRESSURE = 3     /* pressure acceleration only -> acc (phase access) */
};

/* block: threads per block of the pass kernels (128 or 256, autotuned) */
void launch_density(const SimParams& P, const DeviceArrays& A, bool alpha, bool eos, int block, cudaStream_t s);
void launch_normals(const SimParams& P, const DeviceArrays& A, int block, cudaStream_t s);
void launch_forces(const SimParams& P, const DeviceArrays& A, int mode, int block, cudaStream_t s);
/* occ: blocks per SM of the persistent DFSPH solver variant (4 or 8);
   tpp: lanes per particle in its neighbour passes (1, 2 or 4) */
int launch_dfsph_solve(const SimParams& P, const DeviceArrays& A, bool divergence, int grid, int occ, int tpp,
                       cudaStream_t s);
int launch_pcisph_solve(const SimParams& P, const DeviceArrays& A, int grid, cudaStream_t s);
int launch_dfsph_solve_batch(const SimParams& P, const DeviceArrays& A, bool divergence, int grid, cudaStream_t s);
int launch_barrier_timeout_probe(DevState* st, cudaStream_t s);
/* cube boundaries: clamp the active particles into each box in order */
void launch_cube_correct(const SimParams& P, const DeviceArrays& A, const CubeBox* cubes, int ncubes, cudaStream_t s);
/* PCISPH boundary method: mark the cells of n particles as listed by the
   search now completing, then count it (two launches) */
void launch_mark_entries(const SimParams& P, const float4* pos, int n, const unsigned* n_dev, unsigned* entry,
                         DevState* st, bool advance, cudaStream_t s);
/* boundary densities with the cubic spline at the current fluid positions,
   the Tait pressure and p / rho^2 (WCSPH, SPHSolver.cpp:91-124,
   WCSPHSolver.cpp:97-114) */
void launch_boundary_density(const SimParams& P, const DeviceArrays& A, cudaStream_t s);
/* collision correction of positions (and, for WCSPH, velocities) after the
   position update (PCISPHBoundaryObject.cpp:218-388); wcsph selects the
   velocity pass */
void launch_pcib_correct(const SimParams& P, const DeviceArrays& A, bool wcsph, cudaStream_t s);
/* emission of the nemit emitters' due groups (one block); advance: then t += dt */
void launch_emit(const SimParams& P, const DeviceArrays& A, EmitterState* E, const float4* group, int nemit,
                 bool advance, cudaStream_t s);

/* sph_adjoint.cu: reverse-mode WCSPH step. Sorted-order arrays of the
   recomputed step (pos .. cnt_b), caller-order adjoint state (xbar, vbar),
   sorted-order work arrays (abar .. rhobar) and per-block FP64 partial sums
   part[3 b + q] (q = 0: dL/dk, 1: dL/dnu, 2: loss * N), adjoint_blocks(n)
   blocks, which launch_adjoint_finish reduces into red[0..2]. */
struct AdjointArrays {
    const float4* pos;
    const float4* vel;
    const float* rho;
    const float* press;
    const unsigned* orig;
    const float4* bpos;
    const unsigned* nbr_f;
    const unsigned* cnt_f;
    const unsigned* nbr_b;
    const unsigned* cnt_b;
    const DevState* st;
    float4* xbar;
    float4* vbar;
    float4* abar;
    float4* xacc;
    float4* vacc;
    float* Ap;
    float* rhobar;
    double* part;
};
int adjoint_blocks(int n);
void launch_adjoint_seed(int n, const float4* pos, const unsigned* orig, const float* target, float4* xbar,
                         float4* vbar, double* part, cudaStream_t s);
void launch_adjoint_finish(int n, const double* part, double* red, cudaStream_t s);
/* load + forces + density adjoint kernels of one step (3 launches) */
void launch_adjoint_step(const SimParams& P, const AdjointArrays& J, cudaStream_t s);
void launch_adjoint_unpack(int n, const float4* in, float* out3, cudaStream_t s);

/* co-resident grid size of the persistent solver kernels (0 on error) */
int persistent_grid(bool pcisph, bool divergence, bool batch = false, int occ = 8, int tpp = 1);
constexpr int kSolverBlock = 256;

} // namespace sph

#endif
