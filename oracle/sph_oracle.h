/*
 * CPU restatement of SPH2O's per-step particle path -- TEST INFRASTRUCTURE.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker. It mirrors the C ABI of
 * include/sph2o_cuda.h (same scene description, same caller particle order)
 * so the same scenario can run through both. Real is float (fp64 = 0) or
 * double (fp64 = 1); the float variant reproduces the reference's FP32
 * arithmetic operation by operation, the double variant its FP64 build.
 * Parity pinned: tests/test_oracle.py checks it against the golden vectors
 * generated by running the reference itself (tests/golden/).
 */
#ifndef SPH2O_ORACLE_H
#define SPH2O_ORACLE_H

#include <stddef.h>

#include "../include/sph2o_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sph_oracle sph_oracle;

sph_oracle* sph_oracle_create(const sph_scene_desc* desc, int fp64);
int sph_oracle_set_fluid(sph_oracle* o, unsigned n, const float* xyz, const float* v);
int sph_oracle_set_boundary(sph_oracle* o, unsigned n, const float* xyz);
/* PCISPH boundary method: normals of the boundary particles (same order) and
   the object's normalFct / tangFct */
int sph_oracle_set_boundary_normals(sph_oracle* o, unsigned n, const float* nxyz, float normal_fct,
                                    float tangential_fct);
/* PCISPH boundary method: the last computed boundary densities / pressures */
int sph_oracle_boundary_state(sph_oracle* o, double* dens, double* press);
/* cube boundary (boundary method 0), applied after integration in order */
int sph_oracle_add_cube(sph_oracle* o, const float* mn, const float* mx, float normal_fct, float tangential_fct);
int sph_oracle_init(sph_oracle* o);
/* stats: [time, dt, iterations, iterationsV, avg density residual, avg divergence residual] per step */
int sph_oracle_step(sph_oracle* o, int nsteps, double* stats);
int sph_oracle_get_state(sph_oracle* o, double* xyz, double* v, double* rho);
int sph_oracle_get_boundary_volume(sph_oracle* o, double* vol);
/* phases as in sph_phase: density, alpha, non-pressure acc, pressure, pressure acc */
int sph_oracle_phase(sph_oracle* o, int phase, double* out);
/* CSR neighbour sets (|xi - xj| <= h over the 27 cells), caller order */
int sph_oracle_neighbors(sph_oracle* o, unsigned* f_off, unsigned* f_idx, size_t f_cap, unsigned* b_off,
                         unsigned* b_idx, size_t b_cap, size_t* nf_total, size_t* nb_total);
void sph_oracle_destroy(sph_oracle* o);

/* wcsph_adjoint.cpp: FP64 WCSPH run from (x0, v0) for nsteps steps with
   viscosity nu and stiffness k, loss (1/N) sum |x_i(T) - target_i|^2, and
   (when dv0 is not NULL) its gradients dL/dx0, dL/dv0, dL/dnu, dL/dk. */
int sph_oracle_wcsph_adjoint(const sph_scene_desc* d, double nu, double k, unsigned nf, const double* x0,
                             const double* v0, unsigned nb, const double* bxyz, int nsteps, const double* target,
                             double* loss, double* x_out, double* dx0, double* dv0, double* dnu, double* dk);

/* Regular triangle sampling of a mesh (mesh_sampling.cpp): vertices xyz,
   0-based faces, spacing max_distance; rotate_xyz / translate (NULL: none)
   place the samples as AkinciBoundaryObject::sampleGeometry does. Two-call
   convention as sph_sample_mesh. */
int sph_oracle_sample_mesh(const float* vertices, unsigned nv, const unsigned* faces, unsigned nf,
                           float max_distance, const float rotate_xyz[3], const float translate[3], float* out,
                           size_t capacity, size_t* count);

#ifdef __cplusplus
}
#endif
#endif
