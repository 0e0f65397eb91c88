/*
 * Particle-pass kernels of the WCSPH / PCISPH / DFSPH steps (sm_100a).
 *
 * Every pass is one thread per fluid particle walking that particle's
 * neighbour lists (built once per step by sph_grid.cu); positions and
 * velocities of neighbours are gathered as float4 from the cell-sorted
 * arrays, so a warp's gathers fall on a few cache lines of nearby cells.
 * The DFSPH and PCISPH iteration loops each run as ONE persistent,
 * cooperative kernel: phases are separated by a bounded grid barrier and
 * the convergence residual is reduced in FP64 on the device (warp shuffles,
 * a block reduction, one atomicAdd per block), so no host round trip occurs
 * inside a step.
 *
 * Reference correspondence (file:line in SPH2O):
 *   k_density            SPHSolver::computeFluidDensities     SPHSolver.cpp:42-89
 *                        DFSPHSolver::computeAlpha            DFSPHSolver.cpp:109-178
 *                        WCSPHSolver::computeFluidPressures   WCSPHSolver.cpp:80-95
 *   k_normals            SurfaceTensionAkinci::step, pass 1   SurfaceTensionAkinci.cpp:14-31
 *   k_forces             ArtificialViscosity::step            ArtificialViscosity.cpp:6-54
 *                        StandardViscosityForce::step         StandardViscosity.cpp:5-50
 *                        XSPHViscosity::step                  XSPHViscosity.cpp:6-43
 *                        SurfaceTensionAkinci::step, pass 2   SurfaceTensionAkinci.cpp:33-70
 *                        AdhesionForce::step                  AdhesionForce.cpp:5-33
 *                        WCSPHSolver::computePressureForce    WCSPHSolver.cpp:132-188
 *                        SPHSolver::integrate                 SPHSolver.cpp:139-168
 *   k_dfsph_solve<false> updateTimeStep, predictVelocities, densityWarmStart,
 *                        correctDensityError, updatePositions DFSPHSolver.cpp:1090-1162,
 *                                                              180-224, 851-955, 414-536
 *   k_dfsph_solve<true>  divergenceWarmStart, correctDivergenceError,
 *                        computeDivergenceError               DFSPHSolver.cpp:957-1059, 730-849, 538-621
 *   k_pcisph_solve       initPressure, pressureSolver, predictVelocityAndPosition,
 *                        predictFluidDensities, updatePressure, computePressureAcc,
 *                        integrate                            PCISPHSolver.cpp:82-401, 459-488
 */
#include "sph_device.cuh"
#include "sph_internal.h"



namespace sph {

struct Pair {
    float rx, ry, rz, s, rl, inv_rl;
};

__device__ __forceinline__ Pair make_pair(float4 a, float4 b)
{
    Pair p;
    p.rx = a.x - b.x;
    p.ry = a.y - b.y;
    p.rz = a.z - b.z;
    p.s = (p.rx * p.rx + p.ry * p.ry) + p.rz * p.rz;
    len_inv(p.s, p.rl, p.inv_rl);
    return p;
}

/* Calls f(j, x_j) for the fluid neighbours of sorted particle i in list
   order, issuing the list loads and position gathers of U entries before the
   first of them is used (more loads in flight per thread; same order, so the
   sums it feeds are unchanged). With TPP lanes per particle, lane sub visits
   the entries sub, sub + TPP, ... */
template <int U, int TPP = 1, typename F>
__device__ __forceinline__ void for_fluid_neighbors(const DeviceArrays& A, int i, size_t nf, unsigned n, F&& f,
                                                    unsigned sub = 0)
{
    unsigned kk = sub;
    for (; kk + (U - 1) * TPP < n; kk += U * TPP) {
        unsigned jj[U];
        float4 xj[U];
#pragma unroll
        for (int u = 0; u < U; ++u) jj[u] = list_at(A.nbr_f, kk + u * TPP, nf, i);
#pragma unroll
        for (int u = 0; u < U; ++u) xj[u] = A.pos[jj[u]];
#pragma unroll
        for (int u = 0; u < U; ++u) f(jj[u], xj[u]);
    }
    for (; kk < n; kk += TPP) {
        const unsigned j = list_at(A.nbr_f, kk, nf, i);
        f(j, A.pos[j]);
    }
}

/* Sum over the TPP adjacent lanes of a particle's lane group. */
template <int TPP>
__device__ __forceinline__ float group_sum(float v)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gmask = TPP == 32 ? 0xffffffffu : ((1u << TPP) - 1u) << (lane - lane % TPP);
    for (int o = TPP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
    return v;
}

/* ---------------------------------------------------------------------- */
/* PCISPH boundary method (PCISPHBoundaryObject.cpp:218-447)                 */

/* Collision sums over the boundary candidates of x's cell: particles within
   rest_r of x (test position) weigh w = max(0, (rest_r - |y - x_b|) / rest_r)
   with y the weight position (x itself, or the predicted position), and
   contribute w, w (rest_r - |y - x_b|) and w n_b. */
__device__ __forceinline__ void pcib_collide(const SimParams& P, const DeviceArrays& A, float4 x, float4 y,
                                             float& wsum, float& w2sum, float3& avg)
{
    wsum = 0.0f;
    w2sum = 0.0f;
    avg = make_float3(0.0f, 0.0f, 0.0f);
    for_cells27(x, P.h, grid_single(P), [&](unsigned c) {
        const unsigned e = A.bcell_start[c + 1];
        for (unsigned q = A.bcell_start[c]; q < e; ++q) {
            const float4 xb = A.bpos[q];
            if (!(glm_length(__fsub_rn(x.x, xb.x), __fsub_rn(x.y, xb.y), __fsub_rn(x.z, xb.z)) < P.rest_r)) continue;
            const float l = glm_length(__fsub_rn(y.x, xb.x), __fsub_rn(y.y, xb.y), __fsub_rn(y.z, xb.z));
            const float gap = __fsub_rn(P.rest_r, l);
            const float w = fmaxf(0.0f, __fdiv_rn(gap, P.rest_r));
            wsum = __fadd_rn(wsum, w);
            w2sum = __fadd_rn(w2sum, __fmul_rn(w, gap));
            const float4 nb = A.bnormal[q];
            avg.x = __fadd_rn(avg.x, __fmul_rn(w, nb.x));
            avg.y = __fadd_rn(avg.y, __fmul_rn(w, nb.y));
            avg.z = __fadd_rn(avg.z, __fmul_rn(w, nb.z));
        }
    });
}

/* n = normalize(avg) (NaN for a zero sum, as glm computes it); when some
   weight is positive the point moves by (w2sum / wsum) n. */
__device__ __forceinline__ float4 pcib_push(float4 p, float wsum, float w2sum, float3 avg, float4& n)
{
    const float inv = __fdiv_rn(1.0f, __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(avg.x, avg.x), __fmul_rn(avg.y, avg.y)),
                                                          __fmul_rn(avg.z, avg.z))));
    n = make_float4(__fmul_rn(avg.x, inv), __fmul_rn(avg.y, inv), __fmul_rn(avg.z, inv), 0.0f);
    if (wsum > 0.0f) {
        const float s = __fmul_rn(__fdiv_rn(1.0f, wsum), w2sum);
        p.x = __fadd_rn(p.x, __fmul_rn(s, n.x));
        p.y = __fadd_rn(p.y, __fmul_rn(s, n.y));
        p.z = __fadd_rn(p.z, __fmul_rn(s, n.z));
    }
    return p;
}

/* correctVelocities: where |n| > 0, v_out = tf (u - (u.n) n) - nf (u.n) n
   for the reference velocity u */
__device__ __forceinline__ void pcib_velocity(const SimParams& P, float4 n, float4 u, float4& v_out)
{
    if (!(glm_length(n.x, n.y, n.z) > 0.0f)) return;
    const float d = __fadd_rn(__fadd_rn(__fmul_rn(u.x, n.x), __fmul_rn(u.y, n.y)), __fmul_rn(u.z, n.z));
    const float nx = __fmul_rn(d, n.x), ny = __fmul_rn(d, n.y), nz = __fmul_rn(d, n.z);
    v_out.x = __fsub_rn(__fmul_rn(P.pcib_tf, __fsub_rn(u.x, nx)), __fmul_rn(P.pcib_nf, nx));
    v_out.y = __fsub_rn(__fmul_rn(P.pcib_tf, __fsub_rn(u.y, ny)), __fmul_rn(P.pcib_nf, ny));
    v_out.z = __fsub_rn(__fmul_rn(P.pcib_tf, __fsub_rn(u.z, nz)), __fmul_rn(P.pcib_nf, nz));
}

/* Density of boundary particle q: fluid candidates of its 27 cells first,
   then boundary candidates, each term m W(x_q - x_j) added in turn. POLY6:
   PCISPHSolver::predictBoundaryDensities (PCISPHSolver.cpp:211-244) at the
   predicted fluid positions; else SPHSolver::computeBoundaryDensities
   (SPHSolver.cpp:91-124) with the cubic spline at the current ones. */
template <bool POLY6>
__device__ __forceinline__ float boundary_density(const SimParams& P, const DeviceArrays& A, unsigned q)
{
    const float4 xq = A.bpos[q];
    const Grid g = grid_single(P);
    float rho = 0.0f;
    for_cells27(xq, P.h, g, [&](unsigned c) {
        const unsigned e = A.cell_start[c + 1];
        for (unsigned j = A.cell_start[c]; j < e; ++j) {
            const float4 xj = POLY6 ? A.predr[j] : A.pos[j];
            const float s2 = dist2_exact(xq, xj);
            if (!(s2 <= P.h2_guard)) continue;
            const float w = POLY6 ? poly6_W(__fsub_rn(xq.x, xj.x), __fsub_rn(xq.y, xj.y), __fsub_rn(xq.z, xj.z), P)
                                  : cs_W_exact(s2, P);
            rho = __fadd_rn(rho, __fmul_rn(P.mass, w));
        }
    });
    for_cells27(xq, P.h, g, [&](unsigned c) {
        const unsigned e = A.bcell_start[c + 1];
        for (unsigned b = A.bcell_start[c]; b < e; ++b) {
            const float4 xb = A.bpos[b];
            const float s2 = dist2_exact(xq, xb);
            if (!(s2 <= P.h2_guard)) continue;
            const float w = POLY6 ? poly6_W(__fsub_rn(xq.x, xb.x), __fsub_rn(xq.y, xb.y), __fsub_rn(xq.z, xb.z), P)
                                  : cs_W_exact(s2, P);
            rho = __fadd_rn(rho, __fmul_rn(xb.w, w));
        }
    });
    return rho;
}

/* ---------------------------------------------------------------------- */

/* DIVRES: also the divergence error of the current velocities
   (DFSPHSolver::computeDivergenceError, DFSPHSolver.cpp:538-621), which the
   divergence solver's warm start reads (A.divres) instead of spending a
   neighbour pass on it: the velocities do not change between this pass
   and that solver. */
template <bool ALPHA, bool EOS, bool DIVRES = false>
__global__ void __launch_bounds__(256, 8) k_density(SimParams P, DeviceArrays A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active_n(P, A.st)) return;
    const size_t nf = (size_t)P.nf;
    const float4 xi = A.pos[i];
    const float4 vi = DIVRES ? A.vel[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float rho = 0.0f, sgx = 0.0f, sgy = 0.0f, sgz = 0.0f, ssq = 0.0f, div = 0.0f;
    const unsigned nF = A.cnt_f[i];
    for_fluid_neighbors<2>(A, i, nf, nF, [&](unsigned j, const float4& xj) {
        rho = __fadd_rn(rho, __fmul_rn(P.mass, cs_W_exact(dist2_exact(xi, xj), P)));
        if (ALPHA) {
            const Pair p = make_pair(xi, xj);
            const float fg = cs_gradf(p.rl, p.inv_rl, P);
            const float f = P.mass * fg;
            const float gx = f * p.rx, gy = f * p.ry, gz = f * p.rz;
            sgx += gx; sgy += gy; sgz += gz;
            ssq += (gx * gx + gy * gy) + gz * gz;
            if (DIVRES) {
                const float4 vj = A.vel[j];
                div += P.mass * (fg * (((vi.x - vj.x) * p.rx + (vi.y - vj.y) * p.ry) + (vi.z - vj.z) * p.rz));
            }
        }
    });
    const unsigned nB = A.cnt_b[i];
    for (unsigned kk = 0; kk < nB; ++kk) {
        const float4 xb = A.bpos[list_at(A.nbr_b, kk, nf, i)];
        rho = __fadd_rn(rho, __fmul_rn(xb.w, cs_W_exact(dist2_exact(xi, xb), P)));
        if (ALPHA) {
            const Pair p = make_pair(xi, xb);
            const float fg = cs_gradf(p.rl, p.inv_rl, P);
            const float f = xb.w * fg;
            sgx += f * p.rx; sgy += f * p.ry; sgz += f * p.rz;
            if (DIVRES) div += xb.w * (fg * ((vi.x * p.rx + vi.y * p.ry) + vi.z * p.rz));
        }
    }
    A.rho[i] = rho;
    if (ALPHA) {
        const float denom = ((sgx * sgx + sgy * sgy) + sgz * sgz) + ssq;
        A.alpha[i] = denom > P.eps ? rho / denom : 0.0f;
    }
    if (EOS) A.press[i] = tait_pressure(rho, P, P.kr_g);
    /* fewer than 20 neighbours within h: no correction (DFSPHSolver.cpp:608-611) */
    if (DIVRES) A.divres[i] = (nF + nB < 20u) ? 0.0f : fmaxf(div, 0.0f);
}

/* Density (and the Tait pressure when EOS) of small scenes with TPP lanes per
   particle: in each round the group's lanes evaluate m W for TPP consecutive
   list entries, and lane 0 adds the TPP terms in list order (shuffled to
   it), so the sum is the sequential one bit for bit; the terms of entries
   past the end are +0, which leaves a non-negative sum unchanged. */
template <bool EOS, int TPP>
__device__ __forceinline__ void density_lanes_at(const SimParams& P, const DeviceArrays& A, int t)
{
    const int i = t / TPP;
    /* a group's lanes share i, so a group leaves together */
    if (i >= active_n(P, A.st)) return;
    const unsigned lane = threadIdx.x & 31u, sub = lane % TPP, first = lane - sub;
    const unsigned gmask = ((1u << TPP) - 1u) << first;
    const size_t nf = (size_t)P.nf;
    const float4 xi = A.pos[i];
    float rho = 0.0f;
    const unsigned nF = A.cnt_f[i];
    for (unsigned k0 = 0; k0 < nF; k0 += TPP) {
        const unsigned kk = k0 + sub;
        float w = 0.0f;
        if (kk < nF) w = __fmul_rn(P.mass, cs_W_exact(dist2_exact(xi, A.pos[list_at(A.nbr_f, kk, nf, i)]), P));
#pragma unroll
        for (int l = 0; l < TPP; ++l) rho = __fadd_rn(rho, __shfl_sync(gmask, w, first + l));
    }
    const unsigned nB = A.cnt_b[i];
    for (unsigned k0 = 0; k0 < nB; k0 += TPP) {
        const unsigned kk = k0 + sub;
        float w = 0.0f;
        if (kk < nB) {
            const float4 xb = A.bpos[list_at(A.nbr_b, kk, nf, i)];
            w = __fmul_rn(xb.w, cs_W_exact(dist2_exact(xi, xb), P));
        }
#pragma unroll
        for (int l = 0; l < TPP; ++l) rho = __fadd_rn(rho, __shfl_sync(gmask, w, first + l));
    }
    if (sub != 0) return;
    A.rho[i] = rho;
    if (EOS) A.press[i] = tait_pressure(rho, P, P.kr_g);
}

template <bool EOS, int TPP>
__global__ void __launch_bounds__(256) k_density_lanes(SimParams P, DeviceArrays A)
{
    density_lanes_at<EOS, TPP>(P, A, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(256, 8) k_normals(SimParams P, DeviceArrays A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active_n(P, A.st)) return;
    const size_t nf = (size_t)P.nf;
    const float4 xi = A.pos[i];
    float nx = 0.0f, ny = 0.0f, nz = 0.0f;
    const unsigned nF = A.cnt_f[i];
    for (unsigned kk = 0; kk < nF; ++kk) {
        const unsigned j = list_at(A.nbr_f, kk, nf, i);
        const Pair p = make_pair(xi, A.pos[j]);
        const float f = (P.mass / A.rho[j]) * cs_gradf(p.rl, p.inv_rl, P);
        nx += f * p.rx; ny += f * p.ry; nz += f * p.rz;
    }
    A.normal[i] = make_float4(nx * P.h, ny * P.h, nz * P.h, 0.0f);
}

/* Non-pressure and pressure accelerations (MODE). TPP adjacent lanes share
   particle i (small scenes), each summing the list entries sub, sub + TPP,
   ...; the group's sums are combined by shuffles and lane 0 of the group
   finishes the particle. */
template <int MODE, int TPP = 1>
__device__ __forceinline__ void forces_at(const SimParams& P, const DeviceArrays& A, int t, bool first_thread,
                                          float* s_red)
{
    const int i = t / TPP;
    const unsigned sub = (unsigned)t % TPP;
    const bool active = i < active_n(P, A.st);
    const size_t nf = (size_t)P.nf;
    /* per-scene coefficients and time step of a batch */
    const unsigned scene = (A.sst && active) ? A.sref.scene_of[i] : 0u;
    const float dt = A.sst ? (active ? A.sst[scene].dt : 0.0f) : A.st->dt;
    const float visc_c = A.sst ? (active ? A.sref.scenes[scene].visc : 0.0f) : P.visc;
    const float bvisc_c = A.sst ? (active ? A.sref.scenes[scene].bvisc : 0.0f) : P.bvisc;
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    float4 xi = make_float4(0, 0, 0, 0), vi = xi;
    if (active) {
        xi = A.pos[i];
        vi = A.vel[i];
        const float rho_i = A.rho[i];
        const unsigned nF = A.cnt_f[i], nB = A.cnt_b[i];
        const bool pressure = MODE == FORCE_WCSPH || MODE == FORCE_PRESSURE;
        const bool np = MODE != FORCE_PRESSURE;
        const int vm = np ? P.visc_method : -1;
        const bool st_on = np && P.st_on;
        const float dpi = pressure ? A.press[i] / (rho_i * rho_i) : 0.0f;
        const float dpb = pressure ? A.press[i] / (P.rho0 * P.rho0) : 0.0f;
        const float4 ni = st_on ? A.normal[i] : make_float4(0, 0, 0, 0);
        const float eps_h2 = 0.01f * P.h2;
        float svx = 0.0f, svy = 0.0f, svz = 0.0f; /* standard viscosity sum */
        for_fluid_neighbors<2, TPP>(A, i, nf, nF, [&](unsigned j, const float4& xj) {
            const Pair p = make_pair(xi, xj);
            const float rho_j = A.rho[j];
            const float f = cs_gradf(p.rl, p.inv_rl, P);
            if (pressure) {
                const float pj = A.press[j];
                const float c = P.mass * (dpi + pj / (rho_j * rho_j)) * f;
                ax -= c * p.rx; ay -= c * p.ry; az -= c * p.rz;
            }
            if (vm >= 0) {
                const float4 vj = A.vel[j];
                const float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
                if (vm == 1) {
                    const float dot = (dvx * p.rx + dvy * p.ry) + dvz * p.rz;
                    /* nu (m / rho_j) dot / (|r|^2 + 0.01 h^2) gradW with one fast
                       division (this pass is compared with the reference to a
                       relative tolerance, not bit for bit) */
                    const float c = visc_c * __fdividef(P.mass * dot, rho_j * (p.s + eps_h2)) * f;
                    ax += c * p.rx; ay += c * p.ry; az += c * p.rz;
                } else if (vm == 0) {
                    const float c = P.mass / rho_j * visco_lapl(p.rl, P);
                    svx -= c * dvx; svy -= c * dvy; svz -= c * dvz;
                } else {
                    const float c = visc_c * (P.mass / rho_j) * cs_W(p.rl * P.inv_h, P) / dt;
                    ax -= c * dvx; ay -= c * dvy; az -= c * dvz;
                }
            }
            if (st_on && p.s > 0.0f) {
                const float4 nj = A.normal[j];
                const float kij = 2.0f * P.rho0 / (rho_i + rho_j);
                const float c = P.st * P.mass * cohesion_W(p.rl, P) * p.inv_rl;
                ax += kij * (-c * p.rx - P.st * (ni.x - nj.x));
                ay += kij * (-c * p.ry - P.st * (ni.y - nj.y));
                az += kij * (-c * p.rz - P.st * (ni.z - nj.z));
            }
        }, sub);
        if (TPP > 1) {
            ax = group_sum<TPP>(ax); ay = group_sum<TPP>(ay); az = group_sum<TPP>(az);
            svx = group_sum<TPP>(svx); svy = group_sum<TPP>(svy); svz = group_sum<TPP>(svz);
            /* lane 0 of the group carries the fluid sums on; the boundary sums
               below are split over the lanes again and combined at the end */
            if (sub != 0) ax = ay = az = svx = svy = svz = 0.0f;
        }
        if (vm == 0) {
            const float c = visc_c / rho_i;
            ax += svx * c; ay += svy * c; az += svz * c;
        }
        const bool bvisc = vm >= 0 && bvisc_c != 0.0f;
        if (pressure || bvisc || (np && P.adh_on)) {
            float bvx = 0.0f, bvy = 0.0f, bvz = 0.0f;
            for (unsigned kk = sub; kk < nB; kk += TPP) {
                const unsigned bq = list_at(A.nbr_b, kk, nf, i);
                const float4 xb = A.bpos[bq];
                const Pair p = make_pair(xi, xb);
                const float psi = xb.w;
                const float f = cs_gradf(p.rl, p.inv_rl, P);
                if (pressure) {
                    /* Akinci: rho0 V_b (p_i / rho_i^2 + p_i / rho0^2); PCISPH boundary
                       particles: m_b (p_i / rho_i^2 + p_b / rho_b^2) (WCSPHSolver.cpp:160-184) */
                    const float c = psi * (dpi + (P.pcib ? A.bdp[bq] : dpb)) * f;
                    ax -= c * p.rx; ay -= c * p.ry; az -= c * p.rz;
                }
                if (bvisc) {
                    if (vm == 1) {
                        const float dot = (vi.x * p.rx + vi.y * p.ry) + vi.z * p.rz;
                        const float c = bvisc_c * (psi / rho_i) * dot / (p.s + eps_h2) * f;
                        ax += c * p.rx; ay += c * p.ry; az += c * p.rz;
                    } else if (vm == 0) {
                        const float c = psi / rho_i * visco_lapl(p.rl, P);
                        bvx -= c * vi.x; bvy -= c * vi.y; bvz -= c * vi.z;
                    } else {
                        const float c = bvisc_c * (psi / rho_i) * cs_W(p.rl * P.inv_h, P) / dt;
                        ax -= c * vi.x; ay -= c * vi.y; az -= c * vi.z;
                    }
                }
                if (np && P.adh_on && p.s > 0.0f) {
                    const float c = P.adh * psi * adhesion_W(p.rl, P) * p.inv_rl;
                    ax -= c * p.rx; ay -= c * p.ry; az -= c * p.rz;
                }
            }
            if (bvisc && vm == 0) {
                const float c = bvisc_c / rho_i;
                ax += bvx * c; ay += bvy * c; az += bvz * c;
            }
        }
        if (TPP > 1) {
            ax = group_sum<TPP>(ax); ay = group_sum<TPP>(ay); az = group_sum<TPP>(az);
        }
    }
    /* from here on, lane 0 of each group stands for its particle */
    const bool owner = active && sub == 0;

    if (MODE == FORCE_WCSPH) {
        if (owner) {
            /* SPHSolver::integrate: a += g; v += a dt; x += v dt (unfused, as the reference rounds) */
            ax = __fadd_rn(ax, P.gx); ay = __fadd_rn(ay, P.gy); az = __fadd_rn(az, P.gz);
            const float nvx = __fadd_rn(vi.x, __fmul_rn(ax, dt)), nvy = __fadd_rn(vi.y, __fmul_rn(ay, dt)),
                        nvz = __fadd_rn(vi.z, __fmul_rn(az, dt));
            float4 lo = P.pos_lo ? A.plo[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const float px = pos_add(xi.x, lo.x, __fmul_rn(nvx, dt), P.pos_lo),
                        py = pos_add(xi.y, lo.y, __fmul_rn(nvy, dt), P.pos_lo),
                        pz = pos_add(xi.z, lo.z, __fmul_rn(nvz, dt), P.pos_lo);
            A.vel_alt[i] = make_float4(nvx, nvy, nvz, 0.0f);
            A.pos_alt[i] = make_float4(px, py, pz, 0.0f);
            if (P.pos_lo) A.plo_alt[i] = lo;
            if (!isfinite(px) || !isfinite(py) || !isfinite(pz)) atomicOr(&A.st->err, ERRBIT_NAN);
        }
        if (A.sst) {
            if (owner && (unsigned)i == A.sref.scenes[scene].fbegin) {
                A.sst[scene].time = advance_time(A.sst[scene].time, dt);
                A.sst[scene].steps += 1u;
            }
        } else if (first_thread && !P.dynamic) {
            /* with emitters the step's emission comes first (k_emit advances the time) */
            A.st->time = advance_time(A.st->time, dt);
            A.st->steps += 1u;
        }
        return;
    }
    if (owner) A.acc[i] = make_float4(ax, ay, az, 0.0f);
    if (MODE == FORCE_NP_CFL) {
        float speed = 0.0f;
        if (owner) {
            const float cx = __fadd_rn(vi.x, __fmul_rn(__fadd_rn(ax, P.gx), dt));
            const float cy = __fadd_rn(vi.y, __fmul_rn(__fadd_rn(ay, P.gy), dt));
            const float cz = __fadd_rn(vi.z, __fmul_rn(__fadd_rn(az, P.gz), dt));
            speed = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz)));
            if (!(speed == speed)) speed = 3.0e38f;
        }
        if (A.sst) {
            /* per-scene maximum: one atomic per warp when the warp holds one scene */
            const unsigned s0 = __shfl_sync(0xffffffffu, scene, 0);
            if (__all_sync(0xffffffffu, !active || scene == s0)) {
                const float m = warp_max(speed);
                if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(&A.sst[s0].vmax_bits, __float_as_uint(m));
            } else if (active) {
                atomicMax(&A.sst[scene].vmax_bits, __float_as_uint(speed));
            }
        } else {
            const float m = block_max(speed, s_red);
            if (threadIdx.x == 0) atomicMax(&A.st->vmax_bits, __float_as_uint(m));
        }
    }
}

template <int MODE, int TPP = 1>
__global__ void __launch_bounds__(256, 6) k_forces(SimParams P, DeviceArrays A)
{
    __shared__ float s_red[32];
    forces_at<MODE, TPP>(P, A, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.x == 0 && threadIdx.x == 0, s_red);
}

/* ---------------------------------------------------------------------- */
/* DFSPH pieces                                                             */

/* Sum of the residual terms of particle i over the neighbour-list entries
   sub, sub + TPP, ... (fluid, then boundary). The fluid loop issues the
   gathers of U entries before using any of them (more loads in flight per
   lane) and adds the terms in list order, so U changes no bit. */
template <bool DIV, int TPP, int U = 1>
__device__ __forceinline__ float dfsph_residual_part(const SimParams& P, const DeviceArrays& A, int i, int sub,
                                                     size_t nf)
{
    const float4 xi = A.pos[i];
    const float4 vi = A.vel[i];
    float sum = 0.0f;
    const unsigned nF = A.cnt_f[i], nB = A.cnt_b[i];
    unsigned kk = sub;
    for (; kk + (U - 1) * TPP < nF; kk += U * TPP) {
        unsigned jj[U];
        float4 xj[U], vj[U];
#pragma unroll
        for (int u = 0; u < U; ++u) jj[u] = list_at(A.nbr_f, kk + u * TPP, nf, i);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            xj[u] = A.pos[jj[u]];
            vj[u] = A.vel[jj[u]];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const Pair p = make_pair(xi, xj[u]);
            const float f = cs_gradf(p.rl, p.inv_rl, P);
            sum += P.mass * (f * (((vi.x - vj[u].x) * p.rx + (vi.y - vj[u].y) * p.ry) + (vi.z - vj[u].z) * p.rz));
        }
    }
    for (; kk < nF; kk += TPP) {
        const unsigned j = list_at(A.nbr_f, kk, nf, i);
        const Pair p = make_pair(xi, A.pos[j]);
        const float4 vj = A.vel[j];
        const float f = cs_gradf(p.rl, p.inv_rl, P);
        sum += P.mass * (f * (((vi.x - vj.x) * p.rx + (vi.y - vj.y) * p.ry) + (vi.z - vj.z) * p.rz));
    }
    for (unsigned kk = sub; kk < nB; kk += TPP) {
        const float4 xb = A.bpos[list_at(A.nbr_b, kk, nf, i)];
        const Pair p = make_pair(xi, xb);
        const float f = cs_gradf(p.rl, p.inv_rl, P);
        sum += xb.w * (f * ((vi.x * p.rx + vi.y * p.ry) + vi.z * p.rz));
    }
    return sum;
}

/* The residual from the summed terms: predicted density (DIV=false) or
   divergence error (DIV=true) of particle i. */
template <bool DIV>
__device__ __forceinline__ float dfsph_residual_finish(const SimParams& P, const DeviceArrays& A, int i, float sum,
                                                       float dt)
{
    if (DIV) {
        /* particles with fewer than 20 neighbours within h are not corrected
           (DFSPHSolver.cpp:608-611); the lists hold exactly those neighbours */
        if (A.cnt_f[i] + A.cnt_b[i] < 20u) return 0.0f;
        return fmaxf(sum, 0.0f);
    }
    /* rho_i + dt * change, rounded as the reference rounds it: the result
       enters (rho* - rho0), where a contracted FMA would shift it by an ulp */
    return fmaxf(__fadd_rn(A.rho[i], __fmul_rn(sum, dt)), P.rho0);
}

/* predicted density (DIV=false) or divergence error (DIV=true) of particle i */
template <bool DIV>
__device__ __forceinline__ float dfsph_residual(const SimParams& P, const DeviceArrays& A, int i, size_t nf,
                                                float dt)
{
    return dfsph_residual_finish<DIV>(P, A, i, dfsph_residual_part<DIV, 1>(P, A, i, 0, nf), dt);
}

/* Partial sums over list entries sub, sub + TPP, ... of
   sum_j m (k_i + k_j) gradW  (+ boundary with k_i), the fluid gathers issued
   U at a time as in dfsph_residual_part. K is written inside the same
   persistent kernel (before a grid barrier), so it is a plain pointer: a
   read-only (non-coherent) load path would be wrong for it. */
template <int TPP, int U = 1>
__device__ __forceinline__ void dfsph_correct_part(const SimParams& P, const DeviceArrays& A, const float* K, int i,
                                                   int sub, size_t nf, float& sx, float& sy, float& sz)
{
    const float4 xi = A.pos[i];
    const float ki = K[i];
    sx = sy = sz = 0.0f;
    const unsigned nF = A.cnt_f[i];
    unsigned kk = sub;
    for (; kk + (U - 1) * TPP < nF; kk += U * TPP) {
        unsigned jj[U];
        float kj[U];
        float4 xj[U];
#pragma unroll
        for (int u = 0; u < U; ++u) jj[u] = list_at(A.nbr_f, kk + u * TPP, nf, i);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            kj[u] = K[jj[u]];
            xj[u] = A.pos[jj[u]];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const float ks = ki + kj[u];
            if (fabsf(ks) > P.eps) {
                const Pair p = make_pair(xi, xj[u]);
                const float c = P.mass * ks * cs_gradf(p.rl, p.inv_rl, P);
                sx += c * p.rx; sy += c * p.ry; sz += c * p.rz;
            }
        }
    }
    for (; kk < nF; kk += TPP) {
        const unsigned j = list_at(A.nbr_f, kk, nf, i);
        const float ks = ki + K[j];
        if (fabsf(ks) > P.eps) {
            const Pair p = make_pair(xi, A.pos[j]);
            const float c = P.mass * ks * cs_gradf(p.rl, p.inv_rl, P);
            sx += c * p.rx; sy += c * p.ry; sz += c * p.rz;
        }
    }
    if (fabsf(ki) > P.eps) {
        const unsigned nB = A.cnt_b[i];
        for (unsigned kk = sub; kk < nB; kk += TPP) {
            const float4 xb = A.bpos[list_at(A.nbr_b, kk, nf, i)];
            const Pair p = make_pair(xi, xb);
            const float c = xb.w * ki * cs_gradf(p.rl, p.inv_rl, P);
            sx += c * p.rx; sy += c * p.ry; sz += c * p.rz;
        }
    }
}

__device__ __forceinline__ void dfsph_apply(const DeviceArrays& A, int i, float dt, float sx, float sy, float sz)
{
    float4 v = A.vel[i];
    v.x = __fsub_rn(v.x, __fmul_rn(dt, sx));
    v.y = __fsub_rn(v.y, __fmul_rn(dt, sy));
    v.z = __fsub_rn(v.z, __fmul_rn(dt, sz));
    A.vel[i] = v;
}

/* v_i -= dt * sum_j m (k_i + k_j) gradW  (+ boundary with k_i) */
__device__ __forceinline__ void dfsph_correct(const SimParams& P, const DeviceArrays& A, const float* K, int i,
                                              size_t nf, float dt)
{
    float sx, sy, sz;
    dfsph_correct_part<1>(P, A, K, i, 0, nf, sx, sy, sz);
    dfsph_apply(A, i, dt, sx, sy, sz);
}

/* Sum over the TPP adjacent lanes that share a particle (all lanes call). */
template <int TPP>
__device__ __forceinline__ float lane_group_sum(float v)
{
    for (int o = TPP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* Calls f(i, sub, valid) for every particle i < n, TPP adjacent lanes per
   particle (sub = lane index within the group), up to 32 / TPP particles per
   warp and round. In each full round the warps take consecutive groups of
   32 / TPP particles, so at any moment the whole grid works on one stretch
   of the cell-ordered arrays (whose state and lists then stay in L2); the
   particles left over for the last round are spread evenly over all warps,
   so that no warp sits out the last round while others run a full group.
   The trip count is uniform per warp, so f may use warp shuffles; lanes
   without a particle get valid = false. */
template <int TPP, typename F>
__device__ __forceinline__ void for_particles(int n, F&& f)
{
    constexpr int PPW = 32 / TPP;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int per_round = nw * PPW;
    const int full = n / per_round;
    for (int r = 0; r < full; ++r) f(r * per_round + gw * PPW + lane / TPP, lane % TPP, true);
    const int base = full * per_round, rem = n - base;
    if (rem > 0) {
        const int lo = base + (int)(((long long)rem * gw) / nw);
        const int hi = base + (int)(((long long)rem * (gw + 1)) / nw);
        const int i = lo + lane / TPP;
        f(i, lane % TPP, i < hi);
    }
}

/* residual of particle i with its list split over TPP lanes (all lanes call) */
template <bool DIV, int TPP, int U>
__device__ __forceinline__ float dfsph_residual_lanes(const SimParams& P, const DeviceArrays& A, int i, int sub,
                                                      bool valid, size_t nf, float dt)
{
    float part = valid ? dfsph_residual_part<DIV, TPP, U>(P, A, i, sub, nf) : 0.0f;
    if (TPP > 1) part = lane_group_sum<TPP>(part);
    return valid ? dfsph_residual_finish<DIV>(P, A, i, part, dt) : 0.0f;
}

/* velocity correction of particle i with its list split over TPP lanes */
template <int TPP, int U>
__device__ __forceinline__ void dfsph_correct_lanes(const SimParams& P, const DeviceArrays& A, const float* K, int i,
                                                    int sub, bool valid, size_t nf, float dt)
{
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    if (valid) dfsph_correct_part<TPP, U>(P, A, K, i, sub, nf, sx, sy, sz);
    if (TPP > 1) {
        sx = lane_group_sum<TPP>(sx);
        sy = lane_group_sum<TPP>(sy);
        sz = lane_group_sum<TPP>(sz);
    }
    if (valid && sub == 0) dfsph_apply(A, i, dt, sx, sy, sz);
}

/* OCC blocks of 256 per SM: 8 (32 registers) by default -- the passes are
   bound by the latency of dependent neighbour gathers and full occupancy
   hides most of it; 4 (64 registers, no spills) is the autotuner's other
   candidate. TPP lanes share a particle in the neighbour passes (1, 2 or 4):
   more gathers in flight per particle, fewer particles per warp. Each lane
   issues U gathers before using them: 2 within the 32 registers of the
   8-block variant, 4 in the 64-register variant (measured best for each on
   the 1M-particle scene). */
template <bool DIV, int OCC, int TPP>
__global__ void __launch_bounds__(kSolverBlock, OCC) k_dfsph_solve(SimParams P, DeviceArrays A)
{
    constexpr int U = OCC == 4 ? 4 : 2;
    __shared__ double s_red[32];
    DevState* st = A.st;
    const int nfi = active_n(P, st);
    const size_t nf = (size_t)P.nf;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;

    float dt;
    float vmax = 0.0f;
    if (!DIV) {
        /* DFSPHSolver::updateTimeStep: CFL bound and iteration-count rule */
        const float dt_old = st->dt;
        vmax = __uint_as_float(st->vmax_bits);
        if (vmax < 1.0e-9f) vmax = 1.0e-9f;
        const float cfl_ts = P.cfl * 0.4f * (2.0f * P.r) / vmax;
        const unsigned its = max(st->its, st->its_v);
        float hs = dt_old;
        if (its > 6u) hs *= 0.9f;
        else if (its < 4u) hs *= 1.05f;
        hs = fminf(hs, cfl_ts);
        hs = fmaxf(hs, P.min_ts);
        hs = fminf(hs, P.max_ts);
        dt = hs;
        /* DFSPHSolver::predictVelocities */
        for (int i = tid; i < nfi; i += nthr) {
            const float4 a = A.acc[i];
            float4 v = A.vel[i];
            v.x = __fadd_rn(v.x, __fmul_rn(__fadd_rn(a.x, P.gx), dt));
            v.y = __fadd_rn(v.y, __fmul_rn(__fadd_rn(a.y, P.gy), dt));
            v.z = __fadd_rn(v.z, __fmul_rn(__fadd_rn(a.z, P.gz), dt));
            /* PCISPH boundary method: PCISPHBoundaryObject::correctVelocities
               with the normals left by the last collision pass (or by the
               surface-tension pass of this step, which shares the array) */
            if (P.pcib) pcib_velocity(P, A.normal[i], v, v);
            A.vel[i] = v;
            A.acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (!grid_barrier(st)) return;
    } else {
        dt = st->dt;
    }
    const float ts2 = dt * dt;
    float* kws = DIV ? A.kvws : A.kws;

    /* warm start: residual at the current velocities, keep the previous
       step's accumulated k only where the residual is positive */
    for_particles<TPP>(nfi, [&](int i, int sub, bool valid) {
        /* the divergence error may come from the density pass (A.divres) */
        const float r = (DIV && A.divres) ? (valid ? A.divres[i] : 0.0f)
                                          : dfsph_residual_lanes<DIV, TPP, U>(P, A, i, sub, valid, nf, dt);
        if (valid && sub == 0) {
            if (DIV) kws[i] = r > 0.0f ? kws[i] / dt : 0.0f;
            else kws[i] = r > P.rho0 ? kws[i] / ts2 : 0.0f;
        }
    });
    if (!grid_barrier(st)) return;
    for_particles<TPP>(nfi, [&](int i, int sub, bool valid) { dfsph_correct_lanes<TPP, U>(P, A, kws, i, sub, valid, nf, dt); });
    if (!grid_barrier(st)) return;
    /* same particle-to-lane mapping as the accumulation below (no barrier between) */
    for_particles<TPP>(nfi, [&](int i, int sub, bool valid) {
        if (valid && sub == 0) kws[i] = 0.0f;
    });

    const double limit = DIV ? (double)(P.eta_v / dt) : (double)P.eta;
    const unsigned min_it = DIV ? P.min_it_v : P.min_it;
    /* the divergence loop is capped by maxIterations, not maxIterationsV
       (DFSPHSolver.cpp:746) */
    const unsigned max_it = P.max_it;
    unsigned it = 0;
    double avg = 0.0;
    while ((avg > limit || it < min_it) && it < max_it) {
        double local = 0.0;
        for_particles<TPP>(nfi, [&](int i, int sub, bool valid) {
            const float r = dfsph_residual_lanes<DIV, TPP, U>(P, A, i, sub, valid, nf, dt);
            if (!valid || sub != 0) return;
            float k;
            if (DIV) {
                k = r * A.alpha[i] / (dt * A.rho[i]);
                local += (double)(r / P.rho0);
            } else {
                k = __fdiv_rn(__fmul_rn(__fsub_rn(r, P.rho0), A.alpha[i]), __fmul_rn(ts2, A.rho[i]));
                local += (double)((r - P.rho0) / P.rho0);
            }
            A.k[i] = k;
            kws[i] += k;
        });
        const double bs = block_sum(local, s_red);
        if (threadIdx.x == 0) atomicAdd(&A.accum[it], bs);
        if (!grid_barrier(st)) return;
        avg = *(volatile double*)&A.accum[it] / (double)nfi;
        for_particles<TPP>(nfi, [&](int i, int sub, bool valid) { dfsph_correct_lanes<TPP, U>(P, A, A.k, i, sub, valid, nf, dt); });
        if (!grid_barrier(st)) return;
        ++it;
    }

    const float scale = DIV ? dt : ts2;
    /* the particle-to-lane mapping of the zeroing and accumulation passes:
       with no iteration there is no barrier after the zeroing */
    for_particles<TPP>(nfi, [&](int i, int sub, bool valid) {
        if (valid && sub == 0) kws[i] *= scale;
    });
    if (!DIV) {
        /* DFSPHSolver::updatePositions */
        bool bad = false;
        for (int i = tid; i < nfi; i += nthr) {
            const float4 v = A.vel[i];
            float4 x = A.pos[i];
            float4 lo = P.pos_lo ? A.plo[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            x.x = pos_add(x.x, lo.x, __fmul_rn(v.x, dt), P.pos_lo);
            x.y = pos_add(x.y, lo.y, __fmul_rn(v.y, dt), P.pos_lo);
            x.z = pos_add(x.z, lo.z, __fmul_rn(v.z, dt), P.pos_lo);
            A.pos[i] = x;
            if (P.pos_lo) A.plo[i] = lo;
            bad |= !isfinite(x.x) || !isfinite(x.y) || !isfinite(x.z);
        }
        if (bad) atomicOr(&st->err, ERRBIT_NAN);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (!DIV) {
            st->dt = dt;
            st->its = it;
            st->avg_dens = avg;
            st->sum_its += it;
            st->last_vmax = vmax;
        } else {
            st->its_v = it;
            st->avg_div = avg;
            st->sum_its_v += it;
            st->time = advance_time(st->time, dt);
            st->steps += 1u;
            st->vmax_bits = 0u;
        }
    }
}

/* ---------------------------------------------------------------------- */
/* DFSPH over a batch of independent scenes: the same passes, each scene with
   its own dt (CFL + iteration rule), residual and convergence test. A scene
   that has converged stops contributing; the loop runs until no scene is
   active (masked convergence). Residuals are reduced per scene in FP64 with
   one atomic per warp when the warp holds a single scene.                  */

__device__ __forceinline__ void scene_accumulate(double* accum, unsigned stride, unsigned it, unsigned scene,
                                                 bool valid, double v)
{
    const unsigned s0 = __shfl_sync(0xffffffffu, scene, 0);
    if (__all_sync(0xffffffffu, !valid || scene == s0)) {
        v = warp_sum(valid ? v : 0.0);
        if ((threadIdx.x & 31) == 0) atomicAdd(&accum[(size_t)s0 * stride + it], v);
    } else if (valid) {
        atomicAdd(&accum[(size_t)scene * stride + it], v);
    }
}

template <bool DIV>
__global__ void __launch_bounds__(kSolverBlock, 8) k_dfsph_solve_batch(SimParams P, DeviceArrays A)
{
    DevState* st = A.st;
    SceneState* sst = A.sst;
    const SceneInfo* sc = A.sref.scenes;
    const unsigned* so = A.sref.scene_of;
    const int nfi = P.nf, ns = A.nscenes;
    const size_t nf = (size_t)nfi;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const unsigned stride = A.accum_stride;
    const unsigned min_it = DIV ? P.min_it_v : P.min_it;
    const unsigned max_it = P.max_it;

    /* per-scene time step (DFSPHSolver::updateTimeStep) and first activity */
    for (int s = tid; s < ns; s += nthr) {
        float dt;
        if (!DIV) {
            float vmax = __uint_as_float(sst[s].vmax_bits);
            if (vmax < 1.0e-9f) vmax = 1.0e-9f;
            const float cfl_ts = P.cfl * 0.4f * (2.0f * P.r) / vmax;
            const unsigned its = max(sst[s].its, sst[s].its_v);
            float hs = sst[s].dt;
            if (its > 6u) hs *= 0.9f;
            else if (its < 4u) hs *= 1.05f;
            hs = fminf(hs, cfl_ts);
            hs = fmaxf(hs, P.min_ts);
            dt = fminf(hs, P.max_ts);
            sst[s].last_vmax = vmax;
        } else {
            dt = sst[s].dt;
        }
        sst[s].dt_next = dt;
        sst[s].active = (min_it > 0u && max_it > 0u) ? 1u : 0u;  /* parity 0: iteration 0 */
    }
    if (!grid_barrier(st)) return;
    if (!DIV) {
        for (int i = tid; i < nfi; i += nthr) {
            const float dt = sst[so[i]].dt_next;
            const float4 a = A.acc[i];
            float4 v = A.vel[i];
            v.x = __fadd_rn(v.x, __fmul_rn(__fadd_rn(a.x, P.gx), dt));
            v.y = __fadd_rn(v.y, __fmul_rn(__fadd_rn(a.y, P.gy), dt));
            v.z = __fadd_rn(v.z, __fmul_rn(__fadd_rn(a.z, P.gz), dt));
            A.vel[i] = v;
            A.acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (!grid_barrier(st)) return;
    }
    float* kws = DIV ? A.kvws : A.kws;
    for (int i = tid; i < nfi; i += nthr) {
        const float dt = sst[so[i]].dt_next;
        /* the divergence error may come from the density pass (A.divres) */
        const float r = (DIV && A.divres) ? A.divres[i] : dfsph_residual<DIV>(P, A, i, nf, dt);
        if (DIV) kws[i] = r > 0.0f ? kws[i] / dt : 0.0f;
        else kws[i] = r > P.rho0 ? kws[i] / (dt * dt) : 0.0f;
    }
    if (!grid_barrier(st)) return;
    for (int i = tid; i < nfi; i += nthr) dfsph_correct(P, A, kws, i, nf, sst[so[i]].dt_next);
    if (!grid_barrier(st)) return;
    for (int i = tid; i < nfi; i += nthr) kws[i] = 0.0f;

    /* activity for iteration it lives in bit (it & 1) of SceneState::active;
       the convergence test of iteration it keeps that bit (the correction
       pass of the same iteration still reads it) and sets the other one,
       dropping whatever the iteration before left there */
    bool any = min_it > 0u && max_it > 0u && ns > 0;
    unsigned it = 0;
    while (any) {
        const unsigned bit = 1u << (it & 1u);
        for (int i0 = tid - lane; i0 < nfi; i0 += nthr) {
            const int i = i0 + lane;
            const bool valid_i = i < nfi;
            const unsigned s = valid_i ? so[i] : 0u;
            const bool on = valid_i && (sst[s].active & bit);
            double err = 0.0;
            if (on) {
                const float dt = sst[s].dt_next;
                const float r = dfsph_residual<DIV>(P, A, i, nf, dt);
                float k;
                if (DIV) {
                    k = r * A.alpha[i] / (dt * A.rho[i]);
                    err = (double)(r / P.rho0);
                } else {
                    k = __fdiv_rn(__fmul_rn(__fsub_rn(r, P.rho0), A.alpha[i]), __fmul_rn(dt * dt, A.rho[i]));
                    err = (double)((r - P.rho0) / P.rho0);
                }
                A.k[i] = k;
                kws[i] += k;
            } else if (valid_i) {
                A.k[i] = 0.0f;
            }
            scene_accumulate(A.accum, stride, it, s, on, err);
        }
        if (!grid_barrier(st)) return;
        /* convergence test per scene for the next iteration */
        const unsigned nbit = 1u << ((it + 1u) & 1u);
        for (int s = tid; s < ns; s += nthr) {
            const unsigned cur = sst[s].active;
            unsigned nxt = 0u;
            if (cur & bit) {
                const double avg = *(volatile double*)&A.accum[(size_t)s * stride + it] / (double)(sc[s].fend - sc[s].fbegin);
                const float dt = sst[s].dt_next;
                const double limit = DIV ? (double)(P.eta_v / dt) : (double)P.eta;
                if (DIV) sst[s].avg_div = avg;
                else sst[s].avg_dens = avg;
                nxt = ((avg > limit || it + 1u < min_it) && it + 1u < max_it) ? 1u : 0u;
                if (DIV) sst[s].its_v = it + 1u;
                else sst[s].its = it + 1u;
                if (nxt) atomicOr(&A.any_active[it + 1u], 1u);
            }
            sst[s].active = (cur & bit) | (nxt ? nbit : 0u);
        }
        for (int i = tid; i < nfi; i += nthr) {
            const unsigned s = so[i];
            if (sst[s].active & bit) dfsph_correct(P, A, A.k, i, nf, sst[s].dt_next);
        }
        if (!grid_barrier(st)) return;
        any = *(volatile unsigned*)&A.any_active[it + 1u] != 0u;
        ++it;
    }

    for (int i = tid; i < nfi; i += nthr) {
        const float dt = sst[so[i]].dt_next;
        kws[i] *= DIV ? dt : dt * dt;
    }
    if (!DIV) {
        bool bad = false;
        for (int i = tid; i < nfi; i += nthr) {
            const float dt = sst[so[i]].dt_next;
            const float4 v = A.vel[i];
            float4 x = A.pos[i];
            x.x = __fadd_rn(x.x, __fmul_rn(v.x, dt));
            x.y = __fadd_rn(x.y, __fmul_rn(v.y, dt));
            x.z = __fadd_rn(x.z, __fmul_rn(v.z, dt));
            A.pos[i] = x;
            bad |= !isfinite(x.x) || !isfinite(x.y) || !isfinite(x.z);
        }
        if (bad) atomicOr(&st->err, ERRBIT_NAN);
    }
    for (int s = tid; s < ns; s += nthr) {
        if (!DIV) {
            if (min_it == 0u || max_it == 0u) sst[s].its = 0u;
            sst[s].dt = sst[s].dt_next;
            sst[s].sum_its += sst[s].its;
        } else {
            if (min_it == 0u || max_it == 0u) sst[s].its_v = 0u;
            sst[s].sum_its_v += sst[s].its_v;
            sst[s].time = advance_time(sst[s].time, sst[s].dt);
            sst[s].steps += 1u;
            sst[s].vmax_bits = 0u;
        }
        sst[s].active = 0u;
    }
}

/* ---------------------------------------------------------------------- */
/* PCISPH                                                                   */

__global__ void __launch_bounds__(kSolverBlock, 4) k_pcisph_solve(SimParams P, DeviceArrays A)
{
    __shared__ double s_red[32];
    DevState* st = A.st;
    const int nfi = active_n(P, st);
    const size_t nf = (size_t)P.nf;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    const float dt = st->dt;

    /* PCISPHSolver::initPressure (boundary pressures too with PCISPH boundary particles) */
    for (int i = tid; i < nfi; i += nthr) {
        A.press[i] = 0.0f;
        A.pacc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (P.pcib)
        for (int q = tid; q < P.nb; q += nthr) A.bpress[q] = 0.0f;
    unsigned it = 0;
    /* the first test uses the residual left by the previous step (PCISPHSolver.cpp:374) */
    double avg = st->pcisph_avg;
    while ((avg > (double)P.eta || it < P.min_it) && it < P.max_it) {
        /* predictVelocityAndPosition */
        for (int i = tid; i < nfi; i += nthr) {
            const float4 a = A.acc[i], pa = A.pacc[i], v = A.vel[i], x = A.pos[i];
            /* acc = (a + pacc) + g; predV = v + acc dt; predR = r + predV dt */
            const float vx = __fadd_rn(v.x, __fmul_rn(__fadd_rn(__fadd_rn(a.x, pa.x), P.gx), dt));
            const float vy = __fadd_rn(v.y, __fmul_rn(__fadd_rn(__fadd_rn(a.y, pa.y), P.gy), dt));
            const float vz = __fadd_rn(v.z, __fmul_rn(__fadd_rn(__fadd_rn(a.z, pa.z), P.gz), dt));
            float4 pr = make_float4(__fadd_rn(x.x, __fmul_rn(vx, dt)), __fadd_rn(x.y, __fmul_rn(vy, dt)),
                                    __fadd_rn(x.z, __fmul_rn(vz, dt)), 0.0f);
            if (P.pcib) {
                /* PCISPHBoundaryObject::correctPredPositions (:390-438): tested at the
                   current position (whose cell holds lists), weighted at the
                   predicted one, which moves */
                A.predv[i] = make_float4(vx, vy, vz, 0.0f);
                float wsum, w2sum;
                float3 avg;
                pcib_collide(P, A, x, pr, wsum, w2sum, avg);
                float4 n;
                pr = pcib_push(pr, wsum, w2sum, avg, n);
                A.normal[i] = n;
            }
            A.predr[i] = pr;
        }
        if (!grid_barrier(st)) return;
        /* predictFluidDensities over the start-of-step candidates of the 27
           cells around the particle's current cell, then updatePressure */
        double local = 0.0;
        for (int i = tid; i < nfi; i += nthr) {
            const float4 xi = A.pos[i];
            const float4 pi = A.predr[i];
            /* all fluid candidates of the 27 cells first, then all boundary
               candidates: the reference's summation order (PCISPHSolver.cpp:180-206) */
            const Grid g = grid_for(P, A.sref, (unsigned)i);
            float rho = 0.0f;
            for_cells27(xi, P.h, g, [&](unsigned c) {
                const unsigned e = A.cell_start[c + 1];
                for (unsigned q = A.cell_start[c]; q < e; ++q) {
                    const float s2 = dist2_exact(pi, A.predr[q]);
                    if (s2 <= P.h2_guard) rho = __fadd_rn(rho, __fmul_rn(P.mass, cs_W_exact(s2, P)));
                }
            });
            if (P.nb > 0)
                for_cells27(xi, P.h, g, [&](unsigned c) {
                    const unsigned e = A.bcell_start[c + 1];
                    for (unsigned q = A.bcell_start[c]; q < e; ++q) {
                        const float4 xb = A.bpos[q];
                        const float s2 = dist2_exact(pi, xb);
                        if (s2 <= P.h2_guard) rho = __fadd_rn(rho, __fmul_rn(xb.w, cs_W_exact(s2, P)));
                    }
                });
            A.rho[i] = rho;
            const float err = fmaxf(0.0f, __fsub_rn(rho, P.rho0));
            A.press[i] = __fadd_rn(A.press[i], __fmul_rn(P.pcisph_delta, err));
            local += (double)(err / P.rho0);
        }
        if (P.pcib)
            /* predictBoundaryDensities (Poly6) and their pressure update with
               the fluid's scaling factor (PCISPHSolver.cpp:211-244, 279-297) */
            for (int q = tid; q < P.nb; q += nthr) {
                const float rb = boundary_density<true>(P, A, (unsigned)q);
                A.bdens[q] = rb;
                const float err = fmaxf(0.0f, __fsub_rn(rb, P.rho0));
                A.bpress[q] = __fadd_rn(A.bpress[q], __fmul_rn(P.pcisph_delta, err));
            }
        const double bs = block_sum(local, s_red);
        if (threadIdx.x == 0) atomicAdd(&A.accum[it], bs);
        if (!grid_barrier(st)) return;
        avg = *(volatile double*)&A.accum[it] / (double)nfi;
        /* computePressureAcc at the current positions, with the reference's
           exact gradient arithmetic: the result feeds the next predicted
           positions, whose densities enter the ill-conditioned p update */
        for (int i = tid; i < nfi; i += nthr) {
            const float4 xi = A.pos[i];
            const float rho_i = A.rho[i];
            const float dpi = __fdiv_rn(A.press[i], __fmul_rn(rho_i, rho_i));
            float ax = 0.0f, ay = 0.0f, az = 0.0f;
            const unsigned nF = A.cnt_f[i], nB = A.cnt_b[i];
            for (unsigned kk = 0; kk < nF; ++kk) {
                const unsigned j = list_at(A.nbr_f, kk, nf, i);
                const float4 xj = A.pos[j];
                const float rho_j = A.rho[j];
                float gx, gy, gz;
                cs_gradW_exact(__fsub_rn(xi.x, xj.x), __fsub_rn(xi.y, xj.y), __fsub_rn(xi.z, xj.z), P, gx, gy, gz);
                const float c = __fmul_rn(P.mass, __fadd_rn(dpi, __fdiv_rn(A.press[j], __fmul_rn(rho_j, rho_j))));
                ax = __fsub_rn(ax, __fmul_rn(c, gx));
                ay = __fsub_rn(ay, __fmul_rn(c, gy));
                az = __fsub_rn(az, __fmul_rn(c, gz));
            }
            for (unsigned kk = 0; kk < nB; ++kk) {
                const unsigned bq = list_at(A.nbr_b, kk, nf, i);
                const float4 xb = A.bpos[bq];
                float gx, gy, gz, c;
                if (P.pcib) {
                    /* m_b (p_i / rho_i^2 + p_b / rho_b^2) Spiky::gradW (PCISPHSolver.cpp:336-347) */
                    spiky_gradW(__fsub_rn(xi.x, xb.x), __fsub_rn(xi.y, xb.y), __fsub_rn(xi.z, xb.z), P, gx, gy, gz);
                    const float rb = A.bdens[bq];
                    c = __fmul_rn(xb.w, __fadd_rn(dpi, __fdiv_rn(A.bpress[bq], __fmul_rn(rb, rb))));
                } else {
                    cs_gradW_exact(__fsub_rn(xi.x, xb.x), __fsub_rn(xi.y, xb.y), __fsub_rn(xi.z, xb.z), P, gx, gy, gz);
                    c = __fmul_rn(xb.w, dpi);
                }
                ax = __fsub_rn(ax, __fmul_rn(c, gx));
                ay = __fsub_rn(ay, __fmul_rn(c, gy));
                az = __fsub_rn(az, __fmul_rn(c, gz));
            }
            A.pacc[i] = make_float4(ax, ay, az, 0.0f);
        }
        ++it;
    }
    if (!grid_barrier(st)) return;
    /* PCISPHSolver::integrate */
    bool bad = false;
    for (int i = tid; i < nfi; i += nthr) {
        const float4 a = A.acc[i], pa = A.pacc[i];
        float4 v = A.vel[i], x = A.pos[i];
        /* a += g + pacc; v += a dt; x += v dt */
        const float axx = __fadd_rn(a.x, __fadd_rn(P.gx, pa.x));
        const float ayy = __fadd_rn(a.y, __fadd_rn(P.gy, pa.y));
        const float azz = __fadd_rn(a.z, __fadd_rn(P.gz, pa.z));
        v.x = __fadd_rn(v.x, __fmul_rn(axx, dt)); v.y = __fadd_rn(v.y, __fmul_rn(ayy, dt));
        v.z = __fadd_rn(v.z, __fmul_rn(azz, dt));
        float4 lo = P.pos_lo ? A.plo[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        x.x = pos_add(x.x, lo.x, __fmul_rn(v.x, dt), P.pos_lo);
        x.y = pos_add(x.y, lo.y, __fmul_rn(v.y, dt), P.pos_lo);
        x.z = pos_add(x.z, lo.z, __fmul_rn(v.z, dt), P.pos_lo);
        if (P.pos_lo) A.plo[i] = lo;
        if (P.pcib) {
            /* correctPositions (PCISPH branch, :226-262): candidates of the new
               cell if the last search listed it, weights at the predicted
               position; then correctVelocities from the predicted velocity */
            float wsum = 0.0f, w2sum = 0.0f;
            float3 avg = make_float3(0.0f, 0.0f, 0.0f);
            if (cell_listed(A.cell_entry, cell_index(x, P.h, grid_single(P)), st->ns_epoch))
                pcib_collide(P, A, x, A.predr[i], wsum, w2sum, avg);
            float4 n;
            x = pcib_push(x, wsum, w2sum, avg, n);
            A.normal[i] = n;
            pcib_velocity(P, n, A.predv[i], v);
        }
        A.vel[i] = v;
        A.pos[i] = x;
        A.acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        bad |= !isfinite(x.x) || !isfinite(x.y) || !isfinite(x.z);
    }
    if (bad) atomicOr(&st->err, ERRBIT_NAN);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->its = it;
        st->pcisph_avg = avg;
        st->avg_dens = avg;
        st->sum_its += it;
        if (!P.dynamic) {
            /* with emitters the step's emission comes first (k_emit advances the time) */
            st->time = advance_time(st->time, dt);
            st->steps += 1u;
        }
    }
}

/* ---------------------------------------------------------------------- */
/* PCISPH boundary method passes outside the persistent solvers             */

/* SPHSolver::computeBoundaryDensities + WCSPHSolver::computeBoundaryPressures:
   rho_b, p_b = max(0, k rho0 / gamma ((rho_b / rho0)^gamma - 1)), p_b / rho_b^2 */
__global__ void __launch_bounds__(256) k_boundary_density(SimParams P, DeviceArrays A)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.nb) return;
    const float rho = boundary_density<false>(P, A, (unsigned)q);
    const float p = tait_pressure(rho, P, P.kr_g);
    A.bdens[q] = rho;
    A.bpress[q] = p;
    A.bdp[q] = __fdiv_rn(p, __fmul_rn(rho, rho));
}

void launch_boundary_density(const SimParams& P, const DeviceArrays& A, cudaStream_t s)
{
    if (P.nb > 0) k_boundary_density<<<(P.nb + 255) / 256, 256, 0, s>>>(P, A);
}

/* PCISPHBoundaryObject::correctPositions (WCSPH / DFSPH branch, :264-300)
   at the updated positions, and for WCSPH correctVelocities (:338-358) with
   the new normals */
template <bool WCSPH>
__global__ void __launch_bounds__(256) k_pcib_correct(SimParams P, DeviceArrays A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active_n(P, A.st)) return;
    float4 x = A.pos[i];
    float wsum = 0.0f, w2sum = 0.0f;
    float3 avg = make_float3(0.0f, 0.0f, 0.0f);
    if (cell_listed(A.cell_entry, cell_index(x, P.h, grid_single(P)), A.st->ns_epoch))
        pcib_collide(P, A, x, x, wsum, w2sum, avg);
    float4 n;
    x = pcib_push(x, wsum, w2sum, avg, n);
    A.pos[i] = x;
    A.normal[i] = n;
    if (!isfinite(x.x) || !isfinite(x.y) || !isfinite(x.z)) atomicOr(&A.st->err, ERRBIT_NAN);
    if (WCSPH) {
        float4 v = A.vel[i];
        pcib_velocity(P, n, v, v);
        A.vel[i] = v;
    }
}

void launch_pcib_correct(const SimParams& P, const DeviceArrays& A, bool wcsph, cudaStream_t s)
{
    const int grid = (P.nf + 255) / 256;
    if (grid == 0) return;
    if (wcsph) k_pcib_correct<true><<<grid, 256, 0, s>>>(P, A);
    else k_pcib_correct<false><<<grid, 256, 0, s>>>(P, A);
}

/* ---------------------------------------------------------------------- */
/* CubeBoundaryObject::correctPositionAndVelocity (CubeBoundaryObject.cpp:10-88):
   per axis in x, y, z order, a particle below min (above max) is put on the
   face; an outward velocity component is scaled by -normal_fct and the
   other two by tangential_fct; cubes in order.                             */

__device__ __forceinline__ void cube_axis(float& p, float& v, float& t1, float& t2, float lo, float hi, float nf,
                                          float tf)
{
    if (p < lo) {
        p = lo;
        if (v < 0.0f) v = __fmul_rn(v, -nf);
        t1 = __fmul_rn(t1, tf);
        t2 = __fmul_rn(t2, tf);
    } else if (p > hi) {
        p = hi;
        if (v > 0.0f) v = __fmul_rn(v, -nf);
        t1 = __fmul_rn(t1, tf);
        t2 = __fmul_rn(t2, tf);
    }
}

__global__ void __launch_bounds__(256) k_cube_correct(SimParams P, DeviceArrays A, const CubeBox* cubes, int ncubes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active_n(P, A.st)) return;
    const float4 x0 = A.pos[i];
    float4 x = x0, v = A.vel[i];
    for (int c = 0; c < ncubes; ++c) {
        const CubeBox b = cubes[c];
        cube_axis(x.x, v.x, v.y, v.z, b.minx, b.maxx, b.normal_fct, b.tangential_fct);
        cube_axis(x.y, v.y, v.x, v.z, b.miny, b.maxy, b.normal_fct, b.tangential_fct);
        cube_axis(x.z, v.z, v.x, v.y, b.minz, b.maxz, b.normal_fct, b.tangential_fct);
    }
    A.pos[i] = x;
    A.vel[i] = v;
    if (P.pos_lo && (x.x != x0.x || x.y != x0.y || x.z != x0.z)) {
        /* a clamped coordinate sits exactly on the face */
        float4 lo = A.plo[i];
        if (x.x != x0.x) lo.x = 0.0f;
        if (x.y != x0.y) lo.y = 0.0f;
        if (x.z != x0.z) lo.z = 0.0f;
        A.plo[i] = lo;
    }
}

void launch_cube_correct(const SimParams& P, const DeviceArrays& A, const CubeBox* cubes, int ncubes, cudaStream_t s)
{
    if (P.nf <= 0 || ncubes <= 0) return;
    k_cube_correct<<<(P.nf + 255) / 256, 256, 0, s>>>(P, A, cubes, ncubes);
}

/* ---------------------------------------------------------------------- */
/* Emitters (Emitter::emitParticles / emitGroup, Emitter.cpp:82-128).       */

/* glm's quat * vec3 (type_quat.inl:347-354) in FP32, operation for
   operation: uv = cross(q.xyz, v), uuv = cross(q.xyz, uv),
   v + ((uv * w) + uuv) * 2, cross as in func_geometric.inl:74-77. */
__device__ __forceinline__ void quat_rotate(const EmitterState& e, float vx, float vy, float vz, float& ox, float& oy,
                                            float& oz)
{
    const float uvx = __fsub_rn(__fmul_rn(e.qy, vz), __fmul_rn(vy, e.qz));
    const float uvy = __fsub_rn(__fmul_rn(e.qz, vx), __fmul_rn(vz, e.qx));
    const float uvz = __fsub_rn(__fmul_rn(e.qx, vy), __fmul_rn(vx, e.qy));
    const float uuvx = __fsub_rn(__fmul_rn(e.qy, uvz), __fmul_rn(uvy, e.qz));
    const float uuvy = __fsub_rn(__fmul_rn(e.qz, uvx), __fmul_rn(uvz, e.qx));
    const float uuvz = __fsub_rn(__fmul_rn(e.qx, uvy), __fmul_rn(uvx, e.qy));
    ox = __fadd_rn(vx, __fmul_rn(__fadd_rn(__fmul_rn(uvx, e.qw), uuvx), 2.0f));
    oy = __fadd_rn(vy, __fmul_rn(__fadd_rn(__fmul_rn(uvy, e.qw), uuvy), 2.0f));
    oz = __fadd_rn(vz, __fmul_rn(__fadd_rn(__fmul_rn(uvz, e.qw), uuvz), 2.0f));
}

/* One block. Emitters in order: one whose next emission time has come
   (time >= next, the start-of-step time) and that still holds a whole group
   appends the group after the active particles (slots and caller ids
   n_active, n_active + 1, ...) with velocity rot (0, 0, v) at
   rot (g + t (v_z + gravity t)) + r, t = time - next, then its next time
   moves on by its period. With `advance` (WCSPH, PCISPH, whose step ends
   with the emission) the time then moves on by dt. */
__global__ void __launch_bounds__(256) k_emit(SimParams P, DeviceArrays A, EmitterState* E, const float4* group,
                                              int nemit, int advance)
{
    __shared__ unsigned s_n;
    __shared__ int s_go;
    __shared__ float s_off;
    DevState* st = A.st;
    const float time = (float)st->time;
    if (threadIdx.x == 0) s_n = st->n_active;
    __syncthreads();
    for (int e = 0; e < nemit; ++e) {
        if (threadIdx.x == 0) {
            const EmitterState& em = E[e];
            s_go = time >= em.next && em.group_count <= em.remaining && s_n + em.group_count <= (unsigned)P.nf;
            s_off = __fsub_rn(time, em.next);
        }
        __syncthreads();
        if (s_go) {
            const EmitterState em = E[e];
            const float t = s_off;
            /* velocity + gravity * t, with velocity = (0, 0, v) */
            const float wx = __fadd_rn(0.0f, __fmul_rn(P.gx, t));
            const float wy = __fadd_rn(0.0f, __fmul_rn(P.gy, t));
            const float wz = __fadd_rn(em.v, __fmul_rn(P.gz, t));
            float rvx, rvy, rvz;
            quat_rotate(em, 0.0f, 0.0f, em.v, rvx, rvy, rvz);
            for (unsigned k = threadIdx.x; k < em.group_count; k += blockDim.x) {
                const float4 g = group[em.group_begin + k];
                const float px = __fadd_rn(g.x, __fmul_rn(t, wx));
                const float py = __fadd_rn(g.y, __fmul_rn(t, wy));
                const float pz = __fadd_rn(g.z, __fmul_rn(t, wz));
                float rx, ry, rz;
                quat_rotate(em, px, py, pz, rx, ry, rz);
                const unsigned slot = s_n + k;
                A.pos[slot] = make_float4(__fadd_rn(rx, em.px), __fadd_rn(ry, em.py), __fadd_rn(rz, em.pz), 0.0f);
                if (P.pos_lo) A.plo[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                A.vel[slot] = make_float4(rvx, rvy, rvz, 0.0f);
                A.acc[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                A.orig_w[slot] = slot;
                if (A.kws) A.kws[slot] = 0.0f;
                if (A.kvws) A.kvws[slot] = 0.0f;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_go) {
            s_n += E[e].group_count;
            E[e].remaining -= E[e].group_count;
            E[e].next = __fadd_rn(E[e].next, E[e].period);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        st->n_active = s_n;
        if (advance) {
            st->time = advance_time(st->time, st->dt);
            st->steps += 1u;
        }
    }
}

void launch_emit(const SimParams& P, const DeviceArrays& A, EmitterState* E, const float4* group, int nemit,
                 bool advance, cudaStream_t s)
{
    k_emit<<<1, 256, 0, s>>>(P, A, E, group, nemit, advance ? 1 : 0);
}

/* Test kernel: block 1 never arrives, so block 0's wait must run out. */
__global__ void k_barrier_timeout_probe(DevState* st)
{
    if (blockIdx.x == 1) return;
    grid_barrier(st);
}

int launch_barrier_timeout_probe(DevState* st, cudaStream_t s)
{
    void* args[] = {&st};
    return (int)cudaLaunchCooperativeKernel((const void*)k_barrier_timeout_probe, dim3(2), dim3(32), args, 0, s);
}

/* ---------------------------------------------------------------------- */

static inline int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

/* Lanes per particle for the WCSPH density and force passes: 4 below 2^16
   particles, where one lane per particle leaves most of the GPU idle and its
   serial neighbour walk is the critical path (32k particles: forces 42.8 ->
   18.4 us, density 25 -> 14 us); one lane above. */
static int small_scene_lanes(int n)
{
    return n < (1 << 16) ? 4 : 1;
}

void launch_density(const SimParams& P, const DeviceArrays& A, bool alpha, bool eos, int block, cudaStream_t s)
{
    if (P.nf <= 0) return;
    const int g = blocks_for(P.nf, block);
    if (alpha && eos) k_density<true, true><<<g, block, 0, s>>>(P, A);
    else if (alpha && A.divres) k_density<true, false, true><<<g, block, 0, s>>>(P, A);
    else if (alpha) k_density<true, false><<<g, block, 0, s>>>(P, A);
    else if (small_scene_lanes(P.nf) > 1) {
        const int gl = blocks_for((long long)P.nf * 4, block);
        if (eos) k_density_lanes<true, 4><<<gl, block, 0, s>>>(P, A);
        else k_density_lanes<false, 4><<<gl, block, 0, s>>>(P, A);
    }
    else if (eos) k_density<false, true><<<g, block, 0, s>>>(P, A);
    else k_density<false, false><<<g, block, 0, s>>>(P, A);
}

void launch_normals(const SimParams& P, const DeviceArrays& A, int block, cudaStream_t s)
{
    if (P.nf <= 0) return;
    k_normals<<<blocks_for(P.nf, block), block, 0, s>>>(P, A);
}

void launch_forces(const SimParams& P, const DeviceArrays& A, int mode, int block, cudaStream_t s)
{
    const int g = P.nf > 0 ? blocks_for(P.nf, block) : 1;
    switch (mode) {
    case FORCE_NP: k_forces<FORCE_NP><<<g, block, 0, s>>>(P, A); break;
    case FORCE_NP_CFL: k_forces<FORCE_NP_CFL><<<g, block, 0, s>>>(P, A); break;
    case FORCE_WCSPH: {
        const int tpp = small_scene_lanes(P.nf);
        const int gw = P.nf > 0 ? blocks_for((long long)P.nf * tpp, block) : 1;
        if (tpp == 1) k_forces<FORCE_WCSPH, 1><<<gw, block, 0, s>>>(P, A);
        else k_forces<FORCE_WCSPH, 4><<<gw, block, 0, s>>>(P, A);
        break;
    }
    default: k_forces<FORCE_PRESSURE><<<g, block, 0, s>>>(P, A); break;
    }
}

/* k_dfsph_solve instance for (divergence, blocks per SM, lanes per particle) */
static const void* dfsph_solve_fn(bool divergence, int occ, int tpp)
{
#define SPH_SOLVE_FN(D, O)                                                                          \
    (tpp == 4 ? (const void*)k_dfsph_solve<D, O, 4>                                                 \
              : tpp == 2 ? (const void*)k_dfsph_solve<D, O, 2> : (const void*)k_dfsph_solve<D, O, 1>)
    if (divergence) return occ == 4 ? SPH_SOLVE_FN(true, 4) : SPH_SOLVE_FN(true, 8);
    return occ == 4 ? SPH_SOLVE_FN(false, 4) : SPH_SOLVE_FN(false, 8);
#undef SPH_SOLVE_FN
}

int persistent_grid(bool pcisph, bool divergence, bool batch, int occ, int tpp)
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    const void* fn = pcisph ? (const void*)k_pcisph_solve
                     : batch ? (divergence ? (const void*)k_dfsph_solve_batch<true>
                                           : (const void*)k_dfsph_solve_batch<false>)
                             : dfsph_solve_fn(divergence, occ, tpp);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSolverBlock, 0) != cudaSuccess) return 0;
    return per_sm * sms;
}

static int coop_launch(const void* fn, const SimParams& P, const DeviceArrays& A, int grid, cudaStream_t s)
{
    SimParams p = P;
    DeviceArrays a = A;
    void* args[] = {&p, &a};
    return (int)cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kSolverBlock), args, 0, s);
}

int launch_dfsph_solve(const SimParams& P, const DeviceArrays& A, bool divergence, int grid, int occ, int tpp,
                       cudaStream_t s)
{
    const int need = blocks_for((long long)(P.nf > 0 ? P.nf : 1) * tpp, kSolverBlock);
    const int g = grid < need ? grid : need;
    return coop_launch(dfsph_solve_fn(divergence, occ, tpp), P, A, g > 0 ? g : 1, s);
}

int launch_dfsph_solve_batch(const SimParams& P, const DeviceArrays& A, bool divergence, int grid, cudaStream_t s)
{
    const int need = blocks_for(P.nf > 0 ? P.nf : 1, kSolverBlock);
    const int g = grid < need ? grid : need;
    return coop_launch(divergence ? (const void*)k_dfsph_solve_batch<true> : (const void*)k_dfsph_solve_batch<false>,
                       P, A, g > 0 ? g : 1, s);
}

int launch_pcisph_solve(const SimParams& P, const DeviceArrays& A, int grid, cudaStream_t s)
{
    const int need = blocks_for(P.nf > 0 ? P.nf : 1, kSolverBlock);
    const int g = grid < need ? grid : need;
    return coop_launch((const void*)k_pcisph_solve, P, A, g > 0 ? g : 1, s);
}

} // namespace sph
