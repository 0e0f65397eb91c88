/*
 * Reverse-mode adjoint of the WCSPH step (sm_100a). SPH2O has no
 * differentiable path; this differentiates the step that k_forces<FORCE_WCSPH>
 * takes (WCSPHSolver::step, WCSPHSolver.cpp:14-78), with the neighbour lists
 * of each step held fixed:
 *
 *   rho_i = sum_j m W(x_i - x_j) + sum_b psi_b W(x_i - x_b)        (SPHSolver.cpp:42-89)
 *   p_i   = max(0, (k rho0 / gamma) ((rho_i / rho0)^gamma - 1))   (WCSPHSolver.cpp:80-95)
 *   a_i   = - sum_j m (A_i + A_j) gradW_ij - sum_b psi_b (A_i + B_i) gradW_ib
 *           + nu sum_j (m / rho_j) phi_ij gradW_ij
 *           + nu_b sum_b (psi_b / rho_i) phi_ib gradW_ib + g        (WCSPHSolver.cpp:132-188,
 *                                                                    ArtificialViscosity.cpp:6-54)
 *   v' = v + a dt,  x' = x + v' dt                                   (SPHSolver.cpp:139-168)
 *
 * with A = p / rho^2, B = p / rho0^2, phi_ij = (v_ij . r_ij) / (|r_ij|^2 + 0.01 h^2),
 * gradW(r) = f(|r|) r and Hessian H(r) = f I + g r r^T, g = f'(|r|) / |r|.
 *
 * Every sum is a gather: because the neighbour relation is symmetric and
 * gradW antisymmetric, the adjoint of a pair term can be formed from either
 * side, so each particle accumulates its own adjoint from its own list and
 * no atomics are needed. The loss and the two parameter gradients are
 * reduced in FP64 (warp shuffles, then a block sum) into one slot per block
 * that the block adds to across steps, and k_adj_finish sums the slots in a
 * fixed order: results are bit-reproducible run to run.
 *
 * One backward step, in the cell-sorted order of the recomputed step:
 *   k_adj_load     x~ = xbar', v~ = vbar' + dt xbar', abar = dt v~, A = p / rho^2
 *   k_adj_forces   pressure / viscosity adjoint: rhobar, x~ += dF/dx, v~ += dF/dv,
 *                  dL/dk and dL/dnu partial sums
 *   k_adj_density  x~ += sum_j m (rhobar_i + rhobar_j) gradW_ij + boundary,
 *                  scattered to caller order
 * The adjoint state xbar, vbar is kept in caller particle order between steps,
 * since every forward step re-sorts the particles.
 */
#include "sph_device.cuh"
#include "sph_internal.h"

namespace sph {

/* gradW(r) = f r and g = f'(|r|) / |r| for 0 < |r| <= h (CubicSpline.h:52-74):
   q <= 1/2: f = (l / h^2)(3q - 2),        g = 3 l / (h^3 |r|)
   q >  1/2: f = -(l / h)(1 - q)^2 / |r|,  g = (l / h)(1 - q)(1 + q) / |r|^3   */
__device__ __forceinline__ void cs_grad_fg(float rl, float inv_rl, const SimParams& P, float& f, float& g)
{
    const float q = rl * P.inv_h;
    if (!(rl > 1.0e-9f) || q > 1.0f) {
        f = 0.0f;
        g = 0.0f;
        return;
    }
    if (q <= 0.5f) {
        f = P.cs_l_h2 * (3.0f * q - 2.0f);
        g = 3.0f * P.cs_l_h2 * P.inv_h * inv_rl;
    } else {
        const float t = 1.0f - q;
        f = -P.cs_l_h * (t * t) * inv_rl;
        g = P.cs_l_h * t * (1.0f + q) * (inv_rl * inv_rl * inv_rl);
    }
}

__device__ __forceinline__ void pair_of(float4 a, float4 b, float& rx, float& ry, float& rz, float& s, float& rl,
                                        float& inv_rl)
{
    rx = a.x - b.x;
    ry = a.y - b.y;
    rz = a.z - b.z;
    s = (rx * rx + ry * ry) + rz * rz;
    len_inv(s, rl, inv_rl);
}

/* Sum over the TPP adjacent lanes of a group (gmask: the group's lanes). */
template <int TPP>
__device__ __forceinline__ float group_sum(float v, unsigned gmask)
{
    for (int o = TPP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
    return v;
}

template <int TPP>
__device__ __forceinline__ unsigned group_mask()
{
    const unsigned lane = threadIdx.x & 31u;
    return TPP == 32 ? 0xffffffffu : ((1u << TPP) - 1u) << (lane - lane % TPP);
}

/* Loss L = (1/N) sum_i |x_i - t_i|^2 of the current (sorted) positions
   against the caller-order target; seeds xbar = 2 (x - t) / N, vbar = 0. */
__global__ void __launch_bounds__(256) k_adj_seed(int n, const float4* __restrict__ pos,
                                                  const unsigned* __restrict__ orig,
                                                  const float* __restrict__ target, float4* __restrict__ xbar,
                                                  float4* __restrict__ vbar, double* __restrict__ part)
{
    __shared__ double s_red[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < n) {
        const unsigned o = orig[i];
        const float4 x = pos[i];
        const float dx = x.x - target[3 * (size_t)o], dy = x.y - target[3 * (size_t)o + 1],
                    dz = x.z - target[3 * (size_t)o + 2];
        l = ((double)dx * dx + (double)dy * dy) + (double)dz * dz;
        const float c = 2.0f / (float)n;
        xbar[o] = make_float4(c * dx, c * dy, c * dz, 0.0f);
        vbar[o] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    const double t = block_sum(l, s_red);
    if (threadIdx.x == 0) part[3 * blockIdx.x + 2] = t;
}

/* Adjoint of the symplectic Euler update, gathered into sorted order. */
__global__ void __launch_bounds__(256) k_adj_load(SimParams P, AdjointArrays J)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.nf) return;
    const float dt = J.st->dt;
    const unsigned o = J.orig[i];
    const float4 xb = J.xbar[o], vb = J.vbar[o];
    const float vx = vb.x + dt * xb.x, vy = vb.y + dt * xb.y, vz = vb.z + dt * xb.z;
    J.abar[i] = make_float4(dt * vx, dt * vy, dt * vz, 0.0f);
    J.xacc[i] = make_float4(xb.x, xb.y, xb.z, 0.0f);
    J.vacc[i] = make_float4(vx, vy, vz, 0.0f);
    const float r = J.rho[i];
    J.Ap[i] = J.press[i] / (r * r);
}

/* Adjoint of the pressure and viscosity accelerations (and of the EOS).
   TPP adjacent lanes share particle i, each summing the list entries
   sub, sub + TPP, ...; the group's partial sums are then added by shuffles
   in a fixed order, so results are reproducible run to run. */
template <int TPP>
__global__ void __launch_bounds__(256, 4) k_adj_forces(SimParams P, AdjointArrays J)
{
    __shared__ double s_red[32];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / TPP;
    const unsigned sub = (unsigned)t % TPP;
    const size_t nf = (size_t)P.nf;
    double kbar = 0.0, nubar = 0.0;
    float sA = 0.0f, sB = 0.0f, rv = 0.0f, sbv = 0.0f, nup = 0.0f;
    float xrx = 0.0f, xry = 0.0f, xrz = 0.0f, vrx = 0.0f, vry = 0.0f, vrz = 0.0f;
    if (i < P.nf) {
        const float4 xi = J.pos[i];
        const float4 vi = J.vel[i];
        const float4 ai = J.abar[i];
        const float rho_i = J.rho[i], p_i = J.press[i];
        const float Ai = J.Ap[i];
        const float Bi = p_i / (P.rho0 * P.rho0);
        const float m = P.mass;
        const bool visc = P.visc_method == 1;
        const bool bvisc = visc && P.bvisc != 0.0f;
        const float nu = P.visc, nub = P.bvisc;
        const float eps_h2 = 0.01f * P.h2;
        const float inv_rho_i = 1.0f / rho_i;
        const unsigned nF = J.cnt_f[i];
        for (unsigned kk = sub; kk < nF; kk += TPP) {
            const unsigned j = list_at(J.nbr_f, kk, nf, i);
            const float4 xj = J.pos[j];
            float rx, ry, rz, s, rl, inv_rl, f, g;
            pair_of(xi, xj, rx, ry, rz, s, rl, inv_rl);
            cs_grad_fg(rl, inv_rl, P, f, g);
            if (f == 0.0f && g == 0.0f) continue;
            const float4 aj = J.abar[j];
            const float Aj = J.Ap[j];
            const float dax = ai.x - aj.x, day = ai.y - aj.y, daz = ai.z - aj.z;
            const float rda = (rx * dax + ry * day) + rz * daz;
            sA -= m * f * rda;
            /* x~_i += -m (A_i + A_j) H (abar_i - abar_j) */
            const float c1 = -m * (Ai + Aj);
            const float gr = g * rda;
            xrx += c1 * (f * dax + gr * rx);
            xry += c1 * (f * day + gr * ry);
            xrz += c1 * (f * daz + gr * rz);
            if (visc) {
                const float4 vj = J.vel[j];
                const float rho_j = J.rho[j];
                const float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
                const float vr = (vx * rx + vy * ry) + vz * rz;
                const float invD = 1.0f / (s + eps_h2);
                const float phi = vr * invD;
                /* c = nu m (abar_i / rho_j - abar_j / rho_i) */
                const float inv_rho_j = 1.0f / rho_j;
                const float cx = nu * m * (ai.x * inv_rho_j - aj.x * inv_rho_i);
                const float cy = nu * m * (ai.y * inv_rho_j - aj.y * inv_rho_i);
                const float cz = nu * m * (ai.z * inv_rho_j - aj.z * inv_rho_i);
                const float cr = (cx * rx + cy * ry) + cz * rz;
                const float tv = f * cr * invD;
                vrx += tv * rx; vry += tv * ry; vrz += tv * rz;
                const float t1 = f * invD;
                const float t2 = vr * cr * (g * invD - 2.0f * f * invD * invD);
                xrx += t1 * (cr * vx + vr * cx) + t2 * rx;
                xry += t1 * (cr * vy + vr * cy) + t2 * ry;
                xrz += t1 * (cr * vz + vr * cz) + t2 * rz;
                rv += phi * f * ((aj.x * rx + aj.y * ry) + aj.z * rz);
                nup += m * inv_rho_j * phi * f * ((ai.x * rx + ai.y * ry) + ai.z * rz);
            }
        }
        const unsigned nB = J.cnt_b[i];
        for (unsigned kk = sub; kk < nB; kk += TPP) {
            const float4 xb = J.bpos[list_at(J.nbr_b, kk, nf, i)];
            float rx, ry, rz, s, rl, inv_rl, f, g;
            pair_of(xi, xb, rx, ry, rz, s, rl, inv_rl);
            cs_grad_fg(rl, inv_rl, P, f, g);
            if (f == 0.0f && g == 0.0f) continue;
            const float psi = xb.w;
            const float rai = (rx * ai.x + ry * ai.y) + rz * ai.z;
            const float t = psi * f * rai;
            sA -= t;
            sB -= t;
            const float c1 = -psi * (Ai + Bi);
            const float gr = g * rai;
            xrx += c1 * (f * ai.x + gr * rx);
            xry += c1 * (f * ai.y + gr * ry);
            xrz += c1 * (f * ai.z + gr * rz);
            if (bvisc) {
                const float vr = (vi.x * rx + vi.y * ry) + vi.z * rz;
                const float invD = 1.0f / (s + eps_h2);
                const float phi = vr * invD;
                const float cb = nub * psi * inv_rho_i;
                const float cx = cb * ai.x, cy = cb * ai.y, cz = cb * ai.z;
                const float cr = cb * rai;
                const float tv = f * cr * invD;
                vrx += tv * rx; vry += tv * ry; vrz += tv * rz;
                const float t1 = f * invD;
                const float t2 = vr * cr * (g * invD - 2.0f * f * invD * invD);
                xrx += t1 * (cr * vi.x + vr * cx) + t2 * rx;
                xry += t1 * (cr * vi.y + vr * cy) + t2 * ry;
                xrz += t1 * (cr * vi.z + vr * cz) + t2 * rz;
                sbv += psi * phi * f * rai;
            }
        }
        if (TPP > 1) {
            const unsigned gm = group_mask<TPP>();
            sA = group_sum<TPP>(sA, gm); sB = group_sum<TPP>(sB, gm);
            rv = group_sum<TPP>(rv, gm); sbv = group_sum<TPP>(sbv, gm); nup = group_sum<TPP>(nup, gm);
            xrx = group_sum<TPP>(xrx, gm); xry = group_sum<TPP>(xry, gm); xrz = group_sum<TPP>(xrz, gm);
            vrx = group_sum<TPP>(vrx, gm); vry = group_sum<TPP>(vry, gm); vrz = group_sum<TPP>(vrz, gm);
        }
    }
    if (i < P.nf && sub == 0) {
        const float rho_i = J.rho[i], p_i = J.press[i];
        const float inv_rho_i = 1.0f / rho_i;
        const float m = P.mass;
        const bool visc = P.visc_method == 1;
        const float nu = P.visc, nub = P.bvisc;
        /* EOS: p = max(0, kr_g (ratio^gamma - 1)), kr_g = k rho0 / gamma */
        const float pbar = sA * inv_rho_i * inv_rho_i + sB / (P.rho0 * P.rho0);
        float dpdrho = 0.0f;
        if (p_i > 0.0f) {
            const double ratio = (double)rho_i / (double)P.rho0;
            const double pw1 = pow(ratio, (double)P.gamma - 1.0);
            dpdrho = (float)((double)P.kr_g * (double)P.gamma * pw1 / (double)P.rho0);
            kbar = (double)pbar * ((double)P.rho0 / (double)P.gamma) * (pw1 * ratio - 1.0);
        }
        const float rhobar = -2.0f * p_i * sA * inv_rho_i * inv_rho_i * inv_rho_i +
                             nu * m * rv * inv_rho_i * inv_rho_i - nub * sbv * inv_rho_i * inv_rho_i +
                             pbar * dpdrho;
        J.rhobar[i] = rhobar;
        float4 xa = J.xacc[i], va = J.vacc[i];
        xa.x += xrx; xa.y += xry; xa.z += xrz;
        va.x += vrx; va.y += vry; va.z += vrz;
        J.xacc[i] = xa;
        J.vacc[i] = va;
        nubar = visc ? (double)nup : 0.0;
    }
    const double tk = block_sum(kbar, s_red);
    const double tn = block_sum(nubar, s_red);
    if (threadIdx.x == 0) {
        J.part[3 * blockIdx.x] += tk;
        J.part[3 * blockIdx.x + 1] += tn;
    }
}

/* red[q] = sum over blocks of part[3 b + q], in a fixed order. */
__global__ void __launch_bounds__(256) k_adj_finish(int nblocks, const double* __restrict__ part,
                                                    double* __restrict__ red)
{
    __shared__ double s_red[32];
    for (int q = 0; q < 3; ++q) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += part[3 * b + q];
        const double t = block_sum(v, s_red);
        if (threadIdx.x == 0) red[q] = t;
    }
}

/* Adjoint of the density sum; writes the step's input adjoint in caller order. */
template <int TPP>
__global__ void __launch_bounds__(256, 6) k_adj_density(SimParams P, AdjointArrays J)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / TPP;
    const unsigned sub = (unsigned)t % TPP;
    /* a group's lanes share i, so a group leaves together */
    if (i >= P.nf) return;
    const size_t nf = (size_t)P.nf;
    const float4 xi = J.pos[i];
    const float rbi = J.rhobar[i];
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    const unsigned nF = J.cnt_f[i];
    for (unsigned kk = sub; kk < nF; kk += TPP) {
        const unsigned j = list_at(J.nbr_f, kk, nf, i);
        float rx, ry, rz, s, rl, inv_rl;
        pair_of(xi, J.pos[j], rx, ry, rz, s, rl, inv_rl);
        const float f = cs_gradf(rl, inv_rl, P);
        if (f == 0.0f) continue;
        const float c = P.mass * (rbi + J.rhobar[j]) * f;
        sx += c * rx; sy += c * ry; sz += c * rz;
    }
    const unsigned nB = J.cnt_b[i];
    for (unsigned kk = sub; kk < nB; kk += TPP) {
        const float4 xb = J.bpos[list_at(J.nbr_b, kk, nf, i)];
        float rx, ry, rz, s, rl, inv_rl;
        pair_of(xi, xb, rx, ry, rz, s, rl, inv_rl);
        const float c = xb.w * rbi * cs_gradf(rl, inv_rl, P);
        sx += c * rx; sy += c * ry; sz += c * rz;
    }
    if (TPP > 1) {
        const unsigned gm = group_mask<TPP>();
        sx = group_sum<TPP>(sx, gm); sy = group_sum<TPP>(sy, gm); sz = group_sum<TPP>(sz, gm);
        if (sub != 0) return;
    }
    const unsigned o = J.orig[i];
    const float4 xa = J.xacc[i];
    J.xbar[o] = make_float4(xa.x + sx, xa.y + sy, xa.z + sz, 0.0f);
    J.vbar[o] = J.vacc[i];
}

__global__ void k_adj_unpack(int n, const float4* __restrict__ in, float* __restrict__ out3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = in[i];
    out3[3 * (size_t)i] = v.x;
    out3[3 * (size_t)i + 1] = v.y;
    out3[3 * (size_t)i + 2] = v.z;
}

static inline int blocks_for(int n, int b) { return (n + b - 1) / b; }

/* lanes per particle of the adjoint passes: 4 below 2^16 particles, where
   one lane per particle leaves most of the GPU idle; one above */
static inline int adjoint_tpp(int n) { return n < (1 << 16) ? 4 : 1; }

int adjoint_blocks(int n) { return blocks_for(n * adjoint_tpp(n), 256); }

void launch_adjoint_seed(int n, const float4* pos, const unsigned* orig, const float* target, float4* xbar,
                         float4* vbar, double* part, cudaStream_t s)
{
    if (n <= 0) return;
    k_adj_seed<<<blocks_for(n, 256), 256, 0, s>>>(n, pos, orig, target, xbar, vbar, part);
}

void launch_adjoint_finish(int n, const double* part, double* red, cudaStream_t s)
{
    k_adj_finish<<<1, 256, 0, s>>>(adjoint_blocks(n), part, red);
}

void launch_adjoint_step(const SimParams& P, const AdjointArrays& J, cudaStream_t s)
{
    if (P.nf <= 0) return;
    k_adj_load<<<blocks_for(P.nf, 256), 256, 0, s>>>(P, J);
    const int g = adjoint_blocks(P.nf);
    if (adjoint_tpp(P.nf) == 1) {
        k_adj_forces<1><<<g, 256, 0, s>>>(P, J);
        k_adj_density<1><<<g, 256, 0, s>>>(P, J);
    } else {
        k_adj_forces<4><<<g, 256, 0, s>>>(P, J);
        k_adj_density<4><<<g, 256, 0, s>>>(P, J);
    }
}

void launch_adjoint_unpack(int n, const float4* in, float* out3, cudaStream_t s)
{
    if (n <= 0) return;
    k_adj_unpack<<<blocks_for(n, 256), 256, 0, s>>>(n, in, out3);
}

} // namespace sph
