/*
 * FP64 WCSPH forward run and its reverse-mode adjoint on the CPU -- TEST
 * INFRASTRUCTURE (the checker of the GPU adjoint, sph_wcsph_forward /
 * sph_wcsph_backward). Only tests/ load it.
 *
 * Forward step (SPH2O's WCSPHSolver::step, WCSPHSolver.cpp:14-78, in double):
 *   neighbour lists N(i) = { j : |x_i - x_j| <= h } (self included) and
 *   boundary lists, from a uniform grid of cell size h
 *     (HashTable.cpp:23-86 gathers the same sets from its 27 cells);
 *   rho_i = sum_j m W_ij + sum_b psi_b W_ib                 SPHSolver.cpp:42-89
 *   p_i = max(0, k rho0 / gamma ((rho_i / rho0)^gamma - 1)) WCSPHSolver.cpp:80-95
 *   a_i = -sum_j m (p_i / rho_i^2 + p_j / rho_j^2) gradW_ij
 *         -sum_b psi_b (p_i / rho_i^2 + p_i / rho0^2) gradW_ib WCSPHSolver.cpp:132-188
 *         +nu sum_j (m / rho_j) (v_ij . r_ij) / (|r_ij|^2 + 0.01 h^2) gradW_ij
 *         +nu_b sum_b (psi_b / rho_i) (v_i . r_ib) / (|r_ib|^2 + 0.01 h^2) gradW_ib
 *                                                         ArtificialViscosity.cpp:6-54
 *   v += (a + g) dt; x += v dt                            SPHSolver.cpp:139-168
 * with psi_b = rho0 V_b, V_b = 1 / sum_b' W_bb' (AkinciBoundaryObject.cpp:10-34)
 * and the cubic spline of CubicSpline.h:27-74.
 *
 * Loss L = (1/N) sum_i |x_i(T) - t_i|^2. The adjoint is the exact derivative
 * of this forward map with each step's neighbour lists fixed (the
 * contributions of pairs at the support edge vanish smoothly, so this is the
 * derivative central differences converge to). It is written per directed
 * pair in scatter form -- a different arrangement from the GPU's gather
 * form, so the two check each other.
 */
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../include/sph2o_cuda.h"

namespace {

struct V {
    double x = 0, y = 0, z = 0;
    V() = default;
    V(double a, double b, double c) : x(a), y(b), z(c) {}
    V operator+(const V& o) const { return {x + o.x, y + o.y, z + o.z}; }
    V operator-(const V& o) const { return {x - o.x, y - o.y, z - o.z}; }
    V operator*(double s) const { return {x * s, y * s, z * s}; }
    V& operator+=(const V& o) { x += o.x; y += o.y; z += o.z; return *this; }
    V& operator-=(const V& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
};
inline double dot(const V& a, const V& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct Kernel {
    double h, ck, cl;
    double W(double rl) const
    {
        const double q = rl / h;
        if (q > 1.0) return 0.0;
        if (q <= 0.5) return ck * (6.0 * q * q * q - 6.0 * q * q + 1.0);
        const double t = 1.0 - q;
        return ck * 2.0 * t * t * t;
    }
    /* gradW(r) = f r, Hessian f I + g r r^T (g = f'(|r|) / |r|) */
    void fg(const V& r, double& f, double& g) const
    {
        const double rl = std::sqrt(dot(r, r));
        const double q = rl / h;
        f = g = 0.0;
        if (!(rl > 1.0e-9) || q > 1.0) return;
        if (q <= 0.5) {
            f = cl / (h * h) * (3.0 * q - 2.0);
            g = 3.0 * cl / (h * h * h * rl);
        } else {
            const double t = 1.0 - q;
            f = -cl / h * t * t / rl;
            g = cl / h * t * (1.0 + q) / (rl * rl * rl);
        }
    }
};

struct Lists {
    std::vector<uint32_t> fo, fi, bo, bi; /* CSR */
};

struct Grid {
    double h;
    std::unordered_map<uint64_t, std::vector<uint32_t>> cells;
    static uint64_t key(int64_t a, int64_t b, int64_t c)
    {
        return ((uint64_t)(a + (1 << 20)) << 42) | ((uint64_t)(b + (1 << 20)) << 21) | (uint64_t)(c + (1 << 20));
    }
    void build(const std::vector<V>& p)
    {
        cells.clear();
        for (size_t i = 0; i < p.size(); ++i)
            cells[key((int64_t)std::floor(p[i].x / h), (int64_t)std::floor(p[i].y / h), (int64_t)std::floor(p[i].z / h))]
                .push_back((uint32_t)i);
    }
    template <typename F> void around(const V& x, F f) const
    {
        const int64_t cx = (int64_t)std::floor(x.x / h), cy = (int64_t)std::floor(x.y / h), cz = (int64_t)std::floor(x.z / h);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    auto it = cells.find(key(cx + dx, cy + dy, cz + dz));
                    if (it != cells.end())
                        for (uint32_t j : it->second) f(j);
                }
    }
};

struct Problem {
    Kernel K;
    double h, h2, mass, rho0, nu, nub, stiff, gamma, kr_g, dt;
    V g;
    std::vector<V> bx;
    std::vector<double> psi;
    Grid bgrid;

    void lists(const std::vector<V>& x, Lists& L) const
    {
        const size_t n = x.size();
        Grid fg{h, {}};
        fg.build(x);
        /* per-particle sets in parallel (read-only grid lookups), then CSR */
        std::vector<std::vector<uint32_t>> F(n), B(n);
#pragma omp parallel for schedule(dynamic, 256)
        for (long i = 0; i < (long)n; ++i) {
            std::vector<uint32_t>& f = F[i];
            std::vector<uint32_t>& b = B[i];
            fg.around(x[i], [&](uint32_t j) { const V r = x[i] - x[j]; if (std::sqrt(dot(r, r)) <= h) f.push_back(j); });
            bgrid.around(x[i], [&](uint32_t k) { const V r = x[i] - bx[k]; if (std::sqrt(dot(r, r)) <= h) b.push_back(k); });
            std::sort(f.begin(), f.end());
            std::sort(b.begin(), b.end());
        }
        L.fo.assign(n + 1, 0);
        L.bo.assign(n + 1, 0);
        for (size_t i = 0; i < n; ++i) {
            L.fo[i + 1] = L.fo[i] + (uint32_t)F[i].size();
            L.bo[i + 1] = L.bo[i] + (uint32_t)B[i].size();
        }
        L.fi.resize(L.fo[n]);
        L.bi.resize(L.bo[n]);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; ++i) {
            std::copy(F[i].begin(), F[i].end(), L.fi.begin() + L.fo[i]);
            std::copy(B[i].begin(), B[i].end(), L.bi.begin() + L.bo[i]);
        }
    }

    void density(const std::vector<V>& x, const Lists& L, std::vector<double>& rho, std::vector<double>& p) const
    {
        const size_t n = x.size();
        rho.assign(n, 0.0);
        p.assign(n, 0.0);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; ++i) {
            double s = 0.0;
            for (uint32_t k = L.fo[i]; k < L.fo[i + 1]; ++k) {
                const V r = x[i] - x[L.fi[k]];
                s += mass * K.W(std::sqrt(dot(r, r)));
            }
            for (uint32_t k = L.bo[i]; k < L.bo[i + 1]; ++k) {
                const V r = x[i] - bx[L.bi[k]];
                s += psi[L.bi[k]] * K.W(std::sqrt(dot(r, r)));
            }
            rho[i] = s;
            p[i] = std::max(0.0, kr_g * (std::pow(s / rho0, gamma) - 1.0));
        }
    }

    void accel(const std::vector<V>& x, const std::vector<V>& v, const Lists& L, const std::vector<double>& rho,
               const std::vector<double>& p, std::vector<V>& a) const
    {
        const size_t n = x.size();
        a.assign(n, V());
        const double eh2 = 0.01 * h2;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; ++i) {
            V ai;
            const double Ai = p[i] / (rho[i] * rho[i]), Bi = p[i] / (rho0 * rho0);
            for (uint32_t k = L.fo[i]; k < L.fo[i + 1]; ++k) {
                const uint32_t j = L.fi[k];
                const V r = x[i] - x[j];
                double f, gg;
                K.fg(r, f, gg);
                const double Aj = p[j] / (rho[j] * rho[j]);
                ai -= r * (mass * (Ai + Aj) * f);
                ai += r * (nu * (mass / rho[j]) * dot(v[i] - v[j], r) / (dot(r, r) + eh2) * f);
            }
            for (uint32_t k = L.bo[i]; k < L.bo[i + 1]; ++k) {
                const uint32_t b = L.bi[k];
                const V r = x[i] - bx[b];
                double f, gg;
                K.fg(r, f, gg);
                ai -= r * (psi[b] * (Ai + Bi) * f);
                ai += r * (nub * (psi[b] / rho[i]) * dot(v[i], r) / (dot(r, r) + eh2) * f);
            }
            a[i] = ai + g;
        }
    }
};

inline V hess(double f, double g, const V& r, const V& u) { return u * f + r * (g * dot(r, u)); }

} // namespace

extern "C" {

/* FP64 run of nsteps WCSPH steps from (x0, v0) with viscosity nu and EOS
   stiffness k (overriding the description's, so that central differences
   can step them). Returns the loss; when dv0 is not NULL also the gradients
   dL/dx0, dL/dv0 (n*3 each, caller order), dL/dnu and dL/dk. x_out (may be
   NULL) receives x(T). With a gradient every step's state and lists are
   kept in host memory (about 100 B per particle and step); a loss-only run
   (dv0 NULL) keeps one step. Loops run on OpenMP threads. */
int sph_oracle_wcsph_adjoint(const sph_scene_desc* d, double nu, double k, unsigned nf, const double* x0,
                             const double* v0, unsigned nb, const double* bxyz, int nsteps, const double* target,
                             double* loss, double* x_out, double* dx0, double* dv0, double* dnu, double* dk)
{
    if (!d || !x0 || !v0 || !target || !loss || nsteps < 0) return SPH_ERR_ARG;
    Problem P;
    const double r = d->particle_radius;
    P.h = 4.0 * r;
    P.h2 = P.h * P.h;
    P.rho0 = d->density0;
    P.mass = P.rho0 * std::pow(2.0 * r, 3.0);
    P.K = Kernel{P.h, 8.0 / (M_PI * P.h * P.h * P.h), 48.0 / (M_PI * P.h * P.h * P.h)};
    const bool visc = d->viscosity_method == SPH_VISCOSITY_ARTIFICIAL;
    if (d->viscosity_method != -1 && !visc) return SPH_ERR_ARG;
    P.nu = visc ? nu : 0.0;
    P.nub = visc ? (double)d->boundary_viscosity : 0.0;
    P.stiff = k;
    P.gamma = d->gamma;
    P.kr_g = k * P.rho0 / P.gamma;
    P.dt = d->time_step;
    P.g = V(d->gravity[0], d->gravity[1], d->gravity[2]);
    P.bx.resize(nb);
    for (unsigned b = 0; b < nb; ++b) P.bx[b] = V(bxyz[3 * b], bxyz[3 * b + 1], bxyz[3 * b + 2]);
    P.bgrid.h = P.h;
    P.bgrid.build(P.bx);
    P.psi.assign(nb, 0.0);
    for (unsigned b = 0; b < nb; ++b) {
        double s = 0.0;
        P.bgrid.around(P.bx[b], [&](uint32_t c) { const V rr = P.bx[b] - P.bx[c]; s += P.K.W(std::sqrt(dot(rr, rr))); });
        P.psi[b] = P.rho0 / s;
    }

    const size_t n = nf;
    /* every step's state, lists, densities and pressures are kept when the
       gradient is wanted (the backward sweep reads them newest first);
       a loss-only run keeps one slot */
    const bool keep = dv0 != nullptr;
    const int slots = keep ? nsteps : 1;
    std::vector<std::vector<V>> xs(keep ? nsteps + 1 : 2), vs(keep ? nsteps + 1 : 2);
    std::vector<Lists> Ls(slots);
    std::vector<std::vector<double>> rhos(slots), ps(slots);
    xs[0].resize(n);
    vs[0].resize(n);
    for (size_t i = 0; i < n; ++i) {
        xs[0][i] = V(x0[3 * i], x0[3 * i + 1], x0[3 * i + 2]);
        vs[0][i] = V(v0[3 * i], v0[3 * i + 1], v0[3 * i + 2]);
    }
    std::vector<V> a;
    for (int s = 0; s < nsteps; ++s) {
        const int cur = keep ? s : 0, nxt = keep ? s + 1 : 1, slot = keep ? s : 0;
        P.lists(xs[cur], Ls[slot]);
        P.density(xs[cur], Ls[slot], rhos[slot], ps[slot]);
        P.accel(xs[cur], vs[cur], Ls[slot], rhos[slot], ps[slot], a);
        xs[nxt].resize(n);
        vs[nxt].resize(n);
        for (size_t i = 0; i < n; ++i) {
            vs[nxt][i] = vs[cur][i] + a[i] * P.dt;
            xs[nxt][i] = xs[cur][i] + vs[nxt][i] * P.dt;
        }
        if (!keep) {
            xs[0].swap(xs[1]);
            vs[0].swap(vs[1]);
        }
    }
    const std::vector<V>& xT = xs[keep ? nsteps : 0];
    double l = 0.0;
    std::vector<V> xb(n), vb(n);
    for (size_t i = 0; i < n; ++i) {
        const V dd = xT[i] - V(target[3 * i], target[3 * i + 1], target[3 * i + 2]);
        l += dot(dd, dd);
        xb[i] = dd * (2.0 / (double)n);
    }
    *loss = l / (double)n;
    if (x_out)
        for (size_t i = 0; i < n; ++i) {
            x_out[3 * i] = xT[i].x; x_out[3 * i + 1] = xT[i].y; x_out[3 * i + 2] = xT[i].z;
        }
    if (!dv0) return SPH_OK;

    double gnu = 0.0, gk = 0.0;
    const double eh2 = 0.01 * P.h2, m = P.mass, rho0 = P.rho0, dt = P.dt;
    /* The scatter writes to both particles of a pair; each OpenMP thread
       scatters into its own copy of the targets, summed after each sweep. */
    const int T = omp_get_max_threads();
    std::vector<std::vector<V>> txn(T, std::vector<V>(n)), tvn(T, std::vector<V>(n));
    std::vector<std::vector<double>> tA(T, std::vector<double>(n)), tR(T, std::vector<double>(n));
    std::vector<V> abar(n), xn(n), vn(n);
    std::vector<double> Abar(n), Bbar(n), rbar(n);
    auto clear = [&]() {
#pragma omp parallel for schedule(static)
        for (int t = 0; t < T; ++t) {
            std::fill(txn[t].begin(), txn[t].end(), V());
            std::fill(tvn[t].begin(), tvn[t].end(), V());
            std::fill(tA[t].begin(), tA[t].end(), 0.0);
            std::fill(tR[t].begin(), tR[t].end(), 0.0);
        }
    };
    for (int s = nsteps - 1; s >= 0; --s) {
        const std::vector<V>& x = xs[s];
        const std::vector<V>& v = vs[s];
        const Lists& L = Ls[s];
        const std::vector<double>& rho = rhos[s];
        const std::vector<double>& p = ps[s];
        /* x' = x + dt v', v' = v + dt a */
        for (size_t i = 0; i < n; ++i) {
            const V vt = vb[i] + xb[i] * dt;
            abar[i] = vt * dt;
            xn[i] = xb[i];
            vn[i] = vt;
        }
        std::fill(Bbar.begin(), Bbar.end(), 0.0);
        clear();
        /* scatter over directed pairs (i receives from j): a_i's terms */
#pragma omp parallel reduction(+ : gnu)
        {
            const int t = omp_get_thread_num();
            V* XN = txn[t].data();
            V* VN = tvn[t].data();
            double* AB = tA[t].data();
            double* RB = tR[t].data();
#pragma omp for schedule(dynamic, 256)
            for (long i = 0; i < (long)n; ++i) {
                const double Ai = p[i] / (rho[i] * rho[i]), Bi = p[i] / (rho0 * rho0);
                for (uint32_t kk = L.fo[i]; kk < L.fo[i + 1]; ++kk) {
                    const uint32_t j = L.fi[kk];
                    const V rr = x[i] - x[j];
                    double f, g;
                    P.K.fg(rr, f, g);
                    if (f == 0.0 && g == 0.0) continue;
                    const double Aj = p[j] / (rho[j] * rho[j]);
                    /* pressure: a_i -= m (A_i + A_j) f r */
                    const double tt = m * f * dot(abar[i], rr);
                    AB[i] -= tt;
                    AB[j] -= tt;
                    const V hv = hess(f, g, rr, abar[i]) * (-m * (Ai + Aj));
                    XN[i] += hv;
                    XN[j] -= hv;
                    if (P.nu != 0.0) {
                        /* a_i += nu (m / rho_j) phi f r, phi = (v_ij . r) / D */
                        const V vij = v[i] - v[j];
                        const double D = dot(rr, rr) + eh2, vr = dot(vij, rr), phi = vr / D;
                        const V c = abar[i] * (P.nu * m / rho[j]);
                        const double cr = dot(c, rr);
                        const V dv = rr * (f * cr / D);
                        VN[i] += dv;
                        VN[j] -= dv;
                        const V dr = (vij * cr + c * vr) * (f / D) + rr * (vr * cr * (g / D - 2.0 * f / (D * D)));
                        XN[i] += dr;
                        XN[j] -= dr;
                        RB[j] -= P.nu * m / (rho[j] * rho[j]) * phi * f * dot(abar[i], rr);
                        gnu += (m / rho[j]) * phi * f * dot(abar[i], rr);
                    }
                }
                for (uint32_t kk = L.bo[i]; kk < L.bo[i + 1]; ++kk) {
                    const uint32_t b = L.bi[kk];
                    const V rr = x[i] - P.bx[b];
                    double f, g;
                    P.K.fg(rr, f, g);
                    if (f == 0.0 && g == 0.0) continue;
                    const double tt = P.psi[b] * f * dot(abar[i], rr);
                    AB[i] -= tt;
                    Bbar[i] -= tt;
                    XN[i] += hess(f, g, rr, abar[i]) * (-P.psi[b] * (Ai + Bi));
                    if (P.nub != 0.0) {
                        const double D = dot(rr, rr) + eh2, vr = dot(v[i], rr), phi = vr / D;
                        const V c = abar[i] * (P.nub * P.psi[b] / rho[i]);
                        const double cr = dot(c, rr);
                        VN[i] += rr * (f * cr / D);
                        XN[i] += (v[i] * cr + c * vr) * (f / D) + rr * (vr * cr * (g / D - 2.0 * f / (D * D)));
                        RB[i] -= P.nub * P.psi[b] / (rho[i] * rho[i]) * phi * f * dot(abar[i], rr);
                    }
                }
            }
        }
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; ++i) {
            double A = 0.0, R = 0.0;
            for (int t = 0; t < T; ++t) {
                A += tA[t][i];
                R += tR[t][i];
                xn[i] += txn[t][i];
                vn[i] += tvn[t][i];
            }
            Abar[i] = A;
            rbar[i] = R;
        }
        /* A = p / rho^2, B = p / rho0^2, EOS */
#pragma omp parallel for schedule(static) reduction(+ : gk)
        for (long i = 0; i < (long)n; ++i) {
            const double pbar = Abar[i] / (rho[i] * rho[i]) + Bbar[i] / (rho0 * rho0);
            rbar[i] += -2.0 * p[i] * Abar[i] / (rho[i] * rho[i] * rho[i]);
            if (p[i] > 0.0) {
                const double ratio = rho[i] / rho0;
                rbar[i] += pbar * P.kr_g * P.gamma * std::pow(ratio, P.gamma - 1.0) / rho0;
                gk += pbar * rho0 / P.gamma * (std::pow(ratio, P.gamma) - 1.0);
            }
        }
        /* density: rho_i = sum_j m W(x_i - x_j) + sum_b psi_b W(x_i - x_b) */
        clear();
#pragma omp parallel
        {
            V* XN = txn[omp_get_thread_num()].data();
#pragma omp for schedule(dynamic, 256)
            for (long i = 0; i < (long)n; ++i) {
                for (uint32_t kk = L.fo[i]; kk < L.fo[i + 1]; ++kk) {
                    const uint32_t j = L.fi[kk];
                    const V rr = x[i] - x[j];
                    double f, g;
                    P.K.fg(rr, f, g);
                    const V gw = rr * (m * rbar[i] * f);
                    XN[i] += gw;
                    XN[j] -= gw;
                }
                for (uint32_t kk = L.bo[i]; kk < L.bo[i + 1]; ++kk) {
                    const V rr = x[i] - P.bx[L.bi[kk]];
                    double f, g;
                    P.K.fg(rr, f, g);
                    XN[i] += rr * (P.psi[L.bi[kk]] * rbar[i] * f);
                }
            }
        }
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; ++i)
            for (int t = 0; t < T; ++t) xn[i] += txn[t][i];
        xb.swap(xn);
        vb.swap(vn);
    }
    for (size_t i = 0; i < n; ++i) {
        dv0[3 * i] = vb[i].x; dv0[3 * i + 1] = vb[i].y; dv0[3 * i + 2] = vb[i].z;
        if (dx0) { dx0[3 * i] = xb[i].x; dx0[3 * i + 1] = xb[i].y; dx0[3 * i + 2] = xb[i].z; }
    }
    if (dnu) *dnu = gnu;
    if (dk) *dk = gk;
    return SPH_OK;
}

} // extern "C"
