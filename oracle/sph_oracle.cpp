/*
 * CPU restatement of SPH2O's per-step particle path -- TEST INFRASTRUCTURE
 * (see sph_oracle.h). Parity pinned against golden vectors produced by the
 * reference itself (tests/test_oracle.py).
 *
 * Each routine restates the reference routine named in its comment, in this
 * project's own code, keeping the reference's operation order and types so
 * the float variant reproduces its FP32 results: unqualified pow() in the
 * reference resolves to the double overload, so the expressions that use it
 * are evaluated in double exactly where the reference's are. Compiled with
 * -ffp-contract=off (no FMA).
 */
#include "sph_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

template <typename R> struct V3 {
    R x = 0, y = 0, z = 0;
    V3() = default;
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    V3 operator+(const V3& o) const { return {x + o.x, y + o.y, z + o.z}; }
    V3 operator-(const V3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    V3 operator-() const { return {-x, -y, -z}; }
    V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    V3 operator*(R s) const { return {x * s, y * s, z * s}; }
    V3 operator/(R s) const { return {x / s, y / s, z / s}; }
    V3& operator*=(R s) { x *= s; y *= s; z *= s; return *this; }
    V3& operator/=(R s) { x /= s; y /= s; z /= s; return *this; }
};
template <typename R> V3<R> operator*(R s, const V3<R>& v) { return {s * v.x, s * v.y, s * v.z}; }
template <typename R> R dot(const V3<R>& a, const V3<R>& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <typename R> R length(const V3<R>& a) { return std::sqrt(dot(a, a)); }

template <typename R> struct Oracle {
    sph_scene_desc d{};
    /* kernel constants (setSupportRadius of each kernel, Kernels.cpp / *.h) */
    R r = 0, h = 0, mass = 0, rho0 = 0, ck = 0, cl = 0, coh1 = 0, coh2 = 0, lapl = 0, eps = (R)1e-5;
    V3<R> g;
    R dt = 0, time = 0, min_ts = 0, max_ts = 0, delta = 0;
    unsigned its = 0, its_v = 0;
    R avg_dens = 0, avg_div = 0, pci_avg = 0;
    bool visc = false, st = false, adh = false;
    std::vector<V3<R>> x, v, a, nrm, predr, pacc;
    std::vector<R> rho, alpha, press, kk, kv, kws, kvws, pred, div;
    std::vector<V3<R>> bx;
    std::vector<R> bvol;
    struct Cube { V3<R> mn, mx; R nf, tf; };
    std::vector<Cube> cubes;
    /* PCISPH boundary method: normals, velocity factors, boundary densities
       and pressures, predicted velocities, kernel constants */
    bool pcib = false;
    std::vector<V3<R>> bn, predv;
    std::vector<R> bdens, bpress;
    R pnf = 0, ptf = 0, rest = 0, h2 = 0, poly6c = 0, spikyg = 0;
    /* since: the neighbour search that first gave the cell candidate lists
       (HashTable keeps every cell ever touched; a cell first touched by a
       lookup gets lists at the next search); nsc: searches so far */
    struct Cell { std::vector<uint32_t> f, b; unsigned since = 0; };
    std::unordered_map<uint64_t, Cell> cells;
    unsigned nsc = 0;

    /* ---- smoothing kernels ---------------------------------------------- */
    /* CubicSpline::W (CubicSpline.h:27-45) */
    R W(R rl) const
    {
        R res = 0;
        const R q = rl / h;
        if (q <= 1.0) {
            if (q <= 0.5) {
                const R q2 = q * q;
                const R q3 = q2 * q;
                res = ck * ((R)6 * q3 - (R)6 * q2 + (R)1);
            } else {
                res = (R)((double)ck * ((double)(R)2 * std::pow((double)((R)1 - q), 3.0)));
            }
        }
        return res;
    }
    R W(const V3<R>& rv) const { return W(length(rv)); }
    /* CubicSpline::gradW (CubicSpline.h:52-74) */
    V3<R> gradW(const V3<R>& rv) const
    {
        V3<R> res;
        const R rl = length(rv);
        const R q = rl / h;
        if (((double)rl > 1.0e-9) && (q <= 1.0)) {
            V3<R> gq = rv / rl;
            gq /= h;
            if (q <= 0.5) {
                res = (cl * q * ((R)3 * q - (R)2)) * gq;
            } else {
                const R f = (R)1 - q;
                res = (cl * (-f * f)) * gq;
            }
        }
        return res;
    }
    /* Cohesion::W (Cohesion.h:20-40) */
    R cohesion(const V3<R>& rv) const
    {
        R value = 0;
        const R m = length(rv);
        if ((2.0 * m > h) && (m <= h))
            value = (R)((double)coh1 * std::pow((double)(h - m), 3.0) * std::pow((double)m, 3.0));
        else if ((m > 0) && (2.0 * m <= h))
            value = (R)((double)(coh1 * (R)2) * std::pow((double)(h - m), 3.0) * std::pow((double)m, 3.0) -
                        (double)coh2);
        return value;
    }
    /* Adhesion::W (Adhesion.h:18-35) -- its 0.007 / h^3.25 factor is never applied there */
    R adhesionW(const V3<R>& rv) const
    {
        const R m = length(rv);
        if ((2.0 * m > h) && (m <= h)) {
            const R value = -(R)4 * m * m / h + (R)6 * m - (R)2 * h;
            return (R)std::pow((double)value, 1.0 / 4.0);
        }
        return 0;
    }
    /* ViscoK::laplW (ViscoK.h:32-38) */
    R laplW(const V3<R>& rv) const
    {
        const R m = length(rv);
        return m <= h ? lapl * (h - m) : (R)0;
    }
    /* Poly6::W (Poly6.h:29-42) */
    R poly6W(const V3<R>& rv) const
    {
        const R m = length(rv);
        const R m2 = m * m;
        if (m2 <= h2) {
            const R diff = h2 - m2;
            return poly6c * diff * diff * diff;
        }
        return 0;
    }
    /* Spiky::gradW (Spiky.h:44-55) */
    V3<R> spikyGrad(const V3<R>& rv) const
    {
        const R m = length(rv);
        if (m != 0 && m <= h) {
            const R diff = h - m;
            return (-spikyg * diff * diff / m) * rv;
        }
        return V3<R>();
    }

    /* ---- set-up (SPHSimulation::importScene/init, SPHSimulation.cpp:117-155, 201-208) */
    void setup(const sph_scene_desc& desc)
    {
        d = desc;
        r = (R)d.particle_radius;
        h = (R)4 * r;
        rho0 = (R)d.density0;
        const R diameter = (R)2 * r;
        mass = rho0 * (R)std::pow((double)diameter, 3.0);
        const R pi = (R)M_PI;
        const R h3 = h * h * h;
        ck = (R)8 / (pi * h3);
        cl = (R)48 / (pi * h3);
        const R h6 = h * h * h * h * h * h;
        const R h9 = h * h * h * h * h * h * h * h * h;
        coh1 = (R)(32.0 / M_PI) / h9;
        coh2 = h6 / (R)64;
        lapl = (R)45 / ((R)M_PI * h6);
        h2 = h * h;
        poly6c = (R)315 / ((R)(64.0 * M_PI) * h9);
        spikyg = (R)45 / ((R)M_PI * h6);
        rest = (R)0.5 * h;
        pcib = d.boundary_method == SPH_BOUNDARY_PCISPH;
        g = V3<R>((R)d.gravity[0], (R)d.gravity[1], (R)d.gravity[2]);
        dt = (R)d.time_step;
        const R fps_ts = (R)1 / (R)d.fps;
        min_ts = fps_ts < (R)d.min_time_step ? fps_ts : (R)d.min_time_step; /* TimeHelper.h:57 */
        max_ts = (R)d.max_time_step;
        visc = d.viscosity_method > -1 && d.viscosity_method <= 2 && d.viscosity != 0.0f;
        st = d.surface_tension_method == SPH_SURFACE_TENSION_AKINCI && d.surface_tension != 0.0f;
        adh = d.adhesion_method == SPH_ADHESION_AKINCI && d.adhesion != 0.0f;
    }

    /* ---- neighbour search (HashTable.cpp:3-86, SPHSolver.cpp:170-219) -- */
    static int64_t cell1(R p, R hh) { return (int64_t)std::floor(p / hh); }
    static uint64_t key(int64_t a, int64_t b, int64_t c)
    {
        return ((uint64_t)(a + (1 << 20)) << 42) | ((uint64_t)(b + (1 << 20)) << 21) | (uint64_t)(c + (1 << 20));
    }
    void cell_of(const V3<R>& p, int64_t* c) const { c[0] = cell1(p.x, h); c[1] = cell1(p.y, h); c[2] = cell1(p.z, h); }

    void insert_boundary()
    {
        for (auto& kvp : cells) kvp.second.b.clear();
        for (size_t i = 0; i < bx.size(); ++i) {
            int64_t c[3];
            cell_of(bx[i], c);
            Cell& cell = cells[key(c[0], c[1], c[2])];
            if (cell.since == 0) cell.since = nsc + 1;
            cell.b.push_back((uint32_t)i);
        }
    }
    void insert_fluid()
    {
        for (auto& kvp : cells) kvp.second.f.clear();
        ++nsc;
        for (size_t i = 0; i < x.size(); ++i) {
            int64_t c[3];
            cell_of(x[i], c);
            Cell& cell = cells[key(c[0], c[1], c[2])];
            if (cell.since == 0) cell.since = nsc;
            cell.f.push_back((uint32_t)i);
        }
    }
    /* the 27 cells of p's cell in x-major offset order (HashTable.cpp:59-65):
       ff(j) for every fluid candidate, then fb(b) for every boundary one */
    template <typename FF, typename FB> void for_candidates(const V3<R>& p, FF ff, FB fb) const
    {
        int64_t c[3];
        cell_of(p, c);
        const Cell* nb[27];
        int n = 0;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    auto it = cells.find(key(c[0] + dx, c[1] + dy, c[2] + dz));
                    if (it != cells.end()) nb[n++] = &it->second;
                }
        for (int q = 0; q < n; ++q)
            for (uint32_t j : nb[q]->f) ff(j);
        for (int q = 0; q < n; ++q)
            for (uint32_t b : nb[q]->b) fb(b);
    }

    /* AkinciBoundaryObject::computeVolume (AkinciBoundaryObject.cpp:10-34) */
    void boundary_volumes()
    {
        bvol.assign(bx.size(), 0);
        for (size_t i = 0; i < bx.size(); ++i) {
            R delta_ = 0;
            for_candidates(bx[i], [](uint32_t) {}, [&](uint32_t b) { delta_ += W(bx[i] - bx[b]); });
            bvol[i] = (R)1 / delta_;
        }
    }
    /* a boundary particle's density weight: rho0 V_b (Akinci) or its mass
       rho0 (2r)^3 (PCISPH method, SPHSimulation.cpp:435-437) */
    R psi(uint32_t b) const { return pcib ? mass : rho0 * bvol[b]; }

    /* whether p's cell held candidate lists at the last search; a lookup of
       an untouched cell creates its entry (HashTable's operator[]) */
    bool listed(const V3<R>& p)
    {
        int64_t c[3];
        cell_of(p, c);
        auto it = cells.find(key(c[0], c[1], c[2]));
        if (it == cells.end()) {
            cells[key(c[0], c[1], c[2])].since = nsc + 1;
            return false;
        }
        return it->second.since <= nsc;
    }

    /* SPHSolver::computeFluidDensities (SPHSolver.cpp:42-89), Akinci branch */
    void densities()
    {
        for (size_t i = 0; i < x.size(); ++i) {
            R dens = 0;
            for_candidates(x[i], [&](uint32_t j) { dens += mass * W(x[i] - x[j]); },
                           [&](uint32_t b) { dens += psi(b) * W(x[i] - bx[b]); });
            rho[i] = dens;
        }
    }

    /* DFSPHSolver::computeAlpha (DFSPHSolver.cpp:109-178) */
    void compute_alpha()
    {
        for (size_t i = 0; i < x.size(); ++i) {
            V3<R> sg;
            R ssq = 0;
            for_candidates(x[i],
                           [&](uint32_t j) {
                               const V3<R> mg = mass * gradW(x[i] - x[j]);
                               sg += mg;
                               ssq += dot(mg, mg);
                           },
                           [&](uint32_t b) { sg += psi(b) * gradW(x[i] - bx[b]); });
            const R den = dot(sg, sg) + ssq;
            alpha[i] = den > eps ? rho[i] / den : (R)0;
        }
    }

    /* non-pressure forces in creation order (SPHSimulation.cpp:256-265,
       FluidObject.cpp:123-175): viscosity, surface tension, adhesion */
    void nonpressure()
    {
        const size_t n = x.size();
        const R h2 = h * h;
        const R visc_c = (R)d.viscosity, bvisc = pcib ? (R)0 : (R)d.boundary_viscosity; /* an Akinci-only term */
        if (visc && d.viscosity_method == SPH_VISCOSITY_ARTIFICIAL) {
            /* ArtificialViscosity::step (ArtificialViscosity.cpp:6-54) */
            for (size_t i = 0; i < n; ++i) {
                const R dens_i = rho[i];
                for_candidates(x[i],
                               [&](uint32_t j) {
                                   const V3<R> rij = x[i] - x[j];
                                   const R dp = dot(v[i] - v[j], rij);
                                   const R sq = dot(rij, rij);
                                   a[i] += (R)(10.0 * 0.1) * visc_c * (mass / rho[j]) * dp / (sq + (R)0.01 * h2) *
                                           gradW(rij);
                               },
                               [](uint32_t) {});
                if (bvisc != 0)
                    for_candidates(x[i], [](uint32_t) {},
                                   [&](uint32_t b) {
                                       const V3<R> rib = x[i] - bx[b];
                                       const R dp = dot(v[i], rib);
                                       const R sq = dot(rib, rib);
                                       a[i] += (R)(10.0 * 0.1) * bvisc * (psi(b) / dens_i) * dp /
                                               (sq + (R)0.01 * h2) * gradW(rib);
                                   });
            }
        } else if (visc && d.viscosity_method == SPH_VISCOSITY_STANDARD) {
            /* StandardViscosityForce::step (StandardViscosity.cpp:5-50) */
            for (size_t i = 0; i < n; ++i) {
                V3<R> vf;
                for_candidates(x[i], [&](uint32_t j) { vf += mass * (v[j] - v[i]) / rho[j] * laplW(x[i] - x[j]); },
                               [](uint32_t) {});
                vf *= visc_c / rho[i];
                a[i] += vf;
                vf = V3<R>();
                if (bvisc != 0) {
                    for_candidates(x[i], [](uint32_t) {},
                                   [&](uint32_t b) { vf += psi(b) * (-v[i]) / rho[i] * laplW(x[i] - bx[b]); });
                    vf *= bvisc / rho[i];
                    a[i] += vf;
                }
            }
        } else if (visc && d.viscosity_method == SPH_VISCOSITY_XSPH) {
            /* XSPHViscosity::step (XSPHViscosity.cpp:6-43) */
            for (size_t i = 0; i < n; ++i) {
                for_candidates(x[i],
                               [&](uint32_t j) {
                                   a[i] += visc_c * (mass / rho[j]) * (v[j] - v[i]) * W(x[i] - x[j]) / dt;
                               },
                               [](uint32_t) {});
                if (bvisc != 0)
                    for_candidates(x[i], [](uint32_t) {},
                                   [&](uint32_t b) {
                                       a[i] += bvisc * (psi(b) / rho[i]) * (-v[i]) * W(x[i] - bx[b]) / dt;
                                   });
            }
        }
        if (st) {
            /* SurfaceTensionAkinci::step (SurfaceTensionAkinci.cpp:5-71) */
            const R sigma = (R)d.surface_tension;
            for (size_t i = 0; i < n; ++i) {
                V3<R> ni;
                for_candidates(x[i], [&](uint32_t j) { ni += (mass / rho[j]) * gradW(x[i] - x[j]); },
                               [](uint32_t) {});
                ni *= h;
                nrm[i] = ni;
            }
            for (size_t i = 0; i < n; ++i) {
                for_candidates(x[i],
                               [&](uint32_t j) {
                                   V3<R> acc;
                                   const V3<R> rij = x[i] - x[j];
                                   const R mag = length(rij);
                                   const R kij = (R)2 * rho0 / (rho[i] + rho[j]);
                                   if (mag > 0 && mag <= h) {
                                       acc -= sigma * mass * cohesion(rij) * rij / mag;
                                       acc -= sigma * (nrm[i] - nrm[j]);
                                   }
                                   a[i] += kij * acc;
                               },
                               [](uint32_t) {});
            }
        }
        if (adh) {
            /* AdhesionForce::step (AdhesionForce.cpp:5-33) */
            const R beta = (R)d.adhesion;
            for (size_t i = 0; i < n; ++i)
                for_candidates(x[i], [](uint32_t) {},
                               [&](uint32_t b) {
                                   const V3<R> rib = x[i] - bx[b];
                                   const R mag = length(rib);
                                   if (mag > 0) a[i] -= beta * rho0 * bvol[b] * adhesionW(rib) * rib / mag;
                               });
        }
    }

    /* ---- WCSPH (WCSPHSolver.cpp:14-188) ------------------------------- */
    void wcsph_pressures()
    {
        const R k = (R)d.stiffness, gm = (R)d.gamma;
        for (size_t i = 0; i < x.size(); ++i)
            press[i] = std::max((R)0, k * rho0 / gm * (std::pow(rho[i] / rho0, gm) - (R)1));
    }
    void wcsph_pressure_force()
    {
        for (size_t i = 0; i < x.size(); ++i) {
            const R dpi = press[i] / (rho[i] * rho[i]);
            for_candidates(x[i],
                           [&](uint32_t j) {
                               a[i] -= mass * (dpi + press[j] / (rho[j] * rho[j])) * gradW(x[i] - x[j]);
                           },
                           [](uint32_t) {});
            const R dpb = press[i] / (rho0 * rho0);
            if (pcib) /* WCSPHSolver.cpp:160-171 */
                for_candidates(x[i], [](uint32_t) {}, [&](uint32_t b) {
                    a[i] -= mass * (dpi + bpress[b] / (bdens[b] * bdens[b])) * gradW(x[i] - bx[b]);
                });
            else
                for_candidates(x[i], [](uint32_t) {},
                               [&](uint32_t b) { a[i] -= psi(b) * (dpi + dpb) * gradW(x[i] - bx[b]); });
        }
    }
    /* SPHSolver::integrate (SPHSolver.cpp:139-168) */
    void integrate()
    {
        for (size_t i = 0; i < x.size(); ++i) {
            a[i] += g;
            v[i] += a[i] * dt;
            x[i] += v[i] * dt;
            a[i] = V3<R>();
        }
    }
    /* CubeBoundaryObject::correctPositionAndVelocity (CubeBoundaryObject.cpp:10-88) */
    static void cube_axis(R& p, R& v, R& t1, R& t2, R lo, R hi, R nf, R tf)
    {
        if (p < lo) {
            p = lo;
            if (v < 0.0) v *= -nf;
            t1 *= tf;
            t2 *= tf;
        } else if (p > hi) {
            p = hi;
            if (v > 0.0) v *= -nf;
            t1 *= tf;
            t2 *= tf;
        }
    }
    void cube_correct()
    {
        for (const Cube& c : cubes)
            for (size_t i = 0; i < x.size(); ++i) {
                cube_axis(x[i].x, v[i].x, v[i].y, v[i].z, c.mn.x, c.mx.x, c.nf, c.tf);
                cube_axis(x[i].y, v[i].y, v[i].x, v[i].z, c.mn.y, c.mx.y, c.nf, c.tf);
                cube_axis(x[i].z, v[i].z, v[i].x, v[i].y, c.mn.z, c.mx.z, c.nf, c.tf);
            }
    }

    /* ---- PCISPH boundary method (PCISPHBoundaryObject.cpp:218-447) ---- */
    /* boundary densities: SPHSolver::computeBoundaryDensities (cubic spline,
       SPHSolver.cpp:91-124) or PCISPHSolver::predictBoundaryDensities (Poly6
       at the predicted fluid positions, PCISPHSolver.cpp:211-244) */
    void boundary_densities(bool poly6, const std::vector<V3<R>>& fx)
    {
        for (size_t b = 0; b < bx.size(); ++b) {
            R dens = 0;
            for_candidates(bx[b],
                           [&](uint32_t j) { dens += mass * (poly6 ? poly6W(bx[b] - fx[j]) : W(bx[b] - fx[j])); },
                           [&](uint32_t q) { dens += mass * (poly6 ? poly6W(bx[b] - bx[q]) : W(bx[b] - bx[q])); });
            bdens[b] = dens;
        }
    }
    /* WCSPHSolver::computeBoundaryPressures (WCSPHSolver.cpp:97-114) */
    void boundary_pressures()
    {
        const R k = (R)d.stiffness, gm = (R)d.gamma;
        for (size_t b = 0; b < bx.size(); ++b)
            bpress[b] = std::max((R)0, k * rho0 / gm * (std::pow(bdens[b] / rho0, gm) - (R)1));
    }
    /* collision sums of point p (test) weighted at q (correctPositions /
       correctPredPositions): writes the normal (glm::normalize of the
       weighted sum, NaN when it is zero) and returns whether to push, with
       the push length (1 / wsum) w2sum */
    bool collide(size_t i, const V3<R>& p, const V3<R>& q, bool lookup, R& s)
    {
        V3<R> avg;
        R wsum = 0, w2sum = 0;
        if (!lookup || listed(p))
            for_candidates(p, [](uint32_t) {}, [&](uint32_t b) {
                if (length(p - bx[b]) < rest) {
                    const R l = length(q - bx[b]);
                    const R w = std::max((R)0, (rest - l) / rest);
                    wsum += w;
                    w2sum += w * (rest - l);
                    avg += w * bn[b];
                }
            });
        nrm[i] = avg * ((R)1 / std::sqrt(dot(avg, avg)));
        s = (R)1 / wsum * w2sum;
        return wsum > 0;
    }
    /* correctPositions at the updated positions, weighted there (WCSPH,
       DFSPH) or at the predicted positions (PCISPH) */
    void pcib_positions(bool pred)
    {
        for (size_t i = 0; i < x.size(); ++i) {
            R sc;
            if (collide(i, x[i], pred ? predr[i] : x[i], true, sc)) x[i] += sc * nrm[i];
        }
    }
    /* correctPredPositions: tested at the current position, weighted at and
       moving the predicted one */
    void pcib_pred_positions()
    {
        for (size_t i = 0; i < x.size(); ++i) {
            R sc;
            if (collide(i, x[i], predr[i], false, sc)) predr[i] += sc * nrm[i];
        }
    }
    /* correctVelocities from u = v (WCSPH, DFSPH) or the predicted velocity (PCISPH) */
    void pcib_velocities(bool pred)
    {
        for (size_t i = 0; i < x.size(); ++i) {
            const V3<R>& n = nrm[i];
            if (!(length(n) > 0)) continue;
            const V3<R> u = pred ? predv[i] : v[i];
            const V3<R> nv = dot(u, n) * n;
            const V3<R> tv = u - nv;
            v[i] = ptf * tv - pnf * nv;
        }
    }

    void wcsph_step()
    {
        insert_fluid();
        densities();
        if (pcib) boundary_densities(false, x);
        wcsph_pressures();
        if (pcib) boundary_pressures();
        wcsph_pressure_force();
        nonpressure();
        integrate();
        cube_correct();
        if (pcib) { /* WCSPHSolver.cpp:62-72 */
            pcib_positions(false);
            pcib_velocities(false);
        }
        time += dt;
    }

    /* ---- PCISPH (PCISPHSolver.cpp:20-436) ------------------------------ */
    void pcisph_scaling()
    {
        const R dist = (R)2 * r;
        V3<R> sg;
        R ssq = 0;
        for (int i = -1; i <= 1; i++)
            for (int j = -1; j <= 1; j++)
                for (int k = -1; k <= 1; k++) {
                    V3<R> rij((R)(-i), (R)(-j), (R)(-k));
                    rij *= dist;
                    const V3<R> gr = gradW(rij);
                    sg += gr;
                    ssq += dot(gr, gr);
                }
        const R beta = (R)((double)(R)2 * std::pow((double)(mass * dt / rho0), 2.0));
        const R dsg = dot(sg, sg);
        delta = -(R)1 / (beta * (-dsg - ssq));
    }
    void pcisph_step()
    {
        insert_fluid();
        densities();
        nonpressure();
        const size_t n = x.size();
        for (size_t i = 0; i < n; ++i) { press[i] = 0; pacc[i] = V3<R>(); }
        if (pcib) std::fill(bpress.begin(), bpress.end(), (R)0);
        unsigned it = 0;
        while ((pci_avg > (R)d.eta || it < d.min_iterations) && it < d.max_iterations) {
            for (size_t i = 0; i < n; ++i) {
                const V3<R> acc = a[i] + pacc[i] + g;
                const V3<R> pv = v[i] + acc * dt;
                predv[i] = pv;
                predr[i] = x[i] + pv * dt;
            }
            if (pcib) pcib_pred_positions();
            /* predicted densities over the start-of-step candidates of x_i's cell */
            for (size_t i = 0; i < n; ++i) {
                R dens = 0;
                for_candidates(x[i], [&](uint32_t j) { dens += mass * W(predr[i] - predr[j]); },
                               [&](uint32_t b) { dens += psi(b) * W(predr[i] - bx[b]); });
                rho[i] = dens;
            }
            R avg = 0;
            for (size_t i = 0; i < n; ++i) {
                const R err = std::max((R)0, rho[i] - rho0);
                press[i] += delta * err;
                avg += err / rho0;
            }
            pci_avg = avg / (R)n;
            if (pcib) { /* predictBoundaryDensities + the boundary part of updatePressure */
                boundary_densities(true, predr);
                for (size_t b = 0; b < bx.size(); ++b) bpress[b] += delta * std::max((R)0, bdens[b] - rho0);
            }
            for (size_t i = 0; i < n; ++i) {
                V3<R> pa;
                const R dpi = press[i] / (rho[i] * rho[i]);
                for_candidates(x[i],
                               [&](uint32_t j) {
                                   pa -= mass * (dpi + press[j] / (rho[j] * rho[j])) * gradW(x[i] - x[j]);
                               },
                               [&](uint32_t b) {
                                   if (pcib) /* PCISPHSolver.cpp:336-347 */
                                       pa -= mass * (dpi + bpress[b] / (bdens[b] * bdens[b])) * spikyGrad(x[i] - bx[b]);
                                   else
                                       pa -= psi(b) * dpi * gradW(x[i] - bx[b]);
                               });
                pacc[i] = pa;
            }
            ++it;
        }
        its = it;
        avg_dens = pci_avg;
        for (size_t i = 0; i < n; ++i) {
            a[i] += g + pacc[i];
            v[i] += a[i] * dt;
            x[i] += v[i] * dt;
            a[i] = V3<R>();
        }
        cube_correct();
        if (pcib) { /* PCISPHSolver.cpp:64-74 */
            pcib_positions(true);
            pcib_velocities(true);
        }
        time += dt;
    }

    /* ---- DFSPH (DFSPHSolver.cpp:33-1162) ------------------------------- */
    /* predictDensities (:226-299) */
    R predict_densities()
    {
        R avg = 0;
        for (size_t i = 0; i < x.size(); ++i) {
            R change = 0;
            for_candidates(x[i], [&](uint32_t j) { change += mass * dot(v[i] - v[j], gradW(x[i] - x[j])); },
                           [&](uint32_t b) { change += psi(b) * dot(v[i], gradW(x[i] - bx[b])); });
            R pd = rho[i] + change * dt;
            pd = std::max(pd, rho0);
            pred[i] = pd;
            avg += (pd - rho0) / rho0;
        }
        return avg / (R)x.size();
    }
    /* computeDivergenceError (:538-621) */
    R divergence_errors()
    {
        R avg = 0;
        for (size_t i = 0; i < x.size(); ++i) {
            R e = 0;
            unsigned cnt = 0;
            for_candidates(x[i],
                           [&](uint32_t j) {
                               e += mass * dot(v[i] - v[j], gradW(x[i] - x[j]));
                               if (length(x[i] - x[j]) <= h) cnt++;
                           },
                           [&](uint32_t b) {
                               e += psi(b) * dot(v[i], gradW(x[i] - bx[b]));
                               if (length(x[i] - bx[b]) <= h) cnt++;
                           });
            e = cnt < 20 ? (R)0 : std::max(e, (R)0);
            div[i] = e;
            avg += e / rho0;
        }
        return avg / (R)x.size();
    }
    /* the shared velocity update of correctDensityError / correctDivergenceError / warm starts */
    void correct(const std::vector<R>& K)
    {
        const size_t n = x.size();
        std::vector<V3<R>> dv(n);
        for (size_t i = 0; i < n; ++i) {
            const R ki = K[i];
            V3<R> sum;
            for_candidates(x[i],
                           [&](uint32_t j) {
                               const R ks = ki + K[j];
                               if (std::fabs(ks) > eps) sum += mass * ks * gradW(x[i] - x[j]);
                           },
                           [](uint32_t) {});
            if (std::fabs(ki) > eps)
                for_candidates(x[i], [](uint32_t) {}, [&](uint32_t b) { sum += psi(b) * ki * gradW(x[i] - bx[b]); });
            dv[i] = sum;
        }
        for (size_t i = 0; i < n; ++i) v[i] -= dt * dv[i];
    }
    /* updateTimeStep (:1090-1162) */
    void update_time_step()
    {
        R vmax = 0;
        for (size_t i = 0; i < x.size(); ++i) {
            const V3<R> acc = a[i] + g;
            const V3<R> cv = v[i] + acc * dt;
            vmax = std::max(vmax, length(cv));
        }
        if (vmax < 1.0e-9) vmax = (R)1.0e-9;
        R hs = dt;
        const R cfl = (R)d.cfl_factor * (R)0.4 * ((R)2 * r) / vmax;
        const unsigned itmax = std::max(its, its_v);
        if (itmax > 6) hs *= (R)0.9;
        else if (itmax < 4) hs *= (R)1.05;
        hs = std::min(hs, cfl);
        hs = std::max(hs, min_ts);
        hs = std::min(hs, max_ts);
        dt = hs;
    }
    void dfsph_step()
    {
        const size_t n = x.size();
        nonpressure();
        update_time_step();
        for (size_t i = 0; i < n; ++i) { v[i] += (a[i] + g) * dt; a[i] = V3<R>(); }
        if (pcib) pcib_velocities(false); /* DFSPHSolver.cpp:46-52 */
        const R ts2 = dt * dt;
        /* densityWarmStart (:851-955) */
        predict_densities();
        for (size_t i = 0; i < n; ++i) kws[i] = pred[i] > rho0 ? kws[i] / ts2 : (R)0;
        correct(kws);
        std::fill(kws.begin(), kws.end(), (R)0);
        /* correctDensityError (:414-536) */
        unsigned it = 0;
        R avg = 0;
        while ((avg > (R)d.eta || it < d.min_iterations) && it < d.max_iterations) {
            avg = predict_densities();
            for (size_t i = 0; i < n; ++i) {
                kk[i] = (pred[i] - rho0) * alpha[i] / (ts2 * rho[i]);
                kws[i] += kk[i];
            }
            correct(kk);
            ++it;
        }
        for (size_t i = 0; i < n; ++i) kws[i] *= ts2;
        its = it;
        avg_dens = avg;
        for (size_t i = 0; i < n; ++i) x[i] += v[i] * dt;  /* updatePositions (:204-224) */
        if (pcib) pcib_positions(false);                   /* :60-70 */
        insert_fluid();
        densities();
        compute_alpha();
        /* divergenceWarmStart (:957-1059) */
        divergence_errors();
        for (size_t i = 0; i < n; ++i) kvws[i] = div[i] > 0 ? kvws[i] / dt : (R)0;
        correct(kvws);
        std::fill(kvws.begin(), kvws.end(), (R)0);
        /* correctDivergenceError (:730-849), capped by maxIterations (:746) */
        it = 0;
        R avgv = 0;
        while ((avgv > (R)d.eta_v / dt || it < d.min_iterations_v) && it < d.max_iterations) {
            avgv = divergence_errors();
            for (size_t i = 0; i < n; ++i) {
                kv[i] = div[i] * alpha[i] / (dt * rho[i]);
                kvws[i] += kv[i];
            }
            correct(kv);
            ++it;
        }
        for (size_t i = 0; i < n; ++i) kvws[i] *= dt;
        its_v = it;
        avg_div = avgv;
        cube_correct();
        time += dt;
    }

    void resize(size_t n)
    {
        v.resize(n); a.assign(n, V3<R>()); nrm.assign(n, V3<R>()); predr.assign(n, V3<R>()); pacc.assign(n, V3<R>());
        rho.assign(n, 0); alpha.assign(n, 0); press.assign(n, 0); kk.assign(n, 0); kv.assign(n, 0);
        kws.assign(n, 0); kvws.assign(n, 0); pred.assign(n, 0); div.assign(n, 0);
        predv.assign(n, V3<R>());
        bdens.assign(bx.size(), 0); bpress.assign(bx.size(), 0);
    }

    void init()
    {
        resize(x.size());
        insert_boundary();
        if (!pcib) boundary_volumes();
        if (d.simulation_method == SPH_PCISPH) pcisph_scaling();
        insert_fluid();
        if (d.simulation_method == SPH_DFSPH) {
            densities();
            compute_alpha();
        }
    }

    void step()
    {
        if (d.simulation_method == SPH_WCSPH) wcsph_step();
        else if (d.simulation_method == SPH_PCISPH) pcisph_step();
        else dfsph_step();
    }
};

struct Any {
    int fp64;
    Oracle<float> f;
    Oracle<double> dd;
};

} // namespace

struct sph_oracle : Any {};

extern "C" {

sph_oracle* sph_oracle_create(const sph_scene_desc* desc, int fp64)
{
    if (!desc) return nullptr;
    sph_oracle* o = new sph_oracle();
    o->fp64 = fp64 ? 1 : 0;
    o->f.setup(*desc);
    o->dd.setup(*desc);
    return o;
}

int sph_oracle_set_fluid(sph_oracle* o, unsigned n, const float* xyz, const float* v)
{
    if (!o || (n && !xyz)) return SPH_ERR_ARG;
    auto fill = [&](auto& S) {
        using R = std::remove_reference_t<decltype(S.r)>;
        S.x.resize(n);
        S.v.resize(n);
        for (unsigned i = 0; i < n; ++i) {
            S.x[i] = {(R)xyz[3 * i], (R)xyz[3 * i + 1], (R)xyz[3 * i + 2]};
            S.v[i] = v ? V3<R>((R)v[3 * i], (R)v[3 * i + 1], (R)v[3 * i + 2]) : V3<R>();
        }
    };
    fill(o->f);
    fill(o->dd);
    return SPH_OK;
}

int sph_oracle_set_boundary(sph_oracle* o, unsigned n, const float* xyz)
{
    if (!o || (n && !xyz)) return SPH_ERR_ARG;
    auto fill = [&](auto& S) {
        using R = std::remove_reference_t<decltype(S.r)>;
        S.bx.resize(n);
        for (unsigned i = 0; i < n; ++i) S.bx[i] = {(R)xyz[3 * i], (R)xyz[3 * i + 1], (R)xyz[3 * i + 2]};
    };
    fill(o->f);
    fill(o->dd);
    return SPH_OK;
}

int sph_oracle_set_boundary_normals(sph_oracle* o, unsigned n, const float* nxyz, float normal_fct,
                                    float tangential_fct)
{
    if (!o || (n && !nxyz)) return SPH_ERR_ARG;
    auto fill = [&](auto& S) {
        using R = std::remove_reference_t<decltype(S.r)>;
        S.bn.resize(n);
        for (unsigned i = 0; i < n; ++i) S.bn[i] = {(R)nxyz[3 * i], (R)nxyz[3 * i + 1], (R)nxyz[3 * i + 2]};
        S.pnf = (R)normal_fct;
        S.ptf = (R)tangential_fct;
    };
    fill(o->f);
    fill(o->dd);
    return SPH_OK;
}

int sph_oracle_boundary_state(sph_oracle* o, double* dens, double* press)
{
    if (!o) return SPH_ERR_ARG;
    auto get = [&](auto& S) {
        for (size_t b = 0; b < S.bdens.size(); ++b) {
            if (dens) dens[b] = S.bdens[b];
            if (press) press[b] = S.bpress[b];
        }
    };
    if (o->fp64) get(o->dd);
    else get(o->f);
    return SPH_OK;
}

int sph_oracle_add_cube(sph_oracle* o, const float* mn, const float* mx, float normal_fct, float tangential_fct)
{
    if (!o || !mn || !mx) return SPH_ERR_ARG;
    auto add = [&](auto& S) {
        using R = std::remove_reference_t<decltype(S.r)>;
        S.cubes.push_back({V3<R>((R)mn[0], (R)mn[1], (R)mn[2]), V3<R>((R)mx[0], (R)mx[1], (R)mx[2]), (R)normal_fct,
                           (R)tangential_fct});
    };
    add(o->f);
    add(o->dd);
    return SPH_OK;
}

int sph_oracle_init(sph_oracle* o)
{
    if (!o) return SPH_ERR_ARG;
    if (o->fp64) o->dd.init();
    else o->f.init();
    return SPH_OK;
}

int sph_oracle_step(sph_oracle* o, int nsteps, double* stats)
{
    if (!o || nsteps < 0) return SPH_ERR_ARG;
    for (int s = 0; s < nsteps; ++s) {
        auto run = [&](auto& S) {
            S.step();
            if (stats) {
                double* row = stats + 6 * (size_t)s;
                row[0] = (double)S.time; row[1] = (double)S.dt; row[2] = S.its; row[3] = S.its_v;
                row[4] = (double)S.avg_dens; row[5] = (double)S.avg_div;
            }
        };
        if (o->fp64) run(o->dd);
        else run(o->f);
    }
    return SPH_OK;
}

int sph_oracle_get_state(sph_oracle* o, double* xyz, double* v, double* rho)
{
    if (!o) return SPH_ERR_ARG;
    auto get = [&](auto& S) {
        for (size_t i = 0; i < S.x.size(); ++i) {
            if (xyz) { xyz[3 * i] = S.x[i].x; xyz[3 * i + 1] = S.x[i].y; xyz[3 * i + 2] = S.x[i].z; }
            if (v) { v[3 * i] = S.v[i].x; v[3 * i + 1] = S.v[i].y; v[3 * i + 2] = S.v[i].z; }
            if (rho) rho[i] = S.rho[i];
        }
    };
    if (o->fp64) get(o->dd);
    else get(o->f);
    return SPH_OK;
}

int sph_oracle_get_boundary_volume(sph_oracle* o, double* vol)
{
    if (!o || !vol) return SPH_ERR_ARG;
    auto get = [&](auto& S) { for (size_t i = 0; i < S.bvol.size(); ++i) vol[i] = S.bvol[i]; };
    if (o->fp64) get(o->dd);
    else get(o->f);
    return SPH_OK;
}

int sph_oracle_phase(sph_oracle* o, int phase, double* out)
{
    if (!o || !out) return SPH_ERR_ARG;
    auto run = [&](auto& S) -> int {
        using R = std::remove_reference_t<decltype(S.r)>;
        S.insert_fluid();
        S.densities();
        if (S.pcib) { /* computeDensities covers the boundary particles; WCSPH their pressures */
            S.boundary_densities(false, S.x);
            if (S.d.simulation_method == SPH_WCSPH) S.boundary_pressures();
        }
        const size_t n = S.x.size();
        switch (phase) {
        case SPH_PHASE_DENSITY: for (size_t i = 0; i < n; ++i) out[i] = S.rho[i]; break;
        case SPH_PHASE_ALPHA: S.compute_alpha(); for (size_t i = 0; i < n; ++i) out[i] = S.alpha[i]; break;
        case SPH_PHASE_NONPRESSURE_ACC:
            std::fill(S.a.begin(), S.a.end(), V3<R>());
            S.nonpressure();
            for (size_t i = 0; i < n; ++i) { out[3 * i] = S.a[i].x; out[3 * i + 1] = S.a[i].y; out[3 * i + 2] = S.a[i].z; }
            std::fill(S.a.begin(), S.a.end(), V3<R>());
            break;
        case SPH_PHASE_PRESSURE: S.wcsph_pressures(); for (size_t i = 0; i < n; ++i) out[i] = S.press[i]; break;
        case SPH_PHASE_PRESSURE_ACC:
            S.wcsph_pressures();
            std::fill(S.a.begin(), S.a.end(), V3<R>());
            S.wcsph_pressure_force();
            for (size_t i = 0; i < n; ++i) { out[3 * i] = S.a[i].x; out[3 * i + 1] = S.a[i].y; out[3 * i + 2] = S.a[i].z; }
            std::fill(S.a.begin(), S.a.end(), V3<R>());
            break;
        default: return SPH_ERR_ARG;
        }
        return SPH_OK;
    };
    return o->fp64 ? run(o->dd) : run(o->f);
}

int sph_oracle_neighbors(sph_oracle* o, unsigned* f_off, unsigned* f_idx, size_t f_cap, unsigned* b_off,
                         unsigned* b_idx, size_t b_cap, size_t* nf_total, size_t* nb_total)
{
    if (!o) return SPH_ERR_ARG;
    auto run = [&](auto& S) {
        S.insert_fluid();
        size_t tf = 0, tb = 0;
        for (size_t i = 0; i < S.x.size(); ++i) {
            if (f_off) f_off[i] = (unsigned)tf;
            if (b_off) b_off[i] = (unsigned)tb;
            S.for_candidates(S.x[i],
                             [&](uint32_t j) {
                                 if (length(S.x[i] - S.x[j]) <= S.h) { if (f_idx && tf < f_cap) f_idx[tf] = j; ++tf; }
                             },
                             [&](uint32_t b) {
                                 if (length(S.x[i] - S.bx[b]) <= S.h) { if (b_idx && tb < b_cap) b_idx[tb] = b; ++tb; }
                             });
        }
        if (f_off) f_off[S.x.size()] = (unsigned)tf;
        if (b_off) b_off[S.x.size()] = (unsigned)tb;
        if (nf_total) *nf_total = tf;
        if (nb_total) *nb_total = tb;
    };
    if (o->fp64) run(o->dd);
    else run(o->f);
    return SPH_OK;
}

void sph_oracle_destroy(sph_oracle* o) { delete o; }

} // extern "C"
