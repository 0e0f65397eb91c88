/*
 * Device-side parameters, smoothing kernels and helpers shared by all
 * kernels of the particle pipeline (sm_100a).
 *
 * Data layout in HBM (all arrays in cell-sorted particle order):
 *   pos  float4 (x, y, z, unused)      vel  float4 (vx, vy, vz, unused)
 *   acc  float4 non-pressure acceleration
 *   rho, alpha, k, kws, kvws, press    float scalars (SoA)
 *   orig uint32 caller-order id of each sorted slot
 *   bpos float4 (x, y, z, psi = rho0 * V_b) for the static boundary
 *   neighbour lists: column-major uint32 nbrF[k * nf + i] / nbrB[k * nf + i]
 *   with counts cntF[i] / cntB[i], so a warp of consecutive particles reads
 *   its k-th neighbours as one coalesced 128-byte line.
 */
#ifndef SPH2O_DEVICE_CUH
#define SPH2O_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

namespace sph {

/* error bits in DevState::err */
enum : int { ERRBIT_NAN = 1, ERRBIT_OVERFLOW = 2, ERRBIT_TIMEOUT = 4 };

/* bounded spin: ~2^22 polls with >= 256 ns sleep each (> 1 s) */
constexpr unsigned long long kSpinLimit = 1ull << 22;

struct SimParams {
    int nf, nb;
    /* smoothing */
    float r, h, h2, inv_h, mass, rho0;
    float cs_k;         /* CubicSpline k = 8 / (pi h^3)            (CubicSpline.h:23) */
    float cs_l;         /* CubicSpline l = 48 / (pi h^3)           (CubicSpline.h:24) */
    float cs_l_h2;      /* l / h^2: gradient factor for q <= 1/2                      */
    float cs_l_h;       /* l / h:   gradient factor for q > 1/2                       */
    float coh_c1;       /* Cohesion 32 / (pi h^9)                  (Cohesion.h:26)    */
    float coh_c2;       /* Cohesion h^6 / 64                       (Cohesion.h:27)    */
    float lapl_c;       /* ViscoK 45 / (pi h^6)                    (ViscoK.h:24)      */
    float gx, gy, gz;
    /* solvers */
    float stiffness, gamma;
    float kr_g;         /* (stiffness * rho0) / gamma, WCSPHSolver.cpp:93            */
    float h2_guard;     /* h^2 (1 + 1e-5): exact-W candidates above it are 0 anyway  */
    float h2_exact;     /* sqrt_le_bound(h): s <= h2_exact exactly when sqrt_rn(s) <= h */
    float eta, eta_v, cfl, min_ts, max_ts;
    unsigned min_it, max_it, min_it_v, max_it_v;
    float pcisph_delta;
    float eps;          /* DFSPH eps = 1e-5 (DFSPHSolver.cpp:19)                      */
    /* non-pressure forces (effective: method set and coefficient non-zero) */
    int visc_method;    /* -1 none, 0 standard, 1 artificial, 2 XSPH */
    float visc, bvisc;
    int st_on;
    float st;
    int adh_on;
    float adh;
    /* grid */
    int cminx, cminy, cminz;   /* integer cell key of grid cell (0,0,0) */
    int dimx, dimy, dimz;      /* cells per axis (multiples of 4)        */
    int nbx, nby;              /* 4^3 bricks per axis (x, y)             */
    unsigned ncells;
    unsigned capF, capB;       /* neighbour-list capacity per particle   */
    int cell_order;            /* 0: 4^3 bricks, Morton inside; 1: linear, x fastest */
    int dynamic;               /* emitters: passes cover DevState::n_active particles, nf is the capacity */
    /* PCISPH boundary method (boundaryMethod 1): mass boundary particles */
    int pcib;                  /* 1: boundary particles carry normals, densities and pressures */
    float pcib_nf, pcib_tf;    /* normalFct, tangFct of the boundary object                     */
    float rest_r;              /* collision distance 0.5 h (PCISPHBoundaryObject.cpp:222)        */
    float poly6_c;             /* Poly6 315 / (64 pi h^9)                 (Poly6.h:25)            */
    float spiky_g;             /* Spiky gradient 45 / (pi h^6)            (Spiky.h:25)            */
    /* 1: positions carry their rounding residual (DeviceArrays::plo) and
       integrate as float pairs; 0: plain FP32 as the reference rounds */
    int pos_lo;
};

/* Device-resident solver state; read by the host after a step. */
struct DevState {
    double time;
    double avg_dens;
    double avg_div;
    double pcisph_avg;          /* PCISPH residual carried into the next step */
    float dt;
    unsigned vmax_bits;         /* DFSPH CFL speed, float bits (>= 0)         */
    unsigned its, its_v;
    unsigned long long sum_its, sum_its_v;
    unsigned steps;
    int err;
    unsigned overflow;
    unsigned bar_count, bar_gen;
    float last_vmax;
    unsigned n_active;          /* active fluid particles (emitters append to them) */
    unsigned ns_epoch;          /* neighbour searches so far (PCISPH boundary cell entries) */
};

/* Fluid particles a pass covers: all nf, or with emitters the active prefix
   (slots [0, n_active) of the sorted arrays; nf stays the list stride). */
__device__ __forceinline__ int active_n(const SimParams& P, const DevState* st)
{
    return P.dynamic ? (int)st->n_active : P.nf;
}

/* Simulated time advanced as the reference keeps it: a float sum (TimeHelper
   holds Real time, TimeHelper.h:29, and steps add dt to it). */
__device__ __forceinline__ double advance_time(double t, float dt)
{
    return (double)__fadd_rn((float)t, dt);
}

/* x + d for one position coordinate. With the residual on, lo holds what
   the float x has lost of the exact sum of all the steps so far; the pair is
   advanced with an error-free float sum (Knuth's TwoSum), so a long run of
   steps much smaller than x's spacing is integrated to about twice float
   precision while every pass keeps reading the float x. */
__device__ __forceinline__ float pos_add(float x, float& lo, float d, int on)
{
    if (!on) return __fadd_rn(x, d);
    const float t = __fadd_rn(lo, d);
    const float s = __fadd_rn(x, t);
    const float bp = __fsub_rn(s, x);
    lo = __fadd_rn(__fsub_rn(x, __fsub_rn(s, bp)), __fsub_rn(t, bp));
    return s;
}

/* A cube boundary (CubeBoundaryObject.h:6-27): box and velocity factors. */
struct CubeBox {
    float minx, miny, minz, maxx, maxy, maxz;
    float normal_fct, tangential_fct;
};

/* One particle emitter (Emitter.h:10-33) on the device: pose, speed, the
   next emission time, what is left to emit and its group of particle
   offsets in the group table. */
struct EmitterState {
    float px, py, pz;           /* position r */
    float qw, qx, qy, qz;       /* rotation (glm::quat w, x, y, z) */
    float v;                    /* speed along local z */
    float next;                 /* nextTimeEmit */
    float period;               /* spacing * 1.105 * 2r / v, added after each emission */
    unsigned remaining;         /* numParticles still to emit */
    unsigned group_begin, group_count;
    unsigned pad;
};

/* ---------------------------------------------------------------------- */
/* Cubic spline (CubicSpline.h:27-74). q = |r| / h.                        */

__device__ __forceinline__ float cs_W(float q, const SimParams& P)
{
    if (q <= 0.5f) {
        const float q2 = q * q;
        const float q3 = q2 * q;
        return P.cs_k * (6.0f * q3 - 6.0f * q2 + 1.0f);
    }
    const float t = fmaxf(1.0f - q, 0.0f);
    return P.cs_k * (2.0f * (t * t * t));
}

/* W(r) with SPH2O's exact FP32 operation sequence: |r| = sqrt((x x + y y) + z z),
   q = |r| / h, k (6 q^3 - 6 q^2 + 1) or k (2 pow(1 - q, 3)); the reference's
   unqualified pow resolves to the double overload, so k * 2 * (1 - q)^3 is
   formed in double and rounded once. No contraction into FMA anywhere, so densities
   summed in the reference's neighbour order are bit-identical to its strict
   FP32 build. Used where a density enters a cancellation-prone expression
   (Tait EOS, PCISPH pressure update, DFSPH k) and for boundary volumes. */
__device__ __forceinline__ float dist2_exact(float4 a, float4 b)
{
    const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ __forceinline__ float cs_W_exact(float s, const SimParams& P)
{
    const float q = __fdiv_rn(__fsqrt_rn(s), P.h);
    if (!(q <= 1.0f)) return 0.0f;
    if (q <= 0.5f) {
        const float q2 = __fmul_rn(q, q);
        const float q3 = __fmul_rn(q2, q);
        return __fmul_rn(P.cs_k, __fadd_rn(__fsub_rn(__fmul_rn(6.0f, q3), __fmul_rn(6.0f, q2)), 1.0f));
    }
    /* k * (2.0f * pow(1 - q, 3.0)): pow returns double, so the whole
       product is formed in double and rounded to float once */
    const double t = (double)__fsub_rn(1.0f, q);
    const double cube = __dmul_rn(__dmul_rn(t, t), t);
    return (float)__dmul_rn((double)P.cs_k, __dmul_rn(2.0, cube));
}

/* gradW(r) with SPH2O's exact FP32 operation sequence (CubicSpline.h:52-74):
   gradq = (r / |r|) / h, then (l q (3q - 2)) gradq or (l (-(1-q)(1-q))) gradq. */
__device__ __forceinline__ void cs_gradW_exact(float rx, float ry, float rz, const SimParams& P, float& gx,
                                               float& gy, float& gz)
{
    const float s = __fadd_rn(__fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry)), __fmul_rn(rz, rz));
    const float rl = __fsqrt_rn(s);
    const float q = __fdiv_rn(rl, P.h);
    gx = gy = gz = 0.0f;
    if (!((double)rl > 1.0e-9) || !(q <= 1.0f)) return;
    const float qx = __fdiv_rn(__fdiv_rn(rx, rl), P.h);
    const float qy = __fdiv_rn(__fdiv_rn(ry, rl), P.h);
    const float qz = __fdiv_rn(__fdiv_rn(rz, rl), P.h);
    float c;
    if (q <= 0.5f) {
        c = __fmul_rn(__fmul_rn(P.cs_l, q), __fsub_rn(__fmul_rn(3.0f, q), 2.0f));
    } else {
        const float f = __fsub_rn(1.0f, q);
        c = __fmul_rn(P.cs_l, __fmul_rn(-f, f));
    }
    gx = __fmul_rn(c, qx);
    gy = __fmul_rn(c, qy);
    gz = __fmul_rn(c, qz);
}

/* Tait EOS p = max(0, k rho0 / gamma ((rho / rho0)^gamma - 1)) (WCSPHSolver.cpp:93)
   with the power in double and rounded once; kr_g = (k rho0) / gamma. */
__device__ __forceinline__ float tait_pressure(float rho, const SimParams& P, float kr_g)
{
    const float ratio = __fdiv_rn(rho, P.rho0);
    const float pw = (float)pow((double)ratio, (double)P.gamma);
    return fmaxf(0.0f, __fmul_rn(kr_g, __fsub_rn(pw, 1.0f)));
}

/* Scalar f with gradW(r) = f * r for 0 < |r| <= h, else 0.
   q <= 1/2: l q (3q - 2) r / (|r| h) = (l / h^2)(3q - 2) r
   q >  1/2: -l (1 - q)^2 r / (|r| h)                                      */
__device__ __forceinline__ float cs_gradf(float rl, float inv_rl, const SimParams& P)
{
    const float q = rl * P.inv_h;
    if (!(rl > 1.0e-9f) || q > 1.0f) return 0.0f;
    if (q <= 0.5f) return P.cs_l_h2 * (3.0f * q - 2.0f);
    const float t = 1.0f - q;
    return -P.cs_l_h * (t * t) * inv_rl;
}

/* |r| and 1/|r| from s = |r|^2 (0 for s == 0). */
__device__ __forceinline__ void len_inv(float s, float& rl, float& inv_rl)
{
    if (s > 0.0f) {
        inv_rl = rsqrtf(s);
        rl = s * inv_rl;
    } else {
        inv_rl = 0.0f;
        rl = 0.0f;
    }
}

/* Akinci cohesion spline (Cohesion.h:20-40). */
__device__ __forceinline__ float cohesion_W(float rl, const SimParams& P)
{
    const float h = P.h;
    if (2.0f * rl > h && rl <= h) {
        const float a = h - rl;
        return P.coh_c1 * (a * a * a) * (rl * rl * rl);
    }
    if (rl > 0.0f && 2.0f * rl <= h) {
        const float a = h - rl;
        return P.coh_c1 * 2.0f * (a * a * a) * (rl * rl * rl) - P.coh_c2;
    }
    return 0.0f;
}

/* Akinci adhesion spline as SPH2O evaluates it (Adhesion.h:18-35): the
   0.007 / h^3.25 coefficient is computed there but never applied, so the
   value is (-4 r^2 / h + 6 r - 2 h)^(1/4) on (h/2, h]. Negative rounding
   residue at the end points is clamped to 0. */
__device__ __forceinline__ float adhesion_W(float rl, const SimParams& P)
{
    const float h = P.h;
    if (2.0f * rl > h && rl <= h) {
        const float v = fmaxf(-4.0f * rl * rl / h + 6.0f * rl - 2.0f * h, 0.0f);
        return sqrtf(sqrtf(v));
    }
    return 0.0f;
}

/* ViscoK Laplacian (ViscoK.h:32-38). */
__device__ __forceinline__ float visco_lapl(float rl, const SimParams& P)
{
    return rl <= P.h ? P.lapl_c * (P.h - rl) : 0.0f;
}

/* ---------------------------------------------------------------------- */
/* Grid: cell key floor(x / h) (HashTable.cpp:5) with IEEE division, shifted
   by the grid origin and clamped; cells stored as 4x4x4 bricks, bricks in x-
   fastest order, cells inside a brick in Morton order.                     */

__device__ __forceinline__ int cell_coord(float x, float h, int cmin, int dim)
{
    const int c = (int)floorf(__fdiv_rn(x, h)) - cmin;
    return min(max(c, 0), dim - 1);
}

/* One scene's cell grid: origin key, extent (x, y, z multiples of 4) and
   the offset of its cells in the global cell table (0 for a single scene;
   batched scenes own disjoint ranges of one table). */
struct Grid {
    int cminx, cminy, cminz;
    int dimx, dimy, dimz;
    int nbx, nby;
    unsigned base;
    int order;                 /* SimParams::cell_order */
};

/* Per-scene constants of a batch. Slots [fbegin, fend) of the sorted fluid
   arrays and [bbegin, bend) of the boundary arrays belong to the scene; the
   sort is scene-major, so these ranges never change. */
struct SceneInfo {
    Grid grid;
    float visc, bvisc;
    unsigned fbegin, fend, bbegin, bend;
};

/* Per-scene solver state of a batch (the per-scene part of DevState). */
struct SceneState {
    double time, avg_dens, avg_div;
    float dt, dt_next, last_vmax;
    unsigned vmax_bits, its, its_v, steps, active;
    unsigned long long sum_its, sum_its_v;
};

__device__ __forceinline__ Grid grid_single(const SimParams& P)
{
    Grid g;
    g.cminx = P.cminx; g.cminy = P.cminy; g.cminz = P.cminz;
    g.dimx = P.dimx; g.dimy = P.dimy; g.dimz = P.dimz;
    g.nbx = P.nbx; g.nby = P.nby;
    g.base = 0u;
    g.order = P.cell_order;
    return g;
}

/* Cell index of (cx, cy, cz): 4 x 4 x 4 bricks in x-fastest order with
   Morton order inside a brick (order 0), or plain x-fastest (order 1). */
__device__ __forceinline__ unsigned brick_morton(int cx, int cy, int cz, const Grid& g)
{
    if (g.order == 1)
        return g.base + ((unsigned)cz * (unsigned)g.dimy + (unsigned)cy) * (unsigned)g.dimx + (unsigned)cx;
    const unsigned lx = (unsigned)cx & 3u, ly = (unsigned)cy & 3u, lz = (unsigned)cz & 3u;
    const unsigned m = (lx & 1u) | ((ly & 1u) << 1) | ((lz & 1u) << 2) | ((lx & 2u) << 2) |
                       ((ly & 2u) << 3) | ((lz & 2u) << 4);
    const unsigned b = ((unsigned)(cz >> 2) * (unsigned)g.nby + (unsigned)(cy >> 2)) * (unsigned)g.nbx +
                       (unsigned)(cx >> 2);
    return g.base + ((b << 6) | m);
}

__device__ __forceinline__ unsigned cell_index(float4 x, float h, const Grid& g)
{
    return brick_morton(cell_coord(x.x, h, g.cminx, g.dimx), cell_coord(x.y, h, g.cminy, g.dimy),
                        cell_coord(x.z, h, g.cminz, g.dimz), g);
}

/* Calls f(c) for the existing cells among the 27 around x's cell, in the
   reference's offset order (x outermost, z innermost; HashTable.cpp:59-65). */
template <typename F>
__device__ __forceinline__ void for_cells27(float4 x, float h, const Grid& g, F&& f)
{
    const int cx = cell_coord(x.x, h, g.cminx, g.dimx);
    const int cy = cell_coord(x.y, h, g.cminy, g.dimy);
    const int cz = cell_coord(x.z, h, g.cminz, g.dimz);
    for (int dx = -1; dx <= 1; ++dx) {
        const int xx = cx + dx;
        if (xx < 0 || xx >= g.dimx) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int yy = cy + dy;
            if (yy < 0 || yy >= g.dimy) continue;
            for (int dz = -1; dz <= 1; ++dz) {
                const int zz = cz + dz;
                if (zz < 0 || zz >= g.dimz) continue;
                f(brick_morton(xx, yy, zz, g));
            }
        }
    }
}

/* Scene table of a batch (both NULL for a single scene). */
struct SceneRef {
    const SceneInfo* scenes;
    const unsigned* scene_of;   /* scene of each sorted slot */
};

__device__ __forceinline__ Grid grid_for(const SimParams& P, const SceneRef& S, unsigned slot)
{
    return S.scenes ? S.scenes[S.scene_of[slot]].grid : grid_single(P);
}

/* Largest float s with sqrt_rn(s) <= h. The correctly rounded square root
   is monotonic, so the reference's neighbour test glm::length(r) <= h,
   sqrt_rn((dx dx + dy dy) + dz dz) <= h, holds exactly when that rounded
   sum is <= this bound (NaN and infinity fail both forms). The host's
   sqrtf is the IEEE correctly rounded one, as __fsqrt_rn is. */
static inline float sqrt_le_bound(float h)
{
    float s = h * h;
    while (s > 0.0f && std::sqrt(s) > h) s = std::nextafter(s, 0.0f);
    while (std::sqrt(std::nextafter(s, INFINITY)) <= h) s = std::nextafter(s, INFINITY);
    return s;
}

/* Entry kk of sorted particle i's neighbour list (column-major). The lists
   are streamed once per pass and at 1M particles are larger than the L2, so
   they are loaded with the evict-first hint (ld.global.cs): they must not
   push out of L2 the particle state that the neighbour gathers read. */
__device__ __forceinline__ unsigned list_at(const unsigned* list, unsigned kk, size_t nf, int i)
{
    return __ldcs(list + kk * nf + i);
}

/* ---------------------------------------------------------------------- */
/* Reductions                                                               */

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_max(float v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

/* Block-wide sum; result valid in thread 0. `scratch` holds >= 32 doubles. */
__device__ __forceinline__ double block_sum(double v, double* scratch)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        t = lane < nw ? scratch[lane] : 0.0;
        t = warp_sum(t);
    }
    return t;
}

__device__ __forceinline__ float block_max(float v, float* scratch)
{
    v = warp_max(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    float t = 0.0f;
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        t = lane < nw ? scratch[lane] : 0.0f;
        t = warp_max(t);
    }
    return t;
}

/* ---------------------------------------------------------------------- */
/* gpu-scope acquire load, acquire-release add and release store (PTX memory
   model). A barrier built from plain loads and __threadfence() does not stop
   an SM's L1 from serving lines it cached before the barrier, so values other
   SMs wrote in between could be read stale; an acquire at gpu scope makes
   them visible to the acquiring thread, and through bar.sync to its block. */
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

/* Grid-wide barrier for cooperative (co-resident) launches. Each block's
   thread 0 arrives with an acquire-release add (releasing its block's
   writes, ordered by the preceding __syncthreads), the last arrival resets
   the count and publishes the next generation with a release store, and the
   waiters spin on an acquire load of the generation: every block sees every
   other block's writes from before the barrier. The wait is bounded: after
   kSpinLimit polls the block records ERRBIT_TIMEOUT and returns false, and
   the caller leaves the kernel. */
__device__ __forceinline__ bool grid_barrier(DevState* st)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned g = ld_acquire_gpu(&st->bar_gen);
        const unsigned arrived = atom_add_acq_rel_gpu(&st->bar_count, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(&st->bar_count, 0u);
            st_release_gpu(&st->bar_gen, g + 1u);
        } else {
            unsigned long long spins = 0;
            while (ld_acquire_gpu(&st->bar_gen) == g) {
                __nanosleep(256);
                if (++spins > kSpinLimit) {
                    atomicOr(&st->err, ERRBIT_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        s_ok = ok && ((ld_acquire_gpu(reinterpret_cast<const unsigned*>(&st->err)) & ERRBIT_TIMEOUT) == 0);
    }
    __syncthreads();
    return s_ok != 0;
}

/* ---------------------------------------------------------------------- */
/* PCISPH boundary method helpers, in the reference's float operation order. */

/* glm::length: sqrt((x x + y y) + z z) */
__device__ __forceinline__ float glm_length(float x, float y, float z)
{
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}

/* Poly6::W (Poly6.h:29-42): |r| squared after the square root, as written */
__device__ __forceinline__ float poly6_W(float rx, float ry, float rz, const SimParams& P)
{
    const float m = glm_length(rx, ry, rz);
    const float m2 = __fmul_rn(m, m);
    if (!(m2 <= P.h2)) return 0.0f;
    const float d = __fsub_rn(P.h2, m2);
    return __fmul_rn(__fmul_rn(__fmul_rn(P.poly6_c, d), d), d);
}

/* Spiky::gradW (Spiky.h:44-55): (-c (h - |r|)^2 / |r|) r */
__device__ __forceinline__ void spiky_gradW(float rx, float ry, float rz, const SimParams& P, float& gx, float& gy,
                                            float& gz)
{
    const float m = glm_length(rx, ry, rz);
    if (m != 0.0f && m <= P.h) {
        const float d = __fsub_rn(P.h, m);
        const float s = __fdiv_rn(__fmul_rn(__fmul_rn(-P.spiky_g, d), d), m);
        gx = __fmul_rn(s, rx);
        gy = __fmul_rn(s, ry);
        gz = __fmul_rn(s, rz);
    } else {
        gx = gy = gz = 0.0f;
    }
}

/* Whether the reference's hash table held a candidate list for cell c at
   the last neighbour search. Its table keeps every cell ever touched (by an
   insertion or by a lookup, HashTable.cpp:88-96) and computes lists for all
   of them at each search (:23-86); a lookup of a cell first touched since
   then finds empty lists. entry[c] is the search that first listed c (0:
   never touched); a lookup of an untouched cell marks it for the next one. */
__device__ __forceinline__ bool cell_listed(unsigned* entry, unsigned c, unsigned epoch)
{
    const unsigned e = entry[c];
    if (e != 0u) return e <= epoch;
    atomicCAS(&entry[c], 0u, epoch + 1u);
    return false;
}

} // namespace sph

#endif
