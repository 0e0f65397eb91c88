/*
 * Neighbour search on the GPU: the B200 replacement of SPH2O's spatial hash
 * (HashTable::insertFluidParticle / neighborhoodSearch, src/SPH2O/HashTable.cpp:3-86;
 * SPHSolver::insertFluidParticles / neighborhoodSearch, src/SPH2O/SPHSolver/SPHSolver.cpp:170-219).
 *
 * Per step:
 *   1. ns_count        cell key floor(x / h) -> brick-Morton cell index,
 *                      per-cell population by atomicAdd (slot = old count)
 *   2. scan_local/add  exclusive scan of the populations -> cellStart[ncells+1]
 *                      (the scan zeroes the populations for the next step)
 *   3. ns_scatter      (orig id, source index) into its cell segment
 *   4. ns_rank_gather  rank inside the cell by orig id (deterministic, equal
 *                      to the reference's insertion order: ascending index),
 *                      then gather the carried state into sorted order
 *   5. ns_build_lists  for each particle, the 27 cells in the reference's
 *                      offset order (x outermost, HashTable.cpp:59-65), keep
 *                      candidates with |xi - xj| <= h (exact IEEE test), in
 *                      column-major neighbour lists (optionally one block
 *                      per cell brick with the brick's halo staged in
 *                      shared memory: k_ns_build_lists_staged, same lists)
 * The static boundary is sorted once at init with steps 1-4 into its own
 * cellStart table, and AkinciBoundaryObject::computeVolume
 * (src/SPH2O/BoundaryObject/AkinciBoundaryObject.cpp:10-34) runs on it.
 */
#include "sph_device.cuh"
#include "sph_grid_body.cuh"
#include "sph_internal.h"

namespace sph {

__global__ void __launch_bounds__(256) k_ns_count(SimParams P, SceneRef S, int n, const unsigned* n_dev,
                                                  const float4* __restrict__ pos, unsigned* __restrict__ cell_count,
                                                  unsigned* __restrict__ cell_of, unsigned* __restrict__ slot)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (n_dev ? (int)*n_dev : n)) return;
    ns_count_at(P, S, i, pos, cell_count, cell_of, slot);
}

/* Exclusive scan, phase 1: each 256-thread block scans 4096 populations (16
   per thread, four 16-byte loads in flight), writes block-local exclusive
   offsets and zeroes the populations. */
__global__ void __launch_bounds__(256) k_scan_local(unsigned* __restrict__ count, unsigned* __restrict__ start,
                                                    unsigned* __restrict__ block_sums)
{
    __shared__ unsigned warp_tot[8];
    const size_t base = (size_t)blockIdx.x * 4096 + (size_t)threadIdx.x * 16;
    uint4 c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = *reinterpret_cast<const uint4*>(count + base + 4 * k);
#pragma unroll
    for (int k = 0; k < 4; ++k) *reinterpret_cast<uint4*>(count + base + 4 * k) = make_uint4(0, 0, 0, 0);
    unsigned t = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) t += (c[k].x + c[k].y) + (c[k].z + c[k].w);
    unsigned incl = t;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const unsigned w = lane < 8 ? warp_tot[lane] : 0u;
        unsigned wi = w;
        for (int o = 1; o < 8; o <<= 1) {
            const unsigned v = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += v;
        }
        if (lane < 8) warp_tot[lane] = wi - w;
        if (lane == 7) block_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    unsigned run = warp_tot[wid] + incl - t;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint4 o;
        o.x = run; run += c[k].x;
        o.y = run; run += c[k].y;
        o.z = run; run += c[k].z;
        o.w = run; run += c[k].w;
        *reinterpret_cast<uint4*>(start + base + 4 * k) = o;
    }
}

/* Phase 2: each block adds to its chunk the totals of all chunks before it
   (summed by the block itself, so the chunk totals need no scan of their
   own), and the last block writes the grand total. */
__global__ void __launch_bounds__(1024) k_scan_add(unsigned* __restrict__ start,
                                                   const unsigned* __restrict__ block_sums, int nblocks,
                                                   unsigned* __restrict__ total_out)
{
    __shared__ unsigned warp_tot[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned v = 0;
    for (int k = threadIdx.x; k < (int)blockIdx.x; k += 1024) v += block_sums[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        unsigned w = warp_tot[lane];
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (lane == 0) warp_tot[0] = w;
    }
    __syncthreads();
    const unsigned off = warp_tot[0];
    if ((int)blockIdx.x == nblocks - 1 && threadIdx.x == 0) *total_out = off + block_sums[blockIdx.x];
    const size_t base = (size_t)blockIdx.x * 4096 + (size_t)threadIdx.x * 4;
    uint4 s = *reinterpret_cast<uint4*>(start + base);
    s.x += off; s.y += off; s.z += off; s.w += off;
    *reinterpret_cast<uint4*>(start + base) = s;
}

__global__ void __launch_bounds__(256) k_ns_scatter(int n, const unsigned* n_dev, const unsigned* __restrict__ cell_of,
                                                    const unsigned* __restrict__ slot,
                                                    const unsigned* __restrict__ cell_start,
                                                    const unsigned* __restrict__ orig,
                                                    unsigned* __restrict__ tmp_key, unsigned* __restrict__ tmp_src)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (n_dev ? (int)*n_dev : n)) return;
    ns_scatter_at(i, cell_of, slot, cell_start, orig, tmp_key, tmp_src);
}

/* Rank inside the cell by caller-order id, then move the carried state. */
__global__ void __launch_bounds__(256) k_ns_rank_gather(int n, const unsigned* __restrict__ cell_of,
                                                        const unsigned* __restrict__ cell_start,
                                                        const unsigned* __restrict__ tmp_key,
                                                        const unsigned* __restrict__ tmp_src, GatherSet g)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (g.n_dev ? (int)*g.n_dev : n)) return;
    ns_rank_gather_at(p, cell_of, cell_start, tmp_key, tmp_src, g);
}

/* Neighbour lists in the reference's candidate order, filtered at |r| <= h. */
__device__ __forceinline__ void build_lists_at(const SimParams& P, const SceneRef& S, int i,
                                               const float4* __restrict__ pos,
                                               const unsigned* __restrict__ cell_start,
                                               const float4* __restrict__ bpos,
                                               const unsigned* __restrict__ bcell_start,
                                               unsigned* __restrict__ nbr_f, unsigned* __restrict__ cnt_f,
                                               unsigned* __restrict__ nbr_b, unsigned* __restrict__ cnt_b,
                                               DevState* st)
{
    const float4 xi = pos[i];
    const size_t nf = (size_t)P.nf;
    /* |r| <= h as the reference rounds it, without the square root */
    const float s2max = P.h2_exact;
    unsigned nF = 0, nB = 0;
    for_cells27(xi, P.h, grid_for(P, S, (unsigned)i), [&](unsigned c) {
        const unsigned s = cell_start[c], e = cell_start[c + 1];
        for (unsigned q = s; q < e; ++q) {
            if (dist2_exact(xi, pos[q]) <= s2max) {
                if (nF < P.capF) __stcs(nbr_f + (size_t)nF * nf + i, q);
                ++nF;
            }
        }
        if (P.nb > 0) {
            const unsigned bs = bcell_start[c], be = bcell_start[c + 1];
            for (unsigned q = bs; q < be; ++q) {
                if (dist2_exact(xi, bpos[q]) <= s2max) {
                    if (nB < P.capB) __stcs(nbr_b + (size_t)nB * nf + i, q);
                    ++nB;
                }
            }
        }
    });
    cnt_f[i] = min(nF, P.capF);
    cnt_b[i] = min(nB, P.capB);
    if (nF > P.capF || nB > P.capB) {
        atomicAdd(&st->overflow, 1u);
        atomicOr(&st->err, ERRBIT_OVERFLOW);
    }
}

__global__ void __launch_bounds__(128) k_ns_build_lists(SimParams P, SceneRef S, const float4* __restrict__ pos,
                                                        const unsigned* __restrict__ cell_start,
                                                        const float4* __restrict__ bpos,
                                                        const unsigned* __restrict__ bcell_start,
                                                        unsigned* __restrict__ nbr_f, unsigned* __restrict__ cnt_f,
                                                        unsigned* __restrict__ nbr_b, unsigned* __restrict__ cnt_b,
                                                        DevState* st)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= active_n(P, st)) return;
    build_lists_at(P, S, i, pos, cell_start, bpos, bcell_start, nbr_f, cnt_f, nbr_b, cnt_b, st);
}

/* ---------------------------------------------------------------------- */
/* List build with each brick's halo staged in shared memory.               */

/* the global-memory walk of one particle of a single scene, kept out of line */
__device__ __noinline__ void build_lists_global(const SimParams& P, int i, const float4* __restrict__ pos,
                                                const unsigned* __restrict__ cell_start,
                                                const float4* __restrict__ bpos,
                                                const unsigned* __restrict__ bcell_start,
                                                unsigned* __restrict__ nbr_f, unsigned* __restrict__ cnt_f,
                                                unsigned* __restrict__ nbr_b, unsigned* __restrict__ cnt_b,
                                                DevState* st)
{
    build_lists_at(P, SceneRef{}, i, pos, cell_start, bpos, bcell_start, nbr_f, cnt_f, nbr_b, cnt_b, st);
}

/* Fluid particles of one brick's 6 x 6 x 6-cell halo that fit in shared
   memory (45 KB of float4); a brick with more takes the cells from global
   memory instead. */
constexpr unsigned kHaloCap = 2816;
constexpr int kStagedBlock = 256;

/* One block per 4 x 4 x 4-cell brick (single scenes in brick order). The
   block lists the 216 cells around the brick with their fluid and boundary
   ranges, lays the fluid cells' positions end to end in shared memory (one
   warp per cell, coalesced), then every thread walks its particles' 27 cells
   in the reference's offset order over the staged copies: the same
   candidates in the same order, the same exact test, the same global slot
   ids written, so the lists equal k_ns_build_lists's entry for entry. */
__global__ void __launch_bounds__(kStagedBlock) k_ns_build_lists_staged(
    SimParams P, const float4* __restrict__ pos, const unsigned* __restrict__ cell_start,
    const float4* __restrict__ bpos, const unsigned* __restrict__ bcell_start, unsigned* __restrict__ nbr_f,
    unsigned* __restrict__ cnt_f, unsigned* __restrict__ nbr_b, unsigned* __restrict__ cnt_b, DevState* st)
{
    __shared__ float4 s_pos[kHaloCap];
    __shared__ unsigned s_off[217]; /* staged offset of each halo cell; [216] = total */
    __shared__ unsigned s_gs[216];  /* global slot of each halo cell's first fluid particle */
    __shared__ unsigned s_bs[216], s_be[216];
    const Grid g = grid_single(P);
    const unsigned b = blockIdx.x;
    const unsigned c0 = b << 6;
    const unsigned ps = cell_start[c0], pe = cell_start[c0 + 64];
    if (ps == pe) return; /* the whole block leaves */
    const int bx = (int)(b % (unsigned)g.nbx), by = (int)((b / (unsigned)g.nbx) % (unsigned)g.nby);
    const int bz = (int)(b / ((unsigned)g.nbx * (unsigned)g.nby));
    const int lane = (int)(threadIdx.x & 31u), warp = (int)(threadIdx.x >> 5);
    for (int h = (int)threadIdx.x; h < 216; h += kStagedBlock) {
        const int cx = 4 * bx - 1 + h % 6, cy = 4 * by - 1 + (h / 6) % 6, cz = 4 * bz - 1 + h / 36;
        unsigned s = 0, e = 0, bs = 0, be = 0;
        if (cx >= 0 && cx < g.dimx && cy >= 0 && cy < g.dimy && cz >= 0 && cz < g.dimz) {
            const unsigned c = brick_morton(cx, cy, cz, g);
            s = cell_start[c];
            e = cell_start[c + 1];
            if (P.nb > 0) {
                bs = bcell_start[c];
                be = bcell_start[c + 1];
            }
        }
        s_gs[h] = s;
        s_off[h] = e - s; /* the population until the scan below */
        s_bs[h] = bs;
        s_be[h] = be;
    }
    __syncthreads();
    if (warp == 0) {
        /* exclusive scan of the 216 populations: 7 consecutive cells per lane */
        unsigned v[7], t = 0;
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            const int h = 7 * lane + k;
            v[k] = h < 216 ? s_off[h] : 0u;
            t += v[k];
        }
        unsigned incl = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        unsigned run = incl - t;
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            const int h = 7 * lane + k;
            if (h <= 216) s_off[h] = run;
            run += v[k];
        }
    }
    __syncthreads();
    const bool staged = s_off[216] <= kHaloCap;
    if (staged)
        for (int h = warp; h < 216; h += kStagedBlock / 32) {
            const unsigned s = s_gs[h], o = s_off[h], n = s_off[h + 1] - o;
            for (unsigned k = (unsigned)lane; k < n; k += 32u) s_pos[o + k] = pos[s + k];
        }
    __syncthreads();
    const size_t nf = (size_t)P.nf;
    const float s2max = P.h2_exact;
    for (unsigned i = ps + threadIdx.x; i < pe; i += kStagedBlock) {
        const float4 xi = pos[i];
        /* the particle's cell inside the brick (its sort cell) */
        const int lx = cell_coord(xi.x, P.h, g.cminx, g.dimx) - 4 * bx;
        const int ly = cell_coord(xi.y, P.h, g.cminy, g.dimy) - 4 * by;
        const int lz = cell_coord(xi.z, P.h, g.cminz, g.dimz) - 4 * bz;
        if ((unsigned)lx > 3u || (unsigned)ly > 3u || (unsigned)lz > 3u) {
            /* moved out of its sort cell's brick since the sort: walk the
               cells around its position in global memory */
            build_lists_global(P, (int)i, pos, cell_start, bpos, bcell_start, nbr_f, cnt_f, nbr_b, cnt_b, st);
            continue;
        }
        unsigned nF = 0, nB = 0;
        /* x outermost, z innermost (HashTable.cpp:59-65); cells outside the
           grid have empty ranges */
        for (int dx = 0; dx < 3; ++dx)
            for (int dy = 0; dy < 3; ++dy)
                for (int dz = 0; dz < 3; ++dz) {
                    const int h = (lz + dz) * 36 + (ly + dy) * 6 + (lx + dx);
                    const unsigned o = s_off[h], n = s_off[h + 1] - o, s = s_gs[h];
                    for (unsigned k = 0; k < n; ++k) {
                        const float4 xq = staged ? s_pos[o + k] : pos[s + k];
                        if (dist2_exact(xi, xq) <= s2max) {
                            if (nF < P.capF) __stcs(nbr_f + (size_t)nF * nf + i, s + k);
                            ++nF;
                        }
                    }
                    for (unsigned q = s_bs[h]; q < s_be[h]; ++q) {
                        if (dist2_exact(xi, bpos[q]) <= s2max) {
                            if (nB < P.capB) __stcs(nbr_b + (size_t)nB * nf + i, q);
                            ++nB;
                        }
                    }
                }
        cnt_f[i] = min(nF, P.capF);
        cnt_b[i] = min(nB, P.capB);
        if (nF > P.capF || nB > P.capB) {
            atomicAdd(&st->overflow, 1u);
            atomicOr(&st->err, ERRBIT_OVERFLOW);
        }
    }
}

__global__ void __launch_bounds__(128) k_ns_build_lists_warp(SimParams P, SceneRef S,
                                                             const float4* __restrict__ pos,
                                                             const unsigned* __restrict__ cell_start,
                                                             const float4* __restrict__ bpos,
                                                             const unsigned* __restrict__ bcell_start,
                                                             unsigned* __restrict__ nbr_f, unsigned* __restrict__ cnt_f,
                                                             unsigned* __restrict__ nbr_b, unsigned* __restrict__ cnt_b,
                                                             DevState* st)
{
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    /* the whole warp shares i and leaves together */
    if (i >= active_n(P, st)) return;
    build_lists_warp_at(P, S, i, pos, cell_start, bpos, bcell_start, nbr_f, cnt_f, nbr_b, cnt_b, st);
}

/* Akinci boundary volume V_b = 1 / sum_b' W(x_b - x_b') over the 27 cells
   (AkinciBoundaryObject.cpp:10-34); k_boundary_psi then stores
   psi = rho0 V_b in bpos.w for the fluid kernels. */
__global__ void __launch_bounds__(128) k_boundary_volume(SimParams P, SceneRef S, const float4* __restrict__ bpos,
                                                         const unsigned* __restrict__ bcell_start,
                                                         float* __restrict__ bvol)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= P.nb) return;
    const float4 xb = bpos[b];
    float delta = 0.0f;
    for_cells27(xb, P.h, grid_for(P, S, (unsigned)b), [&](unsigned c) {
        for (unsigned q = bcell_start[c]; q < bcell_start[c + 1]; ++q) {
            const float s2 = dist2_exact(xb, bpos[q]);
            if (s2 <= P.h2_guard) delta = __fadd_rn(delta, cs_W_exact(s2, P));
        }
    });
    bvol[b] = __fdiv_rn(1.0f, delta);
}

__global__ void __launch_bounds__(256) k_boundary_psi(SimParams P, float4* __restrict__ bpos,
                                                      const float* __restrict__ bvol)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < P.nb) bpos[b].w = __fmul_rn(P.rho0, bvol[b]);
}

/* out[orig[i]] = in[i]: sorted order -> caller order */
__global__ void k_unsort_v4(int n, const unsigned* __restrict__ orig, const float4* __restrict__ in,
                            float* __restrict__ out3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = in[i];
    const size_t o = (size_t)orig[i] * 3;
    out3[o] = v.x;
    out3[o + 1] = v.y;
    out3[o + 2] = v.z;
}

__global__ void k_unsort_f(int n, const unsigned* __restrict__ orig, const float* __restrict__ in,
                           float* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[orig[i]] = in[i];
}

/* caller order -> sorted slots (set_state between steps) */
__global__ void k_sort_v3(int n, const unsigned* __restrict__ orig, const float* __restrict__ in3,
                          float4* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t o = (size_t)orig[i] * 3;
    out[i] = make_float4(in3[o], in3[o + 1], in3[o + 2], 0.0f);
}

__global__ void k_pack_v3(int n, const float* __restrict__ in3, float4* __restrict__ out, float w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4(in3[3 * (size_t)i], in3[3 * (size_t)i + 1], in3[3 * (size_t)i + 2], w);
}

__global__ void k_iota(int n, unsigned* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (unsigned)i;
}

static inline int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

void launch_sort(const SimParams& P, const SceneRef& S, int n, const float4* pos_for_keys, unsigned* cell_count,
                 unsigned* cell_start,
                 unsigned* block_sums, unsigned* cell_of, unsigned* slot, unsigned* tmp_key, unsigned* tmp_src,
                 const unsigned* orig_in, const GatherSet& g, cudaStream_t s)
{
    if (n <= 0) {
        /* an empty set still needs an all-zero start table */
        cudaMemsetAsync(cell_start, 0, ((size_t)P.ncells + 1) * sizeof(unsigned), s);
        return;
    }
    k_ns_count<<<blocks_for(n, 256), 256, 0, s>>>(P, S, n, g.n_dev, pos_for_keys, cell_count, cell_of, slot);
    const int nblk = (int)(P.ncells / 4096);
    k_scan_local<<<nblk, 256, 0, s>>>(cell_count, cell_start, block_sums);
    k_scan_add<<<nblk, 1024, 0, s>>>(cell_start, block_sums, nblk, cell_start + P.ncells);
    k_ns_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, g.n_dev, cell_of, slot, cell_start, orig_in, tmp_key, tmp_src);
    k_ns_rank_gather<<<blocks_for(n, 256), 256, 0, s>>>(n, cell_of, cell_start, tmp_key, tmp_src, g);
}

void launch_build_lists(const SimParams& P, const SceneRef& S, const float4* pos, const unsigned* cell_start,
                        const float4* bpos,
                        const unsigned* bcell_start, unsigned* nbr_f, unsigned* cnt_f, unsigned* nbr_b,
                        unsigned* cnt_b, DevState* st, cudaStream_t s, bool staged)
{
    if (P.nf <= 0) return;
    if (staged && !S.scenes && P.cell_order == 0 && P.nf >= (1 << 16)) {
        /* one block per brick; bricks without fluid leave at once */
        const int nbricks = P.nbx * P.nby * (P.dimz / 4);
        k_ns_build_lists_staged<<<nbricks, kStagedBlock, 0, s>>>(P, pos, cell_start, bpos, bcell_start, nbr_f, cnt_f,
                                                                  nbr_b, cnt_b, st);
        return;
    }
    /* A warp per particle below 2^16 particles, where one lane's serial walk
       over ~216 candidates is the critical path (32k: 32 vs 56 us per build);
       one lane per particle above, where the particles fill the GPU and the
       warp's extra instructions cost more (125k: 0.069 vs 0.096 ms). */
    if (P.nf < (1 << 16))
        k_ns_build_lists_warp<<<blocks_for((long long)P.nf * 32, 128), 128, 0, s>>>(
            P, S, pos, cell_start, bpos, bcell_start, nbr_f, cnt_f, nbr_b, cnt_b, st);
    else
        k_ns_build_lists<<<blocks_for(P.nf, 128), 128, 0, s>>>(P, S, pos, cell_start, bpos, bcell_start, nbr_f,
                                                                cnt_f, nbr_b, cnt_b, st);
}

void launch_boundary_volume(const SimParams& P, const SceneRef& S, float4* bpos, const unsigned* bcell_start,
                            float* bvol, cudaStream_t s)
{
    if (P.nb <= 0) return;
    k_boundary_volume<<<blocks_for(P.nb, 128), 128, 0, s>>>(P, S, bpos, bcell_start, bvol);
    k_boundary_psi<<<blocks_for(P.nb, 256), 256, 0, s>>>(P, bpos, bvol);
}

void launch_unsort_v4(int n, const unsigned* orig, const float4* in, float* out3, cudaStream_t s)
{
    if (n > 0) k_unsort_v4<<<blocks_for(n, 256), 256, 0, s>>>(n, orig, in, out3);
}
void launch_unsort_f(int n, const unsigned* orig, const float* in, float* out, cudaStream_t s)
{
    if (n > 0) k_unsort_f<<<blocks_for(n, 256), 256, 0, s>>>(n, orig, in, out);
}
void launch_sort_v3(int n, const unsigned* orig, const float* in3, float4* out, cudaStream_t s)
{
    if (n > 0) k_sort_v3<<<blocks_for(n, 256), 256, 0, s>>>(n, orig, in3, out);
}
void launch_pack_v3(int n, const float* in3, float4* out, float w, cudaStream_t s)
{
    if (n > 0) k_pack_v3<<<blocks_for(n, 256), 256, 0, s>>>(n, in3, out, w);
}
void launch_iota(int n, unsigned* out, cudaStream_t s)
{
    if (n > 0) k_iota<<<blocks_for(n, 256), 256, 0, s>>>(n, out);
}

/* Cells of n particles listed by the search now completing: entry = the
   completed searches + 1 where still 0 (single-scene grids). */
__global__ void __launch_bounds__(256) k_mark_entries(SimParams P, const float4* __restrict__ pos, int n,
                                                      const unsigned* n_dev, unsigned* entry, const DevState* st)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (n_dev ? (int)*n_dev : n)) return;
    const unsigned c = cell_index(pos[i], P.h, grid_single(P));
    if (entry[c] == 0u) atomicCAS(&entry[c], 0u, st->ns_epoch + 1u);
}

__global__ void k_epoch_advance(DevState* st) { st->ns_epoch += 1u; }

void launch_mark_entries(const SimParams& P, const float4* pos, int n, const unsigned* n_dev, unsigned* entry,
                         DevState* st, bool advance, cudaStream_t s)
{
    if (n > 0) k_mark_entries<<<(n + 255) / 256, 256, 0, s>>>(P, pos, n, n_dev, entry, st);
    if (advance) k_epoch_advance<<<1, 1, 0, s>>>(st);
}

} // namespace sph
