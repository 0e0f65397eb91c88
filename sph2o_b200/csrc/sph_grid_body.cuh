/*
 * Per-particle bodies of the neighbour search (sph_grid.cu): the counting
 * sort's count, scatter and rank + gather steps and the small-scene list
 * build (a warp per particle), kept apart from their kernels (one thread or
 * warp per index) so that other kernels can run the same steps on their own
 * index ranges, and the GatherSet the sort moves state with.
 */
#ifndef SPH2O_GRID_BODY_CUH
#define SPH2O_GRID_BODY_CUH

#include "sph_device.cuh"

namespace sph {

/* Arrays moved by the rank/gather step of the sort (NULL entries skipped).
   n_dev (may be NULL): device count of the particles to sort, read by the
   kernels in place of n (the fluid's active count when emitters add to it). */
struct GatherSet {
    const unsigned* n_dev;
    unsigned* orig_out;
    unsigned* cell_out;
    const float4* v4_in[4];
    float4* v4_out[4];
    const float* f_in[2];
    float* f_out[2];
};

/* cell of particle i and its arrival slot in that cell */
__device__ __forceinline__ void ns_count_at(const SimParams& P, const SceneRef& S, int i, const float4* __restrict__ pos,
                                            unsigned* __restrict__ cell_count, unsigned* __restrict__ cell_of,
                                            unsigned* __restrict__ slot)
{
    const unsigned c = cell_index(pos[i], P.h, grid_for(P, S, (unsigned)i));
    cell_of[i] = c;
    slot[i] = atomicAdd(&cell_count[c], 1u);
}

/* (orig id, source index) of particle i into its cell segment */
__device__ __forceinline__ void ns_scatter_at(int i, const unsigned* __restrict__ cell_of,
                                              const unsigned* __restrict__ slot, const unsigned* __restrict__ cell_start,
                                              const unsigned* __restrict__ orig, unsigned* __restrict__ tmp_key,
                                              unsigned* __restrict__ tmp_src)
{
    const unsigned p = cell_start[cell_of[i]] + slot[i];
    tmp_key[p] = orig[i];
    tmp_src[p] = (unsigned)i;
}

/* Rank of segment entry p inside its cell by caller-order id (the
   reference's insertion order), then the carried state moved there. */
__device__ __forceinline__ void ns_rank_gather_at(int p, const unsigned* __restrict__ cell_of,
                                                  const unsigned* __restrict__ cell_start,
                                                  const unsigned* __restrict__ tmp_key,
                                                  const unsigned* __restrict__ tmp_src, const GatherSet& g)
{
    const unsigned src = tmp_src[p];
    /* the carried position and velocity are loaded before the cell lookup
       and the rank loop, so their latency overlaps that chain */
    const float4 v0 = g.v4_in[0] ? g.v4_in[0][src] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float4 v1 = g.v4_in[1] ? g.v4_in[1][src] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const unsigned c = cell_of[src];
    const unsigned key = tmp_key[p];
    const unsigned s = cell_start[c], e = cell_start[c + 1];
    unsigned rank = 0;
    for (unsigned q = s; q < e; ++q) rank += tmp_key[q] < key ? 1u : 0u;
    const unsigned dst = s + rank;
    g.orig_out[dst] = key;
    if (g.cell_out) g.cell_out[dst] = c;
    if (g.v4_in[0]) g.v4_out[0][dst] = v0;
    if (g.v4_in[1]) g.v4_out[1][dst] = v1;
    if (g.v4_in[2]) g.v4_out[2][dst] = g.v4_in[2][src];
    if (g.v4_in[3]) g.v4_out[3][dst] = g.v4_in[3][src];
    if (g.f_in[0]) g.f_out[0][dst] = g.f_in[0][src];
    if (g.f_in[1]) g.f_out[1][dst] = g.f_in[1][src];
}

/* The same lists for small scenes, one warp per particle: lane k < 27 loads
   the range of the particle's k-th cell (the reference's offset order), a
   warp scan lays the 27 ranges end to end, and the warp then tests the
   concatenated candidates 32 at a time; a ballot ranks each round's accepted
   candidates, so entries are written in candidate order. The serial walk of a
   particle shrinks from ~216 candidates (or 27 cells) to ~7 rounds. */
__device__ __forceinline__ void warp_candidates(const float4* __restrict__ xs, unsigned s, unsigned e, float4 xi,
                                                float s2max, unsigned lane, unsigned cap, unsigned* __restrict__ list,
                                                size_t nf, int i, unsigned& n)
{
    const unsigned cnt = e - s;
    unsigned incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += v;
    }
    const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
    const unsigned excl = incl - cnt;
    for (unsigned u0 = 0; u0 < total; u0 += 32) {
        const unsigned u = min(u0 + lane, total - 1u);
        /* cell of candidate u: the number of lanes whose ranges end at or before u */
        unsigned k = 0;
#pragma unroll
        for (unsigned step = 16; step >= 1; step >>= 1)
            if (__shfl_sync(0xffffffffu, incl, k + step - 1) <= u) k += step;
        const unsigned q = __shfl_sync(0xffffffffu, s, k) + (u - __shfl_sync(0xffffffffu, excl, k));
        const bool in = u0 + lane < total && dist2_exact(xi, xs[q]) <= s2max;
        const unsigned bits = __ballot_sync(0xffffffffu, in);
        if (in) {
            const unsigned r = n + __popc(bits & ((1u << lane) - 1u));
            if (r < cap) __stcs(list + (size_t)r * nf + i, q);
        }
        n += __popc(bits);
    }
}

/* The lists of particle i, built by the whole warp (every lane calls with
   the same i). */
__device__ __forceinline__ void build_lists_warp_at(const SimParams& P, const SceneRef& S, int i,
                                                    const float4* __restrict__ pos,
                                                    const unsigned* __restrict__ cell_start,
                                                    const float4* __restrict__ bpos,
                                                    const unsigned* __restrict__ bcell_start,
                                                    unsigned* __restrict__ nbr_f, unsigned* __restrict__ cnt_f,
                                                    unsigned* __restrict__ nbr_b, unsigned* __restrict__ cnt_b,
                                                    DevState* st)
{
    const unsigned lane = threadIdx.x & 31u;
    const float4 xi = pos[i];
    const Grid g = grid_for(P, S, (unsigned)i);
    unsigned s = 0, e = 0, bs = 0, be = 0;
    if (lane < 27) {
        const int xx = cell_coord(xi.x, P.h, g.cminx, g.dimx) + (int)lane / 9 - 1;
        const int yy = cell_coord(xi.y, P.h, g.cminy, g.dimy) + ((int)lane / 3) % 3 - 1;
        const int zz = cell_coord(xi.z, P.h, g.cminz, g.dimz) + (int)lane % 3 - 1;
        if (xx >= 0 && xx < g.dimx && yy >= 0 && yy < g.dimy && zz >= 0 && zz < g.dimz) {
            const unsigned c = brick_morton(xx, yy, zz, g);
            s = cell_start[c];
            e = cell_start[c + 1];
            if (P.nb > 0) {
                bs = bcell_start[c];
                be = bcell_start[c + 1];
            }
        }
    }
    const size_t nf = (size_t)P.nf;
    unsigned nF = 0, nB = 0;
    warp_candidates(pos, s, e, xi, P.h2_exact, lane, P.capF, nbr_f, nf, i, nF);
    if (P.nb > 0) warp_candidates(bpos, bs, be, xi, P.h2_exact, lane, P.capB, nbr_b, nf, i, nB);
    if (lane != 0) return;
    cnt_f[i] = min(nF, P.capF);
    cnt_b[i] = min(nB, P.capB);
    if (nF > P.capF || nB > P.capB) {
        atomicAdd(&st->overflow, 1u);
        atomicOr(&st->err, ERRBIT_OVERFLOW);
    }
}

} // namespace sph

#endif
