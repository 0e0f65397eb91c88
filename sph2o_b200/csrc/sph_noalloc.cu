/*
 * sph_density_noalloc: fluid densities for callers that cannot allocate GPU
 * memory.
 *
 * Who needs it: code that runs where cudaMalloc is off limits -- inside a
 * host callback or a custom allocator hook, in a process whose device memory
 * is owned and pooled by a framework, or on a real-time path that must not
 * take the allocator's locks or trigger an implicit synchronisation. Such a
 * caller owns its input and output buffers but no scratch.
 *
 * How: the neighbour-search scratch (cell table, sort buffers, sorted copies)
 * lives in one file-scope static __device__ array of fixed size, so this path
 * calls no cudaMalloc, cudaFree or allocating library routine. Every GPU that
 * loads the library holds the array (about 9.5 MiB) until the process exits.
 *
 * Rules for callers (also in include/sph2o_cuda.h):
 *   - sizes above SPH_NOALLOC_MAX_FLUID / _BOUNDARY / _CELLS are rejected
 *     with SPH_ERR_CAPACITY before anything is launched;
 *   - every call on a device uses the same array and leaves its contents
 *     behind; calls whose work overlaps on the GPU (different streams, or
 *     host threads calling concurrently) race on it and must be serialised
 *     by the caller;
 *   - the first call on each device looks up the array's device address with
 *     cudaGetSymbolAddress (once, with that device current); make that first
 *     call before any stream capture on the device. The address is cached per
 *     device ordinal and CUDA context id, so after cudaDeviceReset (a new
 *     primary context, the module possibly reloaded elsewhere) the next call
 *     looks it up again -- that call, too, belongs outside a stream capture.
 * The kernels reuse the pipeline's sort (sph_grid.cu) and evaluate each
 * density over the 27 cells in the same order and with the same exact
 * arithmetic as the context path, so for particles inside domain_min/max the
 * result equals sph_compute_phase(SPH_PHASE_DENSITY) bit for bit. A particle
 * outside the grid is clamped into an edge cell: it still finds every
 * neighbour, but visits them in another order, so its density can differ
 * from the context path's in the last bits.
 */
#include "../../include/sph2o_cuda.h"
#include "sph_internal.h"

#include <cuda.h> /* driver types only: the two driver calls are fetched at run time */

#include <climits>
#include <cmath>
#include <mutex>
#include <string>

namespace sph {
namespace {

constexpr size_t kMaxFluid = SPH_NOALLOC_MAX_FLUID;
constexpr size_t kMaxBoundary = SPH_NOALLOC_MAX_BOUNDARY;
constexpr size_t kMaxCells = SPH_NOALLOC_MAX_CELLS;  /* multiple of 4096 */
constexpr size_t kMaxN = kMaxFluid > kMaxBoundary ? kMaxFluid : kMaxBoundary;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

/* byte offsets of the regions inside the scratch array */
constexpr size_t kOffCount = 0;
constexpr size_t kOffStart = kOffCount + align256(kMaxCells * 4);
constexpr size_t kOffBStart = kOffStart + align256((kMaxCells + 1) * 4);
constexpr size_t kOffBlockSums = kOffBStart + align256((kMaxCells + 1) * 4);
constexpr size_t kOffCellOf = kOffBlockSums + align256((kMaxCells / 4096 + 1) * 4);
constexpr size_t kOffSlot = kOffCellOf + align256(kMaxN * 4);
constexpr size_t kOffKey = kOffSlot + align256(kMaxN * 4);
constexpr size_t kOffSrc = kOffKey + align256(kMaxN * 4);
constexpr size_t kOffIds = kOffSrc + align256(kMaxN * 4);
constexpr size_t kOffOrig = kOffIds + align256(kMaxN * 4);
constexpr size_t kOffBOrig = kOffOrig + align256(kMaxFluid * 4);
constexpr size_t kOffPosRaw = kOffBOrig + align256(kMaxBoundary * 4);
constexpr size_t kOffPos = kOffPosRaw + align256(kMaxFluid * 16);
constexpr size_t kOffBRaw = kOffPos + align256(kMaxFluid * 16);
constexpr size_t kOffBPos = kOffBRaw + align256(kMaxBoundary * 16);
constexpr size_t kScratchBytes = kOffBPos + align256(kMaxBoundary * 16);

} // namespace

/* The scratch of sph_density_noalloc (see the file comment). */
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_setup_mutex;

/* Device address of the scratch per device ordinal, valid for the CUDA
   context it was looked up in (ctx_id; 0 = unknown). */
struct ScratchAddr {
    unsigned long long ctx_id;
    unsigned char* ptr;
};
ScratchAddr g_scratch_dev[64] = {};

/* Unique id of the context current on this thread (cuCtxGetCurrent +
   cuCtxGetId, fetched through cudaGetDriverEntryPoint so the library does not
   link libcuda). Returns false when no context is current or the driver
   calls are unavailable. Called under g_setup_mutex. */
bool current_context_id(unsigned long long* id)
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {
        cudaDriverEntryPointQueryResult q1{}, q2{};
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrent>(f1);
            get_id = reinterpret_cast<GetId>(f2);
        }
        resolved = true;
    }
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

__global__ void k_na_pack_fluid(int n, const float* __restrict__ xyz, float4* __restrict__ out,
                                unsigned* __restrict__ ids)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2], 0.0f);
    ids[i] = (unsigned)i;
}

__global__ void k_na_pack_boundary(int n, const float* __restrict__ xyzw, float4* __restrict__ out,
                                   unsigned* __restrict__ ids)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4(xyzw[4 * (size_t)i], xyzw[4 * (size_t)i + 1], xyzw[4 * (size_t)i + 2],
                         xyzw[4 * (size_t)i + 3]);
    ids[i] = (unsigned)i;
}

/* Density over the 27 cells: every fluid candidate first, then every boundary
   candidate, cells in the reference's offset order, exact W; written to the
   caller's order. */
__global__ void __launch_bounds__(128) k_na_density(SimParams P, const float4* __restrict__ pos,
                                                    const unsigned* __restrict__ cell_start,
                                                    const unsigned* __restrict__ orig,
                                                    const float4* __restrict__ bpos,
                                                    const unsigned* __restrict__ bcell_start,
                                                    float* __restrict__ rho_out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.nf) return;
    const float4 xi = pos[i];
    const Grid g = grid_single(P);
    float rho = 0.0f;
    for_cells27(xi, P.h, g, [&](unsigned c) {
        for (unsigned q = cell_start[c]; q < cell_start[c + 1]; ++q) {
            const float s2 = dist2_exact(xi, pos[q]);
            if (s2 <= P.h2_guard) rho = __fadd_rn(rho, __fmul_rn(P.mass, cs_W_exact(s2, P)));
        }
    });
    if (P.nb > 0)
        for_cells27(xi, P.h, g, [&](unsigned c) {
            for (unsigned q = bcell_start[c]; q < bcell_start[c + 1]; ++q) {
                const float4 xb = bpos[q];
                const float s2 = dist2_exact(xi, xb);
                if (s2 <= P.h2_guard) rho = __fadd_rn(rho, __fmul_rn(xb.w, cs_W_exact(s2, P)));
            }
        });
    rho_out[orig[i]] = rho;
}

thread_local std::string g_noalloc_error;

int na_fail(int code, const std::string& msg)
{
    g_noalloc_error = msg;
    return code;
}

} // namespace
} // namespace sph

using namespace sph;

extern "C" int sph_density_noalloc(float particle_radius, float density0, const float* xyz, unsigned nf,
                                   const float* bxyzpsi, unsigned nb, const float domain_min[3],
                                   const float domain_max[3], float* rho_out, void* stream)
{
    if (!(particle_radius > 0.0f) || !(density0 > 0.0f) || !domain_min || !domain_max)
        return na_fail(SPH_ERR_ARG, "particle_radius, density0 and the domain bounds are required");
    if (nf > 0 && (!xyz || !rho_out)) return na_fail(SPH_ERR_ARG, "null fluid input or output");
    if (nb > 0 && !bxyzpsi) return na_fail(SPH_ERR_ARG, "null boundary input");
    if (nf > kMaxFluid)
        return na_fail(SPH_ERR_CAPACITY, "sph_density_noalloc: " + std::to_string(nf) + " fluid particles exceed "
                                         "SPH_NOALLOC_MAX_FLUID = " + std::to_string(kMaxFluid));
    if (nb > kMaxBoundary)
        return na_fail(SPH_ERR_CAPACITY, "sph_density_noalloc: " + std::to_string(nb) + " boundary particles "
                                         "exceed SPH_NOALLOC_MAX_BOUNDARY = " + std::to_string(kMaxBoundary));

    /* grid over the caller's domain (+1 cell), brick-padded; particles outside
       it are clamped into the edge cells: still found, in another order */
    SimParams P{};
    P.r = particle_radius;
    P.h = 4.0f * particle_radius;
    P.h2 = P.h * P.h;
    P.h2_guard = (float)((double)P.h * (double)P.h * (1.0 + 1.0e-5));
    P.h2_exact = sqrt_le_bound(P.h);
    P.inv_h = 1.0f / P.h;
    P.rho0 = density0;
    const float diameter = 2.0f * particle_radius;
    P.mass = density0 * (float)std::pow((double)diameter, 3.0);
    const float h3 = P.h * P.h * P.h;
    P.cs_k = 8.0f / ((float)M_PI * h3);
    P.nf = (int)nf;
    P.nb = (int)nb;
    int cmin[3], dim[3];
    for (int k = 0; k < 3; ++k) {
        if (!std::isfinite(domain_min[k]) || !std::isfinite(domain_max[k]))
            return na_fail(SPH_ERR_ARG, "sph_density_noalloc: domain bounds must be finite");
        if (!(domain_max[k] >= domain_min[k])) return na_fail(SPH_ERR_ARG, "domain_max < domain_min");
        const double a = std::floor((double)domain_min[k] / P.h) - 1.0;
        const double b = std::floor((double)domain_max[k] / P.h) + 1.0;
        if (a < (double)(INT_MIN / 2) || b > (double)(INT_MAX / 2))
            return na_fail(SPH_ERR_ARG, "sph_density_noalloc: domain bounds too far from the origin for cell "
                                        "indices of edge 4r");
        if (b - a + 1.0 > (double)kMaxCells) return na_fail(SPH_ERR_CAPACITY, "sph_density_noalloc: domain too large");
        cmin[k] = (int)a;
        dim[k] = ((int)(b - a + 1.0) + 3) / 4 * 4;
    }
    const unsigned long long cells = (unsigned long long)dim[0] * dim[1] * dim[2];
    const unsigned long long padded = (cells + 4095) / 4096 * 4096;
    if (padded > kMaxCells)
        return na_fail(SPH_ERR_CAPACITY, "sph_density_noalloc: the domain needs " + std::to_string(cells) +
                                         " cells of size 4r, above SPH_NOALLOC_MAX_CELLS = " + std::to_string(kMaxCells));
    P.cminx = cmin[0]; P.cminy = cmin[1]; P.cminz = cmin[2];
    P.dimx = dim[0]; P.dimy = dim[1]; P.dimz = dim[2];
    P.nbx = dim[0] / 4; P.nby = dim[1] / 4;
    P.ncells = (unsigned)padded;

    /* once per device, with that device current: the array's device address */
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_fail(SPH_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return na_fail(SPH_ERR_NO_DEVICE, "device ordinal out of range");
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        unsigned long long ctx = 0;
        const bool known = current_context_id(&ctx);
        ScratchAddr& slot = g_scratch_dev[dev];
        if (!slot.ptr || !known || slot.ctx_id != ctx) {
            /* first call on this device, or its context changed (cudaDeviceReset) */
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return na_fail(SPH_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            if (!current_context_id(&ctx)) ctx = 0;  /* the lookup made the primary context current */
            slot.ptr = static_cast<unsigned char*>(p);
            slot.ctx_id = ctx;
        }
        base = slot.ptr;
    }
    if (nf == 0) return SPH_OK;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned* cell_count = reinterpret_cast<unsigned*>(base + kOffCount);
    unsigned* cell_start = reinterpret_cast<unsigned*>(base + kOffStart);
    unsigned* bcell_start = reinterpret_cast<unsigned*>(base + kOffBStart);
    unsigned* block_sums = reinterpret_cast<unsigned*>(base + kOffBlockSums);
    unsigned* cell_of = reinterpret_cast<unsigned*>(base + kOffCellOf);
    unsigned* slot = reinterpret_cast<unsigned*>(base + kOffSlot);
    unsigned* key = reinterpret_cast<unsigned*>(base + kOffKey);
    unsigned* src = reinterpret_cast<unsigned*>(base + kOffSrc);
    unsigned* ids = reinterpret_cast<unsigned*>(base + kOffIds);
    unsigned* orig = reinterpret_cast<unsigned*>(base + kOffOrig);
    unsigned* borig = reinterpret_cast<unsigned*>(base + kOffBOrig);
    float4* pos_raw = reinterpret_cast<float4*>(base + kOffPosRaw);
    float4* pos = reinterpret_cast<float4*>(base + kOffPos);
    float4* braw = reinterpret_cast<float4*>(base + kOffBRaw);
    float4* bpos = reinterpret_cast<float4*>(base + kOffBPos);

    /* the populations must start at zero; the array keeps the last call's contents */
    e = cudaMemsetAsync(cell_count, 0, (size_t)P.ncells * sizeof(unsigned), s);
    if (e != cudaSuccess) return na_fail(SPH_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));

    if (nb > 0) {
        k_na_pack_boundary<<<(nb + 255) / 256, 256, 0, s>>>((int)nb, bxyzpsi, braw, ids);
        GatherSet gb{};
        gb.orig_out = borig;
        gb.v4_in[0] = braw;
        gb.v4_out[0] = bpos;
        launch_sort(P, SceneRef{}, (int)nb, braw, cell_count, bcell_start, block_sums, cell_of, slot, key, src, ids, gb, s);
    } else {
        e = cudaMemsetAsync(bcell_start, 0, ((size_t)P.ncells + 1) * sizeof(unsigned), s);
        if (e != cudaSuccess) return na_fail(SPH_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    }
    k_na_pack_fluid<<<(nf + 255) / 256, 256, 0, s>>>((int)nf, xyz, pos_raw, ids);
    GatherSet gf{};
    gf.orig_out = orig;
    gf.v4_in[0] = pos_raw;
    gf.v4_out[0] = pos;
    launch_sort(P, SceneRef{}, (int)nf, pos_raw, cell_count, cell_start, block_sums, cell_of, slot, key, src, ids, gf, s);
    k_na_density<<<(nf + 127) / 128, 128, 0, s>>>(P, pos, cell_start, orig, bpos, bcell_start, rho_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(SPH_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return SPH_OK;
}

extern "C" const char* sph_noalloc_error(void) { return g_noalloc_error.c_str(); }
