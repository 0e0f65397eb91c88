/*
 * Regular triangle sampling of a mesh on the GPU (boundary particles of OBJ
 * "geometry" entries).
 *
 * Restates SPH::RegularTriangleSampling::sampleMesh
 * (extern/RegularTriangleSampling/RegularTriangleSampling.cpp:12-117) with
 * its default skip flags, as a count / scan / write pipeline:
 *   1. every face emits its three edges as 64-bit keys (min << 32 | max);
 *      a radix sort and a unique pass give the reference's lexicographically
 *      sorted unique edge list (uniqueEdges, :96-117);
 *   2. one counting pass over the items [vertices | edges | faces] sizes
 *      each item's samples: 1 per vertex; the interior stops of an edge at
 *      ceil(l / d) + 1 even stops (a zero-length edge: its first vertex
 *      once); for a face, the interior stops of the interior lines parallel
 *      to its longest edge (ceil(h / d) + 1 lines over the height h, each
 *      at ceil(len / d) + 1 stops);
 *   3. an exclusive scan gives each item's first output slot, so the
 *      samples land in the reference's order (vertices, then edges in
 *      sorted order, then faces in file order);
 *   4. the write pass repeats the walk of pass 2 and stores each sample,
 *      optionally mapped by a 4x4 placement matrix plus a translation
 *      (AkinciBoundaryObject::sampleGeometry,
 *      src/SPH2O/BoundaryObject/AkinciBoundaryObject.cpp:155-214).
 *
 * Every float operation is an explicitly rounded intrinsic in the
 * reference's order (no contraction into FMA): its fixed-size Eigen
 * reductions sum a 3-vector as x + (y + z), glm applies a matrix as
 * (m0 x + m1 y) + (m2 z + m3 w). The samples are bit-identical to those of
 * the reference's FP32 build.
 *
 * A face whose three vertices coincide adds no face samples (the reference
 * reads uninitialised vectors there). Counts that would pass kMaxSamples
 * samples, or kMaxLines lines in one face (which already implies more than
 * kMaxSamples samples), set an error flag instead.
 */
#include "../../include/sph2o_cuda.h"
#include "sph_mesh.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <cmath>
#include <string>
#include <vector>

namespace sph {
namespace {

constexpr unsigned long long kMaxSamples = 1ull << 30;
constexpr unsigned kMaxLines = 1u << 16;
constexpr unsigned ERR_TOO_MANY = 1u;

struct MeshView {
    const float* v;                 /* xyz per vertex */
    const unsigned* f;              /* 3 indices per face */
    const unsigned long long* e;    /* sorted unique edge keys */
    unsigned nv, ne, nf;
    float d;
};

struct Placement {
    float m[4][4]; /* columns, as glm stores them */
    float t[3];
    int apply;
};

__device__ __forceinline__ float3 vtx(const float* v, unsigned i)
{
    return make_float3(v[3ull * i], v[3ull * i + 1], v[3ull * i + 2]);
}
__device__ __forceinline__ float3 sub3(float3 a, float3 b)
{
    return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
/* a + s * d */
__device__ __forceinline__ float3 axpy3(float3 a, float s, float3 d)
{
    return make_float3(__fadd_rn(a.x, __fmul_rn(s, d.x)), __fadd_rn(a.y, __fmul_rn(s, d.y)),
                       __fadd_rn(a.z, __fmul_rn(s, d.z)));
}
/* Eigen's unrolled three-term sum: x + (y + z) */
__device__ __forceinline__ float sum3(float a, float b, float c) { return __fadd_rn(a, __fadd_rn(b, c)); }
__device__ __forceinline__ float sqnorm3(float3 a)
{
    return sum3(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y), __fmul_rn(a.z, a.z));
}
__device__ __forceinline__ float dot3(float3 a, float3 b)
{
    return sum3(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z));
}

/* ceil(len / d) + 1 stops, or 1 with the error flag set past the limit */
__device__ __forceinline__ unsigned stops(float len, float d, unsigned* err)
{
    const float q = ceilf(__fdiv_rn(len, d));
    if (!(q < (float)kMaxSamples)) {
        atomicOr(err, ERR_TOO_MANY);
        return 1u;
    }
    return (unsigned)q + 1u;
}

struct FaceFrame {
    float3 v0, bn, to_top;
    float l;
    unsigned lines; /* 0: no face samples */
};

/* The longest edge (first one on ties) as base, its unit direction, the
   edge to the apex and the number of lines over the height. */
__device__ FaceFrame face_frame(const MeshView& m, unsigned t, unsigned* err)
{
    const unsigned* f = m.f + 3ull * t;
    float l2 = 0.0f;
    float3 v0 = make_float3(0, 0, 0), base = v0, to_top = v0;
    for (unsigned c = 0; c < 3; ++c) {
        const float3 p = vtx(m.v, f[c]);
        const float3 e = sub3(vtx(m.v, f[(c + 1) % 3]), p);
        const float le2 = sqnorm3(e);
        if (le2 > l2) {
            l2 = le2;
            v0 = p;
            base = e;
            to_top = sub3(vtx(m.v, f[(c + 2) % 3]), p);
        }
    }
    FaceFrame fr{v0, make_float3(0, 0, 0), to_top, 0.0f, 0u};
    if (!(l2 > 0.0f)) return fr;
    fr.l = __fsqrt_rn(l2);
    fr.bn = make_float3(__fdiv_rn(base.x, fr.l), __fdiv_rn(base.y, fr.l), __fdiv_rn(base.z, fr.l));
    const float along = dot3(fr.bn, to_top);
    const float3 perp = make_float3(__fsub_rn(to_top.x, __fmul_rn(along, fr.bn.x)),
                                    __fsub_rn(to_top.y, __fmul_rn(along, fr.bn.y)),
                                    __fsub_rn(to_top.z, __fmul_rn(along, fr.bn.z)));
    const float h = __fsqrt_rn(sqnorm3(perp));
    const unsigned lines = stops(h, m.d, err);
    if (lines > kMaxLines) {
        atomicOr(err, ERR_TOO_MANY);
        return fr;
    }
    fr.lines = lines;
    return fr;
}

/* Start and length of interior line `line` of a face */
__device__ __forceinline__ void face_line(const FaceFrame& fr, unsigned line, float3& start, float& len)
{
    const float alpha = __fdiv_rn((float)line, (float)(fr.lines - 1u));
    start = axpy3(fr.v0, alpha, fr.to_top);
    len = __fmul_rn(__fsub_rn(1.0f, alpha), fr.l);
}

__device__ __forceinline__ void edge_ends(const MeshView& m, unsigned k, float3& v0, float3& dir)
{
    const unsigned long long key = m.e[k];
    v0 = vtx(m.v, (unsigned)(key >> 32));
    dir = sub3(vtx(m.v, (unsigned)(key & 0xffffffffull)), v0);
}

__global__ void k_edge_keys(const unsigned* f, unsigned nf, unsigned long long* keys)
{
    for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < 3ull * nf;
         w += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long t = w / 3, c = w % 3;
        const unsigned a = f[3 * t + c], b = f[3 * t + (c + 1) % 3];
        keys[w] = ((unsigned long long)min(a, b) << 32) | (unsigned long long)max(a, b);
    }
}

__global__ void k_mesh_count(MeshView m, unsigned long long* count, unsigned* err)
{
    const unsigned long long items = (unsigned long long)m.nv + m.ne + m.nf;
    for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < items;
         w += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long c = 0;
        if (w < m.nv) {
            c = 1;
        } else if (w < (unsigned long long)m.nv + m.ne) {
            float3 v0, dir;
            edge_ends(m, (unsigned)(w - m.nv), v0, dir);
            const unsigned n = stops(__fsqrt_rn(sqnorm3(dir)), m.d, err);
            c = n == 1u ? 1u : n - 2u;
        } else {
            const FaceFrame fr = face_frame(m, (unsigned)(w - m.nv - m.ne), err);
            for (unsigned line = 1; line + 1u < fr.lines; ++line) {
                float3 start;
                float len;
                face_line(fr, line, start, len);
                const unsigned n = stops(len, m.d, err);
                c += n > 2u ? n - 2u : 0u;
            }
        }
        if (c > kMaxSamples) {
            atomicOr(err, ERR_TOO_MANY);
            c = 0;
        }
        count[w] = c;
    }
}

__device__ __forceinline__ void store(const Placement& pl, float* out, unsigned long long slot, float3 p)
{
    if (pl.apply) {
        /* glm's mat4 * vec4 with w = 1, then the translation */
        float o[3];
        for (int k = 0; k < 3; ++k)
            o[k] = __fadd_rn(__fadd_rn(__fmul_rn(pl.m[0][k], p.x), __fmul_rn(pl.m[1][k], p.y)),
                             __fadd_rn(__fmul_rn(pl.m[2][k], p.z), __fmul_rn(pl.m[3][k], 1.0f)));
        p = make_float3(__fadd_rn(o[0], pl.t[0]), __fadd_rn(o[1], pl.t[1]), __fadd_rn(o[2], pl.t[2]));
    }
    out[3 * slot] = p.x;
    out[3 * slot + 1] = p.y;
    out[3 * slot + 2] = p.z;
}

__global__ void k_mesh_write(MeshView m, Placement pl, const unsigned long long* offs, float* out, unsigned* err)
{
    const unsigned long long items = (unsigned long long)m.nv + m.ne + m.nf;
    for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < items;
         w += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long slot = offs[w];
        if (w < m.nv) {
            store(pl, out, slot, vtx(m.v, (unsigned)w));
        } else if (w < (unsigned long long)m.nv + m.ne) {
            float3 v0, dir;
            edge_ends(m, (unsigned)(w - m.nv), v0, dir);
            const unsigned n = stops(__fsqrt_rn(sqnorm3(dir)), m.d, err);
            if (n == 1u) {
                store(pl, out, slot, v0);
                continue;
            }
            const float den = (float)(n - 1u);
            for (unsigned i = 1; i + 1u < n; ++i) store(pl, out, slot++, axpy3(v0, __fdiv_rn((float)i, den), dir));
        } else {
            const FaceFrame fr = face_frame(m, (unsigned)(w - m.nv - m.ne), err);
            for (unsigned line = 1; line + 1u < fr.lines; ++line) {
                float3 start;
                float len;
                face_line(fr, line, start, len);
                const unsigned n = stops(len, m.d, err);
                const float den = (float)(n - 1u);
                for (unsigned i = 1; i + 1u < n; ++i)
                    store(pl, out, slot++, axpy3(start, __fdiv_rn(__fmul_rn((float)i, len), den), fr.bn));
            }
        }
    }
}

/* Device buffers of one sampling call, released on every return path. */
struct Scratch {
    std::vector<void*> ptrs;
    cudaStream_t s = nullptr;
    ~Scratch()
    {
        for (void* p : ptrs) cudaFree(p);
        if (s) cudaStreamDestroy(s);
    }
    template <class T>
    cudaError_t alloc(T** p, size_t count)
    {
        *p = nullptr;
        if (count == 0) count = 1;
        const cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back((void*)*p);
        return e;
    }
};

unsigned grid_for(unsigned long long items)
{
    const unsigned long long blocks = (items + 255) / 256;
    return (unsigned)std::max(1ull, std::min(blocks, 148ull * 16));
}

} // namespace

int sample_mesh_device(const float* v, unsigned nv, const unsigned* f, unsigned nf, float d, const float* m16,
                       const float* translate, std::vector<float>& out, std::string& err)
{
    out.clear();
    /* the kernels index vertices through the faces: check every index here */
    if (!(d > 0.0f) || !std::isfinite(d)) {
        err = "mesh sampling distance must be positive and finite";
        return SPH_ERR_ARG;
    }
    if ((!v && nv) || (!f && nf)) {
        err = "null mesh array";
        return SPH_ERR_ARG;
    }
    if (nf > (1u << 28) || nv > (1u << 29)) {
        err = "mesh too large (at most 2^29 vertices and 2^28 faces)";
        return SPH_ERR_CAPACITY;
    }
    for (unsigned long long i = 0; i < 3ull * nf; ++i)
        if (f[i] >= nv) {
            err = "face index outside the vertex list";
            return SPH_ERR_ARG;
        }
    for (unsigned long long i = 0; i < 3ull * nv; ++i)
        if (!std::isfinite(v[i])) {
            err = "non-finite mesh vertex";
            return SPH_ERR_ARG;
        }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        err = "mesh sampling needs a CUDA device";
        return SPH_ERR_NO_DEVICE;
    }
    Scratch sc;
#define MESH_TRY(expr)                                                                                 \
    do {                                                                                               \
        const cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess) {                                                                       \
            err = std::string(#expr ": ") + cudaGetErrorString(e_);                                    \
            return SPH_ERR_CUDA;                                                                       \
        }                                                                                              \
    } while (0)
    MESH_TRY(cudaStreamCreateWithFlags(&sc.s, cudaStreamNonBlocking));
    float* dv;
    unsigned* df;
    unsigned long long *keys, *keys_sorted, *edges;
    unsigned *dne, *derr;
    MESH_TRY(sc.alloc(&dv, 3ull * nv));
    MESH_TRY(sc.alloc(&df, 3ull * nf));
    MESH_TRY(sc.alloc(&keys, 3ull * nf));
    MESH_TRY(sc.alloc(&keys_sorted, 3ull * nf));
    MESH_TRY(sc.alloc(&edges, 3ull * nf));
    MESH_TRY(sc.alloc(&dne, 1));
    MESH_TRY(sc.alloc(&derr, 1));
    MESH_TRY(cudaMemcpyAsync(dv, v, 3ull * nv * sizeof(float), cudaMemcpyHostToDevice, sc.s));
    MESH_TRY(cudaMemcpyAsync(df, f, 3ull * nf * sizeof(unsigned), cudaMemcpyHostToDevice, sc.s));
    MESH_TRY(cudaMemsetAsync(dne, 0, sizeof(unsigned), sc.s));
    MESH_TRY(cudaMemsetAsync(derr, 0, sizeof(unsigned), sc.s));

    /* 1. sorted unique edges */
    const int nkeys = (int)(3ull * nf);
    if (nkeys > 0) {
        k_edge_keys<<<grid_for(nkeys), 256, 0, sc.s>>>(df, nf, keys);
        MESH_TRY(cudaGetLastError());
        size_t t1 = 0, t2 = 0;
        MESH_TRY(cub::DeviceRadixSort::SortKeys(nullptr, t1, keys, keys_sorted, nkeys, 0, 64, sc.s));
        MESH_TRY(cub::DeviceSelect::Unique(nullptr, t2, keys_sorted, edges, dne, nkeys, sc.s));
        char* tmp;
        MESH_TRY(sc.alloc(&tmp, std::max(t1, t2)));
        size_t tb = std::max(t1, t2);
        MESH_TRY(cub::DeviceRadixSort::SortKeys(tmp, tb, keys, keys_sorted, nkeys, 0, 64, sc.s));
        tb = std::max(t1, t2);
        MESH_TRY(cub::DeviceSelect::Unique(tmp, tb, keys_sorted, edges, dne, nkeys, sc.s));
    }
    unsigned ne = 0;
    MESH_TRY(cudaMemcpyAsync(&ne, dne, sizeof(unsigned), cudaMemcpyDeviceToHost, sc.s));
    MESH_TRY(cudaStreamSynchronize(sc.s));

    /* 2-3. per-item counts and their exclusive scan */
    const unsigned long long items = (unsigned long long)nv + ne + nf;
    if (items == 0) return SPH_OK;
    unsigned long long *count, *offs;
    MESH_TRY(sc.alloc(&count, items));
    MESH_TRY(sc.alloc(&offs, items));
    const MeshView m{dv, df, edges, nv, ne, nf, d};
    k_mesh_count<<<grid_for(items), 256, 0, sc.s>>>(m, count, derr);
    MESH_TRY(cudaGetLastError());
    size_t ts = 0;
    MESH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, ts, count, offs, (int)items, sc.s));
    char* tmp2;
    MESH_TRY(sc.alloc(&tmp2, ts));
    MESH_TRY(cub::DeviceScan::ExclusiveSum(tmp2, ts, count, offs, (int)items, sc.s));
    unsigned long long last_off = 0, last_cnt = 0;
    unsigned herr = 0;
    MESH_TRY(cudaMemcpyAsync(&last_off, offs + items - 1, sizeof(last_off), cudaMemcpyDeviceToHost, sc.s));
    MESH_TRY(cudaMemcpyAsync(&last_cnt, count + items - 1, sizeof(last_cnt), cudaMemcpyDeviceToHost, sc.s));
    MESH_TRY(cudaMemcpyAsync(&herr, derr, sizeof(herr), cudaMemcpyDeviceToHost, sc.s));
    MESH_TRY(cudaStreamSynchronize(sc.s));
    const unsigned long long total = last_off + last_cnt;
    if (herr != 0 || total > kMaxSamples) {
        err = "mesh sampling exceeds the particle limit (2^30 samples)";
        return SPH_ERR_CAPACITY;
    }

    /* 4. samples in the reference's order */
    float* dout;
    MESH_TRY(sc.alloc(&dout, 3ull * total));
    Placement pl{};
    pl.apply = m16 != nullptr;
    if (m16)
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) pl.m[c][r] = m16[4 * c + r];
    for (int k = 0; k < 3; ++k) pl.t[k] = translate ? translate[k] : 0.0f;
    k_mesh_write<<<grid_for(items), 256, 0, sc.s>>>(m, pl, offs, dout, derr);
    MESH_TRY(cudaGetLastError());
    out.resize(3ull * total);
    MESH_TRY(cudaMemcpyAsync(out.data(), dout, out.size() * sizeof(float), cudaMemcpyDeviceToHost, sc.s));
    MESH_TRY(cudaStreamSynchronize(sc.s));
#undef MESH_TRY
    return SPH_OK;
}

} // namespace sph
