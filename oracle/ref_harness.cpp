/*
 * Headless harness around the UNMODIFIED SPH2O sources (test infrastructure:
 * only tests/, bench.py's CPU-baseline leg and smoke() run what this builds).
 *
 * oracle/Makefile compiles this file together with the reference's own
 * src/SPH2O sources into oracle/_ref/sph2o_ref_<variant>. It replaces
 * src/main.cpp, which pulls in the OpenGL GUI, and avoids two behaviours of
 * the reference driver that make it unusable as a harness:
 *   - SPHSimulation::run() never terminates (src/SPH2O/SPHSimulation.cpp:193-199),
 *     so this harness calls SPHSimulation::step() a fixed number of times;
 *   - "-f" calls exit(0) after loading (src/SPH2O/SPHSimulation.cpp:547-548),
 *     so state is injected through getPosition(i)/getVelocity(i) instead.
 * Two uninitialised solver members are zeroed before the first step:
 * DFSPHSolver::iterationsV (read by updateTimeStep, DFSPHSolver.cpp:1146) and
 * PCISPHSolver::avgDensityError (read by pressureSolver, PCISPHSolver.cpp:374).
 *
 * Usage:
 *   sph2o_ref -c scene.json --mode step|neighbors|phases|time|frames
 *             [--steps N] [--warmup W] [--out file.sphd]
 *             [--state-in file.sphd] [--boundary-in file.sphd] [--threads T]
 *             [--dt-in dt] [--gpu]
 *
 * --mode frames turns saving on and calls SPHSimulation::step() N times, so
 * the reference itself decides when to save (TimeHelper::hasToSave) and
 * writes <scene>_NNNN.json with SceneLoader::writeFluid
 * (SPHSimulation.cpp:179-187, SceneLoader.cpp:211-275).
 *
 * --gpu (only in the sph2o_ref_gpu build, compiled with SPH2O_HARNESS_GPU and
 * linked with libsph2o_cuda.so) installs the reference-side binding
 * include/sph2o_gpu_solver.hpp: after the scene is imported, the configured
 * CPU solver is handed to a GPUSolver that replaces it, as a maintainer
 * would do in SPHSimulation::init(); SPHSimulation::init/step and
 * writeFluid then run unchanged around the GPU step.
 *
 * Output (.sphd): "SPHD0001", then records
 *   u32 name_len, name, char dtype ('f' f32, 'd' f64, 'i' i32, 'u' u32),
 *   u32 ndim, u64 shape[ndim], raw little-endian data.
 * Arrays of Real are written as 'f' or 'd' depending on the build variant.
 */
#include "SPH2O/SPHSimulation.h"
#include "SPH2O/SPHSolver/DFSPHSolver.h"
#include "SPH2O/SPHSolver/PCISPHSolver.h"
#include "SPH2O/SPHSolver/WCSPHSolver.h"
#include "SPH2O/BoundaryObject/AkinciBoundaryObject.h"
#include "SPH2O/BoundaryObject/PCISPHBoundaryObject.h"
#include "SPH2O/HashTable.h"
#include "json/json.hpp"

#include "../sph2o_b200/host/scene_rng.h"
#ifdef SPH2O_HARNESS_GPU
#include "sph2o_gpu_solver.hpp"
#endif

#include <omp.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

/* Access to protected solver counters through the pointer-to-member rule. */
struct SolverAccess : SPHSolver {
    static uint& its(SPHSolver* s) { return s->*(&SolverAccess::iterations); }
};
struct DFAccess : DFSPHSolver {
    static uint& itsV(DFSPHSolver* s) { return s->*(&DFAccess::iterationsV); }
    static Real& avgDens(DFSPHSolver* s) { return s->*(&DFAccess::avgDensError); }
    static Real& avgDiv(DFSPHSolver* s) { return s->*(&DFAccess::avgDivError); }
};
struct PCIAccess : PCISPHSolver {
    static Real& avgDens(PCISPHSolver* s) { return s->*(&PCIAccess::avgDensityError); }
};
/* The simulation's solver slot (to install the GPU binding without editing SPH2O). */
struct SimAccess : SPHSimulation {
    static SPHSolver*& slot(SPHSimulation* s) { return s->*(&SimAccess::solver); }
};
/* Normals of PCISPH boundary particles (a protected member without a getter). */
struct PCIBoundaryAccess : PCISPHBoundaryObject {
    static std::vector<Vector3r>& normals(PCISPHBoundaryObject* o) { return o->*(&PCIBoundaryAccess::n); }
};

namespace {

struct Array {
    char dtype;
    std::vector<uint64_t> shape;
    std::vector<char> data;
};

std::map<std::string, Array> read_sphd(const std::string& path)
{
    std::map<std::string, Array> out;
    std::ifstream f(path, std::ios::binary);
    if (!f) { fprintf(stderr, "cannot open %s\n", path.c_str()); exit(2); }
    char magic[8];
    f.read(magic, 8);
    if (std::memcmp(magic, "SPHD0001", 8) != 0) { fprintf(stderr, "bad magic in %s\n", path.c_str()); exit(2); }
    while (true) {
        uint32_t nl;
        if (!f.read(reinterpret_cast<char*>(&nl), 4)) break;
        std::string name(nl, '\0');
        f.read(&name[0], nl);
        Array a;
        f.read(&a.dtype, 1);
        uint32_t nd;
        f.read(reinterpret_cast<char*>(&nd), 4);
        a.shape.resize(nd);
        uint64_t n = 1;
        for (uint32_t i = 0; i < nd; ++i) { f.read(reinterpret_cast<char*>(&a.shape[i]), 8); n *= a.shape[i]; }
        const size_t es = (a.dtype == 'd') ? 8 : 4;
        a.data.resize(n * es);
        f.read(a.data.data(), (std::streamsize)a.data.size());
        out[name] = std::move(a);
    }
    return out;
}

template <typename T> double as_double(const Array& a, size_t i)
{
    return (double)reinterpret_cast<const T*>(a.data.data())[i];
}
double elem(const Array& a, size_t i)
{
    switch (a.dtype) {
    case 'f': return as_double<float>(a, i);
    case 'd': return as_double<double>(a, i);
    case 'i': return as_double<int32_t>(a, i);
    default: return as_double<uint32_t>(a, i);
    }
}

class Writer {
public:
    explicit Writer(const std::string& path) : f_(path, std::ios::binary)
    {
        if (!f_) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
        f_.write("SPHD0001", 8);
    }
    template <typename T>
    void put(const std::string& name, const std::vector<T>& v, std::vector<uint64_t> shape)
    {
        char dt = std::is_same<T, float>::value ? 'f' : std::is_same<T, double>::value ? 'd'
                 : std::is_same<T, int32_t>::value ? 'i' : 'u';
        uint32_t nl = (uint32_t)name.size();
        f_.write(reinterpret_cast<const char*>(&nl), 4);
        f_.write(name.data(), nl);
        f_.write(&dt, 1);
        uint32_t nd = (uint32_t)shape.size();
        f_.write(reinterpret_cast<const char*>(&nd), 4);
        for (auto s : shape) f_.write(reinterpret_cast<const char*>(&s), 8);
        f_.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
    }
private:
    std::ofstream f_;
};

struct Opts {
    std::string scene, mode = "step", out, state_in, boundary_in;
    int steps = 1, warmup = 0, threads = 0;
    bool gpu = false;
    double dt_in = 0.0;
};

Opts parse(int argc, char** argv)
{
    Opts o;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(2); }
            return argv[++i];
        };
        if (a == "-c") o.scene = next();
        else if (a == "--mode") o.mode = next();
        else if (a == "--steps") o.steps = std::atoi(next().c_str());
        else if (a == "--warmup") o.warmup = std::atoi(next().c_str());
        else if (a == "--out") o.out = next();
        else if (a == "--state-in") o.state_in = next();
        else if (a == "--boundary-in") o.boundary_in = next();
        else if (a == "--threads") o.threads = std::atoi(next().c_str());
        else if (a == "--gpu") o.gpu = true;
        else if (a == "--dt-in") o.dt_in = std::atof(next().c_str());
        else { fprintf(stderr, "unknown option %s\n", a.c_str()); exit(2); }
    }
    if (o.scene.empty()) { fprintf(stderr, "-c scene.json is required\n"); exit(2); }
    return o;
}

/* Seeded jitter of the lattice, applied after FluidObject::build. */
void apply_jitter(SPHSimulation* sim, const std::string& scene)
{
    std::ifstream f(scene);
    nlohmann::json cfg;
    f >> cfg;
    const auto& c = cfg["Configuration"];
    if (c.find("jitter") == c.end()) return;
    const float jitter = c["jitter"];
    const uint64_t seed = c.find("jitterSeed") != c.end() ? (uint64_t)c["jitterSeed"] : 0ull;
    if (jitter == 0.0f) return;
    const float radius = (float)sim->getParticleRadius();
    uint64_t id = 0;
    for (uint m = 0; m < sim->numberFluidModels(); ++m) {
        FluidObject* fo = sim->getFluidModel(m);
        for (uint i = 0; i < fo->getSize(); ++i, ++id) {
            Vector3r& r = fo->getPosition(i);
            for (int k = 0; k < 3; ++k) {
                const float base = (float)r[k];
                r[k] = (Real)(base + sph_jitter_offset(seed, id, k, jitter, radius));
            }
        }
    }
}

void load_state(SPHSimulation* sim, const std::string& path)
{
    auto arrs = read_sphd(path);
    FluidObject* fo = sim->getFluidModel(0);
    const uint n = fo->getSize();
    if (arrs.count("pos")) {
        const Array& p = arrs["pos"];
        if (p.shape.size() != 2 || p.shape[0] != n) { fprintf(stderr, "pos shape mismatch\n"); exit(2); }
        for (uint i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) fo->getPosition(i)[k] = (Real)elem(p, 3ull * i + k);
    }
    if (arrs.count("vel")) {
        const Array& v = arrs["vel"];
        if (v.shape.size() != 2 || v.shape[0] != n) { fprintf(stderr, "vel shape mismatch\n"); exit(2); }
        for (uint i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) fo->getVelocity(i)[k] = (Real)elem(v, 3ull * i + k);
    }
}

/* Replace the boundary particle set: all injected points go to boundary
   object 0 (volumes are computed over the neighbours of every object alike,
   AkinciBoundaryObject.cpp:22-29, so the split between objects does not
   matter); the other objects are emptied. The FP64 build samples boxes with
   a different particle count, so it cannot be overwritten in place. */
void load_boundary(SPHSimulation* sim, const std::string& path)
{
    auto arrs = read_sphd(path);
    const Array& p = arrs.at("bpos");
    if (sim->numberBoundaryModels() == 0) { fprintf(stderr, "scene has no boundary object\n"); exit(2); }
    const uint n = (uint)p.shape[0];
    for (uint b = 1; b < sim->numberBoundaryModels(); ++b) sim->getBoundaryModel(b)->resize(0);
    BoundaryObject* bo = sim->getBoundaryModel(0);
    bo->resize(n);
    for (uint i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) bo->getPosition(i)[k] = (Real)elem(p, 3ull * i + k);
}

std::vector<Real> fluid_vec3(FluidObject* fo, int which)
{
    const uint n = fo->getSize();
    std::vector<Real> out(3ull * n);
    for (uint i = 0; i < n; ++i) {
        const Vector3r& v = which == 0 ? fo->getPosition(i) : which == 1 ? fo->getVelocity(i) : fo->getAcceleration(i);
        for (int k = 0; k < 3; ++k) out[3ull * i + k] = v[k];
    }
    return out;
}

std::vector<Real> fluid_density(FluidObject* fo)
{
    std::vector<Real> out(fo->getSize());
    for (uint i = 0; i < fo->getSize(); ++i) out[i] = fo->getDensity(i);
    return out;
}

/* PCISPH boundary method: per-particle normals, and densities / pressures */
bool pcisph_boundary(SPHSimulation* sim) { return sim->getBoundaryHandlingMethod() == SPHSimulation::PCISPH_BOUNDARY_METHOD; }

std::vector<Real> boundary_scalars(SPHSimulation* sim, bool pressure)
{
    std::vector<Real> out;
    for (uint b = 0; b < sim->numberBoundaryModels(); ++b) {
        PCISPHBoundaryObject* bo = static_cast<PCISPHBoundaryObject*>(sim->getBoundaryModel(b));
        for (uint i = 0; i < bo->getSize(); ++i) out.push_back(pressure ? bo->getPressure(i) : bo->getDensity(i));
    }
    return out;
}

std::vector<Real> boundary_normals(SPHSimulation* sim)
{
    std::vector<Real> out;
    for (uint b = 0; b < sim->numberBoundaryModels(); ++b) {
        PCISPHBoundaryObject* bo = static_cast<PCISPHBoundaryObject*>(sim->getBoundaryModel(b));
        for (const Vector3r& v : PCIBoundaryAccess::normals(bo))
            for (int k = 0; k < 3; ++k) out.push_back(v[k]);
    }
    return out;
}

void boundary_arrays(SPHSimulation* sim, std::vector<Real>& pos, std::vector<Real>& vol)
{
    for (uint b = 0; b < sim->numberBoundaryModels(); ++b) {
        BoundaryObject* bo = sim->getBoundaryModel(b);
        for (uint i = 0; i < bo->getSize(); ++i) {
            for (int k = 0; k < 3; ++k) pos.push_back(bo->getPosition(i)[k]);
            if (sim->getBoundaryHandlingMethod() == SPHSimulation::AKINCI_BOUNDARY_METHOD)
                vol.push_back(static_cast<AkinciBoundaryObject*>(bo)->getVolume(i));
        }
    }
}

/* Aggregate statistics of the fluid in double: centroid, kinetic energy,
   mean density error mean(max(rho - rho0, 0) / rho0). */
void aggregates(SPHSimulation* sim, double* out)
{
    FluidObject* fo = sim->getFluidModel(0);
    const uint n = fo->getNumActiveParticles();
    const double rho0 = fo->getRefDensity();
    double cx = 0, cy = 0, cz = 0, ke = 0, de = 0;
    for (uint i = 0; i < n; ++i) {
        const Vector3r& r = fo->getPosition(i);
        const Vector3r& v = fo->getVelocity(i);
        cx += r.x; cy += r.y; cz += r.z;
        ke += 0.5 * (double)fo->getMass(i) * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
        const double d = (double)fo->getDensity(i) - rho0;
        de += (d > 0 ? d : 0) / rho0;
    }
    out[0] = cx / n; out[1] = cy / n; out[2] = cz / n; out[3] = ke; out[4] = de / n;
}

void neighbor_sets(SPHSimulation* sim, Writer& w)
{
    FluidObject* fo = sim->getFluidModel(0);
    HashTable* grid = sim->getGrid();
    const Real h = sim->getSupportRadius();
    std::vector<uint64_t> boff(sim->numberBoundaryModels() + 1, 0);
    for (uint b = 0; b < sim->numberBoundaryModels(); ++b) boff[b + 1] = boff[b] + sim->getBoundaryModel(b)->getSize();
    std::vector<uint32_t> fo_off{0}, fo_idx, bo_off{0}, bo_idx;
    for (uint i = 0; i < fo->getNumActiveParticles(); ++i) {
        const Vector3r& ri = fo->getPosition(i);
        const Vector3i cellId = floor(ri / h);
        for (auto& pi : grid->table[cellId].neighbors)
            if (glm::length(ri - fo->getPosition(pi.id)) <= h) fo_idx.push_back(pi.id);
        for (auto& pi : grid->table[cellId].boundary_neighbors) {
            const Vector3r& rb = sim->getBoundaryModel(pi.pointSetId)->getPosition(pi.id);
            if (glm::length(ri - rb) <= h) bo_idx.push_back((uint32_t)(boff[pi.pointSetId] + pi.id));
        }
        fo_off.push_back((uint32_t)fo_idx.size());
        bo_off.push_back((uint32_t)bo_idx.size());
    }
    w.put("nbr_f_offsets", fo_off, {fo_off.size()});
    w.put("nbr_f", fo_idx, {fo_idx.size()});
    w.put("nbr_b_offsets", bo_off, {bo_off.size()});
    w.put("nbr_b", bo_idx, {bo_idx.size()});
}

} // namespace

int main(int argc, char** argv)
{
    Opts o = parse(argc, argv);
    if (o.threads > 0) omp_set_num_threads(o.threads);

    SPHSimulation* sim = SPHSimulation::getCurrent();
    sim->activateSave(false);
    if (!sim->importScene(o.scene)) { fprintf(stderr, "cannot import scene\n"); return 2; }
    if (sim->numberFluidModels() != 1) { fprintf(stderr, "harness expects one fluid model\n"); return 2; }
    apply_jitter(sim, o.scene);
    if (!o.state_in.empty()) load_state(sim, o.state_in);
    /* a run resumed from another run's state continues with its time step
       (DFSPH adapts it from the previous one, DFSPHSolver.cpp:1090-1162) */
    if (o.dt_in > 0.0) sim->setTimeStep((Real)o.dt_in);
    if (!o.boundary_in.empty()) load_boundary(sim, o.boundary_in);

    FluidObject* fo = sim->getFluidModel(0);
    std::vector<Real> init_pos = fluid_vec3(fo, 0), init_vel = fluid_vec3(fo, 1);
    const int method = sim->getSimulationMethod();

#ifdef SPH2O_HARNESS_GPU
    GPUSolver* gpu = nullptr;
    if (o.gpu) {
        gpu = new GPUSolver(sim->getSolver());
        SimAccess::slot(sim) = gpu;
    }
#else
    if (o.gpu) { fprintf(stderr, "--gpu needs the sph2o_ref_gpu build\n"); return 2; }
#endif
    if (o.mode == "frames") sim->activateSave(true);
    try {
        sim->init();
    } catch (const std::exception& e) {
        fprintf(stderr, "%s\n", e.what());
#ifdef SPH2O_HARNESS_GPU
        if (gpu) { /* the description the binding read from SPH2O, as 32-bit words */
            const sph_scene_desc& d = gpu->description();
            const unsigned char* p = reinterpret_cast<const unsigned char*>(&d);
            for (size_t k = 0; k < sizeof(d); k += 4) {
                uint32_t w;
                std::memcpy(&w, p + k, 4);
                fprintf(stderr, "%08x%c", w, (k / 4) % 8 == 7 ? '\n' : ' ');
            }
            fprintf(stderr, "\n");
        }
#endif
        return 3;
    }
    SPHSolver* solver = sim->getSolver();
    if (!o.gpu && method == SPHSimulation::DFSPH_METHOD) DFAccess::itsV(static_cast<DFSPHSolver*>(solver)) = 0;
    if (!o.gpu && method == SPHSimulation::PCISPH_METHOD) PCIAccess::avgDens(static_cast<PCISPHSolver*>(solver)) = 0;
    /* after a GPU step the fluid object's arrays are refreshed on demand */
    auto refresh = [&]() {
#ifdef SPH2O_HARNESS_GPU
        if (gpu) gpu->pull();
#endif
    };

    if (o.mode == "frames") {
        for (int s = 0; s < o.steps; ++s) sim->step();
        bool on_gpu = false;
#ifdef SPH2O_HARNESS_GPU
        on_gpu = gpu != nullptr && sim->getSolver() == gpu;
#endif
        printf("{\"steps\": %d, \"frames_written\": %u, \"time\": %.9g, \"gpu_solver\": %s}\n", o.steps,
               sim->getFrame() - 1, (double)sim->getTime(), on_gpu ? "true" : "false");
        return 0;
    }

    const uint64_t n = fo->getSize();
    std::vector<Real> bpos, bvol;
    boundary_arrays(sim, bpos, bvol);
    const uint64_t nb = bpos.size() / 3;

    if (o.gpu && o.mode != "time" && o.mode != "step") {
        fprintf(stderr, "--gpu supports the step, time and frames modes\n");
        return 2;
    }
    if (o.mode == "time") {
        for (int s = 0; s < o.warmup; ++s) sim->step();
        const double t0 = omp_get_wtime();
        uint64_t its = 0, itsv = 0;
        for (int s = 0; s < o.steps; ++s) {
            sim->step();
            its += SolverAccess::its(solver);
            if (method == SPHSimulation::DFSPH_METHOD) itsv += DFAccess::itsV(static_cast<DFSPHSolver*>(solver));
        }
        const double dt = omp_get_wtime() - t0;
        printf("{\"fluid_particles\": %llu, \"boundary_particles\": %llu, \"steps\": %d, \"warmup\": %d, "
               "\"seconds\": %.6f, \"particle_steps_per_s\": %.6e, \"threads\": %d, "
               "\"mean_iterations\": %.3f, \"mean_iterations_v\": %.3f, \"sim_time\": %.9g}\n",
               (unsigned long long)n, (unsigned long long)nb, o.steps, o.warmup, dt,
               (double)n * o.steps / dt, omp_get_max_threads(),
               o.steps ? (double)its / o.steps : 0.0, o.steps ? (double)itsv / o.steps : 0.0,
               (double)sim->getTime());
        return 0;
    }

    if (o.out.empty()) { fprintf(stderr, "--out is required for mode %s\n", o.mode.c_str()); return 2; }
    Writer w(o.out);
    w.put("init_pos", init_pos, {n, 3});
    w.put("init_vel", init_vel, {n, 3});
    w.put("bpos", bpos, {nb, 3});
    if (!bvol.empty()) w.put("bvol", bvol, {nb});
    if (pcisph_boundary(sim)) w.put("bnormal", boundary_normals(sim), {nb, 3});
    std::vector<Real> mass(n);
    for (uint64_t i = 0; i < n; ++i) mass[i] = fo->getMass((uint)i);
    w.put("mass", mass, {n});

    if (o.mode == "neighbors") {
        solver->insertFluidParticles();
        solver->neighborhoodSearch();
        neighbor_sets(sim, w);
        return 0;
    }

    if (o.mode == "phases") {
        solver->insertFluidParticles();
        solver->neighborhoodSearch();
        solver->computeDensities();
        w.put("density", fluid_density(fo), {n});
        if (pcisph_boundary(sim)) w.put("bdensity", boundary_scalars(sim, false), {nb});
        if (method == SPHSimulation::DFSPH_METHOD) {
            DFSPHSolver* df = static_cast<DFSPHSolver*>(solver);
            df->computeAlpha();
            std::vector<Real> alpha(n);
            for (uint64_t i = 0; i < n; ++i) alpha[i] = df->getAlpha(0, (uint)i);
            w.put("alpha", alpha, {n});
        }
        for (uint i = 0; i < n; ++i) fo->getAcceleration(i) = Vector3r(0.0);
        sim->computeNonPressureForces();
        w.put("a_nonpressure", fluid_vec3(fo, 2), {n, 3});
        if (method == SPHSimulation::WCSPH_METHOD) {
            WCSPHSolver* wc = static_cast<WCSPHSolver*>(solver);
            for (uint i = 0; i < n; ++i) fo->getAcceleration(i) = Vector3r(0.0);
            wc->computePressures();
            std::vector<Real> p(n);
            for (uint64_t i = 0; i < n; ++i) p[i] = fo->getPressure((uint)i);
            w.put("pressure", p, {n});
            if (pcisph_boundary(sim)) w.put("bpressure", boundary_scalars(sim, true), {nb});
            wc->computePressureForce(0);
            w.put("a_pressure", fluid_vec3(fo, 2), {n, 3});
        }
        return 0;
    }

    if (o.mode != "step") { fprintf(stderr, "unknown mode %s\n", o.mode.c_str()); return 2; }

    std::vector<Real> init_density = fluid_density(fo);
    w.put("init_density", init_density, {n});
    if (method == SPHSimulation::DFSPH_METHOD) {
        std::vector<Real> alpha(n);
        for (uint64_t i = 0; i < n; ++i) alpha[i] = static_cast<DFSPHSolver*>(solver)->getAlpha(0, (uint)i);
        w.put("init_alpha", alpha, {n});
    }
    /* per-step: time, dt, iterations, iterationsV, solver avg error, solver avg div error,
       centroid xyz, kinetic energy, mean density error */
    std::vector<double> stats, active;
    for (int s = 0; s < o.steps; ++s) {
        sim->step();
        refresh();
        active.push_back((double)fo->getNumActiveParticles());
        double agg[5];
        aggregates(sim, agg);
        double avg = 0, avgv = 0, itv = 0;
        if (o.gpu) {
            /* the GPU binding reports iterations through SPHSolver's counter only */
        } else if (method == SPHSimulation::DFSPH_METHOD) {
            DFSPHSolver* df = static_cast<DFSPHSolver*>(solver);
            avg = DFAccess::avgDens(df); avgv = DFAccess::avgDiv(df); itv = DFAccess::itsV(df);
        } else if (method == SPHSimulation::PCISPH_METHOD) {
            avg = PCIAccess::avgDens(static_cast<PCISPHSolver*>(solver));
        }
        const double row[11] = {(double)sim->getTime(), (double)sim->getTimeStep(),
                                (double)SolverAccess::its(solver), itv, avg, avgv,
                                agg[0], agg[1], agg[2], agg[3], agg[4]};
        stats.insert(stats.end(), row, row + 11);
    }
    w.put("step_stats", stats, {(uint64_t)o.steps, 11});
    w.put("active", active, {(uint64_t)o.steps});
    w.put("pos", fluid_vec3(fo, 0), {n, 3});
    w.put("vel", fluid_vec3(fo, 1), {n, 3});
    w.put("density", fluid_density(fo), {n});
    return 0;
}
