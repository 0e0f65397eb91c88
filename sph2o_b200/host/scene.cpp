/*
 * Scene JSON loading and particle generation on the host.
 *
 * Restates, in this project's own code, what SPH2O does between reading a
 * scene file and the first solver step:
 *   - SceneLoader::readSceneInfo/readFluidInfo/readBoundaryInfo
 *     (src/SPH2O/SceneLoader.cpp:40-209): same keys, same conditional reads;
 *   - SPHSimulation::importScene (src/SPH2O/SPHSimulation.cpp:299-481): one
 *     fluid model, Akinci boundary objects built box, then sphere, then
 *     geometry per object;
 *   - FluidObject::build (src/SPH2O/FluidObject/FluidObject.cpp:30-61);
 *   - AkinciBoundaryObject::sampleCube / sampleSphere
 *     (src/SPH2O/BoundaryObject/AkinciBoundaryObject.cpp:97-153);
 *   - AkinciBoundaryObject::addGeometry (:74-95): OBJ "geometry" entries
 *     sampled at spacing * particleRadius * 2 (SPHSimulation.cpp:422-423)
 *     with scale 1, no translation and a fixed rotation of pi/2 about x
 *     (geometry.cpp holds the loader and the sampler).
 * The arithmetic keeps SPH2O's types operation by operation (float where the
 * reference computes in float, double where its unqualified pow/sin/cos/
 * round/floor calls resolve to the double overloads), so the generated
 * particles are bit-identical to the reference's. This file is compiled with
 * -ffp-contract=off for that reason.
 *
 * Emitters ("emitters" of the fluid model, SceneLoader.cpp:109-143) are
 * read into sph_emitter_desc and handed to the context by
 * sph_create_from_scene (FluidObject::addEmitter, FluidObject.cpp:177-194).
 *
 * With boundaryMethod 0 each boundary object contributes its first box as a
 * cube boundary (SPHSimulation.cpp:459-477), with the zero velocity factors
 * SPH2O's loader leaves it.
 *
 * A relative geometry path is opened as given (relative to the working
 * directory, as the reference does) and, failing that, relative to the
 * directory of the scene file.
 *
 * With boundaryMethod 1 (PCISPH boundary particles) the boxes and spheres
 * are sampled with PCISPHBoundaryObject's samplers, each point with its
 * normal, and the object's "normalFct"/"tangFct" are read
 * (PCISPHBoundaryObject.cpp:6-213, SceneLoader.cpp:168-195).
 *
 * Not supported (rejected with SPH_ERR_ARG): more than one fluid model;
 * more than one boundary object with boundaryMethod 1.
 */
#include "../../include/sph2o_cuda.h"
#include "geometry.h"
#include "json_lite.h"
#include "scene_rng.h"

#include <cmath>
#include <cstring>
#include <fstream>
#include <math.h>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

struct sph_scene {
    sph_scene_desc desc;
    std::vector<float> fluid;     /* n*3 */
    std::vector<float> fluid_v;   /* n*3 */
    std::vector<float> boundary;  /* nb*3 */
    std::vector<sph_emitter_desc> emitters;
    struct Cube { float mn[3], mx[3]; };
    std::vector<Cube> cubes;      /* boundary method 0: first box of each boundary object */
    /* boundary method 1: per-particle normals and the object's velocity factors */
    std::vector<float> boundary_normal; /* nb*3 */
    float normal_fct = 0.0f, tangential_fct = 0.0f;
    std::string path;
};

namespace {

thread_local std::string g_scene_error;

struct V3 { float x, y, z; };

float num(const sphjson::Value& v, const char* what) { return (float)v.as_number(what); }

V3 vec3(const sphjson::Value& v, const char* what)
{
    if (!v.is_array() || v.size() < 3) throw sphjson::JsonError(std::string("expected [x,y,z] for ") + what);
    return {num(v.at(0), what), num(v.at(1), what), num(v.at(2), what)};
}

/* FluidObject::build (FluidObject.cpp:30-61): lattice at spacing 2r,
   origin min + r, count floor((max - min) / 2r + 1e-5) per axis, k fastest. */
void build_lattice(const std::vector<std::pair<V3, V3>>& blocks, float radius, std::vector<float>& out)
{
    const float dist = 2.0f * radius;
    for (const auto& b : blocks) {
        const V3& lo = b.first;
        const V3& hi = b.second;
        const unsigned nx = (unsigned)::floor((double)((hi.x - lo.x) / dist + 1e-5f));
        const unsigned ny = (unsigned)::floor((double)((hi.y - lo.y) / dist + 1e-5f));
        const unsigned nz = (unsigned)::floor((double)((hi.z - lo.z) / dist + 1e-5f));
        const float ox = lo.x + radius, oy = lo.y + radius, oz = lo.z + radius;
        for (unsigned i = 0; i < nx; ++i)
            for (unsigned j = 0; j < ny; ++j)
                for (unsigned k = 0; k < nz; ++k) {
                    out.push_back((float)i * dist + ox);
                    out.push_back((float)j * dist + oy);
                    out.push_back((float)k * dist + oz);
                }
    }
}

/* AkinciBoundaryObject::sampleCube (AkinciBoundaryObject.cpp:97-123):
   single-layer hollow box, ceil(l / 2r) intervals per axis. */
void sample_cube(V3 lo, V3 hi, float radius, std::vector<float>& out)
{
    const float lx = std::fabs(lo.x - hi.x), ly = std::fabs(lo.y - hi.y), lz = std::fabs(lo.z - hi.z);
    const float two_r = 2.0f * radius;
    const float nx = std::ceil(lx / two_r), ny = std::ceil(ly / two_r), nz = std::ceil(lz / two_r);
    const float dx = lx / nx, dy = ly / ny, dz = lz / nz;
    for (unsigned i = 0; (float)i <= nx; i++)
        for (unsigned j = 0; (float)j <= ny; j++)
            for (unsigned k = 0; (float)k <= nz; k++)
                if ((i == 0 || (float)i == nx) || (j == 0 || (float)j == ny) || (k == 0 || (float)k == nz)) {
                    out.push_back((float)i * dx + lo.x);
                    out.push_back((float)j * dy + lo.y);
                    out.push_back((float)k * dz + lo.z);
                }
}

/* AkinciBoundaryObject::sampleSphere (AkinciBoundaryObject.cpp:125-153):
   equal-area points with 1.5x overlap; the trigonometry runs in double
   exactly where the reference's unqualified calls do. float_count: the
   point count formed in float, as PCISPHBoundaryObject::sampleSphere
   (PCISPHBoundaryObject.cpp:185-213) forms it; the rest is the same. */
void sample_sphere(V3 c, float radius, float particle_radius, std::vector<float>& out, bool float_count = false)
{
    const float separation = 1.5f;
    const unsigned num_parts =
        float_count ? (unsigned)::floor((double)((float)(4.0 * M_PI) * radius * radius /
                                                 ((float)M_PI * particle_radius * particle_radius) * separation))
                    : (unsigned)::floor(4.0 * M_PI * (double)radius * (double)radius /
                                        (M_PI * (double)particle_radius * (double)particle_radius) *
                                        (double)separation);
    if (num_parts == 0) return;
    const float a = (float)(4.0 * M_PI) / (float)num_parts;
    const float d = (float)::sqrt((double)a);
    const unsigned m_theta = (unsigned)::round(M_PI / (double)d);
    const float d_theta = (float)M_PI / (float)m_theta;
    const float d_phi = a / d_theta;
    for (unsigned m = 0; m < m_theta; ++m) {
        const float theta = (float)(M_PI * ((double)m + 0.5)) / (float)m_theta;
        const unsigned m_phi = (unsigned)::round(2.0 * M_PI * ::sin((double)theta) / (double)d_phi);
        for (unsigned n = 0; n < m_phi; ++n) {
            const float phi = (float)(2.0 * M_PI) * (float)n / (float)m_phi;
            const float x = (float)(::sin((double)theta) * ::cos((double)phi));
            const float y = (float)(::sin((double)theta) * ::sin((double)phi));
            const float z = (float)::cos((double)theta);
            out.push_back(radius * x + c.x);
            out.push_back(radius * y + c.y);
            out.push_back(radius * z + c.z);
        }
    }
}

/* glm::normalize in float: v * (1 / sqrt((x x + y y) + z z)) */
V3 normalized(V3 v)
{
    const float inv = 1.0f / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x * inv, v.y * inv, v.z * inv};
}
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 scale(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
V3 div3(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }

/* A box side as PCISPHBoundaryObject::sampleCube measures it: its
   unqualified abs takes an int there (PCISPHBoundaryObject.cpp:61-63), so
   the float difference is truncated to a whole number first. A side that
   truncates to 0 would give the reference 0/0 spacings (NaN particles):
   refused here. */
float pcisph_side(float lo, float hi, const char* axis)
{
    const float d = lo - hi;
    if (!(std::fabs(d) < 2147483648.0f)) throw std::invalid_argument("PCISPH boundary box too large");
    const int t = std::abs((int)d);
    if (t == 0)
        throw std::invalid_argument(std::string("PCISPH boundary box side along ") + axis +
                                    " is shorter than 1: SPH2O truncates these sides to whole numbers");
    return (float)t;
}

/* PCISPHBoundaryObject::sampleCube (PCISPHBoundaryObject.cpp:52-183): a
   hollow box at ceil(l / 0.45h) intervals per axis, each point with the
   normal of its face, edge (normalised mean of two face normals) or corner
   (of three), times inv (1 for an inverted box, the container, else -1). */
void sample_cube_pcisph(V3 lo, V3 hi, float h, float inv, std::vector<float>& pts, std::vector<float>& nrm)
{
    const float lx = pcisph_side(lo.x, hi.x, "x"), ly = pcisph_side(lo.y, hi.y, "y"), lz = pcisph_side(lo.z, hi.z, "z");
    const float sp = 0.45f * h;
    const unsigned nx = (unsigned)::ceil((double)(lx / sp)), ny = (unsigned)::ceil((double)(ly / sp)),
                   nz = (unsigned)::ceil((double)(lz / sp));
    const float dx = lx / (float)nx, dy = ly / (float)ny, dz = lz / (float)nz;
    const V3 L{1, 0, 0}, R{-1, 0, 0}, T{0, -1, 0}, B{0, 1, 0}, F{0, 0, -1}, K{0, 0, 1}; /* K: behind */
    auto edge = [](V3 a, V3 b) { return normalized(scale(add(a, b), 0.5f)); };
    auto corner = [](V3 a, V3 b, V3 c) { return normalized(div3(add(add(a, b), c), 3.0f)); };
    const V3 LB = edge(L, B), KB = edge(K, B), FB = edge(F, B), RB = edge(R, B);
    const V3 LT = edge(L, T), KT = edge(K, T), FT = edge(F, T), RT = edge(R, T);
    const V3 LK = edge(L, K), RK = edge(R, K), RF = edge(R, F), LF = edge(L, F);
    const V3 LKB = corner(L, K, B), RKB = corner(R, K, B), LFB = corner(L, F, B), RFB = corner(R, F, B);
    const V3 LKT = corner(L, K, T), RKT = corner(R, K, T), LFT = corner(L, F, T), RFT = corner(R, F, T);
    for (unsigned i = 0; i <= nx; i++)
        for (unsigned j = 0; j <= ny; j++)
            for (unsigned k = 0; k <= nz; k++) {
                const bool i0 = i == 0, iN = i == nx, im = i > 0 && i < nx;
                const bool j0 = j == 0, jN = j == ny, jm = j > 0 && j < ny;
                const bool k0 = k == 0, kN = k == nz, km = k > 0 && k < nz;
                if (!(i0 || iN || j0 || jN || k0 || kN)) continue;
                pts.push_back((float)i * dx + lo.x);
                pts.push_back((float)j * dy + lo.y);
                pts.push_back((float)k * dz + lo.z);
                /* the reference's if-chain, first match wins */
                V3 n;
                if (i0 && j0 && k0) n = LKB;
                else if (iN && j0 && k0) n = RKB;
                else if (i0 && j0 && kN) n = LFB;
                else if (iN && j0 && kN) n = RFB;
                else if (i0 && jN && k0) n = LKT;
                else if (iN && jN && k0) n = RKT;
                else if (i0 && jN && kN) n = LFT;
                else if (iN && jN && kN) n = RFT;
                else if (i0 && j0 && km) n = LB;
                else if (im && j0 && k0) n = KB;
                else if (im && j0 && kN) n = FB;
                else if (iN && j0 && km) n = RB;
                else if (i0 && jN && km) n = LT;
                else if (im && jN && k0) n = KT;
                else if (im && jN && kN) n = FT;
                else if (iN && jN && km) n = RT;
                else if (i0 && jm && k0) n = LK;
                else if (iN && jm && k0) n = RK;
                else if (iN && jm && kN) n = RF;
                else if (i0 && jm && kN) n = LF;
                else if (i0 && jm && km) n = L;
                else if (iN && jm && km) n = R;
                else if (im && jN && km) n = T;
                else if (im && j0 && km) n = B;
                else if (im && jm && kN) n = F;
                else n = K; /* im && jm && k0 */
                nrm.push_back(inv * n.x);
                nrm.push_back(inv * n.y);
                nrm.push_back(inv * n.z);
            }
}

unsigned uint_field(const sphjson::Value& cfg, const char* key)
{
    const double d = cfg.get(key).as_number(key);
    if (d < 0) throw sphjson::JsonError(std::string(key) + " must be non-negative");
    return (unsigned)d;
}

/* AkinciBoundaryObject::addGeometry (AkinciBoundaryObject.cpp:78-80): the
   fixed placement of every scene geometry; the angle is M_PI * 0.5 rounded
   to the reference's float Real */
const float kGeomScale[3] = {1.0f, 1.0f, 1.0f};
const float kGeomTranslate[3] = {0.0f, 0.0f, 0.0f};
const float kGeomRotate[3] = {(float)(M_PI * 0.5), 0.0f, 0.0f};

/* The path as given when it opens (the reference's behaviour), else a
   relative path taken from the scene file's directory. */
std::string resolve_geometry(const std::string& file, const std::string& scene_path)
{
    if (std::ifstream(file) || file.empty() || file[0] == '/' || scene_path.empty()) return file;
    const size_t slash = scene_path.find_last_of('/');
    if (slash == std::string::npos) return file;
    return scene_path.substr(0, slash + 1) + file;
}

sph_scene* build_scene(const std::string& text, const std::string& path)
{
    const sphjson::Value root = sphjson::parse(text);
    auto scene = std::make_unique<sph_scene>();
    sph_scene_desc& d = scene->desc;
    std::memset(&d, 0, sizeof d);
    scene->path = path;

    /* SceneLoader::readSceneInfo (SceneLoader.cpp:40-78) */
    const sphjson::Value& c = root.get("Configuration");
    d.start_time = num(c.get("startTime"), "startTime");
    d.end_time = num(c.get("endTime"), "endTime");
    d.time_step = num(c.get("timeStep"), "timeStep");
    d.fps = num(c.get("fps"), "fps");
    d.min_time_step = num(c.get("minTimeStep"), "minTimeStep");
    d.max_time_step = num(c.get("maxTimeStep"), "maxTimeStep");
    d.cfl_factor = num(c.get("cflFactor"), "cflFactor");
    d.particle_radius = num(c.get("particleRadius"), "particleRadius");
    d.boundary_method = (int)c.get("boundaryMethod").as_number("boundaryMethod");
    d.simulation_method = (int)c.get("simulationMethod").as_number("simulationMethod");
    const V3 g = vec3(c.get("gravity"), "gravity");
    d.gravity[0] = g.x; d.gravity[1] = g.y; d.gravity[2] = g.z;
    if (d.simulation_method == SPH_WCSPH) {
        d.stiffness = num(c.get("stiffness"), "stiffness");
        d.gamma = num(c.get("gamma"), "gamma");
    } else if (d.simulation_method == SPH_PCISPH) {
        d.eta = num(c.get("eta"), "eta");
        d.min_iterations = uint_field(c, "minIterations");
        d.max_iterations = uint_field(c, "maxIterations");
    } else if (d.simulation_method == SPH_DFSPH) {
        d.eta = num(c.get("eta"), "eta");
        d.eta_v = num(c.get("etaV"), "etaV");
        d.min_iterations = uint_field(c, "minIterations");
        d.max_iterations = uint_field(c, "maxIterations");
        d.min_iterations_v = uint_field(c, "minIterationsV");
        d.max_iterations_v = uint_field(c, "maxIterationsV");
    } else {
        throw sphjson::JsonError("simulationMethod must be 0 (WCSPH), 1 (PCISPH) or 2 (DFSPH)");
    }
    if (d.boundary_method < SPH_BOUNDARY_CUBE || d.boundary_method > SPH_BOUNDARY_AKINCI)
        throw std::invalid_argument("boundaryMethod must be 0 (cube), 1 (PCISPH) or 2 (Akinci)");

    /* SceneLoader::readFluidInfo (SceneLoader.cpp:80-146) */
    const sphjson::Value& fl = root.get("Fluid");
    d.viscosity_method = (int)fl.get("viscosityMethod").as_number("viscosityMethod");
    d.surface_tension_method = (int)fl.get("surfaceTensionMethod").as_number("surfaceTensionMethod");
    d.adhesion_method = (int)fl.get("adhesionMethod").as_number("adhesionMethod");
    const sphjson::Value& models = fl.get("FluidModel");
    if (models.size() != 1) throw std::invalid_argument("exactly one FluidModel is supported");
    const sphjson::Value& fm = models.at(0);
    d.density0 = num(fm.get("density0"), "density0");
    if (d.viscosity_method > -1) {
        d.viscosity = num(fm.get("viscosity"), "viscosity");
        d.boundary_viscosity = num(fm.get("boundaryViscosity"), "boundaryViscosity");
    }
    if (d.surface_tension_method > -1) d.surface_tension = num(fm.get("surfaceTension"), "surfaceTension");
    if (d.adhesion_method > -1) d.adhesion = num(fm.get("adhesion"), "adhesion");
    if (const sphjson::Value* em = fm.find("emitters"))
        for (size_t i = 0; i < em->size(); ++i) {
            /* SceneLoader.cpp:128-143; rotation is glm::quat(w, x, y, z) */
            const sphjson::Value& e = em->at(i);
            sph_emitter_desc ed{};
            const V3 p = vec3(e.get("position"), "emitters.position");
            ed.position[0] = p.x; ed.position[1] = p.y; ed.position[2] = p.z;
            const sphjson::Value& q = e.get("rotation");
            if (!q.is_array() || q.size() < 4) throw sphjson::JsonError("expected [w,x,y,z] for emitters.rotation");
            for (int k = 0; k < 4; ++k) ed.rotation[k] = num(q.at(k), "emitters.rotation");
            ed.velocity = num(e.get("velocity"), "emitters.velocity");
            ed.num_particles = (unsigned)e.get("numParticles").as_number("emitters.numParticles");
            ed.start_time = num(e.get("startTime"), "emitters.startTime");
            ed.type = (int)e.get("type").as_number("emitters.type");
            ed.width = num(e.get("width"), "emitters.width");
            ed.height = num(e.get("height"), "emitters.height");
            ed.spacing = num(e.get("spacing"), "emitters.spacing");
            scene->emitters.push_back(ed);
        }
    std::vector<std::pair<V3, V3>> blocks;
    const sphjson::Value& fb = fm.get("fluidBlocks");
    for (size_t i = 0; i < fb.size(); ++i)
        blocks.push_back({vec3(fb.at(i).get("min"), "fluidBlocks.min"), vec3(fb.at(i).get("max"), "fluidBlocks.max")});

    build_lattice(blocks, d.particle_radius, scene->fluid);
    scene->fluid_v.assign(scene->fluid.size(), 0.0f);

    /* seeded jitter (scene_rng.h); absent keys leave the lattice as is */
    if (const sphjson::Value* jit = c.find("jitter")) {
        const float amp = (float)jit->as_number("jitter");
        const sphjson::Value* sv = c.find("jitterSeed");
        const uint64_t seed = sv ? (uint64_t)sv->as_number("jitterSeed") : 0ull;
        if (amp != 0.0f) {
            const size_t n = scene->fluid.size() / 3;
            for (size_t i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k)
                    scene->fluid[3 * i + k] += sph_jitter_offset(seed, i, k, amp, d.particle_radius);
        }
    }

    /* SceneLoader::readBoundaryInfo (SceneLoader.cpp:148-209) + importScene
       (:459-477) for the cube method: the first box of each boundary object */
    if (d.boundary_method == SPH_BOUNDARY_CUBE) {
        if (const sphjson::Value* bnd = root.find("Boundary"))
            for (size_t i = 0; i < bnd->size(); ++i) {
                const sphjson::Value* boxes = bnd->at(i).find("box");
                if (!boxes || boxes->size() == 0)
                    throw std::invalid_argument("a cube boundary object needs a box");
                const V3 mn = vec3(boxes->at(0).get("min"), "box.min"), mx = vec3(boxes->at(0).get("max"), "box.max");
                scene->cubes.push_back({{mn.x, mn.y, mn.z}, {mx.x, mx.y, mx.z}});
            }
        return scene.release();
    }
    /* SceneLoader::readBoundaryInfo with the PCISPH method's keys
       (SceneLoader.cpp:168-195) + importScene (:428-453): boxes, then
       spheres, per object; "geometry" entries are not read for this method */
    if (d.boundary_method == SPH_BOUNDARY_PCISPH) {
        if (const sphjson::Value* bnd = root.find("Boundary")) {
            if (bnd->size() > 1)
                throw std::invalid_argument("the PCISPH boundary method takes one boundary object (SPH2O indexes an "
                                            "object's arrays with the candidates of all objects)");
            const float h = 4.0f * d.particle_radius;
            for (size_t i = 0; i < bnd->size(); ++i) {
                const sphjson::Value& b = bnd->at(i);
                scene->normal_fct = num(b.get("normalFct"), "normalFct");
                scene->tangential_fct = num(b.get("tangFct"), "tangFct");
                if (const sphjson::Value* boxes = b.find("box"))
                    for (size_t j = 0; j < boxes->size(); ++j) {
                        const sphjson::Value& bx = boxes->at(j);
                        const float inv = bx.get("inverted").as_bool("box.inverted") ? 1.0f : -1.0f;
                        sample_cube_pcisph(vec3(bx.get("min"), "box.min"), vec3(bx.get("max"), "box.max"), h, inv,
                                           scene->boundary, scene->boundary_normal);
                    }
                if (const sphjson::Value* sph = b.find("sphere"))
                    for (size_t j = 0; j < sph->size(); ++j) {
                        const sphjson::Value& sv = sph->at(j);
                        const float inv = sv.get("inverted").as_bool("sphere.inverted") ? 1.0f : -1.0f;
                        const V3 c = vec3(sv.get("pos"), "sphere.pos");
                        const size_t first = scene->boundary.size();
                        sample_sphere(c, num(sv.get("radius"), "sphere.radius"), d.particle_radius, scene->boundary,
                                      true);
                        /* n = inv (centre - point) (PCISPHBoundaryObject.cpp:40) */
                        for (size_t q = first; q < scene->boundary.size(); q += 3) {
                            scene->boundary_normal.push_back(inv * (c.x - scene->boundary[q]));
                            scene->boundary_normal.push_back(inv * (c.y - scene->boundary[q + 1]));
                            scene->boundary_normal.push_back(inv * (c.z - scene->boundary[q + 2]));
                        }
                    }
            }
        }
        return scene.release();
    }
    /* SceneLoader::readBoundaryInfo (SceneLoader.cpp:148-209) + importScene (:407-426) */
    if (const sphjson::Value* bnd = root.find("Boundary")) {
        for (size_t i = 0; i < bnd->size(); ++i) {
            const sphjson::Value& b = bnd->at(i);
            if (const sphjson::Value* boxes = b.find("box"))
                for (size_t j = 0; j < boxes->size(); ++j)
                    sample_cube(vec3(boxes->at(j).get("min"), "box.min"), vec3(boxes->at(j).get("max"), "box.max"),
                                d.particle_radius, scene->boundary);
            if (const sphjson::Value* sph = b.find("sphere"))
                for (size_t j = 0; j < sph->size(); ++j)
                    sample_sphere(vec3(sph->at(j).get("pos"), "sphere.pos"),
                                  num(sph->at(j).get("radius"), "sphere.radius"), d.particle_radius, scene->boundary);
            if (const sphjson::Value* geo = b.find("geometry"))
                for (size_t j = 0; j < geo->size(); ++j) {
                    const float spacing = num(geo->at(j).get("spacing"), "geometry.spacing");
                    const std::string file = resolve_geometry(geo->at(j).get("path").as_string("geometry.path"), path);
                    std::vector<float> pts;
                    sphgeo::sample_geometry(file, spacing * d.particle_radius * 2.0f, kGeomScale, kGeomTranslate,
                                            kGeomRotate, pts);
                    scene->boundary.insert(scene->boundary.end(), pts.begin(), pts.end());
                }
        }
    }
    return scene.release();
}

/* Copies `pts` out through the two-call convention of the mesh entry points. */
int emit_samples(const std::vector<float>& pts, float* samples, size_t capacity, size_t* count)
{
    const size_t n = pts.size() / 3;
    if (count) *count = n;
    if (!samples) return SPH_OK;
    if (capacity < n) {
        g_scene_error = "sample buffer holds " + std::to_string(capacity) + " points, " + std::to_string(n) +
                        " needed";
        return SPH_ERR_CAPACITY;
    }
    std::memcpy(samples, pts.data(), pts.size() * sizeof(float));
    return SPH_OK;
}

template <class F>
int guarded(F&& f)
{
    try {
        const int rc = f();
        if (rc == SPH_OK) g_scene_error.clear();
        return rc;
    } catch (const sphgeo::StatusError& e) {
        g_scene_error = e.what();
        return e.code;
    } catch (const std::invalid_argument& e) {
        g_scene_error = e.what();
        return SPH_ERR_ARG;
    } catch (const std::length_error& e) {
        g_scene_error = e.what();
        return SPH_ERR_CAPACITY;
    } catch (const std::exception& e) {
        g_scene_error = e.what();
        return SPH_ERR_IO;
    }
}

int load_common(const std::string& text, const std::string& path, sph_scene** out)
{
    if (!out) { g_scene_error = "null output pointer"; return SPH_ERR_ARG; }
    *out = nullptr;
    try {
        *out = build_scene(text, path);
        g_scene_error.clear();
        return SPH_OK;
    } catch (const sphjson::JsonError& e) {
        g_scene_error = e.what();
        return SPH_ERR_IO;
    } catch (const sphgeo::StatusError& e) {
        g_scene_error = e.what();
        return e.code;
    } catch (const std::invalid_argument& e) {
        g_scene_error = e.what();
        return SPH_ERR_ARG;
    } catch (const std::length_error& e) {
        g_scene_error = e.what();
        return SPH_ERR_CAPACITY;
    } catch (const std::exception& e) {
        g_scene_error = e.what();
        return SPH_ERR_IO;
    }
}

} // namespace

extern "C" {

int sph_scene_load(const char* json_path, sph_scene** out)
{
    if (!json_path) { g_scene_error = "null path"; return SPH_ERR_ARG; }
    std::ifstream f(json_path);
    if (!f) { g_scene_error = std::string("cannot read ") + json_path; return SPH_ERR_IO; }
    std::stringstream ss;
    ss << f.rdbuf();
    return load_common(ss.str(), json_path, out);
}

int sph_scene_parse(const char* json_text, sph_scene** out)
{
    if (!json_text) { g_scene_error = "null text"; return SPH_ERR_ARG; }
    return load_common(json_text, "", out);
}

int sph_scene_get_desc(const sph_scene* s, sph_scene_desc* out)
{
    if (!s || !out) return SPH_ERR_ARG;
    *out = s->desc;
    return SPH_OK;
}

unsigned sph_scene_num_fluid(const sph_scene* s) { return s ? (unsigned)(s->fluid.size() / 3) : 0u; }
unsigned sph_scene_num_emitters(const sph_scene* s) { return s ? (unsigned)s->emitters.size() : 0u; }
unsigned sph_scene_num_cube_boundaries(const sph_scene* s) { return s ? (unsigned)s->cubes.size() : 0u; }

int sph_scene_get_cube_boundary(const sph_scene* s, unsigned k, float mn[3], float mx[3], float* normal_fct,
                                float* tangential_fct)
{
    if (!s || k >= s->cubes.size()) return SPH_ERR_ARG;
    for (int q = 0; q < 3; ++q) {
        if (mn) mn[q] = s->cubes[k].mn[q];
        if (mx) mx[q] = s->cubes[k].mx[q];
    }
    /* SceneLoader::readBoundaryInfo reads normalFct / tangFct only for the
       PCISPH method (SceneLoader.cpp:168-172): the cube objects get the zero
       of a value-initialised Boundary */
    if (normal_fct) *normal_fct = 0.0f;
    if (tangential_fct) *tangential_fct = 0.0f;
    return SPH_OK;
}

int sph_scene_get_emitter(const sph_scene* s, unsigned k, sph_emitter_desc* out)
{
    if (!s || !out || k >= s->emitters.size()) return SPH_ERR_ARG;
    *out = s->emitters[k];
    return SPH_OK;
}
unsigned sph_scene_num_boundary(const sph_scene* s) { return s ? (unsigned)(s->boundary.size() / 3) : 0u; }

int sph_scene_get_boundary_normals(const sph_scene* s, float* xyz, float* normal_fct, float* tangential_fct)
{
    if (!s || s->desc.boundary_method != SPH_BOUNDARY_PCISPH) return SPH_ERR_ARG;
    if (xyz) std::memcpy(xyz, s->boundary_normal.data(), s->boundary_normal.size() * sizeof(float));
    if (normal_fct) *normal_fct = s->normal_fct;
    if (tangential_fct) *tangential_fct = s->tangential_fct;
    return SPH_OK;
}

int sph_scene_get_fluid(const sph_scene* s, float* xyz, float* v)
{
    if (!s) return SPH_ERR_ARG;
    if (xyz) std::memcpy(xyz, s->fluid.data(), s->fluid.size() * sizeof(float));
    if (v) std::memcpy(v, s->fluid_v.data(), s->fluid_v.size() * sizeof(float));
    return SPH_OK;
}

int sph_scene_get_boundary(const sph_scene* s, float* xyz)
{
    if (!s) return SPH_ERR_ARG;
    if (xyz) std::memcpy(xyz, s->boundary.data(), s->boundary.size() * sizeof(float));
    return SPH_OK;
}

const char* sph_scene_error(void) { return g_scene_error.c_str(); }

int sph_load_obj(const char* obj_path, const float scale[3], float* vertices, size_t vertex_capacity,
                 size_t* num_vertices, unsigned* faces, size_t face_capacity, size_t* num_faces)
{
    if (!obj_path) {
        g_scene_error = "null path";
        return SPH_ERR_ARG;
    }
    const float one[3] = {1.0f, 1.0f, 1.0f};
    return guarded([&] {
        std::vector<float> v;
        std::vector<unsigned> f;
        sphgeo::load_obj(obj_path, scale ? scale : one, v, f);
        if (num_vertices) *num_vertices = v.size() / 3;
        if (num_faces) *num_faces = f.size() / 3;
        if ((vertices && vertex_capacity < v.size() / 3) || (faces && face_capacity < f.size() / 3)) {
            g_scene_error = "output arrays too small for the mesh";
            return (int)SPH_ERR_CAPACITY;
        }
        if (vertices) std::memcpy(vertices, v.data(), v.size() * sizeof(float));
        if (faces) std::memcpy(faces, f.data(), f.size() * sizeof(unsigned));
        return (int)SPH_OK;
    });
}

int sph_sample_mesh(const float* vertices, unsigned num_vertices, const unsigned* faces, unsigned num_faces,
                    float max_distance, float* samples, size_t capacity, size_t* count)
{
    return guarded([&] {
        std::vector<float> pts;
        sphgeo::sample_mesh(vertices, num_vertices, faces, num_faces, max_distance, pts);
        return emit_samples(pts, samples, capacity, count);
    });
}

int sph_sample_geometry(const char* obj_path, float max_distance, const float scale[3], const float translate[3],
                        const float rotate[3], float* samples, size_t capacity, size_t* count)
{
    if (!obj_path) {
        g_scene_error = "null path";
        return SPH_ERR_ARG;
    }
    const float one[3] = {1.0f, 1.0f, 1.0f}, zero[3] = {0.0f, 0.0f, 0.0f};
    return guarded([&] {
        std::vector<float> pts;
        sphgeo::sample_geometry(obj_path, max_distance, scale ? scale : one, translate ? translate : zero,
                                rotate ? rotate : zero, pts);
        return emit_samples(pts, samples, capacity, count);
    });
}

void sph_scene_free(sph_scene* s) { delete s; }

int sph_create_from_scene(const sph_scene* s, sph_ctx** out)
{
    if (!s || !out) return SPH_ERR_ARG;
    int rc = sph_create(&s->desc, out);
    if (rc != SPH_OK) return rc;
    sph_ctx* ctx = *out;
    if ((rc = sph_set_fluid(ctx, sph_scene_num_fluid(s), s->fluid.data(), s->fluid_v.data())) != SPH_OK ||
        (rc = sph_set_boundary(ctx, sph_scene_num_boundary(s), s->boundary.data())) != SPH_OK)
        return rc; /* the context stays valid; sph_last_error(ctx) explains */
    if (s->desc.boundary_method == SPH_BOUNDARY_PCISPH &&
        (rc = sph_set_boundary_normals(ctx, sph_scene_num_boundary(s), s->boundary_normal.data(), s->normal_fct,
                                       s->tangential_fct)) != SPH_OK)
        return rc;
    for (const sph_scene::Cube& b : s->cubes)
        if ((rc = sph_add_cube_boundary(ctx, b.mn, b.mx, 0.0f, 0.0f)) != SPH_OK) return rc;
    for (const sph_emitter_desc& e : s->emitters)
        if ((rc = sph_add_emitter(ctx, &e)) != SPH_OK) return rc;
    if ((rc = sph_init(ctx)) != SPH_OK) return rc;
    return SPH_OK;
}

} // extern "C"
