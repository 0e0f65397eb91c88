/*
 * sph2o -- headless driver with SPH2O's command line (src/main.cpp:16-91):
 *
 *   sph2o -c scene.json [-g true|false] [-o true|false] [-f frame]
 *         [--steps N] [--device D] [--quiet]
 *
 *   -c   scene JSON (SPH2O schema, SceneLoader.cpp:11-209)
 *   -g   "true" asks for the OpenGL viewer, which does not exist on this
 *        build (no graphics stack): a note is printed and the run is headless
 *   -o   "true" writes <scene>_NNNN.json frames every 1/fps of simulated time
 *        in SceneLoader::writeFluid's format (SceneLoader.cpp:211-275)
 *   -f   resume from frame file <scene>_NNNN.json and continue (SPH2O loads it
 *        and exits, SPHSimulation.cpp:547-548)
 *   --steps N   stop after N steps at the latest
 *
 * Steps run while startTime <= time <= endTime (SPHSimulation::step,
 * SPHSimulation.cpp:157-191) and the loop ends when time passes endTime
 * (SPH2O's run() never refreshes its copy of the time and spins,
 * SPHSimulation.cpp:193-199). Frame bookkeeping follows TimeHelper::hasToSave
 * (TimeHelper.h:100-110) in float, as the reference does.
 */
#include "../../include/sph2o_cuda.h"
#include "json_lite.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

const char* method_label(int m)
{
    switch (m) {
    case SPH_WCSPH: return "Weakly Compressible SPH";
    case SPH_PCISPH: return "Predictive-Corrective Incompressible SPH";
    case SPH_DFSPH: return "Divergence-Free SPH";
    default: return "none";
    }
}

std::string frame_path(const std::string& scene, unsigned frame)
{
    std::string num = std::to_string(frame);
    while (num.size() < 4) num = "0" + num;  /* SceneLoader::MAX_DIGITS = 4 */
    std::string p = scene;
    const std::string ext = ".json";
    if (p.size() >= ext.size() && p.compare(p.size() - ext.size(), ext.size(), ext) == 0)
        p.insert(p.size() - ext.size(), "_" + num);
    else
        p += "_" + num + ext;
    return p;
}

/* Keys in the order nlohmann::json (an ordered std::map) writes them. */
bool write_frame(const std::string& path, const std::vector<float>& x, const std::vector<float>& v, size_t n_active,
                 double time, float dt)
{
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    const size_t n = x.size() / 3;
    std::fprintf(f, "{\"numActiveParticles\":%zu,\"numParticles\":%zu,\"positions\":[", n_active, n);
    for (size_t i = 0; i < n; ++i)
        std::fprintf(f, "%s[%s,%s,%s]", i ? "," : "", sphjson::format_double((double)x[3 * i]).c_str(),
                     sphjson::format_double((double)x[3 * i + 1]).c_str(),
                     sphjson::format_double((double)x[3 * i + 2]).c_str());
    std::fprintf(f, "],\"time\":%s,\"timeStep\":%s,\"velocities\":[", sphjson::format_double((double)(float)time).c_str(),
                 sphjson::format_double((double)dt).c_str());
    for (size_t i = 0; i < n; ++i)
        std::fprintf(f, "%s[%s,%s,%s]", i ? "," : "", sphjson::format_double((double)v[3 * i]).c_str(),
                     sphjson::format_double((double)v[3 * i + 1]).c_str(),
                     sphjson::format_double((double)v[3 * i + 2]).c_str());
    std::fprintf(f, "]}");
    return std::fclose(f) == 0;
}

bool read_frame(const std::string& path, size_t n, std::vector<float>& x, std::vector<float>& v, double& time,
                float& dt, std::string& err)
{
    std::ifstream in(path);
    if (!in) { err = "cannot read " + path; return false; }
    std::stringstream ss;
    ss << in.rdbuf();
    try {
        const sphjson::Value root = sphjson::parse(ss.str());
        if ((size_t)root.get("numParticles").as_number() != n) {
            err = "Different fluid configuration scene_fluid != frame_fluid";
            return false;
        }
        const sphjson::Value& P = root.get("positions");
        const sphjson::Value& V = root.get("velocities");
        if (P.size() != n || V.size() != n) { err = "frame arrays have the wrong length"; return false; }
        x.resize(3 * n);
        v.resize(3 * n);
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                x[3 * i + k] = (float)P.at(i).at(k).as_number();
                v[3 * i + k] = (float)V.at(i).at(k).as_number();
            }
        time = (double)(float)root.get("time").as_number();
        dt = (float)root.get("timeStep").as_number();
    } catch (const std::exception& e) {
        err = e.what();
        return false;
    }
    return true;
}

struct Args {
    std::string scene;
    bool output = false, graphics = false, quiet = false;
    long frame = -1, steps = -1;
    int device = 0;
};

bool parse_args(int argc, char** argv, Args& a)
{
    for (int i = 1; i < argc; ++i) {
        const std::string t = argv[i];
        auto val = [&]() -> std::string { return i + 1 < argc ? std::string(argv[++i]) : std::string(); };
        if (t == "-c") a.scene = val();
        else if (t == "-o") a.output = val() == "true";
        else if (t == "-g") a.graphics = val() == "true";
        else if (t == "-f") a.frame = std::atol(val().c_str());
        else if (t == "--steps") a.steps = std::atol(val().c_str());
        else if (t == "--device") a.device = std::atoi(val().c_str());
        else if (t == "--quiet") a.quiet = true;
        else if (t == "-h" || t == "--help") return false;
        else { std::fprintf(stderr, "unknown option %s\n", t.c_str()); return false; }
    }
    return !a.scene.empty();
}

} // namespace

int main(int argc, char** argv)
{
    Args a;
    if (!parse_args(argc, argv, a)) {
        std::fprintf(stderr, "usage: sph2o -c scene.json [-g true|false] [-o true|false] [-f frame] "
                             "[--steps N] [--device D] [--quiet]\n");
        return 2;
    }
    if (a.graphics)
        std::printf("graphics unavailable on this box (no OpenGL); running headless\n");
    std::printf("Importing scene from %s...\n", a.scene.c_str());
    sph_scene* scene = nullptr;
    if (sph_scene_load(a.scene.c_str(), &scene) != SPH_OK) {
        std::fprintf(stderr, "Cannot import scene! %s\n", sph_scene_error());
        return 1;
    }
    sph_scene_desc d;
    sph_scene_get_desc(scene, &d);
    if (sph_select_device(a.device) != SPH_OK) {
        std::fprintf(stderr, "%s\n", sph_global_error());
        return 1;
    }
    sph_ctx* ctx = nullptr;
    int rc = sph_create_from_scene(scene, &ctx);
    if (rc != SPH_OK) {
        std::fprintf(stderr, "init failed: %s\n", ctx ? sph_last_error(ctx) : sph_global_error());
        return 1;
    }
    const unsigned nf = sph_num_fluid(ctx);
    std::printf("Pressure solver:           %s\n", method_label(d.simulation_method));
    std::printf("Number of particles:       %u fluid, %u boundary\n", nf, sph_num_boundary(ctx));
    std::printf("Particle radius:           %g m (support radius %g m)\n", (double)d.particle_radius,
                4.0 * (double)d.particle_radius);

    /* TimeHelper state (TimeHelper.h:43-49): frame 1, lastTimeSave 0, float time */
    unsigned frame = 1;
    float last_save = 0.0f;
    float time = 0.0f;
    std::vector<float> x(3ull * nf), v(3ull * nf);
    if (a.frame >= 0 && sph_scene_num_emitters(scene) > 0) {
        /* SPH2O's importFluidState exits before it would restore emitters
           (SPHSimulation.cpp:547-551); there is no state to resume them from */
        std::fprintf(stderr, "resuming a scene with emitters is not supported\n");
        return 1;
    }
    if (a.frame >= 0) {
        double t = 0.0;
        float dt = 0.0f;
        std::string err;
        const std::string path = frame_path(a.scene, (unsigned)a.frame);
        std::printf("Importing fluid state from %s...\n", path.c_str());
        if (!read_frame(path, nf, x, v, t, dt, err)) {
            std::fprintf(stderr, "Cannot import fluid state %ld: %s\n", a.frame, err.c_str());
            return 1;
        }
        if (sph_set_state(ctx, x.data(), v.data()) != SPH_OK || sph_set_time(ctx, t, dt) != SPH_OK) {
            std::fprintf(stderr, "%s\n", sph_last_error(ctx));
            return 1;
        }
        time = (float)t;
        frame = (unsigned)a.frame + 1;
        last_save = (float)a.frame / d.fps;
    }

    const auto t0 = std::chrono::steady_clock::now();
    long steps = 0;
    unsigned long long its = 0, itsv = 0;
    while (time >= d.start_time && time <= d.end_time && (a.steps < 0 || steps < a.steps)) {
        sph_step_stats st;
        rc = sph_step(ctx, 1, &st);
        if (rc != SPH_OK && rc != SPH_ERR_NEIGHBOR_OVERFLOW) {
            std::fprintf(stderr, "step %ld failed: %s\n", steps, sph_last_error(ctx));
            return 1;
        }
        ++steps;
        its += st.total_iterations;
        itsv += st.total_iterations_v;
        time = time + st.dt;  /* SPHSimulation: setTime(getTime() + getTimeStep()) in float */
        if (time - last_save >= 1.0 / d.fps) {  /* TimeHelper::hasToSave */
            last_save = (float)frame / d.fps;
            if (a.output) {
                if (sph_get_state(ctx, x.data(), v.data(), nullptr) != SPH_OK) {
                    std::fprintf(stderr, "%s\n", sph_last_error(ctx));
                    return 1;
                }
                unsigned na = nf;
                sph_get_num_active(ctx, &na);
                const std::string path = frame_path(a.scene, frame);
                if (!write_frame(path, x, v, na, (double)time, st.dt)) std::fprintf(stderr, "Cannot write fluid state\n");
            }
            if (!a.quiet)
                std::printf("frame %u  t=%.5f s  dt=%.3g s  its=%u/%u\n", frame, (double)time, (double)st.dt,
                            st.iterations, st.iterations_v);
            ++frame;
        }
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("{\"steps\": %ld, \"sim_time\": %.9g, \"frames\": %u, \"wall_s\": %.6f, "
                "\"particle_steps_per_s\": %.6e, \"mean_iterations\": %.3f, \"mean_iterations_v\": %.3f}\n",
                steps, (double)time, frame - 1, secs, steps ? (double)nf * steps / secs : 0.0,
                steps ? (double)its / steps : 0.0, steps ? (double)itsv / steps : 0.0);
    sph_destroy(ctx);
    sph_scene_free(scene);
    return 0;
}
