/*
 * GPUSolver: SPH2O's solver interface (class SPHSolver,
 * inc/SPH2O/SPHSolver/SPHSolver.h:6-48) implemented on top of the C ABI of
 * sph2o_cuda.h, so that SPHSimulation::init / step / SceneLoader::writeFluid
 * run unchanged while the step itself runs on the GPU.
 *
 * This header is compiled INSIDE SPH2O: it includes SPH2O's own headers
 * (include path: SPH2O's inc/, extern/, extern/glm/inc) and links
 * libsph2o_cuda.so. It is the reference-side binding of the drop-in.
 *
 * Use: after the scene is imported (SceneLoader configured the CPU solver of
 * the chosen method with the scene's parameters) and before
 * SPHSimulation::init(), replace the simulation's solver by
 *     new GPUSolver(configured_cpu_solver)
 * GPUSolver reads every parameter from the simulation, its fluid object's
 * non-pressure forces and the configured solver, takes ownership of that
 * solver and deletes it. In SPH2O itself that is one line in
 * SPHSimulation::init() (src/SPH2O/SPHSimulation.cpp:116-125) behind a
 * switch, e.g. `if (useGPU) solver = new GPUSolver(solver);` before
 * `solver->init()`.
 *
 * What it replaces:
 *   init()  -- SPHSolver::init of WCSPH/PCISPH/DFSPH (WCSPHSolver.cpp:10-12,
 *              PCISPHSolver.cpp:11-18, DFSPHSolver.cpp:22-31): creates a
 *              context, uploads the fluid and boundary particles, sph_init;
 *   step()  -- WCSPHSolver::step (WCSPHSolver.cpp:14-78), PCISPHSolver::step
 *              (PCISPHSolver.cpp:20-80), DFSPHSolver::step
 *              (DFSPHSolver.cpp:33-107): one sph_step; the simulation's time
 *              and time step are updated as the CPU solvers update them, and
 *              when SPHSimulation::step is about to save a frame
 *              (TimeHelper::hasToSave, TimeHelper.h:100-110, checked right
 *              after solver->step(), SPHSimulation.cpp:168-184) the state is
 *              copied back into the fluid object first, so
 *              SceneLoader::writeFluid writes the current positions and
 *              velocities;
 *   pull()  -- copies positions, velocities and densities back on demand
 *              (for a viewer or any reader of the FluidObject arrays).
 * Covered: one fluid model without emitters, Akinci boundary particles
 * (boundaryMethod 2), every solver, viscosity / surface tension / adhesion
 * model the ABI has. Anything else throws std::runtime_error from init().
 */
#ifndef SPH2O_GPU_SOLVER_HPP
#define SPH2O_GPU_SOLVER_HPP

#include "SPH2O/SPHSimulation.h"
#include "SPH2O/SPHSolver/DFSPHSolver.h"
#include "SPH2O/SPHSolver/PCISPHSolver.h"
#include "SPH2O/SPHSolver/SPHSolver.h"
#include "SPH2O/SPHSolver/WCSPHSolver.h"
#include "SPH2O/NonPressureForce/AdhesionForce.h"
#include "SPH2O/NonPressureForce/ArtificialViscosity.h"
#include "SPH2O/NonPressureForce/StandardViscosityForce.h"
#include "SPH2O/NonPressureForce/SurfaceTensionAkinci.h"
#include "SPH2O/NonPressureForce/XSPHViscosity.h"

#include "sph2o_cuda.h"

#include <stdexcept>
#include <string>
#include <vector>

namespace sph2o_gpu_detail {
/* Members without a public getter, read through the derived-class access
   rule (no change to SPH2O): DFSPHSolver::cflFactor and
   SPHSimulation::activeSave. */
struct DFSPHParams : DFSPHSolver {
    static Real cfl(DFSPHSolver* s) { return s->*(&DFSPHParams::cflFactor); }
};
struct SimulationFlags : SPHSimulation {
    static bool saving(SPHSimulation* s) { return s->*(&SimulationFlags::activeSave); }
};
} // namespace sph2o_gpu_detail

class GPUSolver : public SPHSolver {
public:
    /* `configured`: the CPU solver SceneLoader set up for the scene (owned
       from here on). */
    explicit GPUSolver(SPHSolver* configured) : cpu_(configured)
    {
        iterations = 0;
        steps = 0;
        sumIterations = 0;
        maxVel = 0;
        if (configured) {
            minIterations = configured->getMinIterations();
            maxIterations = configured->getMaxIterations();
            maxError = configured->getMaxError();
        }
    }
    ~GPUSolver() override
    {
        if (ctx_) sph_destroy(ctx_);
        delete cpu_;
    }

    void init() override
    {
        SPHSimulation* sim = SPHSimulation::getCurrent();
        if (sim->numberFluidModels() != 1) fail("one fluid model is supported");
        FluidObject* f = sim->getFluidModel(0);
        if (f->getNumActiveParticles() != f->getSize()) fail("fluid emitters are not supported by this binding");
        if (sim->getBoundaryHandlingMethod() != SPHSimulation::AKINCI_BOUNDARY_METHOD)
            fail("Akinci boundary particles (boundaryMethod 2) only");

        sph_scene_desc d{};
        d.simulation_method = sim->getSimulationMethod();
        d.boundary_method = SPH_BOUNDARY_AKINCI;
        d.viscosity_method = sim->getViscosityMethod();
        d.surface_tension_method = sim->getSurfaceTensionMethod();
        d.adhesion_method = sim->getAdhesionMethod();
        d.particle_radius = (float)sim->getParticleRadius();
        d.density0 = (float)f->getRefDensity();
        const Vector3r g = sim->getGravity();
        d.gravity[0] = (float)g.x; d.gravity[1] = (float)g.y; d.gravity[2] = (float)g.z;
        d.time_step = (float)sim->getTimeStep();
        d.fps = (float)sim->getFPS();
        d.min_time_step = (float)sim->getMinTimeStep();
        d.max_time_step = (float)sim->getMaxTimeStep();
        d.start_time = (float)sim->getStartTime();
        d.end_time = (float)sim->getEndTime();
        if (auto* w = dynamic_cast<WCSPHSolver*>(cpu_)) {
            d.stiffness = (float)w->getStiffness();
            d.gamma = (float)w->getGamma();
        } else if (auto* p = dynamic_cast<PCISPHSolver*>(cpu_)) {
            d.eta = (float)p->getMaxError();
            d.min_iterations = p->getMinIterations();
            d.max_iterations = p->getMaxIterations();
        } else if (auto* df = dynamic_cast<DFSPHSolver*>(cpu_)) {
            d.eta = (float)df->getMaxError();
            d.eta_v = (float)df->getMaxErrorV();
            d.min_iterations = df->getMinIterations();
            d.max_iterations = df->getMaxIterations();
            d.min_iterations_v = df->getMinIterationsV();
            d.max_iterations_v = df->getMaxIterationsV();
            d.cfl_factor = (float)sph2o_gpu_detail::DFSPHParams::cfl(df);
        } else {
            fail("the configured solver is not a WCSPH, PCISPH or DFSPH solver");
        }
        for (uint k = 0; k < f->numberNonPressureForces(); ++k) {
            NonPressureForce* npf = f->getNonPressureForce(k);
            if (auto* a = dynamic_cast<ArtificialViscosity*>(npf)) {
                d.viscosity = (float)a->getViscosityCoef();
                d.boundary_viscosity = (float)a->getBoundaryViscosityCoef();
            } else if (auto* s = dynamic_cast<StandardViscosityForce*>(npf)) {
                d.viscosity = (float)s->getViscosityCoef();
                d.boundary_viscosity = (float)s->getBoundaryViscosityCoef();
            } else if (auto* x = dynamic_cast<XSPHViscosity*>(npf)) {
                d.viscosity = (float)x->getViscosityCoef();
                d.boundary_viscosity = (float)x->getBoundaryViscosityCoef();
            } else if (auto* st = dynamic_cast<SurfaceTensionAkinci*>(npf)) {
                d.surface_tension = (float)st->getSurfaceTensionCoef();
            } else if (auto* ad = dynamic_cast<AdhesionForce*>(npf)) {
                d.adhesion = (float)ad->getAdhesionCoef();
            }
        }
        desc_ = d;
        if (sph_create(&d, &ctx_) != SPH_OK) fail(sph_global_error());

        const uint n = f->getSize();
        std::vector<float> x(3 * (size_t)n), v(3 * (size_t)n), b;
        for (uint i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                x[3 * (size_t)i + k] = (float)f->getPosition(i)[k];
                v[3 * (size_t)i + k] = (float)f->getVelocity(i)[k];
            }
        for (uint o = 0; o < sim->numberBoundaryModels(); ++o) {
            BoundaryObject* bo = sim->getBoundaryModel(o);
            for (uint i = 0; i < bo->getSize(); ++i)
                for (int k = 0; k < 3; ++k) b.push_back((float)bo->getPosition(i)[k]);
        }
        check(sph_set_fluid(ctx_, n, x.data(), v.data()));
        check(sph_set_boundary(ctx_, (unsigned)(b.size() / 3), b.data()));
        check(sph_init(ctx_));
        n_ = n;
    }

    void step() override
    {
        SPHSimulation* sim = SPHSimulation::getCurrent();
        sph_step_stats st{};
        check(sph_step(ctx_, 1, &st));
        sim->setTimeStep((Real)st.dt);
        sim->setTime((Real)st.time);
        iterations = st.iterations;
        sumIterations += st.iterations;
        maxVel = (Real)st.max_velocity;
        ++steps;
        if (sph2o_gpu_detail::SimulationFlags::saving(sim) && will_save(sim)) pull();
    }

    void resize() override {}

    /* Positions, velocities and densities back into the fluid object. */
    void pull()
    {
        std::vector<float> x(3 * (size_t)n_), v(3 * (size_t)n_), rho(n_);
        check(sph_get_state(ctx_, x.data(), v.data(), rho.data()));
        FluidObject* f = SPHSimulation::getCurrent()->getFluidModel(0);
        for (uint i = 0; i < n_; ++i) {
            for (int k = 0; k < 3; ++k) {
                f->getPosition(i)[k] = (Real)x[3 * (size_t)i + k];
                f->getVelocity(i)[k] = (Real)v[3 * (size_t)i + k];
            }
            f->getDensity(i) = (Real)rho[i];
        }
    }

    sph_ctx* context() { return ctx_; }
    /* The description init() built from the simulation (valid once init()
       has read the parameters, even if the context could not be created). */
    const sph_scene_desc& description() const { return desc_; }

private:
    /* TimeHelper::hasToSave's test, evaluated without its side effect: the
       last save happened at frame - 1 (frames start at 1, lastTimeSave at
       0, and each save stores (Real) frame / fps before frame is
       incremented, TimeHelper.h:43-48,100-110). */
    static bool will_save(SPHSimulation* sim)
    {
        const Real fps = sim->getFPS();
        const Real last = (Real)(sim->getFrame() - 1) / fps;
        return sim->getTime() - last >= 1.0 / fps;
    }
    [[noreturn]] static void fail(const std::string& msg) { throw std::runtime_error("GPUSolver: " + msg); }
    void check(int rc)
    {
        if (rc != SPH_OK) fail(std::string(ctx_ ? sph_last_error(ctx_) : sph_global_error()) + " (status " +
                               std::to_string(rc) + ")");
    }

    SPHSolver* cpu_ = nullptr;
    sph_ctx* ctx_ = nullptr;
    sph_scene_desc desc_{};
    uint n_ = 0;
};

#endif
