// ref_shim.cpp — extern "C" access to the UNMODIFIED reference PointVortex code.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the reference's own
// sources (src/compute.cpp, src/timestep.cpp, src/dipole.cpp, ... of jplaurie/PointVortex)
// by oracle/Makefile into oracle/_ref/. Only the tests, the smoke check and the CPU-baseline
// leg of bench.py load the result: it is the checker, never the product.
//
// The same source is linked twice: with the reference's CPU backend (src/backend_cpu.cpp)
// into libpvref.so, and with the reference's CUDA backend (src/backend_cuda.cu) into
// libpvref_cuda.so. Every entry point goes through the reference's public interfaces:
// makeBackendKernel (src/backend.h:16), VelocityKernel (src/compute.h:18-36),
// RungeKuttaIntegrator (src/timestep.h:18-34), computeInvariants (src/compute.h:83-84) and
// DipoleManager (src/dipole.h:18-39).
#include "backend.h"
#include "compute.h"
#include "dipole.h"
#include "print.h"
#include "checkpoint.h"
#include "params.h"
#include "timestep.h"

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
struct pvref_params {
    int geometry; // 0 infinite, 1 periodic, 2 disk
    double core_radius;
    double box_length_x;
    double box_length_y;
    int image_layers;
    double disk_radius;
    double absolute_tolerance;
    double relative_tolerance;
    double minimum_time_step;
    double maximum_time_step;
    int dipole_removal;
    double dipole_removal_distance;
    int dipole_reinjection; // 0 none, 1 independent, 2 paired
    std::uint64_t random_seed;
};
}

namespace {
thread_local std::string lastError;

SimParams toSimParams(const pvref_params *p) {
    SimParams s;
    static const char *names[] = {"infinite", "periodic", "disk"};
    if (p->geometry < 0 || p->geometry > 2)
        throw std::invalid_argument("unsupported boundary condition");
    s.boundaryCondition = names[p->geometry];
    s.coreRadius = p->core_radius;
    s.boxLengthX = p->box_length_x;
    s.boxLengthY = p->box_length_y;
    s.periodicImageLayers = p->image_layers;
    s.diskRadius = p->disk_radius;
    s.absoluteTolerance = p->absolute_tolerance;
    s.relativeTolerance = p->relative_tolerance;
    s.minimumTimeStep = p->minimum_time_step;
    s.maximumTimeStep = p->maximum_time_step;
    s.dipoleRemoval = p->dipole_removal != 0;
    s.dipoleRemovalDistance = p->dipole_removal_distance;
    s.dipoleReinjection = p->dipole_reinjection == 1   ? ReinjectionMode::independent
                          : p->dipole_reinjection == 2 ? ReinjectionMode::paired
                                                       : ReinjectionMode::none;
    s.randomSeed = p->random_seed;
    return s;
}

VortexSystem makeSystem(const double *x, const double *y, const double *g, std::size_t n) {
    VortexSystem s(n);
    if (n) {
        std::memcpy(s.x.data(), x, n * sizeof(double));
        std::memcpy(s.y.data(), y, n * sizeof(double));
        std::memcpy(s.circulation.data(), g, n * sizeof(double));
    }
    return s;
}

// Status codes follow the product's C ABI: 1 invalid_argument, 2 out_of_range,
// 3 runtime_error, 4 logic_error, 9 anything else.
template <typename F> int guarded(F &&body) {
    try {
        body();
        lastError.clear();
        return 0;
    } catch (const std::invalid_argument &e) {
        lastError = e.what();
        return 1;
    } catch (const std::out_of_range &e) {
        lastError = e.what();
        return 2;
    } catch (const std::logic_error &e) {
        lastError = e.what();
        return 4;
    } catch (const std::runtime_error &e) {
        lastError = e.what();
        return 3;
    } catch (const std::exception &e) {
        lastError = e.what();
        return 9;
    }
}

struct Handle {
    SimParams params;
    std::unique_ptr<VelocityKernel> kernel;
    std::unique_ptr<RungeKuttaIntegrator> integrator;
};
} // namespace

extern "C" {

const char *pvref_last_error(void) { return lastError.c_str(); }
const char *pvref_backend_name(void) { return backendName(); }

int pvref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void pvref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0)
        omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// VelocityKernel::evaluate over a half-open target range (src/compute.cpp:57-69 when
// begin=0,end=n; otherwise VelocityKernel::evaluateRange, src/compute.h:26-28).
int pvref_evaluate_range(const pvref_params *p, const double *x, const double *y,
                         const double *g, std::size_t n, std::size_t begin, std::size_t end,
                         double *u, double *v) {
    return guarded([&] {
        const SimParams sp = toSimParams(p);
        auto kernel = makeBackendKernel(sp);
        std::vector<double> vx(x, x + n), vy(y, y + n), vg(g, g + n);
        VelocityField vel;
        if (begin == 0 && end == n)
            kernel->evaluate(vx, vy, vg, vel);
        else
            kernel->evaluateRange(vx, vy, vg, vel, begin, end);
        for (std::size_t i = begin; i < end; ++i) {
            u[i - begin] = vel.x[i];
            v[i - begin] = vel.y[i];
        }
    });
}

// computeInvariants(VortexSystem, VelocityKernel) (src/compute.cpp:157-163):
// out = {circulation, Ix, Iy, angular impulse, Hamiltonian}.
int pvref_invariants(const pvref_params *p, const double *x, const double *y, const double *g,
                     std::size_t n, double *out) {
    return guarded([&] {
        const SimParams sp = toSimParams(p);
        auto kernel = makeBackendKernel(sp);
        const Invariants inv = computeInvariants(makeSystem(x, y, g, n), *kernel);
        out[0] = inv.circulation;
        out[1] = inv.linearImpulseX;
        out[2] = inv.linearImpulseY;
        out[3] = inv.angularImpulse;
        out[4] = inv.hamiltonian;
    });
}

int pvref_hamiltonian(const pvref_params *p, const double *x, const double *y, const double *g,
                      std::size_t n, double *out) {
    return guarded([&] {
        const SimParams sp = toSimParams(p);
        auto kernel = makeBackendKernel(sp);
        *out = kernel->hamiltonian(makeSystem(x, y, g, n));
    });
}

void *pvref_stepper_create(const pvref_params *p, std::size_t n) {
    Handle *h = nullptr;
    const int rc = guarded([&] {
        auto owned = std::make_unique<Handle>();
        owned->params = toSimParams(p);
        owned->kernel = makeBackendKernel(owned->params);
        owned->integrator = std::make_unique<RungeKuttaIntegrator>(n);
        h = owned.release();
    });
    return rc == 0 ? h : nullptr;
}

void pvref_stepper_destroy(void *handle) { delete static_cast<Handle *>(handle); }

void pvref_stepper_invalidate(void *handle) {
    auto *h = static_cast<Handle *>(handle);
    h->integrator->invalidateCachedDerivative();
    h->kernel->invalidateDeviceDerivative();
}

// RungeKuttaIntegrator::rk4Step (src/timestep.cpp:31-61), `steps` times in place.
int pvref_rk4_steps(void *handle, double *x, double *y, const double *g, std::size_t n,
                    double dt, std::size_t steps) {
    auto *h = static_cast<Handle *>(handle);
    return guarded([&] {
        VortexSystem s = makeSystem(x, y, g, n);
        for (std::size_t k = 0; k < steps; ++k)
            h->integrator->rk4Step(s, dt, *h->kernel);
        std::memcpy(x, s.x.data(), n * sizeof(double));
        std::memcpy(y, s.y.data(), n * sizeof(double));
    });
}

// RungeKuttaIntegrator::dopri5Step (src/timestep.cpp:62-120). The integrator keeps its FSAL
// derivative between calls, as in the reference driver. out = {accepted dt, suggested dt,
// normalised error, rejected count}.
int pvref_dopri5_step(void *handle, double *x, double *y, const double *g, std::size_t n,
                      double dt, double *out) {
    auto *h = static_cast<Handle *>(handle);
    return guarded([&] {
        VortexSystem s = makeSystem(x, y, g, n);
        const StepResult r = h->integrator->dopri5Step(s, dt, *h->kernel, h->params);
        std::memcpy(x, s.x.data(), n * sizeof(double));
        std::memcpy(y, s.y.data(), n * sizeof(double));
        out[0] = r.acceptedTimeStep;
        out[1] = r.suggestedTimeStep;
        out[2] = r.normalizedError;
        out[3] = static_cast<double>(r.rejectedSteps);
    });
}

// The device-stepping hooks of VelocityKernel (src/compute.h:30-36). With the CPU backend
// these throw std::logic_error (src/compute.cpp:70-84); with the CUDA backend they drive
// src/backend_cuda.cu.
int pvref_device_upload(void *handle, const double *x, const double *y, const double *g,
                        std::size_t n) {
    auto *h = static_cast<Handle *>(handle);
    return guarded([&] { h->kernel->uploadDeviceState(makeSystem(x, y, g, n)); });
}
int pvref_device_download(void *handle, double *x, double *y, const double *g, std::size_t n) {
    auto *h = static_cast<Handle *>(handle);
    return guarded([&] {
        VortexSystem s = makeSystem(x, y, g, n);
        h->kernel->downloadDeviceState(s);
        std::memcpy(x, s.x.data(), n * sizeof(double));
        std::memcpy(y, s.y.data(), n * sizeof(double));
    });
}
int pvref_device_evaluate(void *handle, double *u, double *v, std::size_t n) {
    auto *h = static_cast<Handle *>(handle);
    return guarded([&] {
        VelocityField vel;
        h->kernel->evaluateDeviceState(vel);
        if (vel.x.size() != n)
            throw std::runtime_error("device population differs");
        std::memcpy(u, vel.x.data(), n * sizeof(double));
        std::memcpy(v, vel.y.data(), n * sizeof(double));
    });
}
int pvref_device_rk4_step(void *handle, double dt) {
    auto *h = static_cast<Handle *>(handle);
    return guarded([&] { h->kernel->deviceRk4Step(dt); });
}
int pvref_device_dopri5_step(void *handle, double dt, double *out) {
    auto *h = static_cast<Handle *>(handle);
    return guarded([&] {
        const SimParams &p = h->params;
        const StepResult r =
            h->kernel->deviceDopri5Step(dt, p.absoluteTolerance, p.relativeTolerance,
                                        p.minimumTimeStep, p.maximumTimeStep);
        out[0] = r.acceptedTimeStep;
        out[1] = r.suggestedTimeStep;
        out[2] = r.normalizedError;
        out[3] = static_cast<double>(r.rejectedSteps);
    });
}

// DipoleManager::process (src/dipole.cpp:42-127). Arrays are in/out with room for `capacity`
// vortices; *n is updated to the surviving population. *events receives the return value.
// DipoleManager(params, state) + process + state() (src/dipole.cpp:32-40, 42-127, 182-186): one
// call of a manager restored from (*removed, *reinjected, engine_in); an empty engine_in keeps
// the fresh seeding. The counts and the engine text after the call are written back.
int pvref_dipole_process_state(const pvref_params *p, double *x, double *y, double *g,
                               std::size_t *n, std::size_t capacity, std::size_t *events,
                               std::uint64_t *removed, std::uint64_t *reinjected,
                               const char *engine_in, char *engine_out,
                               std::size_t engine_capacity) {
    return guarded([&] {
        const SimParams sp = toSimParams(p);
        DipoleEventState in{static_cast<std::size_t>(*removed),
                            static_cast<std::size_t>(*reinjected),
                            engine_in ? std::string(engine_in) : std::string()};
        DipoleManager manager(sp, in);
        VortexSystem s = makeSystem(x, y, g, *n);
        *events = manager.process(s);
        if (s.size() > capacity)
            throw std::runtime_error("dipole result exceeds capacity");
        *n = s.size();
        if (*n) {
            std::memcpy(x, s.x.data(), *n * sizeof(double));
            std::memcpy(y, s.y.data(), *n * sizeof(double));
            std::memcpy(g, s.circulation.data(), *n * sizeof(double));
        }
        const DipoleEventState out = manager.state();
        *removed = out.removedPairs;
        *reinjected = out.reinjectedPairs;
        if (out.randomEngineState.size() >= engine_capacity)
            throw std::runtime_error("engine state exceeds capacity");
        std::memcpy(engine_out, out.randomEngineState.c_str(), out.randomEngineState.size() + 1);
    });
}

int pvref_dipole_process(const pvref_params *p, double *x, double *y, double *g, std::size_t *n,
                         std::size_t capacity, std::size_t *events) {
    return guarded([&] {
        const SimParams sp = toSimParams(p);
        DipoleManager manager(sp);
        VortexSystem s = makeSystem(x, y, g, *n);
        *events = manager.process(s);
        if (s.size() > capacity)
            throw std::runtime_error("dipole result exceeds capacity");
        *n = s.size();
        if (*n) {
            std::memcpy(x, s.x.data(), *n * sizeof(double));
            std::memcpy(y, s.y.data(), *n * sizeof(double));
            std::memcpy(g, s.circulation.data(), *n * sizeof(double));
        }
    });
}

// TrajectoryWriter (src/print.cpp:24-40): a new file at path (overwritten) with its header and one
// frame.
int pvref_write_trajectory(const char *path, double time, std::size_t frame, const double *x,
                           const double *y, const double *g, const double *u, const double *v,
                           std::size_t n) {
    return guarded([&] {
        TrajectoryWriter writer(path, true);
        VortexSystem s = makeSystem(x, y, g, n);
        VelocityField vel;
        vel.x.assign(u, u + n);
        vel.y.assign(v, v + n);
        writer.write(time, frame, s, vel);
    });
}

// writeCheckpoint (src/checkpoint.cpp:23-102) into directory with the given records:
// inv[0..4] initial and seg[0..4] segment invariants; sched[0..4] the OutputSchedule fields;
// prog_d = (time, suggestedTimeStep, nextOutputTime); prog_i = (acceptedSteps, outputIndex,
// eventIndex); the dipole state's counts and engine text.
int pvref_write_checkpoint(const char *directory, const pvref_params *p, const double *x,
                           const double *y, const double *g, std::size_t n, const double *inv,
                           const double *seg, std::uint64_t removed, std::uint64_t reinjected,
                           const char *engine, const double *sched, const double *prog_d,
                           const std::uint64_t *prog_i) {
    return guarded([&] {
        const SimParams sp = toSimParams(p);
        VortexSystem s = makeSystem(x, y, g, n);
        const Invariants a{inv[0], inv[1], inv[2], inv[3], inv[4]};
        const Invariants b{seg[0], seg[1], seg[2], seg[3], seg[4]};
        const DipoleEventState d{static_cast<std::size_t>(removed),
                                 static_cast<std::size_t>(reinjected), engine};
        const OutputSchedule o{sched[0], sched[1], sched[2], sched[3], sched[4]};
        const CheckpointProgress pr{prog_d[0], prog_d[1], prog_d[2],
                                    static_cast<std::size_t>(prog_i[0]),
                                    static_cast<std::size_t>(prog_i[1]),
                                    static_cast<std::size_t>(prog_i[2])};
        writeCheckpoint(directory, s, a, sp, b, d, o, pr, true);
    });
}
}
