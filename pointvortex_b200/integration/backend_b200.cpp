// backend_b200.cpp — PointVortex link-time backend over libpvb200's C ABI.
//
// This is the translation unit a PointVortex build links in place of src/backend_cpu.cpp or
// src/backend_cuda.cu: it defines the free functions of src/backend.h:9-16 and a VelocityKernel
// (src/compute.h:18-36) whose device-stepping hooks drive the B200 kernels. It is compiled against
// the reference's own headers (backend.h, compute.h, params.h, vortex.h); oracle/Makefile target
// `cli` links it with the reference's src/main.cpp and src/print.cpp into point_vortex_b200,
// which keeps the parameter-file format, CSV outputs and checkpoints of the reference unchanged.
//
// Status codes of the C ABI become the reference's exception types, with the library's message:
// PV_ERROR_INVALID_ARGUMENT -> std::invalid_argument, PV_ERROR_OUT_OF_RANGE -> std::out_of_range,
// PV_ERROR_LOGIC -> std::logic_error, anything else -> std::runtime_error.
#include "backend_b200.h"

#include "pvb200.h"

#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

[[noreturn]] void raise(pv_status status, const char *message) {
    const std::string text = message ? message : "libpvb200 failure";
    switch (status) {
    case PV_ERROR_INVALID_ARGUMENT:
        throw std::invalid_argument(text);
    case PV_ERROR_OUT_OF_RANGE:
        throw std::out_of_range(text);
    case PV_ERROR_LOGIC:
        throw std::logic_error(text);
    default:
        throw std::runtime_error(text);
    }
}

int deviceOrdinal() {
    // One process drives one GPU; CUDA_VISIBLE_DEVICES selects it.
    return 0;
}

class B200Kernel final : public VelocityKernel {
  public:
    explicit B200Kernel(const SimParams &params) {
        pv_params p{};
        if (params.boundaryCondition == "infinite")
            p.geometry = PV_GEOMETRY_INFINITE;
        else if (params.boundaryCondition == "periodic")
            p.geometry = PV_GEOMETRY_PERIODIC;
        else if (params.boundaryCondition == "disk")
            p.geometry = PV_GEOMETRY_DISK;
        else
            throw std::invalid_argument("unsupported boundary condition: " +
                                        params.boundaryCondition);
        p.core_radius = params.coreRadius;
        p.box_length_x = params.boxLengthX;
        p.box_length_y = params.boxLengthY;
        p.image_layers = params.periodicImageLayers;
        p.disk_radius = params.diskRadius;
        p.precision = PV_PRECISION_FP64;
        const pv_status st = pv_context_create(&p, deviceOrdinal(), &ctx_);
        if (st != PV_OK)
            raise(st, pv_last_error(nullptr));
    }
    ~B200Kernel() override { pv_context_destroy(ctx_); }
    B200Kernel(const B200Kernel &) = delete;
    B200Kernel &operator=(const B200Kernel &) = delete;

    void evaluateRange(const std::vector<double> &x, const std::vector<double> &y,
                       const std::vector<double> &circulation, VelocityField &velocity,
                       std::size_t begin, std::size_t end) const override {
        validateVortexArrays(x, y, circulation);
        const std::size_t count = x.size();
        if (begin > end || end > count)
            throw std::out_of_range("invalid target-vortex range");
        velocity.resize(count);
        std::vector<double> u(end - begin + 1), v(end - begin + 1);
        check(pv_evaluate_range(ctx_, x.data(), y.data(), circulation.data(), count, begin, end,
                                u.data(), v.data()));
        for (std::size_t i = begin; i < end; ++i) {
            velocity.x[i] = u[i - begin];
            velocity.y[i] = v[i - begin];
        }
    }

    double hamiltonian(const VortexSystem &vortices) const override {
        vortices.validate();
        double h = 0.0;
        check(pv_hamiltonian(ctx_, vortices.x.data(), vortices.y.data(),
                             vortices.circulation.data(), vortices.size(), &h));
        return h;
    }

    bool supportsDeviceStepping() const noexcept override { return true; }

    void uploadDeviceState(const VortexSystem &vortices) const override {
        vortices.validate();
        check(pv_upload_state(ctx_, vortices.x.data(), vortices.y.data(),
                              vortices.circulation.data(), vortices.size()));
    }

    void downloadDeviceState(VortexSystem &vortices) const override {
        std::size_t n = vortices.size();
        if (dipolesOnDevice_) {
            // dipole events on the device may have changed the population and its circulations
            check(pv_state_size(ctx_, &n));
            vortices.resize(n);
            check(pv_download_circulation(ctx_, vortices.circulation.data(), n));
        }
        check(pv_download_state(ctx_, vortices.x.data(), vortices.y.data(), n));
        vortices.validate();
    }

    // DipoleManager::process (src/dipole.cpp:42-127) on the device state, for the driver patch
    // that keeps the population on the GPU. `state` carries the manager's counts and generator
    // text in and out, so the host DipoleManager can be rebuilt from it. Returns the events.
    std::size_t processDipolesOnDevice(const SimParams &p, DipoleEventState &state) {
        if (!dipolesOnDevice_) {
            const pv_dipole_config c{p.dipoleRemoval ? 1 : 0, p.dipoleRemovalDistance,
                                     static_cast<int>(p.dipoleReinjection), p.randomSeed};
            check(pv_dipole_configure(ctx_, &c));
            check(pv_dipole_restore(ctx_, state.removedPairs, state.reinjectedPairs,
                                    state.randomEngineState.c_str()));
            dipolesOnDevice_ = true;
        }
        std::size_t events = 0;
        check(pv_dipole_process(ctx_, &events));
        std::uint64_t removed = 0, reinjected = 0;
        std::size_t length = 0;
        pv_dipole_state(ctx_, &removed, &reinjected, nullptr, 0, &length);
        std::string text(length + 1, '\0');
        check(pv_dipole_state(ctx_, &removed, &reinjected, text.data(), text.size(), &length));
        text.resize(length);
        state = {static_cast<std::size_t>(removed), static_cast<std::size_t>(reinjected), text};
        return events;
    }

    void evaluateDeviceState(VelocityField &velocity) const override {
        std::size_t n = 0;
        check(pv_state_size(ctx_, &n));
        velocity.resize(n);
        check(pv_evaluate_state(ctx_, velocity.x.data(), velocity.y.data(), n));
    }

    void deviceRk4Step(double dt) const override { check(pv_rk4_step(ctx_, dt)); }

    StepResult deviceDopri5Step(double dt, double absoluteTolerance, double relativeTolerance,
                                double minimumTimeStep, double maximumTimeStep) const override {
        pv_step_result r{};
        check(pv_dopri5_step(ctx_, dt, absoluteTolerance, relativeTolerance, minimumTimeStep,
                             maximumTimeStep, &r));
        return {r.accepted_time_step, r.suggested_time_step, r.normalized_error, r.rejected_steps};
    }

    void invalidateDeviceDerivative() const noexcept override { pv_invalidate_derivative(ctx_); }

  private:
    void check(pv_status st) const {
        if (st != PV_OK)
            raise(st, pv_last_error(ctx_));
    }
    pv_context *ctx_ = nullptr;
    bool dipolesOnDevice_ = false;
};

} // namespace

bool b200ProcessDipoles(VelocityKernel &kernel, const SimParams &params, DipoleEventState &state,
                        std::size_t &events) {
    auto *b200 = dynamic_cast<B200Kernel *>(&kernel);
    if (!b200)
        return false;
    events = b200->processDipolesOnDevice(params, state);
    return true;
}

void backendInitialize(int &, char **&) {}
void backendFinalize() {}
void backendAbort(int) {}
bool backendIsRoot() { return true; }
const char *backendName() { return pv_backend_name(); }
std::string backendRuntimeDetails() {
    char buffer[512] = {};
    if (pv_runtime_details(deviceOrdinal(), buffer, sizeof(buffer)) != PV_OK)
        return "cuda_device unavailable";
    return buffer;
}
std::unique_ptr<VelocityKernel> makeBackendKernel(const SimParams &params) {
    return std::make_unique<B200Kernel>(params);
}
