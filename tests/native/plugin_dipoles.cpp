// Drives the backend translation unit's dipole hook (b200ProcessDipoles,
// pointvortex_b200/integration/backend_b200.cpp) and compares every call with the reference's
// own host DipoleManager::process on the same state: events, population, positions,
// circulations, counts and generator text, bit for bit. Built by `make -C oracle plugin-test`
// into oracle/_ref/plugin_dipoles; run by tests/test_cli_gpu.py. Exit status 0 = identical.
#include "backend_b200.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>

namespace {

VortexSystem planted(const SimParams &p, std::size_t n, std::uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> unit(0.0, 1.0);
    VortexSystem s;
    const double pi = 3.141592653589793;
    for (std::size_t i = 0; i < n; ++i) {
        double x, y;
        if (p.boundaryCondition == "periodic") {
            x = (unit(rng) - 0.5) * p.boxLengthX;
            y = (unit(rng) - 0.5) * p.boxLengthY;
        } else {
            const double r = 0.999 * p.diskRadius * std::sqrt(unit(rng));
            const double a = 2.0 * pi * unit(rng);
            x = r * std::cos(a);
            y = r * std::sin(a);
        }
        s.pushBack(x, y, (i % 2) ? -1.0 : 1.0);
    }
    for (std::size_t k = 0; k < 20; k += 2) {  // ten close opposite-sign pairs
        if (p.boundaryCondition == "periodic") {
            s.x[k + 1] = s.x[k] + 0.0005 * static_cast<double>(k + 1);
            s.y[k + 1] = s.y[k] - 0.0003 * static_cast<double>(k + 1);
        } else {  // towards the centre, so the partner stays inside the disk
            const double f = 1.0 - 0.0005 * static_cast<double>(k + 1);
            s.x[k + 1] = s.x[k] * f;
            s.y[k + 1] = s.y[k] * f;
        }
    }
    return s;
}

bool same(const std::vector<double> &a, const std::vector<double> &b) {
    return a.size() == b.size() &&
           (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(double)) == 0);
}

} // namespace

int run();

int main() {
    std::setvbuf(stdout, nullptr, _IOLBF, 0);
    try {
        return run();
    } catch (const std::exception &e) {
        std::printf("FAIL: %s\n", e.what());
        return 3;
    }
}

int run() {
    int failures = 0;
    for (const char *boundary : {"periodic", "disk"}) {
        for (ReinjectionMode mode :
             {ReinjectionMode::none, ReinjectionMode::independent, ReinjectionMode::paired}) {
            SimParams p;
            p.boundaryCondition = boundary;
            p.boxLengthX = p.boxLengthY = 2.0 * 3.141592653589793;
            p.diskRadius = 1.0;
            p.dipoleRemoval = true;
            p.dipoleRemovalDistance = 0.02;
            p.dipoleReinjection = mode;
            p.randomSeed = 99;
            VortexSystem host = planted(p, 400, 7);
            DipoleManager reference(p);
            auto kernel = makeBackendKernel(p);
            kernel->uploadDeviceState(host);
            DipoleEventState device = reference.state();
            for (int call = 0; call < 3; ++call) {
                const std::size_t expected = reference.process(host);
                std::size_t events = 0;
                if (!b200ProcessDipoles(*kernel, p, device, events)) {
                    std::printf("FAIL %s %s: not a B200 kernel\n", boundary, toString(mode));
                    return 2;
                }
                VortexSystem got;
                kernel->downloadDeviceState(got);
                const DipoleEventState want = reference.state();
                const bool ok = events == expected && same(got.x, host.x) && same(got.y, host.y) &&
                                same(got.circulation, host.circulation) &&
                                device.removedPairs == want.removedPairs &&
                                device.reinjectedPairs == want.reinjectedPairs &&
                                device.randomEngineState == want.randomEngineState;
                std::printf("%s %s call %d: events %zu (reference %zu), population %zu: %s\n",
                            boundary, toString(mode), call, events, expected, got.size(),
                            ok ? "identical" : "DIFFERENT");
                failures += ok ? 0 : 1;
            }
        }
    }
    std::printf(failures ? "FAIL\n" : "OK\n");
    return failures ? 1 : 0;
}
