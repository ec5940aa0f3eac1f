// backend_b200.h — the B200 backend's hooks beyond src/backend.h, for a driver patched to keep
// the population on the GPU: device dipole events and the GPU trajectory and checkpoint writers
// (src/main.cpp:327-337 is the loop such a driver changes).
#pragma once

#include "backend.h"
#include "dipole.h"

#include <cstddef>

// DipoleManager::process (src/dipole.cpp:42-127) on the kernel's device state. `state` carries
// the manager's counts and generator text in and out. Returns false (and does nothing) when the
// kernel is not a B200 kernel; otherwise sets `events` to process()'s return value.
bool b200ProcessDipoles(VelocityKernel &kernel, const SimParams &params, DipoleEventState &state,
                        std::size_t &events);
