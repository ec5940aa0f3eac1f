// pv_context.cu — host side of libpvb200: contexts, device buffers, the step flows and the C ABI
// declared in include/pvb200.h.
//
// A context is the B200 counterpart of one VelocityKernel object of the reference
// (src/compute.h:18-36) plus the device-stepping state the reference CUDA backend keeps in mutable
// members (src/backend_cuda.cu:519-532). All device work of a context is ordered on its own
// stream; results are read back at synchronisation points only (one per RK4 step / DOPRI5 attempt
// / query), unlike the reference backend, which synchronises after every evaluation.
#include "pvb200.h"
#include "pv_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <sstream>
#include <string>
#include <vector>

using namespace pvb;

namespace {

thread_local std::string g_create_error;

// Butcher rows of the Dormand–Prince pair, src/timestep.h:8-15, and the weights b5, b4 of
// src/timestep.cpp:69-73, as the reference's constant expressions evaluate them.
constexpr double kDopri[7][7] = {
    {0},
    {1.0 / 5.0},
    {3.0 / 40.0, 9.0 / 40.0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0},
    {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
constexpr double kB5[7] = {35.0 / 384.0,     0.0,         500.0 / 1113.0, 125.0 / 192.0,
                           -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
constexpr double kB4[7] = {5179.0 / 57600.0, 0.0,          7571.0 / 16695.0,   393.0 / 640.0,
                           -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0};

// A growable device allocation.
struct DeviceArray {
    double *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap && p)
            return cudaSuccess;
        if (p)
            cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(n, 64);
        cudaError_t e = cudaMalloc(&p, want * sizeof(double));
        if (e == cudaSuccess)
            cap = want;
        return e;
    }
    void release() {
        if (p)
            cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

size_t padded(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

bool finite_arrays(const double *x, const double *y, const double *g, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(g[i]))
            return false;
    return true;
}

} // namespace

struct pv_context {
    pv_params params{};
    GeometryConsts gc{};
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::string error;

    // device-resident state
    size_t n = 0;
    bool state_valid = false;
    bool fsal_valid = false;
    uint64_t evaluations = 0;
    EvalPlan plan{};
    DeviceArray x, y, gamma, gs;     // state and scaled circulations
    DeviceArray p0x, p0y, p1x, p1y;  // stage positions (ping-pong)
    DeviceArray kx[7], ky[7];        // stage velocities
    DeviceArray pu, pv;              // chunk partials (or symmetric-kernel rows)
    cudaGraphExec_t attempt_graph = nullptr; // one DOPRI5 attempt with a valid FSAL derivative
    SymmetricPlan sym{};             // one evaluation per unordered pair (when planned)
    DeviceArray sym_items, sym_counter;
    DeviceArray rk4_barrier;         // arrival counter of the cooperative RK4 steps' grid barrier
    int sym_items_blocks = 0;        // the block count the item table was built for
    DeviceArray inv_scratch, inv_out;
    DeviceArray cand;                // dipole candidates (3 doubles-worth each)
    DeviceControl *ctl = nullptr;    // device control block
    DeviceControl *ctl_host = nullptr; // pinned mirror
    double *pinned = nullptr;        // pinned staging for small results (16 doubles)

    // host-array evaluation (kept apart from the device state)
    DeviceArray ex, ey, eg, egs, eu, ev, epu, epv;

    // dipole events (DipoleManager, src/dipole.h:19-40)
    pv_dipole_config dipole{};
    bool dipole_configured = false;
    std::mt19937_64 dipole_random;
    uint64_t removed_pairs = 0, reinjected_pairs = 0;
    std::vector<double> gamma_host;  // the device state's circulations (they change only here)
    DeviceArray removed_index;
    // With removal configured, every DOPRI5 attempt also scans its accepted state for dipoles in
    // the same synchronisation; pv_dipole_process then needs no GPU work when none was found.
    bool prescan_valid = false;        // the device state is the one the last scan saw
    unsigned long long prescan_count = 0;

    // text output (pv_format_*): row slots, row lengths, block offsets, the packed frame
    DeviceArray fmt_stage, fmt_len, fmt_block, fmt_out;

    // FP32C near field (pv_set_near_field): the lists of pairs left to the FP64 pass, and the
    // radius (< 0: the default for the population, 0: none)
    DeviceArray near_count, near_slot;
    // an evaluation's near-field pass, left to the stage launched after it (StageArgs::near)
    NearPass pending_near{};
    double near_radius = -1.0;

    // polls of the bounded device waits (pv_set_wait_limits): tile copies, grid barrier
    uint32_t wait_limit = kWaitLimit;
    uint32_t spin_limit = kGridSpinLimit;

    // launch accounting and optional per-launch CUDA-event timing (pv_set_profiling)
    bool profiling = false;
    uint64_t launches[PV_KERNEL_KINDS] = {};
    uint64_t timed[PV_KERNEL_KINDS] = {};
    double milliseconds[PV_KERNEL_KINDS] = {};
    struct Timer {
        cudaEvent_t start, stop;
        int kind;
        bool in_graph;  // recorded by the captured attempt on every replay; owned by it
    };
    std::vector<Timer> pending, pool;
    bool capturing = false;             // counted() during a graph capture
    std::vector<Timer> capture_timers;  // the timers a capture recorded
    std::vector<Timer> graph_timers;    // those of attempt_graph
    bool graph_profiled = false;        // attempt_graph records per-launch events
    std::vector<const void *> graph_key; // buffers and plan attempt_graph was captured for

    ~pv_context() {
        if (attempt_graph)
            cudaGraphExecDestroy(attempt_graph);
        for (DeviceArray *a : {&x, &y, &gamma, &gs, &p0x, &p0y, &p1x, &p1y, &pu, &pv, &inv_scratch,
                               &inv_out, &cand, &ex, &ey, &eg, &egs, &eu, &ev, &epu, &epv,
                               &removed_index, &fmt_stage, &fmt_len, &fmt_block, &fmt_out,
                               &sym_items, &sym_counter, &rk4_barrier, &near_count, &near_slot})
            a->release();
        for (int s = 0; s < 7; ++s) {
            kx[s].release();
            ky[s].release();
        }
        if (ctl)
            cudaFree(ctl);
        if (ctl_host)
            cudaFreeHost(ctl_host);
        if (pinned)
            cudaFreeHost(pinned);
        for (auto &t : pending)
            if (!t.in_graph)
                pool.push_back(t);
        for (auto &t : graph_timers)
            pool.push_back(t);
        for (auto &t : pool) {
            cudaEventDestroy(t.start);
            cudaEventDestroy(t.stop);
        }
        if (stream)
            cudaStreamDestroy(stream);
    }
};

namespace {

// Keeps the caller's current device and restores it on exit.
struct DeviceGuard {
    int previous = -1;
    bool ok = false;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&previous) != cudaSuccess)
            previous = -1;
        ok = cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceGuard() {
        if (previous >= 0)
            cudaSetDevice(previous);
    }
};

pv_status fail(pv_context *c, pv_status code, const std::string &message) {
    c->error = message;
    return code;
}

pv_status cuda_fail(pv_context *c, cudaError_t e, const char *what) {
    return fail(c, PV_ERROR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PV_CUDA(ctx, call)                                                                         \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return cuda_fail((ctx), e_, #call);                                                    \
    } while (0)

// Runs `launch` (which enqueues `count` kernels of one kind on the context stream), counting the
// launches and, when profiling is on, bracketing them with CUDA events on the same stream.
template <class F> cudaError_t counted(pv_context *c, int kind, int count, F &&launch) {
    c->launches[kind] += static_cast<uint64_t>(count);
    if (!c->profiling)
        return launch();
    pv_context::Timer t{};
    if (!c->pool.empty()) {
        t = c->pool.back();
        c->pool.pop_back();
    } else {
        cudaError_t e = cudaEventCreate(&t.start);
        if (e == cudaSuccess)
            e = cudaEventCreate(&t.stop);
        if (e != cudaSuccess)
            return e;
    }
    t.kind = kind;
    t.in_graph = c->capturing;
    // inside a capture the records become event-record nodes that fire on every replay
    const unsigned flags = c->capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    cudaError_t e = cudaEventRecordWithFlags(t.start, c->stream, flags);
    if (e != cudaSuccess)
        return e;
    e = launch();
    const cudaError_t e2 = cudaEventRecordWithFlags(t.stop, c->stream, flags);
    (c->capturing ? c->capture_timers : c->pending).push_back(t);
    return e != cudaSuccess ? e : e2;
}

// Folds the timings of completed launches into the totals (call after a stream synchronisation).
void collect_timers(pv_context *c) {
    for (auto &t : c->pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, t.start, t.stop) == cudaSuccess) {
            c->milliseconds[t.kind] += ms;
            ++c->timed[t.kind];
        }
        if (!t.in_graph)
            c->pool.push_back(t);
    }
    c->pending.clear();
}

const char *coincident_message(int geometry, bool hamiltonian) {
    if (geometry == GEO_PERIODIC)
        return "coincident periodic vortices";
    if (geometry == GEO_DISK)
        return "coincident vortices in disk";
    return hamiltonian ? "coincident vortices" : "coincident vortices in singular point-vortex kernel";
}

// Maps a device status word to the reference's exception type and message.
pv_status status_error(pv_context *c, int status, bool hamiltonian = false) {
    switch (status) {
    case ST_OK:
        return PV_OK;
    case ST_NONFINITE_POSITION:
        return fail(c, PV_ERROR_INVALID_ARGUMENT, "vortex data must be finite");
    case ST_OUTSIDE_DISK:
        return fail(c, PV_ERROR_INVALID_ARGUMENT, "vortex lies on or outside the disk");
    case ST_COINCIDENT:
        return fail(c, PV_ERROR_RUNTIME, coincident_message(c->params.geometry, hamiltonian));
    case ST_NONFINITE_VELOCITY:
        return fail(c, PV_ERROR_RUNTIME, "non-finite velocity; check scales and close encounters");
    case ST_DOPRI_NONFINITE:
        return fail(c, PV_ERROR_RUNTIME, "non-finite adaptive error estimate or invalid tolerance");
    case ST_DOPRI_FAILED:
        return fail(c, PV_ERROR_RUNTIME, "adaptive integrator could not satisfy tolerance");
    case ST_NONFINITE_MOMENT:
        return fail(c, PV_ERROR_RUNTIME, "non-finite vortex moment; check input scales");
    case ST_NONFINITE_HAMILTONIAN:
        return fail(c, PV_ERROR_RUNTIME, "non-finite Hamiltonian; check input scales");
    case ST_OUTSIDE_DISK_H:
        return fail(c, PV_ERROR_INVALID_ARGUMENT, "vortex outside disk");
    case ST_TIMEOUT:
        return fail(c, PV_ERROR_RUNTIME, "a bounded device wait timed out");
    default:
        return fail(c, PV_ERROR_RUNTIME, "device reported status " + std::to_string(status));
    }
}

// Kernel constructors' validation (src/compute.cpp:50-56, 165-173, 258-261) and the derived
// constants of the fast paths.
pv_status make_consts(const pv_params &p, GeometryConsts &g, std::string &message) {
    std::memset(&g, 0, sizeof(g));
    g.geometry = p.geometry;
    g.image_layers = p.image_layers;
    if (p.precision != PV_PRECISION_FP64 && p.precision != PV_PRECISION_FP32C) {
        message = "unsupported precision";
        return PV_ERROR_INVALID_ARGUMENT;
    }
    if (p.geometry == PV_GEOMETRY_INFINITE) {
        const double r = p.core_radius, r2 = r * r;
        if (!(r >= 0.0) || !std::isfinite(r2) || (r > 0.0 && r2 == 0.0)) {
            message = "core radius is negative or outside the supported numeric range";
            return PV_ERROR_INVALID_ARGUMENT;
        }
        g.eps2 = r2;
        return PV_OK;
    }
    if (p.geometry == PV_GEOMETRY_PERIODIC) {
        const double lx = p.box_length_x, ly = p.box_length_y;
        if (!(lx > 0.0) || !(ly > 0.0) || !std::isfinite(lx) || !std::isfinite(ly) ||
            !std::isfinite(2.0 * kPi / lx) || p.image_layers < 0 || p.image_layers > 64) {
            message = "invalid periodic-box parameters";
            return PV_ERROR_INVALID_ARGUMENT;
        }
        if (std::fabs(lx - ly) > 1e-13 * std::max(lx, ly)) {
            message = "Weiss-McWilliams kernel requires a square periodic box";
            return PV_ERROR_INVALID_ARGUMENT;
        }
        g.lx = lx;
        g.ly = ly;
        g.inv_lx = 1.0 / lx;
        g.inv_ly = 1.0 / ly;
        g.half_lx = 0.5 * lx;
        g.half_ly = 0.5 * ly;
        g.wave = 2.0 * kPi / lx;
        g.half_wave = 0.5 * g.wave;
        g.scale = 0.5 / lx;
        g.m_exact = std::min(p.image_layers, 2);
        for (int m = 0; m <= 2; ++m) {
            const double a = 2.0 * kPi * m;
            g.cosh_m[m] = std::cosh(a);
            g.two_cosh_m[m] = 2.0 * g.cosh_m[m];
            const double s = std::sinh(a);
            g.sinh2_m[m] = s * s;
        }
        // images m = 3..6 enter through 2u C + 2u^2 c cosh 2x^, u = sech(2 pi m) (|m| >= 7 are
        // beyond the reference's |shift| <= 40 cut for every x^)
        g.k1 = 0.0;
        g.k2 = 0.0;
        for (int m = 3; m <= std::min(p.image_layers, 6); ++m) {
            const double u = 1.0 / std::cosh(2.0 * kPi * m);
            g.k1 += 2.0 * u;
            g.k2 += 2.0 * u * u;
        }
        return PV_OK;
    }
    if (p.geometry == PV_GEOMETRY_DISK) {
        const double r = p.disk_radius, r2 = r * r;
        if (!(r > 0.0) || !std::isfinite(r2) || r2 == 0.0) {
            message = "invalid disk parameters";
            return PV_ERROR_INVALID_ARGUMENT;
        }
        g.radius = r;
        g.radius2 = r2;
        g.inv_radius = 1.0 / r;
        g.inv_radius2 = 1.0 / r2;
        return PV_OK;
    }
    message = "unsupported boundary condition";
    return PV_ERROR_INVALID_ARGUMENT;
}

// Geometry validation of evaluateRange (src/compute.cpp:31-48, 211, 293).
pv_status validate_geometry(pv_context *c, const double *x, const double *y, const double *g,
                            size_t n) {
    if (c->params.geometry == PV_GEOMETRY_PERIODIC) {
        double total = 0.0, absolute_total = 0.0;
        for (size_t i = 0; i < n; ++i) {
            total += g[i];
            absolute_total += std::fabs(g[i]);
        }
        if (std::fabs(total) > 1e-12 * std::max(1.0, absolute_total))
            return fail(c, PV_ERROR_INVALID_ARGUMENT, "periodic box requires zero total circulation");
    } else if (c->params.geometry == PV_GEOMETRY_DISK) {
        for (size_t i = 0; i < n; ++i)
            if (x[i] * x[i] + y[i] * y[i] >= c->gc.radius2)
                return fail(c, PV_ERROR_INVALID_ARGUMENT, "vortex lies on or outside the disk");
    }
    return PV_OK;
}

pv_status reset_control(pv_context *c) {
    std::memset(c->ctl_host, 0, sizeof(DeviceControl));
    PV_CUDA(c, cudaMemcpyAsync(c->ctl, c->ctl_host, sizeof(DeviceControl), cudaMemcpyHostToDevice,
                               c->stream));
    return PV_OK;
}

pv_status read_control(pv_context *c) {
    PV_CUDA(c, cudaMemcpyAsync(c->ctl_host, c->ctl, sizeof(DeviceControl), cudaMemcpyDeviceToHost,
                               c->stream));
    PV_CUDA(c, cudaStreamSynchronize(c->stream));
    collect_timers(c);
    return PV_OK;
}

std::vector<double> scaled(const GeometryConsts &g, const double *gamma, size_t n) {
    std::vector<double> out(n);
    for (size_t i = 0; i < n; ++i)
        out[i] = scaled_circulation(g, gamma[i]);
    return out;
}

// The FP32-compensated form's near field: periodic pairs and disk wall images closer than the
// radius are evaluated in FP64 (pv_near.cu). The plane has none.
bool near_field_used(const pv_context *c) {
    return c->params.precision == PV_PRECISION_FP32C &&
           (c->gc.geometry == GEO_PERIODIC || c->gc.geometry == GEO_DISK);
}

double near_radius_for(const pv_context *c, size_t n) {
    return c->near_radius < 0.0 ? default_near_radius(c->gc, n) : c->near_radius;
}

// Lists for n targets; the counts start at zero (the FP64 pass leaves them zero).
pv_status ensure_near_lists(pv_context *c, size_t n) {
    const double *before = c->near_count.p;
    PV_CUDA(c, c->near_count.ensure((n + 1) / 2));
    if (c->near_count.p != before)
        PV_CUDA(c, cudaMemsetAsync(c->near_count.p, 0, c->near_count.cap * sizeof(double),
                                   c->stream));
    PV_CUDA(c, c->near_slot.ensure(n * static_cast<size_t>(f32::kNearSlots) / 2));
    return PV_OK;
}

f32::NearLists near_lists(const pv_context *c) {
    return {reinterpret_cast<unsigned *>(c->near_count.p),
            reinterpret_cast<unsigned *>(c->near_slot.p)};
}

// Velocity of the state positions (px, py) into k_s via partials + stage kernel.
pv_status launch_eval(pv_context *c, const double *px, const double *py) {
    if (c->pending_near.lists.count) {  // a near pass no stage took over: it still resets the lists
        const NearPass stale = c->pending_near;
        c->pending_near = NearPass{};
        PV_CUDA(c, counted(c, PV_KERNEL_NEAR, 1, [&] { return launch_near_field(stale, c->stream); }));
    }
    const bool near = near_field_used(c);
    const f32::NearLists lists = near ? near_lists(c) : f32::NearLists{nullptr, nullptr};
    NearPass np{};
    np.lists = lists;
    np.x = px;
    np.y = py;
    np.gs = c->gs.p;
    np.n = c->n;
    np.t_begin = 0;
    np.t_end = c->n;
    np.stride = padded(c->n);
    np.g = c->gc;
    if (c->sym.enabled()) {
        PV_CUDA(c, counted(c, PV_KERNEL_VELOCITY, 1, [&] {
                    return launch_symmetric(
                        px, py, c->gs.p, c->n, c->sym,
                        reinterpret_cast<const unsigned *>(c->sym_items.p),
                        reinterpret_cast<unsigned *>(c->sym_counter.p),
                        reinterpret_cast<double2 *>(c->pu.p), padded(c->n), c->gc, lists,
                        c->stream);
                }));
        if (near) {
            np.pr = reinterpret_cast<double2 *>(c->pu.p);
            np.rows = c->sym.blocks;
            c->pending_near = np;  // the stage after this evaluation runs it
        }
        ++c->evaluations;
        return PV_OK;
    }
    EvalArgs a{};
    a.tx = px;
    a.ty = py;
    a.sx = px;
    a.sy = py;
    a.sg = c->gs.p;
    a.t_begin = 0;
    a.t_end = c->n;
    a.n_src = c->n;
    a.pu = c->pu.p;
    a.pv = c->pv.p;
    a.stride = padded(c->n);
    a.chunk = c->plan.chunk;
    a.num_chunks = c->plan.num_chunks;
    a.status = &c->ctl->status;
    a.g = c->gc;
    a.wait_limit = c->wait_limit;
    a.near = lists;
    PV_CUDA(c, counted(c, PV_KERNEL_VELOCITY, 1, [&] {
                return c->params.precision == PV_PRECISION_FP32C
                           ? launch_velocity_fp32c(a, c->plan, c->stream)
                           : launch_velocity(a, c->plan, c->stream);
            }));
    if (near) {
        np.pu = c->pu.p;
        np.pv = c->pv.p;
        np.rows = c->plan.num_chunks;
        c->pending_near = np;  // the stage after this evaluation runs it
    }
    ++c->evaluations;
    return PV_OK;
}

// The stage launched after an evaluation takes over its near-field pass, if launch_eval left one.
void attach_pending_near(pv_context *c, StageArgs &s) {
    s.near = c->pending_near;
    c->pending_near = NearPass{};
}

StageArgs stage_base(pv_context *c) {
    StageArgs s{};
    s.n = c->n;
    s.reduce = 1;
    s.num_chunks = c->sym.enabled() ? c->sym.blocks : c->plan.num_chunks;
    s.stride = padded(c->n);
    if (c->sym.enabled()) {  // interleaved (u, v) rows in pu's room
        s.pr = reinterpret_cast<const double2 *>(c->pu.p);
    } else {
        s.pu = c->pu.p;
        s.pv = c->pv.p;
    }
    for (int j = 0; j < 7; ++j) {
        s.kx[j] = c->kx[j].p;
        s.ky[j] = c->ky[j].p;
    }
    s.gamma = c->gamma.p;
    s.n_src = c->n;
    s.x0 = c->x.p;
    s.y0 = c->y.p;
    s.ctl = c->ctl;
    s.g = c->gc;
    return s;
}

// A captured attempt bakes in the population, the plan and the buffer addresses.
void drop_graphs(pv_context *c) {
    if (c->attempt_graph) {
        cudaGraphExecDestroy(c->attempt_graph);
        c->attempt_graph = nullptr;
    }
    for (auto &t : c->graph_timers)
        c->pool.push_back(t);
    c->graph_timers.clear();
    c->graph_key.clear();
}

// What a captured attempt depends on: the population, the plan and every buffer it touches.
std::vector<const void *> attempt_key(const pv_context *c) {
    std::vector<const void *> k = {reinterpret_cast<const void *>(c->n),
                                   reinterpret_cast<const void *>(
                                       static_cast<uintptr_t>(c->profiling ? 1 : 0)),
                                   reinterpret_cast<const void *>(
                                       static_cast<uintptr_t>(c->plan.num_chunks)),
                                   reinterpret_cast<const void *>(
                                       static_cast<uintptr_t>(c->sym.blocks)),
                                   c->x.p, c->y.p, c->gamma.p, c->gs.p, c->p0x.p, c->p0y.p,
                                   c->p1x.p, c->p1y.p, c->pu.p, c->pv.p, c->sym_items.p,
                                   c->sym_counter.p, c->ctl, c->cand.p,
                                   reinterpret_cast<const void *>(static_cast<uintptr_t>(
                                       c->dipole_configured && c->dipole.removal ? 1 : 0)),
                                   reinterpret_cast<const void *>(
                                       static_cast<uintptr_t>(c->wait_limit)),
                                   c->near_count.p, c->near_slot.p};
    uint64_t near_bits;
    std::memcpy(&near_bits, &c->gc.near2, sizeof near_bits);
    k.push_back(reinterpret_cast<const void *>(static_cast<uintptr_t>(near_bits)));
    uint64_t bits;
    std::memcpy(&bits, &c->dipole.distance, sizeof bits);
    k.push_back(reinterpret_cast<const void *>(static_cast<uintptr_t>(bits)));
    for (int s = 0; s < 7; ++s) {
        k.push_back(c->kx[s].p);
        k.push_back(c->ky[s].p);
    }
    return k;
}

pv_status ensure_state_capacity(pv_context *c, size_t n) {
    const size_t np = padded(std::max<size_t>(n, 1));
    for (DeviceArray *a : {&c->x, &c->y, &c->gamma, &c->gs, &c->p0x, &c->p0y, &c->p1x, &c->p1y})
        PV_CUDA(c, a->ensure(np));
    for (int s = 0; s < 7; ++s) {
        PV_CUDA(c, c->kx[s].ensure(np));
        PV_CUDA(c, c->ky[s].ensure(np));
    }
    c->plan = plan_evaluation(c->gc.geometry, n, n, c->sm_count, 0, c->params.precision);
    c->sym = plan_symmetric(n, c->sm_count, c->params.precision, c->gc.geometry);
    if (near_field_used(c)) {
        const double r = near_radius_for(c, n);
        c->gc.near2 = r * r;
        pv_status st = ensure_near_lists(c, n);
        if (st != PV_OK)
            return st;
    }
    const size_t rows = c->sym.enabled() ? static_cast<size_t>(c->sym.blocks)
                                         : static_cast<size_t>(c->plan.num_chunks);
    const size_t partial = rows * np;
    // the symmetric kernels' rows hold (u, v) pairs in pu's room; the chunk partials use both
    PV_CUDA(c, c->pu.ensure(c->sym.enabled() ? 2 * partial : partial));
    PV_CUDA(c, c->pv.ensure(c->sym.enabled() ? 1 : partial));
    if (c->sym.enabled() && c->sym_items_blocks != c->sym.blocks) {
        std::vector<unsigned> items(c->sym.items);
        symmetric_items(c->sym, items.data());
        PV_CUDA(c, c->sym_items.ensure((items.size() + 1) / 2));
        PV_CUDA(c, c->sym_counter.ensure(1));
        PV_CUDA(c, cudaMemsetAsync(c->sym_counter.p, 0, 2 * sizeof(unsigned), c->stream));
        PV_CUDA(c, cudaMemcpyAsync(c->sym_items.p, items.data(), items.size() * sizeof(unsigned),
                                   cudaMemcpyHostToDevice, c->stream));
        PV_CUDA(c, cudaStreamSynchronize(c->stream));
        c->sym_items_blocks = c->sym.blocks;
    }
    return PV_OK;
}

pv_status require_state(pv_context *c) {
    if (!c->state_valid)
        return fail(c, PV_ERROR_LOGIC, "device state has not been uploaded");
    return PV_OK;
}

// Host-array evaluation of targets [begin, end) (evaluateRange). nonfinite_is_error: the
// VelocityKernel::evaluate finiteness check.
pv_status evaluate_host(pv_context *c, const double *x, const double *y, const double *g, size_t n,
                        size_t begin, size_t end, double *u, double *v, bool nonfinite_is_error) {
    if (!finite_arrays(x, y, g, n))
        return fail(c, PV_ERROR_INVALID_ARGUMENT, "vortex data must be finite");
    if (begin > end || end > n)
        return fail(c, PV_ERROR_OUT_OF_RANGE, "invalid target-vortex range");
    pv_status st = validate_geometry(c, x, y, g, n);
    if (st != PV_OK)
        return st;
    if (begin == end)
        return PV_OK;
    DeviceGuard guard(c->device);
    const size_t np = padded(n);
    const size_t nt = end - begin;
    for (DeviceArray *a : {&c->ex, &c->ey, &c->eg, &c->egs})
        PV_CUDA(c, a->ensure(np));
    PV_CUDA(c, c->eu.ensure(padded(nt)));
    PV_CUDA(c, c->ev.ensure(padded(nt)));
    const EvalPlan plan = plan_evaluation(c->gc.geometry, nt, n, c->sm_count, 0, c->params.precision);
    const size_t stride = padded(nt);
    PV_CUDA(c, c->epu.ensure(static_cast<size_t>(plan.num_chunks) * stride));
    PV_CUDA(c, c->epv.ensure(static_cast<size_t>(plan.num_chunks) * stride));
    const std::vector<double> gs = scaled(c->gc, g, n);
    const size_t bytes = n * sizeof(double);
    PV_CUDA(c, cudaMemcpyAsync(c->ex.p, x, bytes, cudaMemcpyHostToDevice, c->stream));
    PV_CUDA(c, cudaMemcpyAsync(c->ey.p, y, bytes, cudaMemcpyHostToDevice, c->stream));
    PV_CUDA(c, cudaMemcpyAsync(c->eg.p, g, bytes, cudaMemcpyHostToDevice, c->stream));
    PV_CUDA(c, cudaMemcpyAsync(c->egs.p, gs.data(), bytes, cudaMemcpyHostToDevice, c->stream));
    if ((st = reset_control(c)) != PV_OK)
        return st;
    EvalArgs a{};
    a.tx = c->ex.p;
    a.ty = c->ey.p;
    a.sx = c->ex.p;
    a.sy = c->ey.p;
    a.sg = c->egs.p;
    a.t_begin = begin;
    a.t_end = end;
    a.n_src = n;
    a.pu = c->epu.p;
    a.pv = c->epv.p;
    a.stride = stride;
    a.chunk = plan.chunk;
    a.num_chunks = plan.num_chunks;
    a.status = &c->ctl->status;
    a.g = c->gc;
    a.wait_limit = c->wait_limit;
    const bool near = near_field_used(c);
    if (near) {
        const double r = near_radius_for(c, n);
        a.g.near2 = r * r;
        if ((st = ensure_near_lists(c, n)) != PV_OK)
            return st;
        a.near = near_lists(c);
    }
    PV_CUDA(c, counted(c, PV_KERNEL_VELOCITY, 1, [&] {
                return c->params.precision == PV_PRECISION_FP32C
                           ? launch_velocity_fp32c(a, plan, c->stream)
                           : launch_velocity(a, plan, c->stream);
            }));
    if (near) {
        NearPass np{};
        np.lists = a.near;
        np.x = c->ex.p;
        np.y = c->ey.p;
        np.gs = c->egs.p;
        np.n = n;
        np.t_begin = begin;
        np.t_end = end;
        np.pu = c->epu.p;
        np.pv = c->epv.p;
        np.stride = stride;
        np.rows = plan.num_chunks;
        np.g = a.g;
        c->pending_near = np;  // the stage below runs it
    }
    StageArgs s{};
    s.n = nt;
    s.mode = STAGE_REDUCE_ONLY;
    s.reduce = 1;
    s.num_chunks = plan.num_chunks;
    s.stride = stride;
    s.pu = c->epu.p;
    s.pv = c->epv.p;
    s.s = 0;
    s.kx[0] = c->eu.p;
    s.ky[0] = c->ev.p;
    s.ex = c->ex.p;
    s.ey = c->ey.p;
    s.gamma = c->eg.p;
    s.t_offset = begin;
    s.n_src = n;
    s.nonfinite_ok = nonfinite_is_error ? 0 : 1;
    s.ctl = c->ctl;
    s.g = c->gc;
    attach_pending_near(c, s);
    PV_CUDA(c, counted(c, PV_KERNEL_STAGE, 1, [&] { return launch_stage(s, c->stream, c->sm_count); }));
    PV_CUDA(c, cudaMemcpyAsync(u, c->eu.p, nt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PV_CUDA(c, cudaMemcpyAsync(v, c->ev.p, nt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((st = read_control(c)) != PV_OK)
        return st;
    return status_error(c, c->ctl_host->status);
}

pv_status invariants_of(pv_context *c, const double *x, const double *y, const double *g, size_t n,
                        double out[5]) {
    if (n == 0) {
        for (int k = 0; k < 5; ++k)
            out[k] = 0.0;
        return PV_OK;
    }
    PV_CUDA(c, c->inv_scratch.ensure(invariants_scratch_doubles(n, c->sm_count)));
    PV_CUDA(c, c->inv_out.ensure(8));
    pv_status st = reset_control(c);
    if (st != PV_OK)
        return st;
    PV_CUDA(c, counted(c, PV_KERNEL_INVARIANTS, 3, [&] {
                return launch_invariants(x, y, g, n, c->gc, c->inv_scratch.p, c->inv_out.p,
                                         &c->ctl->status, &c->ctl->status2, c->stream);
            }));
    PV_CUDA(c, cudaMemcpyAsync(c->pinned, c->inv_out.p, 5 * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream));
    if ((st = read_control(c)) != PV_OK)
        return st;
    if ((st = status_error(c, c->ctl_host->status)) != PV_OK)
        return st;
    if ((st = status_error(c, c->ctl_host->status2, true)) != PV_OK)
        return st;
    std::memcpy(out, c->pinned, 5 * sizeof(double));
    return PV_OK;
}

} // namespace

namespace pvb {
int make_geometry_consts(const pv_params &p, GeometryConsts &g, std::string &message) {
    return make_consts(p, g, message);
}
void set_thread_error(const std::string &message) { g_create_error = message; }
} // namespace pvb

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

pv_status pv_context_create(const pv_params *params, int device, pv_context **out) {
    if (!out || !params) {
        g_create_error = "null argument";
        return PV_ERROR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    GeometryConsts gc;
    std::string message;
    pv_status st = make_consts(*params, gc, message);
    if (st != PV_OK) {
        g_create_error = message;
        return st;
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || device < 0 || device >= count) {
        g_create_error = std::string("cudaGetDeviceCount: ") +
                         (e != cudaSuccess ? cudaGetErrorString(e) : "device ordinal out of range");
        return PV_ERROR_CUDA;
    }
    DeviceGuard guard(device);
    auto *c = new pv_context();
    c->params = *params;
    c->gc = gc;
    c->device = device;
    const auto bail = [&](cudaError_t err, const char *what) {
        g_create_error = std::string(what) + ": " + cudaGetErrorString(err);
        delete c;
        return PV_ERROR_CUDA;
    };
    if ((e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return bail(e, "cudaDeviceGetAttribute");
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(e, "cudaStreamCreate");
    if ((e = cudaMalloc(&c->ctl, sizeof(DeviceControl))) != cudaSuccess)
        return bail(e, "cudaMalloc(control)");
    if ((e = cudaMallocHost(&c->ctl_host, sizeof(DeviceControl))) != cudaSuccess)
        return bail(e, "cudaMallocHost(control)");
    if ((e = cudaMallocHost(&c->pinned, 16 * sizeof(double))) != cudaSuccess)
        return bail(e, "cudaMallocHost(staging)");
    std::memset(c->ctl_host, 0, sizeof(DeviceControl));
    if ((e = cudaMemcpy(c->ctl, c->ctl_host, sizeof(DeviceControl), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return bail(e, "cudaMemcpy(control)");
    *out = c;
    return PV_OK;
}

void pv_context_destroy(pv_context *ctx) {
    if (!ctx)
        return;
    DeviceGuard guard(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

const char *pv_last_error(const pv_context *ctx) {
    return ctx ? ctx->error.c_str() : g_create_error.c_str();
}

const char *pv_backend_name(void) { return "CUDA/B200"; }

pv_status pv_runtime_details(int device, char *buf, size_t len) {
    cudaDeviceProp prop{};
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        g_create_error = std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e);
        return PV_ERROR_CUDA;
    }
    const std::string text = "cuda_device " + std::to_string(device) + "\ncuda_device_name \"" +
                             prop.name + "\"\ncuda_compute_capability " +
                             std::to_string(prop.major) + "." + std::to_string(prop.minor) +
                             "\ncuda_multiprocessors " + std::to_string(prop.multiProcessorCount);
    if (buf && len) {
        const size_t k = std::min(len - 1, text.size());
        std::memcpy(buf, text.data(), k);
        buf[k] = '\0';
    }
    return PV_OK;
}

pv_status pv_evaluate_range(pv_context *ctx, const double *x, const double *y,
                            const double *circulation, size_t n, size_t begin, size_t end,
                            double *u, double *v) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    return evaluate_host(ctx, x, y, circulation, n, begin, end, u, v, false);
}

pv_status pv_evaluate(pv_context *ctx, const double *x, const double *y, const double *circulation,
                      size_t n, double *u, double *v) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    return evaluate_host(ctx, x, y, circulation, n, 0, n, u, v, true);
}

pv_status pv_invariants(pv_context *ctx, const double *x, const double *y,
                        const double *circulation, size_t n, double out[5]) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    if (!finite_arrays(x, y, circulation, n))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "vortex data must be finite");
    DeviceGuard guard(ctx->device);
    const size_t np = padded(n);
    for (DeviceArray *a : {&ctx->ex, &ctx->ey, &ctx->eg})
        PV_CUDA(ctx, a->ensure(np));
    const size_t bytes = n * sizeof(double);
    if (n) {
        PV_CUDA(ctx, cudaMemcpyAsync(ctx->ex.p, x, bytes, cudaMemcpyHostToDevice, ctx->stream));
        PV_CUDA(ctx, cudaMemcpyAsync(ctx->ey.p, y, bytes, cudaMemcpyHostToDevice, ctx->stream));
        PV_CUDA(ctx, cudaMemcpyAsync(ctx->eg.p, circulation, bytes, cudaMemcpyHostToDevice,
                                     ctx->stream));
    }
    return invariants_of(ctx, ctx->ex.p, ctx->ey.p, ctx->eg.p, n, out);
}

pv_status pv_hamiltonian(pv_context *ctx, const double *x, const double *y,
                         const double *circulation, size_t n, double *hamiltonian) {
    double out[5];
    const pv_status st = pv_invariants(ctx, x, y, circulation, n, out);
    if (st == PV_OK)
        *hamiltonian = out[4];
    return st;
}

pv_status pv_upload_state(pv_context *ctx, const double *x, const double *y,
                          const double *circulation, size_t n) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    if (!finite_arrays(x, y, circulation, n))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "vortex data must be finite");
    pv_status st = validate_geometry(ctx, x, y, circulation, n);
    if (st != PV_OK)
        return st;
    DeviceGuard guard(ctx->device);
    if ((st = ensure_state_capacity(ctx, n)) != PV_OK)
        return st;
    ctx->n = n;
    ctx->fsal_valid = false;
    ctx->prescan_valid = false;
    ctx->state_valid = true;
    ctx->gamma_host.assign(circulation, circulation + n);
    if (n == 0)
        return PV_OK;
    const size_t bytes = n * sizeof(double);
    const std::vector<double> gs = scaled(ctx->gc, circulation, n);
    PV_CUDA(ctx, cudaMemcpyAsync(ctx->x.p, x, bytes, cudaMemcpyHostToDevice, ctx->stream));
    PV_CUDA(ctx, cudaMemcpyAsync(ctx->y.p, y, bytes, cudaMemcpyHostToDevice, ctx->stream));
    PV_CUDA(ctx, cudaMemcpyAsync(ctx->gamma.p, circulation, bytes, cudaMemcpyHostToDevice, ctx->stream));
    PV_CUDA(ctx, cudaMemcpyAsync(ctx->gs.p, gs.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
    PV_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PV_OK;
}

pv_status pv_download_state(pv_context *ctx, double *x, double *y, size_t n) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    if (n != ctx->n)
        return fail(ctx, PV_ERROR_RUNTIME, "host and device vortex populations differ");
    if (n == 0)
        return PV_OK;
    DeviceGuard guard(ctx->device);
    PV_CUDA(ctx, cudaMemcpyAsync(x, ctx->x.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PV_CUDA(ctx, cudaMemcpyAsync(y, ctx->y.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PV_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PV_OK;
}

namespace {
// Enqueues the velocity of the device state into p1x / p1y (stage scratch; the stage velocities
// and the FSAL derivative stay untouched) after clearing the control block. Not counted as a
// stepping evaluation. The status is read by the caller's next read_control.
pv_status enqueue_state_velocity(pv_context *ctx) {
    pv_status st;
    if ((st = reset_control(ctx)) != PV_OK)
        return st;
    if ((st = launch_eval(ctx, ctx->x.p, ctx->y.p)) != PV_OK)
        return st;
    --ctx->evaluations;
    StageArgs s = stage_base(ctx);
    s.mode = STAGE_REDUCE_ONLY;
    s.s = 0;
    s.kx[0] = ctx->p1x.p;
    s.ky[0] = ctx->p1y.p;
    s.ex = ctx->x.p;
    s.ey = ctx->y.p;
    attach_pending_near(ctx, s);
    PV_CUDA(ctx, counted(ctx, PV_KERNEL_STAGE, 1,
                         [&] { return launch_stage(s, ctx->stream, ctx->sm_count); }));
    return PV_OK;
}
} // namespace

pv_status pv_evaluate_state(pv_context *ctx, double *u, double *v, size_t n) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    if (n != ctx->n)
        return fail(ctx, PV_ERROR_RUNTIME, "host and device vortex populations differ");
    if (n == 0)
        return PV_OK;
    DeviceGuard guard(ctx->device);
    if ((st = enqueue_state_velocity(ctx)) != PV_OK)
        return st;
    PV_CUDA(ctx, cudaMemcpyAsync(u, ctx->p1x.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PV_CUDA(ctx, cudaMemcpyAsync(v, ctx->p1y.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if ((st = read_control(ctx)) != PV_OK)
        return st;
    return status_error(ctx, ctx->ctl_host->status);
}

namespace {
// Enqueues one RK4 step (src/timestep.cpp:31-61) on the context stream.
// Stage s of an RK4 step (src/timestep.cpp:31-61): evaluated at the state (s = 0) or at the
// previous stage's position, writing the next position into the ping-pong buffers; stage 3
// writes the combined state.
StageArgs rk4_stage(pv_context *c, double dt, int s) {
    static const double rows[3][3] = {{0.5}, {0.0, 0.5}, {0.0, 0.0, 1.0}};
    double *pos_x[2] = {c->p0x.p, c->p1x.p};
    double *pos_y[2] = {c->p0y.p, c->p1y.p};
    StageArgs a = stage_base(c);
    a.s = s;
    a.ex = s == 0 ? c->x.p : pos_x[(s - 1) & 1];
    a.ey = s == 0 ? c->y.p : pos_y[(s - 1) & 1];
    a.dt = dt;
    a.xt = pos_x[s & 1];
    a.yt = pos_y[s & 1];
    if (s < 3) {
        a.mode = STAGE_POSITION;
        a.ncoef = s + 1;
        for (int j = 0; j <= s; ++j)
            a.coef[j] = rows[s][j];
    } else {
        a.mode = STAGE_RK4_COMBINE;
    }
    return a;
}

// Whole RK4 steps in one cooperative launch: FP64, the ordered kernel's plan (no symmetric
// rows), a small enough population, and no per-launch profiling.
bool rk4_steps_apply(const pv_context *c) {
    return !c->profiling && c->params.precision == PV_PRECISION_FP64 && !c->sym.enabled() &&
           rk4_steps_eligible(c->n, c->plan.num_chunks);
}

pv_status enqueue_rk4_steps(pv_context *c, double dt, uint64_t steps) {
    Rk4Steps p{};
    for (int s = 0; s < 4; ++s)
        p.stage[s] = rk4_stage(c, dt, s);
    p.x = c->x.p;
    p.y = c->y.p;
    p.gs = c->gs.p;
    p.n = c->n;
    p.chunk = c->plan.chunk;
    p.num_chunks = c->plan.num_chunks;
    p.steps = steps;
    p.spin_limit = c->spin_limit;
    PV_CUDA(c, c->rk4_barrier.ensure(1));
    PV_CUDA(c, cudaMemsetAsync(c->rk4_barrier.p, 0, sizeof(unsigned long long), c->stream));
    p.barrier = reinterpret_cast<unsigned long long *>(c->rk4_barrier.p);
    PV_CUDA(c, counted(c, PV_KERNEL_VELOCITY, 1,
                       [&] { return launch_rk4_steps(p, c->sm_count, c->stream); }));
    c->evaluations += 4 * steps;
    return PV_OK;
}

pv_status enqueue_rk4(pv_context *c, double dt) {
    const double *px = c->x.p, *py = c->y.p;
    pv_status st;
    for (int s = 0; s < 4; ++s) {
        if ((st = launch_eval(c, px, py)) != PV_OK)
            return st;
        StageArgs a = rk4_stage(c, dt, s);
        attach_pending_near(c, a);
        PV_CUDA(c, counted(c, PV_KERNEL_STAGE, 1, [&] { return launch_stage(a, c->stream, c->sm_count); }));
        px = a.xt;
        py = a.yt;
    }
    PV_CUDA(c, counted(c, PV_KERNEL_ACCEPT, 1, [&] {
                return launch_accept(c->x.p, c->y.p, px, py, nullptr, nullptr, nullptr, nullptr, c->n,
                                     0, c->ctl, c->stream);
            }));
    return PV_OK;
}
} // namespace

pv_status pv_rk4_step(pv_context *ctx, double dt) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    if (!std::isfinite(dt) || !(dt > 0.0))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "timestep must be finite and positive");
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    ctx->fsal_valid = false;
    ctx->prescan_valid = false;
    if (ctx->n == 0)
        return PV_OK;
    DeviceGuard guard(ctx->device);
    if ((st = reset_control(ctx)) != PV_OK)
        return st;
    if ((st = rk4_steps_apply(ctx) ? enqueue_rk4_steps(ctx, dt, 1) : enqueue_rk4(ctx, dt)) != PV_OK)
        return st;
    if ((st = read_control(ctx)) != PV_OK)
        return st;
    return status_error(ctx, ctx->ctl_host->status);
}

pv_status pv_rk4_advance(pv_context *ctx, double dt, uint64_t steps) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    if (!std::isfinite(dt) || !(dt > 0.0))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "timestep must be finite and positive");
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    ctx->fsal_valid = false;
    ctx->prescan_valid = false;
    if (ctx->n == 0 || steps == 0)
        return PV_OK;
    DeviceGuard guard(ctx->device);
    if ((st = reset_control(ctx)) != PV_OK)
        return st;
    if (rk4_steps_apply(ctx)) {
        if ((st = enqueue_rk4_steps(ctx, dt, steps)) != PV_OK)
            return st;
    } else if (ctx->profiling || steps < 4) {
        for (uint64_t k = 0; k < steps; ++k)
            if ((st = enqueue_rk4(ctx, dt)) != PV_OK)
                return st;
    } else {
        // one step (9 launches at small N, each a few microseconds) captured as a CUDA graph
        // and replayed: the step loop is launch-bound below N ~ 10^4
        uint64_t launches0[PV_KERNEL_KINDS];
        std::copy(ctx->launches, ctx->launches + PV_KERNEL_KINDS, launches0);
        const uint64_t evals0 = ctx->evaluations;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        PV_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        st = enqueue_rk4(ctx, dt);
        const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        if (st != PV_OK || e != cudaSuccess) {
            if (graph)
                cudaGraphDestroy(graph);
            return st != PV_OK ? st
                               : fail(ctx, PV_ERROR_CUDA,
                                      std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
        }
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess)
            return fail(ctx, PV_ERROR_CUDA,
                        std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
        for (uint64_t k = 0; k < steps; ++k) {
            const cudaError_t el = cudaGraphLaunch(exec, ctx->stream);
            if (el != cudaSuccess) {
                cudaGraphExecDestroy(exec);
                return fail(ctx, PV_ERROR_CUDA,
                            std::string("cudaGraphLaunch: ") + cudaGetErrorString(el));
            }
        }
        // the capture counted one step's launches and evaluations
        for (int kind = 0; kind < PV_KERNEL_KINDS; ++kind)
            ctx->launches[kind] += (ctx->launches[kind] - launches0[kind]) * (steps - 1);
        ctx->evaluations += (ctx->evaluations - evals0) * (steps - 1);
        st = read_control(ctx);
        cudaGraphExecDestroy(exec);
        if (st != PV_OK)
            return st;
        return status_error(ctx, ctx->ctl_host->status);
    }
    if ((st = read_control(ctx)) != PV_OK)
        return st;
    return status_error(ctx, ctx->ctl_host->status);
}

namespace {
// One DOPRI5 attempt (src/timestep.cpp:62-120) on the context stream: k0 when it is not cached,
// stages 1..6 with their positions, the error norm and step control of the last stage, and the
// accept kernel. Everything it needs from the host is in the control block.
pv_status enqueue_dopri_attempt(pv_context *ctx, bool need_k0) {
    double *pos_x[2] = {ctx->p0x.p, ctx->p1x.p};
    double *pos_y[2] = {ctx->p0y.p, ctx->p1y.p};
    double w[7];
    for (int j = 0; j < 7; ++j)
        w[j] = kB5[j] - kB4[j];
    pv_status st;
    const double *px = ctx->x.p, *py = ctx->y.p;
    if (need_k0 && (st = launch_eval(ctx, px, py)) != PV_OK)
        return st;
    for (int s = 0; s < 7; ++s) {
        if (s > 0 && (st = launch_eval(ctx, px, py)) != PV_OK)
            return st;
        StageArgs a = stage_base(ctx);
        a.s = s;
        a.reduce = (s > 0 || need_k0) ? 1 : 0;
        a.ex = px;
        a.ey = py;
        a.dt_from_control = 1;
        if (s < 6) {
            a.mode = STAGE_POSITION;
            a.ncoef = s + 1;
            for (int j = 0; j <= s; ++j)
                a.coef[j] = kDopri[s + 1][j];
            a.xt = pos_x[s & 1];
            a.yt = pos_y[s & 1];
        } else {
            a.mode = STAGE_DOPRI_ERROR;
            a.xt = const_cast<double *>(px); // y5, the position k6 was evaluated at
            a.yt = const_cast<double *>(py);
            for (int j = 0; j < 7; ++j)
                a.w[j] = w[j];
        }
        attach_pending_near(ctx, a);
        PV_CUDA(ctx, counted(ctx, PV_KERNEL_STAGE, 1,
                             [&] { return launch_stage(a, ctx->stream, ctx->sm_count); }));
        if (s < 6) {
            px = a.xt;
            py = a.yt;
        }
    }
    PV_CUDA(ctx, counted(ctx, PV_KERNEL_ACCEPT, 1, [&] {
                return launch_accept(ctx->x.p, ctx->y.p, px, py, ctx->kx[0].p, ctx->ky[0].p,
                                     ctx->kx[6].p, ctx->ky[6].p, ctx->n, 1, ctx->ctl, ctx->stream);
            }));
    if (ctx->dipole_configured && ctx->dipole.removal) {
        // the dipole scan of the accepted state (the kernel returns at once after a rejection)
        auto *dev = reinterpret_cast<DipoleCandidateDev *>(ctx->cand.p);
        auto *dev_count = reinterpret_cast<unsigned long long *>(&ctx->ctl->dipole_count);
        PV_CUDA(ctx, counted(ctx, PV_KERNEL_DIPOLE, 1, [&] {
                    return launch_dipole_scan(ctx->x.p, ctx->y.p, ctx->gamma.p, ctx->n, ctx->gc,
                                              ctx->dipole.distance, dev, ctx->cand.cap / 3,
                                              dev_count, ctx->stream, ctx->ctl);
                }));
    }
    return PV_OK;
}
} // namespace

pv_status pv_dopri5_step(pv_context *ctx, double dt, double absolute_tolerance,
                         double relative_tolerance, double minimum_time_step,
                         double maximum_time_step, pv_step_result *result) {
    if (!ctx || !result)
        return PV_ERROR_INVALID_ARGUMENT;
    if (!std::isfinite(dt) || !(dt > 0.0))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "timestep must be finite and positive");
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    if (ctx->n == 0) {
        // Empty population: the reference's error is 0, so the step is accepted with factor 5.
        ctx->evaluations += ctx->fsal_valid ? 6 : 7;
        ctx->fsal_valid = true;
        const double s = dt * 5.0;
        result->accepted_time_step = dt;
        result->suggested_time_step =
            s < minimum_time_step ? minimum_time_step : (maximum_time_step < s ? maximum_time_step : s);
        result->normalized_error = 0.0;
        result->rejected_steps = 0;
        return PV_OK;
    }
    DeviceGuard guard(ctx->device);
    std::memset(ctx->ctl_host, 0, sizeof(DeviceControl));
    ctx->ctl_host->dt = dt;
    ctx->ctl_host->absolute_tolerance = absolute_tolerance;
    ctx->ctl_host->relative_tolerance = relative_tolerance;
    ctx->ctl_host->minimum_time_step = minimum_time_step;
    ctx->ctl_host->maximum_time_step = maximum_time_step;
    PV_CUDA(ctx, cudaMemcpyAsync(ctx->ctl, ctx->ctl_host, sizeof(DeviceControl),
                                 cudaMemcpyHostToDevice, ctx->stream));
    ctx->prescan_valid = false;
    const bool prescan = ctx->dipole_configured && ctx->dipole.removal;
    if (prescan)
        PV_CUDA(ctx, ctx->cand.ensure(3 * 64));
    bool need_k0 = !ctx->fsal_valid;
    for (int attempt = 0; attempt < 40; ++attempt) {
        if (need_k0) {
            if ((st = enqueue_dopri_attempt(ctx, need_k0)) != PV_OK)
                return st;
        } else {
            // the FSAL attempt is the same launch sequence every time (dt lives in the control
            // block): one CUDA graph, captured again only when the population, the plan, a
            // buffer or the profiling switch changes. With profiling on, the capture holds the
            // per-launch events, which every replay records.
            const std::vector<const void *> key = attempt_key(ctx);
            if (ctx->attempt_graph && key != ctx->graph_key)
                drop_graphs(ctx);
            if (!ctx->attempt_graph) {
                const uint64_t evals0 = ctx->evaluations;
                uint64_t launches0[PV_KERNEL_KINDS];
                std::copy(ctx->launches, ctx->launches + PV_KERNEL_KINDS, launches0);
                cudaGraph_t graph = nullptr;
                PV_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
                ctx->capturing = true;
                ctx->capture_timers.clear();
                st = enqueue_dopri_attempt(ctx, false);
                ctx->capturing = false;
                const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
                ctx->graph_timers.swap(ctx->capture_timers);
                ctx->capture_timers.clear();
                if (st != PV_OK || e != cudaSuccess) {
                    if (graph)
                        cudaGraphDestroy(graph);
                    drop_graphs(ctx);
                    return st != PV_OK ? st
                                       : fail(ctx, PV_ERROR_CUDA, std::string("cudaStreamEndCapture: ") +
                                                                      cudaGetErrorString(e));
                }
                const cudaError_t ei = cudaGraphInstantiate(&ctx->attempt_graph, graph, 0);
                cudaGraphDestroy(graph);
                if (ei != cudaSuccess) {
                    ctx->attempt_graph = nullptr;
                    drop_graphs(ctx);
                    return fail(ctx, PV_ERROR_CUDA,
                                std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
                }
                // the capture counted; the launch below counts again
                ctx->evaluations = evals0;
                std::copy(launches0, launches0 + PV_KERNEL_KINDS, ctx->launches);
                ctx->graph_key = key;
            }
            PV_CUDA(ctx, cudaGraphLaunch(ctx->attempt_graph, ctx->stream));
            for (const auto &t : ctx->graph_timers)
                ctx->pending.push_back(t);
            ctx->evaluations += 6;
            ctx->launches[PV_KERNEL_VELOCITY] += 6;
            if (near_field_used(ctx))
                ctx->launches[PV_KERNEL_NEAR] += 6;
            ctx->launches[PV_KERNEL_STAGE] += 7;
            ctx->launches[PV_KERNEL_ACCEPT] += 1;
            if (prescan)
                ctx->launches[PV_KERNEL_DIPOLE] += 1;
        }
        need_k0 = false;
        if ((st = read_control(ctx)) != PV_OK)
            return st;
        if (ctx->ctl_host->status != 0) {
            ctx->fsal_valid = false;
            return status_error(ctx, ctx->ctl_host->status);
        }
        if (ctx->ctl_host->accepted) {
            ctx->fsal_valid = true;
            ctx->prescan_valid = prescan;
            ctx->prescan_count = ctx->ctl_host->dipole_count;
            result->accepted_time_step = ctx->ctl_host->result[0];
            result->suggested_time_step = ctx->ctl_host->result[1];
            result->normalized_error = ctx->ctl_host->result[2];
            result->rejected_steps = static_cast<unsigned>(ctx->ctl_host->result[3]);
            return PV_OK;
        }
    }
    return fail(ctx, PV_ERROR_RUNTIME, "adaptive integrator could not satisfy tolerance");
}

pv_status pv_invalidate_derivative(pv_context *ctx) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    ctx->fsal_valid = false;
    return PV_OK;
}

pv_status pv_state_invariants(pv_context *ctx, double out[5]) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    DeviceGuard guard(ctx->device);
    return invariants_of(ctx, ctx->x.p, ctx->y.p, ctx->gamma.p, ctx->n, out);
}

pv_status pv_dipole_scan(pv_context *ctx, double threshold, pv_dipole_candidate *out,
                         size_t capacity, size_t *count) {
    if (!ctx || !count)
        return PV_ERROR_INVALID_ARGUMENT;
    if (!std::isfinite(threshold) || !(threshold > 0.0))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "dipoleRemovalDistance must be positive");
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    *count = 0;
    if (ctx->n == 0)
        return PV_OK;
    DeviceGuard guard(ctx->device);
    static_assert(sizeof(DipoleCandidateDev) == 3 * sizeof(double), "candidate layout");
    static_assert(sizeof(pv_dipole_candidate) == sizeof(DipoleCandidateDev), "candidate layout");
    const size_t cap = std::max<size_t>(capacity, 1);
    PV_CUDA(ctx, ctx->cand.ensure(3 * cap));
    auto *dev = reinterpret_cast<DipoleCandidateDev *>(ctx->cand.p);
    auto *dev_count = reinterpret_cast<unsigned long long *>(&ctx->ctl->dipole_count);
    PV_CUDA(ctx, counted(ctx, PV_KERNEL_DIPOLE, 1, [&] {
                return launch_dipole_scan(ctx->x.p, ctx->y.p, ctx->gamma.p, ctx->n, ctx->gc,
                                          threshold, dev, cap, dev_count, ctx->stream);
            }));
    if ((st = read_control(ctx)) != PV_OK)
        return st;
    const unsigned long long found = ctx->ctl_host->dipole_count;
    *count = static_cast<size_t>(found);
    const size_t k = std::min<size_t>(static_cast<size_t>(found), capacity);
    if (k && out) {
        PV_CUDA(ctx, cudaMemcpyAsync(out, dev, k * sizeof(pv_dipole_candidate),
                                     cudaMemcpyDeviceToHost, ctx->stream));
        PV_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return PV_OK;
}

namespace {

// Every candidate of the device state (rescanning once with room for all of them).
pv_status scan_all(pv_context *ctx, double threshold, std::vector<pv_dipole_candidate> &out) {
    size_t cap = std::max<size_t>(ctx->cand.cap / 3, 256), count = 0;
    out.resize(cap);
    pv_status st = pv_dipole_scan(ctx, threshold, out.data(), cap, &count);
    if (st == PV_OK && count > cap) {
        if (count > (static_cast<size_t>(1) << 26))
            return fail(ctx, PV_ERROR_CAPACITY, "more than 2^26 close-dipole candidates");
        out.resize(count);
        st = pv_dipole_scan(ctx, threshold, out.data(), count, &count);
    }
    out.resize(std::min(count, out.size()));
    return st;
}

struct Position {
    double x, y;
};

// The reinjection draws of src/dipole.cpp:129-180, in the reference's order and arithmetic.
struct Reinjector {
    pv_context *ctx;
    std::uniform_real_distribution<double> unit{0.0, 1.0};

    bool periodic() const { return ctx->params.geometry == PV_GEOMETRY_PERIODIC; }
    double u() { return unit(ctx->dipole_random); }

    Position random_position() {
        const pv_params &p = ctx->params;
        if (periodic()) {
            const double px = (u() - 0.5) * p.box_length_x;
            const double py = (u() - 0.5) * p.box_length_y;
            return {px, py};
        }
        const double radius = p.disk_radius * std::sqrt(u());
        const double angle = 2.0 * kPi * u();
        return {radius * std::cos(angle), radius * std::sin(angle)};
    }

    // injectSingle: a wall event puts its one vortex back uniformly in the disk.
    Position single() {
        const double radius = ctx->params.disk_radius * std::sqrt(u());
        const double angle = 2.0 * kPi * u();
        return {radius * std::cos(angle), radius * std::sin(angle)};
    }

    // injectPair: two independent positions, or (paired) a first position and a second one at the
    // mean spacing of the original population in a random direction.
    bool pair(size_t population, Position &first, Position &second) {
        const pv_params &p = ctx->params;
        const double area = periodic() ? p.box_length_x * p.box_length_y
                                       : kPi * p.disk_radius * p.disk_radius;
        const double spacing = std::sqrt(area / static_cast<double>(population));
        first = random_position();
        second = random_position();
        if (ctx->dipole.reinjection != PV_REINJECT_PAIRED)
            return true;
        for (size_t attempt = 0; attempt < 100000; ++attempt) {
            first = random_position();
            const double angle = 2.0 * kPi * u();
            second = {first.x + spacing * std::cos(angle), first.y + spacing * std::sin(angle)};
            if (periodic()) {
                second.x = std::remainder(second.x, p.box_length_x);
                second.y = std::remainder(second.y, p.box_length_y);
                return true;
            }
            if (second.x * second.x + second.y * second.y < p.disk_radius * p.disk_radius)
                return true;
        }
        return false;
    }
};

} // namespace

pv_status pv_dipole_configure(pv_context *ctx, const pv_dipole_config *config) {
    if (!ctx || !config)
        return PV_ERROR_INVALID_ARGUMENT;
    // the dipole checks of SimParams::validate (src/read.cpp:55-99)
    const double d = config->distance;
    if (!std::isfinite(d))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "simulation parameters must be finite");
    if (!std::isfinite(d * d) || (d > 0.0 && d * d == 0.0))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT,
                    "radius or distance is outside the supported numeric range");
    if (!(d > 0.0))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "dipoleRemovalDistance must be positive");
    if (config->reinjection < PV_REINJECT_NONE || config->reinjection > PV_REINJECT_PAIRED)
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT,
                    "dipoleReinjection must be none, independent, or paired");
    if (!config->removal && config->reinjection != PV_REINJECT_NONE)
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "dipoleReinjection requires dipoleRemoval true");
    if (ctx->params.geometry == PV_GEOMETRY_INFINITE && config->reinjection != PV_REINJECT_NONE)
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT,
                    "dipole reinjection is available only for periodic and disk geometries");
    ctx->dipole = *config;
    ctx->dipole_configured = true;
    ctx->prescan_valid = false;
    // DipoleManager seeds its engine with the run seed mixed by this constant
    // (src/dipole.cpp:29-30); runs and checkpoints stay interchangeable only with the same seeding
    ctx->dipole_random.seed(config->random_seed ^ 0xd1b54a32d192ed03ULL);
    ctx->removed_pairs = ctx->reinjected_pairs = 0;
    return PV_OK;
}

pv_status pv_dipole_process(pv_context *ctx, size_t *events) {
    if (!ctx || !events)
        return PV_ERROR_INVALID_ARGUMENT;
    *events = 0;
    if (!ctx->dipole_configured)
        return fail(ctx, PV_ERROR_LOGIC, "dipole events have not been configured");
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    const size_t n = ctx->n;
    if (!ctx->dipole.removal || n == 0)
        return PV_OK;
    if (ctx->prescan_valid && ctx->prescan_count == 0)
        return PV_OK;  // the last accepted DOPRI5 attempt scanned this very state: no candidate
    ctx->prescan_valid = false;
    std::vector<pv_dipole_candidate> cands;
    if ((st = scan_all(ctx, ctx->dipole.distance, cands)) != PV_OK)
        return st;
    if (cands.empty())
        return PV_OK;  // before any use of the generator, as the reference returns
    // closest first; ties by (first, second) -- src/dipole.cpp:79-85
    std::sort(cands.begin(), cands.end(), [](const pv_dipole_candidate &a,
                                             const pv_dipole_candidate &b) {
        if (a.distance_squared != b.distance_squared)
            return a.distance_squared < b.distance_squared;
        return a.first != b.first ? a.first < b.first : a.second < b.second;
    });
    // greedy disjoint selection (src/dipole.cpp:87-100)
    struct Event {
        double first_gamma, second_gamma;
        bool wall;
    };
    std::vector<unsigned char> selected(n, 0);
    std::vector<Event> chosen;
    std::vector<unsigned long long> removed;
    for (const pv_dipole_candidate &c : cands) {
        if (selected[c.first] || (c.second < n && selected[c.second]))
            continue;
        selected[c.first] = 1;
        removed.push_back(c.first);
        if (c.second < n) {
            selected[c.second] = 1;
            removed.push_back(c.second);
            chosen.push_back({ctx->gamma_host[c.first], ctx->gamma_host[c.second], false});
        } else {
            chosen.push_back({ctx->gamma_host[c.first], 0.0, true});
        }
    }
    std::sort(removed.begin(), removed.end());
    const size_t m = removed.size();
    const size_t survivors = n - m;

    DeviceGuard guard(ctx->device);
    // compaction on the device: state -> stage-position scratch, then the buffers trade places
    // (the cached derivative is invalidated below, so the scratch holds nothing live)
    PV_CUDA(ctx, ctx->removed_index.ensure(m));
    PV_CUDA(ctx, cudaMemcpyAsync(ctx->removed_index.p, removed.data(),
                                 m * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                 ctx->stream));
    PV_CUDA(ctx, counted(ctx, PV_KERNEL_DIPOLE, 1, [&] {
                return launch_compact_survivors(
                    ctx->x.p, ctx->y.p, ctx->gamma.p, ctx->gs.p, n,
                    reinterpret_cast<const unsigned long long *>(ctx->removed_index.p), m,
                    ctx->p0x.p, ctx->p0y.p, ctx->p1x.p, ctx->p1y.p, ctx->stream);
            }));
    std::swap(ctx->x, ctx->p0x);
    std::swap(ctx->y, ctx->p0y);
    std::swap(ctx->gamma, ctx->p1x);
    std::swap(ctx->gs, ctx->p1y);
    std::vector<double> gamma_new;
    gamma_new.reserve(n);
    for (size_t i = 0; i < n; ++i)
        if (!selected[i])
            gamma_new.push_back(ctx->gamma_host[i]);
    ctx->removed_pairs += chosen.size();
    ctx->fsal_valid = false;
    ctx->n = survivors;

    // reinjection, appended after the survivors (src/dipole.cpp:116-124)
    std::vector<double> ax, ay, ag;
    if (ctx->dipole.reinjection != PV_REINJECT_NONE) {
        Reinjector r{ctx};
        for (const Event &e : chosen) {
            if (e.wall) {
                const Position q = r.single();
                ax.push_back(q.x);
                ay.push_back(q.y);
                ag.push_back(e.first_gamma);
                continue;
            }
            Position a{}, b{};
            if (!r.pair(n, a, b)) {
                ctx->gamma_host = gamma_new;
                return fail(ctx, PV_ERROR_RUNTIME,
                            "could not find a valid paired reinjection position");
            }
            ax.push_back(a.x);
            ay.push_back(a.y);
            ag.push_back(e.first_gamma);
            ax.push_back(b.x);
            ay.push_back(b.y);
            ag.push_back(e.second_gamma);
        }
        ctx->reinjected_pairs += chosen.size();
    }
    const size_t added = ax.size();
    if (added) {
        const std::vector<double> ags = scaled(ctx->gc, ag.data(), added);
        const size_t bytes = added * sizeof(double);
        PV_CUDA(ctx, cudaMemcpyAsync(ctx->x.p + survivors, ax.data(), bytes, cudaMemcpyHostToDevice,
                                     ctx->stream));
        PV_CUDA(ctx, cudaMemcpyAsync(ctx->y.p + survivors, ay.data(), bytes, cudaMemcpyHostToDevice,
                                     ctx->stream));
        PV_CUDA(ctx, cudaMemcpyAsync(ctx->gamma.p + survivors, ag.data(), bytes,
                                     cudaMemcpyHostToDevice, ctx->stream));
        PV_CUDA(ctx, cudaMemcpyAsync(ctx->gs.p + survivors, ags.data(), bytes,
                                     cudaMemcpyHostToDevice, ctx->stream));
        gamma_new.insert(gamma_new.end(), ag.begin(), ag.end());
    }
    ctx->n = survivors + added;
    ctx->gamma_host.swap(gamma_new);
    PV_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    collect_timers(ctx);
    if ((st = ensure_state_capacity(ctx, ctx->n)) != PV_OK)
        return st;
    *events = chosen.size();
    // the checks the reference's driver meets when it re-uploads the new population
    // (src/main.cpp:329-333 -> uploadDeviceState): zero net circulation in the periodic box and
    // reinjected vortices strictly inside the disk
    if (ctx->params.geometry == PV_GEOMETRY_PERIODIC &&
        (st = validate_geometry(ctx, nullptr, nullptr, ctx->gamma_host.data(), ctx->n)) != PV_OK)
        return st;
    if (ctx->params.geometry == PV_GEOMETRY_DISK &&
        (st = validate_geometry(ctx, ax.data(), ay.data(), ag.data(), added)) != PV_OK)
        return st;
    return PV_OK;
}

pv_status pv_dipole_state(const pv_context *ctx, uint64_t *removed, uint64_t *reinjected,
                          char *engine_state, size_t capacity, size_t *length) {
    if (!ctx || !length)
        return PV_ERROR_INVALID_ARGUMENT;
    if (removed)
        *removed = ctx->removed_pairs;
    if (reinjected)
        *reinjected = ctx->reinjected_pairs;
    std::ostringstream text;
    text << ctx->dipole_random;
    const std::string s = text.str();
    *length = s.size();
    if (!engine_state || capacity <= s.size())
        return PV_ERROR_CAPACITY;
    std::memcpy(engine_state, s.c_str(), s.size() + 1);
    return PV_OK;
}

pv_status pv_dipole_restore(pv_context *ctx, uint64_t removed, uint64_t reinjected,
                            const char *engine_state) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    if (!ctx->dipole_configured)
        return fail(ctx, PV_ERROR_LOGIC, "dipole events have not been configured");
    if (engine_state && *engine_state) {
        std::istringstream input(engine_state);
        std::mt19937_64 engine;
        if (!(input >> engine))
            return fail(ctx, PV_ERROR_RUNTIME, "invalid random-generator state in checkpoint");
        ctx->dipole_random = engine;
    }
    ctx->removed_pairs = removed;
    ctx->reinjected_pairs = reinjected;
    return PV_OK;
}

namespace {

// Formats rows of (x, y, g[, u, v]) device arrays on the device and copies the packed text to
// out when it fits. One synchronisation for the byte count (and the velocity status), one for the
// copy.
pv_status format_rows(pv_context *ctx, RowFormat f, char *out, size_t capacity, size_t *length,
                      bool check_velocity) {
    const size_t n = f.n;
    const size_t blocks = (n + 255) / 256;
    auto words = [](size_t bytes) { return (bytes + 7) / 8; };
    PV_CUDA(ctx, ctx->fmt_stage.ensure(words(n * static_cast<size_t>(f.stride))));
    PV_CUDA(ctx, ctx->fmt_out.ensure(words(n * static_cast<size_t>(f.stride))));
    PV_CUDA(ctx, ctx->fmt_len.ensure(words(n * sizeof(uint32_t))));
    PV_CUDA(ctx, ctx->fmt_block.ensure(blocks + 1));
    char *dev_out = reinterpret_cast<char *>(ctx->fmt_out.p);
    auto *block = reinterpret_cast<unsigned long long *>(ctx->fmt_block.p);
    PV_CUDA(ctx, counted(ctx, PV_KERNEL_OUTPUT, 3, [&] {
                return launch_format_rows(f, reinterpret_cast<char *>(ctx->fmt_stage.p),
                                          reinterpret_cast<uint32_t *>(ctx->fmt_len.p), block,
                                          dev_out, ctx->stream);
            }));
    auto *total = reinterpret_cast<unsigned long long *>(ctx->pinned);
    PV_CUDA(ctx, cudaMemcpyAsync(total, block + blocks, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    pv_status st;
    if ((st = read_control(ctx)) != PV_OK)
        return st;
    if (check_velocity && (st = status_error(ctx, ctx->ctl_host->status)) != PV_OK)
        return st;
    *length = static_cast<size_t>(*total);
    if (*length > capacity || (!out && *length))
        return fail(ctx, PV_ERROR_CAPACITY, "output buffer is smaller than the formatted frame");
    if (*length) {
        PV_CUDA(ctx, cudaMemcpyAsync(out, dev_out, *length, cudaMemcpyDeviceToHost, ctx->stream));
        PV_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return PV_OK;
}

} // namespace

pv_status pv_format_trajectory(pv_context *ctx, double time, uint64_t frame, char *out,
                               size_t capacity, size_t *length) {
    if (!ctx || !length)
        return PV_ERROR_INVALID_ARGUMENT;
    *length = 0;
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    if (ctx->n == 0)
        return PV_OK;
    DeviceGuard guard(ctx->device);
    if ((st = enqueue_state_velocity(ctx)) != PV_OK)
        return st;
    RowFormat f{};
    f.x = ctx->x.p;
    f.y = ctx->y.p;
    f.g = ctx->gamma.p;
    f.u = ctx->p1x.p;
    f.v = ctx->p1y.p;
    f.n = ctx->n;
    f.kind = ROWS_TRAJECTORY;
    f.stride = kTrajectoryRowStride;
    f.prefix_len = format_prefix(time, frame, f.prefix);
    return format_rows(ctx, f, out, capacity, length, true);
}

pv_status pv_format_trajectory_host(pv_context *ctx, double time, uint64_t frame, const double *x,
                                    const double *y, const double *circulation, const double *u,
                                    const double *v, size_t n, char *out, size_t capacity,
                                    size_t *length) {
    if (!ctx || !length || (n && (!x || !y || !circulation || !u || !v)))
        return PV_ERROR_INVALID_ARGUMENT;
    *length = 0;
    if (n == 0)
        return PV_OK;
    DeviceGuard guard(ctx->device);
    const size_t np = padded(n);
    for (DeviceArray *a : {&ctx->ex, &ctx->ey, &ctx->eg, &ctx->eu, &ctx->ev})
        PV_CUDA(ctx, a->ensure(np));
    const size_t bytes = n * sizeof(double);
    const double *src[5] = {x, y, circulation, u, v};
    DeviceArray *dst[5] = {&ctx->ex, &ctx->ey, &ctx->eg, &ctx->eu, &ctx->ev};
    for (int k = 0; k < 5; ++k)
        PV_CUDA(ctx, cudaMemcpyAsync(dst[k]->p, src[k], bytes, cudaMemcpyHostToDevice, ctx->stream));
    RowFormat f{};
    f.x = ctx->ex.p;
    f.y = ctx->ey.p;
    f.g = ctx->eg.p;
    f.u = ctx->eu.p;
    f.v = ctx->ev.p;
    f.n = n;
    f.kind = ROWS_TRAJECTORY;
    f.stride = kTrajectoryRowStride;
    f.prefix_len = format_prefix(time, frame, f.prefix);
    return format_rows(ctx, f, out, capacity, length, false);
}

pv_status pv_format_checkpoint_vortices(pv_context *ctx, char *out, size_t capacity,
                                        size_t *length) {
    if (!ctx || !length)
        return PV_ERROR_INVALID_ARGUMENT;
    *length = 0;
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    if (ctx->n == 0)
        return PV_OK;
    DeviceGuard guard(ctx->device);
    RowFormat f{};
    f.x = ctx->x.p;
    f.y = ctx->y.p;
    f.g = ctx->gamma.p;
    f.n = ctx->n;
    f.kind = ROWS_CHECKPOINT;
    f.stride = kCheckpointRowStride;
    return format_rows(ctx, f, out, capacity, length, false);
}

pv_status pv_download_circulation(pv_context *ctx, double *circulation, size_t n) {
    if (!ctx || (n && !circulation))
        return PV_ERROR_INVALID_ARGUMENT;
    pv_status st = require_state(ctx);
    if (st != PV_OK)
        return st;
    if (n != ctx->n)
        return fail(ctx, PV_ERROR_RUNTIME, "host and device vortex populations differ");
    std::copy(ctx->gamma_host.begin(), ctx->gamma_host.end(), circulation);
    return PV_OK;
}

pv_status pv_state_plan(const pv_context *ctx, pv_plan_info *info) {
    if (!ctx || !info)
        return PV_ERROR_INVALID_ARGUMENT;
    info->symmetric = ctx->sym.enabled() ? 1 : 0;
    info->rows = ctx->sym.enabled() ? ctx->sym.blocks : ctx->plan.num_chunks;
    info->targets_per_thread = ctx->plan.per_thread;
    info->chunk = ctx->plan.chunk;
    info->symmetric_min_ctas = ctx->sym.enabled() ? ctx->sym.min_ctas : 0;
    info->symmetric_targets = ctx->sym.enabled() ? ctx->sym.targets : 0;
    info->symmetric_grid_ctas = ctx->sym.enabled() ? ctx->sym.grid_ctas : 0;
    return PV_OK;
}

pv_status pv_state_size(const pv_context *ctx, size_t *n) {
    if (!ctx || !n)
        return PV_ERROR_INVALID_ARGUMENT;
    *n = ctx->n;
    return PV_OK;
}

pv_status pv_evaluation_count(const pv_context *ctx, uint64_t *count) {
    if (!ctx || !count)
        return PV_ERROR_INVALID_ARGUMENT;
    *count = ctx->evaluations;
    return PV_OK;
}

pv_status pv_set_tuning(int geometry, int precision, int log2_n, int per_thread) {
    if (!tuning_store(geometry, precision, log2_n, per_thread)) {
        g_create_error = "invalid tuning entry";
        return PV_ERROR_INVALID_ARGUMENT;
    }
    return PV_OK;
}

pv_status pv_set_symmetric_tuning(int geometry, int precision, int log2_n, int mode, int min_ctas,
                                  int targets) {
    if (!symmetric_tuning_store(geometry, precision, log2_n, mode, min_ctas, targets)) {
        g_create_error = "invalid symmetric tuning entry";
        return PV_ERROR_INVALID_ARGUMENT;
    }
    return PV_OK;
}

pv_status pv_get_symmetric_tuning(int geometry, int precision, int log2_n, int *mode,
                                  int *min_ctas, int *targets) {
    if (!mode || !min_ctas || !targets || log2_n < 0 || log2_n >= 40)
        return PV_ERROR_INVALID_ARGUMENT;
    const int packed = symmetric_tuning_lookup(geometry, precision, size_t(1) << log2_n);
    *mode = packed & 15;
    *min_ctas = (packed >> 4) & 15;
    *targets = (packed >> 8) & 15;
    return PV_OK;
}

pv_status pv_set_symmetric_grid(int geometry, int precision, int log2_n, int ctas_per_sm) {
    if (!symmetric_grid_store(geometry, precision, log2_n, ctas_per_sm)) {
        g_create_error = "invalid symmetric grid entry";
        return PV_ERROR_INVALID_ARGUMENT;
    }
    return PV_OK;
}

pv_status pv_get_symmetric_grid(int geometry, int precision, int log2_n, int *ctas_per_sm) {
    if (!ctas_per_sm || log2_n < 0 || log2_n >= 40)
        return PV_ERROR_INVALID_ARGUMENT;
    *ctas_per_sm = symmetric_grid_lookup(geometry, precision, size_t(1) << log2_n);
    return PV_OK;
}

pv_status pv_get_tuning(int geometry, int precision, int log2_n, int *per_thread) {
    if (!per_thread || log2_n < 0 || log2_n >= 40)
        return PV_ERROR_INVALID_ARGUMENT;
    *per_thread = tuning_lookup(geometry, precision, size_t(1) << log2_n);
    return PV_OK;
}

pv_status pv_context_stream(const pv_context *ctx, void **stream) {
    if (!ctx || !stream)
        return PV_ERROR_INVALID_ARGUMENT;
    *stream = static_cast<void *>(ctx->stream);
    return PV_OK;
}

pv_status pv_set_near_field(pv_context *ctx, double radius) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    if (std::isnan(radius) || std::isinf(radius))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "near-field radius must be finite");
    ctx->near_radius = radius < 0.0 ? -1.0 : radius;
    if (ctx->state_valid && near_field_used(ctx)) {
        DeviceGuard guard(ctx->device);
        const double r = near_radius_for(ctx, ctx->n);
        ctx->gc.near2 = r * r;
        const pv_status st = ensure_near_lists(ctx, ctx->n);
        if (st != PV_OK)
            return st;
        PV_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return PV_OK;
}

pv_status pv_get_near_field(const pv_context *ctx, double *radius) {
    if (!ctx || !radius)
        return PV_ERROR_INVALID_ARGUMENT;
    *radius = near_field_used(ctx) ? std::sqrt(ctx->gc.near2) : 0.0;
    return PV_OK;
}

pv_status pv_set_wait_limits(pv_context *ctx, int64_t copy_polls, int64_t barrier_polls) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    if (copy_polls > static_cast<int64_t>(UINT32_MAX) ||
        barrier_polls > static_cast<int64_t>(UINT32_MAX))
        return fail(ctx, PV_ERROR_INVALID_ARGUMENT, "wait limit out of range");
    ctx->wait_limit = copy_polls < 0 ? kWaitLimit : static_cast<uint32_t>(copy_polls);
    ctx->spin_limit = barrier_polls < 0 ? kGridSpinLimit : static_cast<uint32_t>(barrier_polls);
    return PV_OK;
}

pv_status pv_set_profiling(pv_context *ctx, int enabled) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    ctx->profiling = enabled != 0;
    return PV_OK;
}

pv_status pv_get_kernel_stats(pv_context *ctx, pv_kernel_stats *out) {
    if (!ctx || !out)
        return PV_ERROR_INVALID_ARGUMENT;
    DeviceGuard guard(ctx->device);
    PV_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    collect_timers(ctx);
    for (int k = 0; k < PV_KERNEL_KINDS; ++k) {
        out->launches[k] = ctx->launches[k];
        out->timed_launches[k] = ctx->timed[k];
        out->milliseconds[k] = ctx->milliseconds[k];
    }
    return PV_OK;
}

pv_status pv_reset_kernel_stats(pv_context *ctx) {
    if (!ctx)
        return PV_ERROR_INVALID_ARGUMENT;
    DeviceGuard guard(ctx->device);
    PV_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    collect_timers(ctx);
    for (int k = 0; k < PV_KERNEL_KINDS; ++k) {
        ctx->launches[k] = 0;
        ctx->timed[k] = 0;
        ctx->milliseconds[k] = 0.0;
    }
    return PV_OK;
}

pv_status pv_probe_peak(int device, int kind, double *flops_per_second) {
    if (!flops_per_second || (kind != 0 && kind != 1))
        return PV_ERROR_INVALID_ARGUMENT;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        g_create_error = "no such CUDA device";
        return PV_ERROR_CUDA;
    }
    DeviceGuard guard(device);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *sink = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess)
        return PV_ERROR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256;
    // Double the work until one launch runs for at least 100 ms (after two warm-up launches), and
    // keep the iteration count and the time of that same launch.
    int iterations = 1024, timed_iterations = 0;
    float ms = 0.0f;
    cudaError_t e = cudaSuccess;
    for (int pass = 0; pass < 16 && e == cudaSuccess; ++pass) {
        cudaEventRecord(e0);
        e = launch_peak_probe(kind, blocks, threads, iterations, sink, nullptr);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        timed_iterations = iterations;
        if (ms >= 100.0f && pass >= 2)
            break;
        if (ms < 100.0f && iterations < (1 << 22))
            iterations *= 2;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) {
        g_create_error = std::string("peak probe: ") + cudaGetErrorString(e);
        return PV_ERROR_CUDA;
    }
    const double fmas = static_cast<double>(blocks) * threads * timed_iterations * 8.0;
    *flops_per_second = 2.0 * fmas / (ms * 1e-3);
    return PV_OK;
}

} // extern "C"
