// pv_noalloc.cu — velocity evaluation that allocates nothing.
//
// pv_evaluate_device_noalloc() serves callers that must not allocate GPU memory themselves or let
// a library do it for them: a host application that owns every byte of device memory through its
// own pool and hands out only the buffers it placed, or a tight time-stepping loop that cannot
// afford the implicit device-wide synchronisation of cudaMalloc/cudaFree. The caller passes its
// inputs and outputs as device pointers; everything else the evaluation needs (the scaled
// circulations, the per-chunk partial sums and the status word) lives in one fixed array in this
// file, sized at build time. Every GPU that loads the library holds that array until the process
// exits.
//
// The array is shared by all calls on a device and keeps whatever the previous call left in it:
// each call clears the status word and overwrites every scratch value it reads. Calls whose GPU
// work overlaps in time (different streams, or different host threads, on one device) race on the
// array and corrupt each other's results; callers must order them.
//
// In host code the array's name is only a host-side stand-in for the symbol, not a device
// address: the first call on each device (with that device current) asks the runtime for the
// array's device address with cudaGetSymbolAddress and caches it. Make that first call on a
// device before any stream capture begins. The cache is keyed by device ordinal and assumes the
// runtime's primary context of that device for the life of the process: after cudaDeviceReset,
// or with another context current, the cached address is not valid.
#include "pvb200.h"
#include "pv_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

using namespace pvb;

namespace {

// 8 MiB: the first 32 doubles hold the DeviceControl block, then the scaled circulations (one
// padded array) and the u/v chunk partials (two arrays per chunk).
constexpr size_t kScratchDoubles = size_t(1) << 20;
constexpr size_t kControlDoubles = sizeof(DeviceControl) / sizeof(double);
constexpr size_t kPad = 256;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr size_t padded_n(size_t n) { return (n + kPad - 1) / kPad * kPad; }

// Largest population that fits with a single chunk: control + scaled circulations + 2 partials.
constexpr size_t kMaxVortices = (kScratchDoubles - kControlDoubles) / 3 / kPad * kPad;
static_assert(kMaxVortices == PV_NOALLOC_MAX_VORTICES, "header limit matches the scratch array");

std::mutex g_setup_mutex;
double *g_scratch_address[64] = {};

// Failures are reported through pv_last_error(NULL), like those of pv_context_create.
pv_status noalloc_fail(pv_status code, const std::string &message) {
    set_thread_error(message);
    return code;
}

// Device address of the scratch array on the current device (looked up once per device).
pv_status scratch_for_device(int device, double **out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (device < 0 || device >= 64)
        return noalloc_fail(PV_ERROR_CUDA, "device ordinal outside the supported range");
    if (!g_scratch_address[device]) {
        void *address = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&address, g_noalloc_scratch);
        if (e != cudaSuccess)
            return noalloc_fail(PV_ERROR_CUDA,
                                std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_address[device] = static_cast<double *>(address);
    }
    *out = g_scratch_address[device];
    return PV_OK;
}

// Status of a periodic population whose circulations do not sum to zero. Set together with
// status2 = 1, so that the velocity and reduction kernels (which return at once on a non-zero
// status) leave u and v untouched; map_status reports it as the reference's invalid_argument.
constexpr int kStatusNotNeutral = 100;
constexpr int kNeutralTile = 2048;  // circulations staged in shared memory per pass

// One block: scaled circulations and the input checks of the reference, in the reference's order
// (src/compute.cpp:203-211 for the box): finiteness of every value (validateVortexArrays,
// src/vortex.h:7-14), then the box's zero net circulation (validatePeriodicCirculation,
// src/compute.cpp:31-38) or the disk's containment (validateDiskPositions, src/compute.cpp:41-48).
// The net circulation and the sum of |Gamma| are added by one thread in index order, as the
// reference adds them, so that a population near the 1e-12 threshold gets the same verdict here
// as from the reference and from pv_evaluate; the block stages the circulations in shared memory
// for it.
__global__ void __launch_bounds__(1024)
    prepare_kernel(const double *x, const double *y, const double *gamma, size_t n,
                   GeometryConsts g, double *scaled, DeviceControl *ctl) {
    __shared__ double s_gamma[kNeutralTile];
    __shared__ int s_bad;
    if (threadIdx.x == 0)
        s_bad = 0;
    __syncthreads();
    int bad = 0;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double xi = x[i], yi = y[i], gi = gamma[i];
        if (!isfinite(xi) || !isfinite(yi) || !isfinite(gi))
            bad = max(bad, 2);
        else if (g.geometry == GEO_DISK &&
                 __dadd_rn(__dmul_rn(xi, xi), __dmul_rn(yi, yi)) >= g.radius2)
            bad = max(bad, 1);
        scaled[i] = scaled_circulation(g, gi);
    }
    if (bad)
        atomicMax(&s_bad, bad);
    __syncthreads();
    if (s_bad == 2) {
        if (threadIdx.x == 0)
            set_status(&ctl->status, ST_NONFINITE_POSITION);
        return;
    }
    if (g.geometry == GEO_PERIODIC) {
        double total = 0.0, absolute = 0.0;  // meaningful in thread 0 only
        for (size_t base = 0; base < n; base += kNeutralTile) {
            const size_t len = min(static_cast<size_t>(kNeutralTile), n - base);
            for (size_t k = threadIdx.x; k < len; k += blockDim.x)
                s_gamma[k] = gamma[base + k];
            __syncthreads();
            if (threadIdx.x == 0)
                for (size_t k = 0; k < len; ++k) {
                    total += s_gamma[k];
                    absolute += fabs(s_gamma[k]);
                }
            __syncthreads();
        }
        if (threadIdx.x == 0 && fabs(total) > 1e-12 * fmax(1.0, absolute)) {
            ctl->status2 = 1;
            set_status(&ctl->status, kStatusNotNeutral);
        }
        return;
    }
    if (threadIdx.x == 0 && s_bad == 1)
        set_status(&ctl->status, ST_OUTSIDE_DISK);
}

pv_status map_status(const DeviceControl &c, int geometry) {
    if (c.status2 == 1)  // set only for finite data, and no later kernel ran
        return noalloc_fail(PV_ERROR_INVALID_ARGUMENT,
                            "periodic box requires zero total circulation");
    switch (c.status) {
    case ST_OK:
        return PV_OK;
    case ST_NONFINITE_POSITION:
        return noalloc_fail(PV_ERROR_INVALID_ARGUMENT, "vortex data must be finite");
    case ST_OUTSIDE_DISK:
        return noalloc_fail(PV_ERROR_INVALID_ARGUMENT, "vortex lies on or outside the disk");
    case ST_COINCIDENT:
        return noalloc_fail(PV_ERROR_RUNTIME,
                            geometry == GEO_PERIODIC ? "coincident periodic vortices"
                            : geometry == GEO_DISK   ? "coincident vortices in disk"
                                 : "coincident vortices in singular point-vortex kernel");
    case ST_NONFINITE_VELOCITY:
        return noalloc_fail(PV_ERROR_RUNTIME,
                            "non-finite velocity; check scales and close encounters");
    case ST_TIMEOUT:
        return noalloc_fail(PV_ERROR_RUNTIME, "a bounded device wait timed out");
    default:
        return noalloc_fail(PV_ERROR_RUNTIME, "device reported status " + std::to_string(c.status));
    }
}

} // namespace

extern "C" {

pv_status pv_evaluate_device_noalloc(const pv_params *params, const double *x, const double *y,
                                     const double *circulation, size_t n, double *u, double *v,
                                     void *stream_handle) {
    if (!params)
        return noalloc_fail(PV_ERROR_INVALID_ARGUMENT, "null parameters");
    GeometryConsts g;
    std::string message;
    pv_status st = static_cast<pv_status>(make_geometry_consts(*params, g, message));
    if (st != PV_OK)
        return noalloc_fail(st, message);
    if (params->precision != PV_PRECISION_FP64)
        return noalloc_fail(PV_ERROR_INVALID_ARGUMENT,
                            "the allocation-free entry point evaluates in FP64 only");
    if (n > kMaxVortices)
        return noalloc_fail(PV_ERROR_INVALID_ARGUMENT,
                            "population " + std::to_string(n) +
                                " exceeds the allocation-free limit of " +
                                std::to_string(kMaxVortices) + " vortices");
    if (n == 0)
        return PV_OK;
    if (!x || !y || !circulation || !u || !v)
        return noalloc_fail(PV_ERROR_INVALID_ARGUMENT, "null device pointer");
    for (const void *p : {static_cast<const void *>(x), static_cast<const void *>(y),
                          static_cast<const void *>(circulation)})
        if (reinterpret_cast<uintptr_t>(p) % 16 != 0)
            return noalloc_fail(PV_ERROR_INVALID_ARGUMENT,
                                "input device arrays must be 16-byte aligned");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
        return noalloc_fail(PV_ERROR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    double *scratch = nullptr;
    if ((st = scratch_for_device(device, &scratch)) != PV_OK)
        return st;
    int sm_count = 0;
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);

    // Split the sources into as many chunks as the plan wants and the scratch array can hold.
    const size_t np = padded_n(n);
    const size_t max_chunks = (kScratchDoubles - kControlDoubles - np) / (2 * np);
    EvalPlan plan = plan_evaluation(g.geometry, n, n, sm_count);
    if (static_cast<size_t>(plan.num_chunks) > max_chunks) {
        size_t chunk = (n + max_chunks - 1) / max_chunks;
        chunk = (chunk + 1) & ~static_cast<size_t>(1);
        plan.chunk = static_cast<int>(chunk);
        plan.num_chunks = static_cast<int>((n + chunk - 1) / chunk);
    }
    auto *ctl = reinterpret_cast<DeviceControl *>(scratch);
    double *scaled = scratch + kControlDoubles;
    double *pu = scaled + np;
    double *pv = pu + static_cast<size_t>(plan.num_chunks) * np;

    const auto cuda = [](cudaError_t err, const char *what) {
        return noalloc_fail(PV_ERROR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    };
    if ((e = cudaMemsetAsync(ctl, 0, sizeof(DeviceControl), stream)) != cudaSuccess)
        return cuda(e, "cudaMemsetAsync");
    prepare_kernel<<<1, 1024, 0, stream>>>(x, y, circulation, n, g, scaled, ctl);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return cuda(e, "prepare kernel");

    EvalArgs a{};
    a.tx = x;
    a.ty = y;
    a.sx = x;
    a.sy = y;
    a.sg = scaled;
    a.t_begin = 0;
    a.t_end = n;
    a.n_src = n;
    a.pu = pu;
    a.pv = pv;
    a.stride = np;
    a.chunk = plan.chunk;
    a.num_chunks = plan.num_chunks;
    a.status = &ctl->status;
    a.g = g;
    if ((e = launch_velocity(a, plan, stream)) != cudaSuccess)
        return cuda(e, "velocity kernel");

    StageArgs s{};
    s.n = n;
    s.mode = STAGE_REDUCE_ONLY;
    s.reduce = 1;
    s.num_chunks = plan.num_chunks;
    s.stride = np;
    s.pu = pu;
    s.pv = pv;
    s.s = 0;
    s.kx[0] = u;
    s.ky[0] = v;
    s.ex = x;
    s.ey = y;
    s.gamma = circulation;
    s.n_src = n;
    s.ctl = ctl;
    s.g = g;
    if ((e = launch_stage(s, stream, sm_count)) != cudaSuccess)
        return cuda(e, "reduction kernel");

    DeviceControl host{};
    if ((e = cudaMemcpyAsync(&host, ctl, sizeof(DeviceControl), cudaMemcpyDeviceToHost, stream)) !=
        cudaSuccess)
        return cuda(e, "cudaMemcpyAsync");
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess)
        return cuda(e, "cudaStreamSynchronize");
    return map_status(host, g.geometry);
}

} // extern "C"
