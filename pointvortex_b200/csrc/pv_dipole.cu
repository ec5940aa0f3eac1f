// pv_dipole.cu — close-dipole candidate scan on the GPU, plus the peak-throughput probes.
//
// The scan replaces the O(N^2/2) candidate loop of DipoleManager::process (src/dipole.cpp:49-78)
// that the reference runs on the host after every accepted step, with a full download of the
// state first (src/main.cpp:327-328). A candidate count of zero means process() would return 0
// before touching its random generator (src/dipole.cpp:101-102), so nothing else runs. Otherwise
// only the candidates cross to the host (pv_dipole_process selects there) and the survivors are
// compacted in place of the state by compact_survivors_kernel (src/dipole.cpp:104-113), so the
// state itself never leaves the device.
//
// Candidate test, bit for bit as the reference computes it (g++ on x86-64 does not contract):
//   opposite signs (Gamma != 0, signbit differs);
//   dx = remainder(x_i - x_j, Lx) in the periodic box (exactly rounded by definition), else x_i - x_j;
//   d2 = dx*dx + dy*dy (two products, one sum, each rounded) < threshold*threshold;
//   disk wall image: r2 = x*x + y*y > 0, image = (R*R - r2)/sqrt(r2), image*image < threshold^2.
#include "pv_internal.h"

namespace pvb {

namespace {
constexpr int kDT = 128;  // targets per block
constexpr int kDS = 32;   // sources per block

__device__ __forceinline__ void push(DipoleCandidateDev *out, size_t capacity,
                                     unsigned long long *count, unsigned long long a,
                                     unsigned long long b, double d2) {
    const unsigned long long slot = atomicAdd(count, 1ull);
    if (slot < capacity) {
        out[slot].first = a;
        out[slot].second = b;
        out[slot].distance_squared = d2;
    }
}

// Block (source tile of kDS, target block of kDT): every unordered pair i < j once. Short source
// tiles give many CTAs, so the scan hides its latency at small N too.
__global__ void __launch_bounds__(kDT)
    dipole_scan_kernel(const double *x, const double *y, const double *g, size_t n,
                       GeometryConsts gc, double thr2, DipoleCandidateDev *out, size_t capacity,
                       unsigned long long *count, const DeviceControl *gate) {
    pdl_enter();
    if (gate && !gate->accepted)  // after a DOPRI5 attempt: only the accepted state is scanned
        return;
    const size_t i0 = static_cast<size_t>(blockIdx.y) * kDT;
    const size_t j0 = static_cast<size_t>(blockIdx.x) * kDS;
    if (j0 + kDS <= i0 + 1)  // every source of the tile precedes every target of the block
        return;
    __shared__ double sx[kDS], sy[kDS], sg[kDS];
    if (threadIdx.x < kDS) {
        const size_t jl = j0 + threadIdx.x;
        sx[threadIdx.x] = jl < n ? x[jl] : 0.0;
        sy[threadIdx.x] = jl < n ? y[jl] : 0.0;
        sg[threadIdx.x] = jl < n ? g[jl] : 0.0;
    }
    __syncthreads();
    const size_t i = i0 + threadIdx.x;
    if (i >= n)
        return;
    const double xi = x[i], yi = y[i], gi = g[i];
    if (gi == 0.0)
        return;
    const bool periodic = gc.geometry == GEO_PERIODIC;
    const int jcount = static_cast<int>(min(static_cast<size_t>(kDS), n - j0));
    const bool neg_i = signbit(gi);
    // every pair's distance first (no divergence); the order and sign conditions only for the
    // rare pair closer than the threshold
#pragma unroll 4
    for (int jj = 0; jj < jcount; ++jj) {
        double dx = xi - sx[jj], dy = yi - sy[jj];
        if (periodic) {
            dx = exact_remainder(dx, gc.lx, gc.inv_lx, gc.half_lx);
            dy = exact_remainder(dy, gc.ly, gc.inv_ly, gc.half_ly);
        }
        const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        if (d2 < thr2) {
            const double gj = sg[jj];
            if (j0 + jj > i && gj != 0.0 && neg_i != static_cast<bool>(signbit(gj)))
                push(out, capacity, count, i, j0 + jj, d2);
        }
    }
    // the wall image of each target once: in the block whose source tile starts at the target block
    if (gc.geometry == GEO_DISK && j0 == i0) {
        const double r2 = __dadd_rn(__dmul_rn(xi, xi), __dmul_rn(yi, yi));
        if (r2 > 0.0) {
            const double image = __ddiv_rn(__dsub_rn(gc.radius2, r2), __dsqrt_rn(r2));
            const double i2 = __dmul_rn(image, image);
            if (i2 < thr2)
                push(out, capacity, count, i, n, i2);
        }
    }
}

// Peak probes: independent FMA chains (8 per thread) on the FP64 or FP32 pipe, or chains of the
// FP64 reciprocal approximation, to measure the arithmetic roofline of this GPU at load clocks.
__global__ void probe_dfma(int iterations, double *sink) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        a[k] = 1.0 + 1e-9 * (threadIdx.x + k);
    const double b = 0.999999999, c = 1e-12;
    for (int it = 0; it < iterations; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        s += a[k];
    if (s == 12345.678)
        sink[0] = s;
}

__global__ void probe_ffma(int iterations, double *sink) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        a[k] = 1.0f + 1e-6f * (threadIdx.x + k);
    const float b = 0.9999999f, c = 1e-7f;
    for (int it = 0; it < iterations; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            a[k] = fmaf(a[k], b, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        s += a[k];
    if (s == 12345.678f)
        sink[0] = s;
}
} // namespace

cudaError_t launch_dipole_scan(const double *x, const double *y, const double *gamma, size_t n,
                               const GeometryConsts &g, double threshold,
                               DipoleCandidateDev *out, size_t capacity,
                               unsigned long long *count, cudaStream_t stream,
                               const DeviceControl *gate) {
    // Gated (inside a DOPRI5 attempt): the count is the control block's, which the attempt's
    // step control has zeroed, so no memset node splits the attempt's chain of kernels.
    if (gate && count != &gate->dipole_count)
        return cudaErrorInvalidValue;
    if (!gate) {
        const cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess)
            return e;
    }
    if (n == 0)
        return cudaSuccess;
    const size_t nt = (n + kDT - 1) / kDT, ns = (n + kDS - 1) / kDS;
    if (nt > 65535)
        return cudaErrorInvalidValue;
    const dim3 grid(static_cast<unsigned>(ns), static_cast<unsigned>(nt));
    return launch_pdl(dipole_scan_kernel, grid, dim3(kDT), 0, stream, x, y, gamma, n, g,
                      threshold * threshold, out, capacity, count, gate);
}

namespace {
// Survivor i (not in the sorted removal list) moves to i - (removals below i): the order of
// src/dipole.cpp:110-113. Reads the state arrays, writes the compacted copies.
__global__ void __launch_bounds__(256)
    compact_survivors_kernel(const double *__restrict__ x, const double *__restrict__ y,
                             const double *__restrict__ g, const double *__restrict__ gs, size_t n,
                             const unsigned long long *__restrict__ removed, size_t m,
                             double *__restrict__ ox, double *__restrict__ oy,
                             double *__restrict__ og, double *__restrict__ ogs) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    size_t lo = 0, hi = m;
    while (lo < hi) {
        const size_t mid = (lo + hi) >> 1;
        if (removed[mid] < i)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo < m && removed[lo] == i)
        return;
    const size_t o = i - lo;
    ox[o] = x[i];
    oy[o] = y[i];
    og[o] = g[i];
    ogs[o] = gs[i];
}
} // namespace

cudaError_t launch_compact_survivors(const double *x, const double *y, const double *g,
                                     const double *gs, size_t n, const unsigned long long *removed,
                                     size_t m, double *ox, double *oy, double *og, double *ogs,
                                     cudaStream_t stream) {
    if (n == 0)
        return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    compact_survivors_kernel<<<blocks, 256, 0, stream>>>(x, y, g, gs, n, removed, m, ox, oy, og,
                                                         ogs);
    return cudaGetLastError();
}

cudaError_t launch_peak_probe(int kind, int blocks, int threads, int iterations, double *sink,
                              cudaStream_t stream) {
    if (kind == 0)
        probe_dfma<<<blocks, threads, 0, stream>>>(iterations, sink);
    else
        probe_ffma<<<blocks, threads, 0, stream>>>(iterations, sink);
    return cudaGetLastError();
}

} // namespace pvb
