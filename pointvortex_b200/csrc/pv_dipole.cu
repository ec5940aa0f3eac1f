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
#include "pv_pair32.cuh"

#include <cmath>
#include <limits>

namespace pvb {

namespace {
constexpr int kDT = 64;  // targets per block (one per thread)
constexpr int kDS = 64;  // sources per block

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

// The exact test of one pair (i < j), bit for bit the reference's (see the file comment).
__device__ __forceinline__ void exact_pair(const GeometryConsts &gc, double xi, double yi,
                                           bool neg_i, size_t i, double xj, double yj, double gj,
                                           size_t j, double thr2, DipoleCandidateDev *out,
                                           size_t capacity, unsigned long long *count) {
    double dx = xi - xj, dy = yi - yj;
    if (gc.geometry == GEO_PERIODIC) {
        dx = exact_remainder(dx, gc.lx, gc.inv_lx, gc.half_lx);
        dy = exact_remainder(dy, gc.ly, gc.inv_ly, gc.half_ly);
    }
    const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
    if (d2 < thr2 && gj != 0.0 && neg_i != static_cast<bool>(signbit(gj)))
        push(out, capacity, count, i, j, d2);
}

// Blocks cover the tiles (target block I, source block J >= I), b = J (J + 1) / 2 + I: every
// unordered pair i < j once, and no block starts only to find its tile below the diagonal.
//
// Prefilter (prefilter != 0): the squared minimum-image distance in FP32 from double-float
// coordinates (hi = fp32(x), lo = fp32(x - hi)): d = (t_hi - s_hi) + (t_lo - s_lo), then
// r = d - m L with m = round(d / L) and L = l_hi + l_lo, in f32x2 lanes (x, y). Only a pair whose
// FP32 distance is not above the target's bound thr2f, or is not finite, takes the exact FP64
// test, so the candidates are exactly the reference's. The bound covers the FP32 errors: with M
// the largest coordinate magnitude of the target and the block's sources, each component of d
// is within 2^-22 * 2M of the exact difference (two roundings of differences of coordinates up
// to M, the lo parts' own error below 2^-48 M), and r adds 2^-22 |r| (two roundings; a wrong m
// is only possible for |r| near L/2, a pair out of reach); so a true candidate (|r| < thr) has
// |r_fp32| < thr + e per component with e = 2^-21 M + 2^-22 thr, and its computed squared
// distance is below thr2f = (thr + 2e)^2 (1 + 2^-20). The host turns the prefilter off when the
// threshold is not small against the box (0.125 L).
__global__ void __launch_bounds__(kDT)
    dipole_scan_kernel(const double *x, const double *y, const double *g, size_t n,
                       GeometryConsts gc, double thr2, int prefilter,
                       DipoleCandidateDev *out, size_t capacity, unsigned long long *count,
                       const DeviceControl *gate) {
    __shared__ alignas(16) float4 s_neg[kDS];  // (-x_hi, -y_hi, -x_lo, -y_lo) of the sources
    __shared__ double sx[kDS], sy[kDS], sg[kDS];
    __shared__ unsigned s_mag;                  // bits of the sources' largest |coordinate|
    pdl_enter();
    if (gate && !gate->accepted)  // after a DOPRI5 attempt: only the accepted state is scanned
        return;
    const unsigned b = blockIdx.x;
    unsigned J = static_cast<unsigned>((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
    while (static_cast<unsigned long long>(J + 1) * (J + 2) / 2 <= b)
        ++J;
    while (static_cast<unsigned long long>(J) * (J + 1) / 2 > b)
        --J;
    const unsigned I = b - J * (J + 1) / 2;
    const size_t i0 = static_cast<size_t>(I) * kDT;
    const size_t j0 = static_cast<size_t>(J) * kDS;
    if (threadIdx.x == 0)
        s_mag = 0u;
    __syncthreads();
    for (int t = threadIdx.x; t < kDS; t += kDT) {
        const size_t jl = j0 + t;
        const double xj = jl < n ? x[jl] : 0.0, yj = jl < n ? y[jl] : 0.0;
        sx[t] = xj;
        sy[t] = yj;
        sg[t] = jl < n ? g[jl] : 0.0;
        const float4 f = f32::split_position(xj, yj);
        s_neg[t] = make_float4(-f.x, -f.y, -f.z, -f.w);
        // non-negative floats order as their bits; a NaN's bits exceed every finite one's
        const float mag = fmaxf(fabsf(static_cast<float>(xj)), fabsf(static_cast<float>(yj)));
        atomicMax(&s_mag, __float_as_uint(isnan(xj) || isnan(yj) ? __int_as_float(0x7fc00000)
                                                                   : mag));
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
    if (prefilter) {
        // this target's bound (see above), rounded up to FP32; a NaN coordinate makes it NaN,
        // and then every pair takes the exact test
        const float smag = __uint_as_float(s_mag);
        const double m = fmax(fmax(fabs(xi), fabs(yi)), static_cast<double>(smag));
        const double thr = sqrt(thr2);
        const double e = 0x1p-21 * m + 0x1p-22 * thr;
        const double bound = (thr + 2.0 * e) * (thr + 2.0 * e) * (1.0 + 0x1p-20);
        const float thr2f = isnan(smag) || isnan(xi) || isnan(yi) ? __int_as_float(0x7fc00000)
                                                                  : __double2float_ru(bound);
        const float4 t = f32::split_position(xi, yi);
        const float2 th = make_float2(t.x, t.y), tl = make_float2(t.z, t.w);
        const float inv_l = static_cast<float>(gc.inv_lx);
        const float l_hi = static_cast<float>(gc.lx);
        const float l_lo = static_cast<float>(gc.lx - static_cast<double>(l_hi));
        // the squared FP32 distance to source jj; rounding to an integer by adding and subtracting
        // 1.5 * 2^23 (round to nearest even for |q| < 2^22, as rintf) keeps it on the FMA pipe
        const auto dist2 = [&](int jj) {
            const float4 s = s_neg[jj];
            float2 r = f32::add2(f32::add2(th, make_float2(s.x, s.y)),
                                 f32::add2(tl, make_float2(s.z, s.w)));
            if (periodic) {
                const float2 q = f32::mul2(r, f32::splat2(inv_l));
                const float2 m = f32::add2(f32::add2(q, f32::splat2(12582912.0f)),
                                           f32::splat2(-12582912.0f));
                r = f32::fma2(m, f32::splat2(-l_lo), f32::fma2(m, f32::splat2(-l_hi), r));
            }
            return fmaf(r.x, r.x, r.y * r.y);
        };
        // no branch per pair: the smallest distance decides whether the exact tests run (rarely).
        // In the diagonal tile only sources after the target count (the target itself is at 0).
        float closest = __int_as_float(0x7f800000);
        bool nonfinite = false;
        const int first = I == J ? static_cast<int>(i - j0) + 1 : 0;
#pragma unroll 4
        for (int jj = first; jj < jcount; ++jj) {
            const float d2f = dist2(jj);
            closest = fminf(closest, d2f);
            nonfinite |= !(d2f == d2f);
        }
        if (!(closest > thr2f) || nonfinite)
            for (int jj = first; jj < jcount; ++jj)
                if (!(dist2(jj) > thr2f))
                    exact_pair(gc, xi, yi, neg_i, i, sx[jj], sy[jj], sg[jj], j0 + jj, thr2, out,
                               capacity, count);
    } else {
#pragma unroll 4
        for (int jj = 0; jj < jcount; ++jj)
            if (j0 + jj > i)
                exact_pair(gc, xi, yi, neg_i, i, sx[jj], sy[jj], sg[jj], j0 + jj, thr2, out,
                           capacity, count);
    }
    // the wall image of each target once: in the block of its own tile
    if (gc.geometry == GEO_DISK && I == J) {
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
    const size_t nb = (n + kDT - 1) / kDT;  // kDT == kDS: target and source blocks alike
    const size_t blocks = nb * (nb + 1) / 2;
    if (blocks > 0x7fffffffu)
        return cudaErrorInvalidValue;
    const double thr2 = threshold * threshold;
    // the FP32 prefilter needs a threshold well inside the FP32 range and, in the box, small
    // against the box (so the FP32 minimum image is the exact one for every pair within reach)
    const bool small = thr2 > 0.0 && thr2 < 1e30 &&
                       (g.geometry != GEO_PERIODIC ||
                        (threshold < 0.125 * g.lx && threshold < 0.125 * g.ly &&
                         g.lx == g.ly));
    return launch_pdl(dipole_scan_kernel, dim3(static_cast<unsigned>(blocks)), dim3(kDT), 0,
                      stream, x, y, gamma, n, g, thr2, small ? 1 : 0, out, capacity, count, gate);
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
