// pv_common.cuh — device helpers shared by every kernel of libpvb200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pvb {

// ---------------------------------------------------------------------------------------------
// Device status word. Codes are ranked so that atomicMax keeps the error the reference would have
// thrown first when several vortices fail in one kernel (its evaluateRange reports a singular pair
// before evaluate() checks finiteness; a stage's velocity errors precede the next position's
// validation; finiteness is validated before disk containment). Every kernel of a step returns
// at once when the word is non-zero, so an earlier kernel's error always stands. The host maps
// the codes to the reference's exception types and messages (pv_context.cu).
enum DeviceStatus : int {
    ST_OK = 0,
    ST_DOPRI_FAILED = 1,          // src/timestep.cpp:116-117 (runtime_error)
    ST_OUTSIDE_DISK = 2,          // validateDiskPositions, src/compute.cpp:41-48 (invalid_argument)
    ST_NONFINITE_POSITION = 3,    // validateVortexArrays, src/vortex.h:7-14 (invalid_argument)
    ST_DOPRI_NONFINITE = 4,       // src/timestep.cpp:92-94 (runtime_error)
    ST_NONFINITE_VELOCITY = 5,    // VelocityKernel::evaluate, src/compute.cpp:66-68 (runtime_error)
    ST_COINCIDENT = 6,            // singular pair (runtime_error; message depends on the geometry)
    ST_NONFINITE_MOMENT = 7,      // computeMoments, src/compute.cpp:22-25 (runtime_error)
    ST_NONFINITE_HAMILTONIAN = 8, // src/compute.cpp:153-154, 160-161 (runtime_error)
    ST_OUTSIDE_DISK_H = 9,        // DiskKernel::hamiltonian, src/compute.cpp:267-268 (invalid_argument)
    ST_TIMEOUT = 10,              // a bounded device wait gave up (runtime_error)
};

// Per-context control block in device memory. One 256-byte line; the host mirrors it in pinned
// memory and reads it back once per synchronisation point.
struct DeviceControl {
    int status;
    int accepted;              // DOPRI5: last attempt accepted
    unsigned rejected;         // DOPRI5: rejections in the current step
    unsigned blocks_done;      // last-block-done counter of the error reduction
    unsigned long long err_bits; // max scaled error of the attempt, as ordered bits (>= 0)
    unsigned long long dipole_count;
    int status2;               // status word of the Hamiltonian pass (invariants)
    int pad0;
    double dt;                 // DOPRI5: step size of the current attempt
    double absolute_tolerance, relative_tolerance, minimum_time_step, maximum_time_step;
    double result[4];          // accepted dt, suggested dt, normalised error, rejected
    double pad[18];
};
static_assert(sizeof(DeviceControl) == 256, "control block is one 256-byte line");

// Programmatic dependent launch. The kernels of a step are launched so that the next one may be
// scheduled while the previous one drains (launch_pdl); each of them first waits until the grid
// before it has completed and its memory is visible, then lets its own successor be scheduled.
// Without a programmatic predecessor the wait returns at once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void set_status(int *status, int code) { atomicMax(status, code); }
// For end-of-operation checks that the reference makes only when nothing failed earlier.
__device__ __forceinline__ void set_status_if_clean(int *status, int code) {
    atomicCAS(status, 0, code);
}

// ---------------------------------------------------------------------------------------------
// Shared-memory staging with the Tensor Memory Accelerator's bulk (non-tensor) copy engine:
// one elected thread arms an mbarrier with the expected byte count and issues
// cp.async.bulk global->shared copies that complete on that barrier. No cluster multicast.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned) into this CTA's shared
// memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gmem_src, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}

// Bounded wait: gives up after `limit` polls (each try_wait may itself suspend the thread for a
// hardware-chosen interval), reports ST_TIMEOUT and returns false. A bulk copy from valid global
// memory always completes, so the bound only turns an impossible hang into an error status.
// limit = 0 gives up without polling (the tests of the timeout exits use it).
constexpr uint32_t kWaitLimit = 1u << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *status,
                                                  uint32_t limit = kWaitLimit) {
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity))
            return true;
    set_status(status, ST_TIMEOUT);
    return false;
}

// After a bounded wait gave up at tile k of a two-stage ring (tile k on stage k & 1, phase parity
// (k >> 1) & 1), waits for the bulk copies still in flight -- tile k's and, when it was issued,
// tile k + 1's -- so that none lands in shared memory after the CTA has exited. Run by the thread
// that issued them, before it returns. The wait is bounded again, with the default limit.
__device__ __forceinline__ void mbar_drain(uint64_t *bars, uint32_t k, bool next_issued) {
    const uint32_t end = k + (next_issued ? 2u : 1u);
    for (uint32_t q = k; q < end; ++q)
        for (uint32_t it = 0; it < kWaitLimit && !mbar_try_wait(&bars[q & 1], (q >> 1) & 1); ++it) {
        }
}

// ---------------------------------------------------------------------------------------------
// FP64 reciprocal: hardware approximation (rcp.approx.ftz.f64) refined by one third-order
// Newton–Raphson (Householder) step, y1 = y0 (1 + e + e^2) with e = 1 - d y0, which triples the
// number of correct bits. Zero, subnormal and infinite d produce NaN, which the callers treat as
// "recompute this target with the IEEE reference form".
__device__ __forceinline__ double rcp_approx_f64(double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    return r;
}

__device__ __forceinline__ double rcp_refined(double d) {
    const double r = rcp_approx_f64(d);
    double e = fma(-d, r, 1.0);
    e = fma(e, e, e);
    return fma(r, e, r);
}

// IEEE remainder(a, L) (exact by definition), fast path for |a/L| of moderate size: with
// n = rint(a/L) the single-rounding fma gives a - nL exactly whenever |a - nL| < L/2, and the
// test below can only pass in that case; anything else (ties, huge or non-finite a) takes the
// library remainder().
__device__ __forceinline__ double exact_remainder(double a, double L, double inv_L, double half_L) {
    const double n = rint(a * inv_L);
    const double r = fma(-n, L, a);
    if (fabs(r) < half_L)
        return r;
    return remainder(a, L);
}

// sinh, cosh, sin and cos of t for |t| <= pi/2 from the power series of exp(t) and exp(i t),
// grouped by powers t^(4k+r) so that the hyperbolic and circular functions share every term:
//   sinh t = t (E1 + t^2 O1),  sin t = t (E1 - t^2 O1),  cosh t = E0 + t^2 O0,  cos t = E0 - t^2 O0
// with E1 = sum_k w^k/(4k+1)!, O1 = sum_k w^k/(4k+3)!, E0 = sum_k w^k/(4k)!, O0 = sum_k w^k/(4k+2)!,
// w = t^4 in [0, (pi/2)^4]. Horner in w. Every output keeps its exact parity in t (odd: t times a
// polynomial in w; even: a polynomial in w and t^2), which the once-per-unordered-pair kernels rely
// on.
//
// sinh_cosh_sin_cos: the Taylor polynomials, truncated after the w^5 (E) and w^4 (O) terms; the
// first omitted term is below 2e-17 relative. The Hamiltonian uses it: its periodic image product
// adds up to 2M + 1 = 129 factors whose logarithms accumulate the series' error.
__device__ __forceinline__ void sinh_cosh_sin_cos(double t, double &sh, double &ch, double &s,
                                                  double &c) {
    const double t2 = t * t, w = t2 * t2;
    double e1 = fma(w, 1.9572941063391263e-20, 2.8114572543455206e-15); // 1/21!, 1/17!
    e1 = fma(w, e1, 1.6059043836821613e-10);                             // 1/13!
    e1 = fma(w, e1, 2.7557319223985893e-06);                             // 1/9!
    e1 = fma(w, e1, 0.008333333333333333);                             // 1/5!
    e1 = fma(w, e1, 1.0);
    double o1 = fma(w, 8.22063524662433e-18, 7.647163731819816e-13); // 1/19!, 1/15!
    o1 = fma(w, o1, 2.505210838544172e-08);                             // 1/11!
    o1 = fma(w, o1, 0.0001984126984126984);                             // 1/7!
    o1 = fma(w, o1, 0.16666666666666666);                             // 1/3!
    double e0 = fma(w, 4.110317623312165e-19, 4.779477332387385e-14); // 1/20!, 1/16!
    e0 = fma(w, e0, 2.08767569878681e-09);                             // 1/12!
    e0 = fma(w, e0, 2.48015873015873e-05);                             // 1/8!
    e0 = fma(w, e0, 0.041666666666666664);                             // 1/4!
    e0 = fma(w, e0, 1.0);
    double o0 = fma(w, 1.5619206968586225e-16, 1.1470745597729725e-11); // 1/18!, 1/14!
    o0 = fma(w, o0, 2.755731922398589e-07);                             // 1/10!
    o0 = fma(w, o0, 0.001388888888888889);                             // 1/6!
    o0 = fma(w, o0, 0.5);                                                // 1/2!
    const double t3 = t * t2, te1 = t * e1;
    sh = fma(t3, o1, te1);
    s = fma(-t3, o1, te1);
    ch = fma(t2, o0, e0);
    c = fma(-t2, o0, e0);
}

// sinh_cosh_sin_cos_economized: one coefficient fewer per polynomial, for the velocity's pair
// terms. Each of the four is the Taylor polynomial of one degree more economized by Lanczos'
// method (its top term traded for the shifted Chebyshev polynomial of that degree on
// [0, (pi/2)^4], computed in exact rational arithmetic): E1 and E0 keep five coefficients, O1 and
// O0 four. Relative error of the polynomials over the interval: E1 3.2e-19, E0 6.7e-18, O1
// 5.3e-16, O0 3.4e-15; of the functions (double evaluation against 30-digit references): sinh,
// sin below 6e-16 relative, cosh below 1.7e-15 relative, cos below 4.1e-15 absolute. In a pair
// term cos(t) only scales sin(x^) = 2 sin(t) cos(t), a factor of the term, so the term's error
// stays at the 1e-15 level, three orders below the parity tolerance.
__device__ __forceinline__ void sinh_cosh_sin_cos_economized(double t, double &sh, double &ch,
                                                             double &s, double &c) {
    const double t2 = t * t, w = t2 * t2;
    double e1 = fma(w, 2.8117551578451845e-15, 1.6059043678126643e-10);
    e1 = fma(w, e1, 2.7557319224020396e-06);
    e1 = fma(w, e1, 0.008333333333333331);
    e1 = fma(w, e1, 1.0);
    double o1 = fma(w, 7.648164687578687e-13, 2.5052108004573786e-08);
    o1 = fma(w, o1, 0.00019841269841316215);
    o1 = fma(w, o1, 0.16666666666666657);
    double e0 = fma(w, 4.780102929736679e-14, 2.0876756654608657e-09);
    e0 = fma(w, e0, 2.4801587301659764e-05);
    e0 = fma(w, e0, 0.04166666666666661);
    e0 = fma(w, e0, 1.0);
    double o0 = fma(w, 1.1472647413671577e-11, 2.755731850033682e-07);
    o0 = fma(w, o0, 0.0013888888888977);
    o0 = fma(w, o0, 0.49999999999999833);
    const double t3 = t * t2, te1 = t * e1;
    sh = fma(t3, o1, te1);
    s = fma(-t3, o1, te1);
    ch = fma(t2, o0, e0);
    c = fma(-t2, o0, e0);
}

// Ordered bits of a non-negative double, so that atomicMax on the integers is max on the values.
__device__ __forceinline__ unsigned long long ordered_bits(double nonnegative) {
    return static_cast<unsigned long long>(__double_as_longlong(nonnegative));
}

} // namespace pvb
