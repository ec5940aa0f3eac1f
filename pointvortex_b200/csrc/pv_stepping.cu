// pv_stepping.cu — the Runge–Kutta stage work between two velocity evaluations, on the GPU.
//
// Replaces RungeKuttaIntegrator::makeStage / rk4Step / dopri5Step (src/timestep.cpp:19-120)
// and the reference CUDA backend's stage, combine, validation and error kernels with their
// host round trips (src/backend_cuda.cu:115-200, 299-357, 387-450). One kernel per stage:
//
//   1. reduce the evaluation's chunk partials into k_s in fixed chunk order; a target whose sum is
//      non-finite is recomputed in the reference form (IEEE divisions, the reference's singular
//      test), which either yields the reference's finite value or its error;
//   2. per mode: the next stage position y0 + dt * sum_j a_j k_j, or the RK4 combination, or the
//      DOPRI5 scaled error (max-reduced with one atomicMax per block), each validated like the
//      reference (finite positions; in a disk, inside the wall);
//   3. DOPRI5: the last block to finish runs the step-size control of src/timestep.cpp:97-118 on
//      the device (accept/reject, suggested step, rejection cap), so the state never leaves the GPU
//      between attempts.
//
// All combination arithmetic uses explicitly rounded operations (__dmul_rn/__dadd_rn/__ddiv_rn)
// in the reference's order, so that given the same stage velocities the new state is bit-identical
// to the reference's (which x86-64 g++ computes without FMA contraction).
#include "pv_internal.h"

#include <algorithm>
#include <type_traits>

namespace pvb {

namespace {
__device__ __forceinline__ double max_ref(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double min_ref(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double clamp_ref(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

// Validation of a new position, src/vortex.h:7-14 and src/compute.cpp:41-48.
__device__ __forceinline__ void validate_position(const StageArgs &a, double x, double y) {
    if (!isfinite(x) || !isfinite(y))
        set_status(&a.ctl->status, ST_NONFINITE_POSITION);
    else if (a.g.geometry == GEO_DISK &&
             __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)) >= a.g.radius2)
        set_status(&a.ctl->status, ST_OUTSIDE_DISK);
}

// DOPRI5 step-size control, src/timestep.cpp:95-118, run by one thread.
__device__ void dopri_control(DeviceControl *ctl) {
    const double error = __longlong_as_double(static_cast<long long>(ctl->err_bits));
    const double dt = ctl->dt;
    const double factor = error == 0.0 ? 5.0 : clamp_ref(0.9 * pow(error, -0.2), 0.2, 5.0);
    const double suggested =
        clamp_ref(__dmul_rn(dt, factor), ctl->minimum_time_step, ctl->maximum_time_step);
    if (ctl->status == 0) {
        if (error <= 1.0) {
            ctl->accepted = 1;
            ctl->result[0] = dt;
            ctl->result[1] = suggested;
            ctl->result[2] = error;
            ctl->result[3] = static_cast<double>(ctl->rejected);
        } else {
            ctl->accepted = 0;
            if (dt <= ctl->minimum_time_step || ++ctl->rejected > 32u)
                set_status(&ctl->status, ST_DOPRI_FAILED);
            else
                ctl->dt = max_ref(ctl->minimum_time_step, min_ref(suggested, __dmul_rn(dt, 0.9)));
        }
    }
    ctl->err_bits = 0ull;
    ctl->blocks_done = 0u;
    ctl->dipole_count = 0ull;  // the attempt's gated dipole scan counts from here
}
} // namespace

// What a target's finish reads besides its own velocity: the step-start position, the earlier
// stage velocities k_j (j != s) that its combination uses, and for the DOPRI5 error the
// fifth-order point. All of them were written by kernels that completed before this stage kernel
// was launched (the earlier stage kernels; the velocity launch it waits for writes only partial
// rows), so the stage kernel may load them before its wait on the velocity launch.
struct FinishInputs {
    double x0, y0, xt, yt;
    double kx[7], ky[7];
};

template <int MODE>
__device__ __forceinline__ void load_finish_inputs(const StageArgs &a, size_t i, FinishInputs &p) {
    p.x0 = a.x0[i];
    p.y0 = a.y0[i];
    if (MODE == STAGE_DOPRI_ERROR) {
        p.xt = a.xt[i];
        p.yt = a.yt[i];
    }
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        bool used = false;
        if (MODE == STAGE_POSITION)
            used = j < a.ncoef && a.coef[j] != 0.0;
        else if (MODE == STAGE_DOPRI_ERROR)
            used = a.w[j] != 0.0;
        else if (MODE == STAGE_RK4_COMBINE)
            used = j < 3;
        if (used && j != a.s) {
            p.kx[j] = a.kx[j][i];
            p.ky[j] = a.ky[j][i];
        }
    }
}

// Everything a stage does for one target once its velocity (ku, kv) is summed: the slow path of
// a non-finite sum, the stage velocity, and the stage position / RK4 combination / DOPRI5 error.
// ex, ey: the positions the slow path recomputes from (a.ex, a.ey, or a copy of them). p: the
// target's FinishInputs.
template <int MODE>
__device__ __forceinline__ void finish_target(const StageArgs &a, size_t i, double ku, double kv,
                                              double dt, double &local_max, const double *ex,
                                              const double *ey, const FinishInputs &p) {
    if (a.reduce) {
        if (!isfinite(ku) || !isfinite(kv)) {
            const int verdict =
                slow_target(a.g, ex, ey, a.gamma, a.n_src, a.t_offset + i, ku, kv);
            if (verdict == ST_COINCIDENT || (verdict && !a.nonfinite_ok))
                set_status(&a.ctl->status, verdict);
        }
        a.kx[a.s][i] = ku;
        a.ky[a.s][i] = kv;
    }
    if (MODE == STAGE_POSITION) {
        // makeStage, src/timestep.cpp:19-30 (zero coefficients add an exact zero: skipped)
        double dx = 0.0, dy = 0.0;
#pragma unroll
        for (int j = 0; j < 7; ++j) {  // unrolled: p's fields stay in registers
            const double c = a.coef[j];
            if (j >= a.ncoef || c == 0.0)
                continue;
            const double kxj = j == a.s ? ku : p.kx[j];
            const double kyj = j == a.s ? kv : p.ky[j];
            dx = __dadd_rn(dx, __dmul_rn(c, kxj));
            dy = __dadd_rn(dy, __dmul_rn(c, kyj));
        }
        const double nx = __dadd_rn(p.x0, __dmul_rn(dt, dx));
        const double ny = __dadd_rn(p.y0, __dmul_rn(dt, dy));
        a.xt[i] = nx;
        a.yt[i] = ny;
        validate_position(a, nx, ny);
    } else if (MODE == STAGE_RK4_COMBINE) {
        // src/timestep.cpp:52-57: x0 + dt * (k1 + 2 k2 + 2 k3 + k4) / 6
        const double sx = __dadd_rn(__dadd_rn(__dadd_rn(p.kx[0], __dmul_rn(2.0, p.kx[1])),
                                              __dmul_rn(2.0, p.kx[2])),
                                    ku);
        const double sy = __dadd_rn(__dadd_rn(__dadd_rn(p.ky[0], __dmul_rn(2.0, p.ky[1])),
                                              __dmul_rn(2.0, p.ky[2])),
                                    kv);
        const double nx = __dadd_rn(p.x0, __ddiv_rn(__dmul_rn(dt, sx), 6.0));
        const double ny = __dadd_rn(p.y0, __ddiv_rn(__dmul_rn(dt, sy), 6.0));
        a.xt[i] = nx;
        a.yt[i] = ny;
        if (!isfinite(nx) || !isfinite(ny))
            set_status(&a.ctl->status, ST_NONFINITE_POSITION);
    } else if (MODE == STAGE_DOPRI_ERROR) {
        // src/timestep.cpp:78-95: xt holds the fifth-order point y5 (stage 7's position).
        double xe = 0.0, ye = 0.0;
#pragma unroll
        for (int j = 0; j < 7; ++j) {
            const double w = a.w[j];
            if (w == 0.0)
                continue;
            const double h = __dmul_rn(dt, w);
            const double kxj = j == a.s ? ku : p.kx[j];
            const double kyj = j == a.s ? kv : p.ky[j];
            xe = __dadd_rn(xe, __dmul_rn(h, kxj));
            ye = __dadd_rn(ye, __dmul_rn(h, kyj));
        }
        const double x5 = p.xt, y5 = p.yt;
        const double xs = __dadd_rn(a.ctl->absolute_tolerance,
                                    __dmul_rn(a.ctl->relative_tolerance,
                                              max_ref(fabs(p.x0), fabs(x5))));
        const double ys = __dadd_rn(a.ctl->absolute_tolerance,
                                    __dmul_rn(a.ctl->relative_tolerance,
                                              max_ref(fabs(p.y0), fabs(y5))));
        if (!isfinite(xe) || !isfinite(ye) || !isfinite(xs) || !isfinite(ys) || !(xs > 0.0) ||
            !(ys > 0.0)) {
            set_status(&a.ctl->status, ST_DOPRI_NONFINITE);
        } else {
            local_max = max_ref(local_max, __ddiv_rn(fabs(xe), xs));
            local_max = max_ref(local_max, __ddiv_rn(fabs(ye), ys));
        }
    }
}

// The near-field terms of the block's kWideTargets targets, fused into the wide stage (the work of
// pv_near.cu's near_field_kernel): the kWideGroups threads of a target share its listed entries
// (at most f32::kNearSlots), each computes its entries' FP64 terms (the plain kernels' pair
// functions) and their rank in (source, image) order, and the target's first thread adds them in
// that order, so the sum does not depend on the order of the listing. A target with more
// entries than slots is evaluated whole in FP64 instead (the threads striding over the sources,
// their sums added in thread order), replacing its partial rows. Every count is reset.
// Returns, for the calling first thread (group 0) of target `lane`, the near sum (nu, nv) and
// whether it replaces the rows.
struct NearScratch {
    unsigned key[16][f32::kNearSlots];
    double tu[16][f32::kNearSlots], tv[16][f32::kNearSlots];
};

__device__ __forceinline__ bool fused_near(const NearPass &np, size_t i, bool valid, int lane,
                                           int group, int groups, NearScratch &sc, double &nu,
                                           double &nv) {
    const size_t gi = np.t_begin + i;
    // every thread of the target reads its count (the first one resets it after the barrier
    // below, once all have read it)
    const unsigned count = valid ? np.lists.count[gi] : 0u;
    bool whole = false;
    nu = nv = 0.0;
    const double tx = valid && count ? np.x[gi] : 0.0, ty = valid && count ? np.y[gi] : 0.0;
    if (count > static_cast<unsigned>(f32::kNearSlots)) {
        // overflow: the whole target in FP64
        double su = 0.0, sv = 0.0;
        for (size_t j = group; j < np.n; j += groups) {
            if (np.g.geometry == GEO_PERIODIC)
                PeriodicPair::pair<true>(np.g, tx, ty, np.x[j], np.y[j], np.gs[j], j == gi, su,
                                         sv);
            else
                DiskPair::pair<true>(np.g, tx, ty, np.x[j], np.y[j], np.gs[j], j == gi, su, sv);
        }
        sc.tu[lane][group] = su;
        sc.tv[lane][group] = sv;
        whole = true;
    } else if (count) {
        for (int e = group; e < static_cast<int>(count); e += groups) {
            const unsigned v = np.lists.slot[gi * f32::kNearSlots + e];
            sc.key[lane][e] = (v & ~f32::kNearImage) * 2u + (v >> 31);
        }
    }
    __syncthreads();
    if (group == 0 && count)
        np.lists.count[gi] = 0u;
    if (!whole && count) {
        for (int e = group; e < static_cast<int>(count); e += groups) {
            const unsigned key = sc.key[lane][e];
            int rank = 0;
            for (int k = 0; k < static_cast<int>(count); ++k)
                rank += sc.key[lane][k] < key ? 1 : 0;
            double du = 0.0, dv = 0.0;
            const size_t j = key >> 1;
            if (key & 1u)
                DiskPair::image(np.g, tx, ty, np.x[j], np.y[j], np.gs[j], du, dv);
            else if (np.g.geometry == GEO_PERIODIC)
                PeriodicPair::pair<false>(np.g, tx, ty, np.x[j], np.y[j], np.gs[j], false, du, dv);
            else
                DiskPair::direct(tx, ty, np.x[j], np.y[j], np.gs[j], du, dv);
            sc.tu[lane][rank] = du;
            sc.tv[lane][rank] = dv;
        }
    }
    __syncthreads();
    if (group == 0 && count) {
        const int terms = whole ? groups : static_cast<int>(count);
        for (int r = 0; r < terms; ++r) {
            nu += sc.tu[lane][r];
            nv += sc.tv[lane][r];
        }
    }
    return whole;
}

// WIDE: many partial rows (the symmetric kernel's). A block then covers kWideTargets targets with
// 256 / kWideTargets row groups: thread (group, t) sums rows group, group + groups, ...
// (coalesced over the targets), and the threads of group 0 add the group sums in fixed order.
// Otherwise one thread per target sums its rows in order.
constexpr int kWideTargets = 16;
constexpr int kWideGroups = 256 / kWideTargets;

template <int MODE, bool WIDE, bool NEAR = false>
__global__ void __launch_bounds__(256) stage_kernel(const StageArgs a) {
    __shared__ int s_status;
    __shared__ double s_max[8];
    __shared__ double s_u[WIDE ? kWideGroups : 1][kWideTargets],
        s_v[WIDE ? kWideGroups : 1][kWideTargets];
    __shared__ typename std::conditional<NEAR, NearScratch, char>::type s_near;
    const int tid = threadIdx.x;
    // WIDE: the finishing threads load their first target's FinishInputs before the wait
    FinishInputs early;
    const size_t first = static_cast<size_t>(blockIdx.x) * kWideTargets + tid % kWideTargets;
    if (WIDE && tid < kWideTargets && first < a.n && MODE != STAGE_REDUCE_ONLY)
        load_finish_inputs<MODE>(a, first, early);
    pdl_enter();
    if (tid == 0)
        s_status = *reinterpret_cast<volatile int *>(&a.ctl->status);
    __syncthreads();
    if (s_status != 0) {
        if (NEAR)  // the next evaluation starts from empty lists
            for (size_t i = static_cast<size_t>(blockIdx.x) * kWideTargets + tid; i < a.n;
                 i += static_cast<size_t>(gridDim.x) * kWideTargets)
                if (tid < kWideTargets)
                    a.near.lists.count[a.near.t_begin + i] = 0u;
        return;
    }

    const double dt = a.dt_from_control ? a.ctl->dt : a.dt;
    double local_max = 0.0;
    if (WIDE) {
        const int lane = tid % kWideTargets, group = tid / kWideTargets;
        for (size_t base = static_cast<size_t>(blockIdx.x) * kWideTargets; base < a.n;
             base += static_cast<size_t>(gridDim.x) * kWideTargets) {
            const size_t i = base + lane;
            double su = 0.0, sv = 0.0;
            if (i < a.n && a.pr) {
                // interleaved rows: one 16-byte load per row, eight rows in flight per thread
                // before they are added (in row order, so the sum does not depend on timing)
                const double2 *col = a.pr + i;
                const size_t step = static_cast<size_t>(kWideGroups) * a.stride;
                int c = group;
                for (; c + 7 * kWideGroups < a.num_chunks; c += 8 * kWideGroups) {
                    double2 r[8];
                    const double2 *p = col + static_cast<size_t>(c) * a.stride;
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        r[q] = __ldcg(p + q * step);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        su += r[q].x;
                        sv += r[q].y;
                    }
                }
                for (; c < a.num_chunks; c += kWideGroups) {
                    const double2 r = __ldcg(col + static_cast<size_t>(c) * a.stride);
                    su += r.x;
                    sv += r.y;
                }
            } else if (i < a.n) {
                for (int c = group; c < a.num_chunks; c += kWideGroups) {
                    su += a.pu[static_cast<size_t>(c) * a.stride + i];
                    sv += a.pv[static_cast<size_t>(c) * a.stride + i];
                }
            }
            s_u[group][lane] = su;
            s_v[group][lane] = sv;
            double nu = 0.0, nv = 0.0;
            bool whole = false;
            if constexpr (NEAR)  // its barriers also order the row sums above
                whole = fused_near(a.near, i, i < a.n, lane, group, kWideGroups, s_near, nu, nv);
            __syncthreads();
            if (group == 0 && i < a.n) {
                double ku = s_u[0][lane], kv = s_v[0][lane];
                for (int g = 1; g < kWideGroups; ++g) {
                    ku += s_u[g][lane];
                    kv += s_v[g][lane];
                }
                if (NEAR) {  // the near terms after the rows, or instead of them
                    ku = whole ? nu : ku + nu;
                    kv = whole ? nv : kv + nv;
                }
                if (i != first && MODE != STAGE_REDUCE_ONLY)
                    load_finish_inputs<MODE>(a, i, early);
                finish_target<MODE>(a, i, ku, kv, dt, local_max, a.ex, a.ey, early);
            }
            __syncthreads();
        }
    } else {
        for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + tid; i < a.n;
             i += static_cast<size_t>(gridDim.x) * blockDim.x) {
            double ku, kv;
            if (a.reduce) {
                ku = 0.0;
                kv = 0.0;
                for (int c = 0; c < a.num_chunks; ++c) {
                    if (a.pr) {
                        const double2 r = a.pr[static_cast<size_t>(c) * a.stride + i];
                        ku += r.x;
                        kv += r.y;
                    } else {
                        ku += a.pu[static_cast<size_t>(c) * a.stride + i];
                        kv += a.pv[static_cast<size_t>(c) * a.stride + i];
                    }
                }
            } else {
                ku = a.kx[a.s][i];
                kv = a.ky[a.s][i];
            }
            FinishInputs in;
            if (MODE != STAGE_REDUCE_ONLY)
                load_finish_inputs<MODE>(a, i, in);
            finish_target<MODE>(a, i, ku, kv, dt, local_max, a.ex, a.ey, in);
        }
    }

    if (MODE == STAGE_DOPRI_ERROR) {
        // Block max (max is exact, so the order of the reduction cannot change the result).
        for (int off = 16; off > 0; off >>= 1)
            local_max = max_ref(local_max, __shfl_xor_sync(0xffffffffu, local_max, off));
        if ((tid & 31) == 0)
            s_max[tid >> 5] = local_max;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w)
                m = max_ref(m, s_max[w]);
            atomicMax(&a.ctl->err_bits, ordered_bits(m));
            __threadfence();
            const unsigned done = atomicAdd(&a.ctl->blocks_done, 1u);
            if (done == gridDim.x - 1) {
                __threadfence();
                dopri_control(a.ctl);
            }
        }
    }
}

__global__ void __launch_bounds__(256)
    accept_kernel(double *x, double *y, const double *xt, const double *yt, double *k0x,
                  double *k0y, const double *k6x, const double *k6y, size_t n, int dopri,
                  const DeviceControl *ctl) {
    pdl_enter();
    if (ctl->status != 0 || (dopri && !ctl->accepted))
        return;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        x[i] = xt[i];
        y[i] = yt[i];
        if (dopri) { // FSAL: k7 of the accepted step is k1 of the next (src/timestep.cpp:104-108)
            k0x[i] = k6x[i];
            k0y[i] = k6y[i];
        }
    }
}

namespace {
unsigned grid_for(size_t n, int sm_count) {
    const size_t blocks = (n + 255) / 256;
    const size_t cap = static_cast<size_t>(sm_count > 0 ? sm_count : 148) * 8;
    return static_cast<unsigned>(blocks < 1 ? 1 : (blocks < cap ? blocks : cap));
}
} // namespace

// Partial rows from which a block of 32 targets x 8 row groups beats one thread per target.
constexpr int kWideRows = 32;

template <int MODE>
cudaError_t launch_stage_mode(const StageArgs &a, cudaStream_t stream, int sm_count) {
    const bool near = a.near.lists.count != nullptr;
    if (near && !a.reduce)
        return cudaErrorInvalidValue;
    // the near-field terms need the wide layout (a target's threads share its list), whatever
    // the number of rows
    if (a.reduce && (a.num_chunks >= kWideRows || near)) {
        const size_t blocks = (a.n + kWideTargets - 1) / kWideTargets;
        const size_t cap = static_cast<size_t>(sm_count > 0 ? sm_count : 148) * 8;
        const unsigned grid = static_cast<unsigned>(blocks < 1 ? 1 : (blocks < cap ? blocks : cap));
        if (near)
            return launch_pdl(stage_kernel<MODE, true, true>, dim3(grid), dim3(256), 0, stream, a);
        return launch_pdl(stage_kernel<MODE, true>, dim3(grid), dim3(256), 0, stream, a);
    }
    return launch_pdl(stage_kernel<MODE, false>, dim3(grid_for(a.n, sm_count)), dim3(256), 0,
                      stream, a);
}

cudaError_t launch_stage(const StageArgs &a, cudaStream_t stream, int sm_count) {
    switch (a.mode) {
    case STAGE_REDUCE_ONLY:
        return launch_stage_mode<STAGE_REDUCE_ONLY>(a, stream, sm_count);
    case STAGE_POSITION:
        return launch_stage_mode<STAGE_POSITION>(a, stream, sm_count);
    case STAGE_RK4_COMBINE:
        return launch_stage_mode<STAGE_RK4_COMBINE>(a, stream, sm_count);
    case STAGE_DOPRI_ERROR:
        return launch_stage_mode<STAGE_DOPRI_ERROR>(a, stream, sm_count);
    default:
        return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------------------------
// RK4 steps of a small population in one cooperative launch. Below N ~ 2000 a step's nine
// launches take longer to schedule than to run, so one CTA per SM keeps the whole step loop: each
// CTA owns a range of targets, and a grid barrier separates the four evaluations of a step.
//
// The results are bit for bit those of the launch sequence (enqueue_rk4): a target's velocity is
// summed chunk by chunk (the ordered kernel's chunks, sources in index order, pair<true> with the
// self flag) and the chunk sums are added in chunk order from 0.0, as the stage kernel does with
// fewer than kWideRows chunks; finish_target then runs unchanged. The previous step's combined
// state (stage 3's output) is the next step's evaluation point and is copied into the state target
// by target in the phase that reads it, so a step costs four barriers.

// Grid barrier over the CTAs of a cooperative launch. The arrival counter starts at zero (the
// host clears it before the launch) and only grows: the r-th barrier is open once it reaches
// r * gridDim.x. One fence and one atomic per CTA, then polling with an acquire load.
//
// A wait that outlasts `limit` polls breaks the barrier instead of walking away from it: a
// compare-and-swap sets kBarrierBroken in the counter, and succeeds only if the counter has not
// moved since it was read. Every CTA therefore agrees on each barrier: either it opened (the last
// arrival came before the swap) and all pass it, or it is broken and none does -- later arrivals
// and pollers see the flag and return. The breaker sets ST_TIMEOUT. Since the state is written
// only in phases that follow an open barrier, a timeout leaves it at the last completed step.
constexpr unsigned long long kBarrierBroken = 1ull << 62;
__device__ bool grid_barrier(unsigned long long *arrivals, unsigned long long open_at,
                             int *status, uint32_t limit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();  // this CTA's writes, ordered by the __syncthreads, before its arrival
        unsigned long long now = atomicAdd(arrivals, 1ull) + 1ull;
        ok = 1;
        uint32_t it = 0;
        for (;;) {
            if (now & kBarrierBroken) {
                ok = 0;
                break;
            }
            if (now >= open_at)
                break;
            if (it >= limit) {
                const unsigned long long seen = atomicCAS(arrivals, now, now | kBarrierBroken);
                if (seen == now) {
                    set_status(status, ST_TIMEOUT);
                    ok = 0;
                    break;
                }
                now = seen;  // another CTA arrived (or broke it) meanwhile: look again
                continue;
            }
            ++it;
            if (it > 64)
                __nanosleep(32);
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(now) : "l"(arrivals) : "memory");
        }
        __threadfence();  // the other CTAs' writes before their arrivals are visible from here
    }
    __syncthreads();
    return ok != 0;
}

template <class Pair>
__global__ void __launch_bounds__(256) rk4_steps_kernel(const Rk4Steps p) {
    extern __shared__ double smem[];
    const size_t n = p.n;
    const int nc = p.num_chunks;
    const size_t per_cta = (n + gridDim.x - 1) / gridDim.x;
    const size_t t0 = static_cast<size_t>(blockIdx.x) * per_cta;
    const size_t t1 = t0 < n ? min(t0 + per_cta, n) : t0;
    const int mine = static_cast<int>(t1 - t0);
    double *sx = smem, *sy = smem + n, *sg = smem + 2 * n;
    double *qu = smem + 3 * n, *qv = qu + per_cta * nc;
    int *status = &p.stage[0].ctl->status;
    for (size_t j = threadIdx.x; j < n; j += blockDim.x)
        sg[j] = p.gs[j];
    double local_max = 0.0;
    unsigned long long open_at = 0;
    for (uint64_t step = 0; step < p.steps; ++step) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const StageArgs &a = p.stage[s];
            // evaluation point: the state, or for a step's first stage after the first step the
            // previous step's combination (not yet copied into the state)
            const bool carried = s == 0 && step > 0;
            const double *px = carried ? p.stage[3].xt : a.ex;
            const double *py = carried ? p.stage[3].yt : a.ey;
#pragma unroll 8  // the loads of several iterations in flight at once
            for (size_t j = threadIdx.x; j < n; j += blockDim.x) {
                sx[j] = __ldcg(px + j);
                sy[j] = __ldcg(py + j);
            }
            __syncthreads();
            for (int w = threadIdx.x; w < mine * nc; w += blockDim.x) {
                const int li = w % mine, c = w / mine;
                const size_t i = t0 + li;
                const size_t j0 = static_cast<size_t>(c) * p.chunk;
                const size_t j1 = min(j0 + static_cast<size_t>(p.chunk), n);
                const double tx = sx[i], ty = sy[i];
                double u = 0.0, v = 0.0;
                // unrolled so that the independent work of several sources overlaps; the sums
                // still take the sources in index order
#pragma unroll 4
                for (size_t j = j0; j < j1; ++j)
                    Pair::template pair<true>(a.g, tx, ty, sx[j], sy[j], sg[j], i == j, u, v);
                qu[li * nc + c] = u;
                qv[li * nc + c] = v;
            }
            __syncthreads();
            for (int li = threadIdx.x; li < mine; li += blockDim.x) {
                const size_t i = t0 + li;
                if (carried) {  // the accept of the previous step
                    p.x[i] = px[i];
                    p.y[i] = py[i];
                }
                double ku = 0.0, kv = 0.0;
                for (int c = 0; c < nc; ++c) {
                    ku += qu[li * nc + c];
                    kv += qv[li * nc + c];
                }
                // the slow path recomputes from this phase's positions, held in shared memory
                FinishInputs in;
                if (s < 3) {
                    load_finish_inputs<STAGE_POSITION>(a, i, in);
                    finish_target<STAGE_POSITION>(a, i, ku, kv, a.dt, local_max, sx, sy, in);
                } else {
                    load_finish_inputs<STAGE_RK4_COMBINE>(a, i, in);
                    finish_target<STAGE_RK4_COMBINE>(a, i, ku, kv, a.dt, local_max, sx, sy, in);
                }
            }
            open_at += gridDim.x;
            if (!grid_barrier(p.barrier, open_at, status, p.spin_limit))
                return;
            // every CTA reads the same word after an open barrier: errors are set before arrival
            if (*reinterpret_cast<volatile int *>(status) != 0)
                return;
        }
    }
    for (int li = threadIdx.x; li < mine; li += blockDim.x) {  // the last step's accept
        const size_t i = t0 + li;
        p.x[i] = __ldcg(p.stage[3].xt + i);
        p.y[i] = __ldcg(p.stage[3].yt + i);
    }
}

size_t rk4_steps_smem(size_t n, int num_chunks, int grid) {
    const size_t per_cta = (n + grid - 1) / grid;
    return (3 * n + 2 * per_cta * static_cast<size_t>(num_chunks)) * sizeof(double);
}

bool rk4_steps_eligible(size_t n, int num_chunks) {
    return n >= 1 && n <= kRk4StepsMaxN && num_chunks >= 1 && num_chunks < kWideRows;
}

template <class Pair>
cudaError_t launch_rk4_steps_t(const Rk4Steps &p, int grid, cudaStream_t stream) {
    const size_t smem = rk4_steps_smem(p.n, p.num_chunks, grid);
    cudaError_t e = cudaFuncSetAttribute(rk4_steps_kernel<Pair>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // every CTA resident, or no launch at all
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, rk4_steps_kernel<Pair>, p);
}

cudaError_t launch_rk4_steps(const Rk4Steps &p, int sm_count, cudaStream_t stream) {
    if (!rk4_steps_eligible(p.n, p.num_chunks) || p.steps == 0 || !p.barrier)
        return cudaErrorInvalidValue;
    const int grid = static_cast<int>(
        std::min<size_t>(static_cast<size_t>(sm_count > 0 ? sm_count : 148), p.n));
    switch (p.stage[0].g.geometry) {
    case GEO_INFINITE:
        return launch_rk4_steps_t<InfinitePair>(p, grid, stream);
    case GEO_PERIODIC:
        return launch_rk4_steps_t<PeriodicPair>(p, grid, stream);
    case GEO_DISK:
        return launch_rk4_steps_t<DiskPair>(p, grid, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

cudaError_t launch_accept(double *x, double *y, const double *xt, const double *yt, double *k0x,
                          double *k0y, const double *k6x, const double *k6y, size_t n, int dopri,
                          DeviceControl *ctl, cudaStream_t stream) {
    return launch_pdl(accept_kernel, dim3(grid_for(n, 0)), dim3(256), 0, stream, x, y, xt, yt, k0x,
                      k0y, k6x, k6y, n, dopri, ctl);
}

} // namespace pvb
