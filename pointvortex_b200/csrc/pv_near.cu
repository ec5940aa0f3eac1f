// pv_near.cu — the FP64 near-field pass of the FP32-compensated form.
//
// The FP32 kernels (pv_velocity32.cu, pv_symmetric.cu) leave out of their sums the pairs whose
// terms are large -- periodic pairs closer than the near-field radius at their minimum image, disk
// pairs closer than it, and disk wall images closer than it to their target -- and list them per
// target (pv_pair32.cuh).
// This pass, one warp per target, evaluates the listed terms with the FP64 pair functions of the
// plain kernels (pv_geometry.cuh: the reference's truncated Weiss-McWilliams series,
// src/compute.cpp:203-256, its direct term and its disk image term, src/compute.cpp:286-336),
// sorted by source, adds them in a fixed tree, and adds that sum to the target's entry of the
// evaluation's last partial row, which the stage kernel then reduces with the others in fixed
// order: results stay deterministic.
//
// A target with more listed pairs than its slots hold is evaluated whole in FP64 instead (every
// source, the same pair functions): its partial rows are replaced by that one sum.
//
// Every target's list count is reset to zero here, also after a failed or timed-out evaluation, so
// the next evaluation starts from empty lists.
//
// The stage kernel that reduces an evaluation's partial rows runs this pass itself
// (StageArgs::near, pv_stepping.cu: the threads of a target share its list, and the sum enters
// after the rows). This kernel runs only for a pass that no stage took over, to reset the lists.
#include "pv_internal.h"

#include <cmath>

namespace pvb {

namespace {

constexpr int kNearWarps = 8;  // targets per CTA: one warp each

// Sum of a warp's values in a fixed tree (lane 0 receives it): the same order on every run.
__device__ __forceinline__ double warp_sum(double v) {
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

// One warp per target. The listed entries (at most 32: one per lane) are sorted across the warp
// (a bitonic network over the lanes), each lane evaluates one in FP64, and the warp adds the terms
// in a fixed tree; so the sum does not depend on the order in which the FP32 kernel listed them.
// Four CTAs per SM (at most 64 registers): a population's targets are then one wave, and each
// warp's chain of dependent loads (list count and slots, the listed sources, the partial row)
// overlaps the others'. The count, the slots and the target are loaded together.
__global__ void __launch_bounds__(kNearWarps * 32, 4) near_field_kernel(const NearPass a) {
    pdl_enter();
    const int lane = threadIdx.x & 31;
    const size_t i = a.t_begin + static_cast<size_t>(blockIdx.x) * kNearWarps + (threadIdx.x >> 5);
    if (i >= a.t_end)
        return;  // the whole warp
    const unsigned count = a.lists.count[i];
    const unsigned listed = a.lists.slot[i * f32::kNearSlots + lane];  // meaningful below count
    const double tx = a.x[i], ty = a.y[i];
    if (count == 0)
        return;
    __syncwarp();
    if (lane == 0)
        a.lists.count[i] = 0u;
    const size_t local = i - a.t_begin;
    const size_t last = static_cast<size_t>(a.rows - 1) * a.stride + local;
    double du = 0.0, dv = 0.0;
    if (count > static_cast<unsigned>(f32::kNearSlots)) {
        // overflow: the whole target in FP64, the lanes striding over the sources; its FP32 rows
        // are dropped
        for (size_t j = lane; j < a.n; j += 32) {
            if (a.g.geometry == GEO_PERIODIC)
                PeriodicPair::pair<true>(a.g, tx, ty, a.x[j], a.y[j], a.gs[j], j == i, du, dv);
            else
                DiskPair::pair<true>(a.g, tx, ty, a.x[j], a.y[j], a.gs[j], j == i, du, dv);
        }
        du = warp_sum(du);
        dv = warp_sum(dv);
        for (int r = lane; r + 1 < a.rows; r += 32) {
            const size_t e = static_cast<size_t>(r) * a.stride + local;
            if (a.pr) {
                a.pr[e] = make_double2(0.0, 0.0);
            } else {
                a.pu[e] = 0.0;
                a.pv[e] = 0.0;
            }
        }
        if (lane == 0) {
            if (a.pr) {
                a.pr[last] = make_double2(du, dv);
            } else {
                a.pu[last] = du;
                a.pv[last] = dv;
            }
        }
        return;
    }
    // the listed entries in increasing (source, image) order across the lanes; a source's image
    // sorts after the source itself, empty lanes last
    unsigned key = 0xffffffffu;
    if (lane < static_cast<int>(count))
        key = (listed & ~f32::kNearImage) * 2u + (listed >> 31);
    for (int k = 2; k <= 32; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned other = __shfl_xor_sync(0xffffffffu, key, j);
            key = (((lane & j) == 0) == ((lane & k) == 0)) ? min(key, other) : max(key, other);
        }
    if (key != 0xffffffffu) {
        const size_t j = key >> 1;
        if (key & 1u)
            DiskPair::image(a.g, tx, ty, a.x[j], a.y[j], a.gs[j], du, dv);
        else if (a.g.geometry == GEO_PERIODIC)
            PeriodicPair::pair<false>(a.g, tx, ty, a.x[j], a.y[j], a.gs[j], false, du, dv);
        else
            DiskPair::direct(tx, ty, a.x[j], a.y[j], a.gs[j], du, dv);
    }
    du = warp_sum(du);
    dv = warp_sum(dv);
    if (lane == 0) {
        if (a.pr) {
            double2 r = a.pr[last];
            r.x += du;
            r.y += dv;
            a.pr[last] = r;
        } else {
            a.pu[last] += du;
            a.pv[last] += dv;
        }
    }
}

}  // namespace

cudaError_t launch_near_field(const NearPass &a, cudaStream_t stream) {
    if (a.t_end <= a.t_begin || !a.lists.count || a.rows < 1)
        return cudaSuccess;
    const size_t targets = a.t_end - a.t_begin;
    const unsigned grid = static_cast<unsigned>((targets + kNearWarps - 1) / kNearWarps);
    return launch_pdl(near_field_kernel, dim3(grid), dim3(kNearWarps * 32), 0, stream, a);
}

double default_near_radius(const GeometryConsts &g, size_t n) {
    if (n < 2)
        return 0.0;
    // periodic box: twice the mean spacing of N uniform vortices, about 12 neighbours per vortex
    // (at one spacing the largest FP32 terms left in the sums raise the maximum error above
    // 2^-20). Disk: one mean spacing. Its wall images are already exact virtual vortices, so
    // only the closest pairs and images matter; at one spacing the maximum error is the same as at
    // two (3.4e-7 against 3.3e-7 on the 16384-vortex workload state) with a quarter of the
    // entries, and targets near the wall, which list both pairs and images, rarely overflow their
    // slots (an overflowing target is evaluated whole in FP64).
    if (g.geometry == GEO_PERIODIC)
        return 2.0 * g.lx / std::sqrt(static_cast<double>(n));
    if (g.geometry == GEO_DISK)
        return g.radius * std::sqrt(kPi / static_cast<double>(n));
    return 0.0;
}

}  // namespace pvb
