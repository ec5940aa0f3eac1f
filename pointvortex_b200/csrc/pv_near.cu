// pv_near.cu — the FP64 near-field pass of the FP32-compensated form.
//
// The FP32 kernels (pv_velocity32.cu, pv_symmetric.cu) leave out of their sums the pairs whose
// terms are large -- periodic pairs closer than the near-field radius at their minimum image, disk
// pairs closer than it, and disk wall images closer than it to their target -- and list them per
// target (pv_pair32.cuh).
// This pass, one thread per target, evaluates the listed terms with the FP64 pair functions of the
// plain kernels (pv_geometry.cuh: the reference's truncated Weiss-McWilliams series,
// src/compute.cpp:203-256, and its disk image term, src/compute.cpp:314-333), in increasing source
// order, and adds their sum to the target's entry of the evaluation's last partial row, which the
// stage kernel then reduces with the others in fixed order: results stay deterministic.
//
// A target with more listed pairs than its slots hold is evaluated whole in FP64 instead (every
// source, the same pair functions): its partial rows are replaced by that one sum.
//
// Every target's list count is reset to zero here, also after a failed or timed-out evaluation, so
// the next evaluation starts from empty lists.
#include "pv_internal.h"

#include <cmath>

namespace pvb {

namespace {

__global__ void __launch_bounds__(256) near_field_kernel(const NearPass a) {
    pdl_enter();
    const size_t i = a.t_begin + blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= a.t_end)
        return;
    const unsigned count = a.lists.count[i];
    if (count == 0)
        return;
    a.lists.count[i] = 0u;
    const double tx = a.x[i], ty = a.y[i];
    const size_t local = i - a.t_begin;
    const size_t last = static_cast<size_t>(a.rows - 1) * a.stride + local;
    double du = 0.0, dv = 0.0;
    if (count > static_cast<unsigned>(f32::kNearSlots)) {
        // overflow: the whole target in FP64, in source order; its FP32 rows are dropped
        for (size_t j = 0; j < a.n; ++j) {
            if (a.g.geometry == GEO_PERIODIC)
                PeriodicPair::pair<true>(a.g, tx, ty, a.x[j], a.y[j], a.gs[j], j == i, du, dv);
            else
                DiskPair::pair<true>(a.g, tx, ty, a.x[j], a.y[j], a.gs[j], j == i, du, dv);
        }
        for (int r = 0; r + 1 < a.rows; ++r) {
            const size_t e = static_cast<size_t>(r) * a.stride + local;
            if (a.pr) {
                a.pr[e] = make_double2(0.0, 0.0);
            } else {
                a.pu[e] = 0.0;
                a.pv[e] = 0.0;
            }
        }
        if (a.pr) {
            a.pr[last] = make_double2(du, dv);
        } else {
            a.pu[last] = du;
            a.pv[last] = dv;
        }
        return;
    }
    // the listed sources in increasing order (insertion sort of at most kNearSlots entries; a
    // source's image sorts after the source itself)
    unsigned e[f32::kNearSlots];
    const unsigned *slot = a.lists.slot + i * f32::kNearSlots;
    for (unsigned k = 0; k < count; ++k) {
        const unsigned v = slot[k];
        const unsigned key = (v & ~f32::kNearImage) * 2u + (v >> 31);
        unsigned m = k;
        while (m > 0 && e[m - 1] > key) {
            e[m] = e[m - 1];
            --m;
        }
        e[m] = key;
    }
    for (unsigned k = 0; k < count; ++k) {
        const size_t j = e[k] >> 1;
        if (e[k] & 1u)
            DiskPair::image(a.g, tx, ty, a.x[j], a.y[j], a.gs[j], du, dv);
        else if (a.g.geometry == GEO_PERIODIC)
            PeriodicPair::pair<false>(a.g, tx, ty, a.x[j], a.y[j], a.gs[j], false, du, dv);
        else
            DiskPair::direct(tx, ty, a.x[j], a.y[j], a.gs[j], du, dv);
    }
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

}  // namespace

cudaError_t launch_near_field(const NearPass &a, cudaStream_t stream) {
    if (a.t_end <= a.t_begin || !a.lists.count || a.rows < 1)
        return cudaSuccess;
    const size_t targets = a.t_end - a.t_begin;
    const unsigned grid = static_cast<unsigned>((targets + 255) / 256);
    return launch_pdl(near_field_kernel, dim3(grid), dim3(256), 0, stream, a);
}

double default_near_radius(const GeometryConsts &g, size_t n) {
    if (n < 2)
        return 0.0;
    // about 12 neighbours per vortex at uniform density: twice the mean spacing
    if (g.geometry == GEO_PERIODIC)
        return 2.0 * g.lx / std::sqrt(static_cast<double>(n));
    if (g.geometry == GEO_DISK)
        return 2.0 * g.radius * std::sqrt(kPi / static_cast<double>(n));
    return 0.0;
}

}  // namespace pvb
