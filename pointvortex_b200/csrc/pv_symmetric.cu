// pv_symmetric.cu — the velocity of a whole population evaluated once per unordered pair: the
// periodic box and the infinite plane, each in FP64 and in the FP32-compensated form.
//
// The reference evaluates every ordered pair (src/compute.cpp:203-256 for the box, :88-133 for
// the plane). The Weiss–McWilliams pair term is antisymmetric: exchanging target and source
// negates x^ and y^ exactly (IEEE remainder is odd), and every quantity of PeriodicPair::terms is
// an exactly odd or even function of them, so the source's term is the target's with the other
// circulation and the opposite sign, bit for bit. The plane's (dy, dx) / (r^2 + eps^2) is odd in
// the same way. One evaluation therefore serves both vortices, and the work per velocity
// evaluation halves. Only the order of summation differs from the ordered-pair kernel.
//
// Work decomposition (warp-level, persistent):
//   * vortices form blocks of 32a (a = 1..16 sub-blocks of 32); an item is a block pair (I, J),
//     I <= J, taken by one warp from an atomic queue;
//   * for a sub-block pair each lane holds one target; the 32 sources and their accumulated
//     reactions rotate through the lanes by shuffles, so in 32 steps every (target, source) pair
//     is met once and every source comes back to its home lane;
//   * sub-blocks on the diagonal of a diagonal item are evaluated one-sided (31 rotations, the
//     self pair skipped, as in the reference);
//   * the plane's pair term is cheap next to the five shuffles of a rotation step, so off the
//     diagonal each lane holds 4 or 8 targets against the rotating sources;
//   * partial sums go to rows of a [blocks][N] array of (u, v) pairs (one 16-byte store per entry):
//     vortices of block I receive row J from item (I, J), vortices of block J receive row I, and
//     each (row, vortex) is written exactly once, so the stage kernel's fixed-order sum over rows
//     keeps results deterministic.
#include "pvb200.h"
#include "pv_internal.h"
#include "pv_symmetric.cuh"

#include <algorithm>
#include <atomic>

namespace pvb {

namespace {

constexpr int kThreads = 128;  // 4 independent warps per CTA

// The work queue resets itself at the end of a launch, so no memset precedes the kernel:
// counter[0] hands out items and counter[1] counts the warps that found the queue empty. Every warp
// draws exactly one ticket past the end, and only after that increments counter[1]; the warp that
// brings counter[1] to the grid's warp count is the last to touch either word, and zeroes both.
__device__ __forceinline__ void release_queue(unsigned *counter) {
    if ((threadIdx.x & 31) != 0)
        return;
    const unsigned warps = gridDim.x * (kThreads / 32);
    __threadfence();
    if (atomicAdd(counter + 1, 1u) == warps - 1) {
        atomicExch(counter, 0u);
        atomicExch(counter + 1, 0u);
    }
}

// P: the pair kernel (sym::PeriodicSym, sym::PlaneSym). T: targets per lane in the items off the
// diagonal (a multiple of T sub-blocks per block); diagonal items hold one target per lane.
// MINB: resident CTAs per SM the register allocation must allow (0: the compiler's own choice;
// the periodic kernel is also built for 7 and 8, fewer registers for more warps to hide latency).
template <class P, int T, int MINB = 0>
__global__ void __launch_bounds__(kThreads, MINB)
    symmetric_kernel(const double *__restrict__ x, const double *__restrict__ y,
                     const double *__restrict__ gs, size_t n, int a,
                     const unsigned *__restrict__ items, unsigned n_items, unsigned *counter,
                     double2 *__restrict__ pr, size_t stride, GeometryConsts g) {
    extern __shared__ double2 reaction_smem[];
    pdl_enter();
    const int lane = threadIdx.x & 31;
    double2 *reaction = reaction_smem + (threadIdx.x >> 5) * a * 32;  // this warp's sources
    const size_t block_len = static_cast<size_t>(32) * a;
    for (;;) {
        unsigned item = 0;
        if (lane == 0)
            item = atomicAdd(counter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= n_items)
            break;
        const unsigned packed = items[item];
        const unsigned I = packed >> 16, J = packed & 0xffffu;
        const bool diagonal = I == J;
        for (int jb = 0; jb < a; ++jb)
            reaction[jb * 32 + lane] = make_double2(0.0, 0.0);
        if (T > 1 && !diagonal) {
            for (int ib = 0; ib < a; ib += T) {
                double tx[T], ty[T], tg[T], u[T], v[T];
                bool t_ok[T], all_ok = true;
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    const size_t ti = I * block_len + static_cast<size_t>(ib + t) * 32 + lane;
                    t_ok[t] = ti < n;
                    all_ok = all_ok && t_ok[t];
                    tx[t] = t_ok[t] ? x[ti] : 0.0;
                    ty[t] = t_ok[t] ? y[ti] : 0.0;
                    tg[t] = t_ok[t] ? P::kScale * gs[ti] : 0.0;
                    u[t] = 0.0;
                    v[t] = 0.0;
                }
                for (int jb = 0; jb < a; ++jb) {
                    const size_t sj = J * block_len + static_cast<size_t>(jb) * 32 + lane;
                    const int s_ok = sj < n ? 1 : 0;
                    const double sx = s_ok ? x[sj] : 0.0, sy = s_ok ? y[sj] : 0.0;
                    const double sg = s_ok ? P::kScale * gs[sj] : 0.0;
                    double ru = reaction[jb * 32 + lane].x, rv = reaction[jb * 32 + lane].y;
                    if (__all_sync(0xffffffffu, all_ok && s_ok)) {
                        sym::react_tiles_full<P, T>(g, tx, ty, tg, sx, sy, sg, u, v, ru, rv);
                    } else {
#pragma unroll
                        for (int t = 0; t < T; ++t)
                            sym::react_tile<P>(g, tx[t], ty[t], tg[t], t_ok[t], sx, sy, sg, s_ok,
                                               u[t], v[t], ru, rv);
                    }
                    reaction[jb * 32 + lane] = make_double2(ru, rv);
                }
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    const size_t ti = I * block_len + static_cast<size_t>(ib + t) * 32 + lane;
                    if (t_ok[t]) {
                        pr[J * stride + ti] = make_double2(u[t], v[t]);
                    }
                }
            }
        } else {
            for (int ib = 0; ib < a; ++ib) {
                const size_t ti = I * block_len + static_cast<size_t>(ib) * 32 + lane;
                const bool t_ok = ti < n;
                const double tx = t_ok ? x[ti] : 0.0, ty = t_ok ? y[ti] : 0.0;
                const double tg = t_ok ? P::kScale * gs[ti] : 0.0;
                double u = 0.0, v = 0.0;
                for (int jb = diagonal ? ib : 0; jb < a; ++jb) {
                    const size_t sj = J * block_len + static_cast<size_t>(jb) * 32 + lane;
                    const int s_ok = sj < n ? 1 : 0;
                    const double sx = s_ok ? x[sj] : 0.0, sy = s_ok ? y[sj] : 0.0;
                    const double sg = s_ok ? P::kScale * gs[sj] : 0.0;
                    if (diagonal && jb == ib) {
                        sym::one_sided_tile<P>(g, tx, ty, t_ok, sx, sy, sg, s_ok, true, u, v);
                        continue;
                    }
                    double ru = reaction[jb * 32 + lane].x, rv = reaction[jb * 32 + lane].y;
                    sym::react_tile<P>(g, tx, ty, tg, t_ok, sx, sy, sg, s_ok, u, v, ru, rv);
                    reaction[jb * 32 + lane] = make_double2(ru, rv);
                }
                if (diagonal) {  // reactions from the sub-blocks before this one in the same block
                    const double2 r = reaction[ib * 32 + lane];
                    u += r.x;
                    v += r.y;
                }
                if (t_ok) {
                    pr[J * stride + ti] = make_double2(u, v);
                }
            }
        }
        if (!diagonal) {
            for (int jb = 0; jb < a; ++jb) {
                const size_t sj = J * block_len + static_cast<size_t>(jb) * 32 + lane;
                if (sj < n) {
                    pr[I * stride + sj] = reaction[jb * 32 + lane];
                }
            }
        }
        __syncwarp();
    }
    release_queue(counter);
}

// The FP32-compensated form of the same decomposition: the pair terms on the FP32 pipe from
// double-float coordinates; each tile's FP32 sums (32 sources) are promoted into FP64. The
// sources of a tile sit in this warp's shared buffer and only the FP32 reactions rotate.
// V: the pair kernel (f32::Periodic32, f32::Plane32). T: targets per lane in the items off the
// diagonal, as in symmetric_kernel.
template <class V, int T>
__global__ void __launch_bounds__(kThreads)
    symmetric32_kernel(const double *__restrict__ x, const double *__restrict__ y,
                       const double *__restrict__ gs, size_t n, int a,
                       const unsigned *__restrict__ items, unsigned n_items, unsigned *counter,
                       double2 *__restrict__ pr, size_t stride, GeometryConsts g,
                       f32::NearLists near) {
    extern __shared__ double2 reaction_smem[];
    __shared__ float4 src_f[kThreads];
    __shared__ float src_g[kThreads];
    pdl_enter();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double2 *reaction = reaction_smem + warp * a * 32;
    float4 *sf = src_f + warp * 32;
    float *sgf = src_g + warp * 32;
    const f32::F32Geometry f = f32::make_f32(g);
    const size_t block_len = static_cast<size_t>(32) * a;
    for (;;) {
        unsigned item = 0;
        if (lane == 0)
            item = atomicAdd(counter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= n_items)
            break;
        const unsigned packed = items[item];
        const unsigned I = packed >> 16, J = packed & 0xffffu;
        const bool diagonal = I == J;
        for (int jb = 0; jb < a; ++jb)
            reaction[jb * 32 + lane] = make_double2(0.0, 0.0);
        if (T > 1 && !diagonal) {
            for (int ib = 0; ib < a; ib += T) {
                float4 t[T];
                float tg[T];
                bool t_ok[T], all_ok = true;
                double ud[T], vd[T];
#pragma unroll
                for (int q = 0; q < T; ++q) {
                    const size_t ti = I * block_len + static_cast<size_t>(ib + q) * 32 + lane;
                    t_ok[q] = ti < n;
                    all_ok = all_ok && t_ok[q];
                    t[q] = sym::split32(t_ok[q] ? x[ti] : 0.0, t_ok[q] ? y[ti] : 0.0);
                    tg[q] = t_ok[q] ? static_cast<float>(gs[ti]) : 0.0f;
                    ud[q] = 0.0;
                    vd[q] = 0.0;
                }
                for (int jb = 0; jb < a; ++jb) {
                    const size_t j0 = J * block_len + static_cast<size_t>(jb) * 32;
                    const size_t sj = j0 + lane;
                    const int s_count =
                        j0 < n ? static_cast<int>(min(static_cast<size_t>(32), n - j0)) : 0;
                    __syncwarp();  // the previous tile's reads of the buffer are done
                    sf[lane] = sym::split32(sj < n ? x[sj] : 0.0, sj < n ? y[sj] : 0.0);
                    sgf[lane] = sj < n ? static_cast<float>(gs[sj]) : 0.0f;
                    __syncwarp();
                    float u[T], v[T];
#pragma unroll
                    for (int q = 0; q < T; ++q) {
                        u[q] = 0.0f;
                        v[q] = 0.0f;
                    }
                    double rud = 0.0, rvd = 0.0;
                    if (__all_sync(0xffffffffu, all_ok && s_count == 32)) {
                        sym::react_tiles32_full<V, T>(f, t, tg, sf, sgf, u, v, rud, rvd);
                    } else {
#pragma unroll
                        for (int q = 0; q < T; ++q) {
                            float ru = 0.0f, rv = 0.0f;
                            const size_t tq = I * block_len + static_cast<size_t>(ib + q) * 32 + lane;
                            sym::react_tile32<V>(f, t[q], tg[q], t_ok[q], sf, sgf, s_count, u[q],
                                                 v[q], ru, rv, sym::NearTile{near, tq, j0});
                            rud += static_cast<double>(ru);
                            rvd += static_cast<double>(rv);
                        }
                    }
                    double2 r = reaction[jb * 32 + lane];
                    r.x += rud;
                    r.y += rvd;
                    reaction[jb * 32 + lane] = r;
#pragma unroll
                    for (int q = 0; q < T; ++q) {
                        ud[q] += static_cast<double>(u[q]);
                        vd[q] += static_cast<double>(v[q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < T; ++q) {
                    const size_t ti = I * block_len + static_cast<size_t>(ib + q) * 32 + lane;
                    if (t_ok[q]) {
                        pr[J * stride + ti] = make_double2(ud[q], vd[q]);
                    }
                }
            }
        } else {
            for (int ib = 0; ib < a; ++ib) {
                const size_t t0 = I * block_len + static_cast<size_t>(ib) * 32;
                const size_t ti = t0 + lane;
                const bool t_ok = ti < n;
                const float4 t = sym::split32(t_ok ? x[ti] : 0.0, t_ok ? y[ti] : 0.0);
                const float tg = t_ok ? static_cast<float>(gs[ti]) : 0.0f;
                double ud = 0.0, vd = 0.0;
                for (int jb = diagonal ? ib : 0; jb < a; ++jb) {
                    const size_t j0 = J * block_len + static_cast<size_t>(jb) * 32;
                    const size_t sj = j0 + lane;
                    const int s_count =
                        j0 < n ? static_cast<int>(min(static_cast<size_t>(32), n - j0)) : 0;
                    __syncwarp();  // the previous tile's reads of the buffer are done
                    sf[lane] = sym::split32(sj < n ? x[sj] : 0.0, sj < n ? y[sj] : 0.0);
                    sgf[lane] = sj < n ? static_cast<float>(gs[sj]) : 0.0f;
                    __syncwarp();
                    float u = 0.0f, v = 0.0f;
                    const sym::NearTile nt{near, ti, j0};
                    if (diagonal && jb == ib) {
                        sym::one_sided_tile32<V>(f, t, t_ok, sf, sgf, s_count, true, u, v, nt);
                    } else {
                        float ru = 0.0f, rv = 0.0f;
                        sym::react_tile32<V>(f, t, tg, t_ok, sf, sgf, s_count, u, v, ru, rv, nt);
                        double2 r = reaction[jb * 32 + lane];
                        r.x += static_cast<double>(ru);
                        r.y += static_cast<double>(rv);
                        reaction[jb * 32 + lane] = r;
                    }
                    ud += static_cast<double>(u);
                    vd += static_cast<double>(v);
                }
                if (diagonal) {
                    const double2 r = reaction[ib * 32 + lane];
                    ud += r.x;
                    vd += r.y;
                }
                if (t_ok) {
                    pr[J * stride + ti] = make_double2(ud, vd);
                }
            }
        }
        if (!diagonal) {
            for (int jb = 0; jb < a; ++jb) {
                const size_t sj = J * block_len + static_cast<size_t>(jb) * 32 + lane;
                if (sj < n) {
                    pr[I * stride + sj] = reaction[jb * 32 + lane];
                }
            }
        }
        __syncwarp();
    }
    release_queue(counter);
}

// Targets per lane of the plane's items off the diagonal: 4 below kSymmetricPlaneWideN, 8 from
// there up. Eight divide the shuffles per pair further but hold 168 registers (3 CTAs per SM), and
// their blocks of at least 8 sub-blocks leave too few items to balance below that size.
constexpr int kPlaneTargets = 4;
constexpr int kPlaneTargetsWide = 8;

enum SymKernel : int {
    SYM_PERIODIC = 0,
    SYM_PERIODIC32 = 1,
    SYM_PLANE = 2,
    SYM_PLANE_WIDE = 3,
    SYM_PLANE32 = 4,
    SYM_PLANE32_WIDE = 5,
    SYM_PERIODIC_7 = 6,   // the periodic FP64 kernel built for 7 resident CTAs per SM
    SYM_PERIODIC_8 = 7,   // ... and for 8
    SYM_PERIODIC_T2 = 8,  // the periodic FP64 kernel with two targets per lane off the diagonal
    SYM_KERNELS = 9
};

int kernel_of(const SymmetricPlan &p) {
    const bool fp32c = p.precision == PV_PRECISION_FP32C;
    if (p.geometry == GEO_INFINITE) {
        const bool wide = p.targets == kPlaneTargetsWide;
        return fp32c ? (wide ? SYM_PLANE32_WIDE : SYM_PLANE32) : (wide ? SYM_PLANE_WIDE : SYM_PLANE);
    }
    if (fp32c)
        return SYM_PERIODIC32;
    if (p.targets == 2)
        return SYM_PERIODIC_T2;
    return p.min_ctas == 8 ? SYM_PERIODIC_8 : (p.min_ctas == 7 ? SYM_PERIODIC_7 : SYM_PERIODIC);
}

// Autotuner table of the symmetric form (pv_set_symmetric_tuning), by geometry (0 plane,
// 1 periodic), precision and floor(log2 N): 0 = the built-in plan; otherwise
// mode | (min_ctas << 4) | (targets << 8) with mode 1 = the ordered kernel, 2 = the symmetric form.
std::atomic<int> g_sym_tuning[2][2][40] = {};

template <typename K> int occupancy(K kernel, size_t smem) {
    int blocks = 0;
    const cudaError_t e =
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, kThreads, smem);
    return e == cudaSuccess && blocks >= 1 ? blocks : 1;
}

int resident_ctas(int a, int kernel) {
    static std::atomic<int> cached[SYM_KERNELS][17] = {};  // host threads may ask at once
    if (a < 1 || a > 16 || kernel < 0 || kernel >= SYM_KERNELS)
        return 1;
    if (!cached[kernel][a].load(std::memory_order_relaxed)) {
        const size_t smem = static_cast<size_t>(kThreads / 32) * a * 32 * sizeof(double2);
        int blocks = 1;
        switch (kernel) {
        case SYM_PERIODIC32:
            blocks = occupancy(symmetric32_kernel<f32::Periodic32, 1>, smem);
            break;
        case SYM_PLANE:
            blocks = occupancy(symmetric_kernel<sym::PlaneSym, kPlaneTargets>, smem);
            break;
        case SYM_PLANE_WIDE:
            blocks = occupancy(symmetric_kernel<sym::PlaneSym, kPlaneTargetsWide>, smem);
            break;
        case SYM_PLANE32:
            blocks = occupancy(symmetric32_kernel<f32::Plane32, kPlaneTargets>, smem);
            break;
        case SYM_PLANE32_WIDE:
            blocks = occupancy(symmetric32_kernel<f32::Plane32, kPlaneTargetsWide>, smem);
            break;
        case SYM_PERIODIC_7:
            blocks = occupancy(symmetric_kernel<sym::PeriodicSym, 1, 7>, smem);
            break;
        case SYM_PERIODIC_8:
            blocks = occupancy(symmetric_kernel<sym::PeriodicSym, 1, 8>, smem);
            break;
        case SYM_PERIODIC_T2:
            blocks = occupancy(symmetric_kernel<sym::PeriodicSym, 2>, smem);
            break;
        default:
            blocks = occupancy(symmetric_kernel<sym::PeriodicSym, 1>, smem);
            break;
        }
        cached[kernel][a].store(blocks, std::memory_order_relaxed);
    }
    return cached[kernel][a].load(std::memory_order_relaxed);
}

}  // namespace

int symmetric_tuning_lookup(int geometry, int precision, size_t n) {
    if ((geometry != GEO_INFINITE && geometry != GEO_PERIODIC) || precision < 0 || precision > 1 ||
        n == 0)
        return 0;
    int bucket = 0;
    while ((size_t(2) << bucket) <= n && bucket < 39)
        ++bucket;
    return g_sym_tuning[geometry == GEO_PERIODIC ? 1 : 0][precision][bucket].load(
        std::memory_order_relaxed);
}

// Persistent CTAs per SM of the symmetric form's grid (0: as many as fit). Fewer CTAs than fit
// can be faster: the work queue's last round of items is fuller.
std::atomic<int> g_sym_grid[2][2][40] = {};

int symmetric_grid_lookup(int geometry, int precision, size_t n) {
    if ((geometry != GEO_INFINITE && geometry != GEO_PERIODIC) || precision < 0 || precision > 1 ||
        n == 0)
        return 0;
    int bucket = 0;
    while ((size_t(2) << bucket) <= n && bucket < 39)
        ++bucket;
    return g_sym_grid[geometry == GEO_PERIODIC ? 1 : 0][precision][bucket].load(
        std::memory_order_relaxed);
}

bool symmetric_grid_store(int geometry, int precision, int log2_n, int ctas_per_sm) {
    if ((geometry != GEO_INFINITE && geometry != GEO_PERIODIC) || precision < 0 || precision > 1 ||
        log2_n < 0 || log2_n >= 40 || ctas_per_sm < 0 || ctas_per_sm > 16)
        return false;
    g_sym_grid[geometry == GEO_PERIODIC ? 1 : 0][precision][log2_n].store(
        ctas_per_sm, std::memory_order_relaxed);
    return true;
}

bool symmetric_tuning_store(int geometry, int precision, int log2_n, int mode, int min_ctas,
                            int targets) {
    if ((geometry != GEO_INFINITE && geometry != GEO_PERIODIC) || precision < 0 || precision > 1 ||
        log2_n < 0 || log2_n >= 40 || mode < 0 || mode > 2)
        return false;
    if (min_ctas != 0 && !(geometry == GEO_PERIODIC && precision == PV_PRECISION_FP64 &&
                           (min_ctas == 7 || min_ctas == 8)))
        return false;
    if (targets != 0 && !(geometry == GEO_INFINITE && (targets == kPlaneTargets ||
                                                      targets == kPlaneTargetsWide)) &&
        !(geometry == GEO_PERIODIC && precision == PV_PRECISION_FP64 && targets == 2 &&
          min_ctas == 0))
        return false;
    const int packed = mode == 0 ? 0 : (mode | (min_ctas << 4) | (targets << 8));
    g_sym_tuning[geometry == GEO_PERIODIC ? 1 : 0][precision][log2_n].store(
        packed, std::memory_order_relaxed);
    return true;
}

SymmetricPlan plan_symmetric(size_t n, int sm_count, int precision, int geometry) {
    SymmetricPlan p{};
    const bool plane = geometry == GEO_INFINITE;
    if (!plane && geometry != GEO_PERIODIC)
        return p;
    // the measured table overrides the built-in choice of form, occupancy and targets per lane
    const int tuned = symmetric_tuning_lookup(geometry, precision, n);
    const int mode = tuned & 15, tuned_ctas = (tuned >> 4) & 15, tuned_targets = (tuned >> 8) & 15;
    if (mode == 1)
        return p;
    const size_t min_n = plane ? (precision == PV_PRECISION_FP32C ? kSymmetricPlane32MinN
                                                                  : kSymmetricPlaneMinN)
                               : kSymmetricMinN;
    if (mode != 2 && n < min_n)
        return p;
    if (n < 64)
        return p;
    // the smallest block that keeps the partial rows within kSymmetricPartialBytes, or the largest
    // block up to kSymmetricPartialBytesMax (N ~ 3.7e5); beyond that the ordered kernel runs. The
    // plane's blocks hold at least as many sub-blocks as a lane holds targets.
    // the periodic FP64 kernel: two targets per lane only where the table asks for it
    const int targets =
        plane ? (tuned_targets ? tuned_targets
                               : (n >= kSymmetricPlaneWideN ? kPlaneTargetsWide : kPlaneTargets))
              : (precision == PV_PRECISION_FP64 && tuned_targets == 2 ? 2 : 1);
    p.min_ctas = tuned_ctas;
    const size_t np = (n + 255) & ~static_cast<size_t>(255);
    for (int a = targets; a <= 16; a *= 2) {
        const size_t blocks = (n + 32 * static_cast<size_t>(a) - 1) / (32 * static_cast<size_t>(a));
        if (blocks > 0xffffu)
            continue;
        const size_t bytes = blocks * np * 2 * sizeof(double);
        if (bytes <= kSymmetricPartialBytes || (a == 16 && bytes <= kSymmetricPartialBytesMax)) {
            p.a = a;
            p.min_ctas = tuned_ctas;
            p.blocks = static_cast<int>(blocks);
            p.items = static_cast<unsigned>(blocks * (blocks + 1) / 2);
            p.precision = precision;
            p.geometry = geometry;
            p.targets = targets;
            const int fit = resident_ctas(a, kernel_of(p));
            const int want = symmetric_grid_lookup(geometry, precision, n);
            p.grid_ctas = want > 0 && want < fit ? want : fit;
            p.grid = std::max(sm_count, 1) * p.grid_ctas;
            return p;
        }
    }
    return SymmetricPlan{};
}

void symmetric_items(const SymmetricPlan &p, unsigned *out) {
    // the diagonal items (evaluated one-sided) first, then I < J row by row
    size_t k = 0;
    for (unsigned i = 0; i < static_cast<unsigned>(p.blocks); ++i)
        out[k++] = (i << 16) | i;
    for (unsigned i = 0; i < static_cast<unsigned>(p.blocks); ++i)
        for (unsigned j = i + 1; j < static_cast<unsigned>(p.blocks); ++j)
            out[k++] = (i << 16) | j;
}

cudaError_t launch_symmetric(const double *x, const double *y, const double *gs, size_t n,
                             const SymmetricPlan &p, const unsigned *items, unsigned *counter,
                             double2 *rows, size_t stride, const GeometryConsts &g,
                             const f32::NearLists &near, cudaStream_t stream) {
    const size_t smem = static_cast<size_t>(kThreads / 32) * p.a * 32 * sizeof(double2);
    const dim3 grid(static_cast<unsigned>(p.grid)), block(kThreads);
    switch (kernel_of(p)) {
    case SYM_PERIODIC32:
        return launch_pdl(symmetric32_kernel<f32::Periodic32, 1>, grid, block, smem, stream, x, y,
                          gs, n, p.a, items, p.items, counter, rows, stride, g, near);
    case SYM_PLANE:
        return launch_pdl(symmetric_kernel<sym::PlaneSym, kPlaneTargets>, grid, block, smem,
                          stream, x, y, gs, n, p.a, items, p.items, counter, rows, stride, g);
    case SYM_PLANE_WIDE:
        return launch_pdl(symmetric_kernel<sym::PlaneSym, kPlaneTargetsWide>, grid, block, smem,
                          stream, x, y, gs, n, p.a, items, p.items, counter, rows, stride, g);
    case SYM_PLANE32:
        return launch_pdl(symmetric32_kernel<f32::Plane32, kPlaneTargets>, grid, block, smem,
                          stream, x, y, gs, n, p.a, items, p.items, counter, rows, stride, g,
                          near);
    case SYM_PLANE32_WIDE:
        return launch_pdl(symmetric32_kernel<f32::Plane32, kPlaneTargetsWide>, grid, block, smem,
                          stream, x, y, gs, n, p.a, items, p.items, counter, rows, stride, g,
                          near);
    case SYM_PERIODIC_7:
        return launch_pdl(symmetric_kernel<sym::PeriodicSym, 1, 7>, grid, block, smem, stream, x, y,
                          gs, n, p.a, items, p.items, counter, rows, stride, g);
    case SYM_PERIODIC_8:
        return launch_pdl(symmetric_kernel<sym::PeriodicSym, 1, 8>, grid, block, smem, stream, x, y,
                          gs, n, p.a, items, p.items, counter, rows, stride, g);
    case SYM_PERIODIC_T2:
        return launch_pdl(symmetric_kernel<sym::PeriodicSym, 2>, grid, block, smem, stream, x, y,
                          gs, n, p.a, items, p.items, counter, rows, stride, g);
    default:
        return launch_pdl(symmetric_kernel<sym::PeriodicSym, 1>, grid, block, smem, stream, x, y,
                          gs, n, p.a, items, p.items, counter, rows, stride, g);
    }
}

}  // namespace pvb
