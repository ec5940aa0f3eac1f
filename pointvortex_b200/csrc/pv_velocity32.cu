// pv_velocity32.cu — the FP32-compensated precision form of the velocity evaluation.
//
// Same tiling, TMA staging, chunk partials and slow path as pv_velocity.cu; the pair terms are
// evaluated on the FP32 pipe (128 lanes/clk/SM on B200, twice the FP64 pipe) with these
// compensations:
//
//   * coordinates as double-float pairs: every staged source and every target is split into
//     hi = fp32(x), lo = fp32(x - hi), and a displacement is (t_hi - s_hi) + (t_lo - s_lo). The
//     first difference is exact when the coordinates are close (Sterbenz) and carries the relative
//     error of one rounding otherwise, so dx keeps ~2^-24 relative accuracy at every separation,
//     which absolute FP32 coordinates cannot (their rounding is relative to |x|, not |dx|). This
//     is what coordinates relative to a tile centre would buy, without sorting the vortices into
//     compact tiles;
//   * FP32 partial sums over 64 sources are promoted into FP64 accumulators, so the summation error
//     does not grow with N;
//   * the disk's wall image of each source is staged as a position (the vortex -Gamma at
//     R^2 s/|s|^2, computed in FP64 once per CTA and tile), so the image term is a direct term
//     from an accurately known point instead of the cancelling 1 - t.s/R^2 form;
//   * near field: the periodic pairs closer than the near-field radius (minimum image), the disk's
//     direct pairs closer than it and the disk images closer than it to their target are left out
//     of the FP32 sums and listed for the FP64 pass (pv_near.cu), which adds their exact terms.
//
// What remains is the FP32 rounding of each far term (a few ulp, ~1e-7 of the term); the velocity
// error against the FP64 oracle is that, summed over sources (reported by the parity tests).
#include "pv_internal.h"
#include "pv_pair32.cuh"

#include <algorithm>
#include <atomic>

namespace pvb {

namespace {
constexpr int kTile32 = 256;
using namespace f32;

template <int GEO, int B, int T>
__global__ void __launch_bounds__(B) velocity32_kernel(const EvalArgs a) {
    __shared__ alignas(128) double s_x[2][kTile32];
    __shared__ alignas(128) double s_y[2][kTile32];
    __shared__ alignas(128) double s_g[2][kTile32];
    // plane, periodic: s_f = (xh, yh, xl, yl), s_gf. Disk: each source packed with its wall image
    // for the f32x2 pair (disk_pair_x2): s_f = px, s_fi = py, s_g2 = (gf, -gf).
    __shared__ alignas(16) float4 s_f[kTile32];
    __shared__ alignas(16) float4 s_fi[GEO == GEO_DISK ? kTile32 : 1];
    __shared__ float s_gf[GEO == GEO_DISK ? 1 : kTile32];
    __shared__ alignas(8) float2 s_g2[GEO == GEO_DISK ? kTile32 : 1];
    __shared__ alignas(8) uint64_t bars[2];
    __shared__ int s_status;

    pdl_enter();
    const int tid = threadIdx.x;
    if (tid == 0)
        s_status = *reinterpret_cast<volatile int *>(a.status);
    __syncthreads();
    if (s_status != 0)
        return;
    const F32Geometry f = make_f32(a.g);

    const int item = blockIdx.x;
    const int tb = item / a.num_chunks;
    const int chunk = item - tb * a.num_chunks;
    const size_t src0 = static_cast<size_t>(chunk) * a.chunk;
    const size_t src1 = min(src0 + static_cast<size_t>(a.chunk), a.n_src);
    const size_t blk0 = a.t_begin + static_cast<size_t>(tb) * (B * T);
    const size_t blk1 = min(blk0 + static_cast<size_t>(B * T), a.t_end);

    Target32 tg[T];
    float u[T], v[T];
    double ud[T], vd[T];
    size_t ti[T];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        ti[k] = blk0 + static_cast<size_t>(k) * B + tid;
        const bool ok = ti[k] < blk1;
        tg[k].x = ok ? a.tx[ti[k]] : 0.0;
        tg[k].y = ok ? a.ty[ti[k]] : 0.0;
        tg[k].xh = static_cast<float>(tg[k].x);
        tg[k].xl = static_cast<float>(tg[k].x - static_cast<double>(tg[k].xh));
        tg[k].yh = static_cast<float>(tg[k].y);
        tg[k].yl = static_cast<float>(tg[k].y - static_cast<double>(tg[k].yh));
        u[k] = v[k] = 0.0f;
        ud[k] = vd[k] = 0.0;
    }
    DiskTarget2 t2[GEO == GEO_DISK ? T : 1];
    float2 u2[GEO == GEO_DISK ? T : 1], v2[GEO == GEO_DISK ? T : 1];
    if (GEO == GEO_DISK) {
#pragma unroll
        for (int k = 0; k < T; ++k) {
            t2[k] = disk_target2(tg[k]);
            u2[k] = v2[k] = make_float2(0.0f, 0.0f);
        }
    }

    const int ntiles = src1 > src0 ? static_cast<int>((src1 - src0 + kTile32 - 1) / kTile32) : 0;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    auto issue = [&](int t) {
        const int st = t & 1;
        const size_t j0 = src0 + static_cast<size_t>(t) * kTile32;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTile32), src1 - j0));
        const int even = cnt & ~1;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bars[st], static_cast<uint32_t>(3 * even * sizeof(double)));
        if (even) {
            const uint32_t bytes = static_cast<uint32_t>(even * sizeof(double));
            bulk_g2s(s_x[st], a.sx + j0, bytes, &bars[st]);
            bulk_g2s(s_y[st], a.sy + j0, bytes, &bars[st]);
            bulk_g2s(s_g[st], a.sg + j0, bytes, &bars[st]);
        }
        if (cnt & 1) {
            s_x[st][cnt - 1] = a.sx[j0 + cnt - 1];
            s_y[st][cnt - 1] = a.sy[j0 + cnt - 1];
            s_g[st][cnt - 1] = a.sg[j0 + cnt - 1];
        }
    };
    if (tid == 0) {
        if (ntiles > 0)
            issue(0);
        if (ntiles > 1)
            issue(1);
    }
    __syncthreads();

    for (int t = 0; t < ntiles; ++t) {
        const int st = t & 1;
        const bool ok = mbar_wait_bounded(&bars[st], static_cast<uint32_t>((t >> 1) & 1), a.status,
                                          a.wait_limit);
        if (__syncthreads_or(!ok)) {
            if (tid == 0)  // the copies of tiles t and t + 1 may still be in flight
                mbar_drain(bars, static_cast<uint32_t>(t), t + 1 < ntiles);
            return;
        }
        const size_t j0 = src0 + static_cast<size_t>(t) * kTile32;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTile32), src1 - j0));
        // split the tile into double-float FP32 coordinates (and, in the disk, the sources' wall
        // images) once per CTA
        for (int j = tid; j < cnt; j += B) {
            const double xj = s_x[st][j], yj = s_y[st][j];
            if (GEO == GEO_DISK) {
                disk_pack_source(split_position(xj, yj), image_position(a.g, xj, yj),
                                 static_cast<float>(s_g[st][j]), s_f[j], s_fi[j], s_g2[j]);
            } else {
                s_f[j] = split_position(xj, yj);
                s_gf[j] = static_cast<float>(s_g[st][j]);
            }
        }
        __syncthreads();
        const bool diagonal = j0 < blk1 && blk0 < j0 + cnt;
        // near terms are left to the FP64 pass: listed under their target
        for (int jb = 0; jb < cnt; jb += kFlush) {
            const int je = min(cnt, jb + kFlush);
            if (diagonal) {
#pragma unroll 1
                for (int j = jb; j < je; ++j) {
                    float4 sf = s_f[j], si = sf;
                    float gf;
                    if (GEO == GEO_DISK) {
                        disk_unpack_source(sf, s_fi[j], sf, si);
                        gf = s_g2[j].x;
                    } else {
                        gf = s_gf[j];
                    }
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        bool np, nw;
                        if (pair32<GEO, true>(f, tg[k], sf, si, gf, ti[k] == j0 + j, u[k], v[k], np,
                                              nw) &&
                            a.near.count && ti[k] < blk1)
                            list_near(a.near, np, nw, ti[k], static_cast<unsigned>(j0 + j));
                    }
                }
            } else if (GEO == GEO_DISK) {
                float closest[T];
#pragma unroll
                for (int k = 0; k < T; ++k)
                    closest[k] = __int_as_float(0x7f800000);
#pragma unroll 4
                for (int j = jb; j < je; ++j) {
                    const float4 px = s_f[j], py = s_fi[j];
                    const float2 g2 = s_g2[j];
#pragma unroll
                    for (int k = 0; k < T; ++k)
                        disk_pair_x2(f, t2[k], px, py, g2, u2[k], v2[k], closest[k]);
                }
                if (a.near.count) {
#pragma unroll
                    for (int k = 0; k < T; ++k)
                        disk_list_near_x2(f, a.near, t2[k], ti[k],
                                          closest[k] < f.near2 && ti[k] < blk1, s_f, s_fi, jb, je,
                                          j0);
                }
            } else {
#pragma unroll 2
                for (int j = jb; j < je; ++j) {
                    const float4 sf = s_f[j];
                    const float gf = s_gf[j];
#pragma unroll
                    for (int k = 0; k < T; ++k) {
                        bool np, nw;
                        if (pair32<GEO, false>(f, tg[k], sf, sf, gf, false, u[k], v[k], np, nw) &&
                            a.near.count && ti[k] < blk1)
                            list_near(a.near, np, nw, ti[k], static_cast<unsigned>(j0 + j));
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < T; ++k) {
                ud[k] += static_cast<double>(u[k]);
                vd[k] += static_cast<double>(v[k]);
                u[k] = v[k] = 0.0f;
                if (GEO == GEO_DISK) { // the direct and the image lanes, in that order
                    ud[k] += static_cast<double>(u2[k].x);
                    ud[k] += static_cast<double>(u2[k].y);
                    vd[k] += static_cast<double>(v2[k].x);
                    vd[k] += static_cast<double>(v2[k].y);
                    u2[k] = v2[k] = make_float2(0.0f, 0.0f);
                }
            }
        }
        __syncthreads();
        if (tid == 0 && t + 2 < ntiles)
            issue(t + 2);
    }
    const size_t base = static_cast<size_t>(chunk) * a.stride - a.t_begin;
#pragma unroll
    for (int k = 0; k < T; ++k)
        if (ti[k] < blk1) {
            a.pu[base + ti[k]] = ud[k];
            a.pv[base + ti[k]] = vd[k];
        }
}

template <int GEO, int T> int resident32() {
    static std::atomic<int> cached{0};  // host threads may plan at once
    if (!cached.load(std::memory_order_relaxed)) {
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, velocity32_kernel<GEO, 128, T>,
                                                          128, 0) != cudaSuccess ||
            blocks < 1)
            blocks = 1;
        cached.store(blocks, std::memory_order_relaxed);
    }
    return cached.load(std::memory_order_relaxed);
}

template <int GEO> int resident32_t(int per_thread) {
    return per_thread == 1 ? resident32<GEO, 1>()
                           : (per_thread == 2 ? resident32<GEO, 2>() : resident32<GEO, 4>());
}

template <int GEO, int T> cudaError_t launch32_t(const EvalArgs &a, const EvalPlan &p, cudaStream_t s) {
    return launch_pdl(velocity32_kernel<GEO, 128, T>, dim3(static_cast<unsigned>(p.items())),
                      dim3(128), 0, s, a);
}

template <int GEO> cudaError_t launch32_geo(const EvalArgs &a, const EvalPlan &p, cudaStream_t s) {
    switch (p.per_thread) {
    case 1:
        return launch32_t<GEO, 1>(a, p, s);
    case 2:
        return launch32_t<GEO, 2>(a, p, s);
    case 4:
        return launch32_t<GEO, 4>(a, p, s);
    default:
        return cudaErrorInvalidConfiguration;
    }
}
} // namespace

int resident_fp32c(int geometry, int per_thread) {
    return geometry == GEO_INFINITE   ? resident32_t<GEO_INFINITE>(per_thread)
           : geometry == GEO_PERIODIC ? resident32_t<GEO_PERIODIC>(per_thread)
                                      : resident32_t<GEO_DISK>(per_thread);
}

cudaError_t launch_velocity_fp32c(const EvalArgs &a, const EvalPlan &p, cudaStream_t stream) {
    if (a.t_end <= a.t_begin)
        return cudaSuccess;
    if (p.block != 128)
        return cudaErrorInvalidConfiguration;
    switch (a.g.geometry) {
    case GEO_INFINITE:
        return launch32_geo<GEO_INFINITE>(a, p, stream);
    case GEO_PERIODIC:
        return launch32_geo<GEO_PERIODIC>(a, p, stream);
    case GEO_DISK:
        return launch32_geo<GEO_DISK>(a, p, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

} // namespace pvb
