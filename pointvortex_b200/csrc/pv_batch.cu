// pv_batch.cu — batched ensembles: many independent simulations of uneven population and mixed
// geometry advanced together, each with its own adaptive DOPRI5 step (src/timestep.cpp:62-120)
// and the reference driver's end-time logic (src/main.cpp:310-323).
//
// The reference runs one simulation per process. Here the states of all simulations live in one
// device arena, and every DOPRI5 stage is one launch of each kernel for the whole ensemble:
//
//   * velocity: a persistent grid (one wave of resident CTAs) drains a work queue of
//     (simulation, block of 128 threads x T targets, chunk of sources) items with an atomic counter. The
//     items are sorted by cost (periodic pairs cost ~15x plane pairs), so the longest go first.
//     Each CTA copies the item's geometry constants to shared memory and runs the same TMA-staged
//     tile loop and pair functions as the single-simulation kernel. Periodic simulations (both
//     forms) from N = 2048 instead take (simulation, block I, block J) items of 128 x 128 evaluated once
//     per unordered pair (the warp tiles of pv_symmetric.cuh, reactions summed across the CTA's
//     warps in fixed order). Simulations in the FP32-compensated form drain a second queue, in a
//     second launch, with the pair terms of pv_pair32.cuh;
//   * stage: one 256-element block per slice of a simulation reduces that simulation's chunk
//     partials in fixed order, then forms the next stage position or the DOPRI5 error;
//   * control: one thread per simulation runs the step-size control, the rejection cap, the end
//     time, a step budget and the simulation's own failure status;
//   * accept: the state update of the simulations whose attempt was accepted.
//
// A simulation's chunking depends only on its own population, and its arithmetic only on its own
// data, so every result is bit-identical whether it runs alone or in any mix. A failing
// simulation stops with its own status; the others are untouched.
#include "pvb200.h"
#include "pv_internal.h"
#include "pv_pair32.cuh"
#include "pv_symmetric.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

using namespace pvb;

namespace {

constexpr int kBlock = 128;          // threads per velocity CTA
constexpr int kTileB = 256;          // sources per shared-memory stage
constexpr size_t kAlign = 256;       // arena granularity (elements)
constexpr int kCounters = 16;        // work-queue counters: two launches per velocity stage

// Default targets per thread of the ordered items by geometry: the plane's cheap pairs share
// each staged source among 4 targets, the disk's among 2. The autotuner's batch table
// (pv_set_batch_tuning) overrides it per geometry, precision and floor(log2 N).
constexpr int default_targets_per_thread(int geometry) {
    return geometry == GEO_INFINITE ? 4 : (geometry == GEO_DISK ? 2 : 1);
}
// Targets per thread the ordered items may hold, by geometry: 1, 2 or 4; the periodic pair's
// registers allow 1 or 2 beside the other forms in the one persistent kernel.
constexpr bool batch_targets_allowed(int geometry, int per_thread) {
    return per_thread == 1 || per_thread == 2 || (per_thread == 4 && geometry != GEO_PERIODIC);
}

// The batch table: targets per thread by (geometry, precision, floor(log2 N)); 0 = the default.
// Atomic entries: a table update may run beside admissions on other host threads.
std::atomic<int> g_batch_tuning[3][2][40] = {};

int batch_targets_for(int geometry, int precision, size_t n) {
    int bucket = 0;
    while ((size_t(2) << bucket) <= n && bucket < 39)
        ++bucket;
    const int t = g_batch_tuning[geometry][precision][bucket].load(std::memory_order_relaxed);
    return t ? t : default_targets_per_thread(geometry);
}
// Sources per work item, a function of the population only (so a simulation's summation order
// never depends on its batch): 512 up to N = 16384, then N/32 rounded up to 512.
constexpr size_t chunk_for(size_t n) { return n <= 16384 ? 512 : (n / 32 + 511) / 512 * 512; }

enum SimState : int { SIM_FREE = 0, SIM_RUNNING = 1, SIM_DONE = 2, SIM_FAILED = 3, SIM_BUDGET = 4 };

struct SimDesc {
    GeometryConsts g;
    unsigned long long off;       // first element of the simulation in the arena
    unsigned long long part_off;  // first element of its chunk partials
    unsigned n;
    unsigned pad_n;
    unsigned num_chunks;          // partial rows (chunks, or 128-blocks of the symmetric form)
    unsigned chunk;
    int precision;                // PV_PRECISION_*
    int symmetric;                // periodic, evaluated once per unordered pair (either form)
    int per_thread;               // targets per thread of the ordered items (1, 2 or 4)
};

struct SimControl {
    int status;
    int state;
    int accepted;
    int fsal;
    unsigned rejected;
    int failure;                   // PV_FAILURE_* of a ST_DOPRI_FAILED stop
    unsigned long long err_bits;
    unsigned long long steps;
    unsigned long long max_steps;
    unsigned long long rejections_total;
    double t, t_end, dt, dt_attempt;
    double atol, rtol, dtmin, dtmax;
};

enum ItemKind : unsigned { ITEM_ORDERED = 0, ITEM_SYMMETRIC = 1 };

struct Item {
    unsigned sim;
    unsigned tb;     // target block (symmetric: block I)
    unsigned chunk;  // source chunk (symmetric: block J >= I)
    unsigned kind;   // ItemKind
};

// Symmetric-form rows: blocks of kBlock vortices (constexpr helper for host and device)
constexpr unsigned symmetric_rows(unsigned n) { return (n + 127u) / 128u; }

struct SliceEntry { // one 256-element slice of one simulation (stage / accept kernels)
    unsigned sim;
    unsigned start;
};

struct Arena {
    double *x, *y, *gamma, *gs;
    double *px[2], *py[2];
    double *kx[7], *ky[7];
    double *pu, *pv;
};

constexpr double kDopriB[7][7] = {
    {0},
    {1.0 / 5.0},
    {3.0 / 40.0, 9.0 / 40.0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0},
    {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
constexpr double kB5b[7] = {35.0 / 384.0,     0.0,         500.0 / 1113.0, 125.0 / 192.0,
                            -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
constexpr double kB4b[7] = {5179.0 / 57600.0, 0.0,          7571.0 / 16695.0,   393.0 / 640.0,
                            -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0};

struct StageCoefs {
    double a[7][7];
    double w[7];
};

__device__ __forceinline__ double max_r(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double min_r(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double clamp_r(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

// ---------------------------------------------------------------------------------------------
// Velocity: persistent CTAs draining the item queue.
template <class Pair, int T>
__device__ __forceinline__ void run_item(const GeometryConsts &g, const double *px, const double *py,
                                         const double *sgs, size_t src0, size_t src1, size_t blk0,
                                         size_t blk1, double *pu, double *pv, size_t out0,
                                         double (*s_x)[kTileB], double (*s_y)[kTileB],
                                         double (*s_g)[kTileB], uint64_t *bars, uint32_t &seq,
                                         int *timeout_status, bool &timed_out) {
    const int tid = threadIdx.x;
    double tx[T], ty[T], u[T], v[T];
    size_t ti[T];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        ti[k] = blk0 + static_cast<size_t>(k) * kBlock + tid;
        const bool ok = ti[k] < blk1;
        tx[k] = ok ? px[ti[k]] : 0.0;
        ty[k] = ok ? py[ti[k]] : 0.0;
        u[k] = 0.0;
        v[k] = 0.0;
    }
    const int ntiles = src1 > src0 ? static_cast<int>((src1 - src0 + kTileB - 1) / kTileB) : 0;
    const uint32_t seq0 = seq;
    auto issue = [&](int t) {
        const int st = (seq0 + t) & 1;
        const size_t j0 = src0 + static_cast<size_t>(t) * kTileB;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTileB), src1 - j0));
        const int even = cnt & ~1;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bars[st], static_cast<uint32_t>(3 * even * sizeof(double)));
        if (even) {
            const uint32_t bytes = static_cast<uint32_t>(even * sizeof(double));
            bulk_g2s(s_x[st], px + j0, bytes, &bars[st]);
            bulk_g2s(s_y[st], py + j0, bytes, &bars[st]);
            bulk_g2s(s_g[st], sgs + j0, bytes, &bars[st]);
        }
        if (cnt & 1) {
            s_x[st][cnt - 1] = px[j0 + cnt - 1];
            s_y[st][cnt - 1] = py[j0 + cnt - 1];
            s_g[st][cnt - 1] = sgs[j0 + cnt - 1];
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
        const uint32_t k = seq0 + t;
        const int st = k & 1;
        const bool ok = mbar_wait_bounded(&bars[st], (k >> 1) & 1, timeout_status);
        if (__syncthreads_or(!ok)) {
            if (tid == 0)  // the copies of tiles k and k + 1 may still be in flight
                mbar_drain(bars, k, t + 1 < ntiles);
            timed_out = true;
            return;
        }
        const size_t j0 = src0 + static_cast<size_t>(t) * kTileB;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTileB), src1 - j0));
        const double *X = s_x[st], *Y = s_y[st], *G = s_g[st];
        if (j0 < blk1 && blk0 < j0 + cnt) {
#pragma unroll 1
            for (int j = 0; j < cnt; ++j) {
                const double sx = X[j], sy = Y[j], sg = G[j];
#pragma unroll
                for (int q = 0; q < T; ++q)
                    Pair::template pair<true>(g, tx[q], ty[q], sx, sy, sg, ti[q] == j0 + j, u[q], v[q]);
            }
        } else {
#pragma unroll 2
            for (int j = 0; j < cnt; ++j) {
                const double sx = X[j], sy = Y[j], sg = G[j];
#pragma unroll
                for (int q = 0; q < T; ++q)
                    Pair::template pair<false>(g, tx[q], ty[q], sx, sy, sg, false, u[q], v[q]);
            }
        }
        __syncthreads();
        if (tid == 0 && t + 2 < ntiles)
            issue(t + 2);
    }
    seq = seq0 + ntiles;
#pragma unroll
    for (int q = 0; q < T; ++q)
        if (ti[q] < blk1) {
            pu[out0 + ti[q]] = u[q];
            pv[out0 + ti[q]] = v[q];
        }
}

// One 128 x 128 block pair of a periodic FP64 simulation, once per unordered pair: warp w holds
// targets I*128 + 32w + lane and meets the four 32-source sub-tiles of block J in turn. Targets'
// sums go to row J, the sources' reactions (summed over the four warps in fixed order) to row I.
// A diagonal item (I == J) is evaluated one-sided. red_u / red_v: 4 x 128 doubles of shared memory.
__device__ __forceinline__ void run_symmetric_item(const GeometryConsts &g, const double *px,
                                                   const double *py, const double *sgs, size_t n,
                                                   unsigned I, unsigned J, double *pu, double *pv,
                                                   size_t pad_n, double *red_u, double *red_v) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool diagonal = I == J;
    const size_t ti = static_cast<size_t>(I) * kBlock + static_cast<size_t>(w) * 32 + lane;
    const bool t_ok = ti < n;
    const double tx = t_ok ? px[ti] : 0.0, ty = t_ok ? py[ti] : 0.0;
    const double tg2 = t_ok ? 2.0 * sgs[ti] : 0.0;  // doubled: the terms carry half sines
    double u = 0.0, v = 0.0;
    for (int qq = 0; qq < 4; ++qq) {
        const int q = (w + qq) & 3;
        const size_t sj = static_cast<size_t>(J) * kBlock + static_cast<size_t>(q) * 32 + lane;
        const int s_ok = sj < n ? 1 : 0;
        const double sx = s_ok ? px[sj] : 0.0, sy = s_ok ? py[sj] : 0.0;
        const double sg2 = s_ok ? 2.0 * sgs[sj] : 0.0;
        if (diagonal) {
            sym::one_sided_tile(g, tx, ty, t_ok, sx, sy, sg2, s_ok, q == w, u, v);
        } else {
            double ru = 0.0, rv = 0.0;
            sym::react_tile(g, tx, ty, tg2, t_ok, sx, sy, sg2, s_ok, u, v, ru, rv);
            red_u[w * kBlock + q * 32 + lane] = ru;
            red_v[w * kBlock + q * 32 + lane] = rv;
        }
    }
    if (t_ok) {
        pu[static_cast<size_t>(J) * pad_n + ti] = u;
        pv[static_cast<size_t>(J) * pad_n + ti] = v;
    }
    if (!diagonal) {
        __syncthreads();
        const size_t sj = static_cast<size_t>(J) * kBlock + threadIdx.x;
        if (sj < n) {
            double su = red_u[threadIdx.x], sv = red_v[threadIdx.x];
            for (int k = 1; k < 4; ++k) {
                su += red_u[k * kBlock + threadIdx.x];
                sv += red_v[k * kBlock + threadIdx.x];
            }
            pu[static_cast<size_t>(I) * pad_n + sj] = su;
            pv[static_cast<size_t>(I) * pad_n + sj] = sv;
        }
        __syncthreads();
    }
}

// The FP32-compensated form of run_symmetric_item: each warp stages the 32 sources of its current
// sub-tile (hi/lo coordinates, FP32 circulation) in its own shared buffer; FP32 sums of each
// 32 x 32 tile are promoted into FP64.
__device__ __forceinline__ void run_symmetric_item32(const GeometryConsts &g, const double *px,
                                                     const double *py, const double *sgs,
                                                     size_t n, unsigned I, unsigned J,
                                                     double *pu, double *pv, size_t pad_n,
                                                     double *red_u, double *red_v, float4 *s_f,
                                                     float *s_gf) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool diagonal = I == J;
    const f32::F32Geometry f = f32::make_f32(g);
    float4 *sf = s_f + w * 32;
    float *sg = s_gf + w * 32;
    const size_t ti = static_cast<size_t>(I) * kBlock + static_cast<size_t>(w) * 32 + lane;
    const bool t_ok = ti < n;
    const float4 t = sym::split32(t_ok ? px[ti] : 0.0, t_ok ? py[ti] : 0.0);
    const float tg = t_ok ? static_cast<float>(sgs[ti]) : 0.0f;
    double ud = 0.0, vd = 0.0;
    for (int qq = 0; qq < 4; ++qq) {
        const int q = (w + qq) & 3;
        const size_t j0 = static_cast<size_t>(J) * kBlock + static_cast<size_t>(q) * 32;
        const size_t sj = j0 + lane;
        const int s_count = j0 < n ? static_cast<int>(min(static_cast<size_t>(32), n - j0)) : 0;
        __syncwarp();
        sf[lane] = sym::split32(sj < n ? px[sj] : 0.0, sj < n ? py[sj] : 0.0);
        sg[lane] = sj < n ? static_cast<float>(sgs[sj]) : 0.0f;
        __syncwarp();
        float u = 0.0f, v = 0.0f;
        const sym::NearTile no_near{{nullptr, nullptr}, ti, j0};  // ensembles: no near field
        if (diagonal) {
            sym::one_sided_tile32(f, t, t_ok, sf, sg, s_count, q == w, u, v, no_near);
        } else {
            float ru = 0.0f, rv = 0.0f;
            sym::react_tile32(f, t, tg, t_ok, sf, sg, s_count, u, v, ru, rv, no_near);
            red_u[w * kBlock + q * 32 + lane] = static_cast<double>(ru);
            red_v[w * kBlock + q * 32 + lane] = static_cast<double>(rv);
        }
        ud += static_cast<double>(u);
        vd += static_cast<double>(v);
    }
    if (t_ok) {
        pu[static_cast<size_t>(J) * pad_n + ti] = ud;
        pv[static_cast<size_t>(J) * pad_n + ti] = vd;
    }
    if (!diagonal) {
        __syncthreads();
        const size_t sj = static_cast<size_t>(J) * kBlock + threadIdx.x;
        if (sj < n) {
            double su = red_u[threadIdx.x], sv = red_v[threadIdx.x];
            for (int k = 1; k < 4; ++k) {
                su += red_u[k * kBlock + threadIdx.x];
                sv += red_v[k * kBlock + threadIdx.x];
            }
            pu[static_cast<size_t>(I) * pad_n + sj] = su;
            pv[static_cast<size_t>(I) * pad_n + sj] = sv;
        }
        __syncthreads();
    }
}

// The FP32-compensated form of run_item: the staged FP64 tile is split once per CTA into
// double-float FP32 coordinates; FP32 sums are promoted into FP64 every f32::kFlush sources.
template <int GEO, int T>
__device__ __forceinline__ void run_item32(const GeometryConsts &g, const double *px,
                                           const double *py, const double *sgs, size_t src0,
                                           size_t src1, size_t blk0, size_t blk1, double *pu,
                                           double *pv, size_t out0, double (*s_x)[kTileB],
                                           double (*s_y)[kTileB], double (*s_g)[kTileB],
                                           float4 *s_f, float4 *s_fi, float *s_gf, uint64_t *bars,
                                           uint32_t &seq, int *timeout_status, bool &timed_out) {
    const int tid = threadIdx.x;
    const f32::F32Geometry f = f32::make_f32(g);
    f32::Target32 tg[T];
    float u[T], v[T];
    double ud[T], vd[T];
    size_t ti[T];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        ti[k] = blk0 + static_cast<size_t>(k) * kBlock + tid;
        const bool ok = ti[k] < blk1;
        tg[k].x = ok ? px[ti[k]] : 0.0;
        tg[k].y = ok ? py[ti[k]] : 0.0;
        tg[k].xh = static_cast<float>(tg[k].x);
        tg[k].xl = static_cast<float>(tg[k].x - static_cast<double>(tg[k].xh));
        tg[k].yh = static_cast<float>(tg[k].y);
        tg[k].yl = static_cast<float>(tg[k].y - static_cast<double>(tg[k].yh));
        u[k] = v[k] = 0.0f;
        ud[k] = vd[k] = 0.0;
    }
    // the disk's pairs in f32x2 lanes (direct term, wall image): f32::disk_pair_x2
    f32::DiskTarget2 t2[GEO == GEO_DISK ? T : 1];
    float2 u2[GEO == GEO_DISK ? T : 1], v2[GEO == GEO_DISK ? T : 1];
    float2 *s_g2 = reinterpret_cast<float2 *>(s_gf);
    if (GEO == GEO_DISK) {
#pragma unroll
        for (int k = 0; k < T; ++k) {
            t2[k] = f32::disk_target2(tg[k]);
            u2[k] = v2[k] = make_float2(0.0f, 0.0f);
        }
    }
    const int ntiles = src1 > src0 ? static_cast<int>((src1 - src0 + kTileB - 1) / kTileB) : 0;
    const uint32_t seq0 = seq;
    auto issue = [&](int t) {
        const int st = (seq0 + t) & 1;
        const size_t j0 = src0 + static_cast<size_t>(t) * kTileB;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTileB), src1 - j0));
        const int even = cnt & ~1;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bars[st], static_cast<uint32_t>(3 * even * sizeof(double)));
        if (even) {
            const uint32_t bytes = static_cast<uint32_t>(even * sizeof(double));
            bulk_g2s(s_x[st], px + j0, bytes, &bars[st]);
            bulk_g2s(s_y[st], py + j0, bytes, &bars[st]);
            bulk_g2s(s_g[st], sgs + j0, bytes, &bars[st]);
        }
        if (cnt & 1) {
            s_x[st][cnt - 1] = px[j0 + cnt - 1];
            s_y[st][cnt - 1] = py[j0 + cnt - 1];
            s_g[st][cnt - 1] = sgs[j0 + cnt - 1];
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
        const uint32_t k = seq0 + t;
        const int st = k & 1;
        const bool ok = mbar_wait_bounded(&bars[st], (k >> 1) & 1, timeout_status);
        if (__syncthreads_or(!ok)) {
            if (tid == 0)  // the copies of tiles k and k + 1 may still be in flight
                mbar_drain(bars, k, t + 1 < ntiles);
            timed_out = true;
            return;
        }
        const size_t j0 = src0 + static_cast<size_t>(t) * kTileB;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTileB), src1 - j0));
        for (int j = tid; j < cnt; j += kBlock) {
            const double xj = s_x[st][j], yj = s_y[st][j];
            if (GEO == GEO_DISK) {
                f32::disk_pack_source(f32::split_position(xj, yj), f32::image_position(g, xj, yj),
                                      static_cast<float>(s_g[st][j]), s_f[j], s_fi[j], s_g2[j]);
            } else {
                s_f[j] = f32::split_position(xj, yj);
                s_gf[j] = static_cast<float>(s_g[st][j]);
            }
        }
        __syncthreads();
        const bool diagonal = j0 < blk1 && blk0 < j0 + cnt;
        for (int jb = 0; jb < cnt; jb += f32::kFlush) {
            const int je = min(cnt, jb + f32::kFlush);
            if (diagonal) {
#pragma unroll 1
                for (int j = jb; j < je; ++j) {
                    float4 sf = s_f[j], si = sf;
                    float gf;
                    if (GEO == GEO_DISK) {
                        f32::disk_unpack_source(sf, s_fi[j], sf, si);
                        gf = s_g2[j].x;
                    } else {
                        gf = s_gf[j];
                    }
#pragma unroll
                    for (int q = 0; q < T; ++q) {  // ensembles: no near field (nothing is listed)
                        bool np, nw;
                        f32::pair32<GEO, true>(f, tg[q], sf, si, gf, ti[q] == j0 + j, u[q], v[q], np,
                                               nw);
                    }
                }
            } else if (GEO == GEO_DISK) {
#pragma unroll 4
                for (int j = jb; j < je; ++j) {
                    const float4 px4 = s_f[j], py4 = s_fi[j];
                    const float2 g2 = s_g2[j];
#pragma unroll
                    for (int q = 0; q < T; ++q) {
                        float closest = 0.0f;  // no near field in ensembles: unused
                        f32::disk_pair_x2(f, t2[q], px4, py4, g2, u2[q], v2[q], closest);
                    }
                }
            } else {
#pragma unroll 2
                for (int j = jb; j < je; ++j) {
                    const float4 sf = s_f[j];
                    const float gf = s_gf[j];
#pragma unroll
                    for (int q = 0; q < T; ++q) {
                        bool np, nw;
                        f32::pair32<GEO, false>(f, tg[q], sf, sf, gf, false, u[q], v[q], np, nw);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < T; ++q) {
                ud[q] += static_cast<double>(u[q]);
                vd[q] += static_cast<double>(v[q]);
                u[q] = v[q] = 0.0f;
                if (GEO == GEO_DISK) { // the direct and the image lanes, in that order
                    ud[q] += static_cast<double>(u2[q].x);
                    ud[q] += static_cast<double>(u2[q].y);
                    vd[q] += static_cast<double>(v2[q].x);
                    vd[q] += static_cast<double>(v2[q].y);
                    u2[q] = v2[q] = make_float2(0.0f, 0.0f);
                }
            }
        }
        __syncthreads();
        if (tid == 0 && t + 2 < ntiles)
            issue(t + 2);
    }
    seq = seq0 + ntiles;
#pragma unroll
    for (int q = 0; q < T; ++q)
        if (ti[q] < blk1) {
            pu[out0 + ti[q]] = ud[q];
            pv[out0 + ti[q]] = vd[q];
        }
}

struct VelocityBatchArgs {
    const Item *items;
    unsigned n_items;
    unsigned *counter;
    const SimDesc *descs;
    const SimControl *ctl;
    Arena arena;
    int stage;          // 0: positions = state; s: positions of stage s
    int only_without_fsal;
    int *timeout_status;
};

// PREC = PV_PRECISION_FP64: ordered and symmetric items; PREC = PV_PRECISION_FP32C: the
// compensated form's ordered items. Built for 5 resident CTAs per SM: the FP64 form then holds
// 96 registers (128 unbounded, 4 CTAs) without spills, and the 512-member mixed-N ensemble runs
// 2 % faster in FP64 and 1 % in FP32C (six alternating runs, spread under 0.3 %); a bound of 6
// spills the FP64 form and gains nothing.
template <int PREC>
__global__ void __launch_bounds__(kBlock, 5) batch_velocity_kernel(const VelocityBatchArgs a) {
    __shared__ alignas(128) double s_x[2][kTileB];
    __shared__ alignas(128) double s_y[2][kTileB];
    __shared__ alignas(128) double s_g[2][kTileB];
    __shared__ alignas(16) float4 s_f[PREC == PV_PRECISION_FP32C ? kTileB : 1];
    __shared__ alignas(16) float4 s_fi[PREC == PV_PRECISION_FP32C ? kTileB : 1];  // disk images
    __shared__ alignas(8) float s_gf[PREC == PV_PRECISION_FP32C ? 2 * kTileB : 1];  // disk: (g, -g)
    __shared__ alignas(8) uint64_t bars[2];
    __shared__ GeometryConsts s_geo;
    __shared__ unsigned s_item;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t seq = 0;
    bool timed_out = false;
    for (;;) {
        if (threadIdx.x == 0)
            s_item = atomicAdd(a.counter, 1u);
        __syncthreads();
        const unsigned item = s_item;
        if (item >= a.n_items)
            break;
        const Item it = a.items[item];
        const SimControl &c = a.ctl[it.sim];
        const bool skip = c.state != SIM_RUNNING || c.status != 0 ||
                          (a.only_without_fsal && c.fsal);
        if (skip) {
            __syncthreads(); // s_item is rewritten next round
            continue;
        }
        const SimDesc &d = a.descs[it.sim];
        for (int w = threadIdx.x; w < static_cast<int>(sizeof(GeometryConsts) / 4); w += blockDim.x)
            reinterpret_cast<int *>(&s_geo)[w] = reinterpret_cast<const int *>(&d.g)[w];
        __syncthreads();
        const double *px = a.stage == 0 ? a.arena.x : a.arena.px[(a.stage - 1) & 1];
        const double *py = a.stage == 0 ? a.arena.y : a.arena.py[(a.stage - 1) & 1];
        px += d.off;
        py += d.off;
        const double *sgs = a.arena.gs + d.off;
        double *pu = a.arena.pu + d.part_off;
        double *pv = a.arena.pv + d.part_off;
        if (it.kind == ITEM_SYMMETRIC) {
            // the TMA ring is idle between items: its buffers hold the cross-warp reactions
            if constexpr (PREC == PV_PRECISION_FP32C)
                run_symmetric_item32(s_geo, px, py, sgs, d.n, it.tb, it.chunk, pu, pv, d.pad_n,
                                     &s_x[0][0], &s_y[0][0], s_f, s_gf);
            else
                run_symmetric_item(s_geo, px, py, sgs, d.n, it.tb, it.chunk, pu, pv, d.pad_n,
                                   &s_x[0][0], &s_y[0][0]);
            __syncthreads();
            continue;
        }
        const size_t src0 = static_cast<size_t>(it.chunk) * d.chunk;
        const size_t src1 = min(src0 + d.chunk, static_cast<size_t>(d.n));
        const size_t per_block = static_cast<size_t>(kBlock) * d.per_thread;
        const size_t blk0 = static_cast<size_t>(it.tb) * per_block;
        const size_t blk1 = min(blk0 + per_block, static_cast<size_t>(d.n));
        const size_t out0 = static_cast<size_t>(it.chunk) * d.pad_n;
        // one instantiation per (geometry, targets per thread) the batch table allows
        auto ordered = [&](auto geo, auto per_thread) {
            constexpr int G = decltype(geo)::value, T = decltype(per_thread)::value;
            if constexpr (PREC == PV_PRECISION_FP32C) {
                run_item32<G, T>(s_geo, px, py, sgs, src0, src1, blk0, blk1, pu, pv, out0, s_x, s_y,
                                 s_g, s_f, s_fi, s_gf, bars, seq, a.timeout_status, timed_out);
            } else {
                using Pair = std::conditional_t<G == GEO_INFINITE, InfinitePair,
                             std::conditional_t<G == GEO_PERIODIC, PeriodicPair, DiskPair>>;
                run_item<Pair, T>(s_geo, px, py, sgs, src0, src1, blk0, blk1, pu, pv, out0, s_x,
                                  s_y, s_g, bars, seq, a.timeout_status, timed_out);
            }
        };
        using I0 = std::integral_constant<int, GEO_INFINITE>;
        using I1 = std::integral_constant<int, GEO_PERIODIC>;
        using I2 = std::integral_constant<int, GEO_DISK>;
        using T1 = std::integral_constant<int, 1>;
        using T2 = std::integral_constant<int, 2>;
        using T4 = std::integral_constant<int, 4>;
        switch (s_geo.geometry * 8 + d.per_thread) {
        case GEO_INFINITE * 8 + 1: ordered(I0{}, T1{}); break;
        case GEO_INFINITE * 8 + 2: ordered(I0{}, T2{}); break;
        case GEO_INFINITE * 8 + 4: ordered(I0{}, T4{}); break;
        case GEO_PERIODIC * 8 + 1: ordered(I1{}, T1{}); break;
        case GEO_PERIODIC * 8 + 2: ordered(I1{}, T2{}); break;
        case GEO_DISK * 8 + 1: ordered(I2{}, T1{}); break;
        case GEO_DISK * 8 + 2: ordered(I2{}, T2{}); break;
        default: ordered(I2{}, T4{}); break;  // admission allows no other combination
        }
        if (timed_out)
            return;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Stage: reduce chunk partials, then the next stage position or the DOPRI5 error.
struct StageBatchArgs {
    const SliceEntry *slices;
    unsigned n_slices;
    const SimDesc *descs;
    SimControl *ctl;
    Arena arena;
    int s;               // stage being produced
    StageCoefs coefs;
};

__global__ void __launch_bounds__(256) batch_stage_kernel(const StageBatchArgs a) {
    __shared__ double s_max[8];
    __shared__ int s_skip;
    const SliceEntry sl = a.slices[blockIdx.x];
    SimControl &c = a.ctl[sl.sim];
    // one decision for the whole block (other blocks may raise the status meanwhile)
    if (threadIdx.x == 0)
        s_skip = c.state != SIM_RUNNING || *reinterpret_cast<volatile int *>(&c.status) != 0;
    __syncthreads();
    if (s_skip)
        return;
    const SimDesc &d = a.descs[sl.sim];
    const size_t i = sl.start + threadIdx.x;
    const bool inside = i < d.n;
    const int s = a.s;
    const double *ex = (s == 0 ? a.arena.x : a.arena.px[(s - 1) & 1]) + d.off;
    const double *ey = (s == 0 ? a.arena.y : a.arena.py[(s - 1) & 1]) + d.off;
    const double dt = c.dt_attempt;
    double local_max = 0.0;
    const bool reduce = s > 0 || !c.fsal;  // uniform over the block: one simulation per slice
    double wide_u = 0.0, wide_v = 0.0;
    if (reduce && d.num_chunks >= 32) {
        // many partial rows (symmetric items): for each 32 targets of the slice, the 8 warps
        // each sum every 8th row, coalesced, and the targets' own warp adds the 8 group sums
        // in fixed order
        __shared__ double s_u[8][32], s_v[8][32];
        const int lane = threadIdx.x & 31, group = threadIdx.x >> 5;
        for (int pass = 0; pass < 8; ++pass) {
            const size_t t = sl.start + static_cast<size_t>(pass) * 32 + lane;
            double su = 0.0, sv = 0.0;
            if (t < d.n)
                for (unsigned ch = group; ch < d.num_chunks; ch += 8) {
                    su += a.arena.pu[d.part_off + static_cast<size_t>(ch) * d.pad_n + t];
                    sv += a.arena.pv[d.part_off + static_cast<size_t>(ch) * d.pad_n + t];
                }
            s_u[group][lane] = su;
            s_v[group][lane] = sv;
            __syncthreads();
            if (group == pass) {
                wide_u = s_u[0][lane];
                wide_v = s_v[0][lane];
                for (int g = 1; g < 8; ++g) {
                    wide_u += s_u[g][lane];
                    wide_v += s_v[g][lane];
                }
            }
            __syncthreads();
        }
    }
    if (inside) {
        const size_t e = d.off + i;
        double ku, kv;
        if (reduce) {
            ku = 0.0;
            kv = 0.0;
            if (d.num_chunks >= 32) {
                ku = wide_u;
                kv = wide_v;
            } else {
                for (unsigned ch = 0; ch < d.num_chunks; ++ch) {
                    ku += a.arena.pu[d.part_off + static_cast<size_t>(ch) * d.pad_n + i];
                    kv += a.arena.pv[d.part_off + static_cast<size_t>(ch) * d.pad_n + i];
                }
            }
            if (!isfinite(ku) || !isfinite(kv)) {
                const int verdict = slow_target(d.g, ex, ey, a.arena.gamma + d.off, d.n, i, ku, kv);
                if (verdict)
                    atomicMax(&c.status, verdict);
            }
            a.arena.kx[s][e] = ku;
            a.arena.ky[s][e] = kv;
        } else {
            ku = a.arena.kx[0][e];
            kv = a.arena.ky[0][e];
        }
        if (s < 6) {
            double dx = 0.0, dy = 0.0;
            for (int j = 0; j <= s; ++j) {
                const double cf = a.coefs.a[s + 1][j];
                if (cf == 0.0)
                    continue;
                dx = __dadd_rn(dx, __dmul_rn(cf, j == s ? ku : a.arena.kx[j][e]));
                dy = __dadd_rn(dy, __dmul_rn(cf, j == s ? kv : a.arena.ky[j][e]));
            }
            const double nx = __dadd_rn(a.arena.x[e], __dmul_rn(dt, dx));
            const double ny = __dadd_rn(a.arena.y[e], __dmul_rn(dt, dy));
            a.arena.px[s & 1][e] = nx;
            a.arena.py[s & 1][e] = ny;
            if (!isfinite(nx) || !isfinite(ny))
                atomicMax(&c.status, ST_NONFINITE_POSITION);
            else if (d.g.geometry == GEO_DISK &&
                     __dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)) >= d.g.radius2)
                atomicMax(&c.status, ST_OUTSIDE_DISK);
        } else {
            double xe = 0.0, ye = 0.0;
            for (int j = 0; j < 7; ++j) {
                const double w = a.coefs.w[j];
                if (w == 0.0)
                    continue;
                const double h = __dmul_rn(dt, w);
                xe = __dadd_rn(xe, __dmul_rn(h, j == 6 ? ku : a.arena.kx[j][e]));
                ye = __dadd_rn(ye, __dmul_rn(h, j == 6 ? kv : a.arena.ky[j][e]));
            }
            const double x5 = ex[i], y5 = ey[i];
            const double xs = __dadd_rn(c.atol, __dmul_rn(c.rtol, max_r(fabs(a.arena.x[e]), fabs(x5))));
            const double ys = __dadd_rn(c.atol, __dmul_rn(c.rtol, max_r(fabs(a.arena.y[e]), fabs(y5))));
            if (!isfinite(xe) || !isfinite(ye) || !isfinite(xs) || !isfinite(ys) || !(xs > 0.0) ||
                !(ys > 0.0))
                atomicMax(&c.status, ST_DOPRI_NONFINITE);
            else
                local_max = max_r(__ddiv_rn(fabs(xe), xs), __ddiv_rn(fabs(ye), ys));
        }
    }
    if (s == 6) {
        for (int off = 16; off > 0; off >>= 1)
            local_max = max_r(local_max, __shfl_xor_sync(0xffffffffu, local_max, off));
        if ((threadIdx.x & 31) == 0)
            s_max[threadIdx.x >> 5] = local_max;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = 0.0;
            for (int w = 0; w < 8; ++w)
                m = max_r(m, s_max[w]);
            atomicMax(&c.err_bits, ordered_bits(m));
        }
    }
}

// Step-size control (src/timestep.cpp:95-118) and the driver's end-time logic
// (src/main.cpp:312-343) for every running simulation.
__global__ void batch_control_kernel(SimControl *ctl, unsigned n_sims) {
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_sims)
        return;
    SimControl &c = ctl[k];
    c.accepted = 0;
    if (c.state != SIM_RUNNING)
        return;
    if (c.status != 0) {
        c.state = SIM_FAILED;
        return;
    }
    const double error = __longlong_as_double(static_cast<long long>(c.err_bits));
    c.err_bits = 0ull;
    c.fsal = 1; // k0 = f(y0) was produced by this attempt (or carried over) and stays valid
    const double dt = c.dt_attempt;
    const double factor = error == 0.0 ? 5.0 : clamp_r(0.9 * pow(error, -0.2), 0.2, 5.0);
    const double suggested = clamp_r(__dmul_rn(dt, factor), c.dtmin, c.dtmax);
    if (error <= 1.0) {
        c.accepted = 1;
        c.fsal = 1;
        c.dt = suggested;
        c.rejected = 0;
        const double t_new = c.t + dt;
        c.t = t_new;
        ++c.steps;
        const double slack = 16.0 * 2.220446049250313e-16 * fabs(t_new);
        if (t_new + slack >= c.t_end) {
            c.t = c.t_end;
            c.state = SIM_DONE;
        } else if (c.steps >= c.max_steps) {
            c.state = SIM_BUDGET;
        } else {
            c.dt_attempt = min_r(c.dt, c.t_end - c.t);
            if (!(c.t + c.dt_attempt > c.t))  // src/main.cpp:314-315
                c.status = ST_DOPRI_FAILED, c.state = SIM_FAILED,
                c.failure = PV_FAILURE_NO_TIME_ADVANCE;
        }
    } else {
        ++c.rejections_total;
        // src/timestep.cpp:116-117: the floor is tested first, as there
        const bool floor = dt <= c.dtmin;
        if (floor || ++c.rejected > 32u) {
            c.status = ST_DOPRI_FAILED;
            c.state = SIM_FAILED;
            c.failure = floor ? PV_FAILURE_DT_FLOOR : PV_FAILURE_REJECTION_CAP;
        } else {
            c.dt_attempt = max_r(c.dtmin, min_r(suggested, __dmul_rn(dt, 0.9)));
        }
    }
}

__global__ void __launch_bounds__(256) batch_accept_kernel(const SliceEntry *slices,
                                                           const SimDesc *descs,
                                                           const SimControl *ctl, Arena arena) {
    const SliceEntry sl = slices[blockIdx.x];
    if (!ctl[sl.sim].accepted)
        return;
    const SimDesc &d = descs[sl.sim];
    const size_t i = sl.start + threadIdx.x;
    if (i >= d.n)
        return;
    const size_t e = d.off + i;
    arena.x[e] = arena.px[1][e];
    arena.y[e] = arena.py[1][e];
    arena.kx[0][e] = arena.kx[6][e];
    arena.ky[0][e] = arena.ky[6][e];
}

__global__ void scale_kernel(const double *gamma, double *gs, size_t n, GeometryConsts g) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        gs[i] = scaled_circulation(g, gamma[i]);
}

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

} // namespace

// =============================================================================================
struct pv_batch {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    size_t capacity = 0;        // vortices
    size_t part_capacity = 0;   // partial elements per array
    unsigned max_sims = 0;
    uint64_t default_max_steps = 0;
    Arena arena{};
    void *arena_block = nullptr;
    SimDesc *d_descs = nullptr;
    SimControl *d_ctl = nullptr;
    SimControl *h_ctl = nullptr;       // pinned mirror
    Item *d_items = nullptr;
    size_t items_cap = 0;
    SliceEntry *d_slices = nullptr;
    size_t slices_cap = 0;
    unsigned *d_counters = nullptr;    // one queue counter per velocity launch of an attempt
    int *d_timeout = nullptr;
    int resident = 1;                  // FP64 velocity CTAs per SM
    int resident32 = 1;                // FP32C velocity CTAs per SM
    std::vector<SimDesc> descs;
    std::vector<int> slot_used;
    std::map<size_t, size_t> free_elems;  // offset -> length (elements), arena
    std::map<size_t, size_t> free_parts;  // offset -> length, partials
    std::vector<std::pair<size_t, size_t>> sim_ranges, part_ranges;
    bool tables_dirty = true;
    unsigned n_items = 0, n_slices = 0;  // n_items = FP64 items, then n_items32 FP32C items
    unsigned n_items32 = 0;
    uint64_t attempts = 0, evaluations_pairs = 0;
    cudaGraphExec_t attempt_graph = nullptr; // one captured attempt for the current tables
    bool use_graph = true;
    // attempts launched directly since the tables last changed: the attempt is captured as a
    // graph only once they have stayed the same for kCaptureAfter attempts, so that a stream of
    // admissions and retirements does not pay a capture and an instantiation for each change
    unsigned unchanged_attempts = 0;

    ~pv_batch() {
        if (attempt_graph)
            cudaGraphExecDestroy(attempt_graph);
        cudaFree(arena_block);
        cudaFree(d_descs);
        cudaFree(d_ctl);
        cudaFreeHost(h_ctl);
        cudaFree(d_items);
        cudaFree(d_slices);
        cudaFree(d_counters);
        cudaFree(d_timeout);
        if (stream)
            cudaStreamDestroy(stream);
    }
};

namespace {

pv_status bfail(pv_batch *b, pv_status code, const std::string &m) {
    b->error = m;
    return code;
}

#define PVB_CUDA(b, call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return bfail((b), PV_ERROR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
    } while (0)

bool take(std::map<size_t, size_t> &free, size_t len, size_t &off) {
    for (auto it = free.begin(); it != free.end(); ++it)
        if (it->second >= len) {
            off = it->first;
            const size_t rest = it->second - len;
            free.erase(it);
            if (rest)
                free[off + len] = rest;
            return true;
        }
    return false;
}

void give(std::map<size_t, size_t> &free, size_t off, size_t len) {
    auto it = free.emplace(off, len).first;
    auto next = std::next(it);
    if (next != free.end() && it->first + it->second == next->first) {
        it->second += next->second;
        free.erase(next);
    }
    if (it != free.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            free.erase(it);
        }
    }
}

// Rebuilds the work queues (items sorted by cost; FP64 first, then FP32C) and the slice table for
// the running simulations.
pv_status rebuild_tables(pv_batch *b) {
    std::vector<Item> items[2];
    std::vector<double> cost[2];
    std::vector<SliceEntry> slices;
    for (unsigned s = 0; s < b->max_sims; ++s) {
        if (b->slot_used[s] != SIM_RUNNING)
            continue;
        const SimDesc &d = b->descs[s];
        const int q = d.precision == PV_PRECISION_FP32C ? 1 : 0;
        const double w = d.g.geometry == GEO_PERIODIC ? 15.0 : (d.g.geometry == GEO_DISK ? 2.7 : 1.0);
        if (d.symmetric) {
            const unsigned nb = symmetric_rows(d.n);
            for (unsigned I = 0; I < nb; ++I)
                for (unsigned J = I; J < nb; ++J) {
                    items[q].push_back({s, I, J, ITEM_SYMMETRIC});
                    const double ni = std::min<double>(kBlock, d.n - I * double(kBlock));
                    const double nj = std::min<double>(kBlock, d.n - J * double(kBlock));
                    cost[q].push_back(w * ni * nj);
                }
        } else {
            const unsigned per_block = kBlock * d.per_thread;
            const unsigned tbs = (d.n + per_block - 1) / per_block;
            for (unsigned tb = 0; tb < tbs; ++tb)
                for (unsigned ch = 0; ch < d.num_chunks; ++ch) {
                    items[q].push_back({s, tb, ch, ITEM_ORDERED});
                    const double nt = std::min<double>(per_block, d.n - tb * double(per_block));
                    const double ns = std::min<double>(d.chunk, d.n - ch * double(d.chunk));
                    cost[q].push_back(w * nt * ns);
                }
        }
        for (unsigned st = 0; st < d.n; st += 256)
            slices.push_back({s, st});
    }
    std::vector<Item> sorted;
    for (int q = 0; q < 2; ++q) {
        std::vector<size_t> order(items[q].size());
        for (size_t i = 0; i < order.size(); ++i)
            order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t c) { return cost[q][a] > cost[q][c]; });
        for (size_t i : order)
            sorted.push_back(items[q][i]);
    }
    if (sorted.size() > b->items_cap) {
        cudaFree(b->d_items);
        b->d_items = nullptr;
        b->items_cap = round_up(sorted.size(), 4096);
        PVB_CUDA(b, cudaMalloc(&b->d_items, b->items_cap * sizeof(Item)));
    }
    if (slices.size() > b->slices_cap) {
        cudaFree(b->d_slices);
        b->d_slices = nullptr;
        b->slices_cap = round_up(slices.size(), 4096);
        PVB_CUDA(b, cudaMalloc(&b->d_slices, b->slices_cap * sizeof(SliceEntry)));
    }
    if (!sorted.empty())
        PVB_CUDA(b, cudaMemcpyAsync(b->d_items, sorted.data(), sorted.size() * sizeof(Item),
                                    cudaMemcpyHostToDevice, b->stream));
    if (!slices.empty())
        PVB_CUDA(b, cudaMemcpyAsync(b->d_slices, slices.data(), slices.size() * sizeof(SliceEntry),
                                    cudaMemcpyHostToDevice, b->stream));
    PVB_CUDA(b, cudaStreamSynchronize(b->stream));
    b->n_items = static_cast<unsigned>(items[0].size());
    b->n_items32 = static_cast<unsigned>(items[1].size());
    b->n_slices = static_cast<unsigned>(slices.size());
    b->tables_dirty = false;
    return PV_OK;
}

StageCoefs stage_coefs() {
    StageCoefs c{};
    for (int i = 0; i < 7; ++i)
        for (int j = 0; j < 7; ++j)
            c.a[i][j] = kDopriB[i][j];
    for (int j = 0; j < 7; ++j)
        c.w[j] = kB5b[j] - kB4b[j];
    return c;
}

// The velocity of one stage: the FP64 queue, then the FP32C queue (counters 2s and 2s + 1).
pv_status launch_velocity_stage(pv_batch *b, int stage, int only_without_fsal, int counter) {
    VelocityBatchArgs a{};
    a.descs = b->d_descs;
    a.ctl = b->d_ctl;
    a.arena = b->arena;
    a.stage = stage;
    a.only_without_fsal = only_without_fsal;
    a.timeout_status = b->d_timeout;
    if (b->n_items) {
        a.items = b->d_items;
        a.n_items = b->n_items;
        a.counter = b->d_counters + 2 * counter;
        // a persistent grid of one wave, or fewer CTAs than that when the queue is short (a
        // small ensemble: CTAs that would only find the queue empty cost launch time)
        const unsigned grid = static_cast<unsigned>(
            std::max(1u, std::min(static_cast<unsigned>(b->sm_count * b->resident), b->n_items)));
        batch_velocity_kernel<PV_PRECISION_FP64><<<grid, kBlock, 0, b->stream>>>(a);
        PVB_CUDA(b, cudaGetLastError());
    }
    if (b->n_items32) {
        a.items = b->d_items + b->n_items;
        a.n_items = b->n_items32;
        a.counter = b->d_counters + 2 * counter + 1;
        const unsigned grid = static_cast<unsigned>(std::max(
            1u, std::min(static_cast<unsigned>(b->sm_count * b->resident32), b->n_items32)));
        batch_velocity_kernel<PV_PRECISION_FP32C><<<grid, kBlock, 0, b->stream>>>(a);
        PVB_CUDA(b, cudaGetLastError());
    }
    return PV_OK;
}

pv_status enqueue_attempt(pv_batch *b) {
    if (b->n_items + b->n_items32 == 0)
        return PV_OK;
    PVB_CUDA(b, cudaMemsetAsync(b->d_counters, 0, kCounters * sizeof(unsigned), b->stream));
    const StageCoefs coefs = stage_coefs();
    pv_status st;
    if ((st = launch_velocity_stage(b, 0, 1, 0)) != PV_OK)
        return st;
    for (int s = 0; s < 7; ++s) {
        if (s > 0 && (st = launch_velocity_stage(b, s, 0, s)) != PV_OK)
            return st;
        StageBatchArgs a{};
        a.slices = b->d_slices;
        a.n_slices = b->n_slices;
        a.descs = b->d_descs;
        a.ctl = b->d_ctl;
        a.arena = b->arena;
        a.s = s;
        a.coefs = coefs;
        batch_stage_kernel<<<b->n_slices, 256, 0, b->stream>>>(a);
        PVB_CUDA(b, cudaGetLastError());
    }
    batch_control_kernel<<<(b->max_sims + 127) / 128, 128, 0, b->stream>>>(b->d_ctl, b->max_sims);
    PVB_CUDA(b, cudaGetLastError());
    batch_accept_kernel<<<b->n_slices, 256, 0, b->stream>>>(b->d_slices, b->d_descs, b->d_ctl,
                                                            b->arena);
    PVB_CUDA(b, cudaGetLastError());
    return PV_OK;
}

// Attempts with unchanged tables after which the attempt is captured as a graph.
constexpr unsigned kCaptureAfter = 8;

// Captures one attempt (17 nodes for the current work queue and slice table) as a CUDA graph, so
// that each further attempt is one graph launch.
pv_status capture_attempt(pv_batch *b) {
    if (b->attempt_graph) {
        cudaGraphExecDestroy(b->attempt_graph);
        b->attempt_graph = nullptr;
    }
    if (!b->use_graph || b->n_items + b->n_items32 == 0)
        return PV_OK;
    cudaGraph_t graph = nullptr;
    PVB_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const pv_status st = enqueue_attempt(b);
    const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (st != PV_OK) {
        if (graph)
            cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess)
        return bfail(b, PV_ERROR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&b->attempt_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess)
        return bfail(b, PV_ERROR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
    return PV_OK;
}

} // namespace

extern "C" {

pv_status pv_batch_create(const pv_batch_config *config, pv_batch **out) {
    if (!config || !out) {
        set_thread_error("null argument");
        return PV_ERROR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (config->max_simulations == 0 || config->capacity_vortices == 0) {
        set_thread_error("a batch needs room for at least one simulation and one vortex");
        return PV_ERROR_INVALID_ARGUMENT;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || config->device < 0 || config->device >= count) {
        set_thread_error("no such CUDA device");
        return PV_ERROR_CUDA;
    }
    cudaSetDevice(config->device);
    auto *b = new pv_batch();
    b->device = config->device;
    b->max_sims = config->max_simulations;
    b->default_max_steps = config->max_steps_per_simulation ? config->max_steps_per_simulation
                                                            : ~0ull;
    const auto bail = [&](cudaError_t e, const char *what) {
        set_thread_error(std::string(what) + ": " + cudaGetErrorString(e));
        delete b;
        return PV_ERROR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device)) != cudaSuccess)
        return bail(e, "cudaDeviceGetAttribute");
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
             &b->resident, batch_velocity_kernel<PV_PRECISION_FP64>, kBlock, 0)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
             &b->resident32, batch_velocity_kernel<PV_PRECISION_FP32C>, kBlock, 0)) != cudaSuccess)
        return bail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    b->resident = std::max(1, b->resident);
    b->resident32 = std::max(1, b->resident32);
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(e, "cudaStreamCreate");
    b->capacity = round_up(config->capacity_vortices, kAlign) + kAlign * b->max_sims;
    // partials: each simulation needs ceil(n/512) chunks of pad(n); bounded by capacity^2/512 but
    // allocated as a multiple of the element capacity (sized by the caller's partial factor)
    const size_t factor = config->partial_chunks_per_vortex_slot ? config->partial_chunks_per_vortex_slot : 16;
    b->part_capacity = b->capacity * factor;
    const size_t arrays = 4 + 4 + 14;
    const size_t bytes = (arrays * b->capacity + 2 * b->part_capacity) * sizeof(double);
    if ((e = cudaMalloc(&b->arena_block, bytes)) != cudaSuccess)
        return bail(e, "cudaMalloc(batch arena)");
    double *p = static_cast<double *>(b->arena_block);
    auto next = [&](size_t n) {
        double *q = p;
        p += n;
        return q;
    };
    b->arena.x = next(b->capacity);
    b->arena.y = next(b->capacity);
    b->arena.gamma = next(b->capacity);
    b->arena.gs = next(b->capacity);
    for (int k = 0; k < 2; ++k) {
        b->arena.px[k] = next(b->capacity);
        b->arena.py[k] = next(b->capacity);
    }
    for (int k = 0; k < 7; ++k) {
        b->arena.kx[k] = next(b->capacity);
        b->arena.ky[k] = next(b->capacity);
    }
    b->arena.pu = next(b->part_capacity);
    b->arena.pv = next(b->part_capacity);
    if ((e = cudaMalloc(&b->d_descs, b->max_sims * sizeof(SimDesc))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_ctl, b->max_sims * sizeof(SimControl))) != cudaSuccess ||
        (e = cudaMallocHost(&b->h_ctl, b->max_sims * sizeof(SimControl))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_counters, kCounters * sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_timeout, sizeof(int))) != cudaSuccess)
        return bail(e, "cudaMalloc(batch tables)");
    std::memset(b->h_ctl, 0, b->max_sims * sizeof(SimControl));
    cudaMemcpy(b->d_ctl, b->h_ctl, b->max_sims * sizeof(SimControl), cudaMemcpyHostToDevice);
    cudaMemset(b->d_timeout, 0, sizeof(int));
    b->descs.assign(b->max_sims, SimDesc{});
    b->slot_used.assign(b->max_sims, SIM_FREE);
    b->sim_ranges.assign(b->max_sims, {0, 0});
    b->part_ranges.assign(b->max_sims, {0, 0});
    b->free_elems[0] = b->capacity;
    b->free_parts[0] = b->part_capacity;
    *out = b;
    return PV_OK;
}

void pv_batch_destroy(pv_batch *b) {
    if (!b)
        return;
    cudaSetDevice(b->device);
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    delete b;
}

const char *pv_batch_last_error(const pv_batch *b) { return b ? b->error.c_str() : ""; }

pv_status pv_batch_add(pv_batch *b, const pv_params *params, const double *x, const double *y,
                       const double *circulation, size_t n, const pv_batch_solve *solve,
                       uint32_t *id) {
    if (!b || !params || !solve || !id)
        return PV_ERROR_INVALID_ARGUMENT;
    GeometryConsts g;
    std::string message;
    pv_status st = static_cast<pv_status>(make_geometry_consts(*params, g, message));
    if (st != PV_OK)
        return bfail(b, st, message);
    if (n == 0)
        return bfail(b, PV_ERROR_INVALID_ARGUMENT, "a batched simulation needs at least one vortex");
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(circulation[i]))
            return bfail(b, PV_ERROR_INVALID_ARGUMENT, "vortex data must be finite");
    if (g.geometry == GEO_PERIODIC) {
        double total = 0.0, absolute = 0.0;
        for (size_t i = 0; i < n; ++i) {
            total += circulation[i];
            absolute += std::fabs(circulation[i]);
        }
        if (std::fabs(total) > 1e-12 * std::max(1.0, absolute))
            return bfail(b, PV_ERROR_INVALID_ARGUMENT, "periodic box requires zero total circulation");
    } else if (g.geometry == GEO_DISK) {
        for (size_t i = 0; i < n; ++i)
            if (x[i] * x[i] + y[i] * y[i] >= g.radius2)
                return bfail(b, PV_ERROR_INVALID_ARGUMENT, "vortex lies on or outside the disk");
    }
    if (!(solve->t_end >= 0.0) || !std::isfinite(solve->t_end) || !(solve->dt > 0.0) ||
        !(solve->absolute_tolerance > 0.0) || !(solve->relative_tolerance >= 0.0) ||
        !(solve->minimum_time_step > 0.0) || !(solve->maximum_time_step >= solve->minimum_time_step))
        return bfail(b, PV_ERROR_INVALID_ARGUMENT, "invalid solve parameters");
    unsigned slot = b->max_sims;
    for (unsigned s = 0; s < b->max_sims; ++s)
        if (b->slot_used[s] == SIM_FREE) {
            slot = s;
            break;
        }
    if (slot == b->max_sims)
        return bfail(b, PV_ERROR_CAPACITY, "no free simulation slot");
    if (params->precision != PV_PRECISION_FP64 && params->precision != PV_PRECISION_FP32C)
        return bfail(b, PV_ERROR_INVALID_ARGUMENT, "unknown precision form");
    const size_t pad = round_up(n, kAlign);
    const size_t chunk = chunk_for(n);
    // periodic populations from kSymmetricMinN up: once per unordered pair, one partial row
    // per 128-block. The autotuner's table of the symmetric form (pv_set_symmetric_tuning) may
    // choose otherwise for the population's size; either way the choice is a function of the
    // simulation's own n, geometry and precision, never of the batch.
    const int tuned = symmetric_tuning_lookup(g.geometry, params->precision, n) & 15;
    const bool symmetric = g.geometry == GEO_PERIODIC && n >= 128 &&
                           (tuned == 2 || (tuned == 0 && n >= kSymmetricMinN));
    const unsigned chunks = symmetric ? symmetric_rows(static_cast<unsigned>(n))
                                      : static_cast<unsigned>((n + chunk - 1) / chunk);
    size_t off = 0, poff = 0;
    if (!take(b->free_elems, pad, off))
        return bfail(b, PV_ERROR_CAPACITY, "the batch arena has no room for this population");
    if (!take(b->free_parts, pad * chunks, poff)) {
        give(b->free_elems, off, pad);
        return bfail(b, PV_ERROR_CAPACITY, "the batch partial buffer has no room for this population");
    }
    SimDesc d{};
    d.g = g;
    d.off = off;
    d.part_off = poff;
    d.n = static_cast<unsigned>(n);
    d.pad_n = static_cast<unsigned>(pad);
    d.num_chunks = chunks;
    d.chunk = static_cast<unsigned>(chunk);
    d.precision = params->precision;
    d.symmetric = symmetric ? 1 : 0;
    d.per_thread = batch_targets_for(g.geometry, params->precision, n);
    b->descs[slot] = d;
    b->sim_ranges[slot] = {off, pad};
    b->part_ranges[slot] = {poff, pad * chunks};
    SimControl c{};
    c.state = SIM_RUNNING;
    c.t = 0.0;
    c.t_end = solve->t_end;
    c.dt = std::min(std::max(solve->dt, solve->minimum_time_step), solve->maximum_time_step);
    c.dt_attempt = std::min(c.dt, c.t_end - c.t);
    c.atol = solve->absolute_tolerance;
    c.rtol = solve->relative_tolerance;
    c.dtmin = solve->minimum_time_step;
    c.dtmax = solve->maximum_time_step;
    c.max_steps = solve->max_steps ? solve->max_steps : b->default_max_steps;
    if (c.t_end <= 0.0)
        c.state = SIM_DONE;
    cudaSetDevice(b->device);
    const size_t bytes = n * sizeof(double);
    PVB_CUDA(b, cudaMemcpyAsync(b->arena.x + off, x, bytes, cudaMemcpyHostToDevice, b->stream));
    PVB_CUDA(b, cudaMemcpyAsync(b->arena.y + off, y, bytes, cudaMemcpyHostToDevice, b->stream));
    PVB_CUDA(b, cudaMemcpyAsync(b->arena.gamma + off, circulation, bytes, cudaMemcpyHostToDevice, b->stream));
    scale_kernel<<<(static_cast<unsigned>(n) + 255) / 256, 256, 0, b->stream>>>(b->arena.gamma + off,
                                                                                b->arena.gs + off, n, g);
    PVB_CUDA(b, cudaGetLastError());
    PVB_CUDA(b, cudaMemcpyAsync(b->d_descs + slot, &b->descs[slot], sizeof(SimDesc),
                                cudaMemcpyHostToDevice, b->stream));
    b->h_ctl[slot] = c;
    PVB_CUDA(b, cudaMemcpyAsync(b->d_ctl + slot, &b->h_ctl[slot], sizeof(SimControl),
                                cudaMemcpyHostToDevice, b->stream));
    PVB_CUDA(b, cudaStreamSynchronize(b->stream));
    b->slot_used[slot] = c.state;
    b->tables_dirty = true;
    *id = slot;
    return PV_OK;
}

pv_status pv_batch_advance(pv_batch *b, uint32_t attempts, uint32_t *running) {
    if (!b)
        return PV_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    pv_status st;
    for (uint32_t k = 0; k < attempts; ++k) {
        if (b->tables_dirty) {
            if ((st = rebuild_tables(b)) != PV_OK)
                return st;
            if (b->attempt_graph) {
                cudaGraphExecDestroy(b->attempt_graph);
                b->attempt_graph = nullptr;
            }
            b->unchanged_attempts = 0;
        }
        if (b->n_items + b->n_items32 == 0)
            break;
        if (!b->attempt_graph && b->unchanged_attempts >= kCaptureAfter &&
            (st = capture_attempt(b)) != PV_OK)
            return st;
        if (b->attempt_graph)
            PVB_CUDA(b, cudaGraphLaunch(b->attempt_graph, b->stream));
        else if ((st = enqueue_attempt(b)) != PV_OK)
            return st;
        ++b->unchanged_attempts;
        ++b->attempts;
    }
    PVB_CUDA(b, cudaMemcpyAsync(b->h_ctl, b->d_ctl, b->max_sims * sizeof(SimControl),
                                cudaMemcpyDeviceToHost, b->stream));
    PVB_CUDA(b, cudaStreamSynchronize(b->stream));
    int timeout = 0;
    PVB_CUDA(b, cudaMemcpy(&timeout, b->d_timeout, sizeof(int), cudaMemcpyDeviceToHost));
    if (timeout)
        return bfail(b, PV_ERROR_RUNTIME, "a bounded device wait timed out");
    uint32_t live = 0;
    for (unsigned s = 0; s < b->max_sims; ++s) {
        if (b->slot_used[s] == SIM_RUNNING && b->h_ctl[s].state != SIM_RUNNING) {
            b->slot_used[s] = b->h_ctl[s].state;
            b->tables_dirty = true;
        }
        if (b->slot_used[s] == SIM_RUNNING)
            ++live;
    }
    if (running)
        *running = live;
    return PV_OK;
}

pv_status pv_batch_info(pv_batch *b, uint32_t id, pv_batch_sim_info *info) {
    if (!b || !info || id >= b->max_sims || b->slot_used[id] == SIM_FREE)
        return PV_ERROR_INVALID_ARGUMENT;
    const SimControl &c = b->h_ctl[id];
    info->state = b->slot_used[id];
    info->status = c.status;
    info->time = c.t;
    info->suggested_time_step = c.dt;
    info->accepted_steps = c.steps;
    info->rejected_steps = c.rejections_total;
    info->population = b->descs[id].n;
    info->failure = c.status == ST_DOPRI_FAILED ? c.failure : PV_FAILURE_NONE;
    info->targets_per_thread = b->descs[id].symmetric ? 0 : b->descs[id].per_thread;
    return PV_OK;
}

pv_status pv_set_batch_tuning(int geometry, int precision, int log2_n, int per_thread) {
    if (geometry < 0 || geometry > 2 || precision < 0 || precision > 1 || log2_n < 0 ||
        log2_n >= 40 || (per_thread != 0 && !batch_targets_allowed(geometry, per_thread))) {
        set_thread_error("invalid batch tuning entry");
        return PV_ERROR_INVALID_ARGUMENT;
    }
    g_batch_tuning[geometry][precision][log2_n].store(per_thread, std::memory_order_relaxed);
    return PV_OK;
}

pv_status pv_get_batch_tuning(int geometry, int precision, int log2_n, int *per_thread) {
    if (!per_thread || geometry < 0 || geometry > 2 || precision < 0 || precision > 1 ||
        log2_n < 0 || log2_n >= 40)
        return PV_ERROR_INVALID_ARGUMENT;
    *per_thread = batch_targets_for(geometry, precision, size_t(1) << log2_n);
    return PV_OK;
}

pv_status pv_batch_result(pv_batch *b, uint32_t id, double *x, double *y, size_t n) {
    if (!b || id >= b->max_sims || b->slot_used[id] == SIM_FREE)
        return PV_ERROR_INVALID_ARGUMENT;
    if (n != b->descs[id].n)
        return bfail(b, PV_ERROR_RUNTIME, "host and device vortex populations differ");
    cudaSetDevice(b->device);
    const size_t off = b->descs[id].off;
    PVB_CUDA(b, cudaMemcpyAsync(x, b->arena.x + off, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    PVB_CUDA(b, cudaMemcpyAsync(y, b->arena.y + off, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    PVB_CUDA(b, cudaStreamSynchronize(b->stream));
    return PV_OK;
}

pv_status pv_batch_release(pv_batch *b, uint32_t id) {
    if (!b || id >= b->max_sims || b->slot_used[id] == SIM_FREE)
        return PV_ERROR_INVALID_ARGUMENT;
    if (b->slot_used[id] == SIM_RUNNING) {
        // stop it on the device first
        b->h_ctl[id].state = SIM_FREE;
        cudaSetDevice(b->device);
        PVB_CUDA(b, cudaMemcpyAsync(&b->d_ctl[id].state, &b->h_ctl[id].state, sizeof(int),
                                    cudaMemcpyHostToDevice, b->stream));
        PVB_CUDA(b, cudaStreamSynchronize(b->stream));
        b->tables_dirty = true;
    }
    give(b->free_elems, b->sim_ranges[id].first, b->sim_ranges[id].second);
    give(b->free_parts, b->part_ranges[id].first, b->part_ranges[id].second);
    b->slot_used[id] = SIM_FREE;
    return PV_OK;
}

pv_status pv_batch_status(pv_batch *b, pv_batch_totals *totals) {
    if (!b || !totals)
        return PV_ERROR_INVALID_ARGUMENT;
    totals->attempts = b->attempts;
    totals->work_items = b->n_items + b->n_items32;
    size_t free_elems = 0;
    for (auto &kv : b->free_elems)
        free_elems += kv.second;
    totals->free_vortices = free_elems;
    unsigned running = 0, used = 0;
    for (unsigned s = 0; s < b->max_sims; ++s) {
        running += b->slot_used[s] == SIM_RUNNING;
        used += b->slot_used[s] != SIM_FREE;
    }
    totals->running = running;
    totals->occupied_slots = used;
    return PV_OK;
}

pv_status pv_batch_stream(const pv_batch *b, void **stream) {
    if (!b || !stream)
        return PV_ERROR_INVALID_ARGUMENT;
    *stream = static_cast<void *>(b->stream);
    return PV_OK;
}

} // extern "C"
