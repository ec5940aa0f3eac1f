// pv_velocity.cu — tiled direct O(N^2) Biot–Savart evaluation, FP64, sm_100a.
//
// Replaces the three evaluateRange loops of the reference (src/compute.cpp:88-133, 203-256,
// 286-336) and its one-thread-per-target CUDA kernel (src/backend_cuda.cu:22-113).
//
// Design (B200):
//   * work item = (block of B*T targets, chunk of sources); the grid covers all items once,
//     sized from the SM count so that every SM gets several items even at small N;
//   * each thread keeps T targets (x, y, u, v) in registers;
//   * source tiles of TILE vortices (x, y, scaled circulation: 3 x TILE doubles) are staged in
//     shared memory by TMA bulk copies (cp.async.bulk, no multicast) into a two-stage ring
//     guarded by mbarriers, so the next tile lands while the current one is consumed;
//   * every thread reads each source with a broadcast shared-memory load and applies it to its
//     T targets; the geometry is a template parameter (no branch in the pair loop) and the self
//     pair test is compiled only into the diagonal tiles;
//   * partial sums of a chunk go to global memory; the stage kernel reduces chunks in fixed order.
#include "pv_internal.h"

#include <algorithm>
#include <atomic>

namespace pvb {

constexpr int kTile = 256; // sources per shared-memory stage

template <class Pair, int B, int T>
__global__ void __launch_bounds__(B) velocity_kernel(const EvalArgs a) {
    __shared__ alignas(128) double s_x[2][kTile];
    __shared__ alignas(128) double s_y[2][kTile];
    __shared__ alignas(128) double s_g[2][kTile];
    __shared__ alignas(8) uint64_t bars[2];
    __shared__ int s_status;

    pdl_enter();
    const int tid = threadIdx.x;
    if (tid == 0)
        s_status = *reinterpret_cast<volatile int *>(a.status);
    __syncthreads();
    if (s_status != 0)
        return;

    const int item = blockIdx.x;
    const int tb = item / a.num_chunks;
    const int chunk = item - tb * a.num_chunks;
    const size_t src0 = static_cast<size_t>(chunk) * a.chunk;
    const size_t src1 = min(src0 + static_cast<size_t>(a.chunk), a.n_src);
    const size_t blk0 = a.t_begin + static_cast<size_t>(tb) * (B * T);
    const size_t blk1 = min(blk0 + static_cast<size_t>(B * T), a.t_end);

    double tx[T], ty[T], u[T], v[T];
    size_t ti[T];
#pragma unroll
    for (int k = 0; k < T; ++k) {
        ti[k] = blk0 + static_cast<size_t>(k) * B + tid;
        const bool ok = ti[k] < blk1;
        tx[k] = ok ? a.tx[ti[k]] : 0.0;
        ty[k] = ok ? a.ty[ti[k]] : 0.0;
        u[k] = 0.0;
        v[k] = 0.0;
    }

    const int ntiles = src1 > src0 ? static_cast<int>((src1 - src0 + kTile - 1) / kTile) : 0;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();

    // Elected thread: arm the stage's barrier and copy tile t (an even number of doubles per
    // array by TMA; an odd last element with a plain load, published by the __syncthreads that
    // separates issue from consumption).
    auto issue = [&](int t) {
        const int st = t & 1;
        const size_t j0 = src0 + static_cast<size_t>(t) * kTile;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTile), src1 - j0));
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
        const size_t j0 = src0 + static_cast<size_t>(t) * kTile;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTile), src1 - j0));
        const double *X = s_x[st];
        const double *Y = s_y[st];
        const double *G = s_g[st];
        const bool diagonal = j0 < blk1 && blk0 < j0 + cnt;
        if (diagonal) {
#pragma unroll 1
            for (int j = 0; j < cnt; ++j) {
                const double sx = X[j], sy = Y[j], sg = G[j];
                const size_t sj = j0 + j;
#pragma unroll
                for (int k = 0; k < T; ++k)
                    Pair::template pair<true>(a.g, tx[k], ty[k], sx, sy, sg, ti[k] == sj, u[k],
                                              v[k]);
            }
        } else {
#pragma unroll 2
            for (int j = 0; j < cnt; ++j) {
                const double sx = X[j], sy = Y[j], sg = G[j];
#pragma unroll
                for (int k = 0; k < T; ++k)
                    Pair::template pair<false>(a.g, tx[k], ty[k], sx, sy, sg, false, u[k], v[k]);
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
            a.pu[base + ti[k]] = u[k];
            a.pv[base + ti[k]] = v[k];
        }
}

namespace {
template <class Pair, int T>
cudaError_t launch_t(const EvalArgs &a, const EvalPlan &p, cudaStream_t stream) {
    constexpr int B = 128;
    if (p.block != B)
        return cudaErrorInvalidConfiguration;
    return launch_pdl(velocity_kernel<Pair, B, T>, dim3(static_cast<unsigned>(p.items())), dim3(B),
                      0, stream, a);
}

template <class Pair>
cudaError_t launch_pair(const EvalArgs &a, const EvalPlan &p, cudaStream_t stream) {
    switch (p.per_thread) {
    case 1:
        return launch_t<Pair, 1>(a, p, stream);
    case 2:
        return launch_t<Pair, 2>(a, p, stream);
    case 4:
        return launch_t<Pair, 4>(a, p, stream);
    default:
        return cudaErrorInvalidConfiguration;
    }
}
} // namespace

namespace {
// Resident CTAs per SM of one kernel instance (registers and shared memory decide it).
// (Contexts on several host threads may ask at once: the cache is an atomic, and a repeated
// query gives the same value.)
template <class Pair, int T> int resident_ctas() {
    static std::atomic<int> cached{-1};
    int v = cached.load(std::memory_order_relaxed);
    if (v < 0) {
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, velocity_kernel<Pair, 128, T>,
                                                          128, 0) != cudaSuccess || blocks < 1)
            blocks = 1;
        cached.store(blocks, std::memory_order_relaxed);
        v = blocks;
    }
    return v;
}

template <class Pair> int resident_for(int per_thread) {
    return per_thread == 1 ? resident_ctas<Pair, 1>()
                           : (per_thread == 2 ? resident_ctas<Pair, 2>() : resident_ctas<Pair, 4>());
}
} // namespace

namespace {
// Autotuner table: targets per thread for (geometry, precision, floor(log2 N)); 0 = heuristic.
// Atomic entries: a table update may run beside evaluations on other host threads.
std::atomic<int> g_tuning[3][2][40] = {};
} // namespace

int tuning_lookup(int geometry, int precision, size_t n) {
    if (geometry < 0 || geometry > 2 || precision < 0 || precision > 1 || n == 0)
        return 0;
    int bucket = 0;
    while ((size_t(2) << bucket) <= n && bucket < 39)
        ++bucket;
    return g_tuning[geometry][precision][bucket].load(std::memory_order_relaxed);
}

bool tuning_store(int geometry, int precision, int log2_n, int per_thread) {
    if (geometry < 0 || geometry > 2 || precision < 0 || precision > 1 || log2_n < 0 ||
        log2_n >= 40 || (per_thread != 0 && per_thread != 1 && per_thread != 2 && per_thread != 4))
        return false;
    g_tuning[geometry][precision][log2_n].store(per_thread, std::memory_order_relaxed);
    return true;
}

EvalPlan plan_evaluation(int geometry, size_t n_targets, size_t n_sources, int sm_count,
                         int per_thread_override, int precision) {
    EvalPlan p{};
    p.block = 128;
    if (per_thread_override == 0)
        per_thread_override = tuning_lookup(geometry, precision, n_sources);
    // Registers per pair grow from the infinite plane to the periodic series; fewer targets per
    // thread keep the heavier geometries at full occupancy.
    p.per_thread = geometry == GEO_INFINITE ? 4 : (geometry == GEO_DISK ? 2 : 1);
    if (per_thread_override == 1 || per_thread_override == 2 || per_thread_override == 4)
        p.per_thread = per_thread_override;
    const auto resident_of = [&](int t) {
        if (precision == 1)
            return resident_fp32c(geometry, t);
        return geometry == GEO_INFINITE   ? resident_for<InfinitePair>(t)
               : geometry == GEO_PERIODIC ? resident_for<PeriodicPair>(t)
                                          : resident_for<DiskPair>(t);
    };
    const auto blocks_of = [&](int t) {
        const size_t per_block = static_cast<size_t>(p.block) * t;
        return std::max<size_t>(1, (n_targets + per_block - 1) / per_block);
    };
    // A chunk shorter than min_chunk spends more on loading targets than on pairs; small
    // populations accept short chunks (and fewer targets per thread) to give every SM work.
    size_t min_chunk = geometry == GEO_PERIODIC ? 64 : 2 * kTile;
    const size_t sms = static_cast<size_t>(std::max(sm_count, 1));
    if (per_thread_override == 0)
        while (p.per_thread > 1 &&
               blocks_of(p.per_thread) * std::max<size_t>(1, n_sources / min_chunk) <
                   sms * resident_of(p.per_thread))
            p.per_thread /= 2;
    if (blocks_of(p.per_thread) * std::max<size_t>(1, n_sources / min_chunk) <
        sms * resident_of(p.per_thread))
        min_chunk = 64;
    p.target_blocks = static_cast<int>(blocks_of(p.per_thread));
    const size_t slots = sms * resident_of(p.per_thread);
    const size_t max_chunks = std::max<size_t>(1, n_sources / min_chunk);
    // Every item costs about the same, so the grid runs in waves of `slots` CTAs: pick the chunk
    // count (up to four waves) whose last wave is fullest; ties go to fewer chunks.
    size_t best_chunks = 1;
    double best_eff = -1.0;
    const size_t limit = std::min<size_t>(max_chunks, std::max<size_t>(1, 4 * slots / p.target_blocks + 1));
    for (size_t c = 1; c <= limit; ++c) {
        const size_t chunk = std::max<size_t>(2, ((n_sources + c - 1) / c + 1) & ~size_t(1));
        const size_t chunks = (n_sources + chunk - 1) / chunk;
        const size_t items = chunks * p.target_blocks;
        const size_t waves = (items + slots - 1) / slots;
        // fraction of the machine busy over the kernel, counting the pair work of each item
        const double eff = static_cast<double>(items) / static_cast<double>(waves * slots);
        if (eff > best_eff + 1e-3) {
            best_eff = eff;
            best_chunks = chunks;
        }
    }
    size_t chunk = (n_sources + best_chunks - 1) / best_chunks;
    chunk = std::max<size_t>(2, (chunk + 1) & ~static_cast<size_t>(1));
    p.chunk = static_cast<int>(chunk);
    p.num_chunks = static_cast<int>(std::max<size_t>(1, (n_sources + chunk - 1) / chunk));
    return p;
}

cudaError_t launch_velocity(const EvalArgs &a, const EvalPlan &p, cudaStream_t stream) {
    if (a.t_end <= a.t_begin)
        return cudaSuccess;
    switch (a.g.geometry) {
    case GEO_INFINITE:
        return launch_pair<InfinitePair>(a, p, stream);
    case GEO_PERIODIC:
        return launch_pair<PeriodicPair>(a, p, stream);
    case GEO_DISK:
        return launch_pair<DiskPair>(a, p, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

} // namespace pvb
