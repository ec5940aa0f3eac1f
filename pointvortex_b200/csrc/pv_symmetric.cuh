// pv_symmetric.cuh — warp tiles evaluated once per unordered pair (periodic box, infinite plane),
// shared by the single-simulation kernels (pv_symmetric.cu) and the batched ensembles
// (pv_batch.cu).
//
// A tile is 32 targets (one per lane) against 32 sources. The sources, with the reactions they
// accumulate, rotate one lane per step by shuffles; after 32 steps every (target, source) pair has
// been met once and every source is back in its home lane. The pair terms are exactly odd under
// exchanging target and source, so one evaluation gives the target's term and, with the other
// circulation and the opposite sign, the source's. Callers pass the scaled circulations times
// the policy's kScale (the periodic terms carry half sines: 2 * Gamma * 0.5/L).
#pragma once

#include "pv_geometry.cuh"
#include "pv_pair32.cuh"

namespace pvb {
namespace sym {

__device__ __forceinline__ double rotate(double v, int from) {
    return __shfl_sync(0xffffffffu, v, from);
}

// Pair kernels K of the geometries evaluated this way: the target's velocity changes by
// u -= c_s K_u, v += c_s K_v and the source's by u += c_t K_u, v -= c_t K_v, where c is the
// stored scaled circulation times kScale.
struct PeriodicSym {
    // the terms carry half sines (PeriodicPair::terms<true>): circulations are doubled
    static constexpr double kScale = 2.0;
    __device__ __forceinline__ static void values(const GeometryConsts &g, double tx, double ty,
                                                  double sx, double sy, double &ku, double &kv) {
        double au, bu, av, bv;
        PeriodicPair::terms<true>(g, tx, ty, sx, sy, au, bu, av, bv);
        ku = au * rcp_refined(bu);
        kv = av * rcp_refined(bv);
    }
};

// The infinite plane (InfinitePair): K = (dy, dx) / (r^2 + eps^2), exactly odd in (dx, dy).
struct PlaneSym {
    static constexpr double kScale = 1.0;
    __device__ __forceinline__ static void values(const GeometryConsts &g, double tx, double ty,
                                                  double sx, double sy, double &ku, double &kv) {
        const double dx = tx - sx, dy = ty - sy;
        const double inv = rcp_refined(fma(dx, dx, fma(dy, dy, g.eps2)));
        ku = dy * inv;
        kv = dx * inv;
    }
};

// Targets (tx, ty, tg) against the sources held in the lanes (sx, sy, sg and their reactions
// ru, rv); adds the targets' sums to u, v and the sources' to ru, rv. Sources end at home.
// FULL: all 32 targets and sources exist (every tile but the last block's), no predicates.
template <class P, bool FULL>
__device__ __forceinline__ void react_tile_t(const GeometryConsts &g, double tx, double ty,
                                             double tg, bool t_ok, double sx, double sy,
                                             double sg, int s_ok, double &u, double &v,
                                             double &ru, double &rv) {
    const int next = (threadIdx.x + 1) & 31;
#pragma unroll 2
    for (int k = 0; k < 32; ++k) {
        if (FULL || (t_ok && s_ok)) {
            double ku, kv;
            P::values(g, tx, ty, sx, sy, ku, kv);
            u = fma(-sg, ku, u);   // target: -c_s K
            v = fma(sg, kv, v);
            ru = fma(tg, ku, ru);  // source: the exchanged pair, +c_t K
            rv = fma(-tg, kv, rv);
        }
        sx = rotate(sx, next);
        sy = rotate(sy, next);
        sg = rotate(sg, next);
        ru = rotate(ru, next);
        rv = rotate(rv, next);
        if (!FULL)
            s_ok = __shfl_sync(0xffffffffu, s_ok, next);
    }
}

template <class P = PeriodicSym>
__device__ __forceinline__ void react_tile(const GeometryConsts &g, double tx, double ty,
                                           double tg, bool t_ok, double sx, double sy, double sg,
                                           int s_ok, double &u, double &v, double &ru,
                                           double &rv) {
    if (__all_sync(0xffffffffu, t_ok && s_ok))
        react_tile_t<P, true>(g, tx, ty, tg, t_ok, sx, sy, sg, s_ok, u, v, ru, rv);
    else
        react_tile_t<P, false>(g, tx, ty, tg, t_ok, sx, sy, sg, s_ok, u, v, ru, rv);
}

// T targets per lane (T sub-blocks of targets) against one sub-block of 32 sources, every target
// and source present. Each rotation step serves T pairs, so the shuffles (five doubles a step)
// per pair fall by T: for a cheap pair term (the plane's) they would otherwise bound the tile.
template <class P, int T>
__device__ __forceinline__ void react_tiles_full(const GeometryConsts &g, const double (&tx)[T],
                                                 const double (&ty)[T], const double (&tg)[T],
                                                 double sx, double sy, double sg, double (&u)[T],
                                                 double (&v)[T], double &ru, double &rv) {
    const int next = (threadIdx.x + 1) & 31;
#pragma unroll 2
    for (int k = 0; k < 32; ++k) {
#pragma unroll
        for (int t = 0; t < T; ++t) {
            double ku, kv;
            P::values(g, tx[t], ty[t], sx, sy, ku, kv);
            u[t] = fma(-sg, ku, u[t]);
            v[t] = fma(sg, kv, v[t]);
            ru = fma(tg[t], ku, ru);
            rv = fma(-tg[t], kv, rv);
        }
        sx = rotate(sx, next);
        sy = rotate(sy, next);
        sg = rotate(sg, next);
        ru = rotate(ru, next);
        rv = rotate(rv, next);
    }
}

// Target side only. same_block: the sources are the targets' own lanes, so the self pair (k = 0)
// is skipped; the reference skips it too (and in the periodic box it contributes exactly 0).
template <class P = PeriodicSym>
__device__ __forceinline__ void one_sided_tile(const GeometryConsts &g, double tx, double ty,
                                               bool t_ok, double sx, double sy, double sg,
                                               int s_ok, bool same_block, double &u, double &v) {
    const int next = (threadIdx.x + 1) & 31;
    for (int k = 0; k < 32; ++k) {
        if (t_ok && s_ok && !(same_block && k == 0)) {
            double ku, kv;
            P::values(g, tx, ty, sx, sy, ku, kv);
            u = fma(-sg, ku, u);
            v = fma(sg, kv, v);
        }
        sx = rotate(sx, next);
        sy = rotate(sy, next);
        sg = rotate(sg, next);
        s_ok = __shfl_sync(0xffffffffu, s_ok, next);
    }
}

// FP32-compensated tiles: the 32 sources (hi/lo coordinates and FP32 circulation) sit in this
// warp's shared buffer, read at index (lane + k) & 31; only their FP32 reactions rotate through
// the lanes. V: the pair kernel (f32::Periodic32, f32::Plane32). The callers promote the FP32
// sums of each tile into FP64.
//
// Near pairs (V::kNear kernels) contribute 0 here and are listed for the FP64 pass, in both
// directions, under the lane's target `ti` and the tile's source j0 + j.
struct NearTile {
    f32::NearLists lists;  // lists.count == nullptr: no near field
    size_t ti;             // this lane's target
    size_t j0;             // the tile's first source
};

template <class V>
__device__ __forceinline__ void list_near_pair(const NearTile &nt, int j, bool both) {
    if (V::kNear && nt.lists.count) {
        f32::near_append(nt.lists, nt.ti, static_cast<unsigned>(nt.j0 + j));
        if (both)
            f32::near_append(nt.lists, nt.j0 + j, static_cast<unsigned>(nt.ti));
    }
}

template <class V, bool FULL>
__device__ __forceinline__ void react_tile32_t(const f32::F32Geometry &f, const float4 t, float tg,
                                               bool t_ok, const float4 *sf, const float *sg,
                                               int s_count, float &u, float &v, float &ru,
                                               float &rv, const NearTile &nt) {
    const int lane = threadIdx.x & 31, next = (lane + 1) & 31;
#pragma unroll 2
    for (int k = 0; k < 32; ++k) {
        const int j = (lane + k) & 31;
        if (FULL || (t_ok && j < s_count)) {
            float ku, kv;
            if (V::values(f, t, sf[j], ku, kv))
                list_near_pair<V>(nt, j, true);
            const float g = sg[j];
            u = fmaf(-g, ku, u);
            v = fmaf(g, kv, v);
            ru = fmaf(tg, ku, ru);
            rv = fmaf(-tg, kv, rv);
        }
        ru = __shfl_sync(0xffffffffu, ru, next);
        rv = __shfl_sync(0xffffffffu, rv, next);
    }
}

template <class V = f32::Periodic32>
__device__ __forceinline__ void react_tile32(const f32::F32Geometry &f, const float4 t, float tg,
                                             bool t_ok, const float4 *sf, const float *sg,
                                             int s_count, float &u, float &v, float &ru,
                                             float &rv, const NearTile &nt) {
    if (__all_sync(0xffffffffu, t_ok && s_count == 32))
        react_tile32_t<V, true>(f, t, tg, t_ok, sf, sg, s_count, u, v, ru, rv, nt);
    else
        react_tile32_t<V, false>(f, t, tg, t_ok, sf, sg, s_count, u, v, ru, rv, nt);
}

// T targets per lane against the 32 sources of the buffer, every target and source present: each
// step serves T pairs per lane, and the reactions' two shuffles are shared by them. Only for pair
// kernels without a near field (the plane): a near verdict is not acted on here. A reaction
// would sum 32T terms in FP32 over the tile; it is restarted every 8 steps instead (8T terms, as
// many as the ordered FP32C kernel sums before promoting), and the four partials of a source,
// left in the lanes 8, 16, 24 and 32 places on, are added in FP64 into rud, rvd.
template <class V, int T>
__device__ __forceinline__ void react_tiles32_full(const f32::F32Geometry &f, const float4 (&t)[T],
                                                   const float (&tg)[T], const float4 *sf,
                                                   const float *sg, float (&u)[T], float (&v)[T],
                                                   double &rud, double &rvd) {
    const int lane = threadIdx.x & 31, next = (lane + 1) & 31;
    float pu[4], pv[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        float ru = 0.0f, rv = 0.0f;
#pragma unroll 2
        for (int kk = 0; kk < 8; ++kk) {
            const int j = (lane + 8 * m + kk) & 31;
            const float4 s = sf[j];
            const float g = sg[j];
#pragma unroll
            for (int q = 0; q < T; ++q) {
                float ku, kv;
                V::values(f, t[q], s, ku, kv);
                u[q] = fmaf(-g, ku, u[q]);
                v[q] = fmaf(g, kv, v[q]);
                ru = fmaf(tg[q], ku, ru);
                rv = fmaf(-tg[q], kv, rv);
            }
            ru = __shfl_sync(0xffffffffu, ru, next);
            rv = __shfl_sync(0xffffffffu, rv, next);
        }
        pu[m] = ru;  // the partial of source (lane + 8 (m + 1)) & 31
        pv[m] = rv;
    }
    rud = static_cast<double>(__shfl_sync(0xffffffffu, pu[0], (lane - 8) & 31));
    rvd = static_cast<double>(__shfl_sync(0xffffffffu, pv[0], (lane - 8) & 31));
    rud += static_cast<double>(__shfl_sync(0xffffffffu, pu[1], (lane - 16) & 31));
    rvd += static_cast<double>(__shfl_sync(0xffffffffu, pv[1], (lane - 16) & 31));
    rud += static_cast<double>(__shfl_sync(0xffffffffu, pu[2], (lane - 24) & 31));
    rvd += static_cast<double>(__shfl_sync(0xffffffffu, pv[2], (lane - 24) & 31));
    rud += static_cast<double>(pu[3]);
    rvd += static_cast<double>(pv[3]);
}

template <class V = f32::Periodic32>
__device__ __forceinline__ void one_sided_tile32(const f32::F32Geometry &f, const float4 t,
                                                 bool t_ok, const float4 *sf, const float *sg,
                                                 int s_count, bool same_block, float &u,
                                                 float &v, const NearTile &nt) {
    const int lane = threadIdx.x & 31;
    for (int k = same_block ? 1 : 0; k < 32; ++k) {
        const int j = (lane + k) & 31;
        if (t_ok && j < s_count) {
            float ku, kv;
            if (V::values(f, t, sf[j], ku, kv))  // the other side lists its own pair
                list_near_pair<V>(nt, j, false);
            u = fmaf(-sg[j], ku, u);
            v = fmaf(sg[j], kv, v);
        }
    }
}

// (x_hi, y_hi, x_lo, y_lo) of a double position.
__device__ __forceinline__ float4 split32(double x, double y) { return f32::split_position(x, y); }

}  // namespace sym
}  // namespace pvb
