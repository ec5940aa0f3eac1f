// pv_pair32.cuh — FP32-compensated pair terms, shared by the single-simulation kernels
// (pv_velocity32.cu, pv_symmetric.cu) and the batched ensembles (pv_batch.cu).
//
// Coordinates enter as double-float pairs (hi = fp32(x), lo = fp32(x - hi)), so a displacement
// (t_hi - s_hi) + (t_lo - s_lo) keeps ~2^-24 relative accuracy at every separation. The periodic
// series, the direct Biot-Savart term and the disk's wall image run on the FP32 pipe. The wall
// image of a source s is the circle theorem's vortex -Gamma at s* = R^2 s / |s|^2 (the
// reference's image term, src/compute.cpp:314-333, is exactly its velocity), so it is evaluated
// as a direct term from s*, whose displacement is as accurate as any other: no cancellation
// near the wall.
//
// Near field: an FP32 term carries ~1e-7 of its own size, so the few pairs whose terms are large
// set the error of a sum. Terms closer than the near-field radius -- the periodic pair at its
// minimum-image distance, the disk's direct pair, and the disk image at its distance to the
// target -- are left out of the FP32 sum and listed (near_append) for the FP64 pass of pv_near.cu,
// which adds their exact FP64 terms in index order. The plane has no near field. Callers promote
// FP32 partial sums into FP64 every kFlush sources.
#pragma once

#include "pv_common.cuh"
#include "pv_geometry.cuh"

namespace pvb {
namespace f32 {

constexpr int kFlush = 64; // sources summed in FP32 before promotion to FP64

// Near-field lists: per target, up to kNearSlots listed sources (a source index, with kNearImage
// set for the disk's wall image of that source). count[t] may exceed kNearSlots: the FP64 pass
// then evaluates the whole target in FP64. count == nullptr: nothing is listed.
constexpr int kNearSlots = 32;
constexpr unsigned kNearImage = 0x80000000u;
struct NearLists {
    unsigned *count;  // [n] zero before an evaluation; the FP64 pass leaves it zero again
    unsigned *slot;   // [n][kNearSlots]
};

__device__ __forceinline__ void near_append(const NearLists &lists, size_t target,
                                            unsigned entry) {
    const unsigned k = atomicAdd(lists.count + target, 1u);
    if (k < kNearSlots)
        lists.slot[target * kNearSlots + k] = entry;
}

__device__ __forceinline__ float rcp_approx_f32(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

struct F32Geometry { // the FP32 constants of one evaluation
    float eps2;
    float l_hi, l_lo, inv_l, half_wave;
    float two_cosh_m[3], cosh_m[3], sinh2_m[3];
    float k1, k2;
    int m_exact;
    float inv_radius2;
    float near2;       // near-field radius squared (0: no near field)
};

__device__ __forceinline__ F32Geometry make_f32(const GeometryConsts &g) {
    F32Geometry f;
    f.eps2 = static_cast<float>(g.eps2);
    f.l_hi = static_cast<float>(g.lx);
    f.l_lo = static_cast<float>(g.lx - static_cast<double>(f.l_hi));
    f.inv_l = static_cast<float>(g.inv_lx);
    f.half_wave = static_cast<float>(0.5 * g.wave);
    for (int m = 0; m < 3; ++m) {
        f.two_cosh_m[m] = static_cast<float>(g.two_cosh_m[m]);
        f.cosh_m[m] = static_cast<float>(g.cosh_m[m]);
        f.sinh2_m[m] = static_cast<float>(g.sinh2_m[m]);
    }
    // In FP32 the images m = +-2 join the m = 3..6 expansion 2u C + 2u^2 c cosh 2x^: with
    // u = sech 4 pi = 7e-6 its remainder O(u^3 C^3) is below 1e-11 of the sum, far under FP32
    // resolution, and the exact pair (six f32x2 instructions per pair) is spared.
    const double u2 = g.m_exact >= 2 ? 1.0 / g.cosh_m[2] : 0.0;
    f.k1 = static_cast<float>(g.k1 + 2.0 * u2);
    f.k2 = static_cast<float>(g.k2 + 2.0 * u2 * u2);
    f.m_exact = g.m_exact;
    f.inv_radius2 = static_cast<float>(g.inv_radius2);
    f.near2 = static_cast<float>(g.near2);
    return f;
}

// (x_hi, y_hi, x_lo, y_lo) of a double position.
__device__ __forceinline__ float4 split_position(double x, double y) {
    const float xh = static_cast<float>(x), yh = static_cast<float>(y);
    return make_float4(xh, yh, static_cast<float>(x - static_cast<double>(xh)),
                       static_cast<float>(y - static_cast<double>(yh)));
}

// The wall image of a disk source at (x, y): the vortex -Gamma at R^2 (x, y) / (x^2 + y^2), as
// double-float coordinates. A source at the centre has its image at infinity and contributes 0
// in the reference; a far finite point (FP32 squares stay finite) gives a term below 1e-15.
__device__ __forceinline__ float4 image_position(const GeometryConsts &g, double x, double y) {
    const double r2 = fma(x, x, y * y);
    if (!(r2 > 1e-30 * g.radius2))
        return make_float4(1e15f, 0.0f, 0.0f, 0.0f);
    const double k = __ddiv_rn(g.radius2, r2);
    return split_position(k * x, k * y);
}

// Two FP32 lanes per instruction (FADD2, FMUL2, FFMA2 on sm_100): the periodic pair's x and y
// axes, or the disk's direct and image terms, run side by side. Each lane is rounded exactly as
// the scalar instruction would round it.
__device__ __forceinline__ float2 splat2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 swap2(float2 a) { return make_float2(a.y, a.x); }

// sinh, sin and cos of t (|t| <= pi/2) for both lanes, from the grouping of the shared series in
// pv_common.cuh (sinh t = t (E1 + t^2 O1), sin t = t (E1 - t^2 O1), cos t = E0 - t^2 O0 in
// w = t^4) at FP32 accuracy: E1, E0 and O0 are their degree-3 Taylor polynomials economized to
// degree 2 over w in [0, (pi/2)^4] (Lanczos: the w^3 term traded for the shifted Chebyshev
// polynomial of that degree), adding at most 1.1e-9, 1.5e-8 and 8e-11 to them; O1 keeps its three
// Taylor terms (economizing it would add 3e-7 to sinh). cosh t is not needed in FP32. O0 is
// evaluated negated, so that cos needs no negation.
__device__ __forceinline__ void sh_sn_cs_x2(float2 t, float2 &sh, float2 &sn, float2 &cs) {
    const float2 t2 = mul2(t, t), w = mul2(t2, t2);
    float2 e1 = fma2(w, splat2(2.7571984e-06f), splat2(8.33333e-03f));
    e1 = fma2(w, e1, splat2(1.0f));
    float2 o1 = fma2(w, splat2(2.505210838544172e-08f), splat2(1.984126984126984e-04f)); // 1/11!, 1/7!
    o1 = fma2(w, o1, splat2(1.6666666666666666e-01f));
    float2 e0 = fma2(w, splat2(2.4820652e-05f), splat2(4.1666623e-02f));
    e0 = fma2(w, e0, splat2(1.0f));
    float2 o0n = fma2(w, splat2(-2.7567793e-07f), splat2(-1.3888887e-03f));
    o0n = fma2(w, o0n, splat2(-0.5f));
    const float2 t3 = mul2(t, t2), te1 = mul2(t, e1);
    sh = fma2(t3, o1, te1);
    sn = fma2(mul2(t3, splat2(-1.0f)), o1, te1);
    cs = fma2(t2, o0n, e0);
}

// The periodic pair's core in FP32, both axes at once (lane 0: the target's u term, lane 1: its v
// term). th/tl and sh/sl are the (x, y) hi and lo parts of target and source. Returns the near
// decision (minimum-image distance below the near-field radius); a2 = (sin y^ N_u, sin x^ N_v)
// and b2 = (d0_u den_u, d0_v den_v): the terms are a2 / b2. skip (near or the self pair) sets
// d0 = 1 so that b2 stays finite; the caller discards those terms.
__device__ __forceinline__ bool periodic_core_x2(const F32Geometry &f, float2 th, float2 tl,
                                                 float2 sh, float2 sl, bool self, float2 &a2,
                                                 float2 &b2) {
    const float2 m1 = splat2(-1.0f);
    // (dx, dy) = (t_hi - s_hi) + (t_lo - s_lo); fma(s, -1, t) is t - s exactly
    const float2 d = add2(fma2(sh, m1, th), fma2(sl, m1, tl));
    // half of x^ = (2 pi/L) remainder(dx, L) from the double-float displacement
    const float2 q = mul2(d, splat2(f.inv_l));
    const float2 n = make_float2(rintf(q.x), rintf(q.y));
    const float2 r = fma2(n, splat2(-f.l_lo), fma2(n, splat2(-f.l_hi), d));
    const float2 h = mul2(splat2(f.half_wave), r);
    const bool near = fmaf(r.x, r.x, r.y * r.y) < f.near2 && !self;
    float2 shh, snh, csh;
    sh_sn_cs_x2(h, shh, snh, csh);
    const float2 tsh = mul2(splat2(2.0f), shh), tsn = mul2(splat2(2.0f), snh);
    const float2 sn2 = mul2(tsn, snh);                          // 2 sin^2
    const float2 cosh_ = fma2(tsh, shh, splat2(1.0f));          // cosh x^ = 1 + 2 sinh^2
    const float2 cos_ = fma2(sn2, splat2(-1.0f), splat2(1.0f)); // cos x^ = 1 - 2 sin^2
    const float2 sin_ = mul2(tsn, csh);                         // sin x^ = 2 sin cos
    // d0 = (2 (sh_x^2 + sn_y^2), 2 (sh_y^2 + sn_x^2))
    float2 d0 = fma2(tsh, shh, swap2(sn2));
    if (near || self)
        d0 = splat2(1.0f);
    // the images m != 0 of each lane's axis, as PeriodicPair::image_sum but with only m = +-1
    // exact; C = cosh of the lane's axis, c = cos of the other.
    const float2 C = cosh_, c = swap2(cos_);
    const float2 ch2 = mul2(C, C);
    const float2 p = fma2(c, c, ch2);
    const float2 m2c = mul2(splat2(-2.0f), c);
    const float2 qq = mul2(m2c, C);
    float2 num = splat2(0.0f), den = splat2(1.0f);
    if (f.m_exact >= 1) {
        num = fma2(C, splat2(f.two_cosh_m[1]), m2c);
        den = fma2(qq, splat2(f.cosh_m[1]), add2(p, splat2(f.sinh2_m[1])));
    }
    // m = +-2 and beyond through k1, k2 (make_f32)
    const float2 rest =
        fma2(C, splat2(f.k1), mul2(c, fma2(splat2(2.0f * f.k2), ch2, splat2(-f.k2))));
    // 1/d0 + num/den + rest = (den + d0 (num + den rest)) / (d0 den)
    a2 = mul2(swap2(sin_), fma2(d0, fma2(den, rest, num), den));
    b2 = mul2(d0, den);
    return near;
}

struct Target32 {
    float xh, xl, yh, yl;
    double x, y;
};

// The periodic pair's terms without its circulation, in FP32: the target's velocity changes by
// u -= g_s ku, v += g_s kv. t and s are (x_hi, y_hi, x_lo, y_lo). Exchanging target and source
// negates the displacement exactly, and every quantity below is an exactly odd or even function
// of it, so ku and kv are exactly odd: the symmetric kernels use one evaluation for both.
// Returns true for a near pair (minimum-image distance below the near-field radius, the same
// decision from either side): its terms are then 0 here and come from the FP64 pass.
__device__ __forceinline__ bool periodic_values32(const F32Geometry &f, const float4 t,
                                                  const float4 s, float &ku, float &kv) {
    float2 a2, b2;
    const bool near = periodic_core_x2(f, make_float2(t.x, t.y), make_float2(t.z, t.w),
                                       make_float2(s.x, s.y), make_float2(s.z, s.w), false, a2, b2);
    ku = near ? 0.0f : a2.x * rcp_approx_f32(b2.x);
    kv = near ? 0.0f : a2.y * rcp_approx_f32(b2.y);
    return near;
}

// The plane's kernel values in FP32: K = (dy, dx) / (r^2 + eps^2) from the double-float
// displacement. Exactly odd under exchanging target and source, as periodic_values32. The plane
// has no near field.
__device__ __forceinline__ void plane_values32(const F32Geometry &f, const float4 t,
                                               const float4 s, float &ku, float &kv) {
    const float dx = (t.x - s.x) + (t.z - s.z);
    const float dy = (t.y - s.y) + (t.w - s.w);
    const float inv = rcp_approx_f32(fmaf(dx, dx, fmaf(dy, dy, f.eps2)));
    ku = dy * inv;
    kv = dx * inv;
}

// The pair kernels of the FP32 symmetric tiles (circulations enter unscaled). values() returns
// true for a near pair (terms 0, listed for the FP64 pass); kNear: the kernel has a near field.
struct Periodic32 {
    static constexpr bool kNear = true;
    __device__ __forceinline__ static bool values(const F32Geometry &f, const float4 t,
                                                  const float4 s, float &ku, float &kv) {
        return periodic_values32(f, t, s, ku, kv);
    }
};
struct Plane32 {
    static constexpr bool kNear = false;
    __device__ __forceinline__ static bool values(const F32Geometry &f, const float4 t,
                                                  const float4 s, float &ku, float &kv) {
        plane_values32(f, t, s, ku, kv);
        return false;
    }
};

// One ordered pair in FP32: t the target, s the source (x_hi, y_hi, x_lo, y_lo), si the source's
// wall image (disk only), sgf its scaled circulation. CHECK/self: the self pair (diagonal tiles)
// has no direct term; the disk keeps its self image, as the reference does. near_pair (the
// pair's own term: periodic box, disk direct term) and near_wall (the source's wall image, disk)
// tell which terms are in the near field: those are left out here, and the caller lists them for
// the FP64 pass. Returns near_pair || near_wall (one test in the caller's common path). The plane
// has no near field.
template <int GEO, bool CHECK>
__device__ __forceinline__ bool pair32(const F32Geometry &f, const Target32 &t, const float4 s,
                                       const float4 si, float sgf, bool self, float &u, float &v,
                                       bool &near_pair, bool &near_wall) {
    near_pair = false;
    near_wall = false;
    const float dx = (t.xh - s.x) + (t.xl - s.z);
    const float dy = (t.yh - s.y) + (t.yl - s.w);
    if (GEO == GEO_PERIODIC) {
        float2 a2, b2;
        const bool self_pair = CHECK && self;
        const bool near = periodic_core_x2(f, make_float2(t.xh, t.yh), make_float2(t.xl, t.yl),
                                           make_float2(s.x, s.y), make_float2(s.z, s.w), self_pair,
                                           a2, b2);
        const bool skip = near || self_pair;
        const float cu = skip ? 0.0f : sgf * a2.x;
        const float cv = skip ? 0.0f : sgf * a2.y;
        u = fmaf(-cu, rcp_approx_f32(b2.x), u);
        v = fmaf(cv, rcp_approx_f32(b2.y), v);
        near_pair = near;
        return near;
    }
    // direct Biot–Savart term (plane, and the disk's j != i term)
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, GEO == GEO_INFINITE ? f.eps2 : 0.0f));
    float c = sgf * rcp_approx_f32(r2);
    if (GEO == GEO_DISK) {
        near_pair = r2 < f.near2 && !(CHECK && self);
        c = near_pair ? 0.0f : c;
    }
    if (CHECK && self)
        c = 0.0f;
    u = fmaf(-c, dy, u);
    v = fmaf(c, dx, v);
    if (GEO == GEO_DISK) {  // the wall image: the vortex -Gamma at si
        const float ix = (t.xh - si.x) + (t.xl - si.z);
        const float iy = (t.yh - si.y) + (t.yl - si.w);
        const float ri2 = fmaf(ix, ix, iy * iy);
        near_wall = ri2 < f.near2;
        const float ci = near_wall ? 0.0f : sgf * rcp_approx_f32(ri2);
        u = fmaf(ci, iy, u);
        v = fmaf(-ci, ix, v);
        return near_pair || near_wall;
    }
    return false;
}

// The disk's pair with both of its terms in one set of f32x2 instructions (FADD2, FMUL2, FFMA2:
// two FP32 lanes per register pair and per issue on sm_100). Lane 0 is the direct term, lane 1
// the source's wall image. The sources are staged packed and with the signs arranged so that no
// negation is issued per pair:
//   px = (-s.xh, -si.xh, -s.xl, -si.xl), py = (s.yh, si.yh, s.yl, si.yl), g2 = (gf, -gf),
// and the target is (xh, xh), (xl, xl), (-yh, -yh), (-yl, -yl). Then dx = t - s and
// dyn = s_y - t_y = -dy exactly (IEEE negation commutes with rounding), so the updates
// u += c dyn, v += c dx are the scalar form's u -= c dy, v += c dx bit for bit, per term; the two
// terms accumulate in separate lanes. A near term gets rcp(inf) = 0.
struct DiskTarget2 {
    float2 xh, xl, nyh, nyl;
};

__device__ __forceinline__ DiskTarget2 disk_target2(const Target32 &t) {
    return {make_float2(t.xh, t.xh), make_float2(t.xl, t.xl), make_float2(-t.yh, -t.yh),
            make_float2(-t.yl, -t.yl)};
}

__device__ __forceinline__ void disk_pack_source(const float4 sf, const float4 si, float gf,
                                                 float4 &px, float4 &py, float2 &g2) {
    px = make_float4(-sf.x, -si.x, -sf.z, -si.z);
    py = make_float4(sf.y, si.y, sf.w, si.w);
    g2 = make_float2(gf, -gf);
}

// The scalar form's source operands of pair32 from the packed ones (exact).
__device__ __forceinline__ void disk_unpack_source(const float4 px, const float4 py, float4 &sf,
                                                   float4 &si) {
    sf = make_float4(-px.x, py.x, -px.z, py.z);
    si = make_float4(-px.y, py.y, -px.w, py.w);
}

__device__ __forceinline__ float2 disk_r2_x2(const DiskTarget2 &t, const float4 px,
                                             const float4 py, float2 &dx, float2 &dyn) {
    dx = __fadd2_rn(__fadd2_rn(t.xh, make_float2(px.x, px.y)),
                    __fadd2_rn(t.xl, make_float2(px.z, px.w)));
    dyn = __fadd2_rn(__fadd2_rn(make_float2(py.x, py.y), t.nyh),
                     __fadd2_rn(make_float2(py.z, py.w), t.nyl));
    return __ffma2_rn(dx, dx, __fmul2_rn(dyn, dyn));
}

// closest: the smallest squared distance of either term met so far, for the caller's near-field
// listing after a block of sources (disk_list_near_x2), so that the pair loop has no branch.
__device__ __forceinline__ void disk_pair_x2(const F32Geometry &f, const DiskTarget2 &t,
                                             const float4 px, const float4 py, const float2 g2,
                                             float2 &u2, float2 &v2, float &closest) {
    float2 dx, dyn;
    const float2 r2 = disk_r2_x2(t, px, py, dx, dyn);
    const float inf = __int_as_float(0x7f800000);
    const float2 c = __fmul2_rn(g2, make_float2(rcp_approx_f32(r2.x < f.near2 ? inf : r2.x),
                                                rcp_approx_f32(r2.y < f.near2 ? inf : r2.y)));
    u2 = __ffma2_rn(c, dyn, u2);
    v2 = __ffma2_rn(c, dx, v2);
    closest = fminf(closest, fminf(r2.x, r2.y));
}

// Lists the near terms that disk_pair_x2 left out among the staged sources [jb, je) (source
// index j0 + j), for every lane whose `flagged` is set, the whole warp at a time: the flagged
// target is broadcast and each lane recomputes the squared distances (the same operations, so
// the same decisions) of every 32nd source. Near terms are rare (a dozen per target at the default
// radius), so this runs for few blocks; all 32 lanes must be present.
__device__ __forceinline__ void disk_list_near_x2(const F32Geometry &f, const NearLists &lists,
                                                  const DiskTarget2 &t, size_t ti, bool flagged,
                                                  const float4 *spx, const float4 *spy, int jb,
                                                  int je, size_t j0) {
    unsigned todo = __ballot_sync(0xffffffffu, flagged);
    const int lane = threadIdx.x & 31;
    while (todo) {
        const int l = __ffs(todo) - 1;
        todo &= todo - 1;
        DiskTarget2 tl;
        tl.xh.x = tl.xh.y = __shfl_sync(0xffffffffu, t.xh.x, l);
        tl.xl.x = tl.xl.y = __shfl_sync(0xffffffffu, t.xl.x, l);
        tl.nyh.x = tl.nyh.y = __shfl_sync(0xffffffffu, t.nyh.x, l);
        tl.nyl.x = tl.nyl.y = __shfl_sync(0xffffffffu, t.nyl.x, l);
        const size_t target = __shfl_sync(0xffffffffu, ti, l);
        for (int j = jb + lane; j < je; j += 32) {
            float2 dx, dyn;
            const float2 r2 = disk_r2_x2(tl, spx[j], spy[j], dx, dyn);
            if (r2.x < f.near2)
                near_append(lists, target, static_cast<unsigned>(j0 + j));
            if (r2.y < f.near2)
                near_append(lists, target, static_cast<unsigned>(j0 + j) | kNearImage);
        }
    }
}

// Lists the near terms pair32 left out, under target ti and source j.
__device__ __forceinline__ void list_near(const NearLists &lists, bool near_pair, bool near_wall,
                                          size_t ti, unsigned j) {
    if (near_pair)
        near_append(lists, ti, j);
    if (near_wall)
        near_append(lists, ti, j | kNearImage);
}

}  // namespace f32
}  // namespace pvb
