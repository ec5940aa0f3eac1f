// pv_pair32.cuh — FP32-compensated pair terms, shared by the single-simulation kernel
// (pv_velocity32.cu) and the batched ensembles (pv_batch.cu).
//
// Coordinates enter as double-float pairs (hi = fp32(x), lo = fp32(x - hi)), so a displacement
// (t_hi - s_hi) + (t_lo - s_lo) keeps ~2^-24 relative accuracy at every separation. The periodic
// series and the direct Biot-Savart term run on the FP32 pipe; the disk image term falls back to
// FP64 where 1 - t.s/R^2 < 1/8. Callers promote FP32 partial sums into FP64 every kFlush sources.
#pragma once

#include "pv_common.cuh"
#include "pv_geometry.cuh"

namespace pvb {
namespace f32 {

constexpr int kFlush = 64; // sources summed in FP32 before promotion to FP64

__device__ __forceinline__ float rcp_approx_f32(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

struct F32Geometry { // the FP32 constants of one evaluation
    float eps2;
    float l_hi, l_lo, inv_l, half_wave;
    float two_cosh_m[3], cosh_m[3], sinh2_m[3];
    float k1, k2, k6, shift6;
    int m_exact, has6;
    float inv_radius2;
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
    f.k1 = static_cast<float>(g.k1);
    f.k2 = static_cast<float>(g.k2);
    f.k6 = static_cast<float>(g.k6);
    f.shift6 = static_cast<float>(0.5 * g.shift6);
    f.m_exact = g.m_exact;
    f.has6 = g.has6;
    f.inv_radius2 = static_cast<float>(g.inv_radius2);
    return f;
}

// sinh, cosh, sin, cos of t (|t| <= pi/2), the FP32 truncation of the shared series in
// pv_common.cuh (first omitted term below 1e-8 relative).
__device__ __forceinline__ void shcs_f32(float t, float &sh, float &ch, float &s, float &c) {
    const float t2 = t * t, w = t2 * t2;
    float e1 = fmaf(w, 1.6059043836821613e-10f, 2.7557319223985893e-06f); // 1/13!, 1/9!
    e1 = fmaf(w, e1, 8.333333333333333e-03f);
    e1 = fmaf(w, e1, 1.0f);
    float o1 = fmaf(w, 2.505210838544172e-08f, 1.984126984126984e-04f); // 1/11!, 1/7!
    o1 = fmaf(w, o1, 1.6666666666666666e-01f);
    float e0 = fmaf(w, 2.08767569878681e-09f, 2.48015873015873e-05f); // 1/12!, 1/8!
    e0 = fmaf(w, e0, 4.1666666666666664e-02f);
    e0 = fmaf(w, e0, 1.0f);
    float o0 = fmaf(w, 1.1470745597729725e-11f, 2.755731922398589e-07f); // 1/14!, 1/10!
    o0 = fmaf(w, o0, 1.388888888888889e-03f);
    o0 = fmaf(w, o0, 0.5f);
    const float t3 = t * t2, te1 = t * e1;
    sh = fmaf(t3, o1, te1);
    s = fmaf(-t3, o1, te1);
    ch = fmaf(t2, o0, e0);
    c = fmaf(-t2, o0, e0);
}

// Half of x^ = (2 pi/L) remainder(dx, L) in FP32 from a double-float displacement.
__device__ __forceinline__ float half_angle_f32(const F32Geometry &f, float dx) {
    const float n = rintf(dx * f.inv_l);
    const float r = fmaf(-n, f.l_lo, fmaf(-n, f.l_hi, dx));
    return f.half_wave * r;
}

__device__ __forceinline__ void image_sum_f32(const F32Geometry &f, float half_hat, float ch,
                                              float sh, float c, float &num, float &den,
                                              float &rest) {
    const float ch2 = ch * ch;
    const float p = fmaf(c, c, ch2);
    const float q = -2.0f * c * ch;
    const float m2c = -2.0f * c;
    num = 0.0f;
    den = 1.0f;
#pragma unroll
    for (int m = 1; m <= 2; ++m) {
        if (m <= f.m_exact) {
            const float pn = fmaf(ch, f.two_cosh_m[m], m2c);
            const float pd = fmaf(q, f.cosh_m[m], p + f.sinh2_m[m]);
            num = fmaf(pn, den, num * pd);
            den *= pd;
        }
    }
    const float ch2x = fmaf(2.0f, ch2, -1.0f);
    rest = fmaf(ch, f.k1, c * ch2x * f.k2);
    if (f.has6) { // |x^ -+ 12 pi| <= 40  <=>  |x^/2 -+ 6 pi| <= 20
        const bool plus = fabsf(half_hat - f.shift6) <= 20.0f;
        const bool minus = fabsf(half_hat + f.shift6) <= 20.0f;
        const float e = (plus ? ch + sh : 0.0f) + (minus ? ch - sh : 0.0f);
        rest = fmaf(f.k6, e, rest);
    }
}

struct Target32 {
    float xh, xl, yh, yl;
    double x, y;
};

// The periodic pair's terms without its circulation, in FP32: the target's velocity changes by
// u -= g_s ku, v += g_s kv. t and s are (x_hi, y_hi, x_lo, y_lo). Exchanging target and source
// negates the displacement exactly, and every quantity below is an exactly odd or even function
// of it, so ku and kv are exactly odd: the symmetric kernels use one evaluation for both.
__device__ __forceinline__ void periodic_values32(const F32Geometry &f, const float4 t,
                                                  const float4 s, float &ku, float &kv) {
    const float dx = (t.x - s.x) + (t.z - s.z);
    const float dy = (t.y - s.y) + (t.w - s.w);
    const float hx = half_angle_f32(f, dx), hy = half_angle_f32(f, dy);
    float shx, chx, snx, csx, shy, chy, sny, csy;
    shcs_f32(hx, shx, chx, snx, csx);
    shcs_f32(hy, shy, chy, sny, csy);
    const float cosh_x = fmaf(2.0f * shx, shx, 1.0f), cosh_y = fmaf(2.0f * shy, shy, 1.0f);
    const float cos_x = fmaf(-2.0f * snx, snx, 1.0f), cos_y = fmaf(-2.0f * sny, sny, 1.0f);
    const float sin_x = 2.0f * snx * csx, sin_y = 2.0f * sny * csy;
    const float sinh_x = 2.0f * shx * chx, sinh_y = 2.0f * shy * chy;
    const float d0u = 2.0f * fmaf(shx, shx, sny * sny);
    const float d0v = 2.0f * fmaf(shy, shy, snx * snx);
    float nu, du, ru, nv, dv, rv;
    image_sum_f32(f, hx, cosh_x, sinh_x, cos_y, nu, du, ru);
    image_sum_f32(f, hy, cosh_y, sinh_y, cos_x, nv, dv, rv);
    ku = sin_y * fmaf(d0u, fmaf(du, ru, nu), du) * rcp_approx_f32(d0u * du);
    kv = sin_x * fmaf(d0v, fmaf(dv, rv, nv), dv) * rcp_approx_f32(d0v * dv);
}

// The plane's kernel values in FP32: K = (dy, dx) / (r^2 + eps^2) from the double-float
// displacement. Exactly odd under exchanging target and source, as periodic_values32.
__device__ __forceinline__ void plane_values32(const F32Geometry &f, const float4 t,
                                               const float4 s, float &ku, float &kv) {
    const float dx = (t.x - s.x) + (t.z - s.z);
    const float dy = (t.y - s.y) + (t.w - s.w);
    const float inv = rcp_approx_f32(fmaf(dx, dx, fmaf(dy, dy, f.eps2)));
    ku = dy * inv;
    kv = dx * inv;
}

// The pair kernels of the FP32 symmetric tiles (circulations enter unscaled).
struct Periodic32 {
    __device__ __forceinline__ static void values(const F32Geometry &f, const float4 t,
                                                  const float4 s, float &ku, float &kv) {
        periodic_values32(f, t, s, ku, kv);
    }
};
struct Plane32 {
    __device__ __forceinline__ static void values(const F32Geometry &f, const float4 t,
                                                  const float4 s, float &ku, float &kv) {
        plane_values32(f, t, s, ku, kv);
    }
};

template <int GEO, bool CHECK>
__device__ __forceinline__ void pair32(const F32Geometry &f, const GeometryConsts &g,
                                       const Target32 &t, const float4 s, float sgf, double sxd,
                                       double syd, double sgd, bool self, float &u, float &v,
                                       double &ud, double &vd) {
    const float dx = (t.xh - s.x) + (t.xl - s.z);
    const float dy = (t.yh - s.y) + (t.yl - s.w);
    if (GEO == GEO_PERIODIC) {
        const float hx = half_angle_f32(f, dx), hy = half_angle_f32(f, dy);
        float shx, chx, snx, csx, shy, chy, sny, csy;
        shcs_f32(hx, shx, chx, snx, csx);
        shcs_f32(hy, shy, chy, sny, csy);
        const float cosh_x = fmaf(2.0f * shx, shx, 1.0f), cosh_y = fmaf(2.0f * shy, shy, 1.0f);
        const float cos_x = fmaf(-2.0f * snx, snx, 1.0f), cos_y = fmaf(-2.0f * sny, sny, 1.0f);
        const float sin_x = 2.0f * snx * csx, sin_y = 2.0f * sny * csy;
        const float sinh_x = 2.0f * shx * chx, sinh_y = 2.0f * shy * chy;
        float d0u = 2.0f * fmaf(shx, shx, sny * sny);
        float d0v = 2.0f * fmaf(shy, shy, snx * snx);
        if (CHECK && self) {
            d0u = 1.0f;
            d0v = 1.0f;
        }
        float nu, du, ru, nv, dv, rv;
        image_sum_f32(f, hx, cosh_x, sinh_x, cos_y, nu, du, ru);
        image_sum_f32(f, hy, cosh_y, sinh_y, cos_x, nv, dv, rv);
        const float numer_u = fmaf(d0u, fmaf(du, ru, nu), du);
        const float numer_v = fmaf(d0v, fmaf(dv, rv, nv), dv);
        float cu = sgf * sin_y * numer_u, cv = sgf * sin_x * numer_v;
        if (CHECK && self) {
            cu = 0.0f;
            cv = 0.0f;
        }
        u = fmaf(-cu, rcp_approx_f32(d0u * du), u);
        v = fmaf(cv, rcp_approx_f32(d0v * dv), v);
        return;
    }
    // direct Biot–Savart term (plane, and the disk's j != i term)
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, GEO == GEO_INFINITE ? f.eps2 : 0.0f));
    float c = sgf * rcp_approx_f32(r2);
    if (CHECK && self)
        c = 0.0f;
    u = fmaf(-c, dy, u);
    v = fmaf(c, dx, v);
    if (GEO == GEO_DISK) {
        const float px = (t.xh + t.xl) * f.inv_radius2, py = (t.yh + t.yl) * f.inv_radius2;
        const float sx = s.x + s.z, sy = s.y + s.w;
        const float a = fmaf(-px, sx, fmaf(-py, sy, 1.0f));
        if (a >= 0.125f) {
            const float b = fmaf(py, sx, -px * sy);
            const float ci = (sgf * f.inv_radius2) * rcp_approx_f32(fmaf(a, a, b * b));
            u = fmaf(ci, fmaf(b, sx, -a * sy), u);
            v = fmaf(ci, fmaf(a, sx, b * sy), v);
        } else { // near the wall: the FP64 image term of DiskPair
            const double pxd = t.x * g.inv_radius2, pyd = t.y * g.inv_radius2;
            const double ad = fma(-pxd, sxd, fma(-pyd, syd, 1.0));
            const double bd = fma(pyd, sxd, -pxd * syd);
            const double cid = (sgd * g.inv_radius2) * rcp_refined(fma(ad, ad, bd * bd));
            ud = fma(cid, fma(bd, sxd, -ad * syd), ud);
            vd = fma(cid, fma(ad, sxd, bd * syd), vd);
        }
    }
}

}  // namespace f32
}  // namespace pvb
