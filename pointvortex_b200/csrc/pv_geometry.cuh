// pv_geometry.cuh — the three Biot–Savart pair interactions of PointVortex, FP64.
//
// Each geometry provides
//   * a per-source record staged in shared memory (x, y, and a scaled circulation),
//   * pair<CHECK>(): the fast form used by the tiled kernels, which adds one source's
//     contribution to one target's (u, v); CHECK enables the self-pair test and is only
//     instantiated for the diagonal tiles,
//   * slow_target(): the reference form with IEEE divisions and the reference's singular-pair
//     test, used to recompute a target whose fast-path sum came out non-finite. It returns the
//     reference's verdict (coincident pair / non-finite / finite).
#pragma once

#include "pv_common.cuh"

namespace pvb {

constexpr double kPi = 3.141592653589793;            // std::numbers::pi
constexpr double kInverseTwoPi = 0.5 / 3.141592653589793;

enum GeometryId : int { GEO_INFINITE = 0, GEO_PERIODIC = 1, GEO_DISK = 2 };

// Constants of one simulation, passed by value to every kernel (kernel parameter space).
struct GeometryConsts {
    int geometry;
    int image_layers;
    // infinite plane
    double eps2;            // coreRadius^2
    // periodic box (Weiss–McWilliams)
    double lx, ly;          // box lengths (square within 1e-13)
    double inv_lx, inv_ly;  // 1/L
    double half_lx, half_ly;
    double wave;            // 2 pi / Lx
    double half_wave;       // pi / Lx (exactly wave / 2)
    double scale;           // 0.5 / Lx
    int m_exact;            // image pairs m = +-1..m_exact summed exactly (min(M, 2))
    double cosh_m[3];       // cosh(2 pi m), m = 0..2
    double two_cosh_m[3];   // 2 cosh(2 pi m)
    double sinh2_m[3];      // sinh(2 pi m)^2
    double k1, k2;          // 2 sum sech(2 pi m), 2 sum sech^2(2 pi m) over m = 3..min(M, 6)
    // disk
    double radius, radius2, inv_radius, inv_radius2;
    // FP32-compensated form: near-field radius squared (0: none), pv_pair32.cuh
    double near2;
};

// Scaled circulation stored per source, chosen so that each pair needs one multiply by it:
// infinite plane and disk Gamma/(2 pi) (the reference's inverseTwoPi * Gamma), periodic box
// Gamma * 0.5/L (the reference's scale * Gamma).
__host__ __device__ __forceinline__ double scaled_circulation(const GeometryConsts &g, double gamma) {
    if (g.geometry == GEO_PERIODIC)
        return g.scale * gamma;
    return kInverseTwoPi * gamma;
}

// ---------------------------------------------------------------------------------------------
// Infinite plane, src/compute.cpp:88-133: u -= (G/2pi) dy/(r^2+eps^2), v += (G/2pi) dx/(r^2+eps^2).
struct InfinitePair {
    template <bool CHECK>
    __device__ __forceinline__ static void pair(const GeometryConsts &g, double tx, double ty,
                                                double sx, double sy, double sg, bool self,
                                                double &u, double &v) {
        const double dx = tx - sx;
        const double dy = ty - sy;
        const double r2 = fma(dx, dx, fma(dy, dy, g.eps2));
        double c = sg * rcp_refined(r2);
        if (CHECK && self)
            c = 0.0;
        u = fma(-c, dy, u);
        v = fma(c, dx, v);
    }
};

// Disk of radius R, src/compute.cpp:286-336, with the source record of the infinite plane
// (x, y, G/(2 pi)). With p = z_i/R^2 and k = G/(2 pi):
//   direct (j != i):  u -= k dy/r^2,  v += k dx/r^2                 (dx = x_i - x_j, ...)
//   image (all j):    a = 1 - p.z_j, b = p_y x_j - p_x y_j,
//                     u += (k/R^2) (b x_j - a y_j)/(a^2 + b^2),  v += (k/R^2) (a x_j + b y_j)/(a^2 + b^2)
// which is the reference's circle-theorem image term written in unscaled source coordinates.
struct DiskPair {
    template <bool CHECK>
    __device__ __forceinline__ static void pair(const GeometryConsts &g, double tx, double ty,
                                                double sx, double sy, double sg, bool self,
                                                double &u, double &v) {
        const double dx = tx - sx;
        const double dy = ty - sy;
        const double r2 = fma(dx, dx, dy * dy);
        double c = sg * rcp_refined(r2);
        if (CHECK && self)
            c = 0.0;
        u = fma(-c, dy, u);
        v = fma(c, dx, v);
        image(g, tx, ty, sx, sy, sg, u, v);
    }
    // The direct term alone (j != i).
    __device__ __forceinline__ static void direct(double tx, double ty, double sx, double sy,
                                                  double sg, double &u, double &v) {
        const double dx = tx - sx;
        const double dy = ty - sy;
        const double c = sg * rcp_refined(fma(dx, dx, dy * dy));
        u = fma(-c, dy, u);
        v = fma(c, dx, v);
    }
    // The image term alone (every j, j == i included).
    __device__ __forceinline__ static void image(const GeometryConsts &g, double tx, double ty,
                                                 double sx, double sy, double sg, double &u,
                                                 double &v) {
        const double px = tx * g.inv_radius2, py = ty * g.inv_radius2;
        const double a = fma(-px, sx, fma(-py, sy, 1.0));
        const double b = fma(py, sx, -px * sy);
        const double ci = (sg * g.inv_radius2) * rcp_refined(fma(a, a, b * b));
        u = fma(ci, fma(b, sx, -a * sy), u);
        v = fma(ci, fma(a, sx, b * sy), v);
    }
};

// Periodic square box, src/compute.cpp:203-256 (Weiss–McWilliams image sum, truncated at
// |m| <= M with the reference's rule that an image whose |shift| exceeds 40 contributes 0).
//
// With x^ = (2 pi/L) remainder(dx, L), y^ likewise, the reference adds per source
//   u -= k sin(y^) sum_m 1/D_u(m),  D_u(m) = 2 (sinh^2((x^ - 2 pi m)/2) + sin^2(y^/2)),
//   v += k sin(x^) sum_m 1/D_v(m),  D_v(m) = 2 (sinh^2((y^ - 2 pi m)/2) + sin^2(x^/2)).
// The same truncated sum is evaluated here with one reciprocal per axis. With C = cosh x^,
// c = cos y^, a = 2 pi m, A = cosh a, D(m) = cosh(x^ - a) - c:
//   * m = 0 keeps the cancellation-free form 2 (sinh^2(x^/2) + sin^2(y^/2));
//   * m = +-1, +-2 (never dropped, since |x^| <= pi) combine exactly in pairs,
//       D(m) + D(-m) = 2 (C A - c),   D(m) D(-m) = C^2 + c^2 - 2 c C A + sinh^2 a,
//     where every term of the product is far from cancelling (sinh^2 a >= 7e4 > 2 |c| C A);
//   * m = +-3..+-6: with u = sech a <= 1.3e-8 the pair sum is
//       2u C + 2u^2 c cosh 2x^ + O(u^3 C^3),
//     and the omitted terms are below 1e-19 of the m = 0 term, far under FP64 rounding;
//   * the reference keeps an m = +-6 image only where |x^ -+ 12 pi| <= 40, so for |x^| > 2.3 it
//     drops one of the pair: a term of at most 2 e^{-12 pi} e^{-2.3} ~ 9e-18, below 1.2e-16 of the
//     sum (whose m = 0 part alone is at least 0.079). Both are kept here, which spares the
//     window test and sinh x^: the difference is at the level of the sum's own rounding;
//   * |m| >= 7 always has |shift| > 40 and is dropped, as in the reference.
// sinh, cosh, sin and cos of x^/2 and y^/2 come from one shared series (|x^/2| <= pi/2).
struct PeriodicPair {
    // Images m != 0 of one axis as num/den + rest: C = cosh of the axis, c = cos of the other.
    __device__ __forceinline__ static void image_sum(const GeometryConsts &g, double ch, double c,
                                                     double &num, double &den, double &rest) {
        const double ch2 = ch * ch;
        const double p = fma(c, c, ch2);   // C^2 + c^2
        const double m2c = -2.0 * c;
        const double q = m2c * ch;         // -2 c C
        // m = 1 starts the fraction, m = 2 joins it: num/den = pn1/pd1 + pn2/pd2
        num = 0.0;
        den = 1.0;
        if (g.m_exact >= 1) {
            num = fma(ch, g.two_cosh_m[1], m2c);
            den = fma(q, g.cosh_m[1], p + g.sinh2_m[1]);
        }
        if (g.m_exact >= 2) {
            const double pair_num = fma(ch, g.two_cosh_m[2], m2c);
            const double pair_den = fma(q, g.cosh_m[2], p + g.sinh2_m[2]);
            num = fma(pair_num, den, num * pair_den);
            den *= pair_den;
        }
        // m = 3..6: 2u C + 2u^2 c cosh 2x^ summed over u = sech(2 pi m), with
        // k2 cosh 2x^ = k2 (2 C^2 - 1) as one fma
        rest = fma(ch, g.k1, c * fma(2.0 * g.k2, ch2, -g.k2));
    }

    // The pair's terms without its circulation: the target's velocity changes by
    // u -= g_s * au / bu, v += g_s * av / bv. Exchanging target and source negates x^ and y^
    // exactly (remainder is odd), which negates au and av and leaves bu and bv unchanged, bit for
    // bit: every quantity below is an exactly odd or even function of (x^, y^).
    // HALF_SINE: au and av carry sin(y^)/2 and sin(x^)/2 (exactly half: the caller doubles the
    // circulation instead, which saves two multiplies per pair and changes no bit of the sums).
    template <bool HALF_SINE = false>
    __device__ __forceinline__ static void terms(const GeometryConsts &g, double tx, double ty,
                                                 double sx, double sy, double &au, double &bu,
                                                 double &av, double &bv) {
        // x^/2 and y^/2: pi/L times the remainder is exactly half of (2 pi/L) times it
        const double hx = g.half_wave * exact_remainder(tx - sx, g.lx, g.inv_lx, g.half_lx);
        const double hy = g.half_wave * exact_remainder(ty - sy, g.ly, g.inv_ly, g.half_ly);
        double shx, chx, snx, csx, shy, chy, sny, csy;
        sinh_cosh_sin_cos_economized(hx, shx, chx, snx, csx);
        sinh_cosh_sin_cos_economized(hy, shy, chy, sny, csy);
        const double tshx = 2.0 * shx, tshy = 2.0 * shy;    // scaling by 2 is exact
        const double nsnx = -2.0 * snx, nsny = -2.0 * sny;
        const double cosh_x = fma(tshx, shx, 1.0); // cosh x^ = 1 + 2 sinh^2(x^/2)
        const double cosh_y = fma(tshy, shy, 1.0);
        const double cos_x = fma(nsnx, snx, 1.0);  // cos x^ = 1 - 2 sin^2(x^/2)
        const double cos_y = fma(nsny, sny, 1.0);
        const double sin_x = HALF_SINE ? snx * csx : 2.0 * snx * csx; // sin x^ (or half)
        const double sin_y = HALF_SINE ? sny * csy : 2.0 * sny * csy;
        // 2 (sinh^2(x^/2) + sin^2(y^/2)) with the factor 2 inside: the same rounding, bit for bit
        const double d0u = fma(tshx, shx, -(nsny * sny));
        const double d0v = fma(tshy, shy, -(nsnx * snx));
        double nu, du, ru, nv, dv, rv;
        image_sum(g, cosh_x, cos_y, nu, du, ru);
        image_sum(g, cosh_y, cos_x, nv, dv, rv);
        // 1/d0 + num/den + rest = (den + d0 (num + den rest)) / (d0 den)
        au = sin_y * fma(d0u, fma(du, ru, nu), du);
        av = sin_x * fma(d0v, fma(dv, rv, nv), dv);
        bu = d0u * du;
        bv = d0v * dv;
    }

    template <bool CHECK>
    __device__ __forceinline__ static void pair(const GeometryConsts &g, double tx, double ty,
                                                double sx, double sy, double sg, bool self,
                                                double &u, double &v) {
        if (CHECK && self) // the self pair contributes exactly 0 in the reference (sin 0 = 0)
            return;
        double au, bu, av, bv;
        terms(g, tx, ty, sx, sy, au, bu, av, bv);
        u = fma(-(sg * au), rcp_refined(bu), u);
        v = fma(sg * av, rcp_refined(bv), v);
    }
};

// ---------------------------------------------------------------------------------------------
// Reference-form recomputation of one target (IEEE divisions, library sinh/sin/remainder,
// the reference's singular-pair rule). Verdict: 0 finite, ST_COINCIDENT, ST_NONFINITE_VELOCITY.
__device__ inline int slow_target(const GeometryConsts &g, const double *x, const double *y,
                                  const double *gamma, size_t n, size_t t, double &u_out,
                                  double &v_out) {
    double u = 0.0, v = 0.0;
    int singular = 0;
    const double tx = x[t], ty = y[t];
    if (g.geometry == GEO_INFINITE) {
        for (size_t s = 0; s < n; ++s) {
            if (s == t)
                continue;
            const double dx = tx - x[s], dy = ty - y[s];
            const double den = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), g.eps2);
            if (den == 0.0) {
                singular = 1;
                continue;
            }
            const double c = __dmul_rn(kInverseTwoPi, gamma[s]) / den;
            u -= c * dy;
            v += c * dx;
        }
    } else if (g.geometry == GEO_PERIODIC) {
        const int layers = g.image_layers;
        for (size_t s = 0; s < n; ++s) {
            const double sdx = g.wave * remainder(tx - x[s], g.lx);
            const double sdy = g.wave * remainder(ty - y[s], g.ly);
            const double sine_x = sin(sdx), sine_y = sin(sdy);
            const double shx = sin(0.5 * sdx), shy = sin(0.5 * sdy);
            for (int m = -layers; m <= layers; ++m) {
                if (s == t && m == 0)
                    continue;
                const double shift = __dmul_rn(2.0 * kPi, static_cast<double>(m));
                const double ax = __dsub_rn(sdx, shift), ay = __dsub_rn(sdy, shift);
                double du, dv;
                if (fabs(ax) > 40.0) {
                    du = __longlong_as_double(0x7ff0000000000000ll);
                } else {
                    const double h = sinh(0.5 * ax);
                    du = 2.0 * __dadd_rn(__dmul_rn(h, h), __dmul_rn(shy, shy));
                }
                if (fabs(ay) > 40.0) {
                    dv = __longlong_as_double(0x7ff0000000000000ll);
                } else {
                    const double h = sinh(0.5 * ay);
                    dv = 2.0 * __dadd_rn(__dmul_rn(h, h), __dmul_rn(shx, shx));
                }
                if (du == 0.0 || dv == 0.0) {
                    singular = 1;
                    continue;
                }
                u -= __dmul_rn(__dmul_rn(g.scale, gamma[s]), sine_y) / du;
                v += __dmul_rn(__dmul_rn(g.scale, gamma[s]), sine_x) / dv;
            }
        }
    } else {
        const double ir = g.inv_radius;
        const double txs = tx * ir, tys = ty * ir;
        for (size_t s = 0; s < n; ++s) {
            if (s != t) {
                const double dx = tx - x[s], dy = ty - y[s];
                const double den = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
                if (den == 0.0) {
                    singular = 1;
                    continue;
                }
                const double c = __dmul_rn(kInverseTwoPi, gamma[s]) / den;
                u -= c * dy;
                v += c * dx;
            }
            const double sx = x[s] * ir, sy = y[s] * ir;
            const double a = 1.0 - __dadd_rn(__dmul_rn(txs, sx), __dmul_rn(tys, sy));
            const double b = __dsub_rn(__dmul_rn(tys, sx), __dmul_rn(txs, sy));
            const double den = __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b));
            const double ix = __dsub_rn(__dmul_rn(-a, sx), __dmul_rn(b, sy));
            const double iy = __dadd_rn(__dmul_rn(-a, sy), __dmul_rn(b, sx));
            const double c = __dmul_rn(__dmul_rn(-kInverseTwoPi, gamma[s]), ir) / den;
            u -= c * iy;
            v += c * ix;
        }
    }
    u_out = u;
    v_out = v;
    if (singular)
        return ST_COINCIDENT;
    if (!isfinite(u) || !isfinite(v))
        return ST_NONFINITE_VELOCITY;
    return 0;
}

} // namespace pvb
