// pv_velocity32.cu — the FP32-compensated precision form of the velocity evaluation.
//
// Same tiling, TMA staging, chunk partials and slow path as pv_velocity.cu; the pair terms are
// evaluated on the FP32 pipe (128 lanes/clk/SM on B200, twice the FP64 pipe) with three
// compensations:
//
//   * coordinates as double-float pairs: every staged source and every target is split into
//     hi = fp32(x), lo = fp32(x - hi), and a displacement is (t_hi - s_hi) + (t_lo - s_lo). The
//     first difference is exact when the coordinates are close (Sterbenz) and carries the relative
//     error of one rounding otherwise, so dx keeps ~2^-24 relative accuracy at every separation,
//     which absolute FP32 coordinates cannot (their rounding is relative to |x|, not |dx|);
//   * FP32 partial sums over 64 sources are promoted into FP64 accumulators, so the summation error
//     does not grow with N;
//   * the disk image term falls back to FP64 where 1 - t.s/R^2 < 1/8 (target and source near the
//     wall and aligned), where the FP32 form would cancel. The periodic m = 0 denominator
//     2 (sinh^2(x^/2) + sin^2(y^/2)) and every m != 0 term have no cancellation, so the periodic
//     series stays in FP32 throughout.
//
// What remains is the FP32 rounding of each pair term (a few ulp, ~1e-7 relative); the velocity
// error against the FP64 oracle is that, summed over sources (reported by the parity tests).
#include "pv_internal.h"

#include <algorithm>

namespace pvb {

namespace {
constexpr int kTile32 = 256;
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

template <int GEO, int B, int T>
__global__ void __launch_bounds__(B) velocity32_kernel(const EvalArgs a) {
    __shared__ alignas(128) double s_x[2][kTile32];
    __shared__ alignas(128) double s_y[2][kTile32];
    __shared__ alignas(128) double s_g[2][kTile32];
    __shared__ alignas(16) float4 s_f[kTile32];
    __shared__ float s_gf[kTile32];
    __shared__ alignas(8) uint64_t bars[2];
    __shared__ int s_status;

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
        const bool ok = mbar_wait_bounded(&bars[st], static_cast<uint32_t>((t >> 1) & 1), a.status);
        if (__syncthreads_or(!ok))
            return;
        const size_t j0 = src0 + static_cast<size_t>(t) * kTile32;
        const int cnt = static_cast<int>(min(static_cast<size_t>(kTile32), src1 - j0));
        // split the tile into double-float FP32 coordinates once per CTA
        for (int j = tid; j < cnt; j += B) {
            const double xj = s_x[st][j], yj = s_y[st][j];
            const float xh = static_cast<float>(xj), yh = static_cast<float>(yj);
            s_f[j] = make_float4(xh, yh, static_cast<float>(xj - static_cast<double>(xh)),
                                 static_cast<float>(yj - static_cast<double>(yh)));
            s_gf[j] = static_cast<float>(s_g[st][j]);
        }
        __syncthreads();
        const bool diagonal = j0 < blk1 && blk0 < j0 + cnt;
        for (int jb = 0; jb < cnt; jb += kFlush) {
            const int je = min(cnt, jb + kFlush);
            if (diagonal) {
#pragma unroll 1
                for (int j = jb; j < je; ++j) {
                    const float4 sf = s_f[j];
                    const float gf = s_gf[j];
#pragma unroll
                    for (int k = 0; k < T; ++k)
                        pair32<GEO, true>(f, a.g, tg[k], sf, gf, s_x[st][j], s_y[st][j], s_g[st][j],
                                          ti[k] == j0 + j, u[k], v[k], ud[k], vd[k]);
                }
            } else {
#pragma unroll 2
                for (int j = jb; j < je; ++j) {
                    const float4 sf = s_f[j];
                    const float gf = s_gf[j];
#pragma unroll
                    for (int k = 0; k < T; ++k)
                        pair32<GEO, false>(f, a.g, tg[k], sf, gf, s_x[st][j], s_y[st][j],
                                           s_g[st][j], false, u[k], v[k], ud[k], vd[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < T; ++k) {
                ud[k] += static_cast<double>(u[k]);
                vd[k] += static_cast<double>(v[k]);
                u[k] = v[k] = 0.0f;
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

template <int GEO, int T> cudaError_t launch32_t(const EvalArgs &a, const EvalPlan &p, cudaStream_t s) {
    velocity32_kernel<GEO, 128, T><<<static_cast<unsigned>(p.items()), 128, 0, s>>>(a);
    return cudaGetLastError();
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
