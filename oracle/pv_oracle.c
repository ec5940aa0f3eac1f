/* pv_oracle.c — plain-C restatement of the PointVortex hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA product is compared with; the
 * product never links, loads or calls it. Every function follows the reference
 * (jplaurie/PointVortex) line by line in the order of its floating-point operations, so that
 * with the same libm it reproduces the reference bit for bit wherever the reference sums
 * sequentially (periodic and disk kernels, Hamiltonians, moments, integrators, dipole scan).
 * The infinite-plane kernel of the reference vectorises its source loop
 * (`omp simd reduction`, src/compute.cpp:111-113), so there this sequential restatement
 * agrees to rounding only.
 *
 * Parity pins: tests/test_oracle.py (against the reference compiled into oracle/_ref/) and
 * tests/test_golden.py (the reference's own known-answer tests).
 */
#include "pv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PVO_OK 0
#define PVO_INVALID 1
#define PVO_RANGE 2
#define PVO_RUNTIME 3

static const double kPi = 3.141592653589793; /* std::numbers::pi */
static _Thread_local const char *last_error = "";

const char *pvo_last_error(void) { return last_error; }

/* std::max / std::min semantics (return the first argument unless the second compares
 * greater / smaller), which differ from C fmax/fmin only for NaN and signed zeros. */
static double fmax_ref(double a, double b) { return (a < b) ? b : a; }
static double fmin_ref(double a, double b) { return (b < a) ? b : a; }

static int fail(int code, const char *message) {
    last_error = message;
    return code;
}

/* validateVortexArrays, src/vortex.h:7-14 */
static int validate_arrays(const double *x, const double *y, const double *g, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!isfinite(x[i]) || !isfinite(y[i]) || !isfinite(g[i]))
            return fail(PVO_INVALID, "vortex data must be finite");
    return PVO_OK;
}

/* validatePeriodicCirculation, src/compute.cpp:31-39 */
static int validate_periodic_circulation(const double *g, size_t n) {
    double total = 0.0, absolute_total = 0.0;
    for (size_t i = 0; i < n; ++i) {
        total += g[i];
        absolute_total += fabs(g[i]);
    }
    if (fabs(total) > 1e-12 * fmax_ref(1.0, absolute_total))
        return fail(PVO_INVALID, "periodic box requires zero total circulation");
    return PVO_OK;
}

/* validateDiskPositions, src/compute.cpp:41-48 */
static int validate_disk_positions(const double *x, const double *y, size_t n, double r2) {
    for (size_t i = 0; i < n; ++i)
        if (x[i] * x[i] + y[i] * y[i] >= r2)
            return fail(PVO_INVALID, "vortex lies on or outside the disk");
    return PVO_OK;
}

/* Kernel constructors: InfinitePlaneKernel src/compute.cpp:50-56, PeriodicBoxKernel :165-173,
 * DiskKernel :258-261. */
static int validate_kernel(const pvo_params *p) {
    if (p->geometry == 0) {
        const double r = p->core_radius, r2 = r * r;
        if (!(r >= 0.0) || !isfinite(r2) || (r > 0.0 && r2 == 0.0))
            return fail(PVO_INVALID,
                        "core radius is negative or outside the supported numeric range");
        return PVO_OK;
    }
    if (p->geometry == 1) {
        const double lx = p->box_length_x, ly = p->box_length_y;
        if (!(lx > 0.0) || !(ly > 0.0) || !isfinite(lx) || !isfinite(ly) ||
            !isfinite(2.0 * kPi / lx) || p->image_layers < 0 || p->image_layers > 64)
            return fail(PVO_INVALID, "invalid periodic-box parameters");
        if (fabs(lx - ly) > 1e-13 * fmax_ref(lx, ly))
            return fail(PVO_INVALID, "Weiss-McWilliams kernel requires a square periodic box");
        return PVO_OK;
    }
    if (p->geometry == 2) {
        const double r = p->disk_radius, r2 = r * r;
        if (!(r > 0.0) || !isfinite(r2) || r2 == 0.0)
            return fail(PVO_INVALID, "invalid disk parameters");
        return PVO_OK;
    }
    return fail(PVO_INVALID, "unsupported boundary condition");
}

/* InfinitePlaneKernel::evaluateRange, src/compute.cpp:88-133 */
static int velocity_infinite(double eps2, const double *x, const double *y, const double *g,
                             size_t n, size_t begin, size_t end, double *u, double *v) {
    const double inverse_two_pi = 0.5 / kPi;
    int singular = 0;
    for (size_t t = begin; t < end; ++t) {
        double uu = 0.0, vv = 0.0;
        for (size_t s = 0; s < n; ++s) {
            if (s == t)
                continue;
            const double dx = x[t] - x[s];
            const double dy = y[t] - y[s];
            const double den = dx * dx + dy * dy + eps2;
            if (den == 0.0) {
                singular = 1;
                continue;
            }
            const double c = inverse_two_pi * g[s] / den;
            uu -= c * dy;
            vv += c * dx;
        }
        u[t - begin] = uu;
        v[t - begin] = vv;
    }
    if (singular)
        return fail(PVO_RUNTIME, "coincident vortices in singular point-vortex kernel");
    return PVO_OK;
}

/* PeriodicBoxKernel::evaluateRange, src/compute.cpp:203-256. The denominator lambda
 * (:235-240) drops images with |shift| > 40 by returning infinity. */
static double periodic_denominator(double a, double sin_half_b) {
    if (fabs(a) > 40.0)
        return INFINITY;
    const double sh = sinh(0.5 * a);
    return 2.0 * (sh * sh + sin_half_b * sin_half_b);
}

static int velocity_periodic(const pvo_params *p, const double *x, const double *y,
                             const double *g, size_t n, size_t begin, size_t end, double *u,
                             double *v) {
    const double lx = p->box_length_x, ly = p->box_length_y;
    const int layers = p->image_layers;
    const double wave = 2.0 * kPi / lx;
    const double scale = 0.5 / lx;
    int singular = 0;
    for (size_t t = begin; t < end; ++t) {
        double uu = 0.0, vv = 0.0;
        for (size_t s = 0; s < n; ++s) {
            const double sdx = wave * remainder(x[t] - x[s], lx);
            const double sdy = wave * remainder(y[t] - y[s], ly);
            const double sine_x = sin(sdx), sine_y = sin(sdy);
            const double sin_half_x = sin(0.5 * sdx);
            const double sin_half_y = sin(0.5 * sdy);
            for (int m = -layers; m <= layers; ++m) {
                if (s == t && m == 0)
                    continue;
                const double shifted_x = sdx - 2.0 * kPi * m;
                const double shifted_y = sdy - 2.0 * kPi * m;
                const double den_u = periodic_denominator(shifted_x, sin_half_y);
                const double den_v = periodic_denominator(shifted_y, sin_half_x);
                if (den_u == 0.0 || den_v == 0.0) {
                    singular = 1;
                    continue;
                }
                uu -= scale * g[s] * sine_y / den_u;
                vv += scale * g[s] * sine_x / den_v;
            }
        }
        u[t - begin] = uu;
        v[t - begin] = vv;
    }
    if (singular)
        return fail(PVO_RUNTIME, "coincident periodic vortices");
    return PVO_OK;
}

/* DiskKernel::evaluateRange, src/compute.cpp:286-336 */
static int velocity_disk(double radius, const double *x, const double *y, const double *g,
                         size_t n, size_t begin, size_t end, double *u, double *v) {
    const double inverse_two_pi = 0.5 / kPi;
    const double inverse_radius = 1.0 / radius;
    int singular = 0;
    for (size_t t = begin; t < end; ++t) {
        double uu = 0.0, vv = 0.0;
        const double tx = x[t] * inverse_radius, ty = y[t] * inverse_radius;
        for (size_t s = 0; s < n; ++s) {
            if (s != t) {
                const double dx = x[t] - x[s];
                const double dy = y[t] - y[s];
                const double den = dx * dx + dy * dy;
                if (den == 0.0) {
                    singular = 1;
                    continue;
                }
                const double c = inverse_two_pi * g[s] / den;
                uu -= c * dy;
                vv += c * dx;
            }
            const double sx = x[s] * inverse_radius, sy = y[s] * inverse_radius;
            const double a = 1.0 - (tx * sx + ty * sy);
            const double b = ty * sx - tx * sy;
            const double den = a * a + b * b;
            const double image_x = -a * sx - b * sy;
            const double image_y = -a * sy + b * sx;
            const double c = -inverse_two_pi * g[s] * inverse_radius / den;
            uu -= c * image_y;
            vv += c * image_x;
        }
        u[t - begin] = uu;
        v[t - begin] = vv;
    }
    if (singular)
        return fail(PVO_RUNTIME, "coincident vortices in disk");
    return PVO_OK;
}

int pvo_evaluate_range(const pvo_params *p, const double *x, const double *y, const double *g,
                       size_t n, size_t begin, size_t end, double *u, double *v) {
    int rc = validate_kernel(p);
    if (rc)
        return rc;
    if ((rc = validate_arrays(x, y, g, n)))
        return rc;
    if (begin > end || end > n)
        return fail(PVO_RANGE, "invalid target-vortex range");
    if (p->geometry == 0)
        return velocity_infinite(p->core_radius * p->core_radius, x, y, g, n, begin, end, u, v);
    if (p->geometry == 1) {
        if ((rc = validate_periodic_circulation(g, n)))
            return rc;
        return velocity_periodic(p, x, y, g, n, begin, end, u, v);
    }
    if ((rc = validate_disk_positions(x, y, n, p->disk_radius * p->disk_radius)))
        return rc;
    return velocity_disk(p->disk_radius, x, y, g, n, begin, end, u, v);
}

/* VelocityKernel::evaluate, src/compute.cpp:60-69 */
int pvo_evaluate(const pvo_params *p, const double *x, const double *y, const double *g,
                 size_t n, double *u, double *v) {
    const int rc = pvo_evaluate_range(p, x, y, g, n, 0, n, u, v);
    if (rc)
        return rc;
    for (size_t i = 0; i < n; ++i)
        if (!isfinite(u[i]) || !isfinite(v[i]))
            return fail(PVO_RUNTIME, "non-finite velocity; check scales and close encounters");
    return PVO_OK;
}

/* computeMoments, src/compute.cpp:11-27 */
static int moments(const double *x, const double *y, const double *g, size_t n, double *out) {
    int rc = validate_arrays(x, y, g, n);
    if (rc)
        return rc;
    double c = 0.0, ix = 0.0, iy = 0.0, l = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double gamma = g[i];
        c += gamma;
        ix += gamma * x[i];
        iy += gamma * y[i];
        l += gamma * (x[i] * x[i] + y[i] * y[i]);
    }
    out[0] = c;
    out[1] = ix;
    out[2] = iy;
    out[3] = l;
    for (int k = 0; k < 4; ++k)
        if (!isfinite(out[k]))
            return fail(PVO_RUNTIME, "non-finite vortex moment; check input scales");
    return PVO_OK;
}

/* computeInvariants(vortices, coreRadius) Hamiltonian part, src/compute.cpp:134-156 */
static int hamiltonian_infinite(double core_radius, const double *x, const double *y,
                                const double *g, size_t n, double *out) {
    if (!(core_radius >= 0.0) || !isfinite(core_radius) || !isfinite(core_radius * core_radius) ||
        (core_radius > 0.0 && core_radius * core_radius == 0.0))
        return fail(PVO_INVALID, "core radius is negative or outside the supported numeric range");
    double m[4];
    int rc = moments(x, y, g, n, m);
    if (rc)
        return rc;
    const double eps2 = core_radius * core_radius;
    double h = 0.0;
    for (size_t i = 0; i < n; ++i)
        for (size_t j = i + 1; j < n; ++j) {
            const double dx = x[i] - x[j];
            const double dy = y[i] - y[j];
            const double r2 = dx * dx + dy * dy + eps2;
            if (r2 == 0.0)
                return fail(PVO_RUNTIME, "coincident vortices");
            h -= g[i] * g[j] * log(r2) / (4.0 * kPi);
        }
    if (!isfinite(h))
        return fail(PVO_RUNTIME, "non-finite Hamiltonian; check input scales");
    *out = h;
    return PVO_OK;
}

/* PeriodicBoxKernel::hamiltonian, src/compute.cpp:174-202 */
static double log_cosh(double a) {
    const double magnitude = fabs(a);
    return magnitude + log1p(exp(-2.0 * magnitude)) - log(2.0);
}

static int hamiltonian_periodic(const pvo_params *p, const double *x, const double *y,
                                const double *g, size_t n, double *out) {
    int rc = validate_arrays(x, y, g, n);
    if (rc)
        return rc;
    const double lx = p->box_length_x, ly = p->box_length_y;
    const int layers = p->image_layers;
    const double wave = 2.0 * kPi / lx;
    double value = 0.0;
    for (size_t i = 0; i < n; ++i)
        for (size_t j = i + 1; j < n; ++j) {
            const double dx = wave * remainder(x[i] - x[j], lx);
            const double dy = wave * remainder(y[i] - y[j], ly);
            double pair = -dx * dx / (2.0 * kPi);
            for (int m = -layers; m <= layers; ++m) {
                const double shifted = dx - 2.0 * kPi * m;
                const double sh = sinh(0.5 * shifted);
                const double sn = sin(0.5 * dy);
                const double den = 2.0 * (sh * sh + sn * sn);
                if (den == 0.0)
                    return fail(PVO_RUNTIME, "coincident periodic vortices");
                pair += log(den) - log_cosh(2.0 * kPi * m);
            }
            value -= g[i] * g[j] * pair / (4.0 * kPi);
        }
    *out = value;
    return PVO_OK;
}

/* DiskKernel::hamiltonian, src/compute.cpp:262-285 */
static int hamiltonian_disk(double radius, const double *x, const double *y, const double *g,
                            size_t n, double *out) {
    int rc = validate_arrays(x, y, g, n);
    if (rc)
        return rc;
    const double r2 = radius * radius;
    double value = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double ri2 = x[i] * x[i] + y[i] * y[i];
        if (ri2 >= r2)
            return fail(PVO_INVALID, "vortex outside disk");
        value += g[i] * g[i] * log((r2 - ri2) / radius) / (4.0 * kPi);
        for (size_t j = i + 1; j < n; ++j) {
            const double dx = x[i] - x[j], dy = y[i] - y[j];
            const double num = (dx * dx + dy * dy) * r2;
            const double dot = x[i] * x[j] + y[i] * y[j];
            const double cross = y[i] * x[j] - x[i] * y[j];
            const double den = (r2 - dot) * (r2 - dot) + cross * cross;
            if (num == 0.0)
                return fail(PVO_RUNTIME, "coincident vortices in disk");
            value -= g[i] * g[j] * log(num / den) / (4.0 * kPi);
        }
    }
    *out = value;
    return PVO_OK;
}

/* VelocityKernel::hamiltonian for the three kernels. InfinitePlaneKernel::hamiltonian
 * (src/compute.cpp:85-87) recovers the core radius as sqrt(coreRadius^2). */
int pvo_hamiltonian(const pvo_params *p, const double *x, const double *y, const double *g,
                    size_t n, double *out) {
    int rc = validate_kernel(p);
    if (rc)
        return rc;
    if (p->geometry == 0)
        return hamiltonian_infinite(sqrt(p->core_radius * p->core_radius), x, y, g, n, out);
    if (p->geometry == 1)
        return hamiltonian_periodic(p, x, y, g, n, out);
    return hamiltonian_disk(p->disk_radius, x, y, g, n, out);
}

/* computeInvariants(vortices, kernel), src/compute.cpp:157-163 */
int pvo_invariants(const pvo_params *p, const double *x, const double *y, const double *g,
                   size_t n, double *out5) {
    int rc = moments(x, y, g, n, out5);
    if (rc)
        return rc;
    if ((rc = pvo_hamiltonian(p, x, y, g, n, &out5[4])))
        return rc;
    if (!isfinite(out5[4]))
        return fail(PVO_RUNTIME, "non-finite Hamiltonian; check input scales");
    return PVO_OK;
}

/* ---------------------------------------------------------------------------------------
 * RungeKuttaIntegrator, src/timestep.h:18-34 and src/timestep.cpp.
 */
struct pvo_stepper {
    pvo_params params;
    size_t n;
    double *x0, *y0, *xt, *yt;
    double *kx[7], *ky[7];
    int fsal_valid;
    size_t evaluations;
};

/* Butcher rows, src/timestep.h:8-15 */
static const double kDopri[7][7] = {
    {0},
    {1.0 / 5.0},
    {3.0 / 40.0, 9.0 / 40.0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0},
    {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
/* src/timestep.cpp:69-73 */
static const double kB5[7] = {35.0 / 384.0,     0.0, 500.0 / 1113.0, 125.0 / 192.0,
                              -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
static const double kB4[7] = {5179.0 / 57600.0,    0.0,           7571.0 / 16695.0,
                              393.0 / 640.0,       -92097.0 / 339200.0, 187.0 / 2100.0,
                              1.0 / 40.0};

static void stepper_free_buffers(pvo_stepper *s) {
    free(s->x0);
    free(s->y0);
    free(s->xt);
    free(s->yt);
    for (int k = 0; k < 7; ++k) {
        free(s->kx[k]);
        free(s->ky[k]);
    }
}

static int stepper_size(pvo_stepper *s, size_t n) {
    if (s->n == n && s->x0)
        return 0;
    stepper_free_buffers(s);
    const size_t bytes = (n ? n : 1) * sizeof(double);
    s->x0 = malloc(bytes);
    s->y0 = malloc(bytes);
    s->xt = malloc(bytes);
    s->yt = malloc(bytes);
    for (int k = 0; k < 7; ++k) {
        s->kx[k] = malloc(bytes);
        s->ky[k] = malloc(bytes);
    }
    s->n = n;
    s->fsal_valid = 0; /* ensureSize, src/timestep.cpp:9-18 */
    return 0;
}

pvo_stepper *pvo_stepper_create(const pvo_params *p, size_t n) {
    if (validate_kernel(p))
        return NULL;
    pvo_stepper *s = calloc(1, sizeof(*s));
    s->params = *p;
    stepper_size(s, n);
    return s;
}

void pvo_stepper_destroy(pvo_stepper *s) {
    if (!s)
        return;
    stepper_free_buffers(s);
    free(s);
}

void pvo_stepper_invalidate(pvo_stepper *s) { s->fsal_valid = 0; }
size_t pvo_stepper_evaluations(const pvo_stepper *s) { return s->evaluations; }

static int stepper_eval(pvo_stepper *s, const double *x, const double *y, const double *g,
                        size_t n, int stage) {
    ++s->evaluations;
    return pvo_evaluate(&s->params, x, y, g, n, s->kx[stage], s->ky[stage]);
}

/* makeStage, src/timestep.cpp:19-30 */
static void make_stage(pvo_stepper *s, int stage, const double *c, double dt) {
    for (size_t i = 0; i < s->n; ++i) {
        double dx = 0.0, dy = 0.0;
        for (int j = 0; j < stage; ++j) {
            dx += c[j] * s->kx[j][i];
            dy += c[j] * s->ky[j][i];
        }
        s->xt[i] = s->x0[i] + dt * dx;
        s->yt[i] = s->y0[i] + dt * dy;
    }
}

/* rk4Step, src/timestep.cpp:31-61 */
int pvo_rk4_step(pvo_stepper *s, double *x, double *y, const double *g, size_t n, double dt) {
    if (!isfinite(dt) || !(dt > 0.0))
        return fail(PVO_INVALID, "timestep must be finite and positive");
    int rc = validate_arrays(x, y, g, n);
    if (rc)
        return rc;
    stepper_size(s, n);
    memcpy(s->x0, x, n * sizeof(double));
    memcpy(s->y0, y, n * sizeof(double));
    s->fsal_valid = 0;
    if ((rc = stepper_eval(s, s->x0, s->y0, g, n, 0)))
        return rc;
    const double a2[7] = {0.5};
    make_stage(s, 1, a2, dt);
    if ((rc = stepper_eval(s, s->xt, s->yt, g, n, 1)))
        return rc;
    const double a3[7] = {0.0, 0.5};
    make_stage(s, 2, a3, dt);
    if ((rc = stepper_eval(s, s->xt, s->yt, g, n, 2)))
        return rc;
    const double a4[7] = {0.0, 0.0, 1.0};
    make_stage(s, 3, a4, dt);
    if ((rc = stepper_eval(s, s->xt, s->yt, g, n, 3)))
        return rc;
    for (size_t i = 0; i < n; ++i) {
        s->xt[i] = s->x0[i] +
                   dt * (s->kx[0][i] + 2.0 * s->kx[1][i] + 2.0 * s->kx[2][i] + s->kx[3][i]) / 6.0;
        s->yt[i] = s->y0[i] +
                   dt * (s->ky[0][i] + 2.0 * s->ky[1][i] + 2.0 * s->ky[2][i] + s->ky[3][i]) / 6.0;
    }
    if ((rc = validate_arrays(s->xt, s->yt, g, n)))
        return rc;
    memcpy(x, s->xt, n * sizeof(double));
    memcpy(y, s->yt, n * sizeof(double));
    return PVO_OK;
}

static double clamp(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }

/* dopri5Step, src/timestep.cpp:62-120 */
int pvo_dopri5_step(pvo_stepper *s, double *x, double *y, const double *g, size_t n, double dt,
                    double *out4) {
    const pvo_params *p = &s->params;
    if (!isfinite(dt) || !(dt > 0.0))
        return fail(PVO_INVALID, "timestep must be finite and positive");
    int rc = validate_arrays(x, y, g, n);
    if (rc)
        return rc;
    stepper_size(s, n);
    memcpy(s->x0, x, n * sizeof(double));
    memcpy(s->y0, y, n * sizeof(double));
    unsigned rejected = 0;
    if (!s->fsal_valid && (rc = stepper_eval(s, s->x0, s->y0, g, n, 0)))
        return rc;
    for (;;) {
        for (int st = 1; st < 7; ++st) {
            make_stage(s, st, kDopri[st], dt);
            if ((rc = stepper_eval(s, s->xt, s->yt, g, n, st)))
                return rc;
        }
        double error = 0.0;
        for (size_t i = 0; i < n; ++i) {
            const double x5 = s->xt[i], y5 = s->yt[i];
            double xe = 0.0, ye = 0.0;
            for (int st = 0; st < 7; ++st) {
                xe += dt * (kB5[st] - kB4[st]) * s->kx[st][i];
                ye += dt * (kB5[st] - kB4[st]) * s->ky[st][i];
            }
            const double xs = p->absolute_tolerance +
                              p->relative_tolerance * fmax_ref(fabs(s->x0[i]), fabs(x5));
            const double ys = p->absolute_tolerance +
                              p->relative_tolerance * fmax_ref(fabs(s->y0[i]), fabs(y5));
            if (!isfinite(xe) || !isfinite(ye) || !isfinite(xs) || !isfinite(ys) || !(xs > 0.0) ||
                !(ys > 0.0))
                return fail(PVO_RUNTIME, "non-finite adaptive error estimate or invalid tolerance");
            error = fmax_ref(error, fabs(xe) / xs);
            error = fmax_ref(error, fabs(ye) / ys);
        }
        const double factor = error == 0.0 ? 5.0 : clamp(0.9 * pow(error, -0.2), 0.2, 5.0);
        const double suggested = clamp(dt * factor, p->minimum_time_step, p->maximum_time_step);
        if (error <= 1.0) {
            memcpy(x, s->xt, n * sizeof(double));
            memcpy(y, s->yt, n * sizeof(double));
            double *tx = s->kx[0], *ty = s->ky[0];
            s->kx[0] = s->kx[6];
            s->ky[0] = s->ky[6];
            s->kx[6] = tx;
            s->ky[6] = ty;
            s->fsal_valid = 1;
            out4[0] = dt;
            out4[1] = suggested;
            out4[2] = error;
            out4[3] = (double)rejected;
            return PVO_OK;
        }
        if (dt <= p->minimum_time_step || ++rejected > 32)
            return fail(PVO_RUNTIME, "adaptive integrator could not satisfy tolerance");
        dt = fmax_ref(p->minimum_time_step, fmin_ref(suggested, dt * 0.9));
    }
}

/* ---------------------------------------------------------------------------------------
 * Close-dipole candidate scan, DipoleManager::process src/dipole.cpp:49-78.
 */
int pvo_dipole_scan(const pvo_params *p, const double *x, const double *y, const double *g,
                    size_t n, pvo_candidate *out, size_t cap, size_t *count) {
    const int periodic = p->geometry == 1;
    const double thr2 = p->dipole_removal_distance * p->dipole_removal_distance;
    size_t found = 0;
#define PUSH(a, b, d)                                                                          \
    do {                                                                                       \
        if (found < cap) {                                                                     \
            out[found].first = (a);                                                            \
            out[found].second = (b);                                                           \
            out[found].distance_squared = (d);                                                 \
        }                                                                                      \
        ++found;                                                                               \
    } while (0)
    for (size_t i = 0; i < n; ++i) {
        if (g[i] == 0.0)
            continue;
        for (size_t j = i + 1; j < n; ++j) {
            if (g[j] == 0.0 || signbit(g[i]) == signbit(g[j]))
                continue;
            const double ddx = x[i] - x[j], ddy = y[i] - y[j];
            const double dx = periodic ? remainder(ddx, p->box_length_x) : ddx;
            const double dy = periodic ? remainder(ddy, p->box_length_y) : ddy;
            const double d2 = dx * dx + dy * dy;
            if (d2 < thr2)
                PUSH(i, j, d2);
        }
        if (p->geometry == 2) {
            const double r2 = p->disk_radius * p->disk_radius;
            const double rad2 = x[i] * x[i] + y[i] * y[i];
            if (rad2 > 0.0) {
                const double image = (r2 - rad2) / sqrt(rad2);
                if (image * image < thr2)
                    PUSH(i, n, image * image);
            }
        }
    }
#undef PUSH
    *count = found;
    return PVO_OK;
}
