"""The FP32 prefilter of the dipole scan never drops a candidate, on the CPU.

The scan (csrc/pv_dipole.cu) first computes each pair's squared minimum-image distance in FP32
from double-float coordinates, and runs the reference's exact FP64 test only for pairs whose FP32
distance is not above a per-target bound thr2f = (thr + 2e)^2 (1 + 2^-20), with
e = 2^-21 M + 2^-22 thr and M the largest coordinate magnitude of the pair. This test restates
that FP32 arithmetic in numpy (float32 adds and multiplies round as the device's; the fused
multiply-adds are formed exactly in float64 and rounded once), places partners just inside the
threshold around targets anywhere in and far outside the box, across periodic images, and checks
that every pair the exact test accepts passes the prefilter."""
import numpy as np

F32 = np.float32
L = 2.0 * np.pi
MAGIC = F32(12582912.0)  # 1.5 * 2^23: adding and subtracting it rounds to the nearest integer


def _split(x):
    hi = x.astype(F32)
    return hi, (x - hi.astype(np.float64)).astype(F32)


def _fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F32)


def _fp32_component(t, s, periodic):
    th, tl = _split(t)
    sh, sl = _split(s)
    d = (th + (-sh)) + (tl + (-sl))
    if not periodic:
        return d
    q = d * F32(1.0 / L)
    m = (q + MAGIC) + (-MAGIC)
    l_hi = F32(L)
    l_lo = F32(L - np.float64(l_hi))
    return _fma32(m, -l_lo, _fma32(m, -l_hi, d))


def _exact_component(t, s, periodic):
    d = t - s
    if periodic:
        d = d - np.rint(d / L) * L
    return d


def _check(periodic, magnitude, thr, seed):
    rng = np.random.default_rng(seed)
    n = 100000
    xi = rng.uniform(-magnitude, magnitude, n)
    yi = rng.uniform(-magnitude, magnitude, n)
    ang = rng.uniform(0.0, 2.0 * np.pi, n)
    rad = thr * rng.uniform(0.95, 1.0, n)
    shift_x = rng.integers(-2, 3, n) * L if periodic else 0.0
    shift_y = rng.integers(-2, 3, n) * L if periodic else 0.0
    xj = xi + rad * np.cos(ang) + shift_x
    yj = yi + rad * np.sin(ang) + shift_y
    dx = _exact_component(xi, xj, periodic)
    dy = _exact_component(yi, yj, periodic)
    candidate = dx * dx + dy * dy < thr * thr
    rx = _fp32_component(xi, xj, periodic)
    ry = _fp32_component(yi, yj, periodic)
    d2f = _fma32(rx, rx, (ry * ry).astype(F32))
    m = np.maximum.reduce([np.abs(xi), np.abs(yi), np.abs(xj), np.abs(yj)])
    e = 2.0 ** -21 * m + 2.0 ** -22 * thr
    bound = ((thr + 2.0 * e) ** 2 * (1.0 + 2.0 ** -20)).astype(F32)
    assert candidate.sum() > n // 4
    missed = candidate & (d2f > bound)
    assert not missed.any(), (periodic, magnitude, thr, int(missed.sum()))


def test_prefilter_keeps_every_candidate_in_the_box():
    for k, (magnitude, thr) in enumerate([(np.pi, 1e-3), (np.pi, 1e-5), (30.0, 1e-3),
                                          (1000.0, 1e-2)]):
        _check(True, magnitude, thr, 100 + k)


def test_prefilter_keeps_every_candidate_in_the_plane():
    for k, (magnitude, thr) in enumerate([(1.0, 1e-3), (1e4, 1e-3), (1e-2, 1e-6)]):
        _check(False, magnitude, thr, 200 + k)
