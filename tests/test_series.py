"""The polynomial sinh/cosh/sin/cos of the periodic pair terms, evaluated on the CPU.

The device evaluates sinh, cosh, sin and cos of t = x^/2 and y^/2 (|t| <= pi/2) as four
polynomials in w = t^4 sharing one set of powers (csrc/pv_common.cuh): sinh(t) = t E1 + t^3 O1,
sin(t) = t E1 - t^3 O1, cosh(t) = E0 + t^2 O0, cos(t) = E0 - t^2 O0. The pair terms use
coefficients economized over the interval (one fewer per polynomial than the Taylor series); the
Hamiltonian keeps the Taylor ones. This test reads the coefficients from the header and checks the
four functions against numpy's long-double ones over the whole interval, within the bounds the
header states."""
import pathlib
import re

import numpy as np

HEADER = pathlib.Path(__file__).resolve().parent.parent / "pointvortex_b200" / "csrc" / "pv_common.cuh"


def _economized_coefficients():
    text = HEADER.read_text()
    body = text[text.index("void sinh_cosh_sin_cos_economized"):]
    body = body[: body.index("\n}\n")]
    polys = {}
    for name in ("e1", "o1", "e0", "o0"):
        # "double e1 = fma(w, c_top, c_next);" then "e1 = fma(w, e1, c);" lines: highest first
        first = re.search(rf"double {name} = fma\(w, ([-0-9.e+]+), ([-0-9.e+]+)\);", body)
        rest = re.findall(rf"\n\s*{name} = fma\(w, {name}, ([-0-9.e+]+)\);", body)
        assert first, name
        polys[name] = [float(first.group(1)), float(first.group(2))] + [float(c) for c in rest]
    return polys


def _horner(coeffs, w):
    acc = np.full_like(w, coeffs[0])
    for c in coeffs[1:]:
        acc = acc * w + c
    return acc


def test_economized_series_matches_the_functions():
    p = _economized_coefficients()
    assert [len(p[k]) for k in ("e1", "o1", "e0", "o0")] == [5, 4, 5, 4]
    t = np.linspace(-np.pi / 2, np.pi / 2, 200001)
    t2 = t * t
    w = t2 * t2
    e1, o1, e0, o0 = (_horner(p[k], w) for k in ("e1", "o1", "e0", "o0"))
    sh = t * e1 + t * t2 * o1
    s = t * e1 - t * t2 * o1
    ch = e0 + t2 * o0
    c = e0 - t2 * o0
    tl = t.astype(np.longdouble)
    ref = {"sinh": np.sinh(tl), "sin": np.sin(tl), "cosh": np.cosh(tl), "cos": np.cos(tl)}
    nz = t != 0
    rel = lambda a, r: float(np.max(np.abs((a[nz] - r[nz]) / r[nz])))  # noqa: E731
    # the header's bounds (fma evaluation) with room for this test's separate multiply-adds
    assert rel(sh, ref["sinh"]) <= 1e-15
    assert rel(s, ref["sin"]) <= 1e-15
    assert rel(ch, ref["cosh"]) <= 3e-15
    assert float(np.max(np.abs(c - ref["cos"]))) <= 6e-15


def test_economized_coefficients_stay_near_taylor():
    """Economization perturbs each Taylor coefficient only slightly (the leading ones by less than
    1e-14 relative): the series is still the Taylor series of exp(t) and exp(it) grouped by
    t^(4k+r)."""
    from math import factorial
    p = _economized_coefficients()
    taylor = {"e1": [1 / factorial(4 * k + 1) for k in range(5)],
              "o1": [1 / factorial(4 * k + 3) for k in range(4)],
              "e0": [1 / factorial(4 * k) for k in range(5)],
              "o0": [1 / factorial(4 * k + 2) for k in range(4)]}
    for name, coeffs in p.items():
        low_first = coeffs[::-1]
        assert abs(low_first[0] - taylor[name][0]) <= 1e-14 * taylor[name][0], name
        for got, exact in zip(low_first, taylor[name]):
            assert abs(got - exact) <= 0.05 * exact, (name, got, exact)


PAIR32 = pathlib.Path(__file__).resolve().parent.parent / "pointvortex_b200" / "csrc" / "pv_pair32.cuh"


def _fp32_coefficients():
    text = PAIR32.read_text()
    body = text[text.index("void sh_sn_cs_x2"):]
    body = body[: body.index("\n}\n")]
    num = r"([-0-9.e+]+)f"
    polys = {}
    for name in ("e1", "o1", "e0", "o0n"):
        first = re.search(rf"float2 {name} = fma2\(w, splat2\({num}\), splat2\({num}\)\);", body)
        rest = re.findall(rf"\n\s*{name} = fma2\(w, {name}, splat2\({num}\)\);", body)
        assert first, name
        polys[name] = [float(first.group(1)), float(first.group(2))] + [float(c) for c in rest]
    return {k: np.array(v, dtype=np.float32).astype(np.float64).tolist() for k, v in polys.items()}


def test_fp32_series_is_accurate_to_fp32():
    """The FP32 periodic pair's economized series (csrc/pv_pair32.cuh): sinh and sin within 1e-7
    and cos within 2e-7 absolute of the functions over |t| <= pi/2, evaluated in float64 with
    the FP32 coefficients (the coefficients' own rounding included)."""
    p = _fp32_coefficients()
    t = np.linspace(-np.pi / 2, np.pi / 2, 200001)
    t2 = t * t
    w = t2 * t2
    e1, o1, e0, o0n = (_horner(p[k], w) for k in ("e1", "o1", "e0", "o0n"))
    sh = t * e1 + t * t2 * o1
    sn = t * e1 - t * t2 * o1
    cs = e0 + t2 * o0n
    nz = t != 0
    assert np.max(np.abs((sh - np.sinh(t))[nz] / np.sinh(t)[nz])) <= 1e-7
    assert np.max(np.abs((sn - np.sin(t))[nz] / np.sin(t)[nz])) <= 1e-7
    assert np.max(np.abs(cs - np.cos(t))) <= 2e-7
