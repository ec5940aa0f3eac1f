"""The GPU text formatter's source (pointvortex_b200/csrc/pv_format.cuh) compiled for the host:
every value must print exactly as `std::ostream << std::setprecision(17)` prints it, i.e. C's
"%.17g" (libstdc++ formats through it). Python's "%.17g" is correctly rounded like glibc's, so it
is the checker for finite values; signs of NaN follow glibc ("-nan")."""
import ctypes
import os
import struct
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("fmt") / "libformat_harness.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    os.path.join(HERE, "native", "format_harness.cpp")], check=True)
    lib = ctypes.CDLL(str(out))
    lib.pvf_format_many.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_size_t,
                                    ctypes.c_char_p, ctypes.c_size_t]
    lib.pvf_format_u64.argtypes = [ctypes.c_ulonglong, ctypes.c_char_p]
    return lib


def fmt_many(lib, values):
    v = np.ascontiguousarray(values, dtype=np.float64)
    stride = 32
    buf = ctypes.create_string_buffer(stride * max(v.size, 1))
    lib.pvf_format_many(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), v.size, buf, stride)
    raw = buf.raw
    return [raw[i * stride:(i + 1) * stride].split(b"\0", 1)[0].decode() for i in range(v.size)]


def expected(v: float) -> str:
    if v != v:
        return "-nan" if struct.pack(">d", v)[0] & 0x80 else "nan"
    return "%.17g" % v


def edge_values():
    vals = [0.0, -0.0, 1.0, -1.0, 0.1, 0.5, 1e17, 1e16, 9.999999999999999e16, 1e-4, 1e-5,
            9.9999999999999995e-5, 123456789012345678.0, 2.0 ** 52, 2.0 ** 53, 2.0 ** 63,
            2.0 ** 64, 1.7976931348623157e308, 2.2250738585072014e-308, 5e-324, 1e-323,
            2.2250738585072009e-308, 1e308, 1e-308, 3.141592653589793, 2.718281828459045,
            float("inf"), float("-inf"), float("nan"), 0.30000000000000004, 100.0, 1e21, 1e22,
            1e23, 4.35e-5, 0.00012345678901234567, 12345678901234567.0]
    # powers of ten and their neighbours, and 17-digit ties
    for e in range(-320, 309):
        p = float(f"1e{e}")
        vals += [p, np.nextafter(p, 0.0), np.nextafter(p, np.inf)]
    return np.array(vals, dtype=np.float64)


def test_edge_values(harness):
    v = edge_values()
    got = fmt_many(harness, v)
    want = [expected(float(x)) for x in v]
    bad = [(float(x), g, w) for x, g, w in zip(v, got, want) if g != w]
    assert not bad, bad[:10]


def test_random_bit_patterns(harness):
    rng = np.random.default_rng(2024)
    bits = rng.integers(0, 2 ** 63, size=200_000, dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=200_000, dtype=np.uint64)
    v = bits.view(np.float64)
    v = v[np.isfinite(v)]
    got = fmt_many(harness, v)
    want = ["%.17g" % float(x) for x in v]
    bad = [(float(x), g, w) for x, g, w in zip(v, got, want) if g != w]
    assert not bad, bad[:10]


def test_domain_values(harness):
    """Values like the files hold: positions in a box, velocities, circulations, small deltas."""
    rng = np.random.default_rng(7)
    v = np.concatenate([rng.uniform(-np.pi, np.pi, 50_000), rng.normal(0, 1e3, 50_000),
                        rng.normal(0, 1e-15, 50_000), np.round(rng.uniform(-5, 5, 10_000)),
                        rng.uniform(0, 1, 10_000) * 10.0 ** rng.integers(-20, 20, 10_000)])
    got = fmt_many(harness, v)
    want = ["%.17g" % float(x) for x in v]
    assert got == want


def test_integers(harness):
    buf = ctypes.create_string_buffer(32)
    for v in (0, 1, 9, 10, 12345, 2 ** 32, 2 ** 64 - 1):
        harness.pvf_format_u64(v, buf)
        assert buf.value.decode() == str(v)
