"""Parity of the CUDA velocity kernels (FP64) with the oracle: per-vortex normalised velocity error
<= 1e-12 (|d(u,v)_i| / max(|(u,v)_i|, rms |(u,v)|)), on seeded states, the golden fixtures made
by the unmodified reference, the reference's edge cases and every size class of the tiling."""
import numpy as np
import pytest

from conftest import golden, normalized_error
from gpu_impl import GpuImpl
from oracle.pyoracle import Geometry
from pointvortex_b200 import ics

pytestmark = pytest.mark.gpu
TOL = 1e-12

GEOS = {
    "infinite": Geometry("infinite"),
    "infinite_core": Geometry("infinite", core_radius=0.05),
    "periodic": Geometry("periodic", box_length_x=2.0, box_length_y=2.0),
    "periodic_m3": Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=3),
    "disk": Geometry("disk", disk_radius=1.0),
}


@pytest.fixture(scope="module")
def gpu():
    return GpuImpl()


def state(geo, n, seed):
    if geo.boundary == "periodic":
        return ics.periodic_box(n + n % 2, seed, geo.box_length_x)
    if geo.boundary == "disk":
        return ics.disk(n, seed, geo.disk_radius, 0.95)
    return ics.infinite_plane(n, seed)


@pytest.mark.parametrize("tag", sorted(GEOS))
def test_small_fixture_velocities(gpu, tag):
    d = golden(f"small_{tag}.npz")
    u, v = gpu.evaluate(GEOS[tag], d["x"], d["y"], d["g"])
    assert normalized_error(u, v, d["u"], d["v"]).max() <= TOL


@pytest.mark.parametrize("geo_name", ["infinite", "periodic", "disk", "infinite_core"])
@pytest.mark.parametrize("n", [1, 2, 3, 31, 33, 127, 128, 129, 255, 256, 257, 511, 513, 1000, 2049])
def test_random_states_against_oracle(gpu, port, geo_name, n):
    geo = GEOS[geo_name]
    x, y, g = state(geo, n, 1000 + n)
    u, v = gpu.evaluate(geo, x, y, g)
    ur, vr = port.evaluate(geo, x, y, g)
    assert normalized_error(u, v, ur, vr).max() <= TOL


@pytest.mark.parametrize("layers", [0, 1, 2, 4, 5, 6, 7, 8, 12, 64])
def test_periodic_image_layers(gpu, port, layers):
    geo = Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=layers)
    x, y, g = ics.periodic_box(150, 77 + layers, 2.0)
    u, v = gpu.evaluate(geo, x, y, g)
    ur, vr = port.evaluate(geo, x, y, g)
    assert normalized_error(u, v, ur, vr).max() <= TOL


def test_periodic_positions_outside_the_box(gpu, port):
    """The reference never wraps positions; displacements use remainder(dx, L)."""
    geo = Geometry("periodic", box_length_x=2.0, box_length_y=2.0)
    x, y, g = ics.periodic_box(200, 5, 2.0)
    x = x + np.round(np.linspace(-7, 7, x.size)) * 2.0
    y = y - np.round(np.linspace(3, -3, y.size)) * 2.0
    u, v = gpu.evaluate(geo, x, y, g)
    ur, vr = port.evaluate(geo, x, y, g)
    assert normalized_error(u, v, ur, vr).max() <= TOL


def test_disk_radius_and_near_wall(gpu, port):
    geo = Geometry("disk", disk_radius=2.5)
    x, y, g = ics.disk(300, 9, 2.5, 0.999)
    u, v = gpu.evaluate(geo, x, y, g)
    ur, vr = port.evaluate(geo, x, y, g)
    assert normalized_error(u, v, ur, vr).max() <= TOL


@pytest.mark.parametrize("geo_name", ["infinite", "periodic", "disk"])
def test_evaluate_range(gpu, port, geo_name):
    geo = GEOS[geo_name]
    x, y, g = state(geo, 700, 4)
    for begin, end in [(0, 700), (3, 5), (129, 600), (699, 700), (10, 10)]:
        u, v = gpu.evaluate_range(geo, x, y, g, begin, end)
        ur, vr = port.evaluate_range(geo, x, y, g, begin, end)
        assert u.size == end - begin
        if end > begin:
            assert normalized_error(u, v, ur, vr).max() <= TOL


def test_workload_fixtures(gpu):
    d = golden("workload_infinite_n1024.npz")
    u, v = gpu.evaluate(Geometry("infinite"), d["x"], d["y"], d["g"])
    assert normalized_error(u, v, d["u"], d["v"]).max() <= TOL
    d = golden("workload_periodic_n4096.npz")
    u, v = gpu.evaluate(Geometry("periodic", box_length_x=2 * np.pi, box_length_y=2 * np.pi),
                        d["x"], d["y"], d["g"])
    k = int(d["targets"][1])
    assert normalized_error(u[:k], v[:k], d["u"], d["v"]).max() <= TOL
    d = golden("workload_disk_n16384.npz")
    u, v = gpu.evaluate(Geometry("disk", disk_radius=1.0), d["x"], d["y"], d["g"])
    k = int(d["targets"][1])
    assert normalized_error(u[:k], v[:k], d["u"], d["v"]).max() <= TOL


def test_deterministic(gpu):
    geo = GEOS["periodic"]
    x, y, g = state(geo, 3000, 8)
    a = gpu.evaluate(geo, x, y, g)
    b = gpu.evaluate(geo, x, y, g)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("case", [
    ("nan", "infinite"), ("coincident", "infinite"), ("coincident", "periodic"),
    ("coincident", "disk"), ("outside", "disk"), ("nonneutral", "periodic"),
])
def test_errors_match_oracle(gpu, port, case):
    kind, geo_name = case
    geo = GEOS[geo_name]
    x = np.array([0.1, -0.2, 0.3, -0.05])
    y = np.array([0.0, 0.1, -0.2, 0.25])
    g = np.array([1.0, -1.0, 1.0, -1.0])
    if kind == "nan":
        x[1] = np.nan
    elif kind == "coincident":
        x[2], y[2] = x[0], y[0]
    elif kind == "outside":
        x[3] = 1.0
    elif kind == "nonneutral":
        g[0] = 2.0
    errs = []
    for impl in (gpu, port):
        with pytest.raises(Exception) as info:
            impl.evaluate(geo, x, y, g)
        errs.append((type(info.value).__mro__[1] if type(info.value).__name__ == "LogicError"
                     else type(info.value), str(info.value)))
    assert errs[0] == errs[1]


def test_range_error(gpu):
    x, y, g = ics.infinite_plane(8, 3)
    with pytest.raises(IndexError, match="invalid target-vortex range"):
        gpu.evaluate_range(Geometry("infinite"), x, y, g, 5, 9)


def test_constructor_validation():
    import pointvortex_b200 as pv
    for make in (lambda: pv.InfinitePlaneKernel(-1.0), lambda: pv.PeriodicBoxKernel(2, 2, 65),
                 lambda: pv.PeriodicBoxKernel(2.0, 2.5), lambda: pv.DiskKernel(0.0)):
        with pytest.raises(ValueError):
            make()
