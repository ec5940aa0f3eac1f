"""Pins the C restatement of the oracle against the unmodified reference compiled from its own
sources (oracle/_ref). Both run on the CPU; agreement is bit for bit."""
import numpy as np
import pytest

from oracle.pyoracle import Geometry
from pointvortex_b200 import ics

GEOMETRIES = [
    Geometry("infinite"),
    Geometry("infinite", core_radius=0.05),
    Geometry("periodic", box_length_x=2.0, box_length_y=2.0),
    Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=0),
    Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=6),
    Geometry("disk", disk_radius=1.0),
    Geometry("disk", disk_radius=2.5),
]


def state_for(geo: Geometry, n: int, seed: int):
    if geo.boundary == "periodic":
        return ics.periodic_box(n + (n % 2), seed, geo.box_length_x)
    if geo.boundary == "disk":
        return ics.disk(n, seed, geo.disk_radius, 0.8, gaussian=False)
    return ics.infinite_plane(n, seed)


@pytest.mark.parametrize("geo", GEOMETRIES, ids=lambda g: f"{g.boundary}-{g.core_radius}-{g.image_layers}-{g.disk_radius}")
@pytest.mark.parametrize("n", [1, 2, 3, 33, 130])
def test_evaluate_and_invariants_bit_exact(port, reference, geo, n):
    x, y, g = state_for(geo, n, 100 + n)
    u1, v1 = port.evaluate(geo, x, y, g)
    u2, v2 = reference.evaluate(geo, x, y, g)
    assert np.array_equal(u1, u2) and np.array_equal(v1, v2)
    assert np.array_equal(port.invariants(geo, x, y, g), reference.invariants(geo, x, y, g))
    if x.size > 4:
        a = port.evaluate_range(geo, x, y, g, 2, x.size - 1)
        b = reference.evaluate_range(geo, x, y, g, 2, x.size - 1)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("geo", GEOMETRIES[::2], ids=lambda g: g.boundary)
def test_integrators_bit_exact(port, reference, geo):
    x, y, g = state_for(geo, 40, 7)
    s1, s2 = port.stepper(geo, x.size), reference.stepper(geo, x.size)
    a, b = (x, y), (x, y)
    for _ in range(3):
        a = s1.rk4_step(a[0], a[1], g, 1e-3)
        b = s2.rk4_step(b[0], b[1], g, 1e-3)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    d1, d2 = port.stepper(geo, x.size), reference.stepper(geo, x.size)
    xa, ya, xb, yb = x, y, x, y
    dt1 = dt2 = 2e-3
    for _ in range(4):
        xa, ya, ra = d1.dopri5_step(xa, ya, g, dt1)
        xb, yb, rb = d2.dopri5_step(xb, yb, g, dt2)
        assert np.array_equal(xa, xb) and np.array_equal(ya, yb)
        assert np.array_equal(ra, rb)
        dt1, dt2 = ra[1], rb[1]


@pytest.mark.parametrize("case", [
    ("nan", Geometry("infinite")),
    ("coincident", Geometry("infinite")),
    ("coincident", Geometry("periodic", box_length_x=2.0, box_length_y=2.0)),
    ("coincident", Geometry("disk", disk_radius=1.0)),
    ("outside", Geometry("disk", disk_radius=1.0)),
    ("nonneutral", Geometry("periodic", box_length_x=2.0, box_length_y=2.0)),
    ("layers", Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=65)),
    ("square", Geometry("periodic", box_length_x=2.0, box_length_y=2.5)),
    ("core", Geometry("infinite", core_radius=-1.0)),
    ("radius", Geometry("disk", disk_radius=0.0)),
], ids=lambda c: f"{c[0]}-{c[1].boundary}")
def test_error_parity(port, reference, case):
    kind, geo = case
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
    for o in (port, reference):
        with pytest.raises(Exception) as info:
            o.evaluate(geo, x, y, g)
        errs.append((type(info.value), str(info.value)))
    assert errs[0] == errs[1]


def test_range_error_parity(port, reference):
    geo = Geometry("infinite")
    x, y, g = ics.infinite_plane(8, 3)
    for o in (port, reference):
        with pytest.raises(IndexError, match="invalid target-vortex range"):
            o.evaluate_range(geo, x, y, g, 5, 9)


def test_hamiltonian_errors_parity(port, reference):
    x = np.array([0.1, 0.1, 0.3])
    y = np.array([0.2, 0.2, -0.1])
    g = np.array([1.0, -1.0, 0.5])
    for geo in (Geometry("infinite"), Geometry("periodic", box_length_x=2.0, box_length_y=2.0),
                Geometry("disk", disk_radius=1.0)):
        errs = []
        for o in (port, reference):
            with pytest.raises(Exception) as info:
                o.hamiltonian(geo, x, y, g)
            errs.append((type(info.value), str(info.value)))
        assert errs[0] == errs[1]


def select_events(candidates, n):
    """Closest-first disjoint selection of DipoleManager::process (src/dipole.cpp:79-100)."""
    chosen = [False] * n
    events = 0
    for a, b, _ in sorted(candidates, key=lambda c: (c[2], c[0], c[1])):
        if chosen[a] or (b < n and chosen[b]):
            continue
        chosen[a] = True
        if b < n:
            chosen[b] = True
        events += 1
    return events, chosen


@pytest.mark.parametrize("tag", ["periodic", "disk", "infinite"])
def test_dipole_scan_matches_reference_process(port, reference, tag):
    from conftest import golden
    d = golden(f"dipole_{tag}.npz")
    geo = {"periodic": Geometry("periodic", box_length_x=2.0, box_length_y=2.0,
                                dipole_removal=True, dipole_removal_distance=0.05),
           "disk": Geometry("disk", disk_radius=1.0, dipole_removal=True, dipole_removal_distance=0.05),
           "infinite": Geometry("infinite", dipole_removal=True, dipole_removal_distance=0.05)}[tag]
    cands = port.dipole_scan(geo, d["x"], d["y"], d["g"])
    events, chosen = select_events(cands, d["x"].size)
    ref_events, sx, sy, sg = reference.dipole_process(geo, d["x"], d["y"], d["g"])
    assert events == ref_events == int(d["events"][0]) and events > 0
    keep = ~np.array(chosen)
    assert np.array_equal(d["x"][keep], sx) and np.array_equal(d["g"][keep], sg)


def test_mt19937_64_known_answer():
    """The C++ standard's required value: the 10000th draw of a default-constructed
    std::mt19937_64 is 9981545732273789042 ([rand.predef])."""
    from oracle.pyoracle import MT19937_64
    e = MT19937_64()
    for _ in range(9999):
        e()
    assert e() == 9981545732273789042


@pytest.mark.parametrize("boundary,mode", [(b, m) for b in ("periodic", "disk") for m in (0, 1, 2)])
def test_dipole_port_matches_reference_fixtures(port, boundary, mode):
    """DipolePort (selection, compaction, reinjection draws, generator text state) against three
    consecutive DipoleManager::process calls of the reference."""
    from conftest import golden
    from golden.make_golden import dipole_event_geometry
    d = golden(f"dipole_events_{boundary}_{mode}.npz")
    geo = dipole_event_geometry(boundary, mode)
    x, y, g, state = d["x"], d["y"], d["g"], None
    for call in range(3):
        events, x, y, g, state = port.dipole_events(geo, x, y, g, state)
        assert events == int(d[f"events{call}"][0])
        assert np.array_equal(x, d[f"x{call}"]) and np.array_equal(y, d[f"y{call}"])
        assert np.array_equal(g, d[f"g{call}"])
        assert state[:2] == tuple(int(c) for c in d[f"counts{call}"])
        assert state[2] == str(d[f"engine{call}"])
    assert int(d["events0"][0]) > 0
