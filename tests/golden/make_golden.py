"""Generates the golden fixtures in this directory from the UNMODIFIED reference.

Run in a tree where the reference sources are available (it builds oracle/_ref/ first):

    python tests/golden/make_golden.py [--reference /path/to/PointVortex]

Every number stored here comes from the reference's own code (src/compute.cpp, src/timestep.cpp,
src/dipole.cpp of jplaurie/PointVortex), called through oracle/ref_shim.cpp. The initial
conditions come from pointvortex_b200/ics.py and are stored beside the results, so the tests
need neither the reference nor a random generator to use them.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pyoracle import Geometry, Oracle  # noqa: E402

_spec = importlib.util.spec_from_file_location("ics", os.path.join(ROOT, "pointvortex_b200", "ics.py"))
ics = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(ics)


def save(name: str, **arrays) -> None:
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"{name}: {os.path.getsize(path) / 1024:.1f} KiB", flush=True)


def small_case(ref: Oracle, geo: Geometry, x, y, g, tag: str) -> None:
    u, v = ref.evaluate(geo, x, y, g)
    inv = ref.invariants(geo, x, y, g)
    st = ref.stepper(geo, x.size)
    rk_x, rk_y = [x.copy()], [y.copy()]
    for _ in range(3):
        nx, ny = st.rk4_step(rk_x[-1], rk_y[-1], g, 1e-3)
        rk_x.append(nx)
        rk_y.append(ny)
    dp = ref.stepper(geo, x.size)
    dp_x, dp_y, dp_r = [x.copy()], [y.copy()], []
    dt = 1e-3
    for _ in range(3):
        nx, ny, r = dp.dopri5_step(dp_x[-1], dp_y[-1], g, dt)
        dp_x.append(nx)
        dp_y.append(ny)
        dp_r.append(r)
        dt = r[1]
    save(f"small_{tag}.npz", x=x, y=y, g=g, u=u, v=v, inv=inv, rk_x=np.array(rk_x),
         rk_y=np.array(rk_y), dp_x=np.array(dp_x), dp_y=np.array(dp_y), dp_r=np.array(dp_r),
         params=np.array([geo.core_radius, geo.box_length_x, geo.image_layers, geo.disk_radius,
                          geo.absolute_tolerance, geo.relative_tolerance]))


def planted_dipoles(boundary: str, n: int, seed: int):
    """A state with ten planted close opposite-sign pairs (and, in the disk, vortices near the
    wall): the input of the dipole-event fixtures."""
    rng = np.random.default_rng(seed)
    if boundary == "periodic":
        x, y, g = ics.periodic_box(n, seed, 2 * np.pi)
    else:
        x, y, g = ics.disk(n, seed, 1.0, 0.999, gaussian=False)
    # move negative vortices next to positive ones (circulations untouched, so the periodic
    # state keeps its zero total)
    for a, b in zip(np.flatnonzero(g > 0)[:10], np.flatnonzero(g < 0)[:10]):
        x[b] = x[a] + rng.uniform(-0.01, 0.01)
        y[b] = y[a] + rng.uniform(-0.01, 0.01)
    if boundary == "periodic":
        x = np.remainder(x + np.pi, 2 * np.pi) - np.pi
    return x, y, g


DIPOLE_EVENT_CASES = [(b, mode) for b in ("periodic", "disk") for mode in (0, 1, 2)]


def dipole_event_geometry(boundary: str, mode: int) -> Geometry:
    return Geometry(boundary, box_length_x=2 * np.pi, box_length_y=2 * np.pi, disk_radius=1.0,
                    dipole_removal=True, dipole_removal_distance=0.02, dipole_reinjection=mode,
                    random_seed=99)


def dipole_event_fixtures(ref: Oracle) -> None:
    """Three consecutive DipoleManager::process calls of one manager (removal, independent and
    paired reinjection; periodic box and disk), with the counts and the generator text state
    after each call."""
    for boundary, mode in DIPOLE_EVENT_CASES:
        geo = dipole_event_geometry(boundary, mode)
        x, y, g = planted_dipoles(boundary, 400, 5)
        out = {"x": x, "y": y, "g": g}
        state = None
        for call in range(3):
            events, x, y, g, state = ref.dipole_events(geo, x, y, g, state)
            out.update({f"events{call}": np.array([events]), f"x{call}": x, f"y{call}": y,
                        f"g{call}": g, f"counts{call}": np.array(state[:2], dtype=np.uint64),
                        f"engine{call}": np.array(state[2])})
        save(f"dipole_events_{boundary}_{mode}.npz", **out)


# The timed periodic workload: N = 4096 in the 2 pi box, M = 8, DOPRI5 rtol 1e-9 / atol 1e-12 from
# dt = 1e-3, close-dipole removal at 1e-3 after every accepted step.
DOPRI_WORKLOAD = dict(boundary="periodic", box_length_x=2 * np.pi, box_length_y=2 * np.pi,
                      image_layers=8, absolute_tolerance=1e-12, relative_tolerance=1e-9,
                      minimum_time_step=1e-12, maximum_time_step=0.1, dipole_removal=True,
                      dipole_removal_distance=1e-3)


def dopri_workload_fixture(ref: Oracle) -> None:
    """Two accepted DOPRI5 steps of the timed periodic workload by the reference's own
    RungeKuttaIntegrator (FSAL kept between them, src/timestep.cpp:62-120), each followed by
    its DipoleManager::process (src/dipole.cpp:42-127): the states, the step results (accepted
    dt, suggested dt, error, rejections) and the event counts."""
    x, y, g = ics.workload_state("periodic_dopri5_n4096")
    geo = Geometry(**DOPRI_WORKLOAD)
    st = ref.stepper(geo, x.size)
    out = {"x0": x, "y0": y, "g": g, "dt0": np.array([1e-3])}
    dt = 1e-3
    for k in (1, 2):
        x, y, r = st.dopri5_step(x, y, g, dt)
        events, x, y, g2 = ref.dipole_process(geo, x, y, g)
        if events:
            raise RuntimeError("the fixture assumes no dipole events in its first steps")
        out.update({f"x{k}": x, f"y{k}": y, f"r{k}": r, f"events{k}": np.array([events])})
        dt = r[1]
        print(f"step {k}: {r}", flush=True)
    save("workload_periodic_dopri5_n4096_steps.npz", **out)


def output_inputs():
    """Inputs of the writer fixtures: a periodic state with velocities, with awkward values
    (negative zero, integers, powers of ten, subnormals, huge and tiny magnitudes) mixed in."""
    x, y, g = ics.periodic_box(300, 31, 2 * np.pi)
    rng = np.random.default_rng(32)
    u = rng.normal(0.0, 50.0, 300)
    v = rng.normal(0.0, 50.0, 300) * 10.0 ** rng.integers(-12, 12, 300)
    odd = np.array([0.0, -0.0, 1.0, -1.0, 1e-5, 1e-4, 1e16, 1e17, 123456789012345678.0, 5e-324,
                    1.7976931348623157e308, 0.1, 2.5, 1e21, -3.0e-310])
    u[:odd.size] = odd
    v[-odd.size:] = odd[::-1]
    return x, y, g, u, v


OUTPUT_GEOMETRY = dict(boundary="periodic", box_length_x=2 * np.pi, box_length_y=2 * np.pi,
                       dipole_removal=True, dipole_removal_distance=1e-3)
OUTPUT_RECORDS = dict(initial=[0.0, 0.123, -0.456, 7.0, -0.0123456789],
                      segment=[0.0, 0.1230000001, -0.4559999, 7.1, -0.012345],
                      schedule=[0.1, 0.05, 0.25, 0.35, 0.5],
                      progress=[0.3, 1.2345e-6, 0.4, 1234, 3, 7])


def output_fixtures(ref: Oracle) -> None:
    """The reference's TrajectoryWriter (one frame) and writeCheckpoint files, as bytes."""
    import tempfile
    x, y, g, u, v = output_inputs()
    with tempfile.TemporaryDirectory() as tmp:
        traj = ref.write_trajectory(os.path.join(tmp, "trajectory.csv"), 0.3, 7, x, y, g, u, v)
        geo = Geometry(**OUTPUT_GEOMETRY)
        engine = ref.dipole_events(Geometry("periodic", box_length_x=2 * np.pi,
                                            box_length_y=2 * np.pi, dipole_removal=True,
                                            dipole_removal_distance=1e-3, random_seed=5),
                                   x, y, g)[4][2]
        r = OUTPUT_RECORDS
        ckpt = ref.write_checkpoint(tmp, geo, x, y, g, r["initial"], r["segment"],
                                    (2, 1, engine), r["schedule"], r["progress"])
    save("writers_periodic_n300.npz", x=x, y=y, g=g, u=u, v=v,
         trajectory=np.frombuffer(traj, dtype=np.uint8),
         checkpoint=np.frombuffer(ckpt, dtype=np.uint8), engine=np.array(engine))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PV_REFERENCE_DIR"),
                    help="the reference checkout (default: $PV_REFERENCE_DIR)")
    ap.add_argument("--only", choices=["dipole_events", "output", "dopri_workload"], default=None,
                    help="regenerate one fixture family only")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference <dir> or set PV_REFERENCE_DIR")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref",
                    f"REF={args.reference}"], check=True)
    ref = Oracle("reference")
    t0 = time.time()
    if args.only == "dipole_events":
        dipole_event_fixtures(ref)
        return 0
    if args.only == "output":
        output_fixtures(ref)
        return 0
    if args.only == "dopri_workload":
        dopri_workload_fixture(ref)
        return 0

    # small cases, all three geometries (+ the core-radius plane)
    for tag, geo, (x, y, g) in [
        ("infinite", Geometry("infinite"), ics.infinite_plane(64, 11)),
        ("infinite_core", Geometry("infinite", core_radius=0.05), ics.infinite_plane(64, 12)),
        ("periodic", Geometry("periodic", box_length_x=2.0, box_length_y=2.0),
         ics.periodic_box(64, 13, 2.0)),
        ("periodic_m3", Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=3),
         ics.periodic_box(64, 14, 2.0)),
        ("disk", Geometry("disk", disk_radius=1.0), ics.disk(64, 15, 1.0, 0.8, gaussian=False)),
    ]:
        small_case(ref, geo, x, y, g, tag)

    # the three single-simulation workloads at full size (target samples where the reference
    # CPU path is too slow for the full matrix)
    x, y, g = ics.workload_state("infinite_rk4_n1024")
    geo = Geometry("infinite")
    u, v = ref.evaluate(geo, x, y, g)
    inv = ref.invariants(geo, x, y, g)
    st = ref.stepper(geo, x.size)
    xs, ys = [x.copy()], [y.copy()]
    for _ in range(5):
        nx, ny = st.rk4_step(xs[-1], ys[-1], g, 1e-3)
        xs.append(nx)
        ys.append(ny)
    save("workload_infinite_n1024.npz", x=x, y=y, g=g, u=u, v=v, inv=inv, rk_x=np.array(xs),
         rk_y=np.array(ys))

    x, y, g = ics.workload_state("periodic_dopri5_n4096")
    geo = Geometry("periodic", box_length_x=2 * np.pi, box_length_y=2 * np.pi)
    u, v = ref.evaluate_range(geo, x, y, g, 0, 256)
    inv = ref.invariants(geo, x, y, g)
    save("workload_periodic_n4096.npz", x=x, y=y, g=g, u=u, v=v, inv=inv, targets=np.array([0, 256]))

    x, y, g = ics.workload_state("disk_rk4_n16384")
    geo = Geometry("disk", disk_radius=1.0)
    u, v = ref.evaluate_range(geo, x, y, g, 0, 256)
    inv = ref.invariants(geo, x, y, g)
    save("workload_disk_n16384.npz", x=x, y=y, g=g, u=u, v=v, inv=inv, targets=np.array([0, 256]))

    # close-dipole removal (removal only): states with planted close opposite-sign pairs
    rng = np.random.default_rng(16)
    for tag, geo, (x, y, g) in [
        ("periodic", Geometry("periodic", box_length_x=2.0, box_length_y=2.0,
                              dipole_removal=True, dipole_removal_distance=0.05),
         ics.periodic_box(200, 17, 2.0)),
        ("disk", Geometry("disk", disk_radius=1.0, dipole_removal=True,
                          dipole_removal_distance=0.05), ics.disk(200, 18, 1.0, 0.999, gaussian=False)),
        ("infinite", Geometry("infinite", dipole_removal=True, dipole_removal_distance=0.05),
         ics.infinite_plane(200, 19)),
    ]:
        x, y = x.copy(), y.copy()
        # move a few positive vortices next to negative ones (and across the periodic seam)
        pos = np.flatnonzero(g > 0)[:6]
        neg = np.flatnonzero(g < 0)[:6]
        for k, (a, b) in enumerate(zip(pos, neg)):
            x[a] = x[b] + 0.01 * (k + 1) * 0.5
            y[a] = y[b] - 0.004 * k
        if tag == "periodic":
            x[pos[5]], x[neg[5]] = 0.995, -0.997
            y[pos[5]] = y[neg[5]]
        events, sx, sy, sg = ref.dipole_process(geo, x, y, g)
        save(f"dipole_{tag}.npz", x=x, y=y, g=g, events=np.array([events]), sx=sx, sy=sy, sg=sg,
             threshold=np.array([geo.dipole_removal_distance]))
    dipole_event_fixtures(ref)
    output_fixtures(ref)
    dopri_workload_fixture(ref)
    print(f"done in {time.time() - t0:.1f} s")
    _ = rng
    return 0


if __name__ == "__main__":
    sys.exit(main())
