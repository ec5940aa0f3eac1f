"""Batched ensembles (pv_batch_*): every simulation advances with its own DOPRI5 step and end
time, its result is bit-identical alone and in any mix, one failing simulation leaves the others
untouched, and each result agrees with the oracle's driver loop."""
import numpy as np
import pytest

from conftest import position_error
from oracle.pyoracle import Geometry
from pointvortex_b200 import ics
from pointvortex_b200.batch import Batch, CapacityError, geometry_params

pytestmark = pytest.mark.gpu

SOLVE = dict(dt=1e-3, atol=1e-10, rtol=1e-8, dtmin=1e-12, dtmax=0.1)


def specs():
    return [
        ("infinite", 300, 1, 0.004),
        ("periodic", 256, 2, 0.003),
        ("disk", 600, 23, 0.002),
        ("infinite", 1000, 4, 0.001),
        ("periodic", 1024, 5, 0.002),
        ("disk", 64, 6, 0.005),
    ]


def state(boundary, n, seed):
    if boundary == "periodic":
        return ics.periodic_box(n, seed, 2.0 * np.pi)
    if boundary == "disk":
        return ics.disk(n, seed, 1.0, 0.8, gaussian=False)
    return ics.infinite_plane(n, seed)


def run_batch(items, capacity=20000, slots=16, **kw):
    """items: (boundary, n, seed, t_end[, precision])."""
    b = Batch(capacity, slots)
    ids = []
    for item in items:
        boundary, n, seed, t_end = item[:4]
        precision = item[4] if len(item) > 4 else "fp64"
        x, y, g = state(boundary, n, seed)
        ids.append(b.add(geometry_params(boundary, precision=precision), x, y, g, t_end,
                         **{**SOLVE, **kw}))
    b.run()
    out = [(b.info(i), b.result(i)) for i in ids]
    b.close()
    return out


def test_alone_equals_in_the_mix():
    mixed = run_batch(specs())
    for k, spec in enumerate(specs()):
        (info_a, (xa, ya)) = run_batch([spec])[0]
        info_m, (xm, ym) = mixed[k]
        assert info_a.state == "done" and info_m.state == "done", (spec, info_a, info_m)
        assert info_a.acceptedSteps == info_m.acceptedSteps
        assert np.array_equal(xa, xm) and np.array_equal(ya, ym), spec


def oracle_driver(oracle, boundary, n, seed, t_end):
    """The reference driver's DOPRI5 loop (src/main.cpp:159-164, 310-343) without output events."""
    geo = Geometry(boundary, box_length_x=2 * np.pi, box_length_y=2 * np.pi, disk_radius=1.0,
                   absolute_tolerance=SOLVE["atol"], relative_tolerance=SOLVE["rtol"],
                   minimum_time_step=SOLVE["dtmin"], maximum_time_step=SOLVE["dtmax"])
    x, y, g = state(boundary, n, seed)
    st = oracle.stepper(geo, n)
    t, dt, steps = 0.0, min(max(SOLVE["dt"], SOLVE["dtmin"]), SOLVE["dtmax"]), 0
    while t < t_end:
        x, y, r = st.dopri5_step(x, y, g, min(dt, t_end - t))
        t += r[0]
        dt = r[1]
        steps += 1
        if t + 16 * np.finfo(float).eps * abs(t) >= t_end:
            t = t_end
    return x, y, steps


def test_batch_matches_oracle_driver(reference):
    """Against the unmodified reference's integrator (OpenMP-parallel, so the periodic cases stay
    affordable on the host)."""
    results = run_batch(specs())
    for spec, (info, (x, y)) in zip(specs(), results):
        rx, ry, steps = oracle_driver(reference, *spec)
        assert info.acceptedSteps == steps, (spec, info)
        assert info.time == spec[3]
        # hundreds of chaotic steps: the 1e-16 per-evaluation differences grow, but stay small
        assert position_error(x, y, rx, ry) <= 1e-9, spec


def test_failure_is_isolated():
    good = specs()[:3]
    alone = run_batch(good)
    b = Batch(20000, 8)
    ids = []
    for boundary, n, seed, t_end in good[:2]:
        ids.append(b.add(geometry_params(boundary), *state(boundary, n, seed), t_end, **SOLVE))
    # a disk vortex next to the wall with a strong partner: leaves the disk within a few steps
    bad = b.add(geometry_params("disk"), np.array([0.9999, -0.2]), np.array([0.0, 0.0]),
                np.array([1.0, 50.0]), 1.0, **SOLVE)
    boundary, n, seed, t_end = good[2]
    ids.append(b.add(geometry_params(boundary), *state(boundary, n, seed), t_end, **SOLVE))
    b.run()
    assert b.info(bad).state == "failed" and b.info(bad).status != 0
    for k, sid in enumerate(ids):
        x, y = b.result(sid)
        assert b.info(sid).state == "done", (k, b.info(sid))
        assert np.array_equal(x, alone[k][1][0]) and np.array_equal(y, alone[k][1][1])


def test_step_budget_and_release():
    # arena room: 1280 requested + 256 per slot = 1792 vortices, in 256-element blocks
    b = Batch(1200, 2)
    x, y, g = state("infinite", 500, 9)
    sid = b.add(geometry_params("infinite"), x, y, g, 10.0, max_steps=3, **SOLVE)
    b.run()
    info = b.info(sid)
    assert info.state == "budget" and info.acceptedSteps == 3
    with pytest.raises(CapacityError):
        b.add(geometry_params("infinite"), *state("infinite", 1500, 1), 1.0, **SOLVE)
    b.release(sid)
    b.add(geometry_params("infinite"), *state("infinite", 1500, 1), 0.0005, **SOLVE)
    assert b.run() >= 1


def test_admission_validation():
    b = Batch(5000, 2)
    x, y, g = state("periodic", 100, 1)
    g = g.copy()
    g[0] += 1.0
    with pytest.raises(ValueError, match="zero total circulation"):
        b.add(geometry_params("periodic"), x, y, g, 0.01, **SOLVE)


def mixed_forms():
    """Periodic from N = 2048 runs once per unordered pair (both forms); fp32c items drain their
    own queue in a second launch per stage."""
    return [
        ("periodic", 2100, 7, 0.0004),
        ("periodic", 2200, 13, 0.0004, "fp32c"),
        ("infinite", 700, 8, 0.002, "fp32c"),
        ("periodic", 512, 9, 0.002, "fp32c"),
        ("disk", 600, 15, 0.002, "fp32c"),
        ("infinite", 500, 11, 0.002),
    ]


def test_alone_equals_in_the_mix_across_forms():
    mixed = run_batch(mixed_forms(), capacity=40000)
    for k, spec in enumerate(mixed_forms()):
        (info_a, (xa, ya)) = run_batch([spec], capacity=40000)[0]
        info_m, (xm, ym) = mixed[k]
        assert info_a.state == "done" and info_m.state == "done", (spec, info_a, info_m)
        assert info_a.acceptedSteps == info_m.acceptedSteps
        assert np.array_equal(xa, xm) and np.array_equal(ya, ym), spec


def test_symmetric_batch_matches_oracle_driver(reference):
    spec = mixed_forms()[0]
    (info, (x, y)), = run_batch([spec], capacity=40000)
    rx, ry, steps = oracle_driver(reference, *spec)
    assert info.acceptedSteps == steps, info
    assert position_error(x, y, rx, ry) <= 1e-9


def test_fp32c_batch_tracks_fp64():
    """The compensated form against the plain form over the same solves: FP32-level terms move
    the vortices by ~1e-7 at most over these few steps."""
    forms = [s for s in mixed_forms() if len(s) > 4]
    fp32 = run_batch(forms, capacity=40000)
    fp64 = run_batch([s[:4] for s in forms], capacity=40000)
    for spec, (i32, (x32, y32)), (i64, (x64, y64)) in zip(forms, fp32, fp64):
        assert i32.state == i64.state == "done", spec
        assert np.max(np.hypot(x32 - x64, y32 - y64)) < 1e-6, spec


@pytest.fixture
def batch_table():
    """Sets batch table entries (pv_set_batch_tuning) and restores the values in effect before."""
    from pointvortex_b200 import autotune
    saved = {}

    def set_entry(boundary, precision, n, per_thread):
        key = (autotune.GEOMETRIES[boundary], autotune.PRECISIONS[precision], n.bit_length() - 1)
        saved.setdefault(key, autotune.get_batch_entry(*key))
        autotune.set_batch_entry(*key, per_thread)

    yield set_entry
    for key, value in saved.items():
        autotune.set_batch_entry(*key, value)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_batch_table_sets_targets_per_thread(batch_table, precision):
    """An entry of the batch table changes the simulation's work items (targets per thread of its
    ordered items) and, where every tile runs the same pair arithmetic, nothing of its result: a
    target's sum over a chunk runs over the same sources in the same order for any T. The FP32C
    disk's tiles that hold the target block itself take the scalar pair form, so its result moves
    within the compensated form's own error when the block size changes: the bound is the one
    test_fp32c_batch_tracks_fp64 holds it to against FP64 (a vortex near the wall moved 1.1e-7
    between 2 and 4 targets per thread, the others 1e-10)."""
    cases = [("infinite", 1000, 4, 0.002, (1, 2, 4)), ("periodic", 700, 5, 0.002, (1, 2)),
             ("disk", 600, 15, 0.002, (1, 2, 4))]
    for boundary, n, seed, t_end, cands in cases:
        runs = {}
        for t in cands:
            batch_table(boundary, precision, n, t)
            (info, (x, y)), = run_batch([(boundary, n, seed, t_end, precision)])
            assert info.state == "done" and info.targetsPerThread == t, (boundary, t, info)
            runs[t] = (info.acceptedSteps, x, y)
        steps0, x0, y0 = runs[cands[0]]
        for t in cands[1:]:
            steps, x, y = runs[t]
            if precision == "fp32c" and boundary == "disk":
                assert np.max(np.hypot(x - x0, y - y0)) < 1e-6, (boundary, t)
            else:
                assert steps == steps0 and np.array_equal(x, x0) and np.array_equal(y, y0), \
                    (boundary, precision, t)


def test_batch_table_skips_the_symmetric_items(batch_table):
    """Periodic FP64 simulations from N = 2048 take the once-per-unordered-pair items, which hold
    no targets per thread: their info reports 0 whatever the table says."""
    batch_table("periodic", "fp64", 2100, 2)
    (info, _), = run_batch([("periodic", 2100, 7, 0.0004)], capacity=40000)
    assert info.state == "done" and info.targetsPerThread == 0
