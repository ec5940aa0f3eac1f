"""Drop-in check of the whole executable: the reference's own driver linked with the B200 backend
(oracle/_ref/point_vortex_b200, built by `make -C oracle cli`) against the reference's CPU
executable (oracle/_ref/point_vortex_cpu) on identical parameter files and initial conditions.
Every field of trajectory.csv and diagnostics.csv must agree to rel 2e-10 / abs 2e-11, the
tolerance of the reference's own backend differential test (tests/backend_consistency.py:29-40)."""
import csv
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CPU = os.path.join(ROOT, "oracle", "_ref", "point_vortex_cpu")
B200 = os.path.join(ROOT, "oracle", "_ref", "point_vortex_b200")


def run(exe, directory, geometry, rows, end, integrator="rk4", extra=""):
    os.makedirs(directory)
    initial = os.path.join(directory, "initial.dat")
    with open(initial, "w") as f:
        f.write("".join(f"{x:.17g} {y:.17g} {g:.17g}\n" for x, y, g in rows))
    params = os.path.join(directory, "run.params")
    with open(params, "w") as f:
        f.write(f"initialConditionFile {initial}\nboundaryCondition {geometry}\nendTime {end}\n"
                f"integrator {integrator}\ntimeStep 0.001\noutputTime 0.002\ndiagnosticsTime 0.001\n"
                f"checkpointTime 0.003\nnumThreads 2\nrunDirectory {directory}\n{extra}")
    r = subprocess.run([exe, params], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def compare(a, b):
    with open(a) as f:
        left = list(csv.DictReader(f))
    with open(b) as f:
        right = list(csv.DictReader(f))
    assert len(left) == len(right) and len(left) > 0
    for p, q in zip(left, right):
        assert p.keys() == q.keys()
        for key in p:
            x, y = float(p[key]), float(q[key])
            assert math.isfinite(x) and math.isfinite(y)
            assert math.isclose(x, y, rel_tol=2e-10, abs_tol=2e-11), (a, key, x, y)


ORDINARY = [(-0.31, -0.12, 1.0), (0.23, 0.14, -1.0), (0.11, -0.29, 2.0), (-0.14, 0.32, -2.0)]


def crowd(n=258, seed=1234):
    rng = np.random.default_rng(seed)
    return [(float(rng.uniform(-0.4, 0.4)), float(rng.uniform(-0.4, 0.4)), 1.0 if i % 2 == 0 else -1.0)
            for i in range(n)]


CASES = (
    [(f"{g}_rk4", g, ORDINARY, 0.003, "rk4") for g in ("infinite", "periodic", "disk")]
    + [(f"{g}_crowd", g, crowd(), 0, "rk4") for g in ("infinite", "periodic", "disk")]
    + [("periodic_close", "periodic", [(0.0, 0.0, 1.0), (1e-10, 0.0, -1.0)], 0, "rk4"),
       ("disk_center", "disk", [(0.2, 0.0, 1.0), (1e-155, 0.0, 1.0)], 0, "rk4")]
    + [(f"{g}_dopri5", g, ORDINARY, 0.003, "dopri5") for g in ("infinite", "periodic", "disk")]
)


@pytest.mark.skipif(not (os.path.exists(CPU) and os.path.exists(B200)),
                    reason="oracle/_ref executables not built")
@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_cli_matches_reference_cpu(tmp_path, case):
    name, geometry, rows, end, integrator = case
    left, right = str(tmp_path / "cpu"), str(tmp_path / "b200")
    run(CPU, left, geometry, rows, end, integrator)
    out = run(B200, right, geometry, rows, end, integrator)
    assert "backend=CUDA/B200" in out.stdout
    for name in ("trajectory.csv", "diagnostics.csv"):
        compare(os.path.join(left, name), os.path.join(right, name))


@pytest.mark.skipif(not (os.path.exists(CPU) and os.path.exists(B200)),
                    reason="oracle/_ref executables not built")
def test_cli_dipole_removal_and_restart(tmp_path):
    """A periodic run with close-dipole removal and a restart from its checkpoint, both through the
    reference driver (checkpoint v6 format, schedules, event counters) on the B200 backend."""
    rows = [(float(x), float(y), g) for x, y, g in
            zip(*np.random.default_rng(3).uniform(-0.5, 0.5, (2, 40)), [1.0, -1.0] * 20)]
    rows[1] = (rows[0][0] + 0.004, rows[0][1], -1.0)
    extra = "boxLengthX 1.0\nboxLengthY 1.0\ndipoleRemoval true\ndipoleRemovalDistance 0.01\n"
    left, right = str(tmp_path / "cpu"), str(tmp_path / "b200")
    run(CPU, left, "periodic", rows, 0.006, "dopri5", extra)
    run(B200, right, "periodic", rows, 0.006, "dopri5", extra)
    for name in ("trajectory.csv", "diagnostics.csv"):
        compare(os.path.join(left, name), os.path.join(right, name))
    with open(os.path.join(right, "diagnostics.csv")) as f:
        last = list(csv.DictReader(f))[-1]
    assert int(last["removed_pairs"]) >= 1
    ckpt = sorted(os.listdir(os.path.join(right, "checkpoints")))[1]
    restart = str(tmp_path / "b200_restart")
    os.makedirs(restart)
    params = os.path.join(restart, "run.params")
    with open(params, "w") as f:
        f.write(f"boundaryCondition periodic\nintegrator dopri5\nendTime 0.009\ntimeStep 0.001\n"
                f"outputTime 0.002\ndiagnosticsTime 0.001\ncheckpointTime 0.003\n{extra}"
                f"restartFile {os.path.join(right, 'checkpoints', ckpt)}\nrunDirectory {restart}\n")
    r = subprocess.run([B200, params], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


PLUGIN_DIPOLES = os.path.join(ROOT, "oracle", "_ref", "plugin_dipoles")


@pytest.mark.skipif(not os.path.exists(PLUGIN_DIPOLES), reason="make -C oracle plugin-test")
def test_backend_dipole_hook_matches_reference_manager():
    """b200ProcessDipoles through the backend translation unit against the reference's host
    DipoleManager: removal, independent and paired reinjection, periodic box and disk, three
    consecutive calls each."""
    r = subprocess.run([PLUGIN_DIPOLES], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout + r.stderr
