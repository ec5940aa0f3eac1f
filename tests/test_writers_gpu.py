"""Trajectory rows and checkpoint vortex blocks formatted on the GPU, byte for byte against the
reference's TrajectoryWriter / writeCheckpoint files (golden fixture) and, for the device-state
frame, against "%.17g" of the downloaded state and its device velocity."""
import os

import numpy as np
import pytest

import pointvortex_b200 as pv
from conftest import golden
from golden.make_golden import OUTPUT_RECORDS
from pointvortex_b200 import ics, output

pytestmark = pytest.mark.gpu


def fixture():
    d = golden("writers_periodic_n300.npz")
    return d, bytes(d["trajectory"]), bytes(d["checkpoint"])


def periodic_kernel():
    return pv.PeriodicBoxKernel(2 * np.pi, 2 * np.pi, 8)


def expected_rows(time, frame, x, y, g, u, v):
    g17 = output.g17
    return "".join(f"{g17(time)},{frame},{i},{g17(x[i])},{g17(y[i])},{g17(g[i])},{g17(u[i])},"
                   f"{g17(v[i])}\n" for i in range(x.size)).encode()


def test_host_frame_matches_reference_writer(tmp_path):
    d, traj, _ = fixture()
    k = periodic_kernel()
    s = pv.VortexSystem(d["x"], d["y"], d["g"])
    vel = pv.VelocityField(d["u"], d["v"])
    assert k.formatTrajectoryHost(0.3, 7, s, vel) == traj[len(output.TRAJECTORY_HEADER):]
    path = str(tmp_path / "run" / "trajectory.csv")
    w = output.TrajectoryWriter(path, False, k)
    w.write(0.3, 7, s, vel)
    w.close()
    assert open(path, "rb").read() == traj
    with pytest.raises(RuntimeError, match="refusing to overwrite output file"):
        output.TrajectoryWriter(path, False, k)


def test_checkpoint_matches_reference_writer(tmp_path):
    d, _, ckpt = fixture()
    k = periodic_kernel()
    k.uploadDeviceState(pv.VortexSystem(d["x"], d["y"], d["g"]))
    r = OUTPUT_RECORDS
    params = {"boundaryCondition": "periodic", "boxLengthX": 2 * np.pi, "boxLengthY": 2 * np.pi,
              "periodicImageLayers": 8, "coreRadius": 0.0, "integrator": "dopri5",
              "dipoleRemoval": True, "dipoleRemovalDistance": 1e-3, "dipoleReinjection": "none"}
    path = output.write_checkpoint(str(tmp_path), k, r["initial"], params, r["segment"],
                                   pv.DipoleEventState(2, 1, str(d["engine"])),
                                   output.OutputSchedule(*r["schedule"]),
                                   output.CheckpointProgress(*r["progress"]))
    assert os.path.basename(path) == "checkpoint_00000003.dat"
    assert open(path, "rb").read() == ckpt
    assert not os.path.exists(path + ".tmp")


@pytest.mark.parametrize("geometry,n", [("infinite", 1), ("infinite", 257), ("disk", 4096),
                                        ("periodic", 20000)])
def test_device_frame_is_exact(geometry, n):
    if geometry == "periodic":
        x, y, g = ics.periodic_box(n, 3)
        k = periodic_kernel()
    elif geometry == "disk":
        x, y, g = ics.disk(n, 4, 1.0, 0.95, gaussian=False)
        k = pv.DiskKernel(1.0)
    else:
        x, y, g = ics.infinite_plane(max(n, 2), 5)
        x, y, g = x[:n], y[:n], g[:n]
        k = pv.InfinitePlaneKernel(0.0)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    rows = k.formatTrajectory(1.5, 12)
    vel = k.evaluateDeviceState()
    assert rows == expected_rows(1.5, 12, x, y, g, vel.x, vel.y)
    block = k.formatCheckpointVortices()
    g17 = output.g17
    assert block == "".join(f"{g17(a)} {g17(b)} {g17(c)}\n" for a, b, c in zip(x, y, g)).encode()


def test_capacity_and_empty_state():
    k = pv.InfinitePlaneKernel(0.0)
    x, y, g = ics.infinite_plane(64, 6)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    import ctypes
    from pointvortex_b200._lib import lib
    buf = ctypes.create_string_buffer(16)
    length = ctypes.c_size_t(0)
    rc = lib.pv_format_trajectory(k._ctx, 0.0, 0, buf, 16, ctypes.byref(length))
    assert rc == 6 and length.value > 16  # PV_ERROR_CAPACITY, the needed size reported
    k.uploadDeviceState(pv.VortexSystem(np.zeros(0), np.zeros(0), np.zeros(0)))
    assert k.formatTrajectory(0.0, 0) == b"" and k.formatCheckpointVortices() == b""
