"""Writers in the reference's formats, host side: the checkpoint header lines and the row layout
that the GPU formatter must reproduce, against the reference's own TrajectoryWriter and
writeCheckpoint output (golden fixture)."""
import numpy as np

from conftest import golden
from golden.make_golden import OUTPUT_GEOMETRY, OUTPUT_RECORDS
from pointvortex_b200 import output


def fixture():
    d = golden("writers_periodic_n300.npz")
    return d, bytes(d["trajectory"]), bytes(d["checkpoint"])


def test_trajectory_rows_are_percent_17g():
    """The reference's frame is exactly "%.17g" per double (the formatter's contract)."""
    d, traj, _ = fixture()
    rows = [f"{output.g17(0.3)},7,{i},{output.g17(d['x'][i])},{output.g17(d['y'][i])},"
            f"{output.g17(d['g'][i])},{output.g17(d['u'][i])},{output.g17(d['v'][i])}\n"
            for i in range(d["x"].size)]
    assert traj == output.TRAJECTORY_HEADER + "".join(rows).encode()


def test_checkpoint_header_matches_reference():
    d, _, ckpt = fixture()
    r = OUTPUT_RECORDS
    params = {"boundaryCondition": "periodic", "boxLengthX": OUTPUT_GEOMETRY["box_length_x"],
              "boxLengthY": OUTPUT_GEOMETRY["box_length_y"], "periodicImageLayers": 8,
              "coreRadius": 0.0, "integrator": "dopri5", "dipoleRemoval": True,
              "dipoleRemovalDistance": 1e-3, "dipoleReinjection": "none"}
    head = output.checkpoint_header(
        d["x"].size, r["initial"], params, r["segment"],
        output.DipoleEventState(2, 1, str(d["engine"])), output.OutputSchedule(*r["schedule"]),
        output.CheckpointProgress(*r["progress"]))
    assert ckpt.startswith(head)
    rows = "".join(f"{output.g17(a)} {output.g17(b)} {output.g17(c)}\n"
                   for a, b, c in zip(d["x"], d["y"], d["g"])).encode()
    assert ckpt == head + rows


def test_g17_nan_sign():
    assert output.g17(float("nan")) == "nan"
    assert output.g17(np.copysign(float("nan"), -1.0)) == "-nan"
