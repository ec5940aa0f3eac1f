"""The allocation-free entry point, pv_evaluate_device_noalloc, through the C ABI.

It serves callers that cannot allocate GPU memory: a host that owns every byte of device memory
through its own pool and hands out only buffers it placed, or a stepping loop that cannot afford
the device-wide synchronisation of cudaMalloc/cudaFree. They pass device arrays they already own;
the library's scratch is one fixed device array. The tests hand it device arrays (allocated here by
torch, as such a host would by its own means) and check, on two calls in a row (the second call
must not see the first call's leftovers in the shared scratch array):

* its velocities against the oracle (the C restatement of the reference) and against the
  context-based pv_evaluate entry point, within the per-vortex tolerance of the other parity
  tests;
* every input and evaluation error against the oracle's exception kind and message, in the
  reference's order (non-finite data, then the box's zero net circulation or the disk's wall, then
  the evaluation's coincident pair), with u and v left untouched by an input error.

This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from conftest import normalized_error

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _states():
    from pointvortex_b200 import ics
    return [
        ("infinite", ics.infinite_plane(3000, 5), dict(geometry=0, core_radius=0.0)),
        ("periodic", ics.periodic_box(1024, 6, 2.0), dict(geometry=1, box_length_x=2.0,
                                                           box_length_y=2.0, image_layers=8)),
        ("disk", ics.disk(2049, 7, 1.0, 0.95), dict(geometry=2, disk_radius=1.0)),
    ]


def _geometry(kw):
    from oracle.pyoracle import Geometry
    name = {0: "infinite", 1: "periodic", 2: "disk"}[kw["geometry"]]
    return Geometry(name, core_radius=kw.get("core_radius", 0.0),
                    box_length_x=kw.get("box_length_x", 2.0),
                    box_length_y=kw.get("box_length_y", 2.0),
                    image_layers=kw.get("image_layers", 8), disk_radius=kw.get("disk_radius", 1.0))


def _params(kw):
    from pointvortex_b200 import _lib
    p = _lib.PvParams()
    p.geometry = kw["geometry"]
    p.core_radius = kw.get("core_radius", 0.0)
    p.box_length_x = kw.get("box_length_x", 2.0)
    p.box_length_y = kw.get("box_length_y", 2.0)
    p.image_layers = kw.get("image_layers", 8)
    p.disk_radius = kw.get("disk_radius", 1.0)
    p.precision = 0
    return p


SENTINEL = 12345.0


def _noalloc(params, x, y, g):
    """(rc, message, u, v); u and v start as SENTINEL so an untouched output is visible."""
    import torch
    from pointvortex_b200._lib import lib
    dev = torch.device("cuda", 0)
    tx, ty, tg = (torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
                  for a in (x, y, g))
    tu = torch.full_like(tx, SENTINEL)
    tv = torch.full_like(tx, SENTINEL)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.pv_evaluate_device_noalloc(ctypes.byref(params), tx.data_ptr(), ty.data_ptr(),
                                        tg.data_ptr(), len(x), tu.data_ptr(), tv.data_ptr(),
                                        ctypes.c_void_p(stream))
    msg = lib.pv_last_error(None).decode() if rc != 0 else ""
    torch.cuda.synchronize(dev)
    return rc, msg, tu.cpu().numpy(), tv.cpu().numpy()


def _with_context(kw, x, y, g):
    import pointvortex_b200 as pv
    k = pv.VelocityKernel(kw["geometry"], core_radius=kw.get("core_radius", 0.0),
                          box_length_x=kw.get("box_length_x", 2.0),
                          box_length_y=kw.get("box_length_y", 2.0),
                          image_layers=kw.get("image_layers", 8),
                          disk_radius=kw.get("disk_radius", 1.0))
    f = k.evaluate(x, y, g)
    k.close()
    return f.x, f.y


@pytest.mark.parametrize("case", range(3), ids=["infinite", "periodic", "disk"])
def test_noalloc_matches_oracle_and_context_entry_point_twice(case, port):
    name, (x, y, g), kw = _states()[case]
    params = _params(kw)
    geo = _geometry(kw)
    x2, y2, g2 = x[: x.size // 2].copy(), y[: x.size // 2].copy(), g[: x.size // 2].copy()
    if name == "periodic":
        g2[-1] = -g2[:-1].sum()
    # two calls in a row, the second on a different state of a different size
    for xs, ys, gs in ((x, y, g), (x2, y2, g2)):
        uo, vo = port.evaluate(geo, xs, ys, gs)
        rc, msg, u, v = _noalloc(params, xs, ys, gs)
        assert rc == 0, msg
        assert normalized_error(u, v, uo, vo).max() <= TOL
        ur, vr = _with_context(kw, xs, ys, gs)
        assert normalized_error(u, v, ur, vr).max() <= TOL


def _oracle_error(port, geo, x, y, g):
    try:
        port.evaluate(geo, x, y, g)
    except Exception as exc:  # noqa: BLE001 -- the kind is compared below
        return type(exc), str(exc)
    return None, ""


def _error_cases():
    from pointvortex_b200 import ics
    box = dict(geometry=1, box_length_x=2.0, box_length_y=2.0, image_layers=8)
    disk = dict(geometry=2, disk_radius=1.0)
    plane = dict(geometry=0, core_radius=0.0)
    cases = []
    x, y, g = ics.periodic_box(256, 11, 2.0)
    gn = g.copy()
    gn[0] += 1e-3  # net circulation far above 1e-12 * max(1, sum |Gamma|)
    cases.append(("box-not-neutral", box, x, y, gn))
    xc, yc = x.copy(), y.copy()
    xc[5], yc[5] = xc[9], yc[9]  # a coincident pair as well: neutrality is reported first
    cases.append(("box-not-neutral-and-coincident", box, xc, yc, gn))
    cases.append(("box-coincident", box, xc, yc, g))
    xf = x.copy()
    xf[3] = np.nan  # non-finite data precedes the neutrality check
    cases.append(("box-nonfinite-and-not-neutral", box, xf, y, gn))
    xd, yd, gd = ics.disk(300, 12, 1.0, 0.9)
    xo = xd.copy()
    xo[7] = 1.0  # on the wall
    cases.append(("disk-outside", disk, xo, yd, gd))
    xp, yp, gp = ics.infinite_plane(200, 13)
    xq, yq = xp.copy(), yp.copy()
    xq[4], yq[4] = xq[8], yq[8]
    cases.append(("plane-coincident", plane, xq, yq, gp))
    gi = gp.copy()
    gi[2] = np.inf
    cases.append(("plane-nonfinite-circulation", plane, xp, yp, gi))
    return cases


_EXPECTED_RC = {ValueError: 1, RuntimeError: 3}


ERROR_CASES = ["box-not-neutral", "box-not-neutral-and-coincident", "box-coincident",
               "box-nonfinite-and-not-neutral", "disk-outside", "plane-coincident",
               "plane-nonfinite-circulation"]


@pytest.mark.parametrize("case", range(len(ERROR_CASES)), ids=ERROR_CASES)
def test_noalloc_errors_match_oracle_twice(case, port):
    name, kw, x, y, g = _error_cases()[case]
    assert name == ERROR_CASES[case]
    kind, text = _oracle_error(port, _geometry(kw), x, y, g)
    assert kind is not None, f"{name}: the oracle accepted the state"
    params = _params(kw)
    for _ in range(2):
        rc, msg, u, v = _noalloc(params, x, y, g)
        assert rc == _EXPECTED_RC[kind], (name, rc, msg, kind, text)
        assert msg == text, (name, msg, text)
        if kind is ValueError:  # input errors are found before any evaluation
            assert np.all(u == SENTINEL) and np.all(v == SENTINEL), name
    # a valid call right after the failed ones starts from a clean status word
    _, (xs, ys, gs), kw_ok = _states()[1]
    rc, msg, u, v = _noalloc(_params(kw_ok), xs, ys, gs)
    assert rc == 0, msg
    uo, vo = port.evaluate(_geometry(kw_ok), xs, ys, gs)
    assert normalized_error(u, v, uo, vo).max() <= TOL


def test_noalloc_rejects_populations_beyond_its_scratch():
    from pointvortex_b200._lib import lib
    limit = 349440
    params = _params(dict(geometry=0))
    rc = lib.pv_evaluate_device_noalloc(ctypes.byref(params), None, None, None, limit + 1, None,
                                        None, None)
    assert rc == 1
    assert "exceeds the allocation-free limit" in lib.pv_last_error(None).decode()
