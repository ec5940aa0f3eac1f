"""The allocation-free entry point, pv_evaluate_device_noalloc, through the C ABI.

It is meant for callers that cannot allocate GPU memory (a host that owns all device memory in
its own pool, a stepping loop that cannot afford cudaMalloc's synchronisation): they pass device
arrays they already own, and the library's scratch is one fixed device array. The test hands it
device arrays (allocated here by torch, as such a host would by its own means) and checks that
its velocities agree with the context-based pv_evaluate entry point, within the same per-vortex
tolerance as the other parity tests, on two calls in a row (the second call must not see the first
call's leftovers in the shared scratch array). This file is collected last on purpose."""
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


def _noalloc(params, x, y, g):
    import torch
    from pointvortex_b200._lib import lib
    dev = torch.device("cuda", 0)
    tx, ty, tg = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (x, y, g))
    tu = torch.empty_like(tx)
    tv = torch.empty_like(tx)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.pv_evaluate_device_noalloc(ctypes.byref(params), tx.data_ptr(), ty.data_ptr(),
                                        tg.data_ptr(), x.size, tu.data_ptr(), tv.data_ptr(),
                                        ctypes.c_void_p(stream))
    if rc != 0:
        raise RuntimeError(lib.pv_last_error(None).decode())
    torch.cuda.synchronize(dev)
    return tu.cpu().numpy(), tv.cpu().numpy()


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
def test_noalloc_matches_context_entry_point_twice(case):
    name, (x, y, g), kw = _states()[case]
    params = _params(kw)
    ur, vr = _with_context(kw, x, y, g)
    u1, v1 = _noalloc(params, x, y, g)
    assert normalized_error(u1, v1, ur, vr).max() <= TOL
    # second call in a row, on a different state of a different size
    x2, y2, g2 = x[: x.size // 2].copy(), y[: x.size // 2].copy(), g[: x.size // 2].copy()
    if name == "periodic":
        g2[-1] = -g2[:-1].sum()
    ur2, vr2 = _with_context(kw, x2, y2, g2)
    u2, v2 = _noalloc(params, x2, y2, g2)
    assert normalized_error(u2, v2, ur2, vr2).max() <= TOL


def test_noalloc_rejects_populations_beyond_its_scratch():
    from pointvortex_b200._lib import lib
    limit = 349440
    params = _params(dict(geometry=0))
    rc = lib.pv_evaluate_device_noalloc(ctypes.byref(params), None, None, None, limit + 1, None,
                                        None, None)
    assert rc == 1
    assert "exceeds the allocation-free limit" in lib.pv_last_error(None).decode()
