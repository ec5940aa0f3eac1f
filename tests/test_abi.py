"""The C ABI library without a GPU: it loads, exports every function include/pvb200.h declares,
and fails cleanly (a CUDA error status and message, no crash) when no device is present."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pvb200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pv_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ["pv_context_create", "pv_context_destroy", "pv_last_error", "pv_evaluate",
                     "pv_evaluate_range", "pv_hamiltonian", "pv_invariants", "pv_upload_state",
                     "pv_download_state", "pv_evaluate_state", "pv_rk4_step", "pv_dopri5_step",
                     "pv_invalidate_derivative", "pv_state_invariants", "pv_dipole_scan"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    from pointvortex_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_backend_name():
    import pointvortex_b200 as pv
    assert pv.backendName() == "CUDA/B200"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device failure path")
def test_context_creation_without_device_is_a_clean_error():
    import pointvortex_b200 as pv
    with pytest.raises(pv.CudaError):
        pv.InfinitePlaneKernel()


def test_parameter_validation_precedes_device_access():
    """The kernel constructors' checks (src/compute.cpp:50-56, 165-173, 258-261) run on the host
    and raise ValueError even on a machine without a GPU."""
    import pointvortex_b200 as pv
    cases = [(lambda: pv.InfinitePlaneKernel(-1.0), "core radius is negative"),
             (lambda: pv.PeriodicBoxKernel(2.0, 2.0, 65), "invalid periodic-box parameters"),
             (lambda: pv.PeriodicBoxKernel(2.0, 2.5), "requires a square periodic box"),
             (lambda: pv.DiskKernel(0.0), "invalid disk parameters")]
    for make, message in cases:
        with pytest.raises(ValueError, match=message):
            make()


def test_symmetric_tuning_table_round_trip_and_validation():
    """The symmetric-form table (pv_set_symmetric_tuning) stores what it accepts, rejects entries
    the planner cannot honour, and mode 0 restores the built-in plan. Host-only: no device."""
    from pointvortex_b200 import autotune
    periodic, plane, fp64, fp32c = 1, 0, 0, 1
    saved = [autotune.get_symmetric_entry(periodic, fp64, 12),
             autotune.get_symmetric_entry(plane, fp32c, 15)]
    try:
        autotune.set_symmetric_entry(periodic, fp64, 12, 2, 8, 0)
        assert autotune.get_symmetric_entry(periodic, fp64, 12) == (2, 8, 0)
        autotune.set_symmetric_entry(plane, fp32c, 15, 2, 0, 8)
        assert autotune.get_symmetric_entry(plane, fp32c, 15) == (2, 0, 8)
        autotune.set_symmetric_entry(periodic, fp64, 12, 2, 0, 2)
        assert autotune.get_symmetric_entry(periodic, fp64, 12) == (2, 0, 2)
        autotune.set_symmetric_entry(periodic, fp64, 12, 1)
        assert autotune.get_symmetric_entry(periodic, fp64, 12) == (1, 0, 0)
        for bad in [(2, fp64, 12, 2, 0, 0),        # the disk has no symmetric form
                    (periodic, fp32c, 12, 2, 8, 0),  # occupancy variants: periodic FP64 only
                    (plane, fp64, 15, 2, 0, 3),      # plane targets: 4 or 8
                    (periodic, fp64, 12, 2, 8, 2),   # periodic two targets: no occupancy variant
                    (periodic, fp32c, 12, 2, 0, 2),  # ... and FP64 only
                    (periodic, fp64, 12, 3, 0, 0)]:  # modes 0..2
            with pytest.raises(ValueError):
                autotune.set_symmetric_entry(*bad)
        autotune.set_symmetric_entry(periodic, fp64, 12, 0)
        assert autotune.get_symmetric_entry(periodic, fp64, 12) == (0, 0, 0)
    finally:
        autotune.set_symmetric_entry(periodic, fp64, 12, *saved[0])
        autotune.set_symmetric_entry(plane, fp32c, 15, *saved[1])


def test_symmetric_grid_table_round_trip_and_validation():
    """The symmetric form's grid table (pv_set_symmetric_grid): CTAs per SM per geometry,
    precision and N bucket, 0 for as many as fit; out-of-range entries are rejected. Host-only."""
    from pointvortex_b200 import autotune
    saved = autotune.get_symmetric_grid(1, 0, 12)
    try:
        autotune.set_symmetric_grid(1, 0, 12, 5)
        assert autotune.get_symmetric_grid(1, 0, 12) == 5
        for bad in [(2, 0, 12, 5), (1, 2, 12, 5), (1, 0, 40, 5), (1, 0, 12, -1), (1, 0, 12, 17)]:
            with pytest.raises(ValueError):
                autotune.set_symmetric_grid(*bad)
        autotune.set_symmetric_grid(1, 0, 12, 0)
        assert autotune.get_symmetric_grid(1, 0, 12) == 0
    finally:
        autotune.set_symmetric_grid(1, 0, 12, saved)


def test_batch_tuning_table_round_trip_and_validation():
    """The batch table (pv_set_batch_tuning): targets per thread of the ordered work items per
    geometry, precision and N bucket; 0 restores the default (plane 4, box 1, disk 2), and the
    box takes no 4. pv_get_batch_tuning returns the value in effect. Host-only."""
    from pointvortex_b200 import autotune
    keys = [(0, 0, 10), (1, 1, 9), (2, 0, 12)]
    saved = [autotune.get_batch_entry(*k) for k in keys]
    try:
        for k, default in zip(keys, (4, 1, 2)):
            autotune.set_batch_entry(*k, 0)
            assert autotune.get_batch_entry(*k) == default
        for k, t in zip(keys, (1, 2, 4)):
            autotune.set_batch_entry(*k, t)
            assert autotune.get_batch_entry(*k) == t
        for bad in [(1, 0, 10, 4), (0, 0, 10, 3), (3, 0, 10, 1), (0, 2, 10, 1), (0, 0, 40, 1),
                    (0, 0, -1, 1)]:
            with pytest.raises(ValueError):
                autotune.set_batch_entry(*bad)
    finally:
        for k, t in zip(keys, saved):
            autotune.set_batch_entry(*k, t)


def test_batch_tuner_sizes_its_batches():
    """The batch tuner's batches admit their simulations: per simulation pad(N) = N rounded up
    to 256 arena elements and pad(N) x rows partial elements, rows = ceil(N/128) for the
    once-per-unordered-pair items or ceil(N/chunk) for ordered ones (chunk 512 up to N = 16384,
    then N/32 rounded up to 512), against the arena and the partial buffer (arena x chunks)."""
    from pointvortex_b200 import autotune
    for log2_n in range(5, 17):
        for n in (1 << log2_n, (1 << log2_n) + 77):
            sims, vortices, chunks = autotune.batch_room(n)
            pad = -(-n // 256) * 256
            chunk = 512 if n <= 16384 else -(-(n // 32) // 512) * 512
            rows = max(-(-n // 128), -(-n // chunk))
            assert sims * pad <= vortices
            assert sims * pad * rows <= vortices * chunks
            assert sims * n * n <= max(1 << 26, n * n)


def test_kernel_stats_struct_matches_the_header():
    """The ctypes mirror of pv_kernel_stats holds PV_KERNEL_KINDS entries per array."""
    from pointvortex_b200 import _lib
    text = open(HEADER).read()
    kinds = int(re.search(r"#define PV_KERNEL_KINDS (\d+)", text).group(1))
    assert len(_lib.KERNEL_KINDS) == kinds
    assert ctypes.sizeof(_lib.PvKernelStats) == kinds * 3 * 8


def test_committed_tuning_table_loads_every_field():
    """The package's tuning.json (the autotuner's output) applies each of its entries: targets per
    thread, the symmetric form's choice and its grid size. Host-only."""
    import json

    from pointvortex_b200 import autotune
    with open(autotune.DEFAULT_PATH) as f:
        table = json.load(f)
    assert autotune.load() == sum(len(table.get(k, [])) for k in ("entries", "symmetric", "batch"))
    for e in table["entries"]:
        got = autotune.get_entry(autotune.GEOMETRIES[e["geometry"]],
                                 autotune.PRECISIONS[e["precision"]], e["log2_n"])
        assert got == e["per_thread"], e
    for e in table["symmetric"]:
        geo, prec = autotune.GEOMETRIES[e["geometry"]], autotune.PRECISIONS[e["precision"]]
        assert autotune.get_symmetric_entry(geo, prec, e["log2_n"]) == (
            e["mode"], e.get("min_ctas", 0), e.get("targets", 0)), e
        assert autotune.get_symmetric_grid(geo, prec, e["log2_n"]) == e.get("grid_ctas", 0), e
    for e in table.get("batch", []):
        geo, prec = autotune.GEOMETRIES[e["geometry"]], autotune.PRECISIONS[e["precision"]]
        assert autotune.get_batch_entry(geo, prec, e["log2_n"]) == e["per_thread"], e
