"""The autotuner's host logic with the timings faked (no device): it keeps the fastest candidate
per geometry, precision and N bucket, skips the sizes its table does not apply to, leaves the
library's table holding its choices, and `--only batch` replaces the batch part of a table file
while keeping the rest."""
import json

import pytest

from pointvortex_b200 import autotune


@pytest.fixture
def restore_batch_table():
    keys = [(g, p, b) for g in range(3) for p in range(2) for b in range(5, 16)]
    saved = {k: autotune.get_batch_entry(*k) for k in keys}
    yield
    for k, v in saved.items():
        autotune.set_batch_entry(*k, v)


def _fake_timings(monkeypatch):
    """ms per attempt: T = 2 fastest below N = 1024, T = 4 (else 1) from there; periodic FP64 from
    N = 2048 takes the once-per-unordered-pair items (None)."""
    calls = []

    def fake(geometry, precision, n, attempts):
        t = autotune.get_batch_entry(autotune.GEOMETRIES[geometry], autotune.PRECISIONS[precision],
                                     n.bit_length() - 1)
        calls.append((geometry, precision, n, t))
        if geometry == "periodic" and precision == "fp64" and n >= 2048:
            return None
        best = 2 if n < 1024 else max(autotune.BATCH_CANDIDATES[geometry])
        return 1.0 + abs(t - best)

    monkeypatch.setattr(autotune, "_time_batch", fake)
    return calls


def test_tune_batch_keeps_the_fastest(monkeypatch, restore_batch_table):
    calls = _fake_timings(monkeypatch)
    entries = autotune.tune_batch(range(9, 13), attempts=2)
    by_key = {(e["geometry"], e["precision"], e["log2_n"]): e for e in entries}
    for geo, cands in autotune.BATCH_CANDIDATES.items():
        for prec in autotune.PRECISIONS:
            for b in range(9, 13):
                key = (geo, prec, b)
                if geo == "periodic" and prec == "fp64" and b >= 11:
                    assert key not in by_key  # the table does not apply: default restored
                    assert autotune.get_batch_entry(1, 0, b) == 1
                    continue
                want = 2 if b < 10 else max(cands)
                assert by_key[key]["per_thread"] == want, key
                assert sorted(by_key[key]["ms"]) == sorted(str(t) for t in cands)
                assert autotune.get_batch_entry(autotune.GEOMETRIES[geo],
                                                autotune.PRECISIONS[prec], b) == want
    # each candidate was timed with its own table entry in effect
    assert all(t in autotune.BATCH_CANDIDATES[g] for g, _, _, t in calls)


def test_tune_batch_skips_a_size_it_cannot_admit(monkeypatch, restore_batch_table, capsys):
    from pointvortex_b200.batch import CapacityError
    _fake_timings(monkeypatch)
    timed = autotune._time_batch

    def fake(geometry, precision, n, attempts):
        if geometry == "disk" and n == 4096:
            raise CapacityError("the batch arena has no room for this population")
        return timed(geometry, precision, n, attempts)

    monkeypatch.setattr(autotune, "_time_batch", fake)
    entries = autotune.tune_batch(range(11, 13), attempts=2)
    keys = {(e["geometry"], e["log2_n"]) for e in entries}
    assert ("disk", 12) not in keys and ("disk", 11) in keys and ("infinite", 12) in keys
    assert autotune.get_batch_entry(2, 0, 12) == 2  # the default
    assert "disk fp64 N = 2^12 skipped" in capsys.readouterr().err


def test_only_batch_replaces_the_batch_part(monkeypatch, tmp_path, restore_batch_table):
    _fake_timings(monkeypatch)
    monkeypatch.setattr(autotune, "tune_batch",
                        lambda: [{"geometry": "disk", "precision": "fp64", "log2_n": 9,
                                  "per_thread": 4, "ms": {"1": 3.0, "2": 2.0, "4": 1.0}}])
    path = tmp_path / "table.json"
    keep = {"entries": [], "symmetric": [], "batch": [{"geometry": "infinite", "precision": "fp64",
                                                      "log2_n": 7, "per_thread": 1}]}
    path.write_text(json.dumps(keep))
    assert autotune.main(["--only", "batch", "--out", str(path)]) == 0
    table = json.loads(path.read_text())
    assert table["entries"] == [] and table["symmetric"] == []
    assert [(e["geometry"], e["log2_n"], e["per_thread"]) for e in table["batch"]] == [("disk", 9, 4)]


@pytest.fixture
def restore_symmetric_tables():
    keys = [(g, p, b) for g in (0, 1) for p in range(2) for b in range(11, 14)]
    saved = {k: (autotune.get_symmetric_entry(*k), autotune.get_symmetric_grid(*k)) for k in keys}
    yield
    for k, (entry, grid) in saved.items():
        autotune.set_symmetric_entry(*k, *entry)
        autotune.set_symmetric_grid(*k, grid)


def test_tune_symmetric_times_forms_then_grids(monkeypatch, restore_symmetric_tables):
    """The form is chosen first (fake: the symmetric form with the default occupancy wins), then
    the grid from as many CTAs as fit (fake: 6) down to three fewer; an entry of 0 means "as many
    as fit". Fake step times: the periodic box is fastest with 5 CTAs per SM, the plane with all."""
    def fake_steps(geometry, precision, n, steps):
        b = n.bit_length() - 1
        mode, min_ctas, targets = autotune.get_symmetric_entry(autotune.GEOMETRIES[geometry],
                                                               precision, b)
        grid = autotune.get_symmetric_grid(autotune.GEOMETRIES[geometry], precision, b) or 6
        form = 0.0 if (mode, min_ctas) == (2, 0) and targets in (0, 4) else 1.0
        return 1.0 + form + (abs(grid - 5) if geometry == "periodic" else 6 - grid) * 0.01

    monkeypatch.setattr(autotune, "_time_steps", fake_steps)
    monkeypatch.setattr(autotune, "_grid_ctas", lambda geometry, precision, n: 6)
    entries = autotune.tune_symmetric(range(11, 13), evals=3)
    assert len(entries) == len(autotune.SYMMETRIC_CANDIDATES) * 2
    for e in entries:
        geo, prec = autotune.GEOMETRIES[e["geometry"]], autotune.PRECISIONS[e["precision"]]
        assert (e["mode"], e["min_ctas"]) == (2, 0)
        assert sorted(e["grid_ms"]) == ["3", "4", "5", "6"]
        assert e["grid_ctas"] == (5 if e["geometry"] == "periodic" else 0)
        assert autotune.get_symmetric_grid(geo, prec, e["log2_n"]) == e["grid_ctas"]
        assert autotune.get_symmetric_entry(geo, prec, e["log2_n"]) == (
            e["mode"], e["min_ctas"], e["targets"])
