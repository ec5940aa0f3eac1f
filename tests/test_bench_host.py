"""The ensemble section's bookkeeping with the batch faked (no device): states, stop reasons and
the targets per thread each simulation's work items held are counted over all 512 members."""
from pointvortex_b200.batch import SimInfo


def test_ensemble_section_counts_members(monkeypatch):
    import bench

    def fake_solve(specs, budget, precision):
        out = []
        for k, (geo, n, _) in enumerate(specs):
            symmetric = geo == "periodic" and n >= 2048
            per_thread = 0 if symmetric else {"infinite": 4, "periodic": 1, "disk": 2}[geo]
            state, status, failure = ("failed", 1, 1) if k % 100 == 0 else ("budget", 0, 0)
            info = SimInfo(state, status, 0.01, 1e-3, budget, 1, n, failure, per_thread)
            out.append((info, float(n * (n - 1))))
        return out, 10, 0.5

    monkeypatch.setattr(bench, "solve_batch", fake_solve)
    r = bench.run_ensemble()
    specs = bench.ensemble_specs()
    assert r["simulations"] == 512 and sum(r["states"].values()) == 512
    assert r["states"] == {"failed": 6, "budget": 506}
    assert sum(r["targets_per_thread"].values()) == 512
    sym = sum(1 for g, n, _ in specs if g == "periodic" and n >= 2048)
    assert r["targets_per_thread"].get("periodic:0", 0) == sym
    assert set(r["targets_per_thread"]) <= {"infinite:4", "periodic:1", "periodic:0", "disk:2"}
    assert sum(v for k, v in r["stop_reasons"].items() if k.endswith("rejection_cap")) == 6
    assert r["budgeted_solves_per_s"] == 512 / 0.5
