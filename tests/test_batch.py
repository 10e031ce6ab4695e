"""The batched form: case sharding (host) and concurrent stepping of several
cases on one GPU, which must give each case exactly its single-case result."""
import numpy as np
import pytest


def test_shard_balances_work_and_covers_every_case():
    from firewebapp_b200.batch import shard
    w = [541, 389, 535, 525, 210, 600, 333, 450]
    parts = [shard(len(w), r, 3, w) for r in range(3)]
    assert sorted(sum(parts, [])) == list(range(len(w)))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert shard(4, 0, 1) == [0, 1, 2, 3]


def test_batch_cases_follow_the_sweep_distribution():
    from firewebapp_b200.cases import batch_cases
    from firewebapp_b200.grid import build_setup
    cs = batch_cases(3, seed0=3)
    assert cs == batch_cases(3, seed0=3)
    for c in cs:
        g = build_setup(c).grid
        assert 200 <= g.Nx <= 600 and g.Ny == 120 and g.Nz == 60 and g.n_z_bed == 4
        assert 1.0 <= c["wind_speed_m_s"] <= 8.0 and 0.02 <= c["initial_moisture_frac"] <= 0.12
        assert 0.2 <= c["bulk_density_kg_m3"] <= 0.6 and 0.1 <= c["fuel_depth_m"] <= 0.4


@pytest.mark.gpu
def test_concurrent_cases_match_single_runs():
    from firewebapp_b200.batch import run_batch
    from firewebapp_b200.cases import TINY
    cases = [dict(TINY, wind_speed_m_s=u, jitter_seed=s)
             for u, s in ((4.0, 0), (6.0, 1), (2.5, 2))]
    alone = run_batch(cases, steps=6, concurrency=1, keep_state=True)
    together = run_batch(cases, steps=6, concurrency=3, keep_state=True)
    for a, b in zip(alone, together):
        assert a.steps == b.steps == 6 and a.t == b.t
        for k, v in a.state.items():
            assert np.array_equal(v, b.state[k]), k


def test_autotune_picks_the_fastest_candidate_and_caches(tmp_path, monkeypatch):
    """The tuner times each candidate through batch.time_concurrent (faked
    here: no GPU), keeps the fastest, skips shapes that fail, and answers the
    same question from its cache."""
    import firewebapp_b200.autotune as A
    import firewebapp_b200.batch as B
    from firewebapp_b200._lib import FireStepError
    from firewebapp_b200.cases import batch_cases
    monkeypatch.setenv("FIREWEBAPP_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(A.torch.cuda, "get_device_name", lambda d=None: "fake")
    calls = []

    def fake(cases, steps, warmup=3, form="plain", device="cuda", solver_kw=None):
        calls.append(dict(solver_kw))
        key = (solver_kw["dom_sweep"], solver_kw["dom_cluster_ctas"])
        if key == (8, 15):
            raise FireStepError(1, "no such sweep shape")
        return {"value": {(8, 0): 1.0e8, (8, 6): 1.5e8}[key], "wall_s": 1.0}

    monkeypatch.setattr(B, "time_concurrent", fake)
    cases = batch_cases(2, seed0=0)
    out = A.tune_batch(cases, concurrency=2)
    assert out["solver_kw"] == {"dom_sweep": 8, "dom_cluster_ctas": 6} and not out["cached"]
    assert len(calls) == len(A.CANDIDATES)
    assert any("error" in t for t in out["trials"])
    again = A.tune_batch(cases, concurrency=2)
    assert again["cached"] and again["solver_kw"] == out["solver_kw"]
    assert len(calls) == len(A.CANDIDATES)


@pytest.mark.gpu
def test_tuned_sweep_shapes_agree():
    """The autotuner's candidates compute the same state to round-off (the
    workload's 60 x 120 cross-section, cut to 40 x-cells)."""
    import numpy as np
    from firewebapp_b200.autotune import CANDIDATES
    from firewebapp_b200.cases import CFG2, scaled
    from firewebapp_b200.solver import Tier3Solver
    case = scaled(CFG2, nx=40)
    states = {}
    for mode, ctas in CANDIDATES:
        s = Tier3Solver(case, dom_sweep=mode, dom_cluster_ctas=ctas)
        for _ in range(2):
            s.step()
        states[(mode, ctas)] = s.state()
        s.close()
    a = states[(8, 0)]
    for key, st in states.items():
        for k in ("T_g", "q_rad", "u", "T_s"):
            d = np.linalg.norm(st[k] - a[k]) / np.linalg.norm(a[k])
            assert d <= 1e-12, (key, k, d)
