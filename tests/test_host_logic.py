"""Host-side logic without a GPU: whole-job aggregation over ranks (gloo,
world size 2), snapshot aggregation and signed flame distance, result-file
key set."""
import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    from bench import job_totals
    # rank r processed (r+1) * 1000 cell-steps in (r+1) * 0.5 s
    work, sec = job_totals((rank + 1) * 1000.0, (rank + 1) * 0.5)
    out.put((rank, work, sec))
    dist.destroy_process_group()


def test_job_totals_sum_work_max_time_over_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, work, sec in res:
        assert work == 3000.0 and sec == 1.0


def test_job_totals_single_process():
    sys.path.insert(0, str(ROOT))
    from bench import job_totals
    assert job_totals(5.0, 2.0) == (5.0, 2.0)


def test_bed_particles_per_cell_matches_loop():
    from firewebapp_b200.api import bed_particles_per_cell
    from firewebapp_b200.grid import build_grid
    g = build_grid(1.2, 0.4, 0.6, 0.1, 0.2, 2)
    rng = np.random.default_rng(3)
    n = 500
    parts = dict(x=rng.uniform(-0.05, 1.25, n), y=rng.uniform(0.0, 0.4, n),
                 z=rng.uniform(0.0, 0.3, n), alive=(rng.random(n) < 0.8).astype(np.int8),
                 m_solid=rng.random(n), m_water=rng.random(n), m_char=rng.random(n),
                 T_s=300 + 500 * rng.random(n))
    got = bed_particles_per_cell(parts, g)
    # loop restatement of the reference's per-particle aggregation
    cnt = np.zeros(g.shape, np.float32)
    tw = np.zeros(g.shape)
    mm = np.zeros(g.shape)
    for p in range(n):
        if parts["alive"][p] == 0:
            continue
        xi, yj = int(parts["x"][p] / g.dx), int(parts["y"][p] / g.dy)
        if not (0 <= xi < g.Nx and 0 <= yj < g.Ny):
            continue
        zk = next((k for k in range(g.Nz) if parts["z"][p] < g.z_face[k + 1]), -1)
        if zk < 0:
            continue
        mt = parts["m_solid"][p] + parts["m_water"][p] + parts["m_char"][p]
        cnt[zk, yj, xi] += 1.0
        tw[zk, yj, xi] += parts["T_s"][p] * mt
        mm[zk, yj, xi] += mt
    assert np.array_equal(got["bp_count"], cnt)
    ref_T = np.where(mm > 0, tw / np.maximum(mm, 1e-30), 0.0).astype(np.float32)
    np.testing.assert_allclose(got["bp_T_s_avg"], ref_T, rtol=1e-6)


def test_phi_flame_signs_and_distance():
    from firewebapp_b200.api import phi_flame_from_state
    shp = (4, 5, 6)
    om = np.zeros(shp)
    om[1, 2, 3] = 1.0
    phi = phi_flame_from_state(om, np.full(shp, 300.0), np.zeros(shp), 0.1, 0.1, np.full(4, 0.1))
    assert phi[1, 2, 3] < 0 and (phi[om == 0] > 0).all()
    assert np.isclose(phi[1, 2, 4], 0.1)
    assert phi_flame_from_state(np.zeros(shp), np.full(shp, 300.0), np.zeros(shp), 0.1, 0.1,
                                np.full(4, 0.1))[0, 0, 0] == 1.0e6


def test_result_save_writes_reference_key_set(tmp_path):
    from firewebapp_b200.api import Spread3DResultGPU
    from firewebapp_b200.grid import build_grid
    g = build_grid(0.6, 0.2, 0.4, 0.1, 0.2, 2)
    z = np.zeros(g.shape)
    st = {k: z for k in ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "alpha_s", "T_s")}
    r = Spread3DResultGPU(ros_m_s=0.1, n_cells_ignited=3, front_t=[0.0, 1.0],
                          front_x=[0.1, 0.2], grid=g, state_final=st)
    path = r.save(tmp_path / "res")
    keys = set(np.load(path, allow_pickle=False).files)
    want = {"_meta_json", "x_mid", "y_mid", "z_mid", "dz_arr", "inv_dz_arr", "z_face",
            "d_face_above", "d_face_below", "rho", "u", "v", "w", "p_dyn", "T_g", "Y_fuel",
            "Y_O2", "Y_H2O", "Y_CO", "alpha_s", "T_s", "m_hemi", "m_cell", "m_lign", "m_char",
            "front_t", "front_x", "diag_t", "diag_Tg_max", "diag_Ts_max", "diag_Sp_max",
            "diag_Qc_max", "diag_omega_max", "diag_Y_max", "diag_n_ign"}
    assert keys == want
    meta = json.loads(str(np.load(path)["_meta_json"]))
    assert meta["Nx"] == g.Nx and meta["ros_m_s"] == 0.1


def _write_deck(case, path):
    lines = ["# test deck", "t_end = 2.5  # seconds"]
    for k, v in case.items():
        if k in ("wind_speed_m_s", "n_quadrature", "jitter_seed"):
            continue
        if isinstance(v, bool):
            v = "true" if v else "false"
        lines.append(f"outdoor.{k} = {v}")
    path.write_text("\n".join(lines) + "\n")


def test_deck_round_trip_gives_the_same_setup(tmp_path):
    from firewebapp_b200.cases import CFG1
    from firewebapp_b200.deck import case_from_deck, read_deck
    from firewebapp_b200.grid import build_setup
    deck = tmp_path / "cfg1.txt"
    _write_deck(CFG1, deck)
    assert read_deck(deck)["t_end"] == 2.5
    case = case_from_deck(deck, wind_speed_m_s=CFG1["wind_speed_m_s"],
                          n_quadrature=CFG1["n_quadrature"], jitter_seed=0)
    a, b = build_setup(CFG1), build_setup(case)
    assert a.grid.shape == b.grid.shape and np.array_equal(a.grid.dz_arr, b.grid.dz_arr)
    for k, v in a.params.items():
        assert b.params[k] == v, k
    for k in a.fields:
        assert np.array_equal(a.fields[k], b.fields[k]), k
    for k in a.particles:
        assert np.array_equal(a.particles[k], b.particles[k]), k


def test_deck_value_parsing_and_precedence(tmp_path):
    from firewebapp_b200.deck import case_from_deck, parse_value
    assert parse_value("1") is True and parse_value("no") is False
    assert parse_value("nan") is None and parse_value(" 0.25 ") == 0.25
    assert parse_value("k_epsilon") == "k_epsilon"
    deck = tmp_path / "d.txt"
    deck.write_text("; comment\noutdoor.n_z_bed = 8\noutdoor.Lx = 12.0\n"
                    "outdoor.dx = 0.1  # inline\n")
    case = case_from_deck(deck, wind_speed_m_s=3.0, n_z_bed=4, Lx=6.0, dx=None)
    assert case["n_z_bed"] == 8.0        # deck wins (spread_3d.py:1041)
    assert case["Lx"] == 6.0 and "lx" not in case   # keyword wins (_pick)
    assert case["dx"] == 0.1 and case["wind_speed_m_s"] == 3.0


def test_unprovided_physics_branches_raise():
    """Decks that ask for a branch the GPU step does not provide fail at setup
    instead of silently running the provided one."""
    from firewebapp_b200.cases import TINY
    from firewebapp_b200.grid import build_setup
    build_setup(TINY)
    for key, bad in (("radiation_solver", "p1"), ("turbulence_model", "smagorinsky"),
                     ("combustion_closure", "mixing_limited"), ("level_set_passive", False),
                     ("empirical_ros_enable", True), ("wall_function", True)):
        with pytest.raises(NotImplementedError, match=key):
            build_setup(dict(TINY, **{key: bad}))
    case = dict(TINY)
    del case["turbulence_model"]  # the reference's default is laminar
    with pytest.raises(NotImplementedError, match="turbulence_model"):
        build_setup(case)


def test_compare_forms_field_errors():
    """The mixed-against-plain error measure: relative L2 per field, the
    velocity components against the norm of the whole velocity vector (a
    crosswind component can be orders of magnitude smaller than the others),
    and the absolute norm for a field that is zero in the plain run."""
    from firewebapp_b200.compare_forms import FIELDS, field_errors
    rng = np.random.default_rng(4)
    plain = {k: rng.random((3, 4, 5)) + 1.0 for k in FIELDS}
    plain["v"] = 1e-6 * rng.standard_normal((3, 4, 5))
    plain["q_rad"] = np.zeros((3, 4, 5))
    mixed = {k: v.copy() for k, v in plain.items()}
    assert all(e == 0.0 for e in field_errors(plain, mixed).values())
    mixed["v"] = plain["v"] + 1e-7
    mixed["T_g"] = plain["T_g"] * (1.0 + 1e-6)
    mixed["q_rad"] = np.full((3, 4, 5), 2e-3)
    err = field_errors(plain, mixed)
    vnorm = np.sqrt(sum(np.linalg.norm(plain[k]) ** 2 for k in ("u", "v", "w")))
    assert err["v"] == pytest.approx(np.linalg.norm(np.full(60, 1e-7)) / vnorm, rel=1e-12)
    assert err["v"] < 1e-6 < np.linalg.norm(mixed["v"] - plain["v"]) / np.linalg.norm(plain["v"])
    assert err["T_g"] == pytest.approx(1e-6, rel=1e-9)
    assert err["q_rad"] == pytest.approx(np.sqrt(60) * 2e-3, rel=1e-12)
    assert err["u"] == 0.0 and set(err) == set(FIELDS)
