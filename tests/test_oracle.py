"""The CPU oracle is pinned to the reference: its kernels against the
reference's committed golden vectors and its whole step against states
captured from the reference solver (tests/golden/*.npz).  No GPU needed."""
import numpy as np
import pytest

from conftest import rel_l2

from oracle import kernels as K

TIGHT = 1e-12


def test_muscl(vectors):
    for name in vectors.cases("muscl"):
        c = vectors.case("muscl", name)
        shp = (c["nz"], c["ny"], c["nx"])
        rhs = c["rhs_in"].reshape(shp).copy()
        K.advect_scalar_muscl(*(c[k].reshape(shp) for k in ("phi", "u", "v", "w")), c["dx"],
                              c["dy"], c["d_face_above"], c["d_face_below"], rhs, c["phi_inlet"])
        assert rel_l2(rhs, c["rhs_out"]) <= TIGHT, name


def test_species(vectors):
    for name in vectors.cases("species"):
        c = vectors.case("species", name)
        shp = (c["nz"], c["ny"], c["nx"])
        r = lambda k: c[k].reshape(shp)  # noqa: E731
        out = K.species_transport(r("Y_in"), r("rho"), r("u"), r("v"), r("w"), r("S"), c["dt"],
                                  c["dx"], c["dy"], c["dz_arr"], c["d_face_above"],
                                  c["d_face_below"], c["D"], c["Y_inlet"])
        assert rel_l2(out, c["Y_out"]) <= TIGHT, name


def test_momentum_and_drag(vectors):
    for name in vectors.cases("momentum"):
        c = vectors.case("momentum", name)
        shp = (c["nz"], c["ny"], c["nx"])
        r = lambda k: c[k].reshape(shp)  # noqa: E731
        i2 = lambda k: c[k].reshape(shp[:2])  # noqa: E731
        u, v, w = K.tentative_velocity(r("u_in"), r("v_in"), r("w_in"), r("rho"), r("T_g"),
                                       r("Fx"), r("Fy"), r("Fz"), c["dt"], c["dx"], c["dy"],
                                       c["dz_arr"], c["d_face_above"], c["d_face_below"],
                                       c["T_amb"], i2("u_inlet"), i2("v_inlet"), i2("w_inlet"))
        for got, k in ((u, "u_out"), (v, "v_out"), (w, "w_out")):
            assert rel_l2(got, c[k]) <= TIGHT, (name, k)
    for name in vectors.cases("drag"):
        c = vectors.case("drag", name)
        F = K.drag_force(c["u"], c["v"], c["w"], c["rho"], c["alpha_s"], c["sigma_sav"], c["C_D"])
        for got, k in zip(F, ("Fx", "Fy", "Fz")):
            assert rel_l2(got, c[k]) <= TIGHT, (name, k)


def test_solid_conduction(vectors):
    for name in vectors.cases("solid_conduction"):
        c = vectors.case("solid_conduction", name)
        shp = (c["nz"], c["ny"], c["nx"])
        out = K.solid_conduction(c["T_s_in"].reshape(shp), c["alpha_s"].reshape(shp),
                                 c["dz_arr"], c["d_face_above"], c["d_face_below"],
                                 c["k_solid"], c["rho_solid"], c["cp_solid"], c["dt"])
        assert rel_l2(out, c["T_s_out"]) <= TIGHT, name


def test_edc(vectors):
    for name in vectors.cases("edc"):
        c = vectors.case("edc", name)
        shp = (c["nz"], c["ny"], c["nx"])
        r = lambda k: c[k].reshape(shp)  # noqa: E731
        Tg, Yf, YO, om = K.edc(r("rho"), r("T_g_in"), r("Y_fuel_in"), r("Y_O2_in"),
                               r("k_turb"), r("eps_turb"), r("Y_H2O"), c["chi_rad"], c["cp_g"],
                               c["dt"], c["n_substeps"], c["s_stoich"], c["hoc_J"],
                               bool(c["extinction_enable"]))
        for got, k in ((Tg, "T_g_out"), (Yf, "Y_fuel_out"), (YO, "Y_O2_out"), (om, "omega_out")):
            assert rel_l2(got, c[k]) <= TIGHT, (name, k)


def test_turbulent_diffusion(vectors):
    for name in vectors.cases("turb_diff"):
        c = vectors.case("turb_diff", name)
        shp = (c["nz"], c["ny"], c["nx"])
        nu = c["nu_t"].reshape(shp)
        n, _ = K.turb_diffusion_nsub(nu, c["sc_t"], c["dt"], c["dx"], c["dy"], c["dz_arr"])
        assert n == c["n_sub"], name
        out = K.turb_diffusion(c["field_in"].reshape(shp), nu, c["sc_t"], c["dt"], c["dx"],
                               c["dy"], c["dz_arr"], c["d_face_above"], c["d_face_below"])
        assert rel_l2(out, c["field_out"]) <= TIGHT, name


def test_k_epsilon(vectors):
    for name in vectors.cases("kepsilon"):
        c = vectors.case("kepsilon", name)
        shp = (c["nz"], c["ny"], c["nx"])
        r = lambda k: c[k].reshape(shp)  # noqa: E731
        k_, e_, nu = K.k_epsilon(r("k_in"), r("eps_in"), r("u"), r("v"), r("w"), r("T_g"),
                                 r("alpha_s"), c["sigma_sav"], c["dt"], c["dx"], c["dy"],
                                 c["dz_arr"], c["d_face_above"], c["d_face_below"], c["T_amb"],
                                 c["u_inlet"].reshape(shp[:2]),
                                 c["k_wall_ghost"].reshape(shp[1:]),
                                 c["eps_wall_ghost"].reshape(shp[1:]), c["beta_p"], c["beta_d"])
        for got, k in ((k_, "k_out"), (e_, "eps_out"), (nu, "nu_t_out")):
            assert rel_l2(got, c[k]) <= TIGHT, (name, k)


def test_dom(vectors):
    from firewebapp_b200.quadrature import level_symmetric
    om, wq = level_symmetric(4)
    for name in vectors.cases("dom"):
        c = vectors.case("dom", name)
        shp = (c["nz"], c["ny"], c["nx"])
        r = lambda k: c[k].reshape(shp)  # noqa: E731
        I = np.zeros((om.shape[0],) + shp)
        qs, qg, qsoil, _ = K.dom_solve(
            I, om, wq, r("T_s"), r("T_g"), r("alpha_s"), r("omega_comb"), c["sigma_sav"],
            c["T_amb"], c["dx"], c["dy"], c["dz_arr"], T_soil0=c["T_soil"].reshape(shp[1:]),
            Y_H2O=r("Y_H2O") if "Y_H2O" in c else None, rho=r("rho") if "rho" in c else None,
            M_local=r("bed_moisture"))
        assert rel_l2(qs, c["q_rad_solid"]) <= 1e-11, name
        assert rel_l2(qg, c["q_rad_gas"]) <= 1e-11, name
        assert rel_l2(qsoil, c["q_in_soil"]) <= 1e-11, name


def test_dom_s8_matches_reference():
    """The oracle's DOM at S8 (80 ordinates) against the reference's own
    DOMRadiationSolver with the S8 set injected (tests/golden/dom_s8.npz):
    two solves in a row on every golden-vector geometry and on a slice of the
    400 x 120 x 60 grid; same iteration counts, outputs to 1e-11."""
    from conftest import dom_s8_cases
    from firewebapp_b200.quadrature import level_symmetric
    om, wq = level_symmetric(8)
    for name, (c, calls) in dom_s8_cases().items():
        shp = (c["nz"], c["ny"], c["nx"])
        I = np.zeros((om.shape[0],) + shp)
        for n, want in enumerate(calls):
            qs, qg, qsoil, it = K.dom_solve(
                I, om, wq, want["T_s"], want["T_g"], c["alpha_s"], c["omega_comb"],
                c["sigma_sav"], c["T_amb"], c["dx"], c["dy"], c["dz_arr"],
                T_soil0=c["T_soil"], Y_H2O=c.get("Y_H2O"), rho=c.get("rho"),
                M_local=c["bed_moisture"])
            assert it == want["iterations"], (name, n)
            assert rel_l2(qs, want["q_rad_solid"]) <= 1e-11, (name, n)
            assert rel_l2(qg, want["q_rad_gas"]) <= 1e-11, (name, n)
            assert rel_l2(qsoil, want["q_in_soil"]) <= 1e-11, (name, n)


def test_lagrangian_bed(vectors):
    for name in vectors.cases("lagrangian_bed"):
        c = vectors.case("lagrangian_bed", name)
        shp = (c["nz"], c["ny"], c["nx"])
        P = {k: np.array(c["in_" + k]) for k in ("x", "y", "z", "m_solid", "m_water", "m_char",
                                                 "T_s", "m_water_0", "sav", "m_char_max")}
        P["alive"] = np.array(c["in_alive"]).astype(np.int8)
        zf = np.asarray(c["z_face"])
        src = K.bed_step(P, c["T_g"].reshape(shp), c["Y_O2"].reshape(shp),
                         c["Q_solid_ext"].reshape(shp), c["n_per_cell"], c["dx"], c["dy"],
                         c["dz_arr"], zf, c["h_conv"], c["rho_solid_true"], c["cp_solid"],
                         c["eps_solid"], c["T_amb"], c["view_factor"],
                         bool(c["view_factor_geometric"]), c["h_bed"], c["kappa_bed_eff"],
                         c["dt"], c["drying_mode"], c["char_ox_flux_cap"], c["char_ox_ash_exp"])
        for k in ("m_solid", "m_water", "m_char", "T_s", "m_char_max"):
            assert rel_l2(P[k], c["out_" + k]) <= TIGHT, (name, k)
        assert np.array_equal(P["alive"].astype(int), np.asarray(c["out_alive"]).astype(int))
        for k, ck in (("S_pyro", "out_S_pyro"), ("S_drying", "out_S_drying"),
                      ("Q_pyro", "out_Q_pyro"), ("Q_drying", "out_Q_drying"),
                      ("Y_F_source", "out_Y_F_source"), ("Q_char", "out_Q_char"),
                      ("Q_smold", "out_Q_smold"), ("Q_g_conv", "out_Q_g_conv")):
            assert rel_l2(src[k], c[ck]) <= TIGHT, (name, k)
        Tg = K.bed_aggregate(P, shp, c["dx"], c["dy"], zf, out=np.full(shp, 300.0), mode=0)
        assert rel_l2(Tg, c["out_T_s_grid"]) <= TIGHT, name
        M = K.bed_aggregate(P, shp, c["dx"], c["dy"], zf, mode=1)
        assert rel_l2(M, c["out_M_local"]) <= TIGHT, name
        Pc = dict(P)
        Pc["T_s"] = P["T_s"].copy()
        Tn = K.bed_hcond(Pc, c["cond_T_in"].reshape(shp), c["alpha_s"].reshape(shp), c["dx"],
                         c["dy"], zf, c["k_solid"], c["rho_solid_true"], c["cp_solid"],
                         c["n_z_bed"], c["dt"])
        assert rel_l2(Tn, c["cond_T_out"]) <= TIGHT, name
        assert rel_l2(Pc["T_s"], c["cond_part_T_out"]) <= TIGHT, name


def test_projection(vectors):
    c = vectors.case("projection", "slab2d")
    shp = (c["nz"], c["ny"], c["nx"])
    A, _ = K.poisson_matrix(c["rho"].reshape(shp), c["dx"], c["dy"], c["dz_arr"],
                            c["d_face_above"], c["d_face_below"])
    assert rel_l2(A @ c["probe"], c["matvec_out"]) <= TIGHT
    u_in = c["u_inlet"].reshape(shp[:2])
    div = K.divergence(c["u_in"].reshape(shp), c["v_in"].reshape(shp), c["w_in"].reshape(shp),
                       c["dx"], c["dy"], c["dz_arr"], u_in)
    assert rel_l2(div, c["div_out"]) <= TIGHT
    tgt = c["div_target"].reshape(shp)
    u, v, w, _ = K.project(c["u_in"].reshape(shp), c["v_in"].reshape(shp),
                           c["w_in"].reshape(shp), c["rho"].reshape(shp), c["dt"], tgt, c["dx"],
                           c["dy"], c["dz_arr"], c["d_face_above"], c["d_face_below"], u_in)
    res = np.max(np.abs(K.divergence(u, v, w, c["dx"], c["dy"], c["dz_arr"], u_in) - tgt))
    assert res <= c["proj_resid"]


def test_level_set(vectors):
    for name in vectors.cases("flame_front"):
        c = vectors.case("flame_front", name)
        shp = (c["nz"], c["ny"], c["nx"])
        phi = c["phi_init"].reshape(shp)
        assert rel_l2(K.godunov_grad(phi, c["dx"], c["dy"], c["dz_arr"]), c["grad_out"]) <= TIGHT
        ev = phi - c["dt"] * c["v_n_in"].reshape(shp) * K.godunov_grad(phi, c["dx"], c["dy"],
                                                                        c["dz_arr"])
        assert rel_l2(ev, c["phi_evolved"]) <= TIGHT, name
        assert rel_l2(K.levelset_reinit(ev, c["dx"], c["dy"], c["dz_arr"]),
                      c["phi_reinit"]) <= TIGHT, name
        act = K.active_flame(c["omega"], c["T_g"], c["Y_fuel"])
        assert int(act.sum()) == c["n_active"]
        assert np.array_equal(act, np.asarray(c["fb_from_phi"]) > 0)
        if "front_x" in c:
            fx = K.front_x(K.levelset_reinit(ev, c["dx"], c["dy"], c["dz_arr"]), 1,
                           c["ny"] // 2, c["dx"])
            assert abs(fx - c["front_x"]) <= 1e-12


def test_support(vectors):
    for name in vectors.cases("support"):
        c = vectors.case("support", name)
        nz, ny, nx = shp = (c["nz"], c["ny"], c["nx"])
        u = K.outflow_sponge(c["sponge_u_in"].reshape(shp), c["sponge_u_target"].reshape(nz, ny),
                             c["sponge_sigma_x"], c["sponge_Y_F"].reshape(shp),
                             c["sponge_Y_F_skip"], c["sponge_dt"])
        assert rel_l2(u, c["sponge_u_out"]) <= TIGHT, name
        ns = c["n_soil"]
        Ts = K.soil_step(c["soil_T_in"].reshape(ns, ny, nx), c["soil_q_in"].reshape(ny, nx),
                         c["soil_dt"], c["soil_dz"], c["soil_d_above"], c["soil_d_below"])
        assert rel_l2(Ts, c["soil_T_out"]) <= TIGHT, name
        T = K.gas_energy_adv(c["Tg_in"].reshape(shp), c["u"].reshape(shp), c["v"].reshape(shp),
                             c["w"].reshape(shp), c["gas_dt"], c["dx"], c["dy"], c["dz_arr"],
                             c["d_face_above"], c["d_face_below"], 2.0e-5, 300.0)
        assert rel_l2(T, c["Tg_out"]) <= TIGHT, name


# ----------------------------------------------------------------- whole step


def _oracle_state(case, snap, t, dt_prev, step):
    from firewebapp_b200.grid import build_setup
    from firewebapp_b200.quadrature import level_symmetric
    from oracle.step import OracleState, geometry_from_setup
    su = build_setup(case)
    om, wq = level_symmetric(case.get("n_quadrature", 4))
    return OracleState(snap, geometry_from_setup(su), su.params, om, wq, t=t, dt_prev=dt_prev,
                       step=step)


STEP_FIELDS = ("rho", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "T_s", "k_turb", "eps_turb", "nu_t",
               "omega", "q_rad", "T_soil", "phi", "p_T_s", "p_m_solid", "p_m_water", "p_m_char",
               "S_pyro_b", "S_dry_b", "Q_gconv_b", "I_set")


def _compare(got, want, tag, tol=1e-9):
    vel = np.sqrt(sum(np.sum(np.asarray(want[c]) ** 2) for c in ("u", "v", "w")))
    bad = {}
    for k in ("u", "v", "w"):
        e = np.linalg.norm((got[k] - want[k]).ravel()) / vel
        if not e <= tol:
            bad[k] = e
    for k in STEP_FIELDS:
        if k in want:
            e = rel_l2(got[k], want[k])
            if not e <= tol:
                bad[k] = e
    assert not bad, f"{tag}: {bad}"


def test_oracle_step_from_initial_state(ref_tiny):
    from firewebapp_b200.cases import TINY
    from firewebapp_b200.grid import build_setup
    from oracle.step import step
    init = dict(ref_tiny["init"])
    su = build_setup(TINY)
    for k in ("k_turb", "eps_turb", "nu_t", "phi"):
        init[k] = su.fields[k]
    init["T_soil"] = su.soil["T"]
    S = _oracle_state(TINY, init, 0.0, None, 0)
    step(S)
    _compare(S.snapshot(), ref_tiny["s1"], "init -> s1")
    step(S)
    _compare(S.snapshot(), ref_tiny["s2"], "s1 -> s2")


def test_oracle_step_from_reference_state(ref_tiny):
    from firewebapp_b200.cases import TINY
    from oracle.step import step
    dts = ref_tiny["trace"]["dt"]
    S = _oracle_state(TINY, ref_tiny["s9"], float(np.sum(dts[:9])), float(dts[8]), 9)
    step(S)
    _compare(S.snapshot(), ref_tiny["s10"], "s9 -> s10")

