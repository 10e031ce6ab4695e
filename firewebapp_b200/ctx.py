"""Whole outer steps driven from C++: ``fs_ctx_create`` / ``fs_step`` /
``fs_batch_run`` of ``libfirestep.so`` behind a small Python handle.

``StepContext(case)`` resolves the case exactly as :class:`Tier3Solver`
does (``grid.build_setup``: grid, constants, initial state, particles, soil,
quadrature), hands everything to ``fs_ctx_create`` and then steps with no
Python on the per-step path: the C++ loop (``csrc/step.cu``) runs the
reference's operator order (``spread_3d.py:1897-3512``) and its host
decisions itself.  The plain and mixed forms are provided; the learned
preconditioner is driven from Python only (:class:`Tier3Solver`).
``batch_run`` steps several contexts at once, one host thread and one pair
of streams per case, inside the library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import FsCaseDesc, FsInitState, FsStepOut, check
from .grid import build_setup
from .quadrature import level_symmetric
from .solver import Tier3Solver

# fs_ctx_read / fs_ctx_write field ids (include/firestep.h, FS_F_* / FS_P_*)
FIELD_IDS = {
    "rho": 0, "u": 1, "v": 2, "w": 3, "T_g": 4, "Y_fuel": 5, "Y_O2": 6, "Y_H2O": 7, "T_s": 8,
    "alpha_s": 9, "k_turb": 10, "eps_turb": 11, "nu_t": 12, "phi": 13, "omega": 14, "q_rad": 15,
    "q_rad_gas": 16, "M_local": 17, "S_pyro_b": 18, "S_dry_b": 19, "Q_gconv_b": 20,
    "Q_comb": 21, "p_prev": 22, "T_soil": 23, "p_x": 24, "p_y": 25, "p_z": 26, "p_m_solid": 27,
    "p_m_water": 28, "p_m_char": 29, "p_T_s": 30, "p_m_water_0": 31, "p_sav": 32,
    "p_m_char_max": 33, "p_alive": 34,
}


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class StepContext:
    """The Tier-3 loop of one case, stepped in C++ (``fs_step``)."""

    def __init__(self, case: dict, projection_cg_rtol: float | None = None,
                 proj_maxiter: int = 200, form: str = "plain", overlap_dom: bool = True):
        if form not in ("plain", "mixed"):
            raise NotImplementedError(
                f"form {form!r}: the C++ step provides the plain and mixed forms (the learned "
                "preconditioner runs through Tier3Solver)")
        self.lib = _lib.lib()
        su = build_setup(case)
        g, p = su.grid, su.params
        self.grid, self.params, self.case = g, p, dict(case)
        self.shape = g.shape
        if projection_cg_rtol is None:
            projection_cg_rtol = 1.0e-6 if form == "plain" else 1.0e-8
        om, wq = level_symmetric(p["n_quadrature"])
        self.Omega = om
        keep = {}

        def arr(name, a, dtype=np.float64):
            keep[name] = np.ascontiguousarray(np.asarray(a, dtype=dtype))
            return keep[name].ctypes.data

        so = su.soil
        desc = FsCaseDesc(
            nx=g.Nx, ny=g.Ny, nz=g.Nz, n_z_bed=g.n_z_bed, dx=g.dx, dy=g.dy,
            dz=arr("dz", g.dz_arr), d_above=arr("da", g.d_face_above),
            d_below=arr("db", g.d_face_below),
            T_amb=p["T_amb"], h_bed=p["h_bed"], sav=p["sav"], cfl=p["cfl"], dz_min=p["dz_min"],
            U_mf=p["U_mf"], min_dt_s=p["min_dt_s"], dt0=p["dt0"],
            ignition_duration_s=p["ignition_duration_s"], ignition_q_mult=p["ignition_q_mult"],
            canopy_C_d=p["canopy_C_d"], canopy_beta_p=p["canopy_beta_p"],
            canopy_beta_d=p["canopy_beta_d"], h_conv=p["h_conv"],
            rho_solid_true=p["rho_solid_true"], cp_solid=p["cp_solid"],
            eps_solid=p["eps_solid"], view_factor=p["view_factor"],
            kappa_bed_eff=p["kappa_bed_eff"], char_ox_flux_cap=p["char_ox_flux_cap"],
            char_ox_ash_exp=p["char_ox_ash_exp"], chi_rad=p["chi_rad"], T_ign=p["T_ign"],
            proj_div_tol=p["proj_div_tol"], x_front0=p["x_front0"],
            bed_x_end=float(case.get("bed_x_end", g.Lx)),
            drying_mode=int(p["drying_mode"]),
            view_factor_geometric=int(p["view_factor_geometric"]),
            n_per_cell=int(p["n_per_cell"]), i_src_start=int(p["i_src_start"]),
            i_src_end=int(p["i_src_end"]), proj_max_iter=int(p["proj_max_iter"]),
            dom_subcycle_every=int(p["dom_subcycle_every"]),
            edc_extinction_enable=int(p["edc_extinction_enable"]),
            M=om.shape[0], ox=arr("ox", om[:, 0]), oy=arr("oy", om[:, 1]),
            oz=arr("oz", om[:, 2]), w=arr("w", wq), n_soil=so["n"],
            soil_dz=arr("sdz", so["dz"]), soil_d_above=arr("sda", so["d_above"]),
            soil_d_below=arr("sdb", so["d_below"]), form=1 if form == "mixed" else 0,
            projection_rtol=float(projection_cg_rtol), proj_maxiter=int(proj_maxiter),
            overlap_dom=1 if overlap_dom else 0)
        fl = su.fields
        k_init = dict(k_turb=fl["k_turb"], eps_turb=fl["eps_turb"], nu_t=fl["nu_t"],
                      phi=fl["phi"])
        parts = su.particles
        init = FsInitState(
            **{k: arr("f_" + k, fl[k]) for k in ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2",
                                                 "Y_H2O", "T_s", "alpha_s")},
            **{k: arr("f_" + k, v) for k, v in k_init.items()},
            u_inlet=arr("u_inlet", su.u_inlet), sigma_x=arr("sigma_x", su.sigma_sponge),
            T_soil=arr("T_soil", so["T"]), n_particles=len(parts["x"]),
            px=arr("px", parts["x"]), py=arr("py", parts["y"]), pz=arr("pz", parts["z"]),
            m_solid=arr("pms", parts["m_solid"]), m_water=arr("pmw", parts["m_water"]),
            m_char=arr("pmc", parts["m_char"]), pT_s=arr("pts", parts["T_s"]),
            m_water_0=arr("pmw0", parts["m_water_0"]), psav=arr("psav", parts["sav"]),
            m_char_max=arr("pmcm", parts["m_char_max"]),
            alive=arr("alive", parts["alive"], np.int8))
        h = C.c_void_p()
        check(self.lib.fs_ctx_create(C.byref(desc), C.byref(init), C.byref(h)), "fs_ctx_create")
        self.h = h
        self.form = form
        self.last = FsStepOut()

    @property
    def t(self):
        return self.last.t

    def step(self, n: int = 1) -> FsStepOut:
        """``n`` outer steps (fewer if the loop's exit tests fire)."""
        out = FsStepOut()
        check(self.lib.fs_step(self.h, int(n), C.byref(out)), "fs_step")
        self.last = out
        return out

    def read(self, name: str) -> np.ndarray:
        fid = FIELD_IDS[name]
        cnt = int(self.lib.fs_ctx_field_size(self.h, fid))
        out = np.empty(cnt, dtype=np.int8 if name == "p_alive" else np.float64)
        check(self.lib.fs_ctx_read(self.h, fid, out.ctypes.data), "fs_ctx_read")
        if fid <= FIELD_IDS["p_prev"]:
            return out.reshape(self.shape)
        if name == "T_soil":
            return out.reshape((-1,) + self.shape[1:])
        return out

    def write(self, name: str, values) -> None:
        fid = FIELD_IDS[name]
        a = np.ascontiguousarray(np.asarray(values, dtype=np.int8 if name == "p_alive"
                                            else np.float64)).ravel()
        if a.size != int(self.lib.fs_ctx_field_size(self.h, fid)):
            raise ValueError(f"{name}: {a.size} values for a field of "
                             f"{self.lib.fs_ctx_field_size(self.h, fid)}")
        check(self.lib.fs_ctx_write(self.h, fid, a.ctypes.data), "fs_ctx_write")

    def state(self) -> dict:
        """Host copy of the state, keyed like :meth:`Tier3Solver.state`."""
        keys = Tier3Solver.FIELDS + ("omega", "q_rad", "q_rad_gas", "T_soil", "S_pyro_b",
                                     "S_dry_b", "Q_gconv_b", "M_local", "p_prev", "p_x", "p_y",
                                     "p_z", "p_alive", "p_m_solid", "p_m_water", "p_m_char",
                                     "p_T_s", "p_m_water_0", "p_sav", "p_m_char_max")
        return {k: self.read(k) for k in keys}

    def close(self):
        if getattr(self, "h", None):
            self.lib.fs_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_run(ctxs, n_steps: int):
    """``n_steps`` outer steps of every context at once (``fs_batch_run``: one
    host thread per case inside the library); returns their summaries."""
    lib = _lib.lib()
    n = len(ctxs)
    hs = (C.c_void_p * n)(*[c.h.value for c in ctxs])
    outs = (FsStepOut * n)()
    check(lib.fs_batch_run(hs, n, int(n_steps), outs), "fs_batch_run")
    for c, o in zip(ctxs, outs):
        c.last = o
    return list(outs)
