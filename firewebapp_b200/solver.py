"""Device-resident Tier-3 time stepper (the ``run_3d_spread`` loop on one GPU).

One :meth:`Tier3Solver.step` performs one outer iteration of the reference
loop (``spread_3d.py:1897-3512``) in the production configuration
(Lagrangian bed, k-epsilon, EDC, DOM, passive level set, periodic y, log-law
inlet), operator by operator in the reference's order, every operator being
a kernel of ``libfirestep.so``.  All state lives in device memory (torch
tensors used as plain buffers); the host only sequences launches and reads
back the few scalars the reference loop branches on (dt, the pressure-
iteration test, the DOM source-iteration test, the turbulent-diffusion
sub-step count, exit tests).

Dead work of the production path is not executed (it cannot change any
state the loop reads): ``step_o2_supply_rate`` and ``tau_mix`` (EDC ignores
both), ``burning_mask``, ``Q_pyro`` in the Lagrangian branch,
``update_cell_age`` and the DOM forward flux at the band (both only feed the
level-set speed, which is zero in passive mode) and the phi_flame distance
values (only its sign is used, and that sign is the active-flame mask).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import FsBedParams, FsBedParticles, FsBedSegments, FsBedSources, FsGrid
from ._lib import check, ptr, ptr_array, dbl_array
from .grid import build_setup, P0, R_AIR, G as G_ACC
from .quadrature import level_symmetric

N_SUB = 10
SC_T = 0.7
PR_T = 0.85
K_MIN = 1.0e-8
EPS_MIN = 1.0e-8
T_CAP = 10_000.0
KAPPA_SOOT_HOT = 0.5


def locate_particle_cells(x, y, z, dx, dy, z_face, nx, ny, nz):
    """Cell index of each particle as ``locate_cell`` computes it
    (lagrangian_particles_3d.py:95-140); -1 for out-of-domain particles."""
    i = np.where(x < 0.0, -1, np.trunc(x / dx)).astype(np.int64)
    i[i >= nx] = -1
    j = np.where(y < 0.0, -1, np.trunc(y / dy)).astype(np.int64)
    j[j >= ny] = -1
    k = np.full(x.shape, -1, dtype=np.int64)
    inside = (z >= z_face[0]) & (z < z_face[nz])
    kk = np.searchsorted(z_face[1:nz + 1], z, side="right")
    k[inside] = np.minimum(kk[inside], nz - 1)
    ok = (i >= 0) & (j >= 0) & (k >= 0)
    cell = np.where(ok, (k * ny + j) * nx + i, -1)
    return cell


def build_segments(cell):
    """Group particle slots by cell, keeping slot order inside a cell."""
    valid = np.nonzero(cell >= 0)[0]
    order = valid[np.argsort(cell[valid], kind="stable")]
    cs = cell[order]
    if cs.size:
        brk = np.nonzero(np.diff(cs))[0] + 1
        starts = np.concatenate([[0], brk, [cs.size]])
        seg_cell = cs[starts[:-1]]
    else:
        starts = np.zeros(1, dtype=np.int64)
        seg_cell = np.zeros(0, dtype=np.int64)
    return order.astype(np.int32), starts.astype(np.int32), seg_cell.astype(np.int32)


@dataclass
class StepDiag:
    t: float = 0.0
    dt: float = 0.0
    proj_iters: int = 0
    cg_iters: list = field(default_factory=list)
    proj_div_max: float = 0.0
    dom_iters: int = 0
    n_sub_sc: int = 0
    n_sub_pr: int = 0


class Tier3Solver:
    """The Tier-3 step on one GPU, from a case dict (deck keys + wind speed).

    ``form="plain"`` is FP64 throughout.  ``form="mixed"`` runs the DOM sweep
    and the multigrid preconditioner in FP32; the state, every other kernel,
    the CG (operator, residuals, dot products), the divergence test and all
    reductions stay FP64.  ``form="learned"`` is the mixed form with the
    pressure solve in flexible CG preconditioned by the U-Net of
    ``learned.py`` (weights from ``learned_weights``, default the packaged
    file), falling back to the V-cycle when it stalls.  ``dom_sweep`` forces a
    DOM sweep path (``fs_dom_set_sweep_mode``; 0 picks automatically),
    ``dom_cluster_ctas`` its CTAs per octant (0: automatic; a nonzero value
    alone selects path 8) and ``dom_kernel`` path 8's kernel
    (``fs_dom_set_sweep_kernel``: 0 automatic, 1 pencil per thread, 2 lane
    column)."""

    FIELDS = ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "T_s", "alpha_s",
              "k_turb", "eps_turb", "nu_t", "phi")

    def __init__(self, case: dict, device="cuda", projection_cg_rtol: float | None = None,
                 proj_maxiter: int = 200, mg_sweeps: int | None = None, form: str = "plain",
                 overlap_dom: bool = True, dom_sweep: int = 0, learned_weights=None,
                 learned_max: int = 30, learned_stall: float = 0.9, dom_cluster_ctas: int = 0,
                 mg_fine_sweeps: int | None = None, dom_kernel: int = 0):
        self.lib = _lib.lib()
        self.dev = torch.device(device)
        if self.dev.type == "cuda" and self.dev.index is None:
            self.dev = torch.device("cuda", torch.cuda.current_device())
        self.case = dict(case)
        su = build_setup(case)
        self.setup = su
        g = su.grid
        self.grid = g
        self.p = dict(su.params)
        if form not in ("plain", "mixed", "learned"):
            raise ValueError(f"unknown solver form {form!r} (plain, mixed or learned)")
        self.form = form
        fp32 = form in ("mixed", "learned")
        if projection_cg_rtol is None:
            # the reference's production tolerance for the plain form; the
            # mixed form's pressure tolerance is 1e-8 relative
            projection_cg_rtol = 1.0e-6 if form == "plain" else 1.0e-8
        self.rtol = float(projection_cg_rtol)
        self.proj_maxiter = int(proj_maxiter)
        dev = self.dev
        f64 = dict(dtype=torch.float64, device=dev)
        self.n = g.n_cells
        self.shape = g.shape
        # geometry
        self.dz_t = torch.tensor(g.dz_arr, **f64)
        self.da_t = torch.tensor(g.d_face_above, **f64)
        self.db_t = torch.tensor(g.d_face_below, **f64)
        self.fsgrid = FsGrid(g.Nx, g.Ny, g.Nz, g.dx, g.dy, ptr(self.dz_t), ptr(self.da_t),
                             ptr(self.db_t))
        self.gp = _ctypes_ref(self.fsgrid)
        # state fields
        self.f = {k: torch.tensor(v, **f64).contiguous() for k, v in su.fields.items()}
        self.u_inlet = torch.tensor(su.u_inlet, **f64).contiguous()
        self.sigma_x = torch.tensor(su.sigma_sponge, **f64)
        z2 = (g.Ny, g.Nx)
        self.k_wall = torch.full(z2, K_MIN, **f64)
        self.eps_wall = torch.full(z2, EPS_MIN, **f64)
        self.zero2 = torch.zeros((g.Nz, g.Ny), **f64)
        # work arrays
        shp = g.shape
        self.w = {}
        for name in ("rho_prev", "omega", "q_rad", "q_rad_gas", "M_local", "S_F", "S_O2",
                     "S_H2O", "div_target", "tmp1", "tmp2", "tmp3", "tmp4", "tmp5", "tmp6",
                     "Q_comb"):
            self.w[name] = torch.zeros(shp, **f64)
        self.bed_out = {name: torch.zeros(shp, **f64) for name in
                        ("S_pyro", "S_drying", "Q_pyro", "Q_drying", "Y_F_source", "Q_char",
                         "Q_smold", "Q_g_conv")}
        nzb = max(g.n_z_bed, 1)
        self.hcond_scratch = torch.zeros((nzb, g.Ny, g.Nx), **f64)
        self.edc_scratch = torch.zeros(int(self.lib.fs_edc_scratch_bytes(self.n)) + 64,
                                       dtype=torch.uint8, device=dev)
        self.active_count = torch.zeros(1, dtype=torch.int64, device=dev)
        # the FP32 forms run the ten chemistry/transport sub-steps on float
        # copies (updated: T_g and the mass fractions; read-only: rho, u, v, w,
        # k, eps, nu_t and the bed sources), made once per step
        self.sub32 = None
        if fp32:
            f32 = dict(dtype=torch.float32, device=dev)
            self.sub32 = {name: torch.zeros(shp, **f32) for name in (
                "T_g", "Y_fuel", "Y_O2", "Y_H2O", "t1", "t2", "t3", "t4", "rho", "u", "v",
                "w", "k_turb", "eps_turb", "nu_t", "S_pyro", "S_drying", "Q_g_conv", "omega",
                "Q_comb")}
            self.edc32_scratch = torch.zeros(int(self.lib.fs_edc_f32_scratch_bytes(self.n)) + 64,
                                             dtype=torch.uint8, device=dev)
        # pinned host mirrors for the per-step scalar reads
        self.h_count = torch.zeros(1, dtype=torch.int64).pin_memory()
        self.h_row = torch.zeros(g.Nx, dtype=torch.float64).pin_memory()
        self.h_rows = torch.zeros((2, g.Nx), dtype=torch.float64).pin_memory()
        self.max_scratch = torch.zeros(64, dtype=torch.float64, device=dev)
        # soil
        so = su.soil
        self.soil_dz = torch.tensor(so["dz"], **f64)
        self.soil_da = torch.tensor(so["d_above"], **f64)
        self.soil_db = torch.tensor(so["d_below"], **f64)
        self.n_soil = so["n"]
        self.T_soil = torch.tensor(so["T"], **f64).contiguous()
        self.q_in_soil = torch.zeros(z2, **f64)
        # particles
        self._load_particles(su.particles)
        # projection and DOM solver objects
        h = _ctypes_void()
        check(self.lib.fs_proj_create(self.gp, _ctypes_byref(h)), "fs_proj_create")
        self.proj = h
        if mg_sweeps is not None:
            # the sweeps on every level (the finest too unless mg_fine_sweeps is
            # given), at the library's default damping
            check(self.lib.fs_proj_configure(self.proj, int(mg_sweeps), 0.9), "fs_proj_configure")
        if mg_fine_sweeps is not None:
            check(self.lib.fs_proj_set_fine_sweeps(self.proj, int(mg_fine_sweeps)),
                  "fs_proj_set_fine_sweeps")
        if fp32:
            check(self.lib.fs_proj_set_precision(self.proj, 1), "fs_proj_set_precision")
        self.net = None
        if form == "learned":
            from . import learned
            path = learned.WEIGHTS if learned_weights is None else learned_weights
            if isinstance(path, np.ndarray):
                self.net = learned.UNetPreconditioner(*g.shape, params=path)
            else:
                self.net = learned.UNetPreconditioner.load(path, *g.shape)
            learned.attach(self, self.net, learned_max, learned_stall)
        om, wq = level_symmetric(self.p["n_quadrature"])
        self.Omega, self.weights = om, wq
        h2 = _ctypes_void()
        check(self.lib.fs_dom_create(self.gp, om.shape[0], dbl_array(om[:, 0]),
                                     dbl_array(om[:, 1]), dbl_array(om[:, 2]), dbl_array(wq),
                                     KAPPA_SOOT_HOT, _ctypes_byref(h2)), "fs_dom_create")
        self.dom = h2
        # The DOM solve reads only fields that momentum, projection, sponge and
        # k-epsilon leave untouched (T_s, T_g, alpha_s, omega, Y_H2O, rho,
        # M_local) and writes only fields they do not read, so it runs on a
        # second stream from a worker thread, concurrently with them.
        self.overlap_dom = bool(overlap_dom)
        # high priority: the DOM is the longer branch, so when SMs free up the
        # block scheduler starts its kernels (each sweep CTA needs a whole SM)
        # before the main stream's
        self.s_dom = (torch.cuda.Stream(device=dev, priority=-1) if self.overlap_dom
                      else None)
        self._pool = None
        if self.overlap_dom:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=1, thread_name_prefix="dom")
        if fp32:
            check(self.lib.fs_dom_set_precision(self.dom, 1), "fs_dom_set_precision")
        if dom_sweep or dom_cluster_ctas:
            check(self.lib.fs_dom_set_sweep_mode(self.dom, int(dom_sweep or 8),
                                                 int(dom_cluster_ctas)),
                  "fs_dom_set_sweep_mode")
        if dom_kernel:
            check(self.lib.fs_dom_set_sweep_kernel(self.dom, int(dom_kernel)),
                  "fs_dom_set_sweep_kernel")
        # clock
        self.t = 0.0
        self.dt = float(self.p["dt0"])
        self.step_count = 0
        self.lset_step = 0
        self.extinct_count = 0
        self.front_t = [0.0]
        self.front_x = [float(self.p["x_front0"])]
        self.diag = StepDiag()
        self.history = []
        self.finished = None

    # ------------------------------------------------------------------ setup
    def _load_particles(self, parts):
        g = self.grid
        dev = self.dev
        self.np_particles = len(parts["x"])
        self.part = {}
        for k in ("x", "y", "z", "m_solid", "m_water", "m_char", "T_s", "m_water_0", "sav",
                  "m_char_max"):
            self.part[k] = torch.tensor(np.asarray(parts[k], dtype=np.float64), device=dev)
        alive = np.asarray(parts["alive"], dtype=np.int8).copy()
        cell = locate_particle_cells(np.asarray(parts["x"]), np.asarray(parts["y"]),
                                     np.asarray(parts["z"]), g.dx, g.dy, g.z_face, g.Nx,
                                     g.Ny, g.Nz)
        alive[cell < 0] = 0
        self.part["alive"] = torch.tensor(alive, device=dev)
        perm, starts, seg_cell = build_segments(cell)
        self.seg_perm = torch.tensor(perm, dtype=torch.int32, device=dev)
        self.seg_start = torch.tensor(starts, dtype=torch.int32, device=dev)
        self.seg_cell = torch.tensor(seg_cell, dtype=torch.int32, device=dev)
        soc = np.full(g.n_cells, -1, dtype=np.int32)
        soc[seg_cell] = np.arange(seg_cell.size, dtype=np.int32)
        self.seg_of_cell = torch.tensor(soc, device=dev)
        pp = self.part
        self.fs_parts = FsBedParticles(*(ptr(pp[k]) for k in (
            "x", "y", "z", "alive", "m_solid", "m_water", "m_char", "T_s", "m_water_0", "sav",
            "m_char_max")))
        self.fs_segs = FsBedSegments(int(seg_cell.size), ptr(self.seg_start),
                                     ptr(self.seg_cell), ptr(self.seg_perm))
        bo = self.bed_out
        self.fs_src = FsBedSources(*(ptr(bo[k]) for k in (
            "S_pyro", "S_drying", "Q_pyro", "Q_drying", "Y_F_source", "Q_char", "Q_smold",
            "Q_g_conv")))

    def load_state(self, snap: dict, t: float, dt_prev: float, step: int):
        """Overwrite the device state with a captured reference state."""
        for k in ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "T_s", "alpha_s"):
            self.f[k].copy_(torch.as_tensor(snap[k]))
        for k_src, k_dst in (("k_turb", "k_turb"), ("eps_turb", "eps_turb"), ("nu_t", "nu_t"),
                             ("phi", "phi")):
            if k_src in snap:
                self.f[k_dst].copy_(torch.as_tensor(snap[k_src]))
        for k_src, k_dst in (("omega", "omega"), ("q_rad", "q_rad"), ("q_rad_gas", "q_rad_gas")):
            if k_src in snap:
                self.w[k_dst].copy_(torch.as_tensor(snap[k_src]))
        if "T_soil" in snap:
            self.T_soil.copy_(torch.as_tensor(snap["T_soil"]))
        for k in ("x", "y", "z", "m_solid", "m_water", "m_char", "T_s", "m_water_0", "sav",
                  "m_char_max"):
            self.part[k].copy_(torch.as_tensor(snap["p_" + k]))
        self.part["alive"].copy_(torch.as_tensor(np.asarray(snap["p_alive"], dtype=np.int8)))
        if "p_prev" in snap:
            pp = torch.as_tensor(np.ascontiguousarray(snap["p_prev"]).reshape(-1))
            self.pressure_view().copy_(pp)
        if "I_set" in snap:
            I = torch.as_tensor(np.ascontiguousarray(snap["I_set"]).reshape(-1)).to(self.dev)
            check(self.lib.fs_dom_load_intensity(self.dom, ptr(I), self._s()), "dom_load")
            torch.cuda.current_stream().synchronize()
            del I
        self.t = float(t)
        self.dt = float(dt_prev)
        self.step_count = int(step)
        self.lset_step = int(snap.get("lset_step", step))
        torch.cuda.synchronize()

    def close(self):
        if getattr(self, "_pool", None) is not None:
            self._pool.shutdown(wait=True)
            self._pool = None
        if getattr(self, "proj", None):
            self.lib.fs_proj_destroy(self.proj)
            self.proj = None
        if getattr(self, "net", None) is not None:
            self.net.close()
            self.net = None
        if getattr(self, "dom", None):
            self.lib.fs_dom_destroy(self.dom)
            self.dom = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --------------------------------------------------------------- helpers
    def enable_phase_timers(self, on=True):
        """Accumulate CUDA-event time per phase of the step (diagnostics)."""
        self._timers = {} if on else None
        self._mark = None

    def _phase(self, label):
        hook = getattr(self, "phase_hook", None)
        if hook is not None:
            hook(label)  # e.g. HostStepper's early download (api.py)
        tm = getattr(self, "_timers", None)
        if tm is None:
            return
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        if self._mark is not None:
            lab0, ev0 = self._mark
            tm.setdefault(lab0, []).append((ev0, ev))
        self._mark = (label, ev) if label else None

    def enable_kernel_timers(self, on=True):
        """Bracket individual kernel launches with CUDA events (same stream)."""
        self._kt_on = bool(on)
        self._kt = {}
        if getattr(self, "dom", None):
            self.lib.fs_dom_sweep_timing(self.dom, 1 if on else 0, None, None)

    def _ktime(self, label):
        if not getattr(self, "_kt_on", False):
            return _NullCtx()
        return _KernelTimer(self._kt, label)

    def kernel_times(self):
        """{kernel: (total ms, launches)} of the bracketed kernels."""
        torch.cuda.synchronize()
        out = {k: (sum(a.elapsed_time(b) for a, b in v), len(v))
               for k, v in getattr(self, "_kt", {}).items()}
        if getattr(self, "dom", None):
            ms = _C.c_double()
            cnt = _C.c_longlong()
            self.lib.fs_dom_sweep_timing(self.dom, -1, _C.byref(ms), _C.byref(cnt))
            if cnt.value:
                out["dom_sweep"] = (ms.value, cnt.value)
        return out

    def phase_times(self):
        """{phase: total milliseconds} of the phases recorded so far."""
        torch.cuda.synchronize()
        out = {}
        for k, pairs in (getattr(self, "_timers", None) or {}).items():
            out[k] = sum(a.elapsed_time(b) for a, b in pairs)
        return out

    def _s(self):
        return torch.cuda.current_stream(self.dev).cuda_stream

    def _max(self, t, mode):
        out = _ctypes_double()
        check(self.lib.fs_field_max(self.gp, ptr(t), mode, _ctypes_byref(out), self._s()),
              "fs_field_max")
        return out.value

    def _swap(self, name, buf):
        old = self.f[name]
        self.f[name] = self.w[buf]
        self.w[buf] = old

    # ------------------------------------------------------------------ step
    def step(self):
        """One outer step; returns False once the reference loop would exit."""
        L, g, p, f, w = self.lib, self.grid, self.p, self.f, self.w
        s = self._s()
        gp = self.gp
        self.step_count += 1
        d = StepDiag()
        # --- 0. adaptive dt (spread_3d.py:1906-1941)
        self._phase("dt")
        mu_, mv_, mw_, mnu_, mT_ = self._maxes([f["u"], f["v"], f["w"], f["nu_t"], f["T_g"]],
                                               [0, 0, 0, 1, 1])
        u_now = max(mu_, mv_, mw_, p["U_mf"], math.sqrt(G_ACC * p["h_bed"] * 0.5), 0.1)
        nu_now = max(mnu_, 1.0e-3)
        dz_min = p["dz_min"]
        dt_adv = p["cfl"] * min(g.dx, g.dy, dz_min) / u_now
        dt_diff = 0.25 * dz_min * dz_min / nu_now
        dt_new = min(dt_adv, dt_diff, 0.05)
        dt_new = min(dt_new, self.dt * 1.5)
        if dt_new < p["min_dt_s"]:
            dt_new = p["min_dt_s"]
        if not math.isfinite(mT_):
            raise RuntimeError(f"State NaN/Inf at t={self.t:.3f}s -- simulation exploded.")
        self.dt = dt = dt_new
        t = self.t
        ign = t < p["ignition_duration_s"]
        # --- 1. rho_prev, EoS, inlet O2 (spread_3d.py:1984-2050)
        self._phase("eos")
        check(L.fs_eos(gp, ptr(f["rho"]), ptr(w["rho_prev"]), ptr(f["T_g"]), ptr(f["Y_O2"]),
                       p["T_amb"], s), "eos")
        # --- 2. Lagrangian bed (spread_3d.py:2064-2181)
        self._phase("bed")
        bp = FsBedParams(dt, p["h_conv"], p["rho_solid_true"], p["cp_solid"], p["eps_solid"],
                         p["T_amb"], p["view_factor"], p["h_bed"], p["kappa_bed_eff"],
                         p["char_ox_flux_cap"], p["char_ox_ash_exp"], 1, 1, 1, 1,
                         p["drying_mode"], int(p["view_factor_geometric"]), p["n_per_cell"],
                         None, ptr(w["q_rad"]), int(ign), g.n_z_bed, p["i_src_start"],
                         p["i_src_end"])
        check(L.fs_bed_step(gp, _ctypes_ref(self.fs_parts), _ctypes_ref(self.fs_segs),
                            _ctypes_ref(self.fs_src), _ctypes_ref(bp), ptr(f["T_g"]),
                            ptr(f["Y_O2"]), s), "bed_step")
        check(L.fs_bed_aggregate(_ctypes_ref(self.fs_parts), _ctypes_ref(self.fs_segs),
                                 ptr(f["T_s"]), 0, s), "bed_aggregate_Ts")
        check(L.fs_bed_hcond(gp, ptr(f["T_s"]), ptr(self.hcond_scratch), ptr(f["alpha_s"]),
                             g.n_z_bed, 0.20, p["rho_solid_true"], p["cp_solid"], dt,
                             _ctypes_ref(self.fs_parts), _ctypes_ref(self.fs_segs),
                             ptr(self.seg_of_cell), s), "bed_hcond")
        Sp, Sd = self.bed_out["S_pyro"], self.bed_out["S_drying"]
        # --- 8 (started here). DOM + M_local aggregation on the second stream
        dom_now = self.step_count % max(p["dom_subcycle_every"], 1) == 0
        dom_job = None
        if dom_now and self.overlap_dom:
            ready = torch.cuda.Event()
            ready.record(torch.cuda.current_stream(self.dev))
            dom_args = (ptr(f["T_s"]), ptr(f["T_g"]), ptr(f["alpha_s"]), ptr(w["omega"]),
                        ptr(f["Y_H2O"]), ptr(f["rho"]), ptr(w["M_local"]), ptr(w["q_rad"]),
                        ptr(w["q_rad_gas"]))
            from concurrent.futures import Future
            self._dom_inputs = Future()
            dom_job = self._pool.submit(self._dom_job, ready, dom_args)
        # --- 3/4. drag + tentative momentum (spread_3d.py:2223-2276)
        self._phase("momentum")
        with self._ktime("momentum_drag"):
            check(L.fs_tentative_velocity(gp, ptr(f["u"]), ptr(f["v"]), ptr(f["w"]),
                                          ptr(f["rho"]), ptr(f["T_g"]), None, None, None,
                                          ptr(f["alpha_s"]), p["sav"], p["canopy_C_d"],
                                          ptr(self.u_inlet), ptr(self.zero2), ptr(self.zero2),
                                          ptr(w["tmp1"]), ptr(w["tmp2"]), ptr(w["tmp3"]), dt,
                                          p["T_amb"], s), "momentum")
        self._swap("u", "tmp1")
        self._swap("v", "tmp2")
        self._swap("w", "tmp3")
        # --- 5. projection (spread_3d.py:2300-2360)
        self._phase("projection")
        self._div_target(dt)
        check(L.fs_proj_rebuild(self.proj, ptr(f["rho"]), s), "proj_rebuild")
        n_it = 0
        div_max = 0.0
        ktp = self._ktime("projection")
        ktp.__enter__()
        for _it in range(p["proj_max_iter"]):
            its = _ctypes_int()
            check(L.fs_proj_project(self.proj, ptr(f["u"]), ptr(f["v"]), ptr(f["w"]),
                                    ptr(self.u_inlet), ptr(w["div_target"]), dt, self.rtol,
                                    self.proj_maxiter, _ctypes_byref(its), s), "proj_project")
            d.cg_iters.append(its.value)
            res = _ctypes_double()
            check(L.fs_divergence_max(gp, ptr(f["u"]), ptr(f["v"]), ptr(f["w"]),
                                      ptr(self.u_inlet), ptr(w["div_target"]), None,
                                      _ctypes_byref(res), s), "divergence")
            div_max = res.value
            n_it = _it + 1
            if div_max < p["proj_div_tol"]:
                break
        ktp.__exit__(None, None, None)
        d.proj_iters = n_it
        d.proj_div_max = div_max
        # --- 6. outflow sponge (spread_3d.py:2369)
        self._phase("sponge")
        check(L.fs_outflow_sponge(gp, ptr(f["u"]), ptr(self.u_inlet), ptr(self.sigma_x),
                                  ptr(f["Y_fuel"]), 1.0e-3, dt, s), "sponge")
        # --- 7. k-epsilon (spread_3d.py:2409)
        self._phase("k_eps")
        with self._ktime("k_epsilon"):
            check(L.fs_k_epsilon(gp, ptr(f["k_turb"]), ptr(f["eps_turb"]), ptr(f["u"]),
                                 ptr(f["v"]), ptr(f["w"]), ptr(f["T_g"]), ptr(f["alpha_s"]),
                                 ptr(self.u_inlet), ptr(self.k_wall), ptr(self.eps_wall),
                                 ptr(w["tmp1"]), ptr(w["tmp2"]), ptr(w["tmp3"]), None, None,
                                 p["sav"], dt, p["T_amb"], p["canopy_beta_p"],
                                 p["canopy_beta_d"], s), "k_eps")
        self._swap("k_turb", "tmp1")
        self._swap("eps_turb", "tmp2")
        self._swap("nu_t", "tmp3")
        # --- 8. DOM (every dom_subcycle_every steps) + soil (spread_3d.py:2472-2514)
        self._phase("dom")
        dt_sub = dt / N_SUB
        drip = int(ign)
        early = None
        if dom_job is not None:
            # Once the DOM has read its input fields, the work that follows it
            # but does not read its outputs (the flame mask, the gas advection
            # and the chemistry and species half of the first sub-step) runs
            # while the sweeps are still going; nothing it writes is read by
            # the soil step or the ignition pulse, so the order of the values
            # is that of the reference loop.
            ev_in = self._dom_inputs.result()
            torch.cuda.current_stream(self.dev).wait_event(ev_in)
            self._flame_mask_and_gas_adv(dt)
            early = self._substep_prep()
            self._to32()
            self._substep_chem(dt_sub, Sp, Sd, *early)
            done = dom_job.result()
            torch.cuda.current_stream(self.dev).wait_event(done)
            d.dom_iters = L.fs_dom_iterations(self.dom)
        elif dom_now:
            check(L.fs_bed_aggregate(_ctypes_ref(self.fs_parts), _ctypes_ref(self.fs_segs),
                                     ptr(w["M_local"]), 1, s), "bed_aggregate_M")
            check(L.fs_dom_solve(self.dom, ptr(f["T_s"]), ptr(f["T_g"]), ptr(f["alpha_s"]),
                                 ptr(w["omega"]), p["sav"], p["T_amb"], ptr(self.T_soil[0]),
                                 ptr(f["Y_H2O"]), ptr(f["rho"]), ptr(w["M_local"]),
                                 ptr(w["q_rad"]), ptr(w["q_rad_gas"]), ptr(self.q_in_soil), s),
                  "dom_solve")
            d.dom_iters = L.fs_dom_iterations(self.dom)
        check(L.fs_soil_step(self.n_soil, g.Ny, g.Nx, ptr(self.T_soil), ptr(self.q_in_soil), dt,
                             ptr(self.soil_dz), ptr(self.soil_da), ptr(self.soil_db), 0.48,
                             1500.0, 800.0, 0.85, p["T_amb"], s), "soil")
        # --- 9. ignition pulse on the top bed layer of the source strip (:2528-2532)
        self._phase("misc")
        if ign and g.n_z_bed > 0:
            check(L.fs_ignition_pulse(gp, ptr(w["q_rad"]), int(g.n_z_bed - 1),
                                      int(p["i_src_start"]), int(p["i_src_end"]),
                                      240_000.0 * float(p["ignition_q_mult"]), s),
                  "ignition_pulse")
        if early is None:
            # --- 10/11. flame mask, gas-temperature advection
            self._flame_mask_and_gas_adv(dt)
            early = self._substep_prep()
            self._to32()
            self._substep_chem(dt_sub, Sp, Sd, *early)
        # --- 12. ten chemistry/transport sub-steps (:2678-3196); the first one's
        # chemistry and species half ran above
        n_sc, dts_sc, n_pr, dts_pr = early
        d.n_sub_sc, d.n_sub_pr = n_sc, n_pr
        for _sub in range(N_SUB):
            if _sub > 0:
                self._substep_chem(dt_sub, Sp, Sd, n_sc, dts_sc, n_pr, dts_pr)
            self._substep_energy(dt_sub, Sp, Sd, drip, n_pr, dts_pr)
        self._from32()
        # --- 13. level set (passive: v_n = 0, so evolve leaves phi; reinit every 10)
        self._phase("levelset")
        self.lset_step += 1
        if self.lset_step % 10 == 0:
            self._reinit_levelset()
        # one wait for the exit tests and the front tracking: the active-cell
        # count and the two phi rows they read (phi does not change again in
        # this step, so the second row may be read before the closing EoS)
        stream = torch.cuda.current_stream(self.dev)
        self.h_count.copy_(self.active_count, non_blocking=True)
        self.h_rows[0].copy_(f["phi"][1, g.Ny // 2, :], non_blocking=True)
        self.h_rows[1].copy_(f["phi"][g.n_z_bed // 2, g.Ny // 2, :], non_blocking=True)
        stream.synchronize()
        if self.lib.fs_stencil_status(1) != 0:
            raise _lib.FireStepError(4, "a stencil kernel's bounded shared-memory staging wait "
                                        "gave up (or the flag could not be read)")
        n_active = int(self.h_count[0])
        front_lset = self._front_from_row(self.h_rows[0].numpy())
        exit_now = False
        if n_active == 0 and t > p["ignition_duration_s"] + 2.0:
            self.extinct_count += 1
            if self.extinct_count > 50:
                exit_now = True
        else:
            self.extinct_count = 0
        if front_lset > float(self.case.get("bed_x_end", g.Lx)) - g.dx:
            exit_now = True
        if exit_now:
            self.finished = "exit"
            return False
        # --- 14. closing EoS (:3440) and clock
        check(L.fs_eos(gp, ptr(f["rho"]), None, ptr(f["T_g"]), None, p["T_amb"], s), "eos2")
        fx = self._front_from_row(self.h_rows[1].numpy())
        if math.isfinite(fx) and fx > self.front_x[-1]:
            self.front_t.append(t)
            self.front_x.append(fx)
        self._phase(None)
        self.t = t + dt
        d.t, d.dt = self.t, dt
        self.diag = d
        return True

    def _flame_mask_and_gas_adv(self, dt):
        """Steps 10-11 of the loop: the flame-mask count and the gas
        temperature advection (spread_3d.py:2648, flame_front_3d.py:756-813)."""
        L, f, w, p, gp = self.lib, self.f, self.w, self.p, self.gp
        s = self._s()
        self.active_count.zero_()
        check(L.fs_active_count(self.n, ptr(w["omega"]), ptr(f["T_g"]), ptr(f["Y_fuel"]),
                                ptr(self.active_count), None, s), "active_count")
        self._phase("gas_adv")
        with self._ktime("gas_energy_adv"):
            check(L.fs_gas_energy_adv(gp, ptr(f["T_g"]), ptr(f["u"]), ptr(f["v"]), ptr(f["w"]),
                                      ptr(w["tmp1"]), dt, 2.0e-5, p["T_amb"], s), "gas_adv")
        self._swap("T_g", "tmp1")

    def _substep_prep(self):
        """Sub-step counts of the turbulent diffusion from the interior maximum
        of nu_t (turbulence_3d.py:880-915), for species and for temperature."""
        self._phase("substeps")
        dt_sub = self.dt / N_SUB
        nu_in = self._maxes([self.f["nu_t"]], [2])[0]
        n_sc, dts_sc = self._nsub_from(nu_in, SC_T, dt_sub)
        n_pr, dts_pr = self._nsub_from(nu_in, PR_T, dt_sub)
        return n_sc, dts_sc, n_pr, dts_pr

    _TO32 = (("T_g", "f"), ("Y_fuel", "f"), ("Y_O2", "f"), ("Y_H2O", "f"), ("rho", "f"),
             ("u", "f"), ("v", "f"), ("w", "f"), ("k_turb", "f"), ("eps_turb", "f"),
             ("nu_t", "f"), ("S_pyro", "b"), ("S_drying", "b"), ("Q_g_conv", "b"))
    _FROM32 = (("T_g", "f"), ("Y_fuel", "f"), ("Y_O2", "f"), ("Y_H2O", "f"), ("omega", "w"),
               ("Q_comb", "w"))

    def _to32(self):
        """FP32 copies of the fields the sub-steps read (FP32 forms only)."""
        if self.sub32 is None:
            return
        src = [(self.f if kind == "f" else self.bed_out)[name] for name, kind in self._TO32]
        dst = [self.sub32[name] for name, _ in self._TO32]
        check(self.lib.fs_convert(self.n, len(src), ptr_array(src), ptr_array(dst), 1,
                                  self._s()), "to_f32")

    def _from32(self):
        """The sub-steps' results back into the FP64 state (FP32 forms only)."""
        if self.sub32 is None:
            return
        src = [self.sub32[name] for name, _ in self._FROM32]
        dst = [(self.f if kind == "f" else self.w)[name] for name, kind in self._FROM32]
        check(self.lib.fs_convert(self.n, len(src), ptr_array(src), ptr_array(dst), 0,
                                  self._s()), "to_f64")

    def _swap32(self, name, buf):
        t = self.sub32
        t[name], t[buf] = t[buf], t[name]

    def _substep_chem32(self, dt_sub, n_sc, dts_sc):
        """The FP32 form of _substep_chem (fs_edc_f32, fs_species_step_f32,
        fs_turb_diffusion_substep_f32 on the float copies)."""
        L, p, gp, t = self.lib, self.p, self.gp, self.sub32
        s = self._s()
        self._phase("edc")
        with self._ktime("edc"):
            check(L.fs_edc_f32(self.n, ptr(t["rho"]), ptr(t["T_g"]), ptr(t["Y_fuel"]),
                               ptr(t["Y_O2"]), ptr(t["k_turb"]), ptr(t["eps_turb"]),
                               ptr(t["Y_H2O"]), ptr(t["omega"]), p["chi_rad"], 1100.0, dt_sub,
                               1, 1.3, 17_000_000.0, int(p["edc_extinction_enable"]),
                               ptr(self.edc32_scratch), s), "edc_f32")
        self._phase("species")
        Ys = [t["Y_fuel"], t["Y_O2"], t["Y_H2O"]]
        Yo = [t["t1"], t["t2"], t["t3"]]
        with self._ktime("species_transport"):
            check(L.fs_species_step_f32(gp, ptr_array(Ys), ptr_array(Yo), ptr(t["S_pyro"]),
                                        ptr(t["S_drying"]), dbl_array([0.0, 0.232, 0.0]),
                                        ptr(t["rho"]), ptr(t["u"]), ptr(t["v"]), ptr(t["w"]),
                                        dt_sub, 1.0e-5, 0.232, s), "species_f32")
        self._swap32("Y_fuel", "t1")
        self._swap32("Y_O2", "t2")
        self._swap32("Y_H2O", "t3")
        self._phase("turb_diff_Y")
        for q in range(n_sc):
            Ys = [t["Y_fuel"], t["Y_O2"], t["Y_H2O"]]
            Yo = [t["t1"], t["t2"], t["t3"]]
            with self._ktime("turb_diffusion_Y"):
                check(L.fs_turb_diffusion_substep_f32(
                    gp, 3, ptr_array(Ys), ptr_array(Yo), ptr(t["nu_t"]), SC_T, dts_sc,
                    int(q == n_sc - 1), dbl_array([0.0, 0.0, 0.0]),
                    dbl_array([1.0, 0.232, 1.0]), s), "turb_diff_Y_f32")
            self._swap32("Y_fuel", "t1")
            self._swap32("Y_O2", "t2")
            self._swap32("Y_H2O", "t3")

    def _substep_energy32(self, dt_sub, drip, n_pr, dts_pr):
        """The FP32 form of _substep_energy (the solid conduction stays FP64)."""
        L, f, w, p, gp, g, t = self.lib, self.f, self.w, self.p, self.gp, self.grid, self.sub32
        s = self._s()
        self._phase("gas_update")
        check(L.fs_gas_energy_update_f32(gp, ptr(t["T_g"]), ptr(t["rho"]), ptr(t["Y_H2O"]),
                                         ptr(f["T_s"]), ptr(t["S_pyro"]), ptr(t["S_drying"]),
                                         ptr(t["Q_g_conv"]), ptr(w["q_rad_gas"]),
                                         ptr(t["Q_comb"]), dt_sub, p["T_amb"], p["h_bed"], drip,
                                         g.n_z_bed, p["i_src_start"], p["i_src_end"], s),
              "gas_update_f32")
        self._phase("solid_cond")
        check(L.fs_solid_conduction_capped(gp, ptr(f["T_s"]), ptr(f["alpha_s"]), ptr(w["tmp4"]),
                                           0.20, 500.0, 1300.0, dt_sub, p["T_amb"], T_CAP, s),
              "solid_cond")
        self._swap("T_s", "tmp4")
        self._phase("turb_diff_T")
        if n_pr > 0:
            for q in range(n_pr):
                check(L.fs_turb_diffusion_substep_f32(
                    gp, 1, ptr_array([t["T_g"]]), ptr_array([t["t4"]]), ptr(t["nu_t"]), PR_T,
                    dts_pr, int(q == n_pr - 1), dbl_array([p["T_amb"]]), dbl_array([T_CAP]),
                    s), "turb_diff_T_f32")
                self._swap32("T_g", "t4")
        else:
            check(L.fs_clip_f32(self.n, ptr(t["T_g"]), p["T_amb"], T_CAP, s), "cap_Tg_f32")

    def _substep_chem(self, dt_sub, Sp, Sd, n_sc, dts_sc, n_pr, dts_pr):
        """First half of a chemistry/transport sub-step: EDC, species sources
        and transport, the O2 clip and the turbulent diffusion of the species
        (spread_3d.py:2678-3060)."""
        if self.sub32 is not None:
            return self._substep_chem32(dt_sub, n_sc, dts_sc)
        L, f, w, p, gp = self.lib, self.f, self.w, self.p, self.gp
        s = self._s()
        self._phase("edc")
        with self._ktime("edc"):
            check(L.fs_edc(self.n, ptr(f["rho"]), ptr(f["T_g"]), ptr(f["Y_fuel"]),
                           ptr(f["Y_O2"]), ptr(f["k_turb"]), ptr(f["eps_turb"]),
                           ptr(f["Y_H2O"]), ptr(w["omega"]), p["chi_rad"], 1100.0, dt_sub,
                           1, 1.3, 17_000_000.0, int(p["edc_extinction_enable"]),
                           ptr(self.edc_scratch), s), "edc")
        self._phase("species")
        # sources with dilution, transport of the three species and the O2
        # clip in one pass (fs_species_step; equal to the three calls)
        Ys = [f["Y_fuel"], f["Y_O2"], f["Y_H2O"]]
        Yo = [w["tmp1"], w["tmp2"], w["tmp3"]]
        with self._ktime("species_transport"):
            check(L.fs_species_step(gp, ptr_array(Ys), ptr_array(Yo), ptr(Sp), ptr(Sd),
                                    dbl_array([0.0, 0.232, 0.0]), ptr(f["rho"]), ptr(f["u"]),
                                    ptr(f["v"]), ptr(f["w"]), dt_sub, 1.0e-5, 0.232, s),
                  "species")
        self._swap("Y_fuel", "tmp1")
        self._swap("Y_O2", "tmp2")
        self._swap("Y_H2O", "tmp3")
        self._phase("turb_diff_Y")
        if n_sc > 0:
            for q in range(n_sc):
                last = q == n_sc - 1
                Ys = [f["Y_fuel"], f["Y_O2"], f["Y_H2O"]]
                Yo = [w["tmp1"], w["tmp2"], w["tmp3"]]
                with self._ktime("turb_diffusion_Y"):
                    check(L.fs_turb_diffusion_substep(
                        gp, 3, ptr_array(Ys), ptr_array(Yo), ptr(f["nu_t"]), SC_T, dts_sc,
                        int(last), dbl_array([0.0, 0.0, 0.0]),
                        dbl_array([1.0, 0.232, 1.0]), s), "turb_diff_Y")
                self._swap("Y_fuel", "tmp1")
                self._swap("Y_O2", "tmp2")
                self._swap("Y_H2O", "tmp3")

    def _substep_energy(self, dt_sub, Sp, Sd, drip, n_pr, dts_pr):
        """Second half of a sub-step: gas-energy update with the radiative
        gas source, vertical solid conduction, turbulent diffusion of T_g and
        the caps (spread_3d.py:3104-3196)."""
        if self.sub32 is not None:
            return self._substep_energy32(dt_sub, drip, n_pr, dts_pr)
        L, f, w, p, gp, g = self.lib, self.f, self.w, self.p, self.gp, self.grid
        s = self._s()
        self._phase("gas_update")
        # the gas-energy update and the vertical solid conduction with the T_s
        # cap of the sub-step's end in one pass: both read the old T_s and
        # nothing between them reads or writes it (spread_3d.py:3104-3196)
        check(L.fs_gas_energy_solid_update(gp, ptr(f["T_g"]), ptr(f["rho"]), ptr(f["Y_H2O"]),
                                           ptr(f["T_s"]), ptr(Sp), ptr(Sd),
                                           ptr(self.bed_out["Q_g_conv"]), ptr(w["q_rad_gas"]),
                                           ptr(w["Q_comb"]), dt_sub, p["T_amb"], p["h_bed"],
                                           drip, g.n_z_bed, p["i_src_start"], p["i_src_end"],
                                           ptr(f["alpha_s"]), ptr(w["tmp4"]), 0.20, 500.0,
                                           1300.0, p["T_amb"], T_CAP, s),
              "gas_update + solid_cond")
        self._swap("T_s", "tmp4")
        self._phase("turb_diff_T")
        if n_pr > 0:
            for q in range(n_pr):
                last = q == n_pr - 1
                check(L.fs_turb_diffusion_substep(
                    gp, 1, ptr_array([f["T_g"]]), ptr_array([w["tmp4"]]), ptr(f["nu_t"]),
                    PR_T, dts_pr, int(last), dbl_array([p["T_amb"]]), dbl_array([T_CAP]),
                    s), "turb_diff_T")
                self._swap("T_g", "tmp4")
        else:
            check(L.fs_clip(self.n, ptr(f["T_g"]), p["T_amb"], T_CAP, s), "cap_Tg")

    def _dom_job(self, ready, a):
        """M_local aggregation and the DOM solve on the second stream, after
        the bed work queued before ``ready``; returns the event that marks the
        end of that work."""
        torch.cuda.set_device(self.dev)
        st = self.s_dom
        st.wait_event(ready)
        sp = st.cuda_stream
        L, p = self.lib, self.p
        Ts, Tg, a_s, om, YH, rho, Ml, qr, qrg = a
        try:
            check(L.fs_bed_aggregate(_ctypes_ref(self.fs_parts), _ctypes_ref(self.fs_segs), Ml,
                                     1, sp), "bed_aggregate_M")
            check(L.fs_dom_begin(self.dom, Ts, Tg, a_s, om, p["sav"], p["T_amb"],
                                 ptr(self.T_soil[0]), YH, rho, Ml, sp), "dom_begin")
            inputs = torch.cuda.Event()
            inputs.record(st)
            self._dom_inputs.set_result(inputs)
        except BaseException as e:
            self._dom_inputs.set_exception(e)
            raise
        check(L.fs_dom_end(self.dom, qr, qrg, ptr(self.q_in_soil), sp), "dom_end")
        done = torch.cuda.Event()
        done.record(st)
        return done

    def _div_target(self, dt):
        # (S_pyro - (rho - rho_prev)/dt) / max(rho, 0.1), S_pyro = Sp + Sd (:2147, :2317)
        f, w = self.f, self.w
        check(self.lib.fs_div_target(self.n, ptr(f["rho"]), ptr(w["rho_prev"]),
                                     ptr(self.bed_out["S_pyro"]), ptr(self.bed_out["S_drying"]),
                                     dt, ptr(w["div_target"]), self._s()), "div_target")

    def _maxes(self, tensors, modes):
        res = (_C.c_double * len(tensors))()
        md = (_C.c_int * len(modes))(*modes)
        check(self.lib.fs_field_max_multi(self.gp, len(tensors), ptr_array(tensors), md, res,
                                          ptr(self.max_scratch), self._s()), "maxima")
        return list(res)

    def _nsub_from(self, nu_max, sc, dt):
        """turbulence_3d.py:880-915 sub-step count from the interior nu_t maximum."""
        g = self.grid
        dz_min = self.p["dz_min"]
        h_min2 = min(g.dx * g.dx, min(g.dy * g.dy, dz_min * dz_min))
        D_max = nu_max / sc
        if D_max <= 1.0e-12 or not math.isfinite(D_max):
            return 0, 0.0
        dt_sub_max = 0.4 * h_min2 / D_max
        if dt_sub_max <= 0.0:
            return 0, 0.0
        target = dt / dt_sub_max
        if target > 1000:
            return 0, 0.0
        n = max(1, int(math.ceil(target)))
        return n, dt / n

    def _nsub(self, sc, dt_sub):
        n = _ctypes_int()
        dts = _ctypes_double()
        check(self.lib.fs_turb_diffusion_nsub(self.gp, ptr(self.f["nu_t"]), sc, dt_sub,
                                              _ctypes_byref(n), _ctypes_byref(dts), self._s()),
              "nsub")
        return n.value, dts.value

    def _reinit_levelset(self):
        # LevelSetFront3D.reinitialize (flame_front_3d.py:339-355)
        g = self.grid
        phi0 = self.f["phi"].clone()
        dtau = 0.5 * min(g.dx, g.dy, float(g.dz_arr.min()))
        for _ in range(5):
            check(self.lib.fs_levelset(self.gp, ptr(self.f["phi"]), ptr(phi0),
                                       ptr(self.w["tmp5"]), dtau, 2, self._s()), "reinit")
            self._swap("phi", "tmp5")

    def _front_x(self, k, j):
        src = self.f["phi"][k, j, :]
        check(self.lib.fs_copy_to_host(self.h_row.data_ptr(), src.data_ptr(),
                                       8 * self.grid.Nx, self._s()), "front_row")
        return self._front_from_row(self.h_row.numpy())

    def _front_from_row(self, row):
        """x of the first sign change of phi along a host row (spread_3d.py:3743)."""
        for i in range(row.size - 1):
            a, b = row[i], row[i + 1]
            if a < 0.0 < b or b < 0.0 < a:
                return (i + (-a / (b - a)) + 0.5) * self.grid.dx
        return float("inf")

    # -------------------------------------------------------------- access
    def state(self):
        """Host copy of the solver state, keyed like the reference fixtures."""
        torch.cuda.synchronize()
        out = {k: self.f[k].cpu().numpy().copy() for k in self.FIELDS}
        out["omega"] = self.w["omega"].cpu().numpy().copy()
        out["q_rad"] = self.w["q_rad"].cpu().numpy().copy()
        out["q_rad_gas"] = self.w["q_rad_gas"].cpu().numpy().copy()
        out["T_soil"] = self.T_soil.cpu().numpy().copy()
        out["S_pyro_b"] = self.bed_out["S_pyro"].cpu().numpy().copy()
        out["S_dry_b"] = self.bed_out["S_drying"].cpu().numpy().copy()
        out["Q_gconv_b"] = self.bed_out["Q_g_conv"].cpu().numpy().copy()
        out["M_local"] = self.w["M_local"].cpu().numpy().copy()
        for k, v in self.part.items():
            out["p_" + k] = v.cpu().numpy().copy()
        out["p_prev"] = self.pressure_view().cpu().numpy().reshape(self.shape).copy()
        iv = self.intensity_view()
        if iv is not None:
            M = self.Omega.shape[0]
            out["I_set"] = iv.cpu().numpy().reshape((M,) + self.shape).copy()
        return out

    def pressure_view(self):
        """Zero-copy view of the projection's pressure (warm-start) buffer."""
        return _DeviceBuffer(self.lib.fs_proj_pressure(self.proj), self.n, self.dev).tensor()

    def intensity_view(self):
        """Zero-copy view of the full DOM intensities (M x cells), or None when
        the sweep path keeps only the periodic inflow rows."""
        addr = self.lib.fs_dom_intensity(self.dom)
        if not addr:
            return None
        M = self.Omega.shape[0]
        return _DeviceBuffer(addr, self.n * M, self.dev).tensor()


# ---- small ctypes helpers --------------------------------------------------
import ctypes as _C  # noqa: E402


class _NullCtx:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class _KernelTimer:
    def __init__(self, store, label):
        self.store, self.label = store, label

    def __enter__(self):
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)
        self.e0.record()
        return self

    def __exit__(self, *a):
        self.e1.record()
        self.store.setdefault(self.label, []).append((self.e0, self.e1))
        return False


def _ctypes_ref(obj):
    return _C.byref(obj)


def _ctypes_byref(obj):
    return _C.byref(obj)


def _ctypes_void():
    return _C.c_void_p()


def _ctypes_int():
    return _C.c_int()


def _ctypes_double():
    return _C.c_double()


class _DeviceBuffer:
    """Expose library-owned device memory as a torch tensor via __cuda_array_interface__."""

    def __init__(self, addr, n, device):
        self.__cuda_array_interface__ = {
            "shape": (int(n),), "typestr": "<f8", "data": (int(addr), False), "version": 3,
            "strides": None,
        }
        self.device = device

    def tensor(self):
        return torch.as_tensor(self, device=self.device)
