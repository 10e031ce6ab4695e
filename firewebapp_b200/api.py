"""Public entry points of the Tier-3 drop-in.

``run_3d_spread_gpu`` is the production mode of the boundary: it takes a case
(the deck keys ``cases.py`` names, plus the wind speed), runs the
``run_3d_spread`` loop (``spread_3d.py:1897-3683``) device-resident, records
the per-step diagnostics the reference appends (``spread_3d.py:3503-3512``)
and returns a :class:`Spread3DResultGPU` whose ``save`` writes the same
``.npz`` keys as ``Spread3DResult.save`` (``spread_3d.py:460-511``).

``HostStepper`` is the kernel-level mode: the caller owns the state in host
memory (as the reference's caller owns its numpy arrays,
``spread_3d.py:1529-1580``) and each ``step`` uploads it, advances one outer
step and downloads it again.  The persistent solver objects (projection
warm-start pressure, DOM intensities) stay on the device, as the reference's
``ProjectionSolver3D`` and ``DOMRadiationSolver`` keep them
(``projection_3d.py:755,791``, ``dom_3d.py:286-300``).
"""
from __future__ import annotations

import ctypes as _C
import gc
import json
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from ._lib import FsColumnDiag, check, ptr, ptr_array
from .solver import Tier3Solver, _ctypes_double

HOC_J = 1.7e7            # heat of combustion, _constants.py:36
T_IGN_ROS = 600.0        # _cheney_phase16_worker.py:208-231 ignition threshold


@dataclass
class Spread3DResultGPU:
    """Fields of ``Spread3DResult`` (``spread_3d.py:425-451``) for a GPU run."""
    ros_m_s: float
    n_cells_ignited: int
    front_t: list
    front_x: list
    grid: object
    state_final: dict
    diag_t: list = field(default_factory=list)
    diag_Tg_max: list = field(default_factory=list)
    diag_Ts_max: list = field(default_factory=list)
    diag_Sp_max: list = field(default_factory=list)
    diag_Qc_max: list = field(default_factory=list)
    diag_omega_max: list = field(default_factory=list)
    diag_Y_max: list = field(default_factory=list)
    diag_n_ign: list = field(default_factory=list)
    diag_proj_div_max: list = field(default_factory=list)
    diag_proj_n_iter: list = field(default_factory=list)
    k_turb_final: np.ndarray | None = None
    eps_turb_final: np.ndarray | None = None
    nu_t_final: np.ndarray | None = None
    ros_Ts: float | None = None
    hrrpua_peak: float | None = None
    snap_t: list = field(default_factory=list)
    snap_lead_x: list = field(default_factory=list)

    def save(self, path, metadata=None):
        """Write the ``Spread3DResult.save`` key set (``spread_3d.py:460-511``).

        State arrays the Lagrangian production path does not carry (p_dyn,
        Y_CO and the Eulerian component masses) are written as zeros, which
        is what they hold in the reference for this path."""
        path = Path(path)
        if not str(path).endswith(".npz"):
            path = path.with_suffix(".npz")
        path.parent.mkdir(parents=True, exist_ok=True)
        g, s = self.grid, self.state_final
        z = np.zeros(g.shape)
        np.savez_compressed(
            path,
            _meta_json=np.array(json.dumps({
                "ros_m_s": float(self.ros_m_s), "n_cells_ignited": int(self.n_cells_ignited),
                "Nx": int(g.Nx), "Ny": int(g.Ny), "Nz": int(g.Nz), "dx": float(g.dx),
                "dy": float(g.dy), "dz": float(g.dz), "Lx": float(g.Lx), "Ly": float(g.Ly),
                "Lz": float(g.Lz), "n_z_bed": int(g.n_z_bed), "user": metadata or {}})),
            x_mid=g.x_mid, y_mid=g.y_mid, z_mid=g.z_mid, dz_arr=g.dz_arr,
            inv_dz_arr=1.0 / g.dz_arr, z_face=g.z_face, d_face_above=g.d_face_above,
            d_face_below=g.d_face_below,
            rho=s["rho"], u=s["u"], v=s["v"], w=s["w"], p_dyn=s.get("p_prev", z),
            T_g=s["T_g"], Y_fuel=s["Y_fuel"], Y_O2=s["Y_O2"], Y_H2O=s["Y_H2O"], Y_CO=z,
            alpha_s=s["alpha_s"], T_s=s["T_s"], m_hemi=z, m_cell=z, m_lign=z, m_char=z,
            front_t=np.array(self.front_t), front_x=np.array(self.front_x),
            diag_t=np.array(self.diag_t), diag_Tg_max=np.array(self.diag_Tg_max),
            diag_Ts_max=np.array(self.diag_Ts_max), diag_Sp_max=np.array(self.diag_Sp_max),
            diag_Qc_max=np.array(self.diag_Qc_max),
            diag_omega_max=np.array(self.diag_omega_max),
            diag_Y_max=np.array(self.diag_Y_max), diag_n_ign=np.array(self.diag_n_ign))
        return path


def compute_steady_ros(front_t, front_x, t_end, source_x, domain_m):
    """``_compute_steady_ros`` (``spread_3d.py:3792-3824``)."""
    if len(front_t) < 2:
        return 0.0
    if front_x[-1] - source_x < 0.1:
        return 0.0
    if t_end - front_t[-1] > 30.0 and not front_x[-1] > domain_m * 0.7:
        return 0.0
    t0 = float(front_t[0])
    if t_end > t0:
        return float((front_x[-1] - front_x[0]) / (t_end - t0))
    return 0.0


def ros_from_snapshots(times, x_lead):
    """ROS_Ts [m/s] as the snapshot worker computes it
    (``_cheney_phase16_worker.py:208-231``): over the snapshots in which some
    column holds T_s >= 600 K (``x_lead`` finite there), at least three, a
    least-squares line through (t, x_lead) of those with t >= 1 s, at least
    three; NaN otherwise.  The worker reports the slope in m/min."""
    t = np.asarray(times, dtype=np.float64)
    x = np.asarray(x_lead, dtype=np.float64)
    burned = np.isfinite(x)
    t, x = t[burned], x[burned]
    if t.size < 3:
        return float("nan")
    late = t >= 1.0
    if int(late.sum()) < 3:
        return float("nan")
    return float(np.polyfit(t[late], x[late], 1)[0])


class _Diag:
    """Per-step diagnostics of ``spread_3d.py:3503-3512`` and the front and
    heat-release columns, on the device (``fs_field_max_multi`` and
    ``fs_column_diag``); one host read per call."""

    def __init__(self, solver: Tier3Solver):
        s = solver
        self.s = s
        g = s.grid
        self.scratch = torch.empty(int(s.lib.fs_column_diag_scratch_bytes(s.gp)),
                                   dtype=torch.uint8, device=s.dev)
        self.hrr = torch.empty(g.Nx, dtype=torch.float64, device=s.dev)
        self.scale = HOC_J * g.dy / g.Ly
        # cell-centre x as the snapshot files hold it (float32, spread_3d.py:3662)
        self.x_mid32 = np.asarray(g.x_mid, dtype=np.float32)
        self.last = None

    def columns(self) -> FsColumnDiag:
        """Ignited cells, max S_pyro, HRRPUA(x) (kept in ``self.hrr``), its
        maximum and the leading column with T_s >= 600 K, from the current state."""
        s = self.s
        out = FsColumnDiag()
        check(s.lib.fs_column_diag(s.gp, ptr(s.f["T_s"]), ptr(s.w["omega"]),
                                   ptr(s.bed_out["S_pyro"]), ptr(s.bed_out["S_drying"]),
                                   float(s.p["T_ign"]), T_IGN_ROS, self.scale, ptr(self.hrr),
                                   ptr(self.scratch), _C.byref(out), s._s()), "fs_column_diag")
        self.last = out
        return out

    def record(self, res: "Spread3DResultGPU"):
        s = self.s
        m = s._maxes([s.f["T_g"], s.f["T_s"], s.w["Q_comb"], s.w["omega"], s.f["Y_fuel"]],
                     [1, 1, 1, 1, 1])
        c = self.columns()
        res.diag_t.append(s.t)
        res.diag_Tg_max.append(m[0])
        res.diag_Ts_max.append(m[1])
        res.diag_Sp_max.append(c.S_pyro_max)
        res.diag_Qc_max.append(m[2])
        res.diag_omega_max.append(m[3])
        res.diag_Y_max.append(m[4])
        res.diag_n_ign.append(int(c.n_ign))
        res.diag_proj_div_max.append(s.diag.proj_div_max)
        res.diag_proj_n_iter.append(int(s.diag.proj_iters))
        return c

    def lead_x_Ts(self):
        """x (float32 cell centre) of the last column with T_s >= 600 K, or NaN."""
        c = self.last if self.last is not None else self.columns()
        return float(self.x_mid32[c.lead_i]) if c.lead_i >= 0 else float("nan")

    def hrrpua_x(self):
        """HRRPUA(x) = (1/Ly) sum_{j,k} omega * HOC_J * dz_k * dy  [W/m^2]."""
        if self.last is None:
            self.columns()
        return self.hrr


def run_3d_spread_gpu(case: dict, *, n_steps: int | None = None, t_end: float | None = None,
                      device="cuda", projection_cg_rtol: float | None = None,
                      snapshot_dir=None, snapshot_interval_s: float = 1.0,
                      form: str = "plain") -> Spread3DResultGPU:
    """Device-resident ``run_3d_spread`` for a case; stops at ``n_steps``
    outer steps, at ``t_end`` simulated seconds or at the reference's own
    exit tests, whichever comes first.

    Snapshot instants follow the reference (``spread_3d.py:3537``): after the
    first step and then whenever ``snapshot_interval_s`` of simulated time has
    passed since the last one.  With ``snapshot_dir`` a ``snap_NNNN.npz`` file
    with the reference's key set is written at each instant; either way the
    leading column with T_s >= 600 K is recorded there, and ``ros_Ts`` is the
    snapshot worker's fit over those instants (``ros_from_snapshots``)."""
    if n_steps is None and t_end is None:
        raise ValueError("run_3d_spread_gpu needs n_steps or t_end")
    s = Tier3Solver(case, device=device, projection_cg_rtol=projection_cg_rtol, form=form)
    # long-lived objects out of the collector's way: full collections during the
    # run then scan only objects made by the run itself
    gc.collect()
    gc.freeze()
    try:
        g = s.grid
        res = Spread3DResultGPU(ros_m_s=0.0, n_cells_ignited=0, front_t=s.front_t,
                                front_x=s.front_x, grid=g, state_final={})
        dg = _Diag(s)
        snap_t, snap_x = [], []
        last_snap_t, snap_idx = -1.0e30, 0
        if snapshot_dir is not None:
            snapshot_dir = Path(snapshot_dir)
            snapshot_dir.mkdir(parents=True, exist_ok=True)
        hrr_peak = 0.0
        k = 0
        while True:
            if n_steps is not None and k >= n_steps:
                break
            if t_end is not None and s.t >= t_end:
                break
            if not s.step():
                break
            k += 1
            c = dg.record(res)
            hrr_peak = max(hrr_peak, c.hrr_max)
            if s.t - last_snap_t >= snapshot_interval_s:
                last_snap_t = s.t
                snap_t.append(s.t)
                snap_x.append(dg.lead_x_Ts())
                if snapshot_dir is not None:
                    write_snapshot(s, snapshot_dir / f"snap_{snap_idx:04d}.npz",
                                   float(case.get("wind_speed_m_s", 0.0)))
                snap_idx += 1
        st = s.state()
        res.state_final = st
        res.k_turb_final = st["k_turb"]
        res.eps_turb_final = st["eps_turb"]
        res.nu_t_final = st["nu_t"]
        res.n_cells_ignited = int(np.sum(st["T_s"] >= s.p["T_ign"]))
        res.ros_m_s = compute_steady_ros(s.front_t, s.front_x, s.t,
                                         source_x=s.p["i_src_end"] * g.dx, domain_m=g.Lx)
        res.ros_Ts = ros_from_snapshots(snap_t, snap_x)
        res.snap_t, res.snap_lead_x = snap_t, snap_x
        res.hrrpua_peak = hrr_peak
        return res
    finally:
        s.close()


class HostStepper:
    """Outer steps on state owned by the caller in (pinned) host memory."""

    FIELDS = Tier3Solver.FIELDS
    WORK = ("omega", "q_rad", "q_rad_gas")
    PARTS = ("x", "y", "z", "alive", "m_solid", "m_water", "m_char", "T_s", "m_water_0",
             "sav", "m_char_max")

    # Fields the step no longer changes from a phase on: their download starts
    # there, on a copy stream, while the rest of the step runs.  At the DOM
    # phase: velocities (after the projection and sponge), k-epsilon (after its
    # update), particles (after the bed phase).  At the first gas-energy update:
    # the radiative sources (after the ignition pulse) and the soil (after its
    # step).
    EARLY_AT = {"dom": ("u", "v", "w", "k_turb", "eps_turb", "nu_t")
                       + tuple("p_" + k for k in PARTS
                               if "p_" + k not in ("p_x", "p_y", "p_z", "p_m_water_0", "p_sav")),
                "gas_update": ("q_rad", "q_rad_gas", "T_soil")}
    EARLY = tuple(k for ks in EARLY_AT.values() for k in ks)
    # Fields the step first reads at the outflow sponge or later (spread_3d.py
    # order: dt, EoS, bed and the DOM's inputs, momentum and the projection come
    # first): their upload runs on the copy stream while those phases compute.
    LATE = ("Y_fuel", "k_turb", "eps_turb", "phi", "q_rad_gas")
    # Fields no step writes (the solid fraction; the particles' positions,
    # initial water mass and surface-to-volume ratio: particles do not move):
    # the device holds what was uploaded, so the host copy needs no download.
    STATIC = ("alpha_s", "p_x", "p_y", "p_z", "p_m_water_0", "p_sav")

    def __init__(self, case: dict, device="cuda", projection_cg_rtol: float | None = None,
                 form: str = "plain"):
        self.solver = Tier3Solver(case, device=device, projection_cg_rtol=projection_cg_rtol,
                                  form=form)
        s = self.solver
        self.host = {}
        for k in self.FIELDS:
            self.host[k] = s.f[k].cpu().pin_memory()
        for k in self.WORK:
            self.host[k] = s.w[k].cpu().pin_memory()
        self.host["T_soil"] = s.T_soil.cpu().pin_memory()
        for k in self.PARTS:
            self.host["p_" + k] = s.part[k].cpu().pin_memory()
        # device copies taken at the DOM phase (the solver swaps field buffers
        # afterwards, so the copy stream reads these, not the live fields)
        self.stage = {k: torch.empty_like(self._dev(k)) for k in self.EARLY}
        self.copy_stream = torch.cuda.Stream(device=s.dev)
        self._sent = set()
        self._late_ev = None
        # bytes moved each way since creation
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        s.phase_hook = self._on_phase

    def _on_phase(self, label):
        if label == "sponge" and self._late_ev is not None:
            torch.cuda.current_stream(self.solver.dev).wait_event(self._late_ev)
            self._late_ev = None
            return
        keys = self.EARLY_AT.get(label)
        if keys is None or label in self._sent:
            return
        cur = torch.cuda.current_stream(self.solver.dev)
        for k in keys:
            self.stage[k].copy_(self._dev(k), non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(cur)
        self.copy_stream.wait_event(ev)
        with torch.cuda.stream(self.copy_stream):
            for k in keys:
                self.host[k].copy_(self.stage[k], non_blocking=True)
                self.d2h_bytes += self._nbytes(k)
        self._sent.add(label)

    def _dev(self, k):
        s = self.solver
        if k in self.FIELDS:
            return s.f[k]
        if k in self.WORK:
            return s.w[k]
        if k == "T_soil":
            return s.T_soil
        return s.part[k[2:]]

    def _nbytes(self, k):
        t = self.host[k]
        return t.numel() * t.element_size()

    def bytes_per_transfer(self):
        return sum(t.numel() * t.element_size() for t in self.host.values())

    def step(self):
        """Upload the host state, advance one outer step, write back what the
        step changed (fields no step writes, and phi on steps without a
        level-set reinitialisation, already hold the right values)."""
        self.h2d_bytes += self.bytes_per_transfer()
        for k, h in self.host.items():
            if k not in self.LATE:
                self._dev(k).copy_(h, non_blocking=True)
        with torch.cuda.stream(self.copy_stream):
            for k in self.LATE:
                self._dev(k).copy_(self.host[k], non_blocking=True)
            self._late_ev = torch.cuda.Event()
            self._late_ev.record(self.copy_stream)
        self._sent = set()
        alive = self.solver.step()
        if self._late_ev is not None:  # the step ended before the sponge
            torch.cuda.current_stream(self.solver.dev).wait_event(self._late_ev)
            self._late_ev = None
        sent = {k for lab in self._sent for k in self.EARLY_AT[lab]}
        sent.update(self.STATIC)
        # the level set changes phi only on its reinitialisation steps
        if self.solver.lset_step % 10 != 0:
            sent.add("phi")
        for k, h in self.host.items():
            if k not in sent:
                h.copy_(self._dev(k), non_blocking=True)
                self.d2h_bytes += self._nbytes(k)
        torch.cuda.current_stream().synchronize()
        self.copy_stream.synchronize()
        return alive

    def close(self):
        self.solver.close()


def run_3d_spread_gpu_e2e(case: dict, steps: int, warmup: int = 1,
                          projection_cg_rtol: float | None = None, form: str = "plain"):
    """Time ``steps`` host-buffer outer steps (uploads and downloads inside
    the timed region), after ``warmup`` untimed ones."""
    hs = HostStepper(case, projection_cg_rtol=projection_cg_rtol, form=form)
    gc.collect()
    gc.freeze()
    try:
        for _ in range(warmup):
            hs.step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        h0, d0 = hs.h2d_bytes, hs.d2h_bytes
        e0.record()
        for _ in range(steps):
            hs.step()
        e1.record()
        torch.cuda.synchronize()
        return {"cells": hs.solver.n, "seconds": e0.elapsed_time(e1) * 1e-3,
                "h2d_bytes": hs.h2d_bytes - h0, "d2h_bytes": hs.d2h_bytes - d0}
    finally:
        hs.close()


# ------------------------------------------------------------------ snapshots
OMEGA_MIN_FLAME = 1.0e-3   # flame_front_3d.py:751-753 active-flame thresholds
T_PLUME_MIN = 1000.0
Y_F_MIN_PLUME = 1.0e-3


def phi_flame_from_state(omega, T_g, Y_fuel, dx, dy, dz_arr):
    """Signed distance to the active-flame region, negative inside
    (``compute_phi_flame_from_state``, flame_front_3d.py:756-800): Euclidean
    distance transforms of the active mask with sampling (mean dz, dy, dx)."""
    from scipy import ndimage
    active = (omega > OMEGA_MIN_FLAME) | ((T_g > T_PLUME_MIN) & (Y_fuel > Y_F_MIN_PLUME))
    sampling = (float(np.mean(dz_arr)), dy, dx)
    if active.any() and (~active).any():
        d_out = ndimage.distance_transform_edt(~active, sampling=sampling)
        d_in = ndimage.distance_transform_edt(active, sampling=sampling)
        return np.where(active, -d_in, d_out)
    return np.full(active.shape, -1.0e6 if active.all() else 1.0e6)


def bed_particles_per_cell(parts, grid):
    """Per-cell particle count, masses and mass-weighted T_s of the live
    particles (the snapshot aggregation of spread_3d.py:3567-3606): x and y
    cells by truncation, z by the first face above the particle."""
    shape = grid.shape
    alive = np.asarray(parts["alive"]) != 0
    xi = np.trunc(np.asarray(parts["x"]) / grid.dx).astype(np.int64)
    yj = np.trunc(np.asarray(parts["y"]) / grid.dy).astype(np.int64)
    zz = np.asarray(parts["z"])
    zk = np.searchsorted(np.asarray(grid.z_face)[1:], zz, side="right")
    ok = alive & (xi >= 0) & (xi < grid.Nx) & (yj >= 0) & (yj < grid.Ny) & (zk < grid.Nz)
    idx = (zk[ok], yj[ok], xi[ok])
    out = {}
    cnt = np.zeros(shape); np.add.at(cnt, idx, 1.0)
    ms, mw, mc = (np.asarray(parts[k])[ok] for k in ("m_solid", "m_water", "m_char"))
    mt = ms + mw + mc
    for name, v in (("bp_m_solid", ms), ("bp_m_water", mw), ("bp_m_char", mc)):
        a = np.zeros(shape); np.add.at(a, idx, v); out[name] = a.astype(np.float32)
    tw = np.zeros(shape); np.add.at(tw, idx, np.asarray(parts["T_s"])[ok] * mt)
    mm = np.zeros(shape); np.add.at(mm, idx, mt)
    out["bp_count"] = cnt.astype(np.float32)
    out["bp_T_s_avg"] = np.where(mm > 0.0, tw / np.maximum(mm, 1e-30), 0.0).astype(np.float32)
    return out


def write_snapshot(solver: Tier3Solver, path, wind_speed_m_s: float):
    """One animation snapshot with the reference's key set
    (spread_3d.py:3613-3669).  Fields this production path does not carry
    (mixing time, level-set drive fields, tendril inventory) are zeros, as
    the reference writes for passive level-set runs without tendrils."""
    s = solver
    g = s.grid
    st = s.state()
    f32 = lambda a: np.asarray(a, dtype=np.float32)  # noqa: E731
    zeros3 = np.zeros(g.shape, np.float32)
    zeros2 = np.zeros((g.Ny, g.Nx), np.float32)
    parts = {k[2:]: v for k, v in st.items() if k.startswith("p_") and k != "p_prev"}
    phi_flame = phi_flame_from_state(st["omega"], st["T_g"], st["Y_fuel"], g.dx, g.dy, g.dz_arr)
    arrays = dict(
        t=np.float64(s.t), step=np.int64(s.step_count),
        T_g=f32(st["T_g"]), T_s=f32(st["T_s"]), Y_fuel=f32(st["Y_fuel"]), Y_O2=f32(st["Y_O2"]),
        Y_H2O=f32(st["Y_H2O"]), u=f32(st["u"]), v=f32(st["v"]), w=f32(st["w"]),
        rho=f32(st["rho"]), omega=f32(st["omega"]),
        S_pyro=f32(np.asarray(st["S_pyro_b"]) + np.asarray(st["S_dry_b"])),
        k_turb=f32(st["k_turb"]), eps_turb=f32(st["eps_turb"]), nu_t=f32(st["nu_t"]),
        tau_mix=zeros3, phi_bed=f32(st["phi"]) if g.n_z_bed > 0 else zeros3,
        phi_flame=f32(phi_flame), front_x=np.float64(s.front_x[-1] if s.front_x else 0.0),
        q_dom_fwd_3d=zeros3, q_frankman_3d=zeros3, q_in_at_front_2d=zeros2, v_n_2d=zeros2,
        ft_sink_M=zeros3, ft_sink_E=zeros3, ft_dep_M=zeros3, ft_dep_E=zeros3,
        ft_sink_t_rem=zeros3, ft_dep_t_rem=zeros3,
        x_mid=f32(g.x_mid), z_mid=f32(g.z_mid), dx=np.float64(g.dx), dy=np.float64(g.dy),
        dz_arr=f32(g.dz_arr), wind_U=np.float64(wind_speed_m_s),
        closure=np.array(["edc"], dtype=object),
    )
    arrays.update(bed_particles_per_cell(parts, g))
    np.savez_compressed(path, **arrays)
    return path


# ---------------------------------------------------------------- checkpoints
_CKPT_WORK = ("omega", "q_rad", "q_rad_gas", "M_local")
_CKPT_PARTS = ("x", "y", "z", "alive", "m_solid", "m_water", "m_char", "T_s", "m_water_0",
               "sav", "m_char_max")


def save_checkpoint(solver: Tier3Solver, path) -> Path:
    """Write everything a later step reads: the state fields, the fields
    carried between steps (omega, q_rad, q_rad_gas, M_local), soil, particles,
    the projection's warm-start pressure, the DOM inflow rows and the clock.
    The reference has no checkpoint; a run restored from this file continues
    bit-identically."""
    s = solver
    torch.cuda.synchronize()
    path = Path(path)
    if not str(path).endswith(".npz"):
        path = path.with_suffix(".npz")
    path.parent.mkdir(parents=True, exist_ok=True)
    arrays = {"f_" + k: s.f[k].cpu().numpy() for k in Tier3Solver.FIELDS}
    arrays.update({"w_" + k: s.w[k].cpu().numpy() for k in _CKPT_WORK})
    arrays.update({"p_" + k: s.part[k].cpu().numpy() for k in _CKPT_PARTS})
    arrays["T_soil"] = s.T_soil.cpu().numpy()
    arrays["pressure"] = s.pressure_view().cpu().numpy()
    nw = int(s.lib.fs_dom_wrap_size(s.dom))
    wrap = torch.empty(nw, dtype=torch.float64, device=s.dev)
    check(s.lib.fs_dom_get_wrap(s.dom, ptr(wrap), s._s()), "fs_dom_get_wrap")
    arrays["dom_wrap"] = wrap.cpu().numpy()
    meta = {"case": s.case, "t": s.t, "dt": s.dt, "step_count": s.step_count,
            "lset_step": s.lset_step, "extinct_count": s.extinct_count,
            "front_t": list(s.front_t), "front_x": list(s.front_x),
            "rtol": s.rtol, "proj_maxiter": s.proj_maxiter, "form": s.form}
    np.savez(path, _meta_json=np.array(json.dumps(meta)), **arrays)
    return path


def load_checkpoint(path, device="cuda") -> Tier3Solver:
    """A solver restored from :func:`save_checkpoint`."""
    z = np.load(Path(path), allow_pickle=False)
    meta = json.loads(str(z["_meta_json"]))
    s = Tier3Solver(meta["case"], device=device, projection_cg_rtol=meta["rtol"],
                    proj_maxiter=meta["proj_maxiter"], form=meta.get("form", "plain"))
    for k in Tier3Solver.FIELDS:
        s.f[k].copy_(torch.as_tensor(z["f_" + k]))
    for k in _CKPT_WORK:
        s.w[k].copy_(torch.as_tensor(z["w_" + k]))
    for k in _CKPT_PARTS:
        s.part[k].copy_(torch.as_tensor(z["p_" + k]))
    s.T_soil.copy_(torch.as_tensor(z["T_soil"]))
    s.pressure_view().copy_(torch.as_tensor(z["pressure"]))
    wrap = torch.as_tensor(z["dom_wrap"]).to(s.dev)
    if wrap.numel() != int(s.lib.fs_dom_wrap_size(s.dom)):
        raise ValueError("checkpoint DOM state does not match the case's grid and quadrature")
    check(s.lib.fs_dom_set_wrap(s.dom, ptr(wrap), s._s()), "fs_dom_set_wrap")
    s.t, s.dt = float(meta["t"]), float(meta["dt"])
    s.step_count, s.lset_step = int(meta["step_count"]), int(meta["lset_step"])
    s.extinct_count = int(meta["extinct_count"])
    s.front_t, s.front_x = list(meta["front_t"]), list(meta["front_x"])
    torch.cuda.synchronize()
    return s
