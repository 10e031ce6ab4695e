"""Host-side set-up of a Tier-3 case: grid, initial state, bed particles, inlet.

This is the one-off initialisation that ``run_3d_spread`` performs before its
time loop (``spread_3d.py:960-1748``), restated in numpy.  Its output is
uploaded to the device once; nothing here runs per step.

Only the production mesh path is provided: the legacy uniform-bed z axis
(``spread_3d.py:303-424`` with ``dz_first``/``bl`` refinement off).  The
segmented ``wall_bl_N > 0`` mesh (``mesh.py``) raises ``NotImplementedError``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Physical constants of the driver (spread_3d.py:67-87).
R_UNIV = 8.314
M_AIR = 0.029
R_AIR = R_UNIV / M_AIR
P0 = 101_325.0
G = 9.81
RHO_PARTICLE = 500.0
CP_SOLID_EULER = 1300.0
T_AMB_DEFAULT = 300.0
Z0_INLET = 0.01            # outdoor_wind.py:32
WAF = {"open": 0.9, "shrub": 0.6}   # boundary.py:40-44


@dataclass
class Grid3D:
    """Cartesian grid with per-cell vertical spacing (fields as in spread_3d.py:158-188)."""
    Nx: int
    Ny: int
    Nz: int
    dx: float
    dy: float
    dz: float
    Lx: float
    Ly: float
    Lz: float
    n_z_bed: int
    x_mid: np.ndarray
    y_mid: np.ndarray
    z_mid: np.ndarray
    dz_arr: np.ndarray
    inv_dz_arr: np.ndarray
    z_face: np.ndarray
    d_face_above: np.ndarray
    d_face_below: np.ndarray

    @property
    def shape(self):
        return (self.Nz, self.Ny, self.Nx)

    @property
    def n_cells(self):
        return self.Nz * self.Ny * self.Nx


def build_grid(Lx, Ly, Lz, dx, h_bed, n_z_bed, dy=None, dz_expansion=1.0,
               wall_bl_N=0) -> Grid3D:
    """Legacy uniform-bed grid (``Grid3D.build`` with the BL options off)."""
    if wall_bl_N and int(wall_bl_N) > 0:
        raise NotImplementedError("segmented wall-BL mesh (wall_bl_N > 0) is not provided")
    if Lz < h_bed:
        raise ValueError(f"Lz={Lz} must exceed h_bed={h_bed}")
    if dz_expansion < 1.0:
        raise ValueError(f"dz_expansion={dz_expansion} must be >= 1.0")
    Nx = max(2, int(round(Lx / dx)))
    dy_t = dy if dy is not None else dx
    Ny = max(1, int(round(Ly / dy_t)))
    dy = Ly / Ny
    dz_bed = h_bed / max(n_z_bed, 1)
    bed_dz = np.full(n_z_bed, dz_bed, dtype=np.float64)
    target = Lz - h_bed
    if dz_expansion <= 1.0 + 1e-12:
        n_buf = max(1, int(round(target / dz_bed)))
        buf_dz = np.full(n_buf, dz_bed, dtype=np.float64)
    else:
        ratio = target * (dz_expansion - 1.0) / dz_bed + 1.0
        n_buf = max(1, int(np.ceil(np.log(ratio) / np.log(dz_expansion))))
        buf_dz = dz_bed * np.power(dz_expansion, np.arange(n_buf, dtype=np.float64))
    dz_arr = np.concatenate([bed_dz, buf_dz])
    Nz = len(dz_arr)
    z_face = np.concatenate([[0.0], np.cumsum(dz_arr)])
    z_mid = z_face[:-1] + 0.5 * dz_arr
    d_above = np.empty(Nz)
    d_below = np.empty(Nz)
    for k in range(Nz):
        d_above[k] = 0.5 * (dz_arr[k] + dz_arr[k + 1]) if k + 1 < Nz else 0.5 * dz_arr[k]
        d_below[k] = 0.5 * (dz_arr[k] + dz_arr[k - 1]) if k - 1 >= 0 else 0.5 * dz_arr[k]
    x_mid = (np.arange(Nx) + 0.5) * (Lx / Nx)
    y_mid = (np.arange(Ny) + 0.5) * dy
    return Grid3D(Nx=Nx, Ny=Ny, Nz=Nz, dx=Lx / Nx, dy=dy, dz=float(dz_bed),
                  Lx=Lx, Ly=Ly, Lz=float(z_face[-1]), n_z_bed=n_z_bed,
                  x_mid=x_mid, y_mid=y_mid, z_mid=z_mid, dz_arr=dz_arr,
                  inv_dz_arr=1.0 / dz_arr, z_face=z_face,
                  d_face_above=d_above, d_face_below=d_below)


def wind_profile_log_law(z, U_ref, z_ref=10.0, z_0=0.01):
    """Log-law inflow u(z) pinned at u(0)=0 and u(z_ref)=U_ref (boundary.py:68-111)."""
    if z <= 0.0 or U_ref <= 0.0 or z_ref <= 0.0:
        return 0.0
    a = U_ref / math.log((z_ref + z_0) / z_0)
    return max(0.0, a * math.log((z + z_0) / z_0))


def midflame_wind_speed(U10, terrain="open"):
    return U10 * WAF.get(terrain.lower(), 0.9)


def init_bed_particles(alpha_s, rho_b_dry, moisture_frac, T_amb, dx, dy, dz_arr,
                       n_z_bed, n_per_cell, sav, i_lo, i_hi):
    """Cell-major coprime-mod particle packing (lagrangian_bed_3d.py:221-329).

    Returns a dict of particle arrays with one slot per particle, in the
    reference's slot order (k, j, i, p).
    """
    Nz, Ny, Nx = alpha_s.shape
    cells = [(k, j, i) for k in range(min(n_z_bed, Nz)) for j in range(Ny)
             for i in range(i_lo, min(i_hi, Nx)) if alpha_s[k, j, i] > 0.0]
    n = len(cells) * n_per_cell
    x = np.zeros(n); y = np.zeros(n); z = np.zeros(n)
    m_solid = np.zeros(n); m_water = np.zeros(n)
    p = np.arange(n_per_cell)
    fx = ((p * 13) % n_per_cell + 0.5) / n_per_cell
    fy = ((p * 7) % n_per_cell + 0.5) / n_per_cell
    fz = (p + 0.5) / n_per_cell
    s = 0
    for (k, j, i) in cells:
        V = dx * dy * dz_arr[k]
        zf = float(np.sum(dz_arr[:k]))
        ms = rho_b_dry * V / n_per_cell
        sl = slice(s, s + n_per_cell)
        x[sl] = (i + fx) * dx
        y[sl] = (j + fy) * dy
        z[sl] = zf + fz * dz_arr[k]
        m_solid[sl] = ms
        m_water[sl] = moisture_frac * ms
        s += n_per_cell
    return dict(x=x, y=y, z=z, alive=np.ones(n, dtype=np.int8),
                m_solid=m_solid, m_water=m_water, m_char=np.zeros(n),
                T_s=np.full(n, T_amb), m_solid_0=m_solid.copy(),
                m_water_0=m_water.copy(), sav=np.full(n, float(sav)),
                m_char_max=np.zeros(n))


def jitter_particle_positions(x, y, z, dx, dy, z_face, seed):
    """Seeded positions uniformly inside each particle's own cell.

    The cell of each slot is taken from its lattice position; the new position
    is drawn from U[0.02, 0.98) of the cell in every axis from a PCG64 stream
    (one (N, 3) draw), so no particle lands on a cell face.
    """
    x = np.asarray(x); y = np.asarray(y); z = np.asarray(z)
    n = x.shape[0]
    rng = np.random.Generator(np.random.PCG64(int(seed)))
    f = 0.02 + 0.96 * rng.random((n, 3))
    i = np.floor(x / dx)
    j = np.floor(y / dy)
    k = np.searchsorted(z_face, z, side="right") - 1
    k = np.clip(k, 0, len(z_face) - 2)
    nx_ = (i + f[:, 0]) * dx
    ny_ = (j + f[:, 1]) * dy
    nz_ = z_face[k] + f[:, 2] * (z_face[k + 1] - z_face[k])
    return nx_, ny_, nz_


def _pick(case, key, default):
    for k in (key, key.lower()):
        if k in case and case[k] is not None:
            return case[k]
    return default


@dataclass
class CaseSetup:
    """Everything the time loop needs, resolved from a case dict."""
    grid: Grid3D
    params: dict
    fields: dict = field(default_factory=dict)     # (Nz,Ny,Nx) float64 initial fields
    particles: dict = field(default_factory=dict)  # particle SoA
    u_inlet: np.ndarray = None                    # (Nz, Ny)
    sigma_sponge: np.ndarray = None               # (Nx,)
    soil: dict = field(default_factory=dict)


# Grid3D.build options that select the boundary-layer or segmented mesh
# kernels (spread_3d.py:190-302) instead of the legacy uniform bed.
_MESH_BRANCH_KEYS = ("dz_first", "dz_first_above", "bed_top_inner_bl_N", "bed_top_outer_bl_N")


def build_grid_from_case(case):
    for key in _MESH_BRANCH_KEYS:
        v = _pick(case, key, None)
        if v is not None and not (isinstance(v, bool) and not v) and float(v) > 0.0:
            raise NotImplementedError(
                f"{key}={v!r} selects the boundary-layer mesh, which the GPU Tier-3 step does "
                "not provide (uniform bed layers only)")
    Lx = float(_pick(case, "Lx", 10.0)); Ly = float(_pick(case, "Ly", 2.0))
    Lz = float(_pick(case, "Lz", 1.5)); dx = float(_pick(case, "dx", 0.05))
    dy = float(_pick(case, "dy", dx))
    n_z_bed = int(_pick(case, "n_z_bed", 4))
    h_bed = float(_pick(case, "fuel_depth_m", 0.30))
    return build_grid(Lx, Ly, Lz, dx, h_bed, n_z_bed, dy=dy,
                      dz_expansion=float(_pick(case, "dz_expansion", 1.0)),
                      wall_bl_N=int(_pick(case, "wall_bl_N", 0)))


# The physics branches this build provides, with the reference driver's
# defaults (spread_3d.py:597-893) for keys a deck leaves out.  Any other
# choice raises NotImplementedError, as the reference's JS port does for the
# branches it lacks, instead of silently running the provided branch.
SUPPORTED = (
    ("turbulence_model", "laminar", ("k_epsilon",)),
    ("combustion_closure", "edc", ("edc",)),
    ("radiation_solver", "dom", ("dom",)),
    ("wall_function", False, (False, None)),
    ("level_set_passive", False, (True,)),
    ("ignition_T_pin_enable", False, (False,)),
    ("empirical_ros_enable", False, (False,)),
    ("finney_tendril_enable", False, (False,)),
    ("moisture_jump_enable", False, (False,)),
)


def check_supported(case: dict) -> None:
    """Raise NotImplementedError for a physics branch this build does not provide."""
    for key, default, ok in SUPPORTED:
        v = _pick(case, key, default)
        if isinstance(v, str):
            v = v.strip().lower()
        elif v is not None and not isinstance(v, bool):
            v = bool(v)
        if v not in ok:
            raise NotImplementedError(
                f"{key}={v!r} is not provided by the GPU Tier-3 step (provided: "
                f"{', '.join(repr(o) for o in ok if o is not None)})")


def build_setup(case: dict) -> CaseSetup:
    """Resolve a case (deck keys + ``wind_speed_m_s``) into initial state and constants."""
    g = build_grid_from_case(case)
    T_amb = T_AMB_DEFAULT
    h_bed = float(_pick(case, "fuel_depth_m", 0.30))
    rho_b = float(_pick(case, "bulk_density_kg_m3", 3.0))
    sav = float(_pick(case, "sav_ratio_1_m", 6562.0))
    M_f = float(_pick(case, "initial_moisture_frac", 0.08) or 0.0)
    U10 = float(case.get("wind_speed_m_s", 0.0))
    Lx = g.Lx
    bed_x_start = float(_pick(case, "bed_x_start", 0.0))
    bed_x_end = float(_pick(case, "bed_x_end", Lx))
    i_bed_start = int(np.searchsorted(g.x_mid, bed_x_start, side="left"))
    i_bed_end = int(np.searchsorted(g.x_mid, bed_x_end, side="right"))
    if i_bed_start >= i_bed_end:
        raise ValueError("bed_x_start >= bed_x_end after grid snapping")
    shape = g.shape
    rho_amb = P0 / (R_AIR * T_amb)
    f = {
        "rho": np.full(shape, rho_amb), "u": np.zeros(shape), "v": np.zeros(shape),
        "w": np.zeros(shape), "T_g": np.full(shape, T_amb), "Y_fuel": np.zeros(shape),
        "Y_O2": np.full(shape, 0.232), "Y_H2O": np.zeros(shape),
        "alpha_s": np.zeros(shape), "T_s": np.full(shape, T_amb),
    }
    alpha_s_avg = rho_b / RHO_PARTICLE
    f["alpha_s"][:g.n_z_bed, :, i_bed_start:i_bed_end] = alpha_s_avg
    if str(_pick(case, "alpha_s_profile_type", "uniform")) != "uniform":
        raise NotImplementedError("only the uniform alpha_s bed profile is provided")

    if not bool(_pick(case, "lagrangian_bed_enable", False)):
        raise NotImplementedError("the Eulerian bed branch is not provided (Lagrangian bed only)")
    check_supported(case)
    n_pc = int(_pick(case, "lagrangian_bed_N_per_cell", 50))
    parts = init_bed_particles(f["alpha_s"], rho_b, M_f, T_amb, g.dx, g.dy, g.dz_arr,
                               g.n_z_bed, n_pc, sav, i_bed_start, i_bed_end)
    seed = case.get("jitter_seed", None)
    if seed is not None and parts["x"].size:
        parts["x"], parts["y"], parts["z"] = jitter_particle_positions(
            parts["x"], parts["y"], parts["z"], g.dx, g.dy,
            np.concatenate([[0.0], np.cumsum(g.dz_arr)]), seed)

    # ignition source strip (spread_3d.py:1486-1495)
    ign_w = float(_pick(case, "ignition_width_mult", 1.0))
    n_src = max(1, int(round(0.5 * ign_w / g.dx)))
    i_src_start = i_bed_start
    i_src_end = min(i_bed_end, i_src_start + n_src)
    n_src = i_src_end - i_src_start
    if bool(_pick(case, "solid_phase_ignition_enable", False)):
        Ts_seed = float(_pick(case, "solid_phase_ignition_T_s_K", 800.0))
        x_lo = g.x_mid[i_src_start] - 0.5 * g.dx
        x_hi = g.x_mid[i_src_end - 1] + 0.5 * g.dx
        sel = (parts["alive"] != 0) & (parts["x"] >= x_lo) & (parts["x"] < x_hi)
        parts["T_s"][sel] = Ts_seed

    terrain = "open"
    U_mf = midflame_wind_speed(U10, terrain)
    u_inlet = np.zeros((g.Nz, g.Ny))
    for k in range(g.Nz):
        u_inlet[k, :] = wind_profile_log_law(g.z_mid[k], U10, 10.0, Z0_INLET)
    f["u"][:] = u_inlet[:, :, None]

    n_sp = max(3, min(int(round(0.5 / g.dx)), g.Nx // 4))
    sig = np.zeros(g.Nx)
    for i in range(g.Nx - n_sp, g.Nx):
        fr = (i - (g.Nx - n_sp)) / n_sp
        sig[i] = 5.0 * fr * fr

    # soil grid (soil_3d.py:73-103), 6 cells from 1 mm x 1.5
    n_soil = 6
    sdz = np.array([0.001 * 1.5 ** k for k in range(n_soil)])
    sda = np.empty(n_soil); sdb = np.empty(n_soil)
    sda[0] = sdz[0] / 2.0
    for k in range(1, n_soil):
        sda[k] = 0.5 * (sdz[k - 1] + sdz[k])
    for k in range(n_soil - 1):
        sdb[k] = 0.5 * (sdz[k] + sdz[k + 1])
    sdb[-1] = sdz[-1] / 2.0

    # k-epsilon initial state (spread_3d.py:1568-1573)
    C_MU = 0.09
    k_init = max(1.5 * (0.10 * max(U_mf, 0.5)) ** 2, 1.0e-4)
    eps_init = C_MU * k_init * k_init / 0.01
    f["k_turb"] = np.full(shape, k_init)
    f["eps_turb"] = np.full(shape, eps_init)
    f["nu_t"] = np.full(shape, 0.01)

    # level set (flame_front_3d.py:304-330), L_burnout = 0.5 m
    L_burn = 0.5
    phi = np.full(shape, 100.0)
    if g.n_z_bed > 0 and i_src_end > i_src_start:
        x_front = g.x_mid[i_src_end - 1] + 0.5 * g.dx
        d = g.x_mid - x_front
        row = np.where(d > 0.0, d, np.maximum(d, -L_burn / 2.0))
        phi[:] = row[None, None, :]
        phi[:g.n_z_bed, :, i_src_start:i_src_end] = -L_burn / 2.0
    f["phi"] = phi

    cfl = float(_pick(case, "cfl_factor", 0.4))
    U_char = max(U_mf, math.sqrt(G * h_bed * 0.5), 0.1)
    dz_min = float(g.dz_arr.min())
    dt_adv = cfl * min(g.dx, g.dy, dz_min) / U_char
    nu_max = max(float(f["nu_t"].max()), 1.0e-3)
    dt_diff = 0.25 * dz_min * dz_min / nu_max
    dt0 = min(dt_adv, dt_diff, 0.05)

    params = dict(
        T_amb=T_amb, h_bed=h_bed, rho_b=rho_b, sav=sav, M_f=M_f, U10=U10, U_mf=U_mf,
        i_bed_start=i_bed_start, i_bed_end=i_bed_end, i_src_start=i_src_start,
        i_src_end=i_src_end, n_src=n_src, n_per_cell=n_pc, cfl=cfl, dt0=dt0,
        dz_min=dz_min, U_char=U_char,
        ignition_duration_s=float(_pick(case, "ignition_duration_s", 30.0)),
        ignition_q_mult=float(_pick(case, "ignition_q_mult", 1.0)),
        canopy_C_d=float(_pick(case, "canopy_C_d", 0.30)),
        canopy_beta_p=float(_pick(case, "canopy_beta_p", 1.0)),
        canopy_beta_d=float(_pick(case, "canopy_beta_d", 4.0)),
        h_conv=float(_pick(case, "lagrangian_bed_h_conv", 25.0)),
        rho_solid_true=380.0, cp_solid=1500.0, eps_solid=0.9, view_factor=1.0,
        view_factor_geometric=bool(_pick(case, "lagrangian_bed_view_factor_geometric", True)),
        drying_mode={"arrhenius": 0, "equilibrium": 1, "combined": 2}[
            str(_pick(case, "lagrangian_bed_drying_mode", "arrhenius"))],
        char_ox_flux_cap=float(_pick(case, "char_ox_flux_cap_W_m2", 1.0e5)),
        char_ox_ash_exp=float(_pick(case, "char_ox_ash_exp", 0.0)),
        kappa_bed_eff=float(sav * rho_b / 380.0),
        min_dt_s=float(_pick(case, "min_dt_s", 1.0e-4)),
        dom_subcycle_every=int(_pick(case, "dom_subcycle_every", 1)),
        n_quadrature=int(case.get("n_quadrature", 4)),
        chi_rad=0.34, T_ign=T_amb + 300.0,
        level_set_passive=bool(_pick(case, "level_set_passive", False)),
        proj_max_iter=int(_pick(case, "proj_max_iter", 50)),
        proj_div_tol=float(_pick(case, "proj_div_tol", 1.0e-3)),
        edc_extinction_enable=bool(_pick(case, "edc_extinction_enable", False)),
        x_front0=(float(g.x_mid[i_src_end - 1] + 0.5 * g.dx)
                  if g.n_z_bed > 0 and i_src_end > i_src_start else 0.0),
    )
    return CaseSetup(grid=g, params=params, fields=f, particles=parts,
                     u_inlet=u_inlet, sigma_sponge=sig,
                     soil=dict(dz=sdz, d_above=sda, d_below=sdb, n=n_soil,
                               T=np.full((n_soil, g.Ny, g.Nx), T_amb)))
