"""Named Tier-3 workloads (deck settings) used by the tests, the bench and the fixtures.

Each case is a flat dict of ``outdoor.*`` deck keys plus the run-time keyword
``wind_speed_m_s`` (the reference driver takes the 10 m wind as a keyword, not
from the deck: ``spread_3d.py:966`` overwrites the deck value with the kwarg).

The production physics switches are the ones the reference's validation decks
use (``data/validation_cases/Outdoor_Cheney_Nat4_U4__empROS_regression.txt``,
``scripts/integration_case.txt``): Lagrangian bed + k-epsilon + EDC + DOM +
``fft_pcg`` projection + periodic y + log-law inlet, passive level set and
solid-phase ignition.
"""
from __future__ import annotations

COMMON = dict(
    turbulence_model="k_epsilon",
    wall_function=False,
    combustion_closure="edc",
    radiation_solver="dom",
    projection_method="fft_pcg",
    lagrangian_bed_enable=True,
    lagrangian_bed_drying_mode="combined",
    lagrangian_bed_h_conv=250.0,
    lagrangian_bed_view_factor_geometric=True,
    level_set_passive=True,
    solid_phase_ignition_enable=True,
    ignition_T_pin_enable=False,
    ignition_duration_s=3.0,
    ignition_q_mult=1.0,
    wall_bl_N=0,
    min_dt_s=1.0e-4,
    canopy_C_d=0.30,
    max_wall_time_s=1.0e9,
)

# 64 x 24 x 20 cells at dx = 0.1 m (the reference's CPU-runnable case).
CFG1 = dict(
    COMMON,
    Lx=6.4, Ly=2.4, Lz=2.0, dx=0.10, dy=0.10, n_z_bed=2,
    bed_x_start=0.5, bed_x_end=6.4,
    fuel_depth_m=0.20, bulk_density_kg_m3=0.30, sav_ratio_1_m=12240.0,
    initial_moisture_frac=0.04, wind_speed_m_s=4.0, cfl_factor=0.5,
    lagrangian_bed_N_per_cell=4, ignition_width_mult=0.4,
    solid_phase_ignition_T_s_K=1200.0, dom_subcycle_every=1,
    n_quadrature=4, jitter_seed=0,
)

# 400 x 120 x 60 cells (2.88M) at dx = dy = 0.1 m, dz = 0.0625 m, S8.
CFG2 = dict(
    COMMON,
    Lx=40.0, Ly=12.0, Lz=3.75, dx=0.10, dy=0.10, n_z_bed=4,
    bed_x_start=1.0, bed_x_end=40.0,
    fuel_depth_m=0.25, bulk_density_kg_m3=0.35, sav_ratio_1_m=12240.0,
    initial_moisture_frac=0.06, wind_speed_m_s=6.0, cfl_factor=0.5,
    lagrangian_bed_N_per_cell=4, ignition_width_mult=0.4,
    solid_phase_ignition_T_s_K=1200.0, dom_subcycle_every=1,
    n_quadrature=8, jitter_seed=0,
)

# 32 x 8 x 12 cells: the small case whose reference states are committed as fixtures.
TINY = dict(
    CFG1,
    Lx=3.2, Ly=0.8, Lz=1.2, bed_x_start=0.5, bed_x_end=3.2,
)

# 24 x 8 x 10 cells with a second (non-uniform-z-free) geometry and S4: parity smoke.
SMOKE = dict(
    CFG1,
    Lx=2.4, Ly=0.8, Lz=1.0, bed_x_start=0.3, bed_x_end=2.4,
)

# The 400 x 120 x 60 workload's geometry and physics (dz = 0.0625 m, n_z_bed 4,
# 16 bed particles per surface cell, S8, U10 6 m/s, moisture 0.06, bulk
# density 0.35) on a 40 x 16 x 60 cell slice, whose reference states are
# committed as fixtures.
CFG2_SLICE = dict(
    CFG2,
    Lx=4.0, Ly=1.6, bed_x_start=1.0, bed_x_end=4.0,
)

# Variants of the 32 x 8 x 12 case that reach the loop's exit tests
# (spread_3d.py:3413-3437): no ignition at all (the flame body stays empty),
# and a bed that ends one cell after the ignition strip (the front is at the
# bed's end from the start).
EXIT_CASES = {
    "extinct": dict(TINY, solid_phase_ignition_enable=False, ignition_duration_s=0.0),
    "front": dict(TINY, bed_x_end=0.75),
}

CASES = {"cfg1": CFG1, "cfg2": CFG2, "tiny": TINY, "smoke": SMOKE, "cfg2_slice": CFG2_SLICE}


def scaled(case: dict, nx: int | None = None, ny: int | None = None,
           nz: int | None = None) -> dict:
    """Return ``case`` with the domain resized to (nz, ny, nx) cells at the same spacing."""
    out = dict(case)
    dx, dy = out["dx"], out.get("dy", out["dx"])
    h = out["fuel_depth_m"]
    dz = h / out["n_z_bed"]
    if nx is not None:
        out["Lx"] = nx * dx
        out["bed_x_end"] = nx * dx
    if ny is not None:
        out["Ly"] = ny * dy
    if nz is not None:
        out["Lz"] = h + (nz - out["n_z_bed"]) * dz
    return out


def batch_cases(n: int = 32, seed0: int = 0, nx_range=(200, 600)) -> list[dict]:
    """The batched sweep of uneven domains: ``n`` cases with Nx drawn uniformly
    from ``nx_range`` (inclusive), Ny = 120, Nz = 60, dx = dy = 0.1 m,
    n_z_bed = 4, dz = h/4 and Lz = 15 h, and per case U10 ~ U(1, 8) m/s,
    moisture ~ U(0.02, 0.12), bulk density ~ U(0.2, 0.6) kg/m3 and fuel depth
    h ~ U(0.1, 0.4) m, each case from its own PCG64 stream seeded with
    ``seed0 + k`` (the seed is also the case's particle-jitter seed)."""
    import numpy as np
    out = []
    for k in range(n):
        rng = np.random.Generator(np.random.PCG64(seed0 + k))
        nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        u10 = float(rng.uniform(1.0, 8.0))
        moist = float(rng.uniform(0.02, 0.12))
        rho_b = float(rng.uniform(0.2, 0.6))
        h = float(rng.uniform(0.1, 0.4))
        out.append(dict(
            CFG2,
            Lx=nx * 0.1, Ly=12.0, Lz=15.0 * h, dx=0.10, dy=0.10, n_z_bed=4,
            bed_x_start=1.0, bed_x_end=nx * 0.1,
            fuel_depth_m=h, bulk_density_kg_m3=rho_b, initial_moisture_frac=moist,
            wind_speed_m_s=u10, jitter_seed=seed0 + k,
        ))
    return out


def learned_cases(n: int = 4, seed0: int = 100, nx: int = 400) -> list[dict]:
    """Cases for the learned preconditioner's training pairs and held-out
    runs: the 400x120x60 workload (``nx`` x-cells) with U10 ~ U(2, 8) m/s and
    moisture ~ U(0.02, 0.12) from a PCG64 stream seeded with ``seed0 + k``
    (also the case's particle-jitter seed).  Grid: (60, 120, nx) cells."""
    import numpy as np
    out = []
    for k in range(n):
        rng = np.random.Generator(np.random.PCG64(seed0 + k))
        c = scaled(CFG2, nx=nx) if nx != 400 else dict(CFG2)
        c.update(wind_speed_m_s=float(rng.uniform(2.0, 8.0)),
                 initial_moisture_frac=float(rng.uniform(0.02, 0.12)),
                 jitter_seed=seed0 + k)
        out.append(c)
    return out
