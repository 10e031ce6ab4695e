"""Run the reference Tier-3 solver in this container and capture its state.

Fixture generation only: this module imports the reference package from its
source tree (default ``/root/reference/src``, override with ``FIRE_REF_SRC``)
and is never imported by the product, by ``smoke()`` or by ``bench.py``.

What it does to the reference, all at import/run time and without copying any
reference file:

* ``pypardiso`` is absent here; ``projection_3d.py:62`` imports it at module
  top, so a stub module is installed in ``sys.modules`` (the ``fft_pcg``
  projection never touches it).
* ``NUMBA_NUM_THREADS=1`` is forced before numba loads: the EDC kernel's
  ``_h2o_quench_substantial`` flag (``edc.py:223``) is only assigned on one
  branch, so its value leaks from the previously visited cell and the result
  depends on the prange chunking.  One thread gives flat k-j-i order.
* The k-epsilon buoyancy gradient at ``turbulence_3d.py:620`` reads
  ``T_g[k+1]``/``T_g[k-1]`` without a guard.  The module source is re-executed
  with that line replaced by the one-sided boundary form the upstream fix uses
  (``docs/js/physics/kepsilon.js:233-236``); the committed ``kepsilon`` golden
  vectors pin that fixed form.
* Bed-particle positions are re-drawn inside each particle's own cell from a
  seeded PCG64 stream (:func:`jitter_positions`), because the reference packs
  them on a deterministic lattice and the workloads ask for seeded jitter.
* S8 (80 ordinates) is injected by replacing ``dom_3d._generate_sn_ordinates``
  when ``n_quadrature == 8`` (the reference raises for N != 4,
  ``dom_3d.py:114-127``).
* A step cap: ``spread_3d._update_front_tracking`` is called once per outer
  step (``spread_3d.py:3453``), after the closing EoS update; the wrapper
  snapshots the state there and stops the run after ``n_steps``.
"""
from __future__ import annotations

import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

REF_SRC = Path(os.environ.get("FIRE_REF_SRC", "/root/reference/src"))


class _Stop(Exception):
    pass


def _install_stubs():
    if "pypardiso" not in sys.modules:
        m = types.ModuleType("pypardiso")

        class PyPardisoSolver:  # noqa: D401 - stub
            def __init__(self, *a, **k):
                raise RuntimeError("pypardiso stub: use projection_method=fft_pcg")

        m.PyPardisoSolver = PyPardisoSolver
        sys.modules["pypardiso"] = m


def _patch_kepsilon(T):
    """Re-execute turbulence_3d with the one-sided dT/dz at k=0 and k=Nz-1."""
    src = Path(T.__file__).read_text(encoding="utf-8")
    old = "dTdz = (T_g[k + 1, j, i] - T_g[k - 1, j, i]) * inv_dz_central"
    assert src.count(old) == 1, "k-epsilon buoyancy line not found"
    indent = src[src.index(old) - 200:src.index(old)].split("\n")[-1]
    new = (
        "if k == 0:\n"
        f"{indent}    dTdz = (T_g[1, j, i] - T_g[0, j, i]) * (1.0 / d_face_above[0])\n"
        f"{indent}elif k == Nz - 1:\n"
        f"{indent}    dTdz = (T_g[Nz - 1, j, i] - T_g[Nz - 2, j, i]) * (1.0 / d_face_below[Nz - 1])\n"
        f"{indent}else:\n"
        f"{indent}    dTdz = (T_g[k + 1, j, i] - T_g[k - 1, j, i]) * inv_dz_central"
    )
    src = src.replace(old, new).replace("cache=True", "cache=False")
    code = compile(src, T.__file__ + ":patched", "exec")
    exec(code, T.__dict__)


_LOADED = {}


def load_reference():
    """Import the reference modules (once) with stubs and patches applied."""
    if _LOADED:
        return _LOADED
    os.environ["NUMBA_NUM_THREADS"] = "1"
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    _install_stubs()
    if str(REF_SRC) not in sys.path:
        sys.path.insert(0, str(REF_SRC))
    from model_outdoor import spread_3d as S
    from model_outdoor.physics_3d import (turbulence_3d, dom_3d, projection_3d,
                                          lagrangian_bed_3d, soil_3d,
                                          flame_front_3d, momentum_3d)
    from model_outdoor.physics_3d import chemistry_closures
    _patch_kepsilon(turbulence_3d)
    _LOADED.update(S=S, T=turbulence_3d, D=dom_3d, P=projection_3d,
                   L=lagrangian_bed_3d, soil=soil_3d, F=flame_front_3d,
                   M=momentum_3d, C=chemistry_closures)
    return _LOADED


def jitter_positions(x, y, z, dx, dy, z_face, seed):
    """Seeded positions inside each particle's own cell (same as the product init)."""
    from firewebapp_b200.grid import jitter_particle_positions
    return jitter_particle_positions(x, y, z, dx, dy, z_face, seed)


def write_deck(case: dict, path: Path):
    skip = {"wind_speed_m_s", "n_quadrature", "jitter_seed"}
    lines = ["t_end = 1.0"]
    for k, v in case.items():
        if k in skip:
            continue
        if isinstance(v, bool):
            v = "true" if v else "false"
        lines.append(f"outdoor.{k} = {v}")
    path.write_text("\n".join(lines) + "\n")


STATE_FIELDS = ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "T_s",
                "alpha_s")
PART_FIELDS = ("x", "y", "z", "alive", "m_solid", "m_water", "m_char", "T_s",
               "m_water_0", "sav", "m_char_max")


def run_reference(case: dict, n_steps: int, capture_steps=None,
                  projection_cg_rtol: float = 1e-12, verbose=False, step_hook=None,
                  snapshot_dir=None):
    """Run the reference for ``n_steps`` outer steps; return per-step snapshots.

    Returns ``(init, snaps, trace)``: ``init`` is the state right after the
    driver's initialisation (before step 1), ``snaps[n]`` the state after step
    ``n`` for every ``n`` in ``capture_steps`` and ``trace`` per-step scalars
    (dt, projection iterations, DOM source iterations).  ``step_hook(n,
    state, extras)``, if given, is called after every step with the
    reference's state object and the captured extra fields.  With
    ``snapshot_dir`` the reference writes its own ``snap_NNNN.npz`` files
    there (``spread_3d.py:3536-3670``).
    """
    R = load_reference()
    S, T, D, P, L, soil, F, C = (R[k] for k in "S T D P L soil F C".split())
    capture_steps = set(capture_steps or range(1, n_steps + 1))
    cap = {}
    trace = {"dt": [], "proj_calls": [], "dom_sweeps": [], "t": []}
    counters = {"step": 0, "proj": 0, "sweeps": 0}
    init = {}

    orig = {}

    def wrap(mod, name, fn):
        orig[(mod, name)] = getattr(mod, name)
        setattr(mod, name, fn)

    # --- state capture hooks -------------------------------------------------
    def alloc(*a, **k):
        st = orig[(S.CellState3D, "allocate")](*a, **k)
        cap["state"] = st
        return st
    orig[(S.CellState3D, "allocate")] = S.CellState3D.allocate
    S.CellState3D.allocate = staticmethod(alloc)

    def bed_alloc(n):
        buf = orig[(L, "allocate_bed_particle_buffers")](n)
        cap["bed"] = buf
        return buf
    wrap(L, "allocate_bed_particle_buffers", bed_alloc)

    def bed_init(buf, alpha_s, *a, **k):
        n = orig[(L, "initialize_bed_particles_from_alpha_s")](buf, alpha_s, *a, **k)
        dx, dy, dz_arr = k["dx"], k["dy"], k["dz_arr"]
        z_face = np.concatenate([[0.0], np.cumsum(dz_arr)])
        nx_, ny_, nz_ = jitter_positions(buf["x"][:n], buf["y"][:n], buf["z"][:n],
                                         dx, dy, z_face, case.get("jitter_seed", 0))
        buf["x"][:n] = nx_
        buf["y"][:n] = ny_
        buf["z"][:n] = nz_
        cap["n_alloc"] = n
        return n
    wrap(L, "initialize_bed_particles_from_alpha_s", bed_init)

    def keps(*a, **k):
        cap["k_turb"], cap["eps_turb"], cap["nu_t"] = a[0], a[1], a[2]
        return orig[(T, "step_k_epsilon")](*a, **k)
    wrap(T, "step_k_epsilon", keps)

    def soil_step(T_soil, q_in, *a, **k):
        cap["T_soil"], cap["q_in_soil"] = T_soil, q_in
        return orig[(soil, "step_soil_conduction")](T_soil, q_in, *a, **k)
    wrap(soil, "step_soil_conduction", soil_step)

    def closure_run(name, **kw):
        cap["omega"] = kw["omega_out"]
        return orig[(C, "run")](name, **kw)
    wrap(C, "run", closure_run)

    def bed_step(*a, **k):
        # positional layout of lagrangian_bed_3d.step_bed_particles
        cap["Q_solid_ext"] = a[12]
        cap["S_pyro_b"], cap["S_dry_b"] = a[14], a[15]
        cap["Q_gconv_b"] = a[21]
        return orig[(L, "step_bed_particles")](*a, **k)
    wrap(L, "step_bed_particles", bed_step)

    DomCls = D.DOMRadiationSolver
    n_quad = int(case.get("n_quadrature", 4))

    class DomWrap(DomCls):
        def __init__(self, *a, **k):
            if n_quad != 4:
                k["N_quadrature"] = n_quad
            super().__init__(*a, **k)
            cap["dom"] = self

        def solve(self, *a, **k):
            cap["q_rad"], cap["q_rad_gas"] = k["q_rad_solid_out"], k["q_rad_gas_out"]
            cap["M_local"] = k.get("bed_moisture_per_cell")
            return super().solve(*a, **k)
    D.DOMRadiationSolver = DomWrap
    if n_quad == 8:
        from firewebapp_b200.quadrature import level_symmetric
        orig_gen = D._generate_sn_ordinates

        def gen(N):
            if N == 8:
                return level_symmetric(8)
            return orig_gen(N)
        wrap(D, "_generate_sn_ordinates", gen)

    ProjCls = P.ProjectionSolver3D

    class ProjWrap(ProjCls):
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            cap["proj"] = self

        def project(self, *a, **k):
            counters["proj"] += 1
            return super().project(*a, **k)
    P.ProjectionSolver3D = ProjWrap

    LsCls = F.LevelSetFront3D

    class LsWrap(LsCls):
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            cap["lset"] = self
    F.LevelSetFront3D = LsWrap

    def sweep(*a, **k):
        counters["sweeps"] += 1
        return orig[(D, "_sweep_one_ordinate")](*a, **k)
    wrap(D, "_sweep_one_ordinate", sweep)

    def sponge(u, u_t, sig, YF, skip, dt):
        trace["dt"].append(float(dt))
        if "u_inlet" not in cap:
            cap["u_inlet"] = np.array(u_t)
        return orig[(_M(), "apply_outflow_sponge")](u, u_t, sig, YF, skip, dt)
    wrap(_M(), "apply_outflow_sponge", sponge)

    snaps = {}

    def snapshot():
        st = cap["state"]
        out = {f: np.array(getattr(st, f)) for f in STATE_FIELDS}
        for f in ("k_turb", "eps_turb", "nu_t", "omega", "T_soil", "q_rad",
                  "q_rad_gas", "S_pyro_b", "S_dry_b", "Q_gconv_b", "M_local"):
            if cap.get(f) is not None:
                out[f] = np.array(cap[f])
        n = cap.get("n_alloc", 0)
        for f in PART_FIELDS:
            out["p_" + f] = np.array(cap["bed"][f][:n])
        out["p_prev"] = np.array(cap["proj"]._p_prev).reshape(out["rho"].shape)
        out["phi"] = np.array(cap["lset"].phi)
        out["lset_step"] = np.int64(cap["lset"]._step)
        return out

    def front(*a, **k):
        counters["step"] += 1
        n = counters["step"]
        trace["proj_calls"].append(counters["proj"])
        trace["dom_sweeps"].append(counters["sweeps"])
        counters["proj"] = 0
        counters["sweeps"] = 0
        if step_hook is not None:
            step_hook(n, cap["state"], cap)
        if n in capture_steps:
            snaps[n] = snapshot()
            if "dom" in cap:
                snaps[n]["I_set"] = np.array(cap["dom"].I_set)
        if n >= n_steps:
            raise _Stop()
        return orig[(S, "_update_front_tracking")](*a, **k)
    wrap(S, "_update_front_tracking", front)

    # The first k-epsilon call happens inside step 1, so the init snapshot is
    # taken by wrapping the DOM constructor's caller-visible state later; the
    # init fields that matter are reconstructed from the allocation hooks.
    def proj_ctor_snapshot():
        st = cap["state"]
        init.update({f: np.array(getattr(st, f)) for f in STATE_FIELDS})
        n = cap.get("n_alloc", 0)
        for f in PART_FIELDS:
            init["p_" + f] = np.array(cap["bed"][f][:n])

    class ProjWrap2(ProjWrap):
        def __init__(self, *a, **k):
            proj_ctor_snapshot()
            super().__init__(*a, **k)
    P.ProjectionSolver3D = ProjWrap2

    with tempfile.TemporaryDirectory() as td:
        deck = Path(td) / "case.txt"
        write_deck(case, deck)
        try:
            import contextlib
            import io
            sink = io.StringIO()
            ctx = contextlib.nullcontext() if verbose else contextlib.redirect_stdout(sink)
            with ctx:
                S.run_3d_spread(deck, wind_speed_m_s=float(case["wind_speed_m_s"]),
                                projection_cg_rtol=projection_cg_rtol,
                                snapshot_dir=snapshot_dir)
        except _Stop:
            pass
        finally:
            S.CellState3D.allocate = orig[(S.CellState3D, "allocate")]
            for (mod, name), fn in orig.items():
                if mod is S.CellState3D:
                    continue
                setattr(mod, name, fn)
            D.DOMRadiationSolver = DomCls
            P.ProjectionSolver3D = ProjCls
            F.LevelSetFront3D = LsCls
    trace["dt"] = trace["dt"][:n_steps]
    return init, snaps, trace


def _M():
    return _LOADED["M"]
