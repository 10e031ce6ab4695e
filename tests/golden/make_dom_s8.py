"""Reference DOM solves at S8 (80 ordinates) for the DOM parity tests.

The reference's ``_generate_sn_ordinates`` raises for N != 4
(``dom_3d.py:114-127``); the benchmarked workload uses S8, so the level-
symmetric S8 set of ``firewebapp_b200/quadrature.py`` is injected into the
reference module (as ``refharness.py`` does for whole runs) and the
reference's own ``DOMRadiationSolver.solve`` (``dom_3d.py:286-473``) is run
on two kinds of input:

* the geometry and fields of every ``dom`` case of the reference's golden
  vectors (``docs/data/kernel_vectors.json``), solved twice in a row (the
  second solve starts from the intensities the first left, as in a run);
* a 40 x 16 x 60 slice with the 400 x 120 x 60 workload's vertical grid
  (dz = 0.0625 m, four bed layers) and seeded fields shaped like a burning
  bed (hot bed cells, a hot plume, water vapour), solved twice.

Writes ``dom_s8.npz`` next to this file: key ``"<case>/<name>"`` for inputs
and ``"<case>/call<n>/<output>"`` for the outputs of solve n (q_rad_solid,
q_rad_gas, q_in_soil, iterations).  Run here, where the reference imports:

    python tests/golden/make_dom_s8.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))


def _slice_inputs(seed=8):
    """Seeded fields on the 40 x 16 x 60 slice of the 400 x 120 x 60 grid."""
    from firewebapp_b200.cases import CFG2_SLICE
    from firewebapp_b200.grid import build_setup
    g = build_setup(CFG2_SLICE).grid
    nz, ny, nx = g.shape
    rng = np.random.default_rng(seed)
    bed = np.zeros(g.shape, dtype=bool)
    bed[:g.n_z_bed, :, 10:] = True
    alpha = np.where(bed, 0.002 * (0.5 + rng.random(g.shape)), 0.0)
    hot = np.zeros(g.shape)
    hot[:, :, 10:16] = 1.0
    T_s = np.where(bed, 300.0 + 800.0 * hot * rng.random(g.shape), 300.0)
    zc = np.asarray(g.z_mid)[:, None, None]
    T_g = 300.0 + 1300.0 * hot * np.exp(-zc / 1.0) * rng.random(g.shape)
    om = np.where(hot > 0, 5e-3 * rng.random(g.shape), 0.0)
    YH = 0.12 * hot * rng.random(g.shape)
    rho = 101325.0 / (8.314 / 0.029 * np.maximum(T_g, 300.0))
    bedM = np.where(bed, 0.06 * (0.5 + rng.random(g.shape)), 0.0)
    Tsoil = 300.0 + 30.0 * rng.random((ny, nx))
    return dict(nz=nz, ny=ny, nx=nx, dx=g.dx, dy=g.dy, dz_arr=np.asarray(g.dz_arr),
                d_face_above=np.asarray(g.d_face_above), d_face_below=np.asarray(g.d_face_below),
                sigma_sav=12240.0, T_amb=300.0, T_s=T_s, T_g=T_g, alpha_s=alpha,
                omega_comb=om, Y_H2O=YH, rho=rho, bed_moisture=bedM, T_soil=Tsoil)


def _vector_inputs():
    """Every ``dom`` case of the golden vectors, as arrays."""
    sys.path.insert(0, str(HERE.parent))
    from conftest import Vectors
    V = Vectors(HERE / "kernel_vectors.npz")
    out = {}
    for name in V.cases("dom"):
        c = V.case("dom", name)
        shp = (c["nz"], c["ny"], c["nx"])
        d = dict(nz=c["nz"], ny=c["ny"], nx=c["nx"], dx=c["dx"], dy=c["dy"],
                 dz_arr=np.asarray(c["dz_arr"]), sigma_sav=c["sigma_sav"], T_amb=c["T_amb"],
                 T_soil=np.asarray(c["T_soil"]).reshape(shp[1:]))
        dz = d["dz_arr"]
        d["d_face_above"] = np.concatenate([0.5 * (dz[:-1] + dz[1:]), [dz[-1]]])
        d["d_face_below"] = np.concatenate([[dz[0]], 0.5 * (dz[:-1] + dz[1:])])
        for k in ("T_s", "T_g", "alpha_s", "omega_comb", "bed_moisture", "Y_H2O", "rho"):
            if k in c:
                d[k] = np.asarray(c[k]).reshape(shp)
        out["vec_" + name] = d
    return out


def _second_call(d, seed):
    """Inputs of the second solve: the fields moved a little (the intensities
    the first solve left are its starting point)."""
    rng = np.random.default_rng(seed)
    e = dict(d)
    e["T_g"] = d["T_g"] * (1.0 + 0.05 * rng.random(d["T_g"].shape))
    e["T_s"] = d["T_s"] * (1.0 + 0.02 * rng.random(d["T_s"].shape))
    return e


def main():
    from refharness import load_reference
    from firewebapp_b200.quadrature import level_symmetric
    R = load_reference()
    D = R["D"]
    orig = D._generate_sn_ordinates
    D._generate_sn_ordinates = lambda N: level_symmetric(8) if N == 8 else orig(N)
    cases = _vector_inputs()
    cases["slice"] = _slice_inputs()
    out = {}
    try:
        for cname, d in cases.items():
            nz, ny, nx = d["nz"], d["ny"], d["nx"]
            sol = D.DOMRadiationSolver(nz, ny, nx, d["dy"], d["dx"], d["dz_arr"],
                                       d["d_face_above"], d["d_face_below"], "periodic", 8)
            for k, v in d.items():
                out[f"{cname}/{k}"] = np.asarray(v)
            for call, inp in enumerate((d, _second_call(d, 17))):
                qs = np.zeros((nz, ny, nx)); qg = np.zeros((nz, ny, nx))
                qsoil = np.zeros((ny, nx))
                for k in ("T_s", "T_g"):
                    out[f"{cname}/call{call}/{k}"] = np.asarray(inp[k])
                sweeps = [0]
                real = D._sweep_one_ordinate

                def count(*a, **kw):
                    sweeps[0] += 1
                    return real(*a, **kw)
                D._sweep_one_ordinate = count
                try:
                    sol.solve(np.ascontiguousarray(inp["T_s"]), np.ascontiguousarray(inp["T_g"]),
                              inp["alpha_s"], inp["omega_comb"], inp["sigma_sav"], inp["T_amb"],
                              qs, qg, inp["T_soil"], qsoil, inp.get("Y_H2O"), inp.get("rho"),
                              inp["bed_moisture"])
                finally:
                    D._sweep_one_ordinate = real
                out[f"{cname}/call{call}/q_rad_solid"] = qs
                out[f"{cname}/call{call}/q_rad_gas"] = qg
                out[f"{cname}/call{call}/q_in_soil"] = qsoil
                out[f"{cname}/call{call}/iterations"] = np.int64(sweeps[0] // 80)
                print(cname, call, "iterations", sweeps[0] // 80, "max q", float(np.abs(qs).max()))
    finally:
        D._generate_sn_ordinates = orig
    np.savez_compressed(HERE / "dom_s8.npz", **out)


if __name__ == "__main__":
    main()
