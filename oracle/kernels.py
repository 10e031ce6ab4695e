"""Vectorised numpy restatement of the Tier-3 kernels (oracle; test infrastructure).

Fields are float64 arrays shaped (Nz, Ny, Nx).  Every function returns new
arrays (or fills the outputs it is given) and cites the reference function it
restates.  The arithmetic follows the reference's expression order so that
results agree to round-off; where the reference's boundary handling is a
branch per cell, this code evaluates both branches and selects with masks.
"""
from __future__ import annotations

import math

import numpy as np

# ---------------------------------------------------------------- stencil helpers


def nb(a, d, axis):
    """a shifted by d along axis with the index clamped (values past the edge
    repeat the edge; callers mask them out or replace them with ghosts)."""
    n = a.shape[axis]
    idx = np.clip(np.arange(n) + d, 0, n - 1)
    return np.take(a, idx, axis=axis)


def yroll(a, d):
    """a[..., j+d, ...] with periodic j (axis 1)."""
    return np.roll(a, -d, axis=1)


def minmod(a, b):
    """muscl_3d.py:37-44"""
    out = np.where(a > 0.0, np.where(a < b, a, b), np.where(a > b, a, b))
    return np.where(a * b <= 0.0, 0.0, out)


def muscl_face(pim1, pi, pip1, pip2, uf):
    """muscl_3d.py:47-64"""
    up = pi + 0.5 * minmod(pi - pim1, pip1 - pi)
    dn = pip1 - 0.5 * minmod(pip1 - pi, pip2 - pip1)
    return np.where(uf >= 0.0, up, dn)


def _kcol(a):
    return np.asarray(a, dtype=np.float64).reshape(-1, 1, 1)


def _masks(shape):
    nz, ny, nx = shape
    i = np.arange(nx)[None, None, :]
    k = np.arange(nz)[:, None, None]
    mx = (i >= 2) & (i <= nx - 3)
    mz = (k >= 2) & (k <= nz - 3)
    return i, k, mx, mz


# ---------------------------------------------------------------- advection


def muscl_fluxes(phi, u, v, w, xL_ghost, xR_self, zL, zR, kind, dx, dy, da, db):
    """The three MUSCL/upwind flux terms shared by the transport kernels.

    kind selects how the reference divides:
      'species'  species_3d.py:288-319 (x,y times inv_dx; z MUSCL divided by
                 0.5*(da+db); z upwind times 1/db or 1/da)
      'scalar'   muscl_3d.py:125-171 (x,y divided by dx, dy)
    Returns (flux_x, flux_y, flux_z).
    """
    shape = phi.shape
    i, k, mx, mz = _masks(shape)
    xm1, xm2 = nb(phi, -1, 2), nb(phi, -2, 2)
    xp1, xp2 = nb(phi, 1, 2), nb(phi, 2, 2)
    fxp = muscl_face(xm1, phi, xp1, xp2, u)
    fxm = muscl_face(xm2, xm1, phi, xp1, u)
    ym1, ym2, yp1, yp2 = yroll(phi, -1), yroll(phi, -2), yroll(phi, 1), yroll(phi, 2)
    fyp = muscl_face(ym1, phi, yp1, yp2, v)
    fym = muscl_face(ym2, ym1, phi, yp1, v)
    zm1, zm2 = nb(phi, -1, 0), nb(phi, -2, 0)
    zp1, zp2 = nb(phi, 1, 0), nb(phi, 2, 0)
    fzp = muscl_face(zm1, phi, zp1, zp2, w)
    fzm = muscl_face(zm2, zm1, phi, zp1, w)
    hz = _kcol(0.5 * (np.asarray(da) + np.asarray(db)))
    idb = _kcol(1.0 / np.asarray(db))
    ida = _kcol(1.0 / np.asarray(da))
    if kind == "species":
        inv_dx, inv_dy = 1.0 / dx, 1.0 / dy
        fx_m = u * (fxp - fxm) * inv_dx
        fx_u = np.where(u >= 0.0, u * (phi - xL_ghost) * inv_dx, u * (xR_self - phi) * inv_dx)
        fy = v * (fyp - fym) * inv_dy
    else:
        fx_m = u * (fxp - fxm) / dx
        fx_u = np.where(u >= 0.0, u * (phi - xL_ghost) / dx, u * (xR_self - phi) / dx)
        fy = v * (fyp - fym) / dy
    fz_m = w * (fzp - fzm) / hz
    fz_u = np.where(w >= 0.0, w * (phi - zL) * idb, w * (zR - phi) * ida)
    return np.where(mx, fx_m, fx_u), fy, np.where(mz, fz_m, fz_u)


def _ghosts_x(phi, inlet):
    nx = phi.shape[2]
    xL = nb(phi, -1, 2).copy()
    xL[:, :, 0] = inlet
    xR = nb(phi, 1, 2).copy()
    xR[:, :, nx - 1] = phi[:, :, nx - 1]
    return xL, xR


def _ghosts_z_wall(phi):
    nz = phi.shape[0]
    zL = nb(phi, -1, 0).copy()
    zL[0] = phi[0]
    zR = nb(phi, 1, 0).copy()
    zR[nz - 1] = phi[nz - 1]
    return zL, zR


def advect_scalar_muscl(phi, u, v, w, dx, dy, da, db, rhs, phi_inlet):
    """muscl_3d.py:67-171 advect_3d_scalar_muscl: rhs -= u.grad(phi) (in place)."""
    xL, xR = _ghosts_x(phi, phi_inlet)
    zL, zR = _ghosts_z_wall(phi)
    fx, fy, fz = muscl_fluxes(phi, u, v, w, xL, xR, zL, zR, "scalar", dx, dy, da, db)
    rhs -= fx + fy + fz
    return rhs


def species_transport(Y, rho, u, v, w, S, dt, dx, dy, dz, da, db, D, Y_inlet):
    """species_3d.py:41-175 step_species_transport; returns the new Y."""
    xL, xR = _ghosts_x(Y, Y_inlet)
    zL, zR = _ghosts_z_wall(Y)
    fx, fy, fz = muscl_fluxes(Y, u, v, w, xL, xR, zL, zR, "species", dx, dy, da, db)
    adv = -(fx + fy + fz)
    inv_dx, inv_dy = 1.0 / dx, 1.0 / dy
    inv_dx2, inv_dy2 = inv_dx * inv_dx, inv_dy * inv_dy
    ida = _kcol(1.0 / np.asarray(da))
    idb = _kcol(1.0 / np.asarray(db))
    idz = _kcol(1.0 / np.asarray(dz))
    d2x = (xR - 2.0 * Y + xL) * inv_dx2
    d2y = (yroll(Y, 1) - 2.0 * Y + yroll(Y, -1)) * inv_dy2
    d2z = ((zR - Y) * ida - (Y - zL) * idb) * idz
    diff = D * (d2x + d2y + d2z)
    src = S / rho
    new = Y + (adv + diff + src) * dt
    return np.where(new < 0.0, 0.0, np.where(new > 1.0, 1.0, new))


def gas_energy_adv(T, u, v, w, dt, dx, dy, dz, da, db, alpha_th, T_amb):
    """spread_3d.py:3827-3897 _adv_gas_energy; returns the new T_g."""
    nz, ny, nx = T.shape
    dT = np.zeros_like(T)
    advect_scalar_muscl(T, u, v, w, dx, dy, da, db, dT, T_amb)
    inv_dx2 = 1.0 / (dx * dx)
    dT[:, :, 1:-1] += alpha_th * (T[:, :, 2:] - 2.0 * T[:, :, 1:-1] + T[:, :, :-2]) * inv_dx2
    dT[:, :, 0] += alpha_th * (T[:, :, 1] - 2.0 * T[:, :, 0] + T_amb) * inv_dx2
    dT[:, :, -1] += alpha_th * (T[:, :, -2] - T[:, :, -1]) * inv_dx2
    dT += alpha_th * (yroll(T, 1) - 2.0 * T + yroll(T, -1)) / (dy * dy)
    ida = (1.0 / np.asarray(da)[1:-1]).reshape(-1, 1, 1)
    idb = (1.0 / np.asarray(db)[1:-1]).reshape(-1, 1, 1)
    idz = (1.0 / np.asarray(dz)[1:-1]).reshape(-1, 1, 1)
    dT[1:-1] += alpha_th * ((T[2:] - T[1:-1]) * ida - (T[1:-1] - T[:-2]) * idb) * idz
    dT[0] += alpha_th * ((T[1] - T[0]) / da[0]) / dz[0]
    dT[-1] += alpha_th * (-(T[-1] - T[-2]) / db[-1]) / dz[-1]
    out = T + dT * dt
    out = np.maximum(out, T_amb)
    return np.minimum(out, 10_000.0)


# ---------------------------------------------------------------- diffusion


def turb_diffusion_nsub(nu_t, sc_t, dt, dx, dy, dz):
    """turbulence_3d.py:880-915: (n_sub, dt_sub) or (0, 0) when skipped."""
    dz_min = float(np.min(dz))
    h_min2 = min(dx * dx, min(dy * dy, dz_min * dz_min))
    inner = nu_t[1:-1, :, 1:-1]
    inner = inner[~np.isnan(inner)]
    nu_max = max(0.0, float(inner.max())) if inner.size else 0.0
    D_max = nu_max / sc_t
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


def turb_diffusion(field, nu_t, sc_t, dt, dx, dy, dz, da, db):
    """turbulence_3d.py:862-949 apply_turbulent_diffusion; returns the new field."""
    n, dts = turb_diffusion_nsub(nu_t, sc_t, dt, dx, dy, dz)
    if n == 0:
        return field.copy()
    f = field.copy()
    inv_dx2, inv_dy2 = 1.0 / (dx * dx), 1.0 / (dy * dy)
    ida = _kcol(1.0 / np.asarray(da))
    idb = _kcol(1.0 / np.asarray(db))
    idz = _kcol(1.0 / np.asarray(dz))
    Dt = nu_t / sc_t
    for _ in range(n):
        xL = nb(f, -1, 2).copy(); xL[:, :, 0] = f[:, :, 0]
        xR = nb(f, 1, 2).copy(); xR[:, :, -1] = f[:, :, -1]
        zL, zR = _ghosts_z_wall(f)
        d2x = (xR - 2.0 * f + xL) * inv_dx2
        d2y = (yroll(f, 1) - 2.0 * f + yroll(f, -1)) * inv_dy2
        d2z = ((zR - f) * ida - (f - zL) * idb) * idz
        f = f + Dt * (d2x + d2y + d2z) * dts
    return f


# ---------------------------------------------------------------- momentum


def drag_force(u, v, w, rho, alpha_s, sigma, C_D):
    """drag_3d.py:100-144 step_drag_force; returns (Fx, Fy, Fz)."""
    a = alpha_s
    speed = np.sqrt(u * u + v * v + w * w)
    om = 1.0 - a
    with np.errstate(divide="ignore", invalid="ignore"):
        K_visc = 50.0 * 3.0e-5 * (sigma * sigma) * a * a / (om * om * om)
    K_quad = C_D * sigma * a * 0.5 * rho * speed
    co = -(K_visc + K_quad)
    fuel = a > 0.0
    return (np.where(fuel, co * u, 0.0), np.where(fuel, co * v, 0.0), np.where(fuel, co * w, 0.0))


def tentative_velocity(u, v, w, rho, T, Fx, Fy, Fz, dt, dx, dy, dz, da, db, T_amb,
                       u_in, v_in, w_in):
    """momentum_3d.py:42-276 step_tentative_velocity; returns (u, v, w)."""
    nz, ny, nx = u.shape
    i, k, mx, mz = _masks(u.shape)
    inv_dx, inv_dy = 1.0 / dx, 1.0 / dy
    inv_dx2, inv_dy2 = inv_dx * inv_dx, inv_dy * inv_dy
    hz_inv = _kcol(1.0 / (0.5 * (np.asarray(da) + np.asarray(db))))
    ida = _kcol(1.0 / np.asarray(da))
    idb = _kcol(1.0 / np.asarray(db))
    idz = _kcol(1.0 / np.asarray(dz))
    nu = 1.8e-5 / rho

    def ghosts(q, qin):
        xL = nb(q, -1, 2).copy(); xL[:, :, 0] = qin
        xR = nb(q, 1, 2).copy(); xR[:, :, -1] = q[:, :, -1]
        zL = nb(q, -1, 0).copy(); zL[0] = 0.0
        zR = nb(q, 1, 0).copy(); zR[-1] = q[-1]
        return xL, xR, zL, zR

    comps = [(u, u_in), (v, v_in), (w, w_in)]
    out = []
    for q, qin in comps:
        xL, xR, zL, zR = ghosts(q, qin)
        fxp = muscl_face(nb(q, -1, 2), q, nb(q, 1, 2), nb(q, 2, 2), u)
        fxm = muscl_face(nb(q, -2, 2), nb(q, -1, 2), q, nb(q, 1, 2), u)
        dqdx = np.where(mx, (fxp - fxm) * inv_dx,
                        np.where(u >= 0.0, (q - xL) * inv_dx, (xR - q) * inv_dx))
        fyp = muscl_face(yroll(q, -1), q, yroll(q, 1), yroll(q, 2), v)
        fym = muscl_face(yroll(q, -2), yroll(q, -1), q, yroll(q, 1), v)
        dqdy = (fyp - fym) * inv_dy
        fzp = muscl_face(nb(q, -1, 0), q, nb(q, 1, 0), nb(q, 2, 0), w)
        fzm = muscl_face(nb(q, -2, 0), nb(q, -1, 0), q, nb(q, 1, 0), w)
        dqdz = np.where(mz, (fzp - fzm) * hz_inv,
                        np.where(w >= 0.0, (q - zL) * idb, (zR - q) * ida))
        adv = -(u * dqdx + v * dqdy + w * dqdz)
        lap = ((xR - 2.0 * q + xL) * inv_dx2 + (yroll(q, 1) - 2.0 * q + yroll(q, -1)) * inv_dy2
               + ((zR - q) * ida - (q - zL) * idb) * idz)
        out.append((adv, nu * lap))
    buoy = 9.81 * (T - T_amb) / T_amb
    du = (out[0][0] + out[0][1] + Fx / rho) * dt
    dv = (out[1][0] + out[1][1] + Fy / rho) * dt
    dw = (out[2][0] + out[2][1] + buoy + Fz / rho) * dt
    return u + du, v + dv, w + dw


def outflow_sponge(u, u_t, sigma_x, Y_F, skip, dt):
    """momentum_3d.py:293-317 apply_outflow_sponge; returns the new u."""
    sig = sigma_x[None, None, :]
    ut = u_t[:, :, None]
    m = (sig > 0.0) & (Y_F < skip)
    return np.where(m, u + sig * dt * (ut - u), u)


# ---------------------------------------------------------------- k-epsilon


def strain_invariants(u, v, w, dx, dy, da, db, u_in):
    """turbulence_3d.py:392-478 (|S|^2, |Omega|^2)."""
    nz = u.shape[0]
    idzc = np.empty(nz)
    for k in range(nz):
        if k == 0:
            idzc[k] = 1.0 / da[0]
        elif k == nz - 1:
            idzc[k] = 1.0 / db[nz - 1]
        else:
            idzc[k] = 1.0 / (db[k] + da[k])
    idzc = _kcol(idzc)
    inv_dx, inv_dy = 1.0 / dx, 1.0 / dy

    def xg(q, inlet):
        L = nb(q, -1, 2).copy(); L[:, :, 0] = inlet
        R = nb(q, 1, 2).copy(); R[:, :, -1] = q[:, :, -1]
        return L, R

    def zg(q):
        L = nb(q, -1, 0).copy(); L[0] = 0.0
        R = nb(q, 1, 0).copy(); R[-1] = q[-1]
        return L, R

    uxL, uxR = xg(u, u_in)
    vxL, vxR = xg(v, 0.0)
    wxL, wxR = xg(w, 0.0)
    uzL, uzR = zg(u); vzL, vzR = zg(v); wzL, wzR = zg(w)
    dudx = (uxR - uxL) * 0.5 * inv_dx
    dudy = (yroll(u, 1) - yroll(u, -1)) * 0.5 * inv_dy
    dudz = (uzR - uzL) * idzc
    dvdx = (vxR - vxL) * 0.5 * inv_dx
    dvdy = (yroll(v, 1) - yroll(v, -1)) * 0.5 * inv_dy
    dvdz = (vzR - vzL) * idzc
    dwdx = (wxR - wxL) * 0.5 * inv_dx
    dwdy = (yroll(w, 1) - yroll(w, -1)) * 0.5 * inv_dy
    dwdz = (wzR - wzL) * idzc
    S12 = 0.5 * (dudy + dvdx); S13 = 0.5 * (dudz + dwdx); S23 = 0.5 * (dvdz + dwdy)
    S2 = 2.0 * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) + 4.0 * (S12 * S12 + S13 * S13 + S23 * S23)
    O12 = 0.5 * (dudy - dvdx); O13 = 0.5 * (dudz - dwdx); O23 = 0.5 * (dvdz - dwdy)
    O2 = 4.0 * (O12 * O12 + O13 * O13 + O23 * O23)
    return S2, O2


def k_epsilon(k_t, eps, u, v, w, T, alpha_s, sigma, dt, dx, dy, dz, da, db, T_amb, u_in,
              k_wall, eps_wall, beta_p=1.0, beta_d=4.0):
    """turbulence_3d.py:482-858 step_k_epsilon with the one-sided dT/dz at the
    wall and top (upstream fix, docs/js/physics/kepsilon.js:182-185,233-236).
    Returns (k_new, eps_new, nu_t)."""
    K_MIN = EPS_MIN = 1.0e-8
    nz, ny, nx = k_t.shape
    i, kk, mx, mz = _masks(k_t.shape)
    S2, O2 = strain_invariants(u, v, w, dx, dy, da, db, u_in)
    kl = np.where(k_t < K_MIN, K_MIN, k_t)
    el = np.where(eps < EPS_MIN, EPS_MIN, eps)
    kxL = nb(k_t, -1, 2).copy(); kxL[:, :, 0] = K_MIN
    exL = nb(eps, -1, 2).copy(); exL[:, :, 0] = EPS_MIN
    kxR = nb(k_t, 1, 2).copy(); kxR[:, :, -1] = kl[:, :, -1]
    exR = nb(eps, 1, 2).copy(); exR[:, :, -1] = el[:, :, -1]
    kzL = nb(k_t, -1, 0).copy(); kzL[0] = k_wall
    ezL = nb(eps, -1, 0).copy(); ezL[0] = eps_wall
    kzR = nb(k_t, 1, 0).copy(); kzR[-1] = kl[-1]
    ezR = nb(eps, 1, 0).copy(); ezR[-1] = el[-1]
    U_star = np.sqrt(0.5 * (S2 + O2))
    C_mu = 1.0 / (4.04 + 4.5 * U_star * kl / el)
    nu_t = C_mu * kl * kl / el
    nu_t = np.where(nu_t < 0.0, 0.0, nu_t)
    P_k = nu_t * S2
    P_lim = np.where(P_k > 10.0 * el, 10.0 * el, P_k)
    dTdz = np.empty_like(T)
    dTdz[1:-1] = (T[2:] - T[:-2]) * _kcol(1.0 / (np.asarray(da)[1:-1] + np.asarray(db)[1:-1]))
    dTdz[0] = (T[1] - T[0]) * (1.0 / da[0])
    dTdz[-1] = (T[-1] - T[-2]) * (1.0 / db[nz - 1])
    Tfb = np.where(T < T_amb, T_amb, T)
    G_k = (nu_t / 0.85) * (9.81 / Tfb) * dTdz
    G_k = np.where(G_k < 0.0, 0.0, G_k)
    G_kk = np.where(G_k > P_lim, P_lim, G_k)
    u_h = np.sqrt(u * u + v * v)
    u_h = np.where(u_h < 0.01, 0.01, u_h)
    C3 = np.tanh(np.abs(w) / u_h)
    speed = np.sqrt(u * u + v * v + w * w)
    cds = 1.0 * (sigma * alpha_s) * speed
    can = alpha_s > 0.0
    Pc = np.where(can, beta_p * cds * speed * speed, 0.0)
    Dc = np.where(can, beta_d * cds * kl, 0.0)
    hz = _kcol(0.5 * (np.asarray(da) + np.asarray(db)))
    ida = _kcol(1.0 / np.asarray(da))
    idb = _kcol(1.0 / np.asarray(db))
    idz = _kcol(1.0 / np.asarray(dz))
    inv_dx, inv_dy = 1.0 / dx, 1.0 / dy
    inv_dx2, inv_dy2 = 1.0 / (dx * dx), 1.0 / (dy * dy)

    def transport(F, Fl, xL, xR, zL, zR):
        fxp = muscl_face(nb(F, -1, 2), Fl, nb(F, 1, 2), nb(F, 2, 2), u)
        fxm = muscl_face(nb(F, -2, 2), nb(F, -1, 2), Fl, nb(F, 1, 2), u)
        ax = np.where(mx, u * (fxp - fxm) * inv_dx,
                      np.where(u >= 0.0, u * (Fl - xL) * inv_dx, u * (xR - Fl) * inv_dx))
        fyp = muscl_face(yroll(F, -1), Fl, yroll(F, 1), yroll(F, 2), v)
        fym = muscl_face(yroll(F, -2), yroll(F, -1), Fl, yroll(F, 1), v)
        ay = v * (fyp - fym) * inv_dy
        fzp = muscl_face(nb(F, -1, 0), Fl, nb(F, 1, 0), nb(F, 2, 0), w)
        fzm = muscl_face(nb(F, -2, 0), nb(F, -1, 0), Fl, nb(F, 1, 0), w)
        az = np.where(mz, w * (fzp - fzm) / hz,
                      np.where(w >= 0.0, w * (Fl - zL) * idb, w * (zR - Fl) * ida))
        lap = ((xR - 2.0 * Fl + xL) * inv_dx2 + (yroll(F, 1) - 2.0 * Fl + yroll(F, -1)) * inv_dy2
               + ((zR - Fl) * ida - (Fl - zL) * idb) * idz)
        return ax + ay + az, lap

    adv_k, lap_k = transport(k_t, kl, kxL, kxR, kzL, kzR)
    diff_k = (1.5e-5 + nu_t / 1.0) * lap_k
    S_pos_k = P_lim + G_kk + Pc + 0.0
    S_neg_k = el + Dc
    k_new = (kl + (-adv_k + diff_k + S_pos_k) * dt) / (1.0 + S_neg_k * dt / kl)
    k_new = np.where(k_new < K_MIN, K_MIN, k_new)
    adv_e, lap_e = transport(eps, el, exL, exR, ezL, ezR)
    diff_e = (1.5e-5 + nu_t / 1.3) * lap_e
    eta = np.sqrt(S2) * kl / el
    eta3 = eta * (eta * eta)
    rng = 0.09 * eta3 * (1.0 - eta / 4.38) / (1.0 + 0.012 * eta3)
    rng = np.where(rng < 0.0, 0.0, rng)
    ek = el / kl
    S_pos_e = 1.44 * (P_lim + C3 * G_k) * ek + 0.9 * Pc * ek
    S_neg_e = (1.92 + rng) * el * ek + 0.9 * Dc * ek
    e_new = (el + (-adv_e + diff_e + S_pos_e) * dt) / (1.0 + S_neg_e * dt / el)
    e_new = np.where(e_new < EPS_MIN, EPS_MIN, e_new)
    C_new = 1.0 / (4.04 + 4.5 * U_star * k_new / e_new)
    nu_new = C_new * k_new * k_new / e_new
    nu_new = np.where(nu_new < 0.0, 0.0, nu_new)
    return k_new, e_new, nu_new


# ---------------------------------------------------------------- chemistry


def edc(rho, T_g, Y_F, Y_O2, k_t, eps, Y_H2O, chi_rad, cp_g, dt, n_substeps, s_stoich,
        hoc_J, extinction):
    """chemistry_closures/edc.py:134-335 step_chemistry_ode_edc.

    The quench flag of the reference (edc.py:223) is only assigned when the
    cell takes the reacting branch; other cells reuse the value left by the
    previous cell in flat k-j-i order (one numba thread).  Here the flag of
    each cell is that forward-filled value.  Returns (T_g, Y_F, Y_O2, omega).
    """
    shape = T_g.shape
    Yf = Y_F.ravel().copy()
    YO = Y_O2.ravel().copy()
    Tg = T_g.ravel().copy()
    YH = Y_H2O.ravel()
    r = rho.ravel()
    kt = np.where(k_t.ravel() < 1.0e-4, 1.0e-4, k_t.ravel())
    et = np.where(eps.ravel() < 1.0e-6, 1.0e-6, eps.ravel())
    ratio = 1.5e-5 * et / (kt * kt)
    ratio = np.where(ratio < 1e-30, 1e-30, ratio)
    gx = 2.1377 * ratio ** 0.25
    gamma = gx * (gx * gx)
    gamma = np.where(gamma > 1.0, 1.0, gamma)
    tau = 0.4083 * np.sqrt(1.5e-5 / et)
    nsub = max(int(n_substeps), 1)
    h = dt / nsub
    HoC = hoc_J * (1.0 - chi_rad)
    relax = 1.0 - math.exp(-h / 0.5)
    # flag: forward fill over flat order of the value assigned in reacting cells
    reacting0 = ~((Yf <= 1e-9) | (YO <= 1e-9))
    fac0 = np.where(YH > 0.0, np.maximum(1.0 - YH / 0.18, 0.0), 1.0)
    own = (YH > 0.0) & (fac0 < 0.5)
    idx = np.where(reacting0, np.arange(Yf.size), -1)
    last = np.maximum.accumulate(idx)
    flag = np.where(last >= 0, own[np.maximum(last, 0)], False)
    acc = np.zeros_like(Tg)
    for _ in range(nsub):
        reacting = ~((Yf <= 1e-9) | (YO <= 1e-9))
        lim = YO / s_stoich
        Y_lim = np.where(Yf < lim, Yf, lim)
        om = gamma * (r * Y_lim / tau)
        fac = 1.0 - YH / 0.18
        fac = np.where(fac < 0.0, 0.0, fac)
        om = np.where(YH > 0.0, om * fac, om)
        om = np.where(reacting, om, 0.0)
        fired = np.zeros(om.shape, dtype=bool)
        if extinction:
            live = om > 0.0
            Yib = 1.0 - Yf - YO
            rs = np.maximum((1.0 - Yib) / (1.0 - 0.88), 0.0)
            b = live & (Yib > 0.88)
            om = np.where(b, om * rs, om)
            fired |= b & (rs < 0.5)
            c = (om > 0.0) & (Tg < 1200.0)
            om = np.where(c, 0.0, om)
            fired |= c
            a = (om > 0.0) & (om * HoC < 75000.0)
            om = np.where(a, 0.0, om)
            fired |= a
        wb = (fired | flag) & (Tg > 373.15) & (YH > 0.0)
        st = np.minimum(YH / 0.10, 1.0)
        Tg = np.where(wb, Tg - (Tg - 373.15) * relax * st, Tg)
        dY = -om * h / r
        Yf = Yf + dY
        Yf = np.where(Yf < 0.0, 0.0, Yf)
        YO = YO + s_stoich * dY
        YO = np.where(YO < 0.0, 0.0, YO)
        cp = (1.0 - YH) * cp_g + YH * 2000.0
        Tg = Tg + om * HoC * h / (r * cp)
        Tg = np.where(Tg > 2400.0, 2400.0, Tg)
        acc = acc + om * h
    omega = acc / dt if dt > 0.0 else np.zeros_like(acc)
    return Tg.reshape(shape), Yf.reshape(shape), YO.reshape(shape), omega.reshape(shape)


# ---------------------------------------------------------------- bed / solid / soil


def solid_conduction(T_s, alpha_s, dz, da, db, k_solid, rho_s, cp_s, dt):
    """solid_conduction_3d.py:56-127 step_solid_conduction_vertical."""
    nz = T_s.shape[0]
    out = T_s.copy()
    irc = 1.0 / (rho_s * cp_s)
    for k in range(nz):
        ac = alpha_s[k]
        fu = np.zeros_like(ac)
        fd = np.zeros_like(ac)
        if k < nz - 1:
            aa = alpha_s[k + 1]
            with np.errstate(divide="ignore", invalid="ignore"):
                ae = 2.0 * ac * aa / (ac + aa)
            fu = np.where(aa > 0.0, k_solid * ae * (T_s[k + 1] - T_s[k]) / da[k], 0.0)
        if k > 0:
            ab = alpha_s[k - 1]
            with np.errstate(divide="ignore", invalid="ignore"):
                ae = 2.0 * ac * ab / (ac + ab)
            fd = np.where(ab > 0.0, k_solid * ae * (T_s[k - 1] - T_s[k]) / db[k], 0.0)
        src = (fu + fd) / dz[k]
        with np.errstate(divide="ignore", invalid="ignore"):
            dT = dt * src * irc / ac
        out[k] = np.where(ac > 0.0, T_s[k] + dT, T_s[k])
    return out


def soil_step(T_soil, q_in, dt, sdz, sda, sdb, k_s=0.48, rho_s=1500.0, cp_s=800.0,
              eps_s=0.85, T_amb=300.0):
    """soil_3d.py:106-153 (sequential in k: cell k sees the updated cell k-1)."""
    T = T_soil.copy()
    n = T.shape[0]
    rci = 1.0 / (rho_s * cp_s)
    ida = 1.0 / np.asarray(sda)
    idb = 1.0 / np.asarray(sdb)
    for k in range(n):
        Tk = T[k].copy()
        if k == 0:
            T2 = Tk * Tk
            qt = q_in - eps_s * 5.67e-8 * (T2 * T2)
        else:
            qt = k_s * (T[k - 1] - Tk) * ida[k]
        if k == n - 1:
            qb = k_s * (Tk - T_amb) * idb[k]
        else:
            qb = k_s * (Tk - T[k + 1]) * idb[k]
        T[k] = Tk + dt * (qt - qb) * rci / sdz[k]
    return T


R_GAS = 8.314


def locate_cells(x, y, z, dx, dy, z_face, nx, ny, nz):
    """lagrangian_particles_3d.py:95-140 (int() truncation, linear k search)."""
    i = np.where(x < 0.0, -1, np.trunc(x / dx)).astype(np.int64)
    i = np.where(i >= nx, -1, i)
    j = np.where(y < 0.0, -1, np.trunc(y / dy)).astype(np.int64)
    j = np.where(j >= ny, -1, j)
    inside = (z >= z_face[0]) & (z < z_face[nz])
    k = np.searchsorted(np.asarray(z_face)[1:nz + 1], z, side="right")
    k = np.where(inside, np.minimum(k, nz - 1), -1)
    return i, j, k


def bed_step(P, T_g, Y_O2, Q_ext, n_split, dx, dy, dz, z_face, h_conv, rho_true, cp_solid,
             eps_solid, T_amb, view, geometric, h_bed, kappa_bed, dt, mode, char_cap,
             ash_exp, do_dry=True, do_pyro=True, do_char=True, do_smold=True):
    """lagrangian_bed_3d.py:594-1070 step_bed_particles.

    P: dict of particle arrays (modified in place).  Returns the eight
    per-cell source grids accumulated in slot order.
    """
    nz, ny, nx = T_g.shape
    src = {k: np.zeros(T_g.shape) for k in ("S_pyro", "S_drying", "Q_pyro", "Q_drying",
                                             "Y_F_source", "Q_char", "Q_smold", "Q_g_conv")}
    alive = P["alive"] != 0
    i, j, k = locate_cells(P["x"], P["y"], P["z"], dx, dy, z_face, nx, ny, nz)
    out = alive & ((i < 0) | (j < 0) | (k < 0))
    P["alive"][out] = 0
    act = np.nonzero(alive & ~out)[0]
    if act.size == 0:
        return src
    ii, jj, kk = i[act], j[act], k[act]
    cell = (kk * ny + jj) * nx + ii
    V = dx * dy * np.asarray(dz)[kk]
    Ts = P["T_s"][act].copy()
    Tg = T_g.ravel()[cell]
    YO = Y_O2.ravel()[cell]
    ms = P["m_solid"][act].copy()
    mw = P["m_water"][act].copy()
    mc = P["m_char"][act].copy()
    mw0 = P["m_water_0"][act]
    sav = P["sav"][act]
    mcmax = P["m_char_max"][act].copy()
    inv_dt = 1.0 / dt if dt > 0.0 else 0.0
    # (1) drying
    dm_evap = np.zeros_like(Ts)
    if do_dry and mode in (0, 2):
        A, E = (4.29e3, 43800.0) if mode == 0 else (4.29e3, 30000.0)
        sel = (mw > 0.0) & (Ts > 0.0)
        with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
            kd = A * np.exp(-E / (R_GAS * Ts))
            mwn = mw * np.exp(-kd * dt)
        dm_evap = np.where(sel, mw - mwn, 0.0)
        mw = np.where(sel, mwn, mw)
    # (2) pyrolysis
    rate = np.zeros_like(Ts)
    f_th = np.ones_like(Ts)
    f_op = np.zeros_like(Ts)
    if do_pyro:
        sel = (ms > 0.0) & (Ts > 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            gate = np.where(mw0 > 0.0, np.where(1.0 - mw / mw0 < 0.0, 0.0, 1.0 - mw / mw0), 1.0)
            kth = 36280.0 * np.exp(-58600.0 / (R_GAS * Ts))
            kop = np.where(YO > 1.0e-3, 7.26e4 * np.exp(-55000.0 / (R_GAS * Ts)) * YO, 0.0)
            ktot = kth + kop
            mnew = ms * np.exp(-ktot * dt)
        go = sel & (gate > 0.0) & (ktot > 0.0)
        dm_pyro = np.where(go, (ms - mnew) * gate, 0.0)
        rate = np.where(go, dm_pyro * inv_dt, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            f_th = np.where(go, kth / ktot, 1.0)
            f_op = np.where(go, kop / ktot, 0.0)
        mc = np.where(go, mc + 0.15 * dm_pyro, mc)
        ms = np.where(go, ms - dm_pyro, ms)
        mcmax = np.where(go & (mc > mcmax), mc, mcmax)
    A_now = sav * (ms + mc) / rho_true
    # (3) char oxidation
    Q_ch = np.zeros_like(Ts)
    if do_char:
        sel = (mc > 1.0e-12) & (Ts >= 600.0) & (YO >= 1.0e-3)
        with np.errstate(over="ignore", invalid="ignore"):
            kch = 7.09e5 * np.exp(-94000.0 / (R_GAS * Ts))
        mcons = kch * mc * YO * dt
        mcons = np.where(mcons > 0.5 * mc, 0.5 * mc, mcons)
        Are = A_now
        if ash_exp > 0.0:
            with np.errstate(divide="ignore", invalid="ignore"):
                bf = np.where(mcmax > 1.0e-15, mc / np.where(mcmax > 0, mcmax, 1.0), 1.0)
            bf = np.where(bf < 0.0, 0.0, bf)
            Are = np.where(mcmax > 1.0e-15, A_now * bf ** ash_exp, A_now)
        Qcap = char_cap * Are
        Qarr = (mcons * 32000000.0) * inv_dt
        mcons = np.where(Qarr > Qcap, Qcap / (32000000.0 * inv_dt), mcons)
        Q_ch = np.where(sel, (mcons * 32000000.0) * inv_dt, 0.0)
        mc = np.where(sel, mc - mcons, mc)
    # (4) smoulder
    Q_sm = np.zeros_like(Ts)
    if do_smold:
        mav = ms + mc
        sel = (Ts >= 473.0) & (YO >= 1.0e-3) & (mav > 1.0e-12)
        with np.errstate(over="ignore", invalid="ignore"):
            ksm = 1.0e6 * np.exp(-80000.0 / (R_GAS * Ts))
        mcons = ksm * mav * YO * dt
        mcons = np.where(mcons > 0.5 * mav, 0.5 * mav, mcons)
        Qcap = 4.0e4 * A_now
        Qarr = (mcons * 28000000.0) * inv_dt
        mcons = np.where(Qarr > Qcap, Qcap / (28000000.0 * inv_dt), mcons)
        with np.errstate(divide="ignore", invalid="ignore"):
            fs = ms / mav
        ms = np.where(sel & (mav > 0.0), ms - fs * mcons, ms)
        mc = np.where(sel & (mav > 0.0), mc - (1.0 - fs) * mcons, mc)
        Q_sm = np.where(sel, (mcons * 28000000.0) * inv_dt, 0.0)
    inv_V = 1.0 / V
    eta = 1.0 - 0.15
    c_Sp = eta * rate * inv_V
    c_Sd1 = dm_evap * inv_dt * inv_V
    c_Qp = (rate * (f_th * 4.0e5 + f_op * -1.0e6)) * inv_V
    c_Qd1 = dm_evap * 2.26e6 * inv_dt * inv_V
    c_Qch = Q_ch * inv_V
    c_Qsm = Q_sm * inv_V
    # (6) T_s update
    mt = ms + mw + mc
    Qconv = np.zeros_like(Ts)
    c_Sd2 = np.zeros_like(Ts)
    c_Qd2 = np.zeros_like(Ts)
    has = mt > 0.0
    A_p = sav * (ms + mc) / rho_true
    Qconv = np.where(has, h_conv * A_p * (Tg - Ts), 0.0)
    Q_rxn = -rate * (f_th * 4.0e5 + f_op * -1.0e6)
    Q_dry = -dm_evap * 2.26e6 * inv_dt
    Q_ext = Q_ext.ravel()[cell] * V / float(n_split) if n_split > 0 else np.zeros_like(Ts)
    if geometric:
        ha = h_bed - P["z"][act]
        ha = np.where(ha < 0.0, 0.0, ha)
        fg = np.exp(-kappa_bed * ha)
    else:
        fg = np.ones_like(Ts)
    C_rad = eps_solid * 5.67e-8 * A_p * view * fg
    mcp = mt * cp_solid
    Ta4 = T_amb * T_amb * T_amb * T_amb
    Qo = Qconv + Q_rxn + Q_dry + Q_ch + Q_sm + Q_ext
    mcdt = mcp / dt
    T_old = Ts.copy()
    Ti = Ts.copy()
    for _ in range(5):
        T2 = Ti * Ti
        T3 = T2 * Ti
        T4 = T3 * Ti
        F = mcdt * (Ti - T_old) - Qo + C_rad * (T4 - Ta4)
        Fp = mcdt + 4.0 * C_rad * T3
        with np.errstate(divide="ignore", invalid="ignore"):
            Ti = Ti - F / Fp
        Ti = np.where(Ti < T_amb, T_amb, Ti)
    Tn = np.where(has, np.where(Ti > 1.0e4, 1.0e4, Ti), Ts)
    if do_dry and mode in (1, 2):
        eq = has & (mw > 0.0) & (Tn > 373.15)
        ex = mcp * (Tn - 373.15)
        dm_eq = ex / 2.26e6
        allw = dm_eq >= mw
        with np.errstate(divide="ignore", invalid="ignore"):
            T_all = 373.15 + np.where(mcp > 0.0, (ex - mw * 2.26e6) / mcp, 0.0)
        dm_eq = np.where(allw, mw, dm_eq)
        Tn = np.where(eq, np.where(allw, T_all, 373.15), Tn)
        mw = np.where(eq, np.where(allw, 0.0, mw - dm_eq), mw)
        c_Sd2 = np.where(eq, dm_eq * inv_dt * inv_V, 0.0)
        c_Qd2 = np.where(eq, dm_eq * 2.26e6 * inv_dt * inv_V, 0.0)
    c_Qgc = Qconv * inv_V
    P["T_s"][act] = Tn
    P["m_solid"][act] = ms
    P["m_water"][act] = mw
    P["m_char"][act] = mc
    P["m_char_max"][act] = mcmax
    dead = mt < 1.0e-8
    P["alive"][act[dead]] = 0
    # deposition in slot order (np.add.at applies repeated indices sequentially)
    for key, contrib in (("S_pyro", c_Sp), ("Q_pyro", c_Qp), ("Y_F_source", c_Sp),
                         ("Q_char", c_Qch), ("Q_smold", c_Qsm), ("Q_g_conv", c_Qgc)):
        np.add.at(src[key].reshape(-1), cell, contrib)
    cell2 = np.repeat(cell, 2)
    for key, a, b in (("S_drying", c_Sd1, c_Sd2), ("Q_drying", c_Qd1, c_Qd2)):
        inter = np.empty(2 * a.size)
        inter[0::2] = a
        inter[1::2] = b
        np.add.at(src[key].reshape(-1), cell2, inter)
    return src


def bed_aggregate(P, shape, dx, dy, z_face, out=None, mode=0):
    """lagrangian_bed_3d.py:501-546 (mode 0: mass-weighted T_s, cells without
    particles keep ``out``) and :550-590 (mode 1: M_local, empty cells 0)."""
    nz, ny, nx = shape
    i, j, k = locate_cells(P["x"], P["y"], P["z"], dx, dy, z_face, nx, ny, nz)
    ok = (P["alive"] != 0) & (i >= 0) & (j >= 0) & (k >= 0)
    num = np.zeros(nz * ny * nx)
    den = np.zeros(nz * ny * nx)
    if mode == 0:
        mt = P["m_solid"] + P["m_water"] + P["m_char"]
        ok &= mt > 0.0
        cell = ((k * ny + j) * nx + i)[ok]
        np.add.at(num, cell, (P["T_s"] * mt)[ok])
        np.add.at(den, cell, mt[ok])
        res = out.copy().ravel()
        with np.errstate(divide="ignore", invalid="ignore"):
            res = np.where(den > 0.0, num / np.where(den > 0, den, 1.0), res)
        return res.reshape(shape)
    cell = ((k * ny + j) * nx + i)[ok]
    np.add.at(num, cell, P["m_water"][ok])
    np.add.at(den, cell, P["m_solid"][ok])
    with np.errstate(divide="ignore", invalid="ignore"):
        res = np.where(den > 0.0, num / np.where(den > 0, den, 1.0), 0.0)
    return res.reshape(shape)


def bed_hcond(P, T_grid, alpha_s, dx, dy, z_face, k_solid, rho_true, cp_solid, n_z_bed, dt):
    """lagrangian_bed_3d.py:428-497; returns the new T_s grid (particles updated)."""
    nz, ny, nx = T_grid.shape
    old = T_grid.copy()
    new = T_grid.copy()
    delta = np.zeros_like(T_grid)
    diff = k_solid / (rho_true * cp_solid)
    nzb = min(n_z_bed, nz)
    a = alpha_s[:nzb]
    T = old[:nzb]
    fuel = a > 0.0
    Txp = np.where(np.concatenate([fuel[:, :, 1:], np.zeros_like(fuel[:, :, :1])], axis=2),
                   nb(T, 1, 2), T)
    Txm = np.where(np.concatenate([np.zeros_like(fuel[:, :, :1]), fuel[:, :, :-1]], axis=2),
                   nb(T, -1, 2), T)
    Typ = np.where(np.roll(fuel, -1, axis=1), np.roll(T, -1, axis=1), T)
    Tym = np.where(np.roll(fuel, 1, axis=1), np.roll(T, 1, axis=1), T)
    lap = (Txp - 2.0 * T + Txm) * (1.0 / (dx * dx)) + (Typ - 2.0 * T + Tym) * (1.0 / (dy * dy))
    dT = diff * lap * dt
    new[:nzb] = np.where(fuel, T + dT, T)
    delta[:nzb] = np.where(fuel, dT, 0.0)
    i, j, k = locate_cells(P["x"], P["y"], P["z"], dx, dy, z_face, nx, ny, nz)
    ok = (P["alive"] != 0) & (i >= 0) & (j >= 0) & (k >= 0) & (k < n_z_bed)
    P["T_s"][ok] += delta[k[ok], j[ok], i[ok]]
    return new


# ---------------------------------------------------------------- radiation


def dom_solve(I_set, Omega, wts, T_s, T_g, alpha_s, omega, sigma, T_amb, dx, dy, dz,
              T_soil0=None, Y_H2O=None, rho=None, M_local=None, kappa_gas_max=0.5,
              eps_w=0.85, max_iter=30, tol=1.0e-3, relax=0.7):
    """dom_3d.py:286-473 DOMRadiationSolver.solve (periodic y).

    I_set (M, Nz, Ny, Nx) persists between calls and is updated in place.
    The sweep of each octant visits hyperplanes i'+j'+k' = d of the flipped
    grid; the y-periodic inflow of the first row reads the previous sweep's
    value (dom_3d.py:184-195).  Returns (q_rad, q_rad_gas, q_in_soil, iters).
    """
    nz, ny, nx = T_s.shape
    ks = sigma * alpha_s
    if M_local is not None:
        ks = ks * (1.0 + 5.0 * M_local)
    of = np.clip(omega / 1.0e-3, 0.0, 1.0)
    tf = np.clip((T_g - 600.0) / 400.0, 0.0, 1.0)
    kg = kappa_gas_max * np.maximum(of, tf)
    if Y_H2O is not None and rho is not None:
        kg = kg + 30.0 * rho * Y_H2O
    kap = ks + kg
    ksafe = np.maximum(kap, 1.0e-3)
    kft = np.where(kap > 1.0e-9, ksafe, 1.0)
    T4 = np.where(kap > 1.0e-9, (ks * T_s ** 4 + kg * T_g ** 4) / kft, T_amb ** 4)
    B = 5.67e-8 * T4 / math.pi
    I_amb = 5.67e-8 * T_amb ** 4 / math.pi
    if T_soil0 is not None:
        Isoil = eps_w * 5.67e-8 * T_soil0 ** 4 / math.pi
    else:
        Isoil = np.full((ny, nx), eps_w * I_amb)
    Ig = Isoil.copy()
    M = Omega.shape[0]
    dzc = np.asarray(dz, dtype=np.float64)
    kB = ksafe * B
    G = np.zeros_like(T_s)
    Gp = None
    qin = np.zeros((ny, nx))
    it_done = 0
    # plane index lists in sweep coordinates
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    dsum = (kk + jj + ii).ravel()
    order = np.argsort(dsum, kind="stable")
    bounds = np.searchsorted(dsum[order], np.arange(nx + ny + nz))
    planes = [order[bounds[d]:bounds[d + 1]] for d in range(nx + ny + nz - 2)]
    groups = {}
    for n in range(M):
        sg = (Omega[n, 0] >= 0.0, Omega[n, 1] >= 0.0, Omega[n, 2] >= 0.0)
        groups.setdefault(sg, []).append(n)
    for it in range(max_iter):
        Gp = G
        for (sx, sy, sz), ns in groups.items():
            ns = np.array(ns)
            # flip into sweep coordinates
            fl = tuple(ax for ax, s in zip((0, 1, 2), (sz, sy, sx)) if not s)
            Iv = np.flip(I_set[ns], axis=tuple(a + 1 for a in fl)).copy() if fl else I_set[ns].copy()
            kf = np.flip(ksafe, axis=fl) if fl else ksafe
            kbf = np.flip(kB, axis=fl) if fl else kB
            dzf = dzc[::-1] if not sz else dzc
            igf = np.flip(Ig, axis=tuple(a - 1 for a in fl if a > 0)) if any(a > 0 for a in fl) else Ig
            ax = np.abs(Omega[ns, 0]) / dx
            ay = np.abs(Omega[ns, 1]) / dy
            az = np.abs(Omega[ns, 2])
            mus = Omega[ns, 2]
            Ivf = Iv.reshape(len(ns), -1)
            for pl in planes:
                k = kk.ravel()[pl]; j = jj.ravel()[pl]; i = ii.ravel()[pl]
                Ix = np.where(i > 0, Iv[:, k, j, np.maximum(i - 1, 0)], I_amb)
                Iy = np.where(j > 0, Iv[:, k, np.maximum(j - 1, 0), i], Iv[:, k, ny - 1, i])
                gin = np.where(mus[:, None] > 0.0, igf[j, i][None, :], 0.0)
                Iz = np.where(k > 0, Iv[:, np.maximum(k - 1, 0), j, i], gin) if sz else \
                    np.where(k > 0, Iv[:, np.maximum(k - 1, 0), j, i], I_amb)
                izk = az[:, None] / dzf[k][None, :]
                kc = kf[k, j, i][None, :]
                num = kbf[k, j, i][None, :] + ax[:, None] * Ix + ay[:, None] * Iy + izk * Iz
                den = kc + ax[:, None] + ay[:, None] + izk
                Iv[:, k, j, i] = num / den
            I_set[ns] = np.flip(Iv, axis=tuple(a + 1 for a in fl)) if fl else Iv
        G = np.zeros_like(T_s)
        for n in range(M):
            G = G + wts[n] * I_set[n]
        qin = np.zeros((ny, nx))
        for n in range(M):
            mu = Omega[n, 2]
            if mu < 0:
                qin = qin + wts[n] * abs(mu) * I_set[n, 0]
        Inew = Isoil + (1.0 - eps_w) / math.pi * qin
        Ig = relax * Inew + (1.0 - relax) * Ig
        it_done = it + 1
        if it > 0:
            Gm = max(float(G.max()), 1e-12)
            err = float(np.abs(G - Gp).max()) / Gm
            if err < tol:
                break
    net = kap * (G - 4.0 * math.pi * B) * dzc.reshape(-1, 1, 1)
    fs = np.where(kap > 1.0e-9, ks / ksafe, 0.0)
    fgas = np.where(kap > 1.0e-9, kg / ksafe, 0.0)
    return net * fs, net * fgas, eps_w * qin, it_done


# ---------------------------------------------------------------- projection


def poisson_matrix(rho, dx, dy, dz, da, db, eps_reg=1.0e-6):
    """projection_3d.py:66-175 _fill_var_density_data (alpha_g = 1) as CSR."""
    import scipy.sparse as sp
    nz, ny, nx = rho.shape
    ir = 1.0 / np.maximum(rho, 0.01)
    n = rho.size
    idx = np.arange(n).reshape(rho.shape)
    rows, cols, vals = [], [], []
    diag = np.full(rho.shape, eps_reg)
    dx2, dy2 = dx * dx, dy * dy
    # x
    cxp = (0.5 * (ir[:, :, :-1] + ir[:, :, 1:])) / dx2
    diag[:, :, :-1] -= cxp
    diag[:, :, 1:] -= cxp
    rows += [idx[:, :, :-1].ravel(), idx[:, :, 1:].ravel()]
    cols += [idx[:, :, 1:].ravel(), idx[:, :, :-1].ravel()]
    vals += [cxp.ravel(), cxp.ravel()]
    diag[:, :, -1] -= (2.0 * ir[:, :, -1]) / dx2
    if ny > 1:
        cyp = (0.5 * (ir + np.roll(ir, -1, axis=1))) / dy2
        diag -= cyp
        diag -= np.roll(cyp, 1, axis=1)
        rows += [idx.ravel(), np.roll(idx, -1, axis=1).ravel()]
        cols += [np.roll(idx, -1, axis=1).ravel(), idx.ravel()]
        vals += [cyp.ravel(), cyp.ravel()]
    idz = 1.0 / np.asarray(dz)
    da_, db_ = np.asarray(da), np.asarray(db)
    irz = 0.5 * (ir[:-1] + ir[1:])
    czp = irz * idz[:-1, None, None] / da_[:-1, None, None]
    czm = irz * idz[1:, None, None] / db_[1:, None, None]
    diag[:-1] -= czp
    diag[1:] -= czm
    rows += [idx[:-1].ravel(), idx[1:].ravel()]
    cols += [idx[1:].ravel(), idx[:-1].ravel()]
    vals += [czp.ravel(), czm.ravel()]
    diag[-1] -= 2.0 * ir[-1] * idz[-1] * idz[-1]
    rows.append(idx.ravel()); cols.append(idx.ravel()); vals.append(diag.ravel())
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    return A, ir


def divergence(u, v, w, dx, dy, dz, u_in):
    """projection_3d.py:847-892 _divergence_compatible (plain branch)."""
    div = np.zeros_like(u)
    div[:, :, 1:] += (u[:, :, 1:] - u[:, :, :-1]) / dx
    div[:, :, 0] += (u[:, :, 0] - u_in) / dx
    if u.shape[1] > 1:
        div += (v - np.roll(v, 1, axis=1)) / dy
    dzk = np.asarray(dz).reshape(-1, 1, 1)
    div[1:] += (w[1:] - w[:-1]) / dzk[1:]
    div[0] += (w[0] - 0.0) / dzk[0]
    return div


class SeparablePoisson:
    """Exact inverse of the constant-coefficient operator, used by the
    reference as the Krylov preconditioner (fft_poisson_3d.py:45-228):
    eigen-decompositions of the 1D x and (sqrt(dz)-symmetrised) z Laplacians,
    FFT along periodic y."""

    def __init__(self, nz, ny, nx, dx, dy, dz, da, db, eps_reg=1.0e-6):
        from scipy.linalg import eigh
        dz = np.asarray(dz, dtype=np.float64)
        Lx = np.zeros((nx, nx))
        c = 1.0 / (dx * dx)
        for i in range(nx):
            if 0 < i < nx - 1:
                Lx[i, i], Lx[i, i + 1], Lx[i, i - 1] = -2.0 * c, c, c
            elif i == 0:
                Lx[0, 0], Lx[0, 1] = -c, c
            else:
                Lx[i, i], Lx[i, i - 1] = -3.0 * c, c
        Lz = np.zeros((nz, nz))
        for k in range(nz):
            idz = 1.0 / dz[k]
            if 0 < k < nz - 1:
                ca, cb = idz / da[k], idz / db[k]
                Lz[k, k], Lz[k, k + 1], Lz[k, k - 1] = -ca - cb, ca, cb
            elif k == 0:
                ca = idz / da[0]
                Lz[0, 0], Lz[0, 1] = -ca, ca
            else:
                cb = idz / db[k]
                Lz[k, k], Lz[k, k - 1] = -2.0 * idz * idz - cb, cb
        D = np.sqrt(dz)
        lx, self.Ux = eigh(Lx)
        lz, self.Uz = eigh((D[:, None] * Lz) / D[None, :])
        ly = (2.0 / (dy * dy)) * (np.cos(2.0 * np.pi * np.arange(ny) / ny) - 1.0)
        self.inv = 1.0 / (lz[:, None, None] + ly[None, :, None] + lx[None, None, :] - eps_reg)
        self.D = D
        self.shape = (nz, ny, nx)

    def solve(self, r):
        nz, ny, nx = self.shape
        q = r.reshape(self.shape) * self.D[:, None, None]
        q = (q.reshape(nz * ny, nx) @ self.Ux).reshape(self.shape)
        q = np.fft.fft(q, axis=1)
        q = (self.Uz.T @ q.reshape(nz, ny * nx)).reshape(self.shape) * self.inv
        q = (self.Uz @ q.reshape(nz, ny * nx)).reshape(self.shape)
        q = np.fft.ifft(q, axis=1).real
        q = (q.reshape(nz * ny, nx) @ self.Ux.T).reshape(self.shape)
        return (q / self.D[:, None, None]).reshape(-1)


def project(u, v, w, rho, dt, div_target, dx, dy, dz, da, db, u_in, solver="direct",
            rtol=1.0e-6, x0=None, precond=None):
    """projection_3d.py:677-844 project.  ``solver='direct'`` solves the
    Poisson system exactly (what the reference's BiCGSTAB reaches at tight
    tolerance); ``'bicgstab'`` is the reference's own iteration (scipy
    BiCGSTAB, warm start x0, separable preconditioner, rtol).
    Returns (u, v, w, p)."""
    import scipy.sparse.linalg as spla
    A, ir = poisson_matrix(rho, dx, dy, dz, da, db)
    div = divergence(u, v, w, dx, dy, dz, u_in)
    if div_target is not None:
        div = div - div_target
    rhs = (div / dt).reshape(-1)
    if solver == "direct":
        p = spla.spsolve(A.tocsc(), rhs).reshape(u.shape)
    else:
        nz, ny, nx = u.shape
        pre = precond or SeparablePoisson(nz, ny, nx, dx, dy, dz, da, db)
        M = spla.LinearOperator(A.shape, matvec=pre.solve)
        p, info = spla.bicgstab(A, rhs, x0=x0, M=M, rtol=rtol, maxiter=200)
        if info != 0:
            raise RuntimeError(f"BiCGSTAB did not converge (info={info})")
        p = p.reshape(u.shape)
    u = u.copy(); v = v.copy(); w = w.copy()
    nz, ny, nx = u.shape
    if nx > 2:
        u[:, :, :-1] -= dt * (p[:, :, 1:] - p[:, :, :-1]) / dx * (0.5 * (ir[:, :, :-1] + ir[:, :, 1:]))
        u[:, :, -1] += 2.0 * dt * p[:, :, -1] / dx * ir[:, :, -1]
    if ny > 1:
        v -= dt * (np.roll(p, -1, axis=1) - p) / dy * (0.5 * (ir + np.roll(ir, -1, axis=1)))
    if nz > 2:
        dac = np.asarray(da)[:-1].reshape(-1, 1, 1)
        w[:-1] -= dt * (p[1:] - p[:-1]) / dac * (0.5 * (ir[:-1] + ir[1:]))
        w[-1] += 2.0 * dt * p[-1] / dz[-1] * ir[-1]
    return u, v, w, p


# ---------------------------------------------------------------- level set


def _ls_inv_dz(dz):
    nz = len(dz)
    im = np.empty(nz); ip = np.empty(nz)
    for k in range(nz):
        if k == 0:
            im[k] = 1.0 / dz[0]
            ip[k] = 2.0 / (dz[0] + dz[1]) if nz > 1 else 1.0 / dz[0]
        elif k == nz - 1:
            ip[k] = 1.0 / dz[nz - 1]
            im[k] = 2.0 / (dz[nz - 1] + dz[nz - 2])
        else:
            im[k] = 2.0 / (dz[k] + dz[k - 1])
            ip[k] = 2.0 / (dz[k] + dz[k + 1])
    return _kcol(im), _kcol(ip)


def godunov_grad(phi, dx, dy, dz, sign=None):
    """flame_front_3d.py:114-188 (sign None) and :192-263 (sign = sign(phi_0))."""
    nz, ny, nx = phi.shape
    im, ip = _ls_inv_dz(dz)
    dmx = np.zeros_like(phi); dpx = np.zeros_like(phi)
    dmx[:, :, 1:] = (phi[:, :, 1:] - phi[:, :, :-1]) * (1.0 / dx)
    dpx[:, :, :-1] = (phi[:, :, 1:] - phi[:, :, :-1]) * (1.0 / dx)
    dmy = (phi - np.roll(phi, 1, axis=1)) * (1.0 / dy)
    dpy = (np.roll(phi, -1, axis=1) - phi) * (1.0 / dy)
    dmz = np.zeros_like(phi); dpz = np.zeros_like(phi)
    dmz[1:] = (phi[1:] - phi[:-1]) * im[1:]
    dpz[:-1] = (phi[1:] - phi[:-1]) * ip[:-1]
    fwd = np.ones(phi.shape, dtype=bool) if sign is None else sign > 0.0
    a = np.where(fwd, np.maximum(dmx, 0.0), np.minimum(dmx, 0.0))
    b = np.where(fwd, np.minimum(dpx, 0.0), np.maximum(dpx, 0.0))
    c = np.where(fwd, np.maximum(dmy, 0.0), np.minimum(dmy, 0.0))
    d = np.where(fwd, np.minimum(dpy, 0.0), np.maximum(dpy, 0.0))
    e = np.where(fwd, np.maximum(dmz, 0.0), np.minimum(dmz, 0.0))
    f = np.where(fwd, np.minimum(dpz, 0.0), np.maximum(dpz, 0.0))
    return np.sqrt(a * a + b * b + c * c + d * d + e * e + f * f)


def levelset_reinit(phi, dx, dy, dz):
    """flame_front_3d.py:339-355 LevelSetFront3D.reinitialize."""
    phi0 = phi.copy()
    s = np.where(phi0 > 0.0, 1.0, np.where(phi0 < 0.0, -1.0, 0.0))
    dtau = 0.5 * min(dx, dy, float(np.min(dz)))
    for _ in range(5):
        g = godunov_grad(phi, dx, dy, dz, sign=s)
        phi = phi - dtau * s * (g - 1.0)
    return phi


def front_x(phi, k, j, dx):
    """flame_front_3d.py:391-403 LevelSetFront3D.front_x."""
    row = phi[k, j]
    for i in range(row.size - 1):
        a, b = row[i], row[i + 1]
        if a < 0.0 < b or b < 0.0 < a:
            return (i + (-a / (b - a)) + 0.5) * dx
    return float("inf")


def active_flame(omega, T_g, Y_F):
    """flame_front_3d.py:756-813: active cells == (phi_flame <= 0)."""
    return (omega > 1.0e-3) | ((T_g > 1000.0) & (Y_F > 1.0e-3))
