"""Discrete-ordinate quadrature sets for the DOM radiation solve.

S4 reproduces the reference's table exactly (``dom_3d.py:98-142``): the
Lathrop-Carlson S4 direction cosines with equal weights, reflected into the 8
octants in the reference's octant order.  The order of ordinates matters for
parity because G = sum_n w_n I_n is accumulated in ordinate order.

S8 does not exist in the reference (``_generate_sn_ordinates`` raises for
N != 4).  It is derived here from the level-symmetric construction instead of
being typed from a table:

* N/2 levels with mu_i^2 = mu_1^2 + (i-1) * 2 (1 - 3 mu_1^2) / (N - 2);
* points (mu_i, mu_j, mu_k) with i + j + k = N/2 + 2 (1-based), 10 per octant;
* one weight per permutation class, fixed by exact integration of the even
  moments <1>, <mu^4>, <mu^6> over the octant (<mu^2> = 1/3 follows from
  mu_x^2 + mu_y^2 + mu_z^2 = 1);
* mu_1 is the root of the remaining <mu^8> = 1/9 condition.

This yields the LQ8 set (mu_1 = sqrt(1/21)) with weights summing to 4 pi.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

# Octant sign order of the reference's reflection loop (dom_3d.py:129-133).
OCTANTS = [
    (1, 1, 1), (1, 1, -1), (1, -1, 1), (-1, 1, 1),
    (1, -1, -1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1),
]

# Reference S4 first-octant direction cosines (dom_3d.py:106-113).
_S4_MU1 = 0.295876
_S4_MU2 = 0.908248


def _ls_points(mu1: float, n_order: int):
    n = n_order // 2
    d = 2.0 * (1.0 - 3.0 * mu1 * mu1) / (n_order - 2)
    mu = np.sqrt(mu1 * mu1 + np.arange(n) * d)
    pts, cls = [], []
    for i, j, k in itertools.product(range(n), repeat=3):
        if i + j + k == n - 1:
            pts.append((mu[i], mu[j], mu[k]))
            cls.append(tuple(sorted((i, j, k))))
    return np.array(pts), cls


def _ls_weights(mu1: float, n_order: int):
    pts, cls = _ls_points(mu1, n_order)
    uniq = sorted(set(cls))
    idx = np.array([uniq.index(c) for c in cls])
    x = pts[:, 0]
    powers = [0] + list(range(4, 4 + 2 * (len(uniq) - 1), 2))
    A = np.array([[(x ** p)[idx == c].sum() for c in range(len(uniq))] for p in powers])
    b = np.array([1.0 / (p + 1) for p in powers])
    w = np.linalg.solve(A, b)
    return pts, w[idx]


def _solve_mu1(n_order: int) -> float:
    """Root of the first unmatched even moment, bracketed on (0.05, 0.55)."""
    n_cls = len(set(_ls_points(0.3, n_order)[1]))
    p_extra = 4 + 2 * (n_cls - 1)

    def f(m):
        pts, w = _ls_weights(m, n_order)
        return float((w * pts[:, 0] ** p_extra).sum() - 1.0 / (p_extra + 1))

    a, b = 0.05, 0.55
    grid = np.linspace(a, b, 101)
    vals = [f(g) for g in grid]
    for g0, g1, v0, v1 in zip(grid[:-1], grid[1:], vals[:-1], vals[1:]):
        if v0 == 0.0:
            return float(g0)
        if v0 * v1 < 0.0:
            lo, hi, flo = g0, g1, v0
            for _ in range(200):
                mid = 0.5 * (lo + hi)
                fm = f(mid)
                if fm == 0.0 or hi - lo < 1e-16:
                    return mid
                if flo * fm < 0.0:
                    hi = mid
                else:
                    lo, flo = mid, fm
            return 0.5 * (lo + hi)
    raise ValueError(f"no level-symmetric S{n_order} root found")


def level_symmetric(n_order: int):
    """Return ``(Omega, w)``: (M, 3) direction cosines and (M,) weights summing to 4 pi."""
    if n_order == 4:
        per_oct = np.array([(_S4_MU1, _S4_MU1, _S4_MU2),
                            (_S4_MU1, _S4_MU2, _S4_MU1),
                            (_S4_MU2, _S4_MU1, _S4_MU1)])
        w_oct = None
    elif n_order in (6, 8):
        mu1 = _solve_mu1(n_order)
        per_oct, w_oct = _ls_weights(mu1, n_order)
    else:
        raise NotImplementedError(f"S{n_order} quadrature is not provided")
    om = []
    ws = []
    for sx, sy, sz in OCTANTS:
        for p, o in enumerate(per_oct):
            om.append((sx * o[0], sy * o[1], sz * o[2]))
            if w_oct is not None:
                ws.append(w_oct[p] * (4.0 * math.pi / 8.0))
    om = np.array(om, dtype=np.float64)
    if w_oct is None:
        w = np.full(om.shape[0], 4.0 * math.pi / om.shape[0], dtype=np.float64)
    else:
        w = np.array(ws, dtype=np.float64)
    return om, w
