"""Plain Roe shallow-water step restated in NumPy float64 (oracle; test infrastructure).

Follows PyExner src/PyExner/solvers/kernels/roe.py:13-315 and
src/PyExner/solvers/roe_solver.py:40-60.  A state is a dict of planes h, hu, hv, z, n
(ring included).  Dry cells are set to h = 0 here (not clamped), so a face whose two
cells are both dry divides by zero exactly as the reference does.
"""
from __future__ import annotations

import numpy as np

from .roe_exner import DRY_TOL, G_ACC, NORMAL_X, NORMAL_Y, VEL_TOL, _pairs, _rotate, _rotate_back

FIELDS = ("h", "hu", "hv", "z", "n")


def roe_face(si, sj, normal, dx):
    """Roe fluctuations with the wet/dry thrust and the beta limiter (roe.py:32-249).

    ``si``/``sj`` = (h, hu, hv, z, n).  Returns (upwP, upwM) in (h, hu, hv) order.
    """
    hi, hui, hvi, zi, ni = si
    hj, huj, hvj, zj, nj = sj
    hi = np.where(hi > DRY_TOL, hi, 0.0)
    hj = np.where(hj > DRY_TOL, hj, 0.0)
    with np.errstate(all="ignore"):
        sqi = np.sqrt(hi)
        sqj = np.sqrt(hj)
        ui = np.where(hi > 0.0, hui / hi, 0.0)
        vi = np.where(hi > 0.0, hvi / hi, 0.0)
        uj = np.where(hj > 0.0, huj / hj, 0.0)
        vj = np.where(hj > 0.0, hvj / hj, 0.0)
        uhi, vhi = _rotate(ui, vi, normal)
        uhj, vhj = _rotate(uj, vj, normal)
        ht = np.where(0.5 * (hi + hj) > DRY_TOL, 0.5 * (hi + hj), 0.0)
        ct = np.sqrt(G_ACC * ht)
        ut = (uhi * sqi + uhj * sqj) / (sqi + sqj)
        vt = (vhi * sqi + vhj * sqj) / (sqi + sqj)
        l1 = ut - ct
        l2 = ut
        l3 = ut + ct
        # Harten-Hyman (roe.py:77-92): the fixed speed replaces lambda first, and the
        # entropy speed is formed from the replaced value.
        ei = uhi - np.sqrt(G_ACC * hi)
        ej = uhj - np.sqrt(G_ACC * hj)
        m1 = (ei < 0.0) & (ej > 0.0)
        l1 = np.where(m1, ei * (ej - l1) / ((ej - ei) + VEL_TOL), l1)
        lE1 = np.where(m1, l1 - ei * (ej - l1) / ((ej - ei) + VEL_TOL), 0.0)
        ei = uhi + np.sqrt(G_ACC * hi)
        ej = uhj + np.sqrt(G_ACC * hj)
        m3 = (ei < 0.0) & (ej > 0.0)
        l3 = np.where(m3, ej * (l3 - ei) / ((ej - ei) + VEL_TOL), l3)
        lE3 = np.where(m3, l3 - ej * (l3 - ei) / ((ej - ei) + VEL_TOL), 0.0)
        den = l1 - l3 + VEL_TOL
        # rows of P^-1 (roe.py:109-113)
        p00 = -l3 / den
        p01 = np.ones_like(ut) / den
        p10 = -vt / ct
        p12 = np.ones_like(ut) / ct
        p20 = l1 / den
        p21 = -np.ones_like(ut) / den
        dh = hj - hi
        dhu = hj * uhj - hi * uhi
        dhv = hj * vhj - hi * vhi
        # alphas = P^-1 dU accumulated over the inner index in order (roe.py:127)
        a1 = p00 * dh + p01 * dhu + 0.0 * dhv
        a2 = p10 * dh + 0.0 * dhu + p12 * dhv
        a3 = p20 * dh + p21 * dhu + 0.0 * dhv
        dz = zj - zi
        di = hi + zi
        dj = hj + zj
        dd = dj - di
        thrust_a = -G_ACC * ht * dz
        mask1 = (dz >= 0) & (di < zj)
        mask2 = (dz < 0) & (dj < zi)
        dzt = np.where(mask1, hi, np.where(mask2, hj, dz))
        hr = np.where(dz >= 0, hi, hj)
        thrust_b = -G_ACC * (hr - 0.5 * np.abs(dzt)) * dzt
        mthr = (dz * dd >= 0.0) & (ut * dz > 0.0)
        thrust = np.where(mthr, np.maximum(thrust_a, thrust_b), thrust_b)
        nt = 0.5 * (ni + nj)
        sf = (nt**2 * np.sqrt(ut**2 + vt**2) * ut) / (np.maximum(DRY_TOL, ht ** (4 / 3)))
        tau = G_ACC * ht * sf * dx
        T1 = thrust - tau
        # betas = P^-1 (0, T1, 0) (roe.py:159-165)
        b1 = p00 * 0.0 + p01 * T1 + 0.0 * 0.0
        b3 = p20 * 0.0 + p21 * T1 + 0.0 * 0.0
        b2 = p10 * 0.0 + 0.0 * T1 + p12 * 0.0
        hs1 = hi + a1 - (b1 / l1)
        hs3 = hj - a3 + (b3 / l3)
        b1min = -(hi + a1) * np.abs(l1)
        b3min = -(hi - a1) * np.abs(l3)
        dtf = dx / np.maximum(np.maximum(np.abs(l1), np.abs(l2)), np.abs(l3))
        dt1s = (dx / 2 * l1) * (hi / (hi - hs1 + VEL_TOL))
        dt3s = (dx / 2 * l3) * (hj / (hj - hs3 + VEL_TOL))
        m = (hs1 < 0.0) & (hs3 > 0.0) & (dt1s < dtf)
        b1 = np.where(m, np.where(-b1min >= b3min, b1min, b1), b1)
        b3 = np.where(m, -b1, b3)
        m = (hs1 > 0.0) & (hs3 < 0.0) & (dt3s < dtf)
        b3 = np.where(m, np.where(-b3min >= b3min, b1min, b3), b3)
        b1 = np.where(m, -b3, b1)
        mk1 = (hi < DRY_TOL) & (hs1 < 0.0)
        mk2 = (hj < DRY_TOL) & (hs3 < 0.0)
        zeros = np.zeros_like(ut)
        lam = (l1, l2, l3)
        alp = (a1, a2, a3)
        bet = (b1, b2, b3)
        P = ((1.0, l1, vt), (zeros, zeros, ct), (1.0, l3, vt))
        pos = [zeros, zeros, zeros]
        neg = [zeros, zeros, zeros]
        for k in range(3):
            w = lam[k] * alp[k] - bet[k]
            for r in range(3):
                f = w * P[k][r]
                pos[r] = pos[r] + np.where(mk2, 0.0, np.where(mk1, f, np.where(lam[k] > 0.0, f, 0.0)))
                neg[r] = neg[r] + np.where(mk2, f, np.where(mk1, 0.0, np.where(lam[k] <= 0.0, f, 0.0)))
        lamE = (lE1, zeros, lE3)
        for k in range(3):
            for r in range(3):
                f = lamE[k] * alp[k] * P[k][r]
                pos[r] = pos[r] + np.where(lamE[k] > 0.0, f, 0.0)
                neg[r] = neg[r] + np.where(lamE[k] <= 0.0, f, 0.0)
    return _rotate_back(*pos, normal), _rotate_back(*neg, normal)


def hydro_update(st, dt, dx):
    """``roe_solve_2D`` (roe.py:251-315): every face, no activity mask."""
    arrs = tuple(st[f] for f in FIELDS)
    ny, nx = st["h"].shape
    flux = [np.zeros((ny, nx)) for _ in range(3)]
    res = {}
    for axis, normal in ((1, NORMAL_X), (0, NORMAL_Y)):
        si, sj = _pairs(arrs, axis)
        res[axis] = roe_face(si, sj, normal, dx)
    for r in range(3):
        flux[r][:, :-1] += res[1][1][r]
        flux[r][:, 1:] += res[1][0][r]
        flux[r][:-1, :] += res[0][1][r]
        flux[r][1:, :] += res[0][0][r]
    return (st["h"] - dt * flux[0] / dx, st["hu"] - dt * flux[1] / dx, st["hv"] - dt * flux[2] / dx)


def stage(st, dt, dx, bcs):
    """``step_fn_roe`` (roe_solver.py:40-54): update, then the boundary handlers."""
    st = dict(st)
    h, hu, hv = hydro_update(st, dt, dx)
    st.update(h=h, hu=hu, hv=hv)
    return bcs.apply(st)


def compute_dt(st, cfl, dx):
    """``compute_dt_roe`` (roe_solver.py:56-60 with roe.py:13-30).

    The interior mask is applied after the minimum, so every cell (ring included)
    counts; there is no lower floor.
    """
    wet = st["h"] > DRY_TOL
    h = np.where(wet, st["h"], 0.0)
    hv = np.where(wet, st["hv"], 0.0)
    hu = np.where(wet, st["hu"], 0.0)
    u = hu / (h + DRY_TOL)
    v = hv / (h + DRY_TOL)
    c = np.sqrt(G_ACC * h)
    dtx = np.min(dx / (np.abs(u) + c + VEL_TOL))
    dty = np.min(dx / (np.abs(v) + c + VEL_TOL))
    return cfl * np.minimum(dtx, dty)
