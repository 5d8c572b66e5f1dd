"""Transposes of the linear passes of the dry iteration, in numpy: the in-loop 4th-order Shapiro
filter (lib/Utils.cpp:334-453, one pass), the zonal column balance of v
(InitValues_Jup.cpp:1500-1538) and the boundary passes on t, u, v, w (BC_Jup.h:185-658,
BoundaryConditions.h:253-360). Test infrastructure only: the specification, checked by
dot-product tests against the oracle's forward passes, that GPU transposes of the whole
iteration follow. Arrays are (im, jm, km) C-ordered; topo is the (jm, km) fluid floor.

Each forward pass maps an input field x to an output y cell by cell from a copy of x, so its
transpose scatters each output's adjoint back through the same stencil: a 4th-order cell
(y = x - c4 d4 x) gives 1 - 6 c4 to itself, 4 c4 to its first and -c4 to its second neighbours, a
2nd-order cell (y = x + c2 d2 x) 1 - 2 c2 and c2, a copied cell 1. The passes are applied in
reverse order.
"""
from __future__ import annotations

import numpy as np


def _shift(a, d, axis):
    """a shifted by d along axis (out-of-range entries 0): out[x] = a[x - d]"""
    out = np.zeros_like(a)
    n = a.shape[axis]
    src = [slice(None)] * a.ndim
    dst = [slice(None)] * a.ndim
    if d >= 0:
        src[axis], dst[axis] = slice(0, n - d), slice(d, n)
    else:
        src[axis], dst[axis] = slice(-d, n), slice(0, n + d)
    out[tuple(dst)] = a[tuple(src)]
    return out


def _scatter(lam, m4, m2, c4, c2, axis):
    """transpose of one out-of-place 4th/2nd-order pass along axis (no wrap): m4, m2 masks of
    the output cells filtered in 4th / 2nd order, the rest copied"""
    l4 = np.where(m4, lam, 0.0)
    l2 = np.where(m2, lam, 0.0)
    out = np.where(m4, (1.0 - 6.0 * c4) * lam, np.where(m2, (1.0 - 2.0 * c2) * lam, lam))
    out += 4.0 * c4 * (_shift(l4, 1, axis) + _shift(l4, -1, axis))
    out += -c4 * (_shift(l4, 2, axis) + _shift(l4, -2, axis))
    out += c2 * (_shift(l2, 1, axis) + _shift(l2, -1, axis))
    return out


def shapiro4_T(lam, topo, strength=1.0):
    """the transpose of one pass of the 4th-order filter with the fluid floor topo"""
    lam = np.array(lam, dtype=np.float64)
    im, jm, km = lam.shape
    c4, c2 = strength / 16.0, strength * 0.25
    floor = np.maximum(np.asarray(topo), 0)                       # (jm, km)
    i_idx = np.arange(im)[:, None, None]
    inf = i_idx >= floor[None, :, :]                                # (im, jm, km)
    # i pass (last forward): column from the floor up, clamped at the top
    fm1, fp1 = i_idx - 1 >= floor[None], i_idx + 1 <= im - 1
    fm2, fp2 = i_idx - 2 >= floor[None], i_idx + 2 <= im - 1
    act = inf & fm1 & fp1
    lam = _scatter(lam, act & fm2 & fp2, act & ~(fm2 & fp2), c4, c2, 0)
    # j pass
    inf_jm1, inf_jp1 = _shift(inf, 1, 1), _shift(inf, -1, 1)       # inf at j-1, j+1 (False outside)
    inf_jm2, inf_jp2 = _shift(inf, 2, 1), _shift(inf, -2, 1)
    act = inf & inf_jm1 & inf_jp1
    lam = _scatter(lam, act & inf_jm2 & inf_jp2, act & ~(inf_jm2 & inf_jp2), c4, c2, 1)
    # k pass (first forward): the ring of km-1 meridians; the output at km-1 is the copy of k = 0
    n = km - 1
    lam = lam.copy()
    lam[:, :, 0] += lam[:, :, n]
    lam[:, :, n] = 0.0
    ring = lam[:, :, :n]
    infr = inf[:, :, :n]
    roll = lambda a, d: np.roll(a, d, axis=2)                     # roll(a, d)[k] = a[k - d]
    act = infr & roll(infr, 1) & roll(infr, -1)
    m4 = act & roll(infr, 2) & roll(infr, -2)
    m2 = act & ~(roll(infr, 2) & roll(infr, -2))
    l4 = np.where(m4, ring, 0.0)
    l2 = np.where(m2, ring, 0.0)
    out = np.where(m4, (1.0 - 6.0 * c4) * ring, np.where(m2, (1.0 - 2.0 * c2) * ring, ring))
    out += 4.0 * c4 * (roll(l4, 1) + roll(l4, -1)) - c4 * (roll(l4, 2) + roll(l4, -2))
    out += c2 * (roll(l2, 1) + roll(l2, -1))
    res = np.zeros_like(lam)
    res[:, :, :n] = out
    return res


def balance_v_T(lam, topo, rad, dr):
    """the transpose of the zonal column balance of v: v -= (per row) the mean over the open
    meridians k < km-1 of the trapezoid column means of r v, subtracted in every open column"""
    lam = np.array(lam, dtype=np.float64)
    im, jm, km = lam.shape
    rad = np.asarray(rad, dtype=np.float64)
    open_ = np.asarray(topo) == 0                                   # (jm, km)
    w = 0.5 * rad * dr
    w[1:-1] *= 2.0                                                  # the trapezoid's weights of r v
    I0 = sum(0.5 * (rad[i] + rad[i + 1]) * dr for i in range(im - 1))
    out = lam.copy()
    for j in range(1, jm - 1):
        mean_cols = np.nonzero(open_[j, : km - 1])[0]
        if mean_cols.size == 0:
            continue
        sub_cols = np.nonzero(open_[j])[0]
        S = lam[:, j, sub_cols].sum()                              # d(sum of the outputs)/d(dv)
        out[:, j, mean_cols] -= (S / mean_cols.size) * (w / I0)[:, None]
    return out


C43, C13 = 4.0 / 3.0, 1.0 / 3.0


def bc_T(lam, solid, lid_u=1, top_taper=3, pole_fill_rows=2, mount_t_ambient=1):
    """the transpose of the dry boundary passes (radius, theta, phi, solid; BC_Jup.h:185-658) on
    (t, u, v, w): lam is a dict of their adjoints after the passes, the result their adjoints
    before. p_stat is frozen and p_dyn's part belongs to the pressure pass, so only t, u, v, w
    are carried."""
    L = {n: np.array(lam[n], dtype=np.float64) for n in ("t", "u", "v", "w")}
    im, jm, km = L["t"].shape
    sol = np.asarray(solid).astype(bool)
    # ---- solid cells, in reverse: the ambient rows, then the extrapolation and the zeroing
    t = L["t"]
    if mount_t_ambient:
        for i in range(im):
            for j in range(jm):
                s_row = sol[i, j]
                n = int((~s_row).sum())
                if not s_row.any() or n == 0:
                    continue
                S = t[i, j, s_row].sum()
                t[i, j, s_row] = 0.0
                t[i, j, ~s_row] += S / n
    for n in ("u", "v", "w"):
        L[n][sol] = 0.0
    fl = ~sol
    def fluid(i, j, k):
        return 0 <= i < im and 0 <= j < jm and 0 <= k < km and fl[i, j, k]
    for i, j, k in zip(*np.nonzero(sol)):
        nb = ((i + 1, j, k), (i - 1, j, k), (i, j + 1, k), (i, j - 1, k), (i, j, k + 1), (i, j, k - 1))
        surf = any(0 <= a < im and 0 <= b < jm and 0 <= c < km and fl[a, b, c] for a, b, c in nb)
        if not surf:
            continue
        pair = None
        for (a1, a2) in (((i + 1, j, k), (i + 2, j, k)), ((i - 1, j, k), (i - 2, j, k)),
                         ((i, j + 1, k), (i, j + 2, k)), ((i, j - 1, k), (i, j - 2, k)),
                         ((i, j, k + 1), (i, j, k + 2)), ((i, j, k - 1), (i, j, k - 2))):
            if fluid(*a1) and fluid(*a2):
                pair = (a1, a2)
                break
        if pair is None:
            continue
        g = t[i, j, k]
        t[i, j, k] = 0.0
        t[pair[0]] += C43 * g
        t[pair[1]] -= C13 * g
    # ---- phi: k = km-1 is the copy of k = 0
    for n in L:
        L[n][:, :, 0] += L[n][:, :, km - 1]
        L[n][:, :, km - 1] = 0.0
    # ---- theta: the pole rows copy row 1 (t, u) or are 0 (v, w), after the fill of rows 1..nfill
    for n in ("t", "u"):
        x = L[n]
        x[:, 1, :] += x[:, 0, :]
        x[:, 0, :] = 0.0
        x[:, jm - 2, :] += x[:, jm - 1, :]
        x[:, jm - 1, :] = 0.0
    for n in ("v", "w"):
        L[n][:, 0, :] = 0.0
        L[n][:, jm - 1, :] = 0.0
    if pole_fill_rows > 0:
        jf = pole_fill_rows + 1
        for r in range(pole_fill_rows, 0, -1):
            ramp = r / jf
            for n in ("t", "u"):
                x = L[n]
                x[:, jf, :] += x[:, r, :]
                x[:, r, :] = 0.0
                x[:, jm - 1 - jf, :] += x[:, jm - 1 - r, :]
                x[:, jm - 1 - r, :] = 0.0
            for n in ("v", "w"):
                z = L[n]
                z[:, jf, :] += ramp * z[:, r, :]
                z[:, r, :] = 0.0
                z[:, jm - 1 - jf, :] += ramp * z[:, jm - 1 - r, :]
                z[:, jm - 1 - r, :] = 0.0
    # ---- radius, in reverse: the zonal-mean sponge, the taper, the lid, the Neumann walls, and
    # the zonal means of the pre-pass v, w at levels im-3 and im-2 that the sponge reads
    zbar = {}
    if top_taper == 3:
        for n in ("v", "w"):
            x = L[n]
            zbar[n] = (C13 * x[im - 3].sum(axis=1),                       # d/d(mean at im-3), per j
                       (2.0 / 3.0) * x[im - 2].sum(axis=1) + x[im - 1].sum(axis=1))   # at im-2
            x[im - 1] = 0.0                                               # overwritten by the mean
    if top_taper != 0:
        for n in ("v", "w"):
            x = L[n]
            if top_taper == 2:
                g2, g3 = x[im - 2].copy(), x[im - 3].copy()
                x[im - 2] = 0.0
                x[im - 3] = 0.0
                x[im - 4] += C13 * g2 + (2.0 / 3.0) * g3
            else:
                x[im - 2] *= C13
                x[im - 3] *= 2.0 / 3.0
            x[im - 1] = 0.0
    if lid_u:
        L["u"][0] = 0.0
        L["u"][im - 1] = 0.0
    for n in L:
        x = L[n]
        g0, g1 = x[0].copy(), x[im - 1].copy()
        x[0] = 0.0
        x[im - 1] = 0.0
        x[1] += C43 * g0
        x[2] -= C13 * g0
        x[im - 2] += C43 * g1
        x[im - 3] -= C13 * g1
    if top_taper == 3:
        kn = km - 1
        for n in ("v", "w"):
            x = L[n]
            g3, g2 = zbar[n]
            x[im - 3, :, :kn] += (g3 / kn)[:, None]
            x[im - 2, :, :kn] += (g2 / kn)[:, None]
    return L
