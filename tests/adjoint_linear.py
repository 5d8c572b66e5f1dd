"""Transposes of the linear passes of the dry iteration, in numpy: the in-loop 4th-order Shapiro
filter (lib/Utils.cpp:334-453, one pass), the zonal column balance of v
(InitValues_Jup.cpp:1500-1538), the boundary passes on t, u, v, w (BC_Jup.h:185-658,
BoundaryConditions.h:253-360) and the pressure pass (PressureSolver.h:144-766 with the radial walls
of its source, cJupiterModel.cpp:1842-1864), and the tangent-linear and transpose of the
mixture density between them and the RK step (computeMixtureDensity). Test infrastructure only: the specification, checked by
dot-product tests against the oracle's forward passes, that GPU transposes of the whole
iteration follow. Arrays are (im, jm, km) C-ordered; topo is the (jm, km) fluid floor.

Each forward pass maps an input field x to an output y cell by cell from a copy of x, so its
transpose scatters each output's adjoint back through the same stencil: a 4th-order cell
(y = x - c4 d4 x) gives 1 - 6 c4 to itself, 4 c4 to its first and -c4 to its second neighbours, a
2nd-order cell (y = x + c2 d2 x) 1 - 2 c2 and c2, a copied cell 1. The passes are applied in
reverse order. The pressure pass updates p in place, one colour at a time; no cell of a colour
reads another of the same colour (the ring of km-1 meridians is even), so each colour's transpose
is a scatter of lam / den to the six neighbours and of -lam / den to the source, the colours
taken black then red and the folds first within each sweep.
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


def _press_weights(P, grid):
    """per interior cell the six neighbour weights of the red-black sweep (PressureSolver.h:
    354-357, 461-479) and their sum den; the k neighbours wrap on the ring of km-1 meridians"""
    im, jm, km = P.im, P.jm, P.km
    sol = np.asarray(grid["solid"]).reshape(im, jm, km).astype(bool)
    rad = np.asarray(grid["rad"], dtype=np.float64)
    the = np.asarray(grid["the"], dtype=np.float64)
    sinthe = np.maximum(P.sinthe_min, np.abs(np.sin(the)))
    inv_rm2 = 1.0 / (rad * rad)
    n1 = np.full((im, jm), 1.0 / (P.dr * P.dr))
    n2 = inv_rm2[:, None] * np.full(jm, 1.0 / (P.dthe * P.dthe))[None, :]
    n3 = (inv_rm2[:, None] / (sinthe * sinthe)[None, :]) * (1.0 / (P.dphi * P.dphi))
    n = km - 1
    ke = np.r_[(np.arange(n) + 1) % n, 0]
    kw = np.r_[(np.arange(n) - 1) % n, 0]
    interior = np.zeros((im, jm, km), bool)
    interior[1:-1, 1:-1, :n] = True
    fl = ~sol
    nb_fluid = (_shift(fl, -1, 0), _shift(fl, 1, 0), _shift(fl, -1, 1), _shift(fl, 1, 1),
                fl[:, :, ke], fl[:, :, kw])                                # +i, -i, +j, -j, +k, -k
    full = ~(bool(P.press_wall) & fl)                                     # every face kept
    W = []
    for d, nn in enumerate((n1, n1, n2, n2, n3, n3)):
        w = np.where(full | nb_fluid[d], nn[:, :, None], 0.0)
        W.append(np.where(interior, w, 0.0))
    den = np.where(interior, W[0] + W[1] + W[2] + W[3] + W[4] + W[5], 0.0)
    return W, den, interior, ke, kw


def _fold_T(lam):
    """transpose of the folds after each sweep: 2-point Neumann in r over the whole shell, then
    in theta, then the seam copy k = km-1 <- k = 0"""
    im, jm, km = lam.shape
    lam[:, :, 0] += lam[:, :, km - 1]
    lam[:, :, km - 1] = 0.0
    for ax, n in ((1, jm), (0, im)):
        for edge, in1, in2 in ((0, 1, 2), (n - 1, n - 2, n - 3)):
            sl = [slice(None)] * 3
            sl[ax] = edge
            g = lam[tuple(sl)].copy()
            lam[tuple(sl)] = 0.0
            sl[ax] = in1
            lam[tuple(sl)] += C43 * g
            sl[ax] = in2
            lam[tuple(sl)] -= C13 * g


def _div_terms(P, grid, i, j, k):
    """the terms (field 0/1/2 = aux_u/v/w, (i, j, k), coefficient) of one cell's divergence
    source (PressureSolver.h:370-459): one-sided at solid cells, the later theta and phi cases
    overriding the earlier as in the reference"""
    im, jm, km = P.im, P.jm, P.km
    sol = grid["_sol3"]
    n = km - 1
    kw, ke = (k - 1) % n, (k + 1) % n
    rm = float(grid["rad"][i])
    sinthe = max(P.sinthe_min, abs(np.sin(grid["the"][j])))
    i2dr, i2dt, i2dp = 1.0 / (2.0 * P.dr), 1.0 / (2.0 * P.dthe), 1.0 / (2.0 * P.dphi)
    idt, idp = 1.0 / P.dthe, 1.0 / P.dphi
    inv_rm, inv_rms = 1.0 / rm, 1.0 / (rm * sinthe)
    sld = sol[i, j, k]
    if i < im - 2 and sld and not sol[i + 1, j, k]:
        du = [((i, j, k), -3.0 * i2dr), ((i + 1, j, k), 4.0 * i2dr), ((i + 2, j, k), -i2dr)]
    else:
        du = [((i + 1, j, k), i2dr), ((i - 1, j, k), -i2dr)]
    dv = [((i, j + 1, k), i2dt), ((i, j - 1, k), -i2dt)]
    if 2 < j < jm - 2:
        ajp, ajm = not sol[i, j + 1, k], not sol[i, j - 1, k]
        if sld and ajp and not sol[i, j + 2, k]:
            dv = [((i, j, k), -3.0 * i2dt), ((i, j + 1, k), 4.0 * i2dt), ((i, j + 2, k), -i2dt)]
        if sld and ajm and not sol[i, j - 2, k]:
            dv = [((i, j, k), 3.0 * i2dt), ((i, j - 1, k), -4.0 * i2dt), ((i, j - 2, k), i2dt)]
        if (sld and ajp and sol[i, j + 2, k]) or (j == jm - 2 and not sld and sol[i, j + 1, k]):
            dv = [((i, j + 1, k), idt), ((i, j, k), -idt)]
        if (sld and ajm and sol[i, j - 2, k]) or (j == 1 and sld and ajm):
            dv = [((i, j - 1, k), idt), ((i, j, k), -idt)]
    dw = [((i, j, ke), i2dp), ((i, j, kw), -i2dp)]
    if 2 < k < km - 2:
        akp, akm = not sol[i, j, ke], not sol[i, j, kw]
        skp2 = sol[i, j, k + 2] if k < km - 2 else False
        skm2 = sol[i, j, k - 2] if k > 2 else False
        if sld and akp and not skp2:
            dw = [((i, j, k), -3.0 * i2dp), ((i, j, k + 1), 4.0 * i2dp), ((i, j, k + 2), -i2dp)]
        if sld and akm and not skm2:
            dw = [((i, j, k), 3.0 * i2dp), ((i, j, k - 1), -4.0 * i2dp), ((i, j, k - 2), i2dp)]
        if (sld and akp and skp2) or (k == km - 2 and not sld and sol[i, j, ke]):
            dw = [((i, j, k + 1), idp), ((i, j, k), -idp)]
        if (sld and akm and skm2) or (k == 1 and sld and akm):
            dw = [((i, j, k - 1), idp), ((i, j, k), -idp)]
    return ([(0, c, a) for c, a in du] + [(1, c, a * inv_rm) for c, a in dv]
            + [(2, c, a * inv_rms) for c, a in dw])


def _with_sol3(P, grid):
    g = dict(grid)
    g["_sol3"] = np.asarray(grid["solid"]).reshape(P.im, P.jm, P.km).astype(bool)
    return g


def pressure_source(P, grid, aux):
    """the unclamped divergence source of (aux_u, aux_v, aux_w) after the radial walls of the
    projection (cJupiterModel.cpp:1842-1864) at the cells the sweep updates (den > 0)"""
    g = _with_sol3(P, grid)
    a = [np.array(x, dtype=np.float64) for x in aux]
    im, jm, km = a[0].shape
    for j in range(1, jm - 1):
        for k in range(km - 1):
            if P.rigid_lid:
                a[0][0, j, k] = a[0][im - 1, j, k] = 0.0
            else:
                a[0][0, j, k] = C43 * a[0][1, j, k] - C13 * a[0][2, j, k]
                a[0][im - 1, j, k] = C43 * a[0][im - 2, j, k] - C13 * a[0][im - 3, j, k]
            for q in (1, 2):
                a[q][0, j, k] = C43 * a[q][1, j, k] - C13 * a[q][2, j, k]
                a[q][im - 1, j, k] = C43 * a[q][im - 2, j, k] - C13 * a[q][im - 3, j, k]
    _, den, interior, _, _ = _press_weights(P, grid)
    src = np.zeros_like(a[0])
    for i, j, k in zip(*np.nonzero(interior & (den > 0))):
        src[i, j, k] = sum(coef * a[q][c] for q, c, coef in _div_terms(P, g, i, j, k))
    return src


def pressure_T(lam, P, grid, sweeps, pass_mask=None):
    """the transpose of the pressure pass (PressureSolver.h:144-766, pointwise branch, omega 1):
    `sweeps` red-black Gauss-Seidel sweeps of p_dyn with the folds after each, the source the
    clamped divergence of aux_u, aux_v, aux_w after their radial walls. The clamp is linearised
    by pass_mask (1 where |div| < cap den, default everywhere). Returns the adjoints of p_dyn
    and of aux_u, aux_v, aux_w before the pass."""
    lp = np.array(lam, dtype=np.float64)
    im, jm, km = lp.shape
    W, den, interior, ke, kw = _press_weights(P, grid)
    n = km - 1
    ii, jj, kk = np.meshgrid(np.arange(im), np.arange(jm), np.arange(km), indexing="ij")
    parity = (ii + jj + kk) & 1
    lsrc = np.zeros_like(lp)
    for _ in range(sweeps):
        _fold_T(lp)
        for colour in (1, 0):
            act = interior & (den > 0) & (parity == colour)
            G = np.where(act, lp, 0.0) / np.where(act, den, 1.0)
            lp[act] = 0.0
            lsrc -= G
            lp += _shift(W[0] * G, 1, 0) + _shift(W[1] * G, -1, 0)
            lp += _shift(W[2] * G, 1, 1) + _shift(W[3] * G, -1, 1)
            lp[:, :, :n] += np.roll((W[4] * G)[:, :, :n], 1, axis=2)
            lp[:, :, :n] += np.roll((W[5] * G)[:, :, :n], -1, axis=2)
    if pass_mask is not None:
        lsrc = lsrc * pass_mask
    g = _with_sol3(P, grid)
    la = [np.zeros_like(lp) for _ in range(3)]
    for i, j, k in zip(*np.nonzero(lsrc)):
        s = lsrc[i, j, k]
        for q, c, coef in _div_terms(P, g, i, j, k):
            la[q][c] += coef * s
    for j in range(1, jm - 1):
        for k in range(km - 1):
            if P.rigid_lid:
                la[0][0, j, k] = la[0][im - 1, j, k] = 0.0
            qs = (1, 2) if P.rigid_lid else (0, 1, 2)
            for q in qs:
                g0, g1 = la[q][0, j, k], la[q][im - 1, j, k]
                la[q][0, j, k] = la[q][im - 1, j, k] = 0.0
                la[q][1, j, k] += C43 * g0
                la[q][2, j, k] -= C13 * g0
                la[q][im - 2, j, k] += C43 * g1
                la[q][im - 3, j, k] -= C13 * g1
    return lp, la


def _rho_base(P, t, p_stat, p_dyn):
    w = 1.0 if P.rho_pdyn else 0.0
    T = np.asarray(t) * P.t_ref
    p_pa = (np.asarray(p_stat) + w * np.asarray(p_dyn) * P.p_dyn_to_bar) * 1.0e5
    with np.errstate(divide="ignore", invalid="ignore"):
        rho = p_pa / (P.R_mix * T)
    live = (T > 0.0) & np.isfinite(rho)
    return w, T, np.where(live, rho, 0.0), live


def mixture_density_tl(P, t, p_stat, p_dyn, dt, dp_stat, dp_dyn):
    """the tangent-linear of the mixture density (rho = (p_stat + p_dyn c) 1e5 / (R_mix t t_ref),
    0 where t <= 0) about (t, p_stat, p_dyn)"""
    w, T, rho, live = _rho_base(P, t, p_stat, p_dyn)
    with np.errstate(divide="ignore", invalid="ignore"):
        d = (1.0e5 * (dp_stat + w * P.p_dyn_to_bar * dp_dyn) / (P.R_mix * T)
             - rho * dt / np.asarray(t))
    return np.where(live, d, 0.0)


def mixture_density_T(P, t, p_stat, p_dyn, lam):
    """its transpose: the adjoints of t, p_stat, p_dyn from that of rho_mix"""
    w, T, rho, live = _rho_base(P, t, p_stat, p_dyn)
    lam = np.where(live, lam, 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        a_p = np.where(live, 1.0e5 * lam / (P.R_mix * T), 0.0)
        a_t = np.where(live, -rho * lam / np.asarray(t), 0.0)
    return a_t, a_p, w * P.p_dyn_to_bar * a_p
