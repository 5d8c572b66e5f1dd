"""Seeded synthetic model state with the shapes and value ranges of ATJUP's initial state.

The reference builds its start state with a long initialisation chain (cJupiterModel.cpp:392-745:
temperature profile, polytropic / isothermal static pressure, measured jets, geostrophic balance,
vortex, SeaMount cone). That chain is not part of the time-step hot path, so benchmarks and
small-grid tests use this generator instead: the same grid geometry (metric radius R/L_atm + i dr,
1-degree colatitude and longitude), the same obstacle construction (an elliptic cone of
half-axes 18 x 12 cells at the base shrinking to 6 x 4 at level 26, centred at j = 112,
k = 180 -- BC_Jup.h:386-413 with ATJUP_CONE_GEOM = 2), a parabolic pole-to-equator temperature
with a 2 K/km lapse clamped at 110 K (InitValues_Jup.cpp:186-264), a polytropic / isothermal
static pressure (InitValues_Jup.cpp:633-693), banded zonal jets, and the i.i.d. Gaussian
perturbations of the dry benchmark configuration (u, v ~ N(0, 0.1 m/s), w ~ N(0, 0.01 m/s),
T ~ N(0, 0.05 K), zero inside the obstacle). Values are nondimensional as in the model.
On grids smaller than 41 x 181 x 361 the obstacle and jets are scaled to the grid.
"""
from __future__ import annotations

import math

import numpy as np

R_PLANET_KM = 69911.0


def grid(im=41, jm=181, km=361, L_atm=140.0, dr=0.025, cone=True):
    """rad, the, solid mask, i_topography for an (im, jm, km) shell."""
    r0 = R_PLANET_KM / L_atm
    rad = r0 + dr * np.arange(im)
    dthe = 1.0 / (180.0 / math.pi)
    the = dthe * np.arange(jm) * (180.0 / (jm - 1))       # 0 .. pi over jm points
    solid = np.zeros((im, jm, km), np.uint8)
    if cone:
        sj, sk = (jm - 1) / 180.0, (km - 1) / 360.0
        j0, k0 = int(round(112 * sj)), int(round(180 * sk))
        i_top = min(26, im - 5)       # the top folds (p[im-1] from im-2, im-3) never read the obstacle
        base_a, base_b = max(2.0, 18 * sk), max(2.0, 12 * sj)
        a_top, b_top = max(1.0, 6 * sk), max(1.0, 4 * sj)
        for i in range(i_top + 1):
            f = i / i_top
            ai = round(base_a + (a_top - base_a) * f)
            bi = round(base_b + (b_top - base_b) * f)
            for k in range(k0 - ai, k0 + ai + 1):
                for j in range(j0 - bi, j0 + bi + 1):
                    x, y = (k - k0) / ai, (j - j0) / bi
                    if x * x + y * y <= 1.0 + 1e-9 and 0 <= j < jm and 0 <= k < km:
                        solid[i, j, k] = 1
    topo = np.zeros((jm, km), np.int32)
    for j in range(jm):
        for k in range(km):
            i = 0
            while i < im and solid[i, j, k]:
                i += 1
            topo[j, k] = i
    return rad, the, solid, topo


def state(im=41, jm=181, km=361, seed=20261203, cone=True, t_ref=165.0, u_0=100.0,
          r_mix=1.2844, R_mix=3531.1847352206946, g=25.92, L_atm=140.0, dr=0.025):
    """Dict of grid arrays and fields (contiguous (i, j, k) float64 arrays)."""
    rad, the, solid, topo = grid(im, jm, km, L_atm, dr, cone)
    rng = np.random.Generator(np.random.Philox(seed))
    shape = (im, jm, km)
    jj = np.arange(jm)
    ratio = jj / ((jm - 1) / 2.0)
    t_pole, t_eq, gam = 310.0, 330.0, 2.0
    t0 = (t_pole + (t_eq - t_pole) * (1.0 - (ratio - 1.0) ** 2))          # K at the base
    height = np.arange(im) * (L_atm / (im - 1))                          # km
    T = t0[None, :] - gam * height[:, None]
    T = np.maximum(T, 110.0) / t_ref
    t = np.broadcast_to(T[:, :, None], shape).copy()
    # polytropic below the clamp, isothermal above
    exp_p = g / (gam * R_mix * 1e-3)
    p_poly = (t * t_ref / t_ref) ** exp_p * 1.0
    p_stat = p_poly.copy()
    for j in range(jm):
        clamp = np.where(T[:, j] * t_ref <= 110.0 + 1e-9)[0]
        if len(clamp):
            ic = clamp[0]
            H = R_mix * 110.0 / g
            z = height * 1e3
            p_stat[ic:, j, :] = p_stat[ic - 1, j, :][None, :] * np.exp(-(z[ic:] - z[ic - 1]) / H)[:, None]
    # banded zonal jets (w), weak meridional cells (v), tiny radial wind (u)
    lat = math.pi / 2 - the
    jet = 1.2 * np.sin(6 * lat) * np.cos(lat) ** 2
    w = np.broadcast_to((jet[None, :] * (0.3 + 0.7 * np.arange(im)[:, None] / (im - 1)))[:, :, None], shape).copy()
    v = np.broadcast_to((0.05 * np.sin(2 * lat)[None, :] * np.cos(math.pi * np.arange(im) / (im - 1))[:, None])[:, :, None], shape).copy()
    u = np.zeros(shape)
    # perturbations of the dry benchmark configuration (model units: / u_0, / t_ref)
    w += rng.normal(0.0, 0.1 / u_0, shape)
    v += rng.normal(0.0, 0.1 / u_0, shape)
    u += rng.normal(0.0, 0.01 / u_0, shape)
    t += rng.normal(0.0, 0.05 / t_ref, shape)
    fluid = solid == 0
    for a in (u, v, w):
        a *= fluid
    p_dyn = 0.5 * np.broadcast_to(np.cos(2 * the)[None, :, None], shape) * (1.0 + 0.1 * rng.standard_normal(shape))
    p_baro = -0.2 * np.broadcast_to(np.cos(the)[None, :, None], shape).copy()
    rho_mix = p_stat * 1e5 / (R_mix * t * t_ref)
    wall_nue = np.zeros(shape)
    # wall viscosity near the obstacle: 0.004 on fluid cells touching it
    if solid.any():
        near = np.zeros(shape, bool)
        for ax in range(3):
            for d in (-1, 1):
                near |= np.roll(solid, d, axis=ax).astype(bool)
        wall_nue[(near & fluid)] = 0.004
    cell_vbar0 = np.zeros(im * jm)
    cell_ubar0 = np.zeros(im * jm)
    return {
        "rad": rad, "the": the, "solid": solid, "topo": topo,
        "cell_vbar0": cell_vbar0, "cell_ubar0": cell_ubar0,
        "t": t, "u": u, "v": v, "w": w, "p_dyn": p_dyn, "p_hydro": np.zeros(shape),
        "p_stat": p_stat, "rho_mix": rho_mix, "wall_nue": wall_nue, "p_baro": p_baro,
        "aux_u": np.zeros(shape), "aux_v": np.zeros(shape), "aux_w": np.zeros(shape),
    }


def saturation_density(T_K, p_bar, rho, gas_consts, ice=False):
    """rho * ep * E(T) / p with E the vapour-pressure fit exp(C + (-L0/T + a ln T + b T) /
    (1e-3 R)) [bar] (the form of ATPhys.h:49-52); used only to place synthetic species near
    saturation."""
    (t_0, t_00, ep, lv, ls, C, L0, R, da, db, Ci, L0i, dai, dbi) = gas_consts
    if ice:
        C, L0, da, db = Ci, L0i, dai, dbi
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        E = np.exp(C + (-L0 / T_K + da * np.log(T_K) + db * T_K) / (1e-3 * R))
        return rho * ep * E / p_bar


def moist(s: dict, gases: dict, seed: int = 20261205, t_ref: float = 165.0) -> dict:
    """Species fields (vapour, cloud, ice of H2O, NH3, CH4) for a state from state(): vapour at
    U(0.3, 1.7) times the liquid saturation density of the cell (capped at 2 % of the mixture
    density), cloud and ice seeded in a third of the fluid cells each at up to half the vapour.
    Every path of the saturation adjustment is taken: condensation, evaporation, melting above
    t_0, the Bergeron branch, dry exits. Zero in solid cells."""
    rng = np.random.Generator(np.random.Philox(seed))
    t, p, rho = s["t"], s["p_stat"], s["rho_mix"]
    shape = t.shape
    fluid = s["solid"] == 0
    out = {}
    for gas, cst in gases.items():
        sat = saturation_density(t * t_ref, p, rho, cst)
        sat = np.where(np.isfinite(sat), np.minimum(sat, 0.02 * rho), 0.0)
        vap = sat * rng.uniform(0.3, 1.7, shape)
        cl = np.where(rng.uniform(size=shape) < 1 / 3, 0.5 * vap * rng.uniform(size=shape), 0.0)
        ic = np.where(rng.uniform(size=shape) < 1 / 3, 0.5 * vap * rng.uniform(size=shape), 0.0)
        name = gas.lower()
        out[name] = np.where(fluid, vap, 0.0)
        out[name + "_cloud"] = np.where(fluid, cl, 0.0)
        out[name + "_ice"] = np.where(fluid, ic, 0.0)
    return out


def physics(s: dict, gases: dict, seed: int = 20261206, u_0: float = 100.0,
            L_atm: float = 140.0) -> dict:
    """Full-physics fields for a state from state(): the species of moist(), h2s and nh4sh,
    k* = k / u_0^2 with k = 1e-4 m2/s2 x U(0.5, 1.5), omega* = omega L / u_0 with
    omega = 1e-3 1/s x U(0.5, 1.5), their time-level-n copies (equal to the live fields), a
    frozen eddy viscosity nue* = k*/omega*, seeded frozen microphysics and chemistry sources of
    1e-6 scale, heating rates of 0.05 W/m3 scale, the friction velocity 0.05 m/s and the level
    heights [km] (float32). Zero in solid cells."""
    rng = np.random.Generator(np.random.Philox(seed))
    t = s["t"]
    shape = t.shape
    im = shape[0]
    fluid = s["solid"] == 0
    out = moist(s, gases, seed=seed + 1)
    out["h2s"] = np.where(fluid, 1e-3 * rng.uniform(0.5, 1.5, shape), 0.0)
    out["nh4sh"] = np.where(fluid, 1e-5 * rng.uniform(0.0, 1.0, shape), 0.0)
    tke = 1e-4 / u_0 ** 2 * rng.uniform(0.5, 1.5, shape)
    om = 1e-3 * (L_atm * 1e3 / u_0) * rng.uniform(0.5, 1.5, shape)
    out["tke"] = np.where(fluid, tke, 0.0)
    out["dis"] = np.where(fluid, om, 0.0)
    out["nue"] = np.where(fluid, tke / om, 0.0)
    for n in ("S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice", "S_precip_nh3",
              "S_precip_nh3_cloud", "S_precip_nh3_ice", "S_precip_ch4", "S_precip_ch4_cloud",
              "S_precip_ch4_ice", "massflux_h2s", "massflux_nh3", "massflux_nh4sh",
              "fluxlim_nh4sh"):
        out[n] = np.where(fluid, 1e-6 * rng.standard_normal(shape), 0.0)
    out["Q_rad"] = np.where(fluid, 0.05 * rng.standard_normal(shape), 0.0)
    out["Q_precip"] = np.where(fluid, 0.05 * rng.standard_normal(shape), 0.0)
    for n in ("prod", "tke_source", "dis_source"):
        out[n] = np.zeros(shape)
    out["vel_star"] = np.full(shape[1:], 0.05)
    out["layer_heights"] = (np.arange(im) * (L_atm / (im - 1))).astype(np.float32)
    return out


def full_physics(s: dict, gases: dict, seed: int = 20261207, u_0: float = 100.0,
                 L_atm: float = 140.0, h2s_fraction: float = 7.0e-4) -> dict:
    """The full-physics benchmark state on a state from state(): vapour of H2O, NH3, CH4 at 90 % of
    the liquid saturation density of the cell (the model's vapour-pressure fits) times seeded
    U(0.95, 1.05), capped at 2 % of the mixture density, no condensate; H2S at h2s_fraction of the
    mixture density, no NH4SH; k = 1e-4 m2/s2 x U(0.5, 1.5) and omega = 1e-3 1/s x U(0.5, 1.5) in
    the model's units (k / u_0^2, omega L / u_0); the diagnostic and source fields zero (the
    iteration computes them); the friction velocity 0.05 m/s and the level heights [km]."""
    rng = np.random.Generator(np.random.Philox(seed))
    t, p, rho = s["t"], s["p_stat"], s["rho_mix"]
    shape = t.shape
    im = shape[0]
    fluid = s["solid"] == 0
    out = {}
    for gas, cst in gases.items():
        sat = saturation_density(t * 165.0, p, rho, cst)
        sat = np.where(np.isfinite(sat), np.minimum(sat, 0.02 * rho), 0.0)
        name = gas.lower()
        out[name] = np.where(fluid, 0.9 * sat * rng.uniform(0.95, 1.05, shape), 0.0)
        out[name + "_cloud"] = np.zeros(shape)
        out[name + "_ice"] = np.zeros(shape)
    out["h2s"] = np.where(fluid, h2s_fraction * rho, 0.0)
    out["nh4sh"] = np.zeros(shape)
    out["tke"] = np.where(fluid, 1e-4 / u_0 ** 2 * rng.uniform(0.5, 1.5, shape), 0.0)
    out["dis"] = np.where(fluid, 1e-3 * (L_atm * 1e3 / u_0) * rng.uniform(0.5, 1.5, shape), 0.0)
    for n in ("nue", "prod", "tke_source", "dis_source", "Q_rad", "Q_precip",
              "S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice", "S_precip_nh3",
              "S_precip_nh3_cloud", "S_precip_nh3_ice", "S_precip_ch4", "S_precip_ch4_cloud",
              "S_precip_ch4_ice", "massflux_h2s", "massflux_nh3", "massflux_nh4sh",
              "fluxlim_nh4sh", "difflux_h2s", "difflux_nh3", "difflux_nh4sh"):
        out[n] = np.zeros(shape)
    out["vel_star"] = np.full(shape[1:], 0.05)
    out["layer_heights"] = (np.arange(im) * (L_atm / (im - 1))).astype(np.float32)
    return out


def smooth121(f: np.ndarray, passes: int = 3) -> np.ndarray:
    """`passes` Shapiro 1-2-1 passes in k (ring of km-1 meridians, seam copy), then j (clamped at
    the poles), then i (clamped), no fluid floor -- damp_wiggles with i_surface = nullptr
    (lib/Utils.cpp:227-323)."""
    f = np.array(f, dtype=np.float64, copy=True)
    im, jm, km = f.shape
    n = km - 1
    for _ in range(passes):
        ring = f[:, :, :n]
        f[:, :, :n] = ring + 0.25 * (np.roll(ring, 1, axis=2) - 2.0 * ring + np.roll(ring, -1, axis=2))
        f[:, :, n] = f[:, :, 0]
        jm1 = np.concatenate([[0], np.arange(jm - 1)])
        jp1 = np.concatenate([np.arange(1, jm), [jm - 1]])
        f = f + 0.25 * (f[:, jm1, :] - 2.0 * f + f[:, jp1, :])
        im1 = np.concatenate([[0], np.arange(im - 1)])
        ip1 = np.concatenate([np.arange(1, im), [im - 1]])
        f = f + 0.25 * (f[im1] - 2.0 * f + f[ip1])
    return f


def poisson_rhs(im=41, jm=181, km=361, seed=20261204) -> np.ndarray:
    """Right-hand side of the isolated Poisson benchmark: seeded N(0, 1) on every cell, smoothed by
    3 passes of the 1-2-1 filter in each direction. (The solver removes its incompatible part.)"""
    rng = np.random.Generator(np.random.Philox(seed))
    return smooth121(rng.standard_normal((im, jm, km)), 3)
