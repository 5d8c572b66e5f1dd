"""Run the reference (oracle/_ref/libatjup_ref.so) in a child process and dump its state.

    python tests/ref_dump.py OUT.npz [--iters N] [--rk4] [--moist] [--satadj] [--threads T]

Writes the reference's dry initial state (species zeroed unless --moist), its grid, its model
constants, and -- with --iters N -- the state after N iterations of the harness loop
(cJupiterModel.cpp:1032-1381 schedule), or with --rk4 the state after one RungeKuttaJup.
With --satadj: the moist initial state, perturbed by seeded noise (perturb_moist) so that every
branch of the adjustment is taken, then SaturationAdjustmentJup for H2O, NH3 and CH4 in the
order of cJupiterModel.cpp:1060-1080, with t and the gas's fields recorded after each gas.
Test infrastructure only.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from oracle_bridge import (DRY_ENV, DYN_FIELDS, MICRO_DIAGNOSTICS, MICRO_FIELDS, MOIST_ENV,  # noqa: E402
                           PHYS_ENV, Reference)

SPECIES = ("h2o", "h2o_cloud", "h2o_ice", "nh3", "nh3_cloud", "nh3_ice",
           "ch4", "ch4_cloud", "ch4_ice")
GASES = ("H2O", "NH3", "CH4")
SATADJ_SEED = 20261204

CONSTS = ("dt", "re", "pr", "g", "omega", "u_0", "t_ref", "L_atm", "r_mix", "R_mix", "cp_mix",
          "Coriolis", "centrifugal", "buoyancy")


def perturb_moist(f: dict, solid: np.ndarray, seed: int = SATADJ_SEED) -> dict:
    """Seeded perturbation of a moist state that sends cells down every path of the adjustment:
    temperature noise of 2 % (warm cells melt ice, cold ones take the Bergeron branch), vapour
    scaled by U(0.3, 1.7) (super- and subsaturated cells), and cloud and ice seeded in a third of
    the cells each, at up to half the local vapour (mixed-phase and evaporating cells)."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = {k: np.array(v, dtype=np.float64, copy=True) for k, v in f.items()}
    shape = out["t"].shape
    fluid = solid == 0
    out["t"] = np.where(fluid, out["t"] * (1.0 + 0.02 * rng.standard_normal(shape)), out["t"])
    for gas in ("h2o", "nh3", "ch4"):
        vap = out[gas] * rng.uniform(0.3, 1.7, shape)
        cl = np.where(rng.uniform(size=shape) < 1 / 3, 0.5 * vap * rng.uniform(size=shape), 0.0)
        ic = np.where(rng.uniform(size=shape) < 1 / 3, 0.5 * vap * rng.uniform(size=shape), 0.0)
        out[gas] = np.where(fluid, vap, out[gas])
        out[gas + "_cloud"] = np.where(fluid, out[gas + "_cloud"] + cl, out[gas + "_cloud"])
        out[gas + "_ice"] = np.where(fluid, out[gas + "_ice"] + ic, out[gas + "_ice"])
    return out


PHYS_FIELDS = ("h2o", "h2o_cloud", "h2o_ice", "h2s", "nh3", "nh3_cloud", "nh3_ice", "ch4",
               "ch4_cloud", "ch4_ice", "nh4sh", "tke", "dis")
PHYS_SOURCES = ("S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice", "S_precip_nh3",
                "S_precip_nh3_cloud", "S_precip_nh3_ice", "S_precip_ch4", "S_precip_ch4_cloud",
                "S_precip_ch4_ice", "massflux_h2s", "massflux_nh3", "massflux_nh4sh",
                "fluxlim_nh4sh", "Q_rad", "Q_precip")


def rk4_phys_case(ref, g, data, seed=SATADJ_SEED + 1):
    """One RungeKuttaJup with every transported field, on the moist initial state with the
    closure on (k_omega_SST): the live k*, omega* and species differ from their time-level-n
    copies by seeded noise (as after the closure's wall passes), the frozen sources are seeded
    fields of realistic size, and so are nue and the heating rates."""
    rng = np.random.Generator(np.random.Philox(seed))
    shape = ref.shape
    fluid = g["solid"] == 0
    for n in PHYS_FIELDS:
        live = ref.get(n)
        data["in_" + n + "n"] = live.copy()
        ref.set(n + "n", live)
        if n in ("tke", "dis", "h2s", "nh4sh"):
            live = np.where(fluid, live * rng.uniform(0.9, 1.1, shape), live)
        ref.set(n, live)
        data["in_" + n] = live
    nue = np.where(fluid, np.abs(ref.get("nue")) + 1e-4 * rng.uniform(size=shape), 0.0)
    ref.set("nue", nue)
    data["in_nue"] = nue
    for n in PHYS_SOURCES:
        scale = {"Q_rad": 0.05, "Q_precip": 0.05}.get(n, 1e-4)
        f = np.where(fluid, scale * rng.standard_normal(shape), 0.0)
        ref.set(n, f)
        data["in_" + n] = f
    for n in ("prod", "tke_source", "dis_source"):
        data["in_" + n] = ref.get(n)
    data["in_vel_star"] = ref.get1("vel_star").reshape(shape[1], shape[2])
    data["in_layer_heights"] = ref.get1("layer_heights").astype(np.float32)
    for k in ("turb_model", "turb_buoy", "nh4sh_cap", "t_limiter", "rk_scalar_sync"):
        data["knob_" + k] = np.array(ref.L.ref_knob(k.encode()))
    for k in ("nue_max_phys", "tke_max", "turb_buoy_prt", "species_divu"):
        data["knobd_" + k] = np.array(ref.L.ref_knob_d(k.encode()))
    for c in ("species_diff_scale", "sc_h2o", "sc_h2s", "sc_nh3", "sc_ch4", "sc_nh4sh",
              "chemical_reaction", "r_p_nh4sh", "rg_nh4sh", "mue_mix", "re_turb",
              "use_turbulence_model"):
        data["phys_" + c] = np.array(ref.scalar(c))
    ref.quiet(ref.L.ref_rk4)
    for n in list(DYN_FIELDS) + list(PHYS_FIELDS) + ["prod", "tke_source", "dis_source"]:
        data["out_" + n] = ref.get(n)
    data["out_buoy_ref"] = ref.get1("buoy_ref_level")


TURB_FIELDS = ("tke", "dis", "tken", "disn", "nue", "prod", "tke_source", "dis_source")


def turb_case(ref, g, data, seed=SATADJ_SEED + 2):
    """One TurbulenceJup::run + turbWallOmega on the moist initial state with the closure on:
    the velocities carry seeded noise of 1 m/s (so the production term is exercised), k* and
    omega* seeded noise of 10 % with some cells driven negative (the clamp passes), the n copies
    are the restored live fields."""
    rng = np.random.Generator(np.random.Philox(seed))
    shape = ref.shape
    fluid = g["solid"] == 0
    for n in ("u", "v", "w"):
        f = ref.get(n)
        f = np.where(fluid, f + 0.01 * rng.standard_normal(shape), f)
        ref.set(n, f)
        data["in_" + n] = f
    for n in ("tke", "dis"):
        f = ref.get(n)
        f = np.where(fluid, f * rng.uniform(0.9, 1.1, shape), f)
        neg = fluid & (rng.uniform(size=shape) < 0.01)
        f = np.where(neg, -np.abs(f), f)
        ref.set(n, f)
        ref.set(n + "n", f)
        data["in_" + n] = f
        data["in_" + n + "n"] = f
    for n in ("nue", "prod", "tke_source", "dis_source", "t"):
        data["in_" + n] = ref.get(n)
    data["in_vel_star"] = ref.get1("vel_star").reshape(shape[1], shape[2])
    data["in_layer_heights"] = ref.get1("layer_heights").astype(np.float32)
    for k in ("turb_model", "turb_buoy"):
        data["knob_" + k] = np.array(ref.L.ref_knob(k.encode()))
    for k in ("nue_max_phys", "abl_height", "turb_free", "turb_k_bg", "turb_clamp_pass"):
        data["knobd_" + k] = np.array(ref.L.ref_knob_d(k.encode()))
    for c in ("re_turb", "mue_mix", "chemical_reaction"):
        data["phys_" + c] = np.array(ref.scalar(c))
    ref.quiet(ref.L.ref_turbulence)
    for n in TURB_FIELDS:
        data["out_" + n] = ref.get(n)
    data["out_vel_star"] = ref.get1("vel_star").reshape(shape[1], shape[2])


BC_FIELDS = ("t", "u", "v", "w", "p_stat", "p_dyn") + PHYS_FIELDS + (
    "tken", "disn", "nue", "prod", "tke_source", "dis_source", "massflux_h2s", "massflux_nh3",
    "massflux_nh4sh", "fluxlim_nh4sh")


def bc_case(ref, g, data, seed=SATADJ_SEED + 3):
    """The four boundary passes of one iteration (BC_Jup::bcRadius, bcTheta, bcPhi,
    bcSolidGround, cJupiterModel.cpp:1263-1272) on the moist initial state with the closure on,
    every listed field carrying seeded noise (a tenth of the species negative, k* and omega*
    with some NaN-free out-of-range values) so that each pass has something to overwrite; the
    state after each pass is recorded."""
    rng = np.random.Generator(np.random.Philox(seed))
    shape = ref.shape
    for n in BC_FIELDS:
        f = ref.get(n)
        scale = np.abs(f).max()
        scale = scale if scale > 0 else 1e-4
        f = f + 0.05 * scale * rng.standard_normal(shape)
        if n in PHYS_FIELDS[:11]:
            f = np.where(rng.uniform(size=shape) < 0.1, -np.abs(f), f)
        if n in ("tke", "tken", "dis", "disn", "nue", "prod"):
            f = np.where(rng.uniform(size=shape) < 0.01, -np.abs(f), f)
            f = np.where(rng.uniform(size=shape) < 0.001, 1e7, f)
        ref.set(n, f)
        data["in_" + n] = f
    data["in_layer_heights"] = ref.get1("layer_heights").astype(np.float32)
    for step, fn in (("radius", ref.L.ref_bc_radius), ("theta", ref.L.ref_bc_theta),
                     ("phi", ref.L.ref_bc_phi), ("solid", ref.L.ref_bc_solid)):
        ref.quiet(fn)
        for n in BC_FIELDS:
            data[f"bc_{step}_{n}"] = ref.get(n)


MICRO_CONSTS = ("m_nh3", "m_h2s", "m_nh4sh", "D_nh3", "D_h2s", "D_nh4sh", "polar_divisor_floor",
                "t_0_nh4sh", "t_00_nh4sh", "coeff_h2o_A", "coeff_h2o_B", "coeff_h2o_A_i",
                "coeff_h2o_B_i", "coeff_nh3_A", "coeff_nh3_B", "coeff_nh3_A_i", "coeff_nh3_B_i",
                "rad_F_int", "rad_S_solar", "rad_albedo_bond", "rad_x_H2", "rad_x_He",
                "rad_cia_strength", "rad_opacity_strength", "rad_solar", "rad_solar_strength",
                "rad_sw_tau_per_bar", "rad_bottom", "precip_rate_scale", "precip_coupling_on")


def micro_case(ref, g, data, seed=SATADJ_SEED + 4):
    """Radiation, precipitation, the NH4SH equilibrium, the chemistry block and the species clamp
    of one iteration, in the loop's order, on the moist initial state: the species carry seeded
    noise of 20 % with a few negative cells, NH4SH is seeded in a third of the cells (so it
    both forms and decomposes), cloud and ice are seeded where there is none (so it rains and
    snows); the state after each routine is recorded."""
    rng = np.random.Generator(np.random.Philox(seed))
    shape = ref.shape
    fluid = g["solid"] == 0
    for n in PHYS_FIELDS[:11]:
        f = ref.get(n)
        f = np.where(fluid, f * rng.uniform(0.8, 1.2, shape), f)
        if n.endswith(("_cloud", "_ice")):
            base = ref.get(n.split("_")[0])
            f = np.where(fluid & (rng.uniform(size=shape) < 0.3), f + 0.3 * base * rng.uniform(size=shape), f)
        if n == "nh4sh":
            f = np.where(fluid & (rng.uniform(size=shape) < 0.3), 1e-4 * rng.uniform(size=shape), f)
        f = np.where(fluid & (rng.uniform(size=shape) < 0.005), -np.abs(f) - 1e-9, f)
        ref.set(n, f)
        data["in_" + n] = f
    for n in ("u", "v", "w"):
        data["in_" + n] = ref.get(n)
    for n in ("massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "difflux_h2s",
              "difflux_nh3", "difflux_nh4sh") + MICRO_DIAGNOSTICS:
        data["in_" + n] = ref.get(n)
    data["in_layer_heights"] = ref.get1("layer_heights").astype(np.float32)
    for c in MICRO_CONSTS:
        data["micro_" + c] = np.array(ref.scalar(c))
    for gas in GASES:
        cst = np.zeros(14)
        ref.L.ref_gas_consts(gas.encode(), cst.ctypes.data_as(ctypes.c_void_p))
        data["gas_" + gas] = cst
    for step, fn in (("radiation", ref.L.ref_radiation), ("precipitation", ref.L.ref_precipitation),
                     ("nh4sh_eq", ref.L.ref_nh4sh_eq), ("chemistry", ref.L.ref_chem_fluxes),
                     ("diagnostics", ref.L.ref_diagnostics),
                     ("clamp_species", ref.L.ref_clamp_species)):
        ref.quiet(fn)
        for n in MICRO_FIELDS + PHYS_FIELDS[:11]:
            data[f"mc_{step}_{n}"] = ref.get(n)


ITER_FIELDS = ("t", "u", "v", "w", "p_dyn", "p_hydro", "p_stat", "rho_mix", "wall_nue", "aux_u",
               "aux_v", "aux_w") + PHYS_FIELDS + tuple(n + "n" for n in PHYS_FIELDS) + (
    "nue", "prod", "tke_source", "dis_source", "Q_rad", "Q_precip", "massflux_h2s",
    "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "difflux_h2s", "difflux_nh3",
    "difflux_nh4sh", "S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice", "S_precip_nh3",
    "S_precip_nh3_cloud", "S_precip_nh3_ice", "S_precip_ch4", "S_precip_ch4_cloud",
    "S_precip_ch4_ice")


# cJupiterModel::restart_arrays() and restart_arrays_carried() (FileIO_Jup.cpp:281-304), in file
# order; vel_star follows them in a JUP2 file.
RESTART_FIELDS = ("t", "u", "v", "w", "tn", "un", "vn", "wn",
                  "h2o", "h2o_cloud", "h2o_ice", "h2on", "h2o_cloudn", "h2o_icen", "h2s", "h2sn",
                  "nh3", "nh3_cloud", "nh3_ice", "nh3n", "nh3_cloudn", "nh3_icen",
                  "ch4", "ch4_cloud", "ch4_ice", "ch4n", "ch4_cloudn", "ch4_icen",
                  "nh4sh", "nh4shn", "p_dyn", "p_dynn", "p_stat", "tke", "dis", "tken", "disn",
                  "nue")
RESTART_CARRIED = ("aux_u", "aux_v", "aux_w", "difflux_h2s", "difflux_nh3", "massflux_h2s",
                   "massflux_nh3", "fluxlim_nh4sh", "thermalmassflux", "Q_precip", "Q_rad",
                   "rho_mix", "S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice",
                   "S_precip_nh3", "S_precip_nh3_ice")


MCA_SEED = 20261205
MCA_FIELDS = ("t", "h2o", "h2o_cloud", "h2o_ice", "nh3", "nh3_cloud", "nh3_ice", "h2s", "nh4sh")


def perturb_unstable(f: dict, solid: np.ndarray, layer_h: np.ndarray, seed: int = MCA_SEED) -> dict:
    """Seeded perturbation that makes the moist convective adjustment fire: in 3 % of the columns
    the lowest four fluid levels are warmed (4 K at the bottom, halving upwards), and in 2 % the
    vapour of the lowest three levels is raised to 1.5 x itself (saturated parcels)."""
    rng = np.random.default_rng(seed)
    im, jm, km = f["t"].shape
    t = f["t"].copy()
    h2o, nh3 = f["h2o"].copy(), f["nh3"].copy()
    fluid = solid == 0
    warm = rng.random((jm, km)) < 0.03
    wet = rng.random((jm, km)) < 0.02
    for j, k in zip(*np.nonzero(warm | wet)):
        col = np.nonzero(fluid[:, j, k])[0]
        col = col[col >= 1]
        if len(col) < 5:
            continue
        i0 = col[0]
        for d in range(4):
            if warm[j, k]:
                t[i0 + d, j, k] += 4.0 / 2 ** d / 165.0
            if wet[j, k] and d < 3:
                h2o[i0 + d, j, k] *= 1.5
                nh3[i0 + d, j, k] *= 1.5
    out = dict(f)
    out.update(t=t, h2o=h2o, nh3=nh3)
    return out


def mca_case(ref, g, data):
    """One MoistConvectiveAdjustmentJup (the loop's gases and tracers) on the reference's moist
    state perturbed by perturb_unstable; inputs as in_*, outputs as mca_*."""
    f = perturb_unstable({n: ref.get(n) for n in MCA_FIELDS}, g["solid"],
                         ref.get1("layer_heights"))
    for n, v in f.items():
        ref.set(n, v)
        data["in_" + n] = v
    data["in_layer_heights"] = ref.get1("layer_heights").astype(np.float32)
    for c in MICRO_CONSTS:
        data["micro_" + c] = np.array(ref.scalar(c))
    for gas in GASES:
        cst = np.zeros(14)
        ref.L.ref_gas_consts(gas.encode(), cst.ctypes.data_as(ctypes.c_void_p))
        data["gas_" + gas] = cst
    data["ep_h2s"] = np.array(ref.scalar("ep_h2s"))
    ref.quiet(ref.L.ref_mca)
    for n in MCA_FIELDS:
        data["mca_" + n] = ref.get(n)


def phys_iters_case(ref, g, data, iters, save_restart=None):
    """`iters` iterations of the loop with the physics on (closure, radiation, precipitation, the
    NH4SH equilibrium, the saturation adjustments), from the reference's own moist initial state;
    every field the iteration reads is recorded before, every field it writes after."""
    shape = ref.shape
    for n in ITER_FIELDS:
        data["in_" + n] = ref.get(n)
    if ref.scalar("has_p_baro") == 1.0:
        data["in_p_baro"] = ref.get1("p_baro").reshape(shape)
    data["in_vel_star"] = ref.get1("vel_star").reshape(shape[1], shape[2])
    data["in_layer_heights"] = ref.get1("layer_heights").astype(np.float32)
    for c in MICRO_CONSTS:
        data["micro_" + c] = np.array(ref.scalar(c))
    for c in ("species_diff_scale", "sc_h2o", "sc_h2s", "sc_nh3", "sc_ch4", "sc_nh4sh",
              "chemical_reaction", "r_p_nh4sh", "rg_nh4sh", "mue_mix", "re_turb"):
        data["phys_" + c] = np.array(ref.scalar(c))
    data["knobd_abl_height"] = np.array(ref.L.ref_knob_d(b"abl_height"))
    for gas in GASES:
        cst = np.zeros(14)
        ref.L.ref_gas_consts(gas.encode(), cst.ctypes.data_as(ctypes.c_void_p))
        data["gas_" + gas] = cst
    for it in range(1, iters + 1):
        rc = ref.quiet(ref.L.ref_iteration, it, 1 if it == 1 else 0, 0)
        if rc != 0:
            raise SystemExit(f"ref_iteration rc={rc}")
        if it in (1, iters):
            for n in ITER_FIELDS:
                data[f"it{it}_{n}"] = ref.get(n)
            data[f"it{it}_vel_star"] = ref.get1("vel_star").reshape(shape[1], shape[2])
        if save_restart and it == save_restart[1]:
            # the reference's restart file after this iteration, and every array it holds
            ref.quiet(ref.L.ref_save_state, save_restart[0].encode(), it)
            for n in RESTART_FIELDS + RESTART_CARRIED:
                data[f"rs{it}_{n}"] = ref.get(n)
            data[f"rs{it}_vel_star"] = ref.get1("vel_star").reshape(shape[1], shape[2])


def cone_call(ref, data: dict, tag: int) -> None:
    """One in-loop projection around the obstacle on the reference's current state: u, v, w
    before, v, w after, and the largest SOR sweep count of its printed summary."""
    import re
    for n in ("u", "v", "w"):
        data[f"cone{tag}_pre_{n}"] = ref.get(n)
    sys.stdout.flush()
    saved = os.dup(1)
    with tempfile.TemporaryFile() as tf:
        os.dup2(tf.fileno(), 1)
        try:
            ref.L.ref_cone_proj(1)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        tf.seek(0)
        txt = tf.read().decode(errors="replace")
    m = re.search(r"SOR iterations up to (\d+)", txt)
    data[f"cone{tag}_itmax"] = np.array(int(m.group(1)) if m else -1)
    for n in ("v", "w"):
        data[f"cone{tag}_post_{n}"] = ref.get(n)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--iters", type=int, default=0)
    ap.add_argument("--rk4", action="store_true")
    ap.add_argument("--pressure", action="store_true")
    ap.add_argument("--moist", action="store_true")
    ap.add_argument("--satadj", action="store_true")
    ap.add_argument("--satadj-synthetic", action="store_true")
    ap.add_argument("--rk4-phys", action="store_true")
    ap.add_argument("--turb", action="store_true")
    ap.add_argument("--bc", action="store_true")
    ap.add_argument("--micro", action="store_true")
    ap.add_argument("--phys-iters", type=int, default=0)
    ap.add_argument("--perturb-ulp", action="store_true",
                    help="with --phys-iters: start from t one ulp above the model's own (fluid cells)")
    ap.add_argument("--mca", action="store_true",
                    help="one moist convective adjustment on the perturbed moist state")
    ap.add_argument("--save-restart", default=None, metavar="DIR:N",
                    help="with --phys-iters: write the reference's restart file to DIR after "
                         "iteration N (and record its arrays as rsN_*)")
    ap.add_argument("--load-restart", default=None, metavar="DIR:N",
                    help="load DIR/jup_restart_N.bin into the reference's moist model with its "
                         "own load_state and record every restart array as rs_*")
    ap.add_argument("--rk4-fd", default=None, metavar="NDIR:EPS",
                    help="central differences of one RungeKuttaJup: for NDIR seeded directions d "
                         "(tests/adjoint_cases.py), the top level's zonal mean of w after one "
                         "step from the initial state +- EPS d (t, u, v, w and their n copies)")
    ap.add_argument("--env", action="append", default=[],
                    help="KEY=VALUE set before the model is built (knobs are read once)")
    ap.add_argument("--iter-fd", default=None, metavar="NDIR:EPS:K",
                    help="with --baseline dry: central differences of K dry iterations along NDIR "
                         "seeded directions (the top level's zonal mean of w)")
    ap.add_argument("--baseline", default=None, choices=("dry", "phys"),
                    help="start from the benchmark configuration's seeded initial state "
                         "(oracle/baseline_state.py) with its knobs: dry with --iters, "
                         "phys (the reference's default physics) with --phys-iters")
    ap.add_argument("--cone-at", default=None, metavar="IT,IT,...",
                    help="with --baseline dry: after each listed iteration (0: before the first) "
                         "record u, v, w, run one in-loop projection around the obstacle and "
                         "record v, w and the largest SOR sweep count it printed")
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    out_dir = tempfile.mkdtemp(prefix="atjup_ref_")
    if a.baseline:
        import baseline_state as BS
        ref = BS.make(a.baseline, out_dir + "/run", threads=a.threads, cls=Reference,
                      env_extra=dict(kv.split("=", 1) for kv in a.env))
        data = {}
        BS.record(ref, data, moist=(a.baseline == "phys"))
        if a.perturb_ulp:
            # the reference's own sensitivity: t one ulp higher in the fluid cells
            t = ref.get("t")
            t = np.where(ref.solid() == 0, np.nextafter(t, np.inf), t)
            ref.set("t", t)
            ref.set("tn", t)
        if a.baseline == "phys":
            iters = a.phys_iters
            for it in range(1, iters + 1):
                rc = ref.quiet(ref.L.ref_iteration, it, 1 if it == 1 else 0, 0)
                if rc != 0:
                    raise SystemExit(f"ref_iteration rc={rc}")
                if it in (1, iters):
                    for n in ITER_FIELDS:
                        data[f"it{it}_{n}"] = ref.get(n)
        elif a.iter_fd:
            # central differences of K dry iterations: for NDIR seeded directions d
            # (tests/adjoint_cases.py) on t, u, v, w and their n copies, the top level's zonal mean
            # of w after K iterations from the state +- EPS d; the model is put back to the
            # state before each run (every field the dry iteration reads or writes)
            import adjoint_cases as AC
            ndir, eps, K = a.iter_fd.split(":")
            ndir, eps, K = int(ndir), float(eps), int(K)
            keep = ("t", "u", "v", "w", "tn", "un", "vn", "wn", "p_dyn", "p_dynn", "p_hydro",
                    "p_stat", "rho_mix", "wall_nue", "aux_u", "aux_v", "aux_w", "acc_t", "acc_u",
                    "acc_v", "acc_w", "rhs_t", "rhs_u", "rhs_v", "rhs_w")
            snap = {n: ref.get(n) for n in keep}

            def run(x):
                for n in keep:
                    ref.set(n, snap[n])
                if x is not None:
                    for f in AC.FIELDS:
                        ref.set(f, x[f])
                        ref.set(f + "n", x[f])
                for it in range(1, K + 1):
                    rc = ref.quiet(ref.L.ref_iteration, it, 1 if it == 1 else 0, 1)
                    if rc != 0:
                        raise SystemExit(f"ref_iteration rc={rc}")
                return AC.zonal_mean_top(ref.get("w"))

            data["fd_zm0"] = run(None)
            data["fd_zm0_again"] = run(None)
            for k in range(ndir):
                d = AC.direction(k, ref.shape)
                for sgn, tag in ((1.0, "p"), (-1.0, "m")):
                    data[f"fd_zm{tag}_{k}"] = run({f: snap[f] + sgn * eps * d[f] for f in AC.FIELDS})
            data["fd_eps"] = np.array(eps)
            data["fd_iters"] = np.array(K)
        else:
            cone_at = {int(x) for x in a.cone_at.split(",")} if a.cone_at else set()
            if 0 in cone_at:
                cone_call(ref, data, 0)
            for it in range(1, a.iters + 1):
                rc = ref.quiet(ref.L.ref_iteration, it, 1 if it == 1 else 0, 1)
                if rc != 0:
                    raise SystemExit(f"ref_iteration rc={rc}")
                if it in cone_at:
                    cone_call(ref, data, it)
            for n in DYN_FIELDS:
                data["out_" + n] = ref.get(n)
        np.savez(a.out, **data)
        sys.stdout.flush()
        os._exit(0)
    env = dict(PHYS_ENV) if (a.rk4_phys or a.turb or a.bc) else dict(DRY_ENV)
    if a.micro or a.phys_iters or a.load_restart or a.mca:
        env = dict(MOIST_ENV)
    env.update(dict(kv.split("=", 1) for kv in a.env))
    ref = Reference(env, out_dir + "/run", threads=a.threads,
                    zero_species=not (a.moist or a.satadj or a.satadj_synthetic or a.rk4_phys or a.turb or a.bc or a.micro or a.phys_iters or a.load_restart or a.mca))
    data = {}
    g = ref.grid()
    for k, v in g.items():
        data["grid_" + k] = v
    for n, v in ref.fields().items():
        data["in_" + n] = v
    for c in CONSTS:
        data["const_" + c] = np.array(ref.scalar(c))
    if a.rk4_phys:
        rk4_phys_case(ref, g, data)
    elif a.turb:
        turb_case(ref, g, data)
    elif a.bc:
        bc_case(ref, g, data)
    elif a.micro:
        micro_case(ref, g, data)
    elif a.phys_iters:
        if a.perturb_ulp:
            t = ref.get("t")
            ref.set("t", np.where(g["solid"] == 0, np.nextafter(t, np.inf), t))
        sr = None
        if a.save_restart:
            d_, n_ = a.save_restart.rsplit(":", 1)
            sr = (d_, int(n_))
        phys_iters_case(ref, g, data, a.phys_iters, sr)
    elif a.mca:
        mca_case(ref, g, data)
    elif a.load_restart:
        d_, n_ = a.load_restart.rsplit(":", 1)
        data["load_rc"] = np.array(ref.quiet(ref.L.ref_load_state, d_.encode(), int(n_)))
        for n in RESTART_FIELDS + RESTART_CARRIED:
            data["rs_" + n] = ref.get(n)
        data["rs_vel_star"] = ref.get1("vel_star").reshape(ref.shape[1], ref.shape[2])
    elif a.satadj or a.satadj_synthetic:
        if a.satadj:
            f = perturb_moist({n: ref.get(n) for n in ("t",) + SPECIES}, g["solid"])
        else:
            # the synthetic shell of atjup_b200.synthetic on the reference's grid size, its cone
            # standing in for the SeaMount mask (the only grid input of the adjustment)
            from atjup_b200 import synthetic
            from atjup_b200.params import DEFAULT_GASES
            s = synthetic.state(*ref.shape)
            f = {n: s[n] for n in ("t", "p_stat", "rho_mix")}
            f.update(synthetic.moist(s, DEFAULT_GASES))
            ref.set("SeaMount", s["solid"].astype(np.float64))
            data["grid_solid"] = s["solid"].astype(np.uint8)
        for n, v in f.items():
            ref.set(n, v)
            data["in_" + n] = v
        data["knob_local_rho"] = np.array(ref.L.ref_knob(b"local_rho"))
        for gas in GASES:
            cst = np.zeros(14)
            if ref.L.ref_gas_consts(gas.encode(), cst.ctypes.data_as(ctypes.c_void_p)) != 0:
                raise SystemExit(f"no constants for {gas}")
            data["gas_" + gas] = cst
            ref.quiet(ref.L.ref_satadj, gas.encode())
            data[f"sat_{gas}_t"] = ref.get("t")
            for n in SPECIES:
                if n.startswith(gas.lower()):
                    data[f"sat_{gas}_{n}"] = ref.get(n)
    elif a.rk4_fd:
        import adjoint_cases as AC
        ndir, eps = a.rk4_fd.split(":")
        ndir, eps = int(ndir), float(eps)
        base = {f: ref.get(f) for f in AC.FIELDS}
        ref.quiet(ref.L.ref_rk4)
        data["fd_zm0"] = AC.zonal_mean_top(ref.get("w"))
        for k in range(ndir):
            d = AC.direction(k, ref.shape)
            for sgn, tag in ((1.0, "p"), (-1.0, "m")):
                for f in AC.FIELDS:
                    x = base[f] + sgn * eps * d[f]
                    ref.set(f, x)
                    ref.set(f + "n", x)
                ref.quiet(ref.L.ref_rk4)
                data[f"fd_zm{tag}_{k}"] = AC.zonal_mean_top(ref.get("w"))
        data["fd_eps"] = np.array(eps)
    elif a.rk4:
        ref.quiet(ref.L.ref_rk4)
        for n in DYN_FIELDS:
            data["out_" + n] = ref.get(n)
        data["out_buoy_ref"] = ref.get1("buoy_ref_level")
    elif a.pressure:
        ref.quiet(ref.L.ref_pressure)
        for n in ("p_dyn", "aux_u", "aux_v", "aux_w"):
            data["out_" + n] = ref.get(n)
    elif a.iters > 0:
        for it in range(1, a.iters + 1):
            rc = ref.quiet(ref.L.ref_iteration, it, 1 if it == 1 else 0, 0 if a.moist else 1)
            if rc != 0:
                raise SystemExit(f"ref_iteration rc={rc}")
        for n in DYN_FIELDS:
            data["out_" + n] = ref.get(n)
    np.savez(a.out, **data)
    sys.stdout.flush()
    os._exit(0)   # the reference's destructor is not needed; skip interpreter teardown


if __name__ == "__main__":
    main()
