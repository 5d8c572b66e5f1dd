"""Resolved parameter block of the hot path (mirror of ``AtjupParams`` in include/atjup_gpu.h).

The reference reads ~200 ``ATJUP_*`` environment knobs into function-local statics at first use
(e.g. planet/cJupiterModel.h:725-943, planet/RHS_Jup_Turb.cpp:103-117, planet/PressureSolver.h:
168-205). The GPU layer never reads the environment: ``resolve_params`` reads the same variables
with the reference's defaults once, on the host, and hands the device a fixed block, so both arms
of a comparison see identical knobs. Knob values the kernels do not implement are rejected by
``check_supported`` with the knob's name.
"""
from __future__ import annotations

import ctypes
import math
import os
from typing import Mapping

ABI_VERSION = 2

# field ids (include/atjup_gpu.h)
F_T, F_U, F_V, F_W, F_P_DYN, F_P_HYDRO, F_P_STAT, F_RHO_MIX, F_WALL_NUE, F_NUE, \
    F_AUX_U, F_AUX_V, F_AUX_W, F_P_BARO, F_Q_RAD, F_Q_PRECIP, \
    F_H2O, F_H2O_CLOUD, F_H2O_ICE, F_NH3, F_NH3_CLOUD, F_NH3_ICE, \
    F_CH4, F_CH4_CLOUD, F_CH4_ICE, F_H2S, F_NH4SH, F_TKE, F_DIS, \
    F_S_PRECIP_H2O, F_S_PRECIP_H2O_CLOUD, F_S_PRECIP_H2O_ICE, \
    F_S_PRECIP_NH3, F_S_PRECIP_NH3_CLOUD, F_S_PRECIP_NH3_ICE, \
    F_S_PRECIP_CH4, F_S_PRECIP_CH4_CLOUD, F_S_PRECIP_CH4_ICE, \
    F_MASSFLUX_H2S, F_MASSFLUX_NH3, F_MASSFLUX_NH4SH, F_FLUXLIM_NH4SH, \
    F_PROD, F_TKE_SOURCE, F_DIS_SOURCE, F_DIFFLUX_H2S, F_DIFFLUX_NH3, F_DIFFLUX_NH4SH, \
    F_CORIOLIS_FORCE, F_CENTRIFUGAL_FORCE, F_BUOYANCY_FORCE, F_PRESGRAD_FORCE, F_Q_LATENT, \
    F_Q_SENSIBLE = range(54)
F2_VEL_STAR = 0
FIELD_IDS = {
    "t": F_T, "u": F_U, "v": F_V, "w": F_W, "p_dyn": F_P_DYN, "p_hydro": F_P_HYDRO,
    "p_stat": F_P_STAT, "rho_mix": F_RHO_MIX, "wall_nue": F_WALL_NUE, "nue": F_NUE,
    "aux_u": F_AUX_U, "aux_v": F_AUX_V, "aux_w": F_AUX_W, "p_baro": F_P_BARO,
    "Q_rad": F_Q_RAD, "Q_precip": F_Q_PRECIP,
    "h2o": F_H2O, "h2o_cloud": F_H2O_CLOUD, "h2o_ice": F_H2O_ICE,
    "nh3": F_NH3, "nh3_cloud": F_NH3_CLOUD, "nh3_ice": F_NH3_ICE,
    "ch4": F_CH4, "ch4_cloud": F_CH4_CLOUD, "ch4_ice": F_CH4_ICE,
    "h2s": F_H2S, "nh4sh": F_NH4SH, "tke": F_TKE, "dis": F_DIS,
    "S_precip_h2o": F_S_PRECIP_H2O, "S_precip_h2o_cloud": F_S_PRECIP_H2O_CLOUD,
    "S_precip_h2o_ice": F_S_PRECIP_H2O_ICE, "S_precip_nh3": F_S_PRECIP_NH3,
    "S_precip_nh3_cloud": F_S_PRECIP_NH3_CLOUD, "S_precip_nh3_ice": F_S_PRECIP_NH3_ICE,
    "S_precip_ch4": F_S_PRECIP_CH4, "S_precip_ch4_cloud": F_S_PRECIP_CH4_CLOUD,
    "S_precip_ch4_ice": F_S_PRECIP_CH4_ICE,
    "massflux_h2s": F_MASSFLUX_H2S, "massflux_nh3": F_MASSFLUX_NH3,
    "massflux_nh4sh": F_MASSFLUX_NH4SH, "fluxlim_nh4sh": F_FLUXLIM_NH4SH,
    "prod": F_PROD, "tke_source": F_TKE_SOURCE, "dis_source": F_DIS_SOURCE,
    "difflux_h2s": F_DIFFLUX_H2S, "difflux_nh3": F_DIFFLUX_NH3, "difflux_nh4sh": F_DIFFLUX_NH4SH,
    "CoriolisForce": F_CORIOLIS_FORCE, "CentrifugalForce": F_CENTRIFUGAL_FORCE,
    "BuoyancyForce": F_BUOYANCY_FORCE, "PresGradForce": F_PRESGRAD_FORCE,
    "Q_Latent": F_Q_LATENT, "Q_Sensible": F_Q_SENSIBLE,
}
# the output diagnostics of Forces and Latent_Heat
DIAGNOSTICS = ("CoriolisForce", "CentrifugalForce", "BuoyancyForce", "PresGradForce", "Q_Latent",
               "Q_Sensible")

# transported scalars in the order of the physics block (ATJUP_S_*), and the fields whose
# time-level-n copies the RK step keeps (the species, then k*, omega*)
SPECIES = ("h2o", "h2o_cloud", "h2o_ice", "h2s", "nh3", "nh3_cloud", "nh3_ice", "ch4",
           "ch4_cloud", "ch4_ice", "nh4sh")
SCALARS = SPECIES + ("tke", "dis")
S_PRECIP = ("S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice", "S_precip_nh3",
            "S_precip_nh3_cloud", "S_precip_nh3_ice", "S_precip_ch4", "S_precip_ch4_cloud",
            "S_precip_ch4_ice")
TURB_K_EPSILON, TURB_K_OMEGA, TURB_K_OMEGA_SST = 0, 1, 2

# gas ids of atjup_gpu_satadj, in the order cJupiterModel.cpp:1060-1080 calls them
GAS_H2O, GAS_NH3, GAS_CH4 = 0, 1, 2
GAS_IDS = {"H2O": GAS_H2O, "NH3": GAS_NH3, "CH4": GAS_CH4}

SOLVE_SWEEPS, SOLVE_RESIDUAL, SOLVE_SOR = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
BC_RADIUS, BC_THETA, BC_PHI, BC_SOLID, BC_ALL = 1, 2, 4, 8, 15
# the passes of atjup_gpu_iteration_tlm / atjup_gpu_iteration_adjoint, and their nine fields
LIN_PRESSURE, LIN_MIXTURE, LIN_RK4, LIN_BC, LIN_SHAPIRO, LIN_BALANCE = 1, 2, 4, 8, 16, 32
LIN_ALL = 63
LIN_FIELDS = ("t", "u", "v", "w", "p_dyn", "aux_u", "aux_v", "aux_w", "rho_mix")

GAS_CONST_NAMES = ("t_0", "t_00", "ep", "lv", "ls", "C", "L0", "R", "del_alf", "del_bet",
                   "C_i", "L0_i", "del_alf_i", "del_bet_i")

_FIELDS = [
    ("abi_version", ctypes.c_int32), ("im", ctypes.c_int32), ("jm", ctypes.c_int32),
    ("km", ctypes.c_int32),
    ("dr", ctypes.c_double), ("dthe", ctypes.c_double), ("dphi", ctypes.c_double),
    ("dt", ctypes.c_double),
    ("re", ctypes.c_double), ("pr", ctypes.c_double), ("g", ctypes.c_double),
    ("omega", ctypes.c_double), ("u_0", ctypes.c_double), ("t_ref", ctypes.c_double),
    ("L_atm", ctypes.c_double),
    ("r_mix", ctypes.c_double), ("R_mix", ctypes.c_double), ("cp_mix", ctypes.c_double),
    ("Coriolis", ctypes.c_double), ("centrifugal", ctypes.c_double), ("buoyancy", ctypes.c_double),
    ("sinthe_min", ctypes.c_double), ("p_dyn_to_bar", ctypes.c_double),
    ("t_diff_scale", ctypes.c_double),
    ("nd_cor", ctypes.c_double), ("nd_cent", ctypes.c_double), ("nd_buoy", ctypes.c_double),
    ("buoy_scale", ctypes.c_double), ("buoy_ramp", ctypes.c_double),
    ("pgrad_scale", ctypes.c_double), ("rad_coupling", ctypes.c_double),
    ("precip_coupling", ctypes.c_double), ("turb_coupling", ctypes.c_double),
    ("pgrad_wall", ctypes.c_int32), ("pgrad_wrap", ctypes.c_int32),
    ("adiabatic", ctypes.c_int32), ("adiabatic_rho", ctypes.c_int32),
    ("metric_split", ctypes.c_int32), ("coriolis_split", ctypes.c_int32),
    ("hydro_split", ctypes.c_int32), ("cell_hold", ctypes.c_int32),
    ("precip_rho_local", ctypes.c_int32), ("local_rho", ctypes.c_int32),
    ("rho_pdyn", ctypes.c_int32), ("has_nue", ctypes.c_int32), ("has_heating", ctypes.c_int32),
    ("p_dyn_cap", ctypes.c_double), ("press_wall", ctypes.c_int32),
    ("rigid_lid", ctypes.c_int32), ("press_sweeps", ctypes.c_int32),
    ("top_taper", ctypes.c_int32), ("lid_u", ctypes.c_int32), ("pole_fill_rows", ctypes.c_int32),
    ("mount_t_ambient", ctypes.c_int32),
    ("shapiro_inloop", ctypes.c_int32), ("shapiro_strength", ctypes.c_double),
    ("v_massbal_stride", ctypes.c_int32), ("v_massbal_zonal", ctypes.c_int32),
    ("precision", ctypes.c_int32),
    ("cone_proj_stride", ctypes.c_int32), ("cone_proj_margin", ctypes.c_int32),
    ("cone_proj_div", ctypes.c_int32),
]


class AtjupParams(ctypes.Structure):
    _fields_ = _FIELDS


class AtjupSolveOpts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("sweeps", ctypes.c_int32),
                ("max_iter", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("rel_tol", ctypes.c_double), ("omega", ctypes.c_double),
                ("external_rhs", ctypes.c_int32)]


class AtjupSolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("inner_solves", ctypes.c_int32),
                ("rel_residual", ctypes.c_double), ("b_norm", ctypes.c_double),
                ("rel_floor", ctypes.c_double)]


class AtjupGasParams(ctypes.Structure):
    """Mirror of AtjupGasParams: the 14 constants of SaturationAdjustmentJup::run
    (SaturationAdjustment.h:236-243) and the ATJUP_SATADJ_* knobs."""
    _fields_ = [(n, ctypes.c_double) for n in GAS_CONST_NAMES] + [
        (n, ctypes.c_int32) for n in ("conserve", "newton", "evap", "ice_entry", "bergeron",
                                      "freeze", "dry_exit", "reserved")]


class AtjupPhysics(ctypes.Structure):
    """Mirror of AtjupPhysics (full physics in the RK4 step)."""
    _fields_ = [("species_on", ctypes.c_int32), ("turb_on", ctypes.c_int32),
                ("turb_model", ctypes.c_int32), ("turb_buoy", ctypes.c_int32)] + [
        (n, ctypes.c_double) for n in ("species_diff_scale", "sc_h2o", "sc_h2s", "sc_nh3",
                                       "sc_ch4", "sc_nh4sh", "chemical_reaction", "r_p_nh4sh",
                                       "rg_nh4sh", "mue_mix", "re_turb", "nue_max_phys",
                                       "tke_max_phys", "turb_buoy_prt")] + [
        (n, ctypes.c_int32) for n in ("turb_free", "turb_curv", "abl_taper", "turb_wall_omega")] + [
        (n, ctypes.c_double) for n in ("turb_k_bg", "vel_star_max", "abl_height")]


# cJupiterModel's constants of the species transport (cJupiterModel.h:290, 470-477, 594) and the
# closure (Turbulence.h:123); mue_mix, chemical_reaction and re_turb are the values the reference
# derives at start-up with its default composition and parameters.
DEFAULT_PHYSICS = {"species_diff_scale": 0.01, "sc_h2o": 0.61, "sc_h2s": 0.94, "sc_nh3": 0.61,
                   "sc_ch4": 0.99, "sc_nh4sh": 0.7, "r_p_nh4sh": 1.0e-5, "rg_nh4sh": 1170.0,
                   "nue_max_phys": 1.0e5}


def resolve_physics(env: Mapping[str, str] | None = None, constants: Mapping[str, float] | None = None,
                    species_on: bool = True) -> AtjupPhysics:
    """Physics block from the environment with the reference's defaults: ATJUP_TURB (else on
    unless ATJUP_TURB_MODEL / turb_model is empty, none or laminar; cJupiterModel.cpp:61-78), ATJUP_TURB_MODEL
    (k_omega_SST), ATJUP_TURB_BUOY 0, ATJUP_SPECIES_DIFF_SCALE 0.01, ATJUP_NUE_MAX 1e5,
    ATJUP_TKE_MAX 1000, ATJUP_TURB_BUOY_PRT 0.9. constants supplies mue_mix,
    chemical_reaction and re_turb (and may override any DEFAULT_PHYSICS entry)."""
    env = os.environ if env is None else env
    c = dict(DEFAULT_PHYSICS)
    c.update({"mue_mix": 1.0819029080091497e-05, "chemical_reaction": 1.0,
              "re_turb": 2222.2222222222226})
    if constants:
        c.update({k: float(v) for k, v in constants.items() if k in c or k in ("mue_mix", "chemical_reaction", "re_turb")})
    model = env.get("ATJUP_TURB_MODEL", "k_omega_SST")
    turb_model = {"k_epsilon": TURB_K_EPSILON, "k_omega": TURB_K_OMEGA}.get(model, TURB_K_OMEGA_SST)
    if "ATJUP_TURB" in env:
        turb_on = _env(env, "ATJUP_TURB", 1) != 0
    else:
        turb_on = model not in ("", "none", "laminar")
    c["species_diff_scale"] = _env(env, "ATJUP_SPECIES_DIFF_SCALE", c["species_diff_scale"], float)
    c["nue_max_phys"] = _env(env, "ATJUP_NUE_MAX", c["nue_max_phys"], float)
    ph = AtjupPhysics(int(species_on), int(turb_on), turb_model, _env(env, "ATJUP_TURB_BUOY", 0))
    for n in ("species_diff_scale", "sc_h2o", "sc_h2s", "sc_nh3", "sc_ch4", "sc_nh4sh",
              "chemical_reaction", "r_p_nh4sh", "rg_nh4sh", "mue_mix", "re_turb", "nue_max_phys"):
        setattr(ph, n, c[n])
    ph.tke_max_phys = _env(env, "ATJUP_TKE_MAX", 1000.0, float)
    ph.turb_buoy_prt = _env(env, "ATJUP_TURB_BUOY_PRT", 0.9, float)
    ph.turb_free = _env(env, "ATJUP_TURB_FREE", 1)
    ph.turb_curv = int(_env(env, "ATJUP_TURB_CURV", 1) != 0)
    ph.abl_taper = int(_env(env, "ATJUP_ABL_TAPER", 0) != 0)
    ph.turb_wall_omega = _env(env, "ATJUP_TURB_WALL_OMEGA", 1)
    ph.turb_k_bg = _env(env, "ATJUP_TURB_K_BG", 1.0, float)
    ph.vel_star_max = _env(env, "ATJUP_VEL_STAR_MAX", math.sqrt(0.002) * 200.0, float)
    ph.abl_height = float((constants or {}).get("abl_height", 20000.0))
    return ph


class AtjupMicro(ctypes.Structure):
    """Mirror of AtjupMicro (the loop's radiation, precipitation and chemistry)."""
    _fields_ = [(n, ctypes.c_int32) for n in ("radiation_on", "precip_on", "nh4sh_eq", "satadj_on",
                                               "solar_on", "rad_bottom", "precip_coupling_on",
                                               "diagnostics_on", "costhe_abs", "qheat_scale",
                                               "pad")] + [
        (n, ctypes.c_double) for n in ("F_int", "S_solar", "albedo_bond", "x_H2", "x_He",
                                       "cia_strength", "opacity_strength", "solar_strength",
                                       "sw_tau_per_bar", "precip_rate_scale", "m_nh3", "m_h2s",
                                       "m_nh4sh", "D_nh3", "D_h2s", "D_nh4sh",
                                       "polar_divisor_floor", "t_0_nh4sh", "t_00_nh4sh")] + [
        ("cc", ctypes.c_double * 8), ("gas", AtjupGasParams * 3)]


# cJupiterModel's radiation constants (cJupiterModel.h:1109-1118), molar masses (255-270) and the
# diffusivities mue / (rg sc) of the chemistry fluxes (ChemistryJup.h:383-385) with its defaults
# (the active set of cJupiterModel.h:385-387 has mue_nh4sh = 0, so NH4SH does not diffuse).
DEFAULT_MICRO = {"F_int": 5.4, "S_solar": 50.5, "albedo_bond": 0.343, "x_H2": 0.863,
                 "x_He": 0.134, "m_nh3": 17.03052, "m_h2s": 34.08088, "m_nh4sh": 51.1114,
                 "D_nh3": 0.92e-5 / (817.0 * 0.61), "D_h2s": 1.3e-5 / (949.0 * 0.94),
                 "D_nh4sh": 0.0, "polar_divisor_floor": 0.4, "t_0_nh4sh": 230.0,
                 "t_00_nh4sh": 200.0,
                 # Latent_Heat's Clausius-Clapeyron pairs (cJupiterModel.h:222-240)
                 "coeff_h2o_A": -4961.04, "coeff_h2o_B": 13.0662, "coeff_h2o_A_i": -4961.04,
                 "coeff_h2o_B_i": 13.0662, "coeff_nh3_A": -2836.56, "coeff_nh3_B": 11.7271,
                 "coeff_nh3_A_i": -2836.56, "coeff_nh3_B_i": 11.7271}
CC_NAMES = ("coeff_h2o_A", "coeff_h2o_B", "coeff_h2o_A_i", "coeff_h2o_B_i", "coeff_nh3_A",
            "coeff_nh3_B", "coeff_nh3_A_i", "coeff_nh3_B_i")


def resolve_micro(env: Mapping[str, str] | None = None, constants: Mapping[str, float] | None = None,
                  gases: Mapping | None = None) -> AtjupMicro:
    """Microphysics block from the environment with the reference's defaults (ATJUP_RADIATION 1,
    ATJUP_PRECIP 1, ATJUP_NH4SH_EQ 1, ATJUP_SOLAR 1, ATJUP_RAD_BOTTOM 0, ATJUP_PRECIP_COUPLING 1,
    ATJUP_CIA_STRENGTH 3.9, ATJUP_OPACITY_STRENGTH 1, ATJUP_SOLAR_STRENGTH 1,
    ATJUP_SW_TAU_PER_BAR 1, ATJUP_PRECIP_SCALE 1, ATJUP_COSTHE_ABS 0, ATJUP_QHEAT_SCALE 0, the
    Forces / Latent_Heat diagnostics on); constants override DEFAULT_MICRO, gases
    the three gas constant sets (DEFAULT_GASES)."""
    env = os.environ if env is None else env
    c = dict(DEFAULT_MICRO)
    if constants:
        c.update({k: float(v) for k, v in constants.items() if k in c})
    mc = AtjupMicro()
    mc.radiation_on = int(_env(env, "ATJUP_RADIATION", 1) != 0)
    mc.precip_on = int(_env(env, "ATJUP_PRECIP", 1) != 0)
    mc.nh4sh_eq = int(_env(env, "ATJUP_NH4SH_EQ", 1) != 0)
    mc.satadj_on = 1
    mc.solar_on = _env(env, "ATJUP_SOLAR", 1)
    mc.rad_bottom = _env(env, "ATJUP_RAD_BOTTOM", 0)
    mc.precip_coupling_on = int(_env(env, "ATJUP_PRECIP_COUPLING", 1.0, float) != 0.0)
    mc.cia_strength = _env(env, "ATJUP_CIA_STRENGTH", 3.9, float)
    mc.opacity_strength = _env(env, "ATJUP_OPACITY_STRENGTH", 1.0, float)
    mc.solar_strength = _env(env, "ATJUP_SOLAR_STRENGTH", 1.0, float)
    mc.sw_tau_per_bar = _env(env, "ATJUP_SW_TAU_PER_BAR", 1.0, float)
    mc.precip_rate_scale = _env(env, "ATJUP_PRECIP_SCALE", 1.0, float)
    mc.diagnostics_on = 1
    mc.costhe_abs = int(_env(env, "ATJUP_COSTHE_ABS", 0) != 0)
    mc.qheat_scale = int(_env(env, "ATJUP_QHEAT_SCALE", 0) != 0)
    for q, n in enumerate(CC_NAMES):
        mc.cc[q] = c[n]
    for n in ("F_int", "S_solar", "albedo_bond", "x_H2", "x_He", "m_nh3", "m_h2s", "m_nh4sh",
              "D_nh3", "D_h2s", "D_nh4sh", "polar_divisor_floor", "t_0_nh4sh", "t_00_nh4sh"):
        setattr(mc, n, c[n])
    gases = gases or DEFAULT_GASES
    for q, g in enumerate(("H2O", "NH3", "CH4")):
        mc.gas[q] = resolve_gas(gases[g], env)
    return mc


class AtjupMca(ctypes.Structure):
    """Mirror of AtjupMca (the moist convective adjustment)."""
    _fields_ = [(n, ctypes.c_int32) for n in ("stride", "ledoux", "loading", "interior",
                                               "max_pass", "pad")] + [
        (n, ctypes.c_double) for n in ("relax", "ep_h2s", "L_nh4sh")]


class AtjupMcaStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("columns", "layers", "moist_triggers",
                                               "dry_triggers", "unstable_t", "held", "skipped")] + [
        ("max_passes", ctypes.c_int32), ("pad", ctypes.c_int32)]


# ChemistryJup::nh4sh_formation_heat (ChemistryJup.h:283): 4705 ln(10) R_univ / m_nh4sh [J/kg]
NH4SH_FORMATION_HEAT = 4705.0 * math.log(10.0) * 8314.46 / 51.1114
EP_H2S = 15.35                      # cJupiterModel.h:418


def resolve_mca(env: Mapping[str, str] | None = None) -> AtjupMca:
    """The moist convective adjustment with the reference's defaults (cJupiterModel.cpp:115-124,
    ConvectiveAdjustment.h:403-420, cJupiterModel.h:1038-1042): ATJUP_MCA 1 (every iteration),
    ATJUP_MCA_LEDOUX 1, ATJUP_MCA_LOADING 1, ATJUP_MCA_INTERIOR 1, ATJUP_MCA_PASSES 64,
    ATJUP_MCA_RELAX 1; NH4SH carries its heat of formation when ATJUP_NH4SH_EQ is on."""
    env = os.environ if env is None else env
    m = AtjupMca()
    m.stride = max(0, _env(env, "ATJUP_MCA", 1))
    m.ledoux = int(_env(env, "ATJUP_MCA_LEDOUX", 1) != 0)
    m.loading = int(_env(env, "ATJUP_MCA_LOADING", 1) != 0)
    m.interior = int(_env(env, "ATJUP_MCA_INTERIOR", 1) != 0)
    passes = _env(env, "ATJUP_MCA_PASSES", 64)
    m.max_pass = passes if passes > 0 else 64
    m.relax = min(1.0, max(0.0, _env(env, "ATJUP_MCA_RELAX", 1.0, float)))
    m.ep_h2s = EP_H2S
    m.L_nh4sh = NH4SH_FORMATION_HEAT if _env(env, "ATJUP_NH4SH_EQ", 1) != 0 else 0.0
    return m


class AtjupSatStats(ctypes.Structure):
    _fields_ = [("adjusted", ctypes.c_int64), ("not_converged", ctypes.c_int64),
                ("dry_exits", ctypes.c_int64)]


# The 14 constants of each gas as cJupiterModel derives them at start-up with its default
# composition and vapour-pressure sets (InitValues_Jup.cpp:880-950, ATPhys.h:55-67), in
# GAS_CONST_NAMES order. A host model passes its own; these serve the synthetic workloads.
DEFAULT_GASES = {
    "H2O": (273.15, 210.15, 7.651416982890988, 2500900.0, 2833900.0, 25.096, 3148.2, 461.52,
            0.0, -0.0087, -1.962499, 2641.4013, 1.629479, -0.003361398),
    "NH3": (195.5, 140.0, 7.232930612074716, 1372000.0, 1832000.0, 196.077451, 3586.5634,
            488.21, -15.978352, 0.02837146, 16.086062, 1857.9898, 0.098768, -0.001179989),
    "CH4": (90.69, 67.36, 6.813102176498581, 511000.0, 511000.0, 1.627, 553.1, 518.28, 1.002,
            -0.0041, 1.627, 553.1, 1.002, -0.0041),
}


def resolve_gas(constants, env: Mapping[str, str] | None = None) -> AtjupGasParams:
    """Gas block from the 14 constants (sequence in GAS_CONST_NAMES order, or a mapping) and the
    ATJUP_SATADJ_* knobs with cJupiterModel's defaults (SaturationAdjustment.h:277-307,
    cJupiterModel.h:1045-1057): CONSERVE 1, NEWTON 1, EVAP 1, ICE_ENTRY 0, BERGERON 2,
    FREEZE 0, DRY_EXIT 1."""
    env = os.environ if env is None else env
    if isinstance(constants, Mapping):
        vals = [float(constants[n]) for n in GAS_CONST_NAMES]
    else:
        vals = [float(v) for v in constants]
    if len(vals) != len(GAS_CONST_NAMES):
        raise ValueError(f"expected {len(GAS_CONST_NAMES)} gas constants, got {len(vals)}")
    knobs = [int(_env(env, "ATJUP_SATADJ_CONSERVE", 1) != 0),
             int(_env(env, "ATJUP_SATADJ_NEWTON", 1) != 0),
             int(_env(env, "ATJUP_SATADJ_EVAP", 1) != 0),
             int(_env(env, "ATJUP_SATADJ_ICE_ENTRY", 0) != 0),
             int(_env(env, "ATJUP_SATADJ_BERGERON", 2)),
             int(_env(env, "ATJUP_SATADJ_FREEZE", 0) != 0),
             int(_env(env, "ATJUP_SATADJ_DRY_EXIT", 1) != 0), 0]
    return AtjupGasParams(*vals, *knobs)


# Mixture constants the reference derives at start-up from its default composition
# (ChemistryJup::ThermalPropertiesJup with ATJUP_COMPOSITION=1, ChemistryJup.h:545-650).
DEFAULT_MIXTURE = {"r_mix": 1.2843999999999998, "R_mix": 3531.1847352206946,
                   "cp_mix": 11810.757033551794}


def _env(env: Mapping[str, str], name: str, default, cast=int):
    v = env.get(name)
    if v is None:
        return default
    try:
        return cast(v)
    except ValueError:
        # atoi / atof of a non-numeric string is 0 in the reference
        return cast(0)


def resolve_params(env: Mapping[str, str] | None = None, *, im=41, jm=181, km=361,
                   constants: Mapping[str, float] | None = None, iter_n: int = 0,
                   has_nue: bool = False, has_heating: bool = False) -> AtjupParams:
    """Resolve every knob that selects a hot-path branch, with the reference's defaults.

    ``constants`` overrides the model constants (re, pr, g, omega, u_0, t_ref, L_atm, r_mix,
    R_mix, cp_mix, Coriolis, centrifugal, buoyancy, dt) -- a driver passes its member values.
    """
    env = os.environ if env is None else env
    c = {"re": 1000.0, "pr": 0.69, "g": 25.92, "omega": 0.000176, "u_0": 100.0, "t_ref": 165.0,
         "L_atm": 140.0, "Coriolis": 1.0, "centrifugal": 1.0, "buoyancy": 1.0}
    c.update(DEFAULT_MIXTURE)
    c["dt"] = _env(env, "ATJUP_DT", 0.005, float)                     # cJupiterModel.cpp:106
    if constants:
        c.update(constants)
    p = AtjupParams()
    p.abi_version = ABI_VERSION
    p.im, p.jm, p.km = im, jm, km
    p.dr = 0.025                                                       # cJupiterModel.cpp:172
    p.dthe = 1.0 / (180.0 / math.pi)                                   # cJupiterModel.cpp:173
    p.dphi = 1.0 / (180.0 / math.pi)
    for k in ("dt", "re", "pr", "g", "omega", "u_0", "t_ref", "L_atm", "r_mix", "R_mix",
              "cp_mix", "Coriolis", "centrifugal", "buoyancy"):
        setattr(p, k, float(c[k]))

    geo_balance = _env(env, "ATJUP_GEO_BALANCE", 1) != 0               # cJupiterModel.h:857
    smin = _env(env, "ATJUP_SINTHE_MIN", 0.55, float)                  # cJupiterModel.h:1121
    p.sinthe_min = smin if 0.0 < smin < 1.0 else 0.55
    pdyn_units = _env(env, "ATJUP_PDYN_UNITS", 1) != 0                 # cJupiterModel.h:1156
    p.p_dyn_to_bar = p.r_mix * p.u_0 * p.u_0 * 1.0e-5 if pdyn_units else 1.0
    p.t_diff_scale = _env(env, "ATJUP_T_DIFF_SCALE", 0.01, float)      # cJupiterModel.h:268

    # body-force scales, RHS_Jup_Turb.cpp:323-346
    nd_all = _env(env, "ATJUP_NONDIM", 0)
    nd_cor_on = _env(env, "ATJUP_ND_COR", 1 if geo_balance else -1)
    nd_cent_on = _env(env, "ATJUP_ND_CENT", -1)
    nd_buoy_on = _env(env, "ATJUP_ND_BUOY", -1)
    L_m = p.L_atm * 1.0e3
    p.nd_cor = L_m / p.u_0 if (nd_cor_on if nd_cor_on >= 0 else nd_all) != 0 else 1.0
    p.nd_cent = L_m * L_m / (p.u_0 * p.u_0) if (nd_cent_on if nd_cent_on >= 0 else nd_all) != 0 else 1.0
    p.nd_buoy = 1.0e5 * L_m / (p.u_0 * p.u_0) if (nd_buoy_on if nd_buoy_on >= 0 else nd_all) != 0 else 1.0
    p.buoy_scale = _env(env, "ATJUP_BUOY_SCALE", 1.0, float)
    ramp_iters = _env(env, "ATJUP_BUOY_RAMP_ITERS", 0)
    p.buoy_ramp = min(1.0, float(iter_n) / float(ramp_iters)) if ramp_iters > 0 else 1.0
    p.pgrad_scale = _env(env, "ATJUP_PGRAD_SCALE", 1.0, float)
    p.rad_coupling = _env(env, "ATJUP_RAD_COUPLING", 1.0, float)
    p.precip_coupling = _env(env, "ATJUP_PRECIP_COUPLING", 1.0, float)
    p.turb_coupling = _env(env, "ATJUP_TURB_COUPLING", 1.0, float)
    p.pgrad_wall = int(_env(env, "ATJUP_PGRAD_WALL", 1) != 0)
    p.pgrad_wrap = int(_env(env, "ATJUP_PGRAD_WRAP", 1) != 0)
    p.adiabatic = int(_env(env, "ATJUP_ADIABATIC", 1) != 0)
    p.adiabatic_rho = int(_env(env, "ATJUP_ADIABATIC_RHO", 1) != 0)
    p.metric_split = int(_env(env, "ATJUP_METRIC_SPLIT", 1) != 0)
    p.coriolis_split = int(_env(env, "ATJUP_CORIOLIS_SPLIT", 1) != 0 and p.metric_split)
    hs = env.get("ATJUP_HYDRO_SPLIT")
    p.hydro_split = int((int(hs) if hs is not None else nd_all) != 0)
    p.cell_hold = int(_env(env, "ATJUP_CELL_HOLD", 1 if geo_balance else 0) != 0)
    p.precip_rho_local = int(_env(env, "ATJUP_PRECIP_RHO_LOCAL", 1) != 0)
    p.local_rho = int(_env(env, "ATJUP_LOCAL_RHO", 1) != 0)
    p.rho_pdyn = int(_env(env, "ATJUP_RHO_PDYN", 0 if geo_balance else 1) != 0)
    p.has_nue = int(bool(has_nue))
    p.has_heating = int(bool(has_heating))

    # pressure solver, PressureSolver.h:168-205
    p.p_dyn_cap = _env(env, "ATJUP_PDYN_CAP", 0.2, float)
    p.press_wall = int(_env(env, "ATJUP_PRESS_WALL", 1) != 0)
    p.rigid_lid = int(_env(env, "ATJUP_BC_RIGID_LID", 1) != 0)
    sw = _env(env, "ATJUP_PRESS_SWEEPS", 1)
    p.press_sweeps = sw if sw > 0 else 1

    # boundary conditions, BoundaryConditions.h:100-140, BC_Jup.h:77-90
    p.top_taper = _env(env, "ATJUP_BC_TOP_TAPER", 3)
    p.lid_u = _env(env, "ATJUP_BC_LID_U", p.rigid_lid)
    p.pole_fill_rows = 2 if _env(env, "ATJUP_BC_POLE_FILL", 1) != 0 else 0
    p.mount_t_ambient = _env(env, "ATJUP_MOUNT_T_AMBIENT", 1)

    # per-iteration glue, cJupiterModel.cpp:44-46 and cJupiterModel.h:937
    p.shapiro_inloop = _env(env, "ATJUP_VEL_SHAPIRO_INLOOP", 0)
    p.shapiro_strength = _env(env, "ATJUP_SHAPIRO_STRENGTH", 1.0, float)
    p.v_massbal_stride = _env(env, "ATJUP_V_MASSBAL_STRIDE", 1)
    vortex = _env(env, "ATJUP_VORTEX", 1) != 0
    p.v_massbal_zonal = int(_env(env, "ATJUP_V_MASSBAL_ZONAL", 1 if vortex else 0) != 0)
    p.precision = PREC_FP64
    # the in-loop projection around the obstacle, cJupiterModel.h:919-933 (a stride or H at or
    # below zero switches its part off, as the reference's "> 0" tests do)
    p.cone_proj_stride = max(0, _env(env, "ATJUP_CONE_PROJ_STRIDE", 10))
    p.cone_proj_margin = _env(env, "ATJUP_CONE_PROJ_MARGIN", 40)
    p.cone_proj_div = max(0, _env(env, "ATJUP_CONE_PROJ_DIV", 3))
    return p


# Knobs whose non-default values select branches this implementation does not provide.
_UNSUPPORTED = {
    "ATJUP_BC_PHI_PERIODIC": ("1", "the periodic phi seam is the only seam implemented"),
    "ATJUP_PRESS_SRC": ("1", "only the projection source div(aux) is implemented"),
    "ATJUP_PRESS_INCR": ("0", "the defect-correction source is not implemented"),
    "ATJUP_PRESS_LINE": ("0", "the reference line pass is replaced by the residual solver"),
    "ATJUP_PRESS_BAROTROPIC": ("0", "the reference barotropic pass is replaced by the residual solver"),
    "ATJUP_PBARO_FOLLOW": ("0", "p_baro follow is not implemented"),
    "ATJUP_T_LIMITER": ("0", "the temperature limiter is not implemented"),
    "ATJUP_BUOY_PDYN": ("0", "the buoyancy reads p_stat only"),
    "ATJUP_PHYDRO_TOP_TAPER": ("0", "the p_hydro top taper is not implemented"),
    "ATJUP_COSTHE_ABS": ("0", "signed cos(theta) only"),
    "ATJUP_SPECIES_DIVU": ("0", "species flux form is not implemented"),
    "ATJUP_BC_SEAM_DAMP": ("0", "seam damping applies only to the non-periodic seam"),
    "ATJUP_BC_T_LID_PIN": ("0", "lid temperature pin is not implemented"),
    "ATJUP_BC_MOUNT_COPY": ("0", "solid cells use the 2-point extrapolation"),
    "ATJUP_BC_RADIUS_COPY": ("0", "radial walls use the 2-point Neumann form"),
    "ATJUP_BC_BOTTOM_FORM": ("0", "radial walls use the 2-point Neumann form"),
    "ATJUP_BC_POLE_COPY": ("1", "pole rows are copies"),
    "ATJUP_DAMP_PDYN": ("0", "no Shapiro pass on p_dyn in the loop"),
    "ATJUP_HYDRO_REF": ("0", "the hydrostatic integral runs upward from the base"),
    "ATJUP_MCA_SMOOTH": ("0", "the latitude-smoothed stability search is not implemented"),
    "ATJUP_CHEM_MOLAR_CONC": ("0", "the rate law's molar-concentration form is not implemented"),
    "ATJUP_CHEM_GATE_ZERO": ("1", "the rate law keeps its last rate outside the window only with 1"),
    "ATJUP_MCA_PHASE": ("0", "the temperature-split phase rule is not implemented"),
    "ATJUP_CHROM": ("0", "the chromophore tracer is not implemented"),
    "ATJUP_CONV_ADJ": ("0", "the dry convective adjustment is not implemented"),
}


def check_supported(env: Mapping[str, str] | None = None) -> list[str]:
    """Names (with reasons) of set knobs whose values the kernels do not implement."""
    env = os.environ if env is None else env
    bad = []
    for name, (ok, why) in _UNSUPPORTED.items():
        v = env.get(name)
        if v is not None and str(int(float(v)) if v.strip().lstrip("-").replace(".", "", 1).isdigit() else v) != ok:
            bad.append(f"{name}={v}: {why}")
    # the dry convective adjustment defaults to ATJUP_NONDIM (cJupiterModel.cpp:125-131)
    if env.get("ATJUP_CONV_ADJ") is None and _env(env, "ATJUP_NONDIM", 0) != 0:
        bad.append("ATJUP_NONDIM set without ATJUP_CONV_ADJ=0: the dry convective adjustment it "
                   "switches on is not implemented")
    return bad
