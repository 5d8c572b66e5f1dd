"""The benchmark configurations' seeded initial states, applied to the reference's own initial
state, and a dump of everything a model needs to start from that state.

TEST AND CPU-BASELINE INFRASTRUCTURE: used by tests/ (parity runs of the two benchmark
configurations against the reference), by bench.py's reference arm and CPU-baseline leg (which
time the reference from this state), and by bench.py to hand the same state, byte for byte, to
the GPU arm. The state comes from the reference built from its sources (oracle/_ref): its
initialisation chain (cJupiterModel.cpp:392-745: temperature profile, static pressure, jets,
geostrophic balance, vortex, SeaMount cone) is not part of the time-step path.

Recipes (model units: velocities / u_0, temperature / t_ref; the reference's velocity names are
u radial, v colatitudinal, w zonal):

* dry (config "dry"): knobs DRY_ENV; the species and their n copies zeroed; i.i.d. Gaussian noise
  on the fluid cells, drawn from one Philox stream in this order: zonal w ~ N(0, 0.1 m/s),
  meridional v ~ N(0, 0.1 m/s), radial u ~ N(0, 0.01 m/s), T ~ N(0, 0.05 K); none inside the
  obstacle; the phi seam k = km-1 repeats k = 0; then the n copies (restoreVar).
* full physics (config "phys"): knobs PHYS_ENV (the reference's default physics: k-omega SST,
  radiation, precipitation, the saturation adjustments, the NH4SH equilibrium, the moist
  convective adjustment every iteration); the dynamics noise above; H2O and NH3 vapour at 90 % of
  the saturation density rho_mix ep E(T) / p of the cell (E the liquid vapour-pressure set above
  the gas's t_0, the ice set below; ATPhys.h:279-282, SaturationAdjustment.h:414-434) times
  U(0.95, 1.05), capped at 2 % of the mixture density (the saturation density grows without
  bound in the deep hot levels), their cloud and ice zero; k = 1e-4 m2/s2 x U(0.5, 1.5) and
  omega = 1e-3 1/s x U(0.5, 1.5) (k* = k / u_0^2, omega* = omega L_atm / u_0); CH4, H2S and NH4SH
  as the reference initialises them; then the n copies.

    python oracle/baseline_state.py OUT.npz --config dry|phys [--threads T]
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from ref_model import RefModel  # noqa: E402

DYN_SEED = 20261203
PHYS_SEED = 20261207

# The dry configuration: obstacle on, microphysics / radiation / turbulence / MCA off, in-loop
# 4th-order Shapiro on u, v, w, the projection around the obstacle at the reference's default
# stride (every 10 iterations).
DRY_ENV = {
    "ATJUP_NO_SEAMOUNT": "0", "ATJUP_PRECIP": "0", "ATJUP_RADIATION": "0", "ATJUP_TURB": "0",
    "ATJUP_MCA": "0", "ATJUP_NH4SH_EQ": "0", "ATJUP_CONE_PROJ_STRIDE": "10",
    "ATJUP_VEL_SHAPIRO_ORDER": "4", "ATJUP_VEL_SHAPIRO_INLOOP": "1",
    "ATJUP_RESTART_STRIDE": "0", "ATJUP_VTK_STRIDE": "100000", "ATJUP_PANORAMA_STRIDE": "100000",
}
# The reference's default full physics on the dry configuration's knobs.
PHYS_ENV = {**DRY_ENV, "ATJUP_TURB": "1", "ATJUP_PRECIP": "1", "ATJUP_RADIATION": "1",
            "ATJUP_NH4SH_EQ": "1", "ATJUP_MCA": "1"}
ENVS = {"dry": DRY_ENV, "phys": PHYS_ENV}

CONSTS = ("dt", "re", "pr", "g", "omega", "u_0", "t_ref", "L_atm", "r_mix", "R_mix", "cp_mix",
          "Coriolis", "centrifugal", "buoyancy")
PHYS_CONSTS = ("species_diff_scale", "sc_h2o", "sc_h2s", "sc_nh3", "sc_ch4", "sc_nh4sh",
               "chemical_reaction", "r_p_nh4sh", "rg_nh4sh", "mue_mix", "re_turb")
MICRO_CONSTS = ("m_nh3", "m_h2s", "m_nh4sh", "D_nh3", "D_h2s", "D_nh4sh", "polar_divisor_floor",
                "t_0_nh4sh", "t_00_nh4sh", "coeff_h2o_A", "coeff_h2o_B", "coeff_h2o_A_i",
                "coeff_h2o_B_i", "coeff_nh3_A", "coeff_nh3_B", "coeff_nh3_A_i", "coeff_nh3_B_i",
                "rad_F_int", "rad_S_solar", "rad_albedo_bond", "rad_x_H2", "rad_x_He",
                "rad_cia_strength", "rad_opacity_strength", "rad_solar", "rad_solar_strength",
                "rad_sw_tau_per_bar", "rad_bottom", "precip_rate_scale", "precip_coupling_on")
GASES = ("H2O", "NH3", "CH4")
DYN_FIELDS = ("t", "u", "v", "w", "p_dyn", "p_hydro", "p_stat", "rho_mix", "wall_nue", "aux_u",
              "aux_v", "aux_w")
PHYS_FIELDS = ("h2o", "h2o_cloud", "h2o_ice", "h2s", "nh3", "nh3_cloud", "nh3_ice", "ch4",
               "ch4_cloud", "ch4_ice", "nh4sh", "tke", "dis")
# every field the full-physics iteration reads
ITER_FIELDS = DYN_FIELDS + PHYS_FIELDS + tuple(n + "n" for n in PHYS_FIELDS) + (
    "nue", "prod", "tke_source", "dis_source", "Q_rad", "Q_precip", "massflux_h2s",
    "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "difflux_h2s", "difflux_nh3",
    "difflux_nh4sh", "S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice", "S_precip_nh3",
    "S_precip_nh3_cloud", "S_precip_nh3_ice", "S_precip_ch4", "S_precip_ch4_cloud",
    "S_precip_ch4_ice")


def _seam(a: np.ndarray) -> np.ndarray:
    a[:, :, -1] = a[:, :, 0]
    return a


def perturb_dynamics(ref: RefModel, seed: int = DYN_SEED) -> None:
    """The dry recipe's noise on t, u, v, w (fluid cells), then the n copies."""
    rng = np.random.Generator(np.random.Philox(seed))
    shape = ref.shape
    fluid = ref.solid() == 0
    u_0, t_ref = ref.scalar("u_0"), ref.scalar("t_ref")
    for name, sd in (("w", 0.1 / u_0), ("v", 0.1 / u_0), ("u", 0.01 / u_0), ("t", 0.05 / t_ref)):
        x = ref.get(name) + np.where(fluid, rng.normal(0.0, sd, shape), 0.0)
        _seam(x)
        ref.set(name, x)
        ref.set(name + "n", x)


def saturation_density(T_K, p_bar, rho, cst, ice):
    """rho ep E(T) / p with E = exp(C + (-L0 / T + del_alf ln T + del_bet T) / (1e-3 R)) [bar]
    (ATPhys.h:49-52, 279-282); cst = the 14 constants of SaturationAdjustmentJup::run."""
    t_0, t_00, ep, lv, ls, C, L0, R, da, db, Ci, L0i, dai, dbi = cst
    C_, L0_, da_, db_ = (Ci, L0i, dai, dbi) if ice else (C, L0, da, db)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        E = np.exp(C_ + (-L0_ / T_K + da_ * np.log(T_K) + db_ * T_K) / (1e-3 * R))
        return rho * ep * E / p_bar


def moist_recipe(ref: RefModel, seed: int = PHYS_SEED) -> None:
    """The full-physics recipe's vapour, condensates, k* and omega* (fluid cells), then the n
    copies of every species and of k*, omega*."""
    rng = np.random.Generator(np.random.Philox(seed))
    shape = ref.shape
    fluid = ref.solid() == 0
    T = ref.get("t") * ref.scalar("t_ref")
    p, rho = ref.get("p_stat"), ref.get("rho_mix")
    for gas in ("H2O", "NH3"):
        cst = ref.gas_consts(gas)
        ice = T <= cst[0]
        sat = np.where(ice, saturation_density(T, p, rho, cst, True),
                       saturation_density(T, p, rho, cst, False))
        sat = np.where(np.isfinite(sat) & (sat > 0), np.minimum(sat, 0.02 * rho), 0.0)
        name = gas.lower()
        vap = 0.9 * sat * rng.uniform(0.95, 1.05, shape)
        ref.set(name, _seam(np.where(fluid, vap, ref.get(name))))
        for c in ("_cloud", "_ice"):
            ref.set(name + c, np.where(fluid, 0.0, ref.get(name + c)))
    u_0, L_atm = ref.scalar("u_0"), ref.scalar("L_atm")
    k = 1e-4 / u_0 ** 2 * rng.uniform(0.5, 1.5, shape)
    om = 1e-3 * (L_atm * 1e3 / u_0) * rng.uniform(0.5, 1.5, shape)
    ref.set("tke", _seam(np.where(fluid, k, ref.get("tke"))))
    ref.set("dis", _seam(np.where(fluid, om, ref.get("dis"))))
    for n in PHYS_FIELDS:
        ref.set(n + "n", ref.get(n))


def describe(config: str) -> str:
    """One line naming the state, identical for every arm that starts from it."""
    what = ("dry recipe: Philox(%d) noise on w, v, u, t" % DYN_SEED if config == "dry" else
            "full-physics recipe: Philox(%d) noise on w, v, u, t; Philox(%d) vapour at 90 %% of "
            "saturation x U(0.95, 1.05), k, omega" % (DYN_SEED, PHYS_SEED))
    return ("the reference's own initial state (its initialisation, %s knobs) with the %s "
            "(oracle/baseline_state.py)" % (config, what))


def make(config: str, out_dir: str, threads: int = 0, cls=RefModel, env_extra=None) -> RefModel:
    """The reference model (an instance of cls, a RefModel) with the configuration's knobs
    (plus env_extra), initialised by the reference and carrying the configuration's seeded
    initial state."""
    env = {**ENVS[config], **(env_extra or {})}
    ref = cls(env, out_dir, threads=threads, zero_species=(config == "dry"))
    perturb_dynamics(ref)
    if config == "phys":
        moist_recipe(ref)
    return ref


def record(ref: RefModel, data: dict, moist: bool) -> None:
    """Everything a model needs to start from ref's current state: the grid (grid_*), the model
    constants (const_*), and every field the iteration reads (in_*); with moist also the physics
    and microphysics constants, the gas constants, vel_star and the level heights."""
    shape = ref.shape
    data["grid_rad"] = ref.get1("rad")
    data["grid_the"] = ref.get1("the")
    data["grid_solid"] = ref.solid()
    data["grid_topo"] = ref.topo()
    if ref.scalar("cell_hold") == 1.0:
        data["grid_cell_vbar0"] = ref.get1("cell_vbar0")
        data["grid_cell_ubar0"] = ref.get1("cell_ubar0")
    for c in CONSTS:
        data["const_" + c] = np.array(ref.scalar(c))
    for n in (ITER_FIELDS if moist else DYN_FIELDS):
        data["in_" + n] = ref.get(n)
    if ref.scalar("has_p_baro") == 1.0:
        data["in_p_baro"] = ref.get1("p_baro").reshape(shape)
    if not moist:
        return
    data["in_vel_star"] = ref.get1("vel_star").reshape(shape[1], shape[2])
    data["in_layer_heights"] = ref.get1("layer_heights").astype(np.float32)
    for c in MICRO_CONSTS:
        data["micro_" + c] = np.array(ref.scalar(c))
    for c in PHYS_CONSTS:
        data["phys_" + c] = np.array(ref.scalar(c))
    data["knobd_abl_height"] = np.array(ref.L.ref_knob_d(b"abl_height"))
    for gas in GASES:
        data["gas_" + gas] = ref.gas_consts(gas)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--config", choices=sorted(ENVS), required=True)
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    ref = make(a.config, tempfile.mkdtemp(prefix="atjup_state_") + "/run",
               threads=a.threads or os.cpu_count() or 1)
    data = {"config": np.array(a.config)}
    record(ref, data, moist=(a.config == "phys"))
    np.savez(a.out, **data)
    sys.stdout.flush()
    os._exit(0)   # the reference's destructor is not needed; skip interpreter teardown


if __name__ == "__main__":
    main()
