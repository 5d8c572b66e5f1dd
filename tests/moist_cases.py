"""Shared set-up of the full-physics iteration tests: the reference's moist iterations and a
small synthetic moist shell, as (params, physics, micro, grid, fields), and a GpuModel built from
them. Test infrastructure only."""
import numpy as np

from atjup_b200 import synthetic
from atjup_b200.params import DEFAULT_GASES, SCALARS, SPECIES, resolve_micro, resolve_physics
from helpers import dump_fields, dump_grid, dump_params, ref_dump, synthetic_case
from oracle_bridge import MOIST_ENV

RENAME = {"rad_F_int": "F_int", "rad_S_solar": "S_solar", "rad_albedo_bond": "albedo_bond",
          "rad_x_H2": "x_H2", "rad_x_He": "x_He"}
PROGNOSTIC = ("t", "u", "v", "w", "p_dyn") + SCALARS


def env_of(extra) -> dict:
    """MOIST_ENV with the "--env KEY=VALUE" pairs of a ref_dump flag list applied"""
    env = dict(MOIST_ENV)
    for flag, kv in zip(extra, extra[1:]):
        if flag == "--env":
            k, v = kv.split("=", 1)
            env[k] = v
    return env


def ref_iters_case(iters=3, *extra):
    d = ref_dump("--phys-iters", str(iters), *extra)
    env = env_of(extra)
    P = dump_params(d, env=env)
    P.has_nue = 1
    P.has_heating = 1
    MC = resolve_micro(env, {RENAME.get(k[6:], k[6:]): float(v) for k, v in d.items()
                             if k.startswith("micro_")},
                       {g: tuple(d["gas_" + g]) for g in ("H2O", "NH3", "CH4")})
    consts = {k[5:]: float(v) for k, v in d.items() if k.startswith("phys_")}
    consts["abl_height"] = float(d["knobd_abl_height"])
    return d, P, resolve_physics(env, consts), MC, dump_grid(d), dump_fields(d)


def synthetic_moist_case(im, jm, km, seed=41, env=None):
    env = MOIST_ENV if env is None else env
    P, g, f = synthetic_case(im, jm, km, seed=seed, env=env)
    P.has_nue = 1
    P.has_heating = 1
    s = dict(f)
    s["solid"] = g["solid"]
    f.update(synthetic.physics(s, DEFAULT_GASES, seed=seed + 1))
    shape = f["t"].shape
    for n in ("difflux_h2s", "difflux_nh3", "difflux_nh4sh"):
        f[n] = np.zeros(shape)
    return P, resolve_physics(env), resolve_micro(env), g, f


def gpu_moist_model(P, PH, MC, g, f):
    from atjup_b200.gpu import GpuModel
    m = GpuModel(P, g)
    m.set_physics(PH, f["layer_heights"])
    m.set_micro(MC)
    m.upload_state(f)
    return m


def baseline_case(config: str, iters: int):
    """The reference from a benchmark configuration's seeded initial state
    (oracle/baseline_state.py), run `iters` iterations: (dump, params, physics, micro, mca, grid,
    fields). physics, micro and mca are None for the dry configuration."""
    import baseline_state as BS
    from atjup_b200.params import resolve_mca
    env = BS.ENVS[config]
    if config == "dry":
        d = ref_dump("--baseline", "dry", "--iters", str(iters))
        return d, dump_params(d, env=env), None, None, None, dump_grid(d), dump_fields(d)
    d = ref_dump("--baseline", "phys", "--phys-iters", str(iters))
    P = dump_params(d, env=env)
    P.has_nue = 1
    P.has_heating = 1
    MC = resolve_micro(env, {RENAME.get(k[6:], k[6:]): float(v) for k, v in d.items()
                             if k.startswith("micro_")},
                       {g: tuple(d["gas_" + g]) for g in ("H2O", "NH3", "CH4")})
    consts = {k[5:]: float(v) for k, v in d.items() if k.startswith("phys_")}
    consts["abl_height"] = float(d["knobd_abl_height"])
    return (d, P, resolve_physics(env, consts), MC, resolve_mca(env), dump_grid(d),
            dump_fields(d))


def gpu_baseline_model(P, PH, MC, MCA, g, f):
    from atjup_b200.gpu import GpuModel
    m = GpuModel(P, g)
    if PH is not None:
        m.set_physics(PH, f["layer_heights"])
        m.set_micro(MC)
        m.set_mca(MCA)
    m.upload_state(f)
    return m
