"""The turbulence closure update (Turbulence<cJupiterModel>::run, Turbulence.h:307-882, and the
driver's turbWallOmega, cJupiterModel.cpp:360-377): the oracle against the reference (CPU), the
CUDA kernels against the oracle and the reference (GPU).

The oracle is bit-exact with the reference for every branch (k-omega SST, k-omega, k-epsilon, the
surface law of ATJUP_TURB_FREE=0, the buoyancy sink, the boundary-layer taper, no curvature
terms). The GPU kernels contract multiply-adds and use CUDA's sqrt, pow, tanh and exp: relative
L2 <= 1e-12 per field after one update (measured ~1e-16)."""
import os

import numpy as np
import pytest

from atjup_b200 import synthetic
from atjup_b200.params import DEFAULT_GASES, resolve_physics
from helpers import dump_fields, dump_grid, dump_params, ref_dump, synthetic_case
from oracle_bridge import PHYS_ENV, oracle_turbulence, rel_l2

TURB_TOL = 1e-12
OUT = ("tke", "dis", "tken", "disn", "nue", "prod", "tke_source", "dis_source", "vel_star")
ALL_VARIANTS = os.environ.get("ATJUP_TEST_ALL_VARIANTS", "0") != "0"
DEFAULT_VARIANTS = [(), ("ATJUP_TURB_MODEL=k_omega", "ATJUP_TURB_FREE=0")]
EXTRA_VARIANTS = [("ATJUP_TURB_MODEL=k_epsilon",), ("ATJUP_TURB_FREE=0",), ("ATJUP_TURB_BUOY=1",),
                  ("ATJUP_TURB_BUOY=2",), ("ATJUP_ABL_TAPER=1",), ("ATJUP_TURB_CURV=0",),
                  ("ATJUP_TURB_MODEL=k_epsilon", "ATJUP_TURB_FREE=0")]
GPU_VARIANTS = [{}, {"ATJUP_TURB_MODEL": "k_omega"}, {"ATJUP_TURB_MODEL": "k_epsilon"},
                {"ATJUP_TURB_FREE": "0"}, {"ATJUP_TURB_MODEL": "k_omega", "ATJUP_TURB_FREE": "0"},
                {"ATJUP_TURB_MODEL": "k_epsilon", "ATJUP_TURB_FREE": "0"}, {"ATJUP_TURB_BUOY": "1"},
                {"ATJUP_TURB_BUOY": "2"}, {"ATJUP_ABL_TAPER": "1"}, {"ATJUP_TURB_CURV": "0"}]


def ref_turb_case(*env):
    d = ref_dump("--turb", *[f"--env={e}" for e in env])
    envd = dict(PHYS_ENV)
    envd.update(dict(e.split("=", 1) for e in env))
    P = dump_params(d, env=envd)
    consts = {k[5:]: float(v) for k, v in d.items() if k.startswith("phys_")}
    consts["abl_height"] = float(d["knobd_abl_height"])
    return d, P, resolve_physics(envd, consts)


def turb_case(im, jm, km, seed=11, env=None):
    envd = dict(PHYS_ENV)
    envd.update(env or {})
    P, g, f = synthetic_case(im, jm, km, seed=seed, env=envd)
    s = dict(f)
    s["solid"] = g["solid"]
    f.update(synthetic.physics(s, DEFAULT_GASES, seed=seed + 3))
    rng = np.random.Generator(np.random.Philox(seed + 4))
    fluid = g["solid"] == 0
    # wind noise of 1 m/s (model units / u_0) and a few negative k*, omega* for the clamps
    for n in ("u", "v", "w"):
        f[n] = np.where(fluid, f[n] + 0.01 * rng.standard_normal(f[n].shape), 0.0)
    for n in ("tke", "dis"):
        neg = fluid & (rng.uniform(size=f[n].shape) < 0.02)
        f[n] = np.where(neg, -f[n], f[n])
        f[n + "n"] = f[n].copy()
    return P, resolve_physics(envd), g, f


@pytest.mark.slow
@pytest.mark.parametrize("env", DEFAULT_VARIANTS + (EXTRA_VARIANTS if ALL_VARIANTS else []))
def test_oracle_turbulence_bit_exact(ref_required, env):
    d, P, PH = ref_turb_case(*env)
    out = oracle_turbulence(P, PH, dump_grid(d), dump_fields(d))
    for n in OUT:
        assert np.array_equal(out[n], d["out_" + n]), f"{n} differs from the reference ({env})"


def gpu_turb(P, PH, g, f):
    from atjup_b200.gpu import GpuModel
    m = GpuModel(P, g)
    m.set_physics(PH, f["layer_heights"])
    m.upload_state(f)
    m.turbulence()
    got = {n: m.download(n) for n in ("tke", "dis", "nue", "prod", "tke_source", "dis_source")}
    got["tken"] = m.download_n("tke")
    got["disn"] = m.download_n("dis")
    got["vel_star"] = m.download2d("vel_star")
    m.close()
    return got


def check(got, want, where):
    out = {}
    for n in OUT:
        assert np.isfinite(got[n]).all(), f"{where}{n}: non-finite"
        r = rel_l2(got[n], want[n])
        out[n] = r
        assert r <= TURB_TOL, f"{where}{n}: relative L2 {r:.3e}"
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("env", GPU_VARIANTS)
def test_gpu_turbulence_matches_oracle(env):
    P, PH, g, f = turb_case(13, 37, 49, env=env)
    check(gpu_turb(P, PH, g, f), oracle_turbulence(P, PH, g, f), f"{env}: ")


@pytest.mark.gpu
def test_gpu_turbulence_matches_oracle_41x61x97():
    P, PH, g, f = turb_case(41, 61, 97)
    check(gpu_turb(P, PH, g, f), oracle_turbulence(P, PH, g, f), "41x61x97: ")


@pytest.mark.gpu
def test_gpu_turbulence_matches_reference_full_grid(ref_required):
    d, P, PH = ref_turb_case()
    f = dump_fields(d)
    got = gpu_turb(P, PH, dump_grid(d), f)
    r = check(got, {n: d["out_" + n] for n in OUT}, "full grid: ")
    print("full-grid turbulence vs reference, rel L2:", {k: f"{v:.1e}" for k, v in r.items()})
