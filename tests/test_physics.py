"""Full physics in the RK4 step (RungeKutta_Jup_Turb.cpp:261-583 with RHS_Jup_Turb.cpp's species
and closure terms): the oracle against the reference (CPU), the CUDA kernels against the oracle
and the reference (GPU).

Tolerances. The oracle keeps the reference's operand order and is bit-exact with it. The GPU
kernels contract multiply-adds into FMAs and evaluate sqrt, pow, tanh and exp with CUDA's
functions, so after one step each field agrees to rounding: relative L2 <= 1e-12 per field
(measured: ~1e-15). The closure diagnostics prod, tke_source and dis_source pass through max/min
clamps; they meet the same bar."""
import os

import numpy as np
import pytest

from atjup_b200 import synthetic
from atjup_b200.params import DEFAULT_GASES, SCALARS, resolve_physics
from helpers import dump_fields, dump_grid, dump_params, ref_dump, synthetic_case
from oracle_bridge import PHYS_ENV, oracle_rk4_phys, rel_l2

PHYS_TOL = 1e-12
DYN = ("t", "u", "v", "w", "p_hydro", "aux_u", "aux_v", "aux_w")
DIAG = ("prod", "tke_source", "dis_source")


def ref_phys_case(*env):
    flags = ["--rk4-phys"] + [f"--env={e}" for e in env]
    d = ref_dump(*flags)
    envd = dict(PHYS_ENV)
    envd.update(dict(e.split("=", 1) for e in env))
    P = dump_params(d, env=envd)
    P.has_nue = 1
    P.has_heating = 1
    consts = {k[5:]: float(v) for k, v in d.items() if k.startswith("phys_")}
    PH = resolve_physics(envd, consts)
    return d, P, PH


def phys_case(im, jm, km, seed=7, env=None):
    envd = dict(PHYS_ENV)
    envd.update(env or {})
    P, g, f = synthetic_case(im, jm, km, seed=seed, env=envd)
    P.has_nue = 1
    P.has_heating = 1
    s = dict(f)
    s["solid"] = g["solid"]
    f.update(synthetic.physics(s, DEFAULT_GASES, seed=seed + 2))
    return P, resolve_physics(envd), g, f


# ---------------------------------------------------------------------------------------------
# CPU: the oracle against the reference
# ---------------------------------------------------------------------------------------------

# knob variants of the reference comparison each need a reference start-up (~15 s): the default
# CPU run takes two, ATJUP_TEST_ALL_VARIANTS=1 all of them
ALL_VARIANTS = os.environ.get("ATJUP_TEST_ALL_VARIANTS", "0") != "0"
REF_VARIANTS = [(), ("ATJUP_TURB_MODEL=k_epsilon",)] + (
    [("ATJUP_TURB_MODEL=k_omega",), ("ATJUP_TURB_BUOY=1",)] if ALL_VARIANTS else [])


@pytest.mark.slow
@pytest.mark.parametrize("env", REF_VARIANTS)
def test_oracle_rk4_phys_bit_exact(ref_required, env):
    d, P, PH = ref_phys_case(*env)
    out = oracle_rk4_phys(P, PH, dump_grid(d), dump_fields(d))
    for n in DYN + SCALARS + DIAG:
        assert np.array_equal(out[n], d["out_" + n]), f"{n} differs from the reference ({env})"


def test_resolve_physics_defaults():
    ph = resolve_physics({})
    assert (ph.species_on, ph.turb_on, ph.turb_model, ph.turb_buoy) == (1, 1, 2, 0)
    assert ph.sc_ch4 == 0.99 and ph.tke_max_phys == 1000.0 and ph.nue_max_phys == 1e5
    assert resolve_physics({"ATJUP_TURB": "0"}).turb_on == 0
    assert resolve_physics({"ATJUP_TURB_MODEL": "none"}).turb_on == 0
    assert resolve_physics({"ATJUP_TURB_MODEL": "none", "ATJUP_TURB": "1"}).turb_model == 2
    assert resolve_physics({"ATJUP_TURB_MODEL": "k_epsilon"}).turb_model == 0


# ---------------------------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------------------------

def gpu_phys(P, PH, g, f):
    from atjup_b200.gpu import GpuModel
    m = GpuModel(P, g)
    m.set_physics(PH, f["layer_heights"])
    m.upload_state(f)
    return m


def check_fields(got, want, names, tol=PHYS_TOL, where=""):
    worst = {}
    for n in names:
        r = rel_l2(got[n], want[n])
        worst[n] = r
        assert np.isfinite(got[n]).all(), f"{where}{n}: non-finite"
        assert r <= tol, f"{where}{n}: relative L2 {r:.3e} > {tol}"
    return worst


@pytest.mark.gpu
@pytest.mark.parametrize("shape,env", [((13, 37, 49), {}), ((9, 21, 33), {}), ((41, 61, 97), {}),
                                       ((13, 37, 49), {"ATJUP_TURB_MODEL": "k_omega"}),
                                       ((13, 37, 49), {"ATJUP_TURB_MODEL": "k_epsilon"}),
                                       ((13, 37, 49), {"ATJUP_TURB_BUOY": "1"})])
def test_gpu_rk4_phys_matches_oracle(shape, env):
    P, PH, g, f = phys_case(*shape, env=env)
    want = oracle_rk4_phys(P, PH, g, f)
    m = gpu_phys(P, PH, g, f)
    m.runge_kutta()
    got = {n: m.download(n) for n in DYN + SCALARS + DIAG}
    m.close()
    check_fields(got, want, DYN + SCALARS + DIAG, where=f"{shape} {env}: ")


@pytest.mark.gpu
def test_gpu_rk4_phys_species_only():
    P, PH, g, f = phys_case(13, 37, 49, env={"ATJUP_TURB": "0"})
    want = oracle_rk4_phys(P, PH, g, f)
    m = gpu_phys(P, PH, g, f)
    m.runge_kutta()
    got = {n: m.download(n) for n in DYN + SCALARS}
    m.close()
    check_fields(got, want, DYN + SCALARS)


@pytest.mark.gpu
def test_gpu_rk4_phys_matches_reference_full_grid(ref_required):
    d, P, PH = ref_phys_case()
    f = dump_fields(d)
    m = gpu_phys(P, PH, dump_grid(d), f)
    m.runge_kutta()
    got = {n: m.download(n) for n in DYN + SCALARS + DIAG}
    m.close()
    want = {n: d["out_" + n] for n in DYN + SCALARS + DIAG}
    worst = check_fields(got, want, DYN + SCALARS + DIAG)
    print("full-grid RK4 with physics vs reference, rel L2:", {k: f"{v:.1e}" for k, v in worst.items()})
