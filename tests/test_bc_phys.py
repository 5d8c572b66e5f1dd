"""The boundary passes over the full-physics field set (BC_Jup::bcRadius, bcTheta, bcPhi,
bcSolidGround with the field lists of BC_Jup.h:275-350: species, chemistry mass fluxes, the
closure fields and their n copies): the oracle against the reference after each pass (CPU), the
CUDA passes against the oracle and the reference (GPU).

The passes are copies, 2-point extrapolations (4/3 a - 1/3 b), tapers and clamps: the oracle is
bit-exact; the GPU may fuse an extrapolation into one FMA, so its bar is relative L2 <= 1e-14 per
field."""
import numpy as np
import pytest

from atjup_b200 import synthetic
from atjup_b200.params import BC_ALL, BC_PHI, BC_RADIUS, BC_SOLID, BC_THETA, DEFAULT_GASES, resolve_physics
from helpers import dump_fields, dump_grid, dump_params, ref_dump, synthetic_case
from oracle_bridge import PHYS_ENV, oracle_bc, rel_l2

BC_TOL = 1e-14
STEPS = ("radius", "theta", "phi", "solid")
STEP_BIT = {"radius": BC_RADIUS, "theta": BC_THETA, "phi": BC_PHI, "solid": BC_SOLID}
FIELDS = ("t", "u", "v", "w", "p_stat", "p_dyn", "h2o", "h2o_cloud", "h2o_ice", "h2s", "nh3",
          "nh3_cloud", "nh3_ice", "ch4", "ch4_cloud", "ch4_ice", "nh4sh", "tke", "dis", "tken",
          "disn", "nue", "prod", "tke_source", "dis_source", "massflux_h2s", "massflux_nh3",
          "massflux_nh4sh", "fluxlim_nh4sh")


@pytest.mark.slow
def test_oracle_bc_phys_bit_exact(ref_required):
    d = ref_dump("--bc")
    P = dump_params(d, env=PHYS_ENV)
    out = oracle_bc(P, dump_grid(d), dump_fields(d))
    for step in STEPS:
        for n in FIELDS:
            assert np.array_equal(out[step][n], d[f"bc_{step}_{n}"], equal_nan=True), \
                f"after {step}: {n} differs from the reference"


def bc_case(im, jm, km, seed=21):
    P, g, f = synthetic_case(im, jm, km, seed=seed, env=PHYS_ENV)
    s = dict(f)
    s["solid"] = g["solid"]
    f.update(synthetic.physics(s, DEFAULT_GASES, seed=seed + 1))
    rng = np.random.Generator(np.random.Philox(seed + 2))
    shape = f["t"].shape
    for n in FIELDS:
        a = np.asarray(f.get(n, np.zeros(shape)), dtype=np.float64)
        scale = np.abs(a).max() or 1e-4
        a = a + 0.05 * scale * rng.standard_normal(shape)
        if n in FIELDS[6:17]:
            a = np.where(rng.uniform(size=shape) < 0.1, -np.abs(a), a)
        if n in ("tke", "tken", "dis", "disn", "nue", "prod"):
            a = np.where(rng.uniform(size=shape) < 0.01, -np.abs(a), a)
            a = np.where(rng.uniform(size=shape) < 0.001, 1e7, a)
        f[n] = a
    return P, resolve_physics(PHYS_ENV), g, f


def gpu_bc(P, PH, g, f, steps=STEPS):
    from atjup_b200.gpu import GpuModel
    m = GpuModel(P, g)
    m.set_physics(PH, f["layer_heights"])
    m.upload_state(f)
    out = {}
    for step in steps:
        m.bc(STEP_BIT[step])
        snap = {n: m.download(n) for n in FIELDS if n not in ("tken", "disn")}
        snap["tken"] = m.download_n("tke")
        snap["disn"] = m.download_n("dis")
        out[step] = snap
    m.close()
    return out


def check(got, want, where=""):
    for step in STEPS:
        for n in FIELDS:
            r = rel_l2(got[step][n], want[step][n])
            assert r <= BC_TOL, f"{where}after {step}: {n} relative L2 {r:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(13, 37, 49), (41, 61, 97)])
def test_gpu_bc_phys_matches_oracle(shape):
    P, PH, g, f = bc_case(*shape)
    check(gpu_bc(P, PH, g, f), oracle_bc(P, g, f), f"{shape}: ")


@pytest.mark.gpu
def test_gpu_bc_phys_matches_reference_full_grid(ref_required):
    d = ref_dump("--bc")
    P = dump_params(d, env=PHYS_ENV)
    f = dump_fields(d)
    got = gpu_bc(P, resolve_physics(PHYS_ENV), dump_grid(d), f)
    want = {step: {n: d[f"bc_{step}_{n}"] for n in FIELDS} for step in STEPS}
    check(got, want, "full grid: ")
