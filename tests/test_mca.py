"""The moist convective adjustment (MoistConvectiveAdjustment<cJupiterModel>::run,
ConvectiveAdjustment.h:403-849; atjup_gpu_mca).

* The oracle (ora_mca) against the reference, bit-exact, on the reference's moist state perturbed
  so that the adjustment fires (warm bottom layers in 3 % of the columns, moist ones in 2 %).
* The oracle's iteration with the adjustment on every iteration (the reference's default,
  ATJUP_MCA=1) against the reference's, bit-exact after 3 iterations.
* The GPU against the oracle on a synthetic shell and against the reference on its perturbed
  state. The parcel test compares a virtual-temperature difference with 1e-7 K and the
  equilibrium solve evaluates exp and log, so a last-bit difference can decide a marginal pair
  differently; a column where that happens is mixed differently from there on. Bar: at most 0.5 %
  of the columns differ (in any cell by more than 1e-12 of the field's maximum), the others agree
  to relative L2 <= 1e-12, and the adjusted-column count agrees to 0.5 %. Measured: identical.
* The GPU iteration with the adjustment against the reference's, after 3 and 20 iterations, with
  the full-physics bars (tests/test_moist_step.py)."""
import numpy as np
import pytest

from atjup_b200.params import DEFAULT_GASES, resolve_gas, resolve_mca, resolve_micro
from helpers import dump_grid, dump_params, ref_dump, synthetic_case
from moist_cases import PROGNOSTIC, gpu_moist_model, ref_iters_case, synthetic_moist_case
from oracle_bridge import MCA_ENV, MOIST_ENV, oracle_iteration_phys, oracle_mca, rel_l2
from test_moist_step import NH4SH_FAMILY_TOL, REF_TOL
import ref_dump as R

FIELDS = R.MCA_FIELDS
COL_FLIP = 5e-3


def mca_ref_case():
    d = ref_dump("--mca")
    P = dump_params(d, env=MOIST_ENV)
    MC = resolve_micro(MOIST_ENV, {k[6:]: float(v) for k, v in d.items() if k.startswith("micro_")},
                       {g: tuple(d["gas_" + g]) for g in ("H2O", "NH3", "CH4")})
    M = resolve_mca(MCA_ENV)
    M.ep_h2s = float(d["ep_h2s"])
    g = dump_grid(d)
    f = {n: d["in_" + n] for n in FIELDS}
    for n in ("p_stat", "rho_mix"):
        f[n] = d["in_" + n]
    f["layer_heights"] = d["in_layer_heights"]
    return d, P, MC, M, g, f


def changed_columns(a, b):
    return np.any(a != b, axis=0)


@pytest.mark.slow
def test_oracle_mca_bit_exact(ref_required):
    d, P, MC, M, g, f = mca_ref_case()
    out, st = oracle_mca(P, MC, M, g, f)
    fired = changed_columns(d["mca_t"], d["in_t"])
    assert fired.sum() > 100, f"the perturbation fired only {fired.sum()} columns"
    for n in FIELDS:
        assert np.array_equal(out[n], d["mca_" + n]), f"{n} differs from the reference"
    assert st["columns"] >= int(fired.sum()), st


@pytest.mark.slow
def test_oracle_iterations_with_mca_bit_exact(ref_required):
    d, P, PH, MC, g, f = ref_iters_case(3, "--env", "ATJUP_MCA=1")
    out = oracle_iteration_phys(P, PH, MC, g, f, 3, mca=resolve_mca(MCA_ENV))
    for n in R.ITER_FIELDS:
        assert np.array_equal(out[3][n], d[f"it3_{n}"], equal_nan=True), f"{n} differs from the reference"


def check_columns(got: dict, want: dict, where: str):
    flipped_any = None
    for n in FIELDS:
        scale = max(np.abs(want[n]).max(), 1e-300)
        flip = np.any(np.abs(got[n] - want[n]) > 1e-12 * scale, axis=0)
        flipped_any = flip if flipped_any is None else flipped_any | flip
    frac = flipped_any.mean()
    assert frac <= COL_FLIP, f"{where}: {frac:.2%} of the columns differ"
    for n in FIELDS:
        r = rel_l2(np.where(flipped_any[None], 0.0, got[n]), np.where(flipped_any[None], 0.0, want[n]))
        assert r <= 1e-12, f"{where}: {n} relative L2 {r:.3e} outside the differing columns"
    return frac


def gpu_mca(P, PH, MC, M, g, f):
    m = gpu_moist_model(P, PH, MC, g, f)
    m.set_mca(M)
    st = m.mca()
    out = {n: m.download(n) for n in FIELDS}
    m.close()
    return out, st


@pytest.mark.gpu
def test_gpu_mca_matches_oracle():
    P, PH, MC, g, f = synthetic_moist_case(41, 61, 97, seed=51)
    f = R.perturb_unstable(f, g["solid"], f["layer_heights"], seed=52)
    M = resolve_mca(MCA_ENV)
    want, wst = oracle_mca(P, MC, M, g, f)
    got, gst = gpu_mca(P, PH, MC, M, g, f)
    assert wst["columns"] > 50, f"the perturbation fired only {wst['columns']} columns"
    frac = check_columns(got, want, "synthetic 41x61x97")
    assert abs(gst["columns"] - wst["columns"]) <= COL_FLIP * wst["columns"] + 1, (gst, wst)
    print("mca GPU vs oracle: differing columns", frac, "counters GPU", gst, "oracle", wst)


@pytest.mark.gpu
def test_gpu_mca_warp_form_matches_oracle():
    """With at most 2048 listed columns the column kernel runs one warp per column (the settles of
    a mixed segment and a sweep's pair tests on the lanes); the shell above lists nearly all of its
    5,917 columns and so runs one thread per column. This smaller shell (1,519 columns) takes the
    warp form, against the oracle with the same bars."""
    P, PH, MC, g, f = synthetic_moist_case(41, 31, 49, seed=53)
    f = R.perturb_unstable(f, g["solid"], f["layer_heights"], seed=54)
    M = resolve_mca(MCA_ENV)
    want, wst = oracle_mca(P, MC, M, g, f)
    got, gst = gpu_mca(P, PH, MC, M, g, f)
    assert 50 < wst["columns"] <= 2048, wst
    frac = check_columns(got, want, "synthetic 41x31x49")
    assert abs(gst["columns"] - wst["columns"]) <= COL_FLIP * wst["columns"] + 1, (gst, wst)
    assert gst["max_passes"] == wst["max_passes"], (gst, wst)
    print("mca (warp form) GPU vs oracle: differing columns", frac, "counters GPU", gst, "oracle", wst)


@pytest.mark.gpu
def test_gpu_mca_matches_reference(ref_required):
    d, P, MC, M, g, f = mca_ref_case()
    from atjup_b200.params import resolve_physics
    PH = resolve_physics(MOIST_ENV)
    full = dict(f)
    for n in ("u", "v", "w", "p_dyn", "nue", "vel_star", "tke", "dis"):
        if "in_" + n in d:
            full[n] = d["in_" + n]
    got, gst = gpu_mca(P, PH, MC, M, g, full)
    frac = check_columns(got, {n: d["mca_" + n] for n in FIELDS}, "reference state")
    print("mca GPU vs reference: differing columns", frac, "counters", gst)


@pytest.mark.gpu
@pytest.mark.parametrize("iters", [3, 20])
def test_gpu_step_with_mca_matches_reference(ref_required, iters):
    d, P, PH, MC, g, f = ref_iters_case(iters, "--env", "ATJUP_MCA=1")
    m = gpu_moist_model(P, PH, MC, g, f)
    m.set_mca(resolve_mca(MCA_ENV))
    for it in range(1, iters + 1):
        m.step(it, first=(it == 1))
    worst = {n: rel_l2(m.download(n), d[f"it{iters}_{n}"]) for n in PROGNOSTIC}
    m.close()
    print(f"full physics with MCA, {iters} iterations vs reference:", {k: f"{v:.1e}" for k, v in worst.items()})
    for n in PROGNOSTIC:
        assert worst[n] <= NH4SH_FAMILY_TOL.get(n, REF_TOL), f"{n} relative L2 {worst[n]:.3e}"
