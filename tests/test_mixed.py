"""The mixed-precision RK step (AtjupParams.precision = ATJUP_PREC_MIXED) against the FP64 step, on
the full-physics configuration's seeded state (the reference's own initial state with the
full-physics recipe, oracle/baseline_state.py; 41x181x361), after 200 iterations.

The mixed step stores the stage inputs and accumulators of the 17 RK fields in FP32 and evaluates
the dynamics, species and closure right-hand sides in FP32; the time-level-n state, the final
update, the differences of the pressures, the buoyancy anomaly against the level mean, the
pressure solve, the level means, the column balance and the loop's microphysics stay FP64. Bar per
prognostic field: relative L2 <= 1e-5 against the FP64 step.

Where the model itself cannot be followed to 1e-5 the bar is its own sensitivity instead. The
saturation adjustment and the precipitation branch on thresholds (saturation, freezing, rain
evaporation), so a perturbation at the level of one FP32 rounding moves the condensates by far more
than 1e-5: the FP64 step started from the same state rounded once to FP32 is measured against the
exact FP64 run in the test, and a field passes when the mixed step's error is <= max(1e-5, 10 x
that self-sensitivity), the factor the full-physics parity tests give the reference's own
sensitivity (tests/test_baseline_configs.py). The mixed step rounds at every stage where the
self-sensitivity run rounds once, and the in-loop projection around the obstacle (every 10
iterations) adds a step of its own: its SOR stops at the first sweep below a relative change of
1e-10, so a rounding-level difference of the flow can move its stopping sweep. Measured: only
h2o_ice needs the second form (mixed 2.5e-3 against a self-sensitivity of 6.8e-4); every other
field is within 1e-5."""
import numpy as np
import pytest

from oracle_bridge import rel_l2

STEPS = 200
MIXED_TOL = 1e-5


def bench_state():
    from moist_cases import baseline_case
    d, P, PH, MC, MCA, grid, fields = baseline_case("phys", 0)
    return P, PH, MC, MCA, grid, fields


def model(P, PH, MC, MCA, grid, fields, precision):
    from moist_cases import gpu_baseline_model
    m = gpu_baseline_model(P, PH, MC, MCA, grid, fields)
    m.set_precision(precision)
    return m


@pytest.mark.gpu
def test_mixed_step_tracks_fp64_200_iterations(ref_required):
    from atjup_b200.params import PREC_FP64, PREC_MIXED, SCALARS
    P, PH, MC, MCA, grid, fields = bench_state()
    names = ("t", "u", "v", "w", "p_dyn") + SCALARS
    rounded = dict(fields)
    for n in names + tuple(x + "n" for x in SCALARS):
        if n in rounded:
            rounded[n] = fields[n].astype(np.float32).astype(np.float64)
    runs = [model(P, PH, MC, MCA, grid, fields, PREC_FP64),
            model(P, PH, MC, MCA, grid, fields, PREC_MIXED),
            model(P, PH, MC, MCA, grid, rounded, PREC_FP64)]
    for it in range(1, STEPS + 1):
        for m in runs:
            m.step(it, it == 1)
    for m in runs:
        assert m.nonfinite_count() == 0
    report = {}
    for n in names:
        ref = runs[0].download(n)
        err = rel_l2(runs[1].download(n), ref)
        sens = rel_l2(runs[2].download(n), ref)
        report[n] = (err, sens)
    for m in runs:
        m.close()
    print("mixed vs FP64 after", STEPS, "iterations (error, FP64 self-sensitivity):",
          {n: f"{e:.1e}/{s:.1e}" for n, (e, s) in report.items()})
    for n, (err, sens) in report.items():
        assert np.isfinite(err) and err <= max(MIXED_TOL, 10.0 * sens), \
            f"{n}: mixed step off by {err:.3e} (FP64 self-sensitivity {sens:.3e})"


@pytest.mark.gpu
def test_precision_switch_is_checked():
    from atjup_b200.gpu import AtjupError, GpuModel
    from helpers import synthetic_case
    P, g, f = synthetic_case(13, 37, 49, seed=5)
    m = GpuModel(P, g)
    with pytest.raises(AtjupError):
        m.set_precision(7)
    m.close()
