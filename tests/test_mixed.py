"""The mixed-precision RK step (AtjupParams.precision = ATJUP_PREC_MIXED) against the FP64 step, on
the full-physics state of the benchmark (41x181x361, seeded), after 200 iterations.

The mixed step stores the stage inputs and accumulators of the 17 RK fields in FP32 and evaluates
the species and closure right-hand sides in FP32; the time-level-n state, the final update, the
dynamics right-hand side, the pressure, the level means, the column balance and the loop's
microphysics stay FP64. Bar per prognostic field: relative L2 <= 1e-5 against the FP64 step.

Where the model itself cannot be followed to 1e-5 the bar is its own sensitivity instead. The
saturation adjustment and the precipitation branch on thresholds (saturation, freezing, rain
evaporation), so a perturbation at the level of one FP32 rounding moves the condensates by far more
than 1e-5: the FP64 step started from the same state rounded once to FP32 differs from the exact
FP64 run after 200 iterations by h2o_cloud 9.4e-4, h2o_ice 3.9e-4, nh3_ice 1.8e-5 (measured). A
field passes when the mixed step's error is <= max(1e-5, 3 x that self-sensitivity), both measured
in the test. Measured mixed-step errors after 200 iterations: h2o_ice 1.1e-4, h2o 1.2e-6, every
other field <= 1.6e-7."""
import numpy as np
import pytest

from oracle_bridge import rel_l2

STEPS = 200
MIXED_TOL = 1e-5


def bench_state():
    import bench
    from atjup_b200 import synthetic
    from atjup_b200.params import DEFAULT_GASES, resolve_params
    im, jm, km = 41, 181, 361
    P = resolve_params(bench.PHYS_ENV, im=im, jm=jm, km=km)
    P.has_nue = 1
    P.has_heating = 1
    s = synthetic.state(im, jm, km, seed=20261203)
    grid = {k: s[k] for k in ("rad", "the", "solid", "topo", "cell_vbar0", "cell_ubar0")}
    fields = {k: v for k, v in s.items() if k not in grid}
    fields.update(synthetic.full_physics(s, DEFAULT_GASES, seed=20261207))
    return P, grid, fields


def model(P, grid, fields, precision):
    import bench
    from atjup_b200.gpu import GpuModel
    from atjup_b200.params import resolve_mca, resolve_micro, resolve_physics
    m = GpuModel(P, grid)
    m.set_physics(resolve_physics(bench.PHYS_ENV), fields["layer_heights"])
    m.set_micro(resolve_micro(bench.PHYS_ENV))
    m.set_mca(resolve_mca(bench.PHYS_ENV))
    m.set_precision(precision)
    m.upload_state(fields)
    return m


@pytest.mark.gpu
def test_mixed_step_tracks_fp64_200_iterations():
    from atjup_b200.params import PREC_FP64, PREC_MIXED, SCALARS
    P, grid, fields = bench_state()
    names = ("t", "u", "v", "w", "p_dyn") + SCALARS
    rounded = dict(fields)
    for n in names:
        rounded[n] = fields[n].astype(np.float32).astype(np.float64)
    runs = [model(P, grid, fields, PREC_FP64), model(P, grid, fields, PREC_MIXED),
            model(P, grid, rounded, PREC_FP64)]
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
        assert np.isfinite(err) and err <= max(MIXED_TOL, 3.0 * sens), \
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
