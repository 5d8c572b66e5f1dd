"""GPU (through the C ABI) against the CPU oracle -- the parity tests proper.

Tolerances: one call of a routine <= 1e-12 relative L2 per field (the kernels contract
multiply-adds into FMA, the oracle does not); 20 dry iterations of the full 41x181x361 shell
<= 1e-10 relative L2 per field (u, v, w, T, p), the bar set for the FP64 GPU path.
"""
import numpy as np
import pytest

from helpers import (DYN_FIELDS, dump_fields, dump_grid, dump_params, gpu_from, oracle_from,
                     ref_dump, rel_l2, synthetic_case)

pytestmark = pytest.mark.gpu

ONE_CALL = 1e-12
TWENTY = 1e-10


def _cmp(m, o, names, tol, where=""):
    for n in names:
        g = m.download(n)
        r = o.f[n]
        e = rel_l2(g, r)
        assert np.isfinite(g).all(), f"{where}{n}: non-finite on GPU"
        assert e <= tol, f"{where}{n}: rel L2 {e:.3e} > {tol:.0e}"


@pytest.fixture(params=[(13, 37, 49), (9, 21, 33), (41, 61, 97)], ids=lambda s: "x".join(map(str, s)))
def small(request):
    return synthetic_case(*request.param)


def test_rk4_small(small):
    p, g, f = small
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    o.rk4()
    m.runge_kutta()
    _cmp(m, o, ["t", "u", "v", "w", "p_hydro", "aux_u", "aux_v", "aux_w"], ONE_CALL)


def test_pressure_sweeps_small(small):
    p, g, f = small
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    o.rk4()                       # realistic aux fields
    m.runge_kutta()
    o.pressure(sweeps=3)
    m.pressure_solver(sweeps=3)
    _cmp(m, o, ["p_dyn", "aux_u", "aux_v", "aux_w"], ONE_CALL)


@pytest.mark.parametrize("order", [2, 4])
def test_shapiro_small(small, order):
    p, g, f = small
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    for n in ("u", "w"):
        o.shapiro(n, order, strength=0.7, passes=2)
        m.shapiro(n, order, strength=0.7, passes=2)
    _cmp(m, o, ["u", "w"], 1e-14)


@pytest.mark.parametrize("order", [2, 4])
def test_shapiro_bit_exact(small, order):
    """The filter's k, j and i passes equal the oracle's (lib/Utils.cpp:227-453) to the bit:
    same rules, same order of operations, no FMA contraction on either side."""
    p, g, f = small
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    for n in ("u", "v", "w"):
        o.shapiro(n, order, strength=1.0, passes=1)
        m.shapiro(n, order, strength=1.0, passes=1)
        assert np.array_equal(m.download(n), o.f[n]), f"{n}: order {order}"
    m.close()


def test_bc_small(small):
    p, g, f = small
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    o.rk4()
    m.runge_kutta()
    for fn in ("ora_bc_radius", "ora_bc_theta", "ora_bc_phi", "ora_bc_solid"):
        o.call(fn)
    m.bc()
    _cmp(m, o, ["t", "u", "v", "w", "p_dyn", "p_stat"], ONE_CALL)


def test_step_small(small):
    p, g, f = small
    p.shapiro_inloop = 1
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    for it in range(1, 6):
        o.iteration(it, it == 1)
        m.step(it, it == 1)
    _cmp(m, o, ["t", "u", "v", "w", "p_dyn", "p_hydro", "rho_mix"], 1e-11)


def test_balance_v_small(small):
    p, g, f = small
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    o.call("ora_balance_column_v")
    m.balance_column_v()
    _cmp(m, o, ["v"], 1e-14)


@pytest.mark.slow
def test_full_grid_rk4_reference_state(ref_required):
    """One RungeKuttaJup on the reference's own initial state (dry config)."""
    d = ref_dump("--rk4")
    p, g, f = dump_params(d), dump_grid(d), dump_fields(d)
    m = gpu_from(p, g, f)
    m.runge_kutta()
    ref_out = dump_fields(d, "out_")
    for n in ("t", "u", "v", "w", "p_hydro", "aux_u", "aux_v", "aux_w"):
        e = rel_l2(m.download(n), ref_out[n])
        assert e <= ONE_CALL, f"{n}: rel L2 vs reference {e:.3e}"


@pytest.mark.slow
def test_full_grid_20_dry_iterations(ref_required):
    """The dry configuration: 20 iterations, GPU FP64 vs the reference <= 1e-10 per field."""
    d = ref_dump("--iters", "20")
    p, g, f = dump_params(d), dump_grid(d), dump_fields(d)
    m = gpu_from(p, g, f)
    for it in range(1, 21):
        m.step(it, it == 1)
    ref_out = dump_fields(d, "out_")
    for n in ("t", "u", "v", "w", "p_dyn", "p_hydro", "rho_mix"):
        e = rel_l2(m.download(n), ref_out[n])
        assert e <= TWENTY, f"{n}: rel L2 vs reference after 20 iterations {e:.3e}"
    assert m.nonfinite_count() == 0
