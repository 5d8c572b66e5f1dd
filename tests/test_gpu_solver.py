"""Residual-controlled pressure solve (ATJUP_SOLVE_RESIDUAL) on the GPU, checked with the CPU
oracle's own application of the reference operator (the sweep's fixed-point equation, oracle
ora_pressure_apply), for FP64 and for FP32-inner / FP64-refinement solves.

Acceptance: ||b - A p|| / ||b|| <= max(1e-10, 8 * floor), floor = eps * || sum |face terms| || /
||b||, the relative residual a single rounding of an FP64 p already produces. On this operator
(radial weight 1600 against horizontal 0.013) the floor is ~1e-9 on the full shell, so a 1e-10
target is met where it is representable and the floor is reported where it is not."""
import numpy as np
import pytest

from atjup_b200 import synthetic
from atjup_b200.params import PREC_FP64, PREC_MIXED, SOLVE_RESIDUAL
from helpers import gpu_from, oracle_from, synthetic_case

pytestmark = pytest.mark.gpu


def _projected(o, b):
    """b minus its y-component on fluid interior cells (the solver's compatibility step)."""
    im, jm, km = o.shape
    s = o.g["solid"].reshape(o.shape)
    a = np.ones(im); a[[1, im - 2]] = 1.5
    d = np.ones(jm); d[[1, jm - 2]] = 1.5
    mask = np.zeros(o.shape, bool)
    mask[1:im - 1, 1:jm - 1, :km - 1] = True
    mask &= (s == 0)
    y = (a[:, None, None] * d[None, :, None]) * mask
    bb = np.where(mask, b, 0.0)
    return bb - (y * bb).sum() / y.sum() * mask, mask


def _rel_residual(o, p, b):
    bp, mask = _projected(o, b)
    r = np.where(mask, bp - o.apply_A(p), 0.0)
    return np.linalg.norm(r) / np.linalg.norm(bp)


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("shape", [(13, 37, 49), (41, 61, 97)], ids=lambda s: "x".join(map(str, s)))
def test_residual_solve_small(shape, prec):
    p, g, f = synthetic_case(*shape)
    b = synthetic.poisson_rhs(*shape, seed=3)
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    m.set_solve_rhs(b)
    st = m.pressure_solver(mode=SOLVE_RESIDUAL, rel_tol=1e-10, max_iter=3000, precision=prec,
                           external_rhs=True)
    tol = max(1e-10, 8 * st.rel_floor)
    assert st.rel_residual <= tol
    e = _rel_residual(o, m.download("p_dyn"), b)
    assert e <= 2 * tol, (f"oracle residual {e:.3e} (solver {st.rel_residual:.3e}, floor "
                          f"{st.rel_floor:.2e}, {st.iterations} it)")


@pytest.mark.slow
@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
def test_residual_solve_full_grid(prec):
    """The isolated Poisson solve (seeded smoothed right-hand side) on the 41x181x361 shell with the
    obstacle, to 1e-10."""
    p, g, f = synthetic_case(41, 181, 361)
    b = synthetic.poisson_rhs(41, 181, 361)
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    m.set_solve_rhs(b)
    st = m.pressure_solver(mode=SOLVE_RESIDUAL, rel_tol=1e-10, max_iter=5000, precision=prec,
                           external_rhs=True)
    tol = max(1e-10, 8 * st.rel_floor)
    e = _rel_residual(o, m.download("p_dyn"), b)
    assert e <= 2 * tol, f"oracle residual {e:.3e} (floor {st.rel_floor:.2e}, {st.iterations} it)"


def test_residual_solve_in_loop_source():
    """The in-loop use: the divergence source of aux, warm-started from p_dyn."""
    p, g, f = synthetic_case(13, 37, 49)
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    o.rk4()
    m.runge_kutta()
    src = o.source()
    st = m.pressure_solver(mode=SOLVE_RESIDUAL, rel_tol=1e-10, max_iter=3000)
    tol = max(1e-10, 8 * st.rel_floor)
    e = _rel_residual(o, m.download("p_dyn"), src)
    assert e <= 2 * tol, f"oracle residual {e:.3e} (floor {st.rel_floor:.2e}, {st.iterations} it)"


@pytest.mark.parametrize("omega", [1.0, 1.7])
def test_sor_arm_small(omega):
    """Point red-black SOR (ATJUP_SOLVE_SOR) on the same operator: the relative residual it reports
    is the oracle's residual of the p it returns, and more sweeps lower it (the slow column modes
    of this operator keep it far from 1e-10 within any practical number of sweeps; with omega 1.7
    the relative residual stays above 1 for the first hundreds of sweeps, while the
    high-frequency error, a small part of ||b||, is removed and the smooth modes barely move)."""
    from atjup_b200.params import SOLVE_SOR
    shape = (13, 37, 49)
    p, g, f = synthetic_case(*shape)
    b = synthetic.poisson_rhs(*shape, seed=5)
    o = oracle_from(p, g, f)
    m = gpu_from(p, g, f)
    m.set_solve_rhs(b)
    rels = []
    for cap in (100, 400):
        st = m.pressure_solver(mode=SOLVE_SOR, omega=omega, rel_tol=1e-10, max_iter=cap,
                               external_rhs=True, allow_not_converged=True)
        assert st.iterations == cap
        e = _rel_residual(o, m.download("p_dyn"), b)
        assert abs(e - st.rel_residual) <= 1e-6 * e + 1e-12, (e, st.rel_residual)
        rels.append(e)
    assert rels[1] < rels[0], rels
