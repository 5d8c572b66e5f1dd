"""The numpy transposes of the dry iteration's linear passes (tests/adjoint_linear.py) against
the oracle's forward passes, by the dot-product test <F d, l> = <d, F^T l> on seeded random d
and l: one pass of the in-loop 4th-order Shapiro filter (lib/Utils.cpp:334-453), the zonal
column balance of v (InitValues_Jup.cpp:1500-1538), the boundary passes on t, u, v, w
(BC_Jup.h:185-658, BoundaryConditions.h:253-360) with each of their knobs, and the pressure pass
(PressureSolver.h:144-766: two red-black sweeps of p_dyn and the one-sided divergence source of
aux_u, aux_v, aux_w), with its clamp off and with a fixed clamp mask; the iteration's tail after
the RK step composed in the loop's order; and the mixture density's tangent-linear against central
differences of the oracle. These transposes
are the specification that GPU transposes of the whole dry iteration follow; the bar is
roundoff (1e-13 relative)."""
import ctypes

import numpy as np
import pytest

import adjoint_linear as AL
from helpers import oracle_from, synthetic_case
from oracle_bridge import oracle_bc

DOT_TOL = 1e-13
SHAPES = [(9, 21, 33), (13, 37, 49)]
NAMES = ("t", "u", "v", "w")


def rel(a, b):
    return abs(a - b) / max(abs(a), 1e-300)


@pytest.mark.parametrize("shape", SHAPES)
def test_shapiro_transpose(shape):
    p, g, f = synthetic_case(*shape, seed=81)
    assert (g["topo"] > 0).any(), "the case has mountains, so the filter's 2nd-order cells act"
    o = oracle_from(p, g, f)
    rng = np.random.default_rng(3)
    d, lam = rng.standard_normal(o.shape), rng.standard_normal(o.shape)
    o.f["u"][...] = d
    o.shapiro("u", 4, p.shapiro_strength, 1, 1)
    lhs = float(np.vdot(o.f["u"], lam))
    rhs = float(np.vdot(d, AL.shapiro4_T(lam, g["topo"], p.shapiro_strength)))
    assert rel(lhs, rhs) <= DOT_TOL, (lhs, rhs)


@pytest.mark.parametrize("shape", SHAPES)
def test_balance_v_transpose(shape):
    p, g, f = synthetic_case(*shape, seed=81)
    o = oracle_from(p, g, f)
    rng = np.random.default_rng(4)
    d, lam = rng.standard_normal(o.shape), rng.standard_normal(o.shape)
    o.f["v"][...] = d
    o.lib.ora_balance_column_v(ctypes.byref(o.P), ctypes.byref(o.G), ctypes.byref(o.S))
    lhs = float(np.vdot(o.f["v"], lam))
    rhs = float(np.vdot(d, AL.balance_v_T(lam, g["topo"], g["rad"], p.dr)))
    assert rel(lhs, rhs) <= DOT_TOL, (lhs, rhs)


@pytest.mark.parametrize("knobs", [{}, {"top_taper": 2}, {"top_taper": 0, "lid_u": 0},
                                   {"pole_fill_rows": 0, "mount_t_ambient": 0}],
                         ids=["default", "taper2", "no_taper_no_lid", "no_fill_no_ambient"])
@pytest.mark.parametrize("shape", SHAPES)
def test_boundary_transpose(shape, knobs):
    p, g, f = synthetic_case(*shape, seed=81)
    for k, v in knobs.items():
        setattr(p, k, v)
    assert g["solid"].any(), "the case has solid cells, so the extrapolation and ambient rows act"
    rng = np.random.default_rng(5)
    d = {n: rng.standard_normal(f["t"].shape) for n in NAMES}
    lam = {n: rng.standard_normal(f["t"].shape) for n in NAMES}
    out = oracle_bc(p, g, {**f, **d}, physics=False)["solid"]
    lhs = sum(float(np.vdot(out[n], lam[n])) for n in NAMES)
    LT = AL.bc_T(lam, g["solid"], lid_u=p.lid_u, top_taper=p.top_taper,
                 pole_fill_rows=p.pole_fill_rows, mount_t_ambient=p.mount_t_ambient)
    rhs = sum(float(np.vdot(d[n], LT[n])) for n in NAMES)
    assert rel(lhs, rhs) <= DOT_TOL, (lhs, rhs)


NO_CLAMP = 1e200      # the source clamp cap * den never binds, so the pass is linear


def aux_case(shape, knobs, seed):
    p, g, f = synthetic_case(*shape, seed=81)
    p.p_dyn_cap = NO_CLAMP
    for k, v in knobs.items():
        setattr(p, k, v)
    rng = np.random.default_rng(seed)
    sh = f["t"].shape
    return p, g, f, rng.standard_normal(sh), [rng.standard_normal(sh) for _ in range(3)], \
        rng.standard_normal(sh)


def set_aux(o, d_a):
    o.f["aux_u"][...], o.f["aux_v"][...], o.f["aux_w"][...] = d_a


@pytest.mark.parametrize("shape", SHAPES)
def test_pressure_source_matches_oracle(shape):
    p, g, f, _, d_a, _ = aux_case(shape, {}, 6)
    o = oracle_from(p, g, f)
    set_aux(o, d_a)
    o.call("ora_prepare_projection")
    want = o.source()
    got = AL.pressure_source(p, g, d_a)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    # the one-sided stencils at the obstacle are exercised
    gg = AL._with_sol3(p, g)
    one_sided = sum(1 for i, j, k in zip(*np.nonzero(gg["_sol3"]))
                    if 0 < i < p.im - 1 and 0 < j < p.jm - 1 and k < p.km - 1
                    and len(AL._div_terms(p, gg, i, j, k)) > 6)
    assert one_sided > 0


@pytest.mark.parametrize("knobs", [{}, {"press_wall": 0}, {"rigid_lid": 0}],
                         ids=["default", "no_press_wall", "free_lid"])
@pytest.mark.parametrize("shape", SHAPES)
def test_pressure_transpose(shape, knobs):
    p, g, f, d_p, d_a, lam = aux_case(shape, knobs, 6)
    o = oracle_from(p, g, f)
    o.f["p_dyn"][...] = d_p
    set_aux(o, d_a)
    o.pressure(sweeps=2)
    lhs = float(np.vdot(o.f["p_dyn"], lam))
    lp, la = AL.pressure_T(lam, p, g, 2)
    rhs = float(np.vdot(d_p, lp)) + sum(float(np.vdot(d_a[q], la[q])) for q in range(3))
    assert rel(lhs, rhs) <= DOT_TOL, (lhs, rhs)


@pytest.mark.parametrize("shape", SHAPES)
def test_pressure_transpose_clamp_mask(shape):
    """the clamp linearised at a base state passes the source's derivative only where it does
    not bind: the forward runs the sweeps on b = mask * source through the oracle's b argument"""
    p, g, f, d_p, d_a, lam = aux_case(shape, {}, 7)
    mask = (np.random.default_rng(8).uniform(size=d_p.shape) < 0.7).astype(np.float64)
    o = oracle_from(p, g, f)
    set_aux(o, d_a)
    o.call("ora_prepare_projection")
    b = mask * o.source()
    o = oracle_from(p, g, f)
    o.f["p_dyn"][...] = d_p
    o.pressure(sweeps=2, b=np.ascontiguousarray(b))
    lhs = float(np.vdot(o.f["p_dyn"], lam))
    lp, la = AL.pressure_T(lam, p, g, 2, pass_mask=mask)
    rhs = float(np.vdot(d_p, lp)) + sum(float(np.vdot(d_a[q], la[q])) for q in range(3))
    assert rel(lhs, rhs) <= DOT_TOL, (lhs, rhs)


@pytest.mark.parametrize("shape", SHAPES)
def test_iteration_tail_transpose(shape):
    """the dry iteration after the RK step, in the loop's order (cJupiterModel.cpp:1032-1381):
    the boundary passes, two in-loop Shapiro passes of u, v, w (ATJUP_VEL_SHAPIRO_INLOOP=2; the
    default is 0), the column balance of v; its transpose is the transposes in reverse order"""
    p, g, f = synthetic_case(*shape, seed=81)
    passes = p.shapiro_inloop = 2
    rng = np.random.default_rng(9)
    d = {n: rng.standard_normal(f["t"].shape) for n in NAMES}
    lam = {n: rng.standard_normal(f["t"].shape) for n in NAMES}
    o = oracle_from(p, g, {**f, **d})
    for step in ("radius", "theta", "phi", "solid"):
        o.call(f"ora_bc_{step}")
    for n in ("u", "v", "w"):
        o.shapiro(n, 4, p.shapiro_strength, passes, 1)
    o.lib.ora_balance_column_v(ctypes.byref(o.P), ctypes.byref(o.G), ctypes.byref(o.S))
    lhs = sum(float(np.vdot(o.f[n], lam[n])) for n in NAMES)
    L = {n: lam[n].copy() for n in NAMES}
    L["v"] = AL.balance_v_T(L["v"], g["topo"], g["rad"], p.dr)
    for n in ("u", "v", "w"):
        for _ in range(passes):
            L[n] = AL.shapiro4_T(L[n], g["topo"], p.shapiro_strength)
    L = AL.bc_T(L, g["solid"], lid_u=p.lid_u, top_taper=p.top_taper,
                pole_fill_rows=p.pole_fill_rows, mount_t_ambient=p.mount_t_ambient)
    rhs = sum(float(np.vdot(d[n], L[n])) for n in NAMES)
    assert rel(lhs, rhs) <= DOT_TOL, (lhs, rhs)


def test_mixture_density_tl_and_transpose():
    """the tangent-linear against central differences of the oracle's mixture density
    (computeMixtureDensity), then the transpose against the tangent-linear by the dot product"""
    p, g, f = synthetic_case(9, 21, 33, seed=81)
    p.rho_pdyn = 1
    rng = np.random.default_rng(10)
    sh = f["t"].shape
    dirs = [rng.standard_normal(sh) * s for s in (np.abs(f["t"]).mean(), np.abs(f["p_stat"]).mean(),
                                                  np.abs(f["p_stat"]).mean() / p.p_dyn_to_bar)]

    def rho(eps):
        o = oracle_from(p, g, {**f, "t": f["t"] + eps * dirs[0], "p_stat": f["p_stat"] + eps * dirs[1],
                               "p_dyn": f["p_dyn"] + eps * dirs[2]})
        o.call("ora_mixture_density")
        return o.f["rho_mix"].copy()

    eps = 1e-6
    fd = (rho(eps) - rho(-eps)) / (2.0 * eps)
    tl = AL.mixture_density_tl(p, f["t"], f["p_stat"], f["p_dyn"], *dirs)
    assert (tl != 0).sum() > 0.5 * tl.size
    assert np.linalg.norm(fd - tl) <= 1e-7 * np.linalg.norm(tl)
    lam = rng.standard_normal(sh)
    lhs = float(np.vdot(tl, lam))
    adj = AL.mixture_density_T(p, f["t"], f["p_stat"], f["p_dyn"], lam)
    rhs = sum(float(np.vdot(d, a)) for d, a in zip(dirs, adj))
    assert rel(lhs, rhs) <= DOT_TOL, (lhs, rhs)
