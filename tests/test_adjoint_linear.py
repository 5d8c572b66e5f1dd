"""The numpy transposes of the dry iteration's linear passes (tests/adjoint_linear.py) against
the oracle's forward passes, by the dot-product test <F d, l> = <d, F^T l> on seeded random d
and l: one pass of the in-loop 4th-order Shapiro filter (lib/Utils.cpp:334-453), the zonal
column balance of v (InitValues_Jup.cpp:1500-1538) and the boundary passes on t, u, v, w
(BC_Jup.h:185-658, BoundaryConditions.h:253-360) with each of their knobs. These transposes
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
