"""Tangent-linear and adjoint of one RK4 step of the dry dynamics (atjup_gpu_rk4_tlm,
atjup_gpu_rk4_adjoint): RungeKuttaJup's four stages with the t, u, v, w right-hand sides, the
buoyancy level mean and the hydrostatic integral, linearised about the current state.

* Dot-product test: <TL dy, l> = <dy, AD l> for seeded dy and l over every cell, relative
  difference <= 1e-12 (synthetic dry shells and the reference's own dry state).
* The tangent-linear against central differences of the GPU's own RK4 step
  (atjup_gpu_rk4_step) along the same direction, eps = 1e-6: relative L2 <= 1e-6 per field.
* The gradient of the zonal-jet loss at the top level (tests/adjoint_cases.py) after one RK4 step,
  from the adjoint, against central differences (eps = 1e-6) of the reference's own
  RungeKuttaJup (oracle/_ref) on its dry initial state, along 16 seeded directions: each
  directional derivative within 1e-6 relative plus the central difference's own rounding,
  10 ulp of J over 2 eps (measured: within 1e-7 relative, 2e-8 absolute, on derivatives of
  order 1; the reference's central differences equal the GPU's to 12 digits).
"""
import numpy as np
import pytest

import adjoint_cases as AC
from helpers import dump_fields, dump_grid, dump_params, gpu_from, ref_dump, synthetic_case

pytestmark = pytest.mark.gpu

EPS = 1e-6
NDIR = 16


def padded(m, arrays):
    """four float64 CUDA tensors (im, jm, pitch) holding arrays (im, jm, km), zero padding"""
    import torch
    im, jm, km = m.shape
    pitch = m.field_ptr("t")[1]
    out = []
    for a in arrays:
        x = torch.zeros((im, jm, pitch), dtype=torch.float64, device="cuda")
        x[:, :, :km] = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
        out.append(x)
    return out


def unpadded(m, tensors):
    km = m.shape[2]
    return [x[:, :, :km].cpu().numpy() for x in tensors]


def tlm(m, d):
    x = padded(m, [d[f] for f in AC.FIELDS])
    m.rk4_tlm(*x)
    return dict(zip(AC.FIELDS, unpadded(m, x)))


def adjoint(m, lam):
    x = padded(m, [lam[f] for f in AC.FIELDS])
    m.rk4_adjoint(*x)
    return dict(zip(AC.FIELDS, unpadded(m, x)))


def dot(a, b):
    return sum(float(np.vdot(a[f], b[f])) for f in AC.FIELDS)


def rk4_from(m, y):
    """the GPU's RK4 step from state y (t, u, v, w); returns the new state"""
    for f in AC.FIELDS:
        m.upload(f, y[f])
    m.runge_kutta()
    return {f: m.download(f) for f in AC.FIELDS}


def dot_product_check(m, seed):
    shape = m.shape
    d = AC.direction(seed, shape)
    lam = AC.direction(seed + 100, shape)
    tl = tlm(m, d)
    ad = adjoint(m, lam)
    lhs, rhs = dot(tl, lam), dot(d, ad)
    rel = abs(lhs - rhs) / max(abs(lhs), abs(rhs))
    return lhs, rhs, rel


@pytest.mark.parametrize("shape", [(13, 37, 49), (41, 61, 97)], ids=lambda s: "x".join(map(str, s)))
def test_dot_product_synthetic(shape):
    p, g, f = synthetic_case(*shape, seed=71)
    m = gpu_from(p, g, f)
    lhs, rhs, rel = dot_product_check(m, 3)
    m.close()
    print(f"{shape}: <TL d, l> = {lhs:.15e}, <d, AD l> = {rhs:.15e}, rel {rel:.2e}")
    assert np.isfinite(lhs) and rel <= 1e-12


def test_tangent_linear_matches_differences():
    p, g, f = synthetic_case(41, 61, 97, seed=72)
    m = gpu_from(p, g, f)
    y0 = {n: m.download(n) for n in AC.FIELDS}
    d = AC.direction(5, m.shape)
    tl = tlm(m, d)
    yp = rk4_from(m, {n: y0[n] + EPS * d[n] for n in AC.FIELDS})
    ym = rk4_from(m, {n: y0[n] - EPS * d[n] for n in AC.FIELDS})
    m.close()
    for n in AC.FIELDS:
        fd = (yp[n] - ym[n]) / (2.0 * EPS)
        rel = np.linalg.norm(tl[n] - fd) / np.linalg.norm(fd)
        print(f"{n}: TL vs central difference rel L2 {rel:.2e}")
        assert rel <= 1e-6, f"{n}: {rel:.3e}"


def test_adjoint_gradient_matches_reference_differences(ref_required):
    d = ref_dump("--rk4-fd", f"{NDIR}:{EPS}")
    p, g, f = dump_params(d), dump_grid(d), dump_fields(d)
    m = gpu_from(p, g, f)
    the = g["the"]
    uref = AC.u_ref(the, p.u_0)
    y0 = {n: m.download(n) for n in AC.FIELDS}
    y1 = rk4_from(m, y0)
    # the linearisation point is the initial state again
    for n in AC.FIELDS:
        m.upload(n, y0[n])
    lam = {n: np.zeros(m.shape) for n in AC.FIELDS}
    lam["w"] = AC.loss_adjoint_w(y1["w"], the, uref)
    grad = adjoint(m, lam)
    j0 = AC.loss(y1["w"], the, uref)
    floor = 10.0 * np.finfo(float).eps * abs(j0) / (2.0 * EPS)
    worst = 0.0
    for k in range(NDIR):
        dk = AC.direction(k, m.shape)
        ad = dot(grad, dk)
        jp = AC.loss_from_mean(d[f"fd_zmp_{k}"], the, uref)
        jm = AC.loss_from_mean(d[f"fd_zmm_{k}"], the, uref)
        fd = (jp - jm) / (2.0 * EPS)
        # the same central difference of the GPU's own step, for scale
        gp = AC.loss(rk4_from(m, {n: y0[n] + EPS * dk[n] for n in AC.FIELDS})["w"], the, uref)
        gm = AC.loss(rk4_from(m, {n: y0[n] - EPS * dk[n] for n in AC.FIELDS})["w"], the, uref)
        fd_gpu = (gp - gm) / (2.0 * EPS)
        rel = abs(ad - fd) / abs(fd)
        worst = max(worst, rel)
        print(f"direction {k}: adjoint {ad:.12e}  reference central difference {fd:.12e} "
              f"(GPU's {fd_gpu:.12e})  rel {rel:.2e}")
        assert abs(ad - fd) <= 1e-6 * abs(fd) + floor, f"direction {k}: {rel:.3e} (floor {floor:.1e})"
    m.close()
    print("J", j0, "rounding floor", floor, "worst relative difference over", NDIR, "directions:",
          f"{worst:.2e}")


def test_dot_product_reference_state(ref_required):
    d = ref_dump("--rk4")
    m = gpu_from(dump_params(d), dump_grid(d), dump_fields(d))
    lhs, rhs, rel = dot_product_check(m, 9)
    m.close()
    print(f"reference state: <TL d, l> = {lhs:.15e}, <d, AD l> = {rhs:.15e}, rel {rel:.2e}")
    assert rel <= 1e-12


def test_refused_outside_the_dry_fp64_step():
    from atjup_b200.gpu import AtjupError
    from atjup_b200.params import PREC_MIXED
    p, g, f = synthetic_case(13, 37, 49, seed=73)
    m = gpu_from(p, g, f)
    m.set_precision(PREC_MIXED)
    x = padded(m, [np.zeros(m.shape)] * 4)
    with pytest.raises(AtjupError):
        m.rk4_tlm(*x)
    m.close()


def test_autograd_three_steps_match_differences():
    """Three RK4 steps through the torch.autograd binding (atjup_b200.autograd.RK4Step, each step
    its own checkpoint) and the loss of the last step's w: the gradient along a seeded direction
    against central differences of three GPU steps, within 1e-6 relative plus the rounding floor."""
    import torch
    from atjup_b200.autograd import rk4_steps
    p, g, f = synthetic_case(41, 61, 97, seed=74)
    m = gpu_from(p, g, f)
    im, jm, km = m.shape
    the = g["the"]
    uref = AC.u_ref(the, p.u_0)
    y0 = {n: m.download(n) for n in AC.FIELDS}
    x = [t.requires_grad_() for t in padded(m, [y0[n] for n in AC.FIELDS])]
    out = rk4_steps(m, *x, steps=3)
    zm = out[3][im - 2, :, : km - 1].mean(dim=1)
    th = torch.tensor(the, device="cuda")
    ur = torch.tensor(uref, device="cuda")
    J = (torch.sin(th) * (zm - ur) ** 2).sum()
    J.backward()
    grad = {n: x[q].grad[:, :, :km].cpu().numpy() for q, n in enumerate(AC.FIELDS)}
    d = AC.direction(11, m.shape)

    def J_of(sign):
        y = {n: y0[n] + sign * EPS * d[n] for n in AC.FIELDS}
        for _ in range(3):
            y = rk4_from(m, y)
        return AC.loss(y["w"], the, uref)

    ad = dot(grad, d)
    fd = (J_of(1.0) - J_of(-1.0)) / (2.0 * EPS)
    m.close()
    floor = 10.0 * np.finfo(float).eps * abs(float(J.detach())) / (2.0 * EPS)
    print(f"autograd, 3 steps: adjoint {ad:.12e}  central difference {fd:.12e}  "
          f"rel {abs(ad - fd) / abs(fd):.2e}  floor {floor:.1e}")
    assert abs(ad - fd) <= 1e-6 * abs(fd) + floor
