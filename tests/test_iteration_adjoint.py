"""Tangent-linear and adjoint of one whole dry iteration (atjup_gpu_iteration_tlm,
atjup_gpu_iteration_adjoint): the pressure pass and the mixture density on even iterations, the
RK4 step, the boundary passes, the in-loop 4th-order Shapiro filter and the column balance of v,
on the nine fields one iteration hands the next (t, u, v, w, p_dyn, aux_u, aux_v, aux_w, rho_mix).

* Dot-product test, each pass alone and the whole iteration, even and odd iterations:
  <TL d, l> = <d, AD l> for seeded d and l over every cell, relative difference <= 1e-12.
* The GPU transposes of the linear passes against their numpy specification
  (tests/adjoint_linear.py, itself held to dot-product tests against the oracle's forward passes):
  boundary passes, Shapiro pass, column balance and pressure pass, relative L2 <= 1e-12.
* The tangent-linear of the whole iteration against central differences of the GPU's own
  iteration (atjup_gpu_step), eps = 1e-6 times the direction: relative L2 <= 1e-6 per field.
* The gradient of the zonal-jet loss after K = 3 iterations of the dry configuration's state,
  through IterationStep (atjup_b200.autograd: each iteration's input is its checkpoint), against
  central differences (eps = 1e-6) of the reference's own dry iterations (oracle/_ref) along 8
  seeded directions: within 1e-6 relative plus 10 ulp of J over 2 eps.
"""
import numpy as np
import pytest

import adjoint_cases as AC
import adjoint_linear as ALIN
from atjup_b200.params import (LIN_ALL, LIN_BALANCE, LIN_BC, LIN_FIELDS, LIN_MIXTURE,
                               LIN_PRESSURE, LIN_RK4, LIN_SHAPIRO)
from helpers import gpu_from, synthetic_case

pytestmark = pytest.mark.gpu

EPS = 1e-6
PARTS = {"pressure": LIN_PRESSURE, "mixture": LIN_MIXTURE, "rk4": LIN_RK4, "bc": LIN_BC,
         "shapiro": LIN_SHAPIRO, "balance": LIN_BALANCE, "all": LIN_ALL}


def padded(m, arrays):
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


def state(m):
    return {n: m.download(n) for n in LIN_FIELDS}


def scales(x):
    """a field's natural size: its RMS (1 where the field is zero)"""
    out = {}
    for n, a in x.items():
        r = float(np.sqrt(np.mean(a * a)))
        out[n] = r if r > 0 else 1.0
    return out


def direction(shape, seed, sc):
    rng = np.random.Generator(np.random.Philox(key=seed))
    return {n: sc[n] * rng.standard_normal(shape) for n in LIN_FIELDS}


def tlm(m, d, it, first, parts=LIN_ALL):
    x = padded(m, [d[n] for n in LIN_FIELDS])
    m.iteration_tlm(x, it, first, parts)
    return dict(zip(LIN_FIELDS, unpadded(m, x)))


def adjoint(m, lam, it, first, parts=LIN_ALL):
    x = padded(m, [lam[n] for n in LIN_FIELDS])
    m.iteration_adjoint(x, it, first, parts)
    return dict(zip(LIN_FIELDS, unpadded(m, x)))


def dot(a, b, names=LIN_FIELDS):
    return sum(float(np.vdot(a[n], b[n])) for n in names)


def prepared(shape, seed):
    """a synthetic dry shell after two iterations (aux and rho_mix realistic)"""
    p, g, f = synthetic_case(*shape, seed=seed)
    m = gpu_from(p, g, f)
    for it in (1, 2):
        m.step(it, it == 1)
    return p, g, m


@pytest.mark.parametrize("part", sorted(PARTS))
@pytest.mark.parametrize("it", [2, 3], ids=["even", "odd"])
def test_dot_product_per_pass(part, it):
    p, g, m = prepared((13, 37, 49), 81)
    x0 = state(m)
    sc = scales(x0)
    d = direction(m.shape, 1, sc)
    lam = direction(m.shape, 2, {n: 1.0 / v for n, v in sc.items()})
    tl = tlm(m, d, it, False, PARTS[part])
    ad = adjoint(m, lam, it, False, PARTS[part])
    after = state(m)
    m.close()
    for n in LIN_FIELDS:        # the context's state is left as it was found
        assert np.array_equal(after[n], x0[n]), f"{n} changed"
    lhs, rhs = dot(tl, lam), dot(d, ad)
    rel = abs(lhs - rhs) / max(abs(lhs), abs(rhs))
    print(f"{part}, iteration {it}: <TL d, l> = {lhs:.15e}  <d, AD l> = {rhs:.15e}  rel {rel:.2e}")
    assert np.isfinite(lhs) and rel <= 1e-12


def test_stage_buffers_must_be_aligned():
    """The dynamics stage kernel reads its input through tensor maps, whose base must lie on a
    16-byte boundary: atjup_gpu_set_stage_buffers refuses a buffer 8 bytes off one
    (ATJUP_ERR_ARG = 1) and keeps the context's own buffers, so the next step leaves the offered
    buffers untouched (NaN) and its own state finite."""
    import ctypes

    import torch
    p, g, m = prepared((13, 37, 49), 83)
    xs = m.state_tensors(LIN_FIELDS)
    stages = [torch.full_like(xs[0], float("nan")) for _ in range(12)]
    spare = torch.full((xs[0].numel() + 2,), float("nan"), dtype=torch.float64, device=xs[0].device)
    ptrs = (ctypes.c_void_p * 12)(*[t.data_ptr() for t in stages])
    ptrs[5] = spare.data_ptr() + 8
    assert m.L.atjup_gpu_set_stage_buffers(m.ctx, ptrs) == 1
    m.step(3, False)
    m.synchronize()
    assert all(bool(torch.isnan(t).all()) for t in stages)
    assert bool(torch.isnan(spare).all())
    assert m.nonfinite_count() == 0
    m.close()


@pytest.mark.parametrize("it", [2, 3], ids=["even", "odd"])
def test_checkpointed_adjoint_equals_recomputed(it):
    """The adjoint that takes the forward step's own RK stage inputs as its checkpoint
    (atjup_gpu_set_stage_buffers, atjup_gpu_iteration_adjoint_ckpt) equals the one that
    recomputes them from the iteration's input, to rounding (<= 1e-12 relative L2 per field: the
    recompute repeats the pressure pass, whose reductions are not bit-reproducible run to run)."""
    import torch
    p, g, m = prepared((13, 37, 49), 83)
    x0 = state(m)
    xs = m.state_tensors(LIN_FIELDS)
    stages = [torch.empty_like(xs[0]) for _ in range(12)]
    m.set_stage_buffers(stages)
    m.step(it, False)
    m.set_stage_buffers(None)
    m.set_state_tensors(xs, names=LIN_FIELDS)
    lam = direction(m.shape, 5, {n: 1.0 / v for n, v in scales(x0).items()})
    a_re = adjoint(m, lam, it, False)
    x = padded(m, [lam[n] for n in LIN_FIELDS])
    m.iteration_adjoint_ckpt(x, stages, it, False)
    a_ck = dict(zip(LIN_FIELDS, unpadded(m, x)))
    m.close()
    worst = {n: _rel(a_ck[n], a_re[n]) for n in LIN_FIELDS}
    print(f"iteration {it}: checkpointed vs recomputed adjoint", {k: f"{v:.1e}" for k, v in worst.items()})
    for n in LIN_FIELDS:
        assert worst[n] <= 1e-12, f"{n}: relative L2 {worst[n]:.3e}"


def test_dot_product_whole_iteration_larger_shell():
    p, g, m = prepared((41, 61, 97), 82)
    sc = scales(state(m))
    for it in (2, 3):
        d = direction(m.shape, 10 + it, sc)
        lam = direction(m.shape, 20 + it, {n: 1.0 / v for n, v in sc.items()})
        lhs, rhs = dot(tlm(m, d, it, False), lam), dot(d, adjoint(m, lam, it, False))
        rel = abs(lhs - rhs) / max(abs(lhs), abs(rhs))
        print(f"41x61x97, iteration {it}: rel {rel:.2e}")
        assert rel <= 1e-12
    m.close()


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def test_transposes_match_numpy_specification():
    p, g, m = prepared((13, 37, 49), 83)
    shape = m.shape
    rng = np.random.Generator(np.random.Philox(key=84))
    lam = {n: rng.standard_normal(shape) for n in LIN_FIELDS}
    # boundary passes on t, u, v, w (p_dyn's adjoint zero: the specification carries t, u, v, w)
    lam_bc = dict(lam, p_dyn=np.zeros(shape))
    got = adjoint(m, lam_bc, 3, False, LIN_BC)
    want = ALIN.bc_T({n: lam[n] for n in ("t", "u", "v", "w")}, g["solid"], lid_u=p.lid_u,
                     top_taper=p.top_taper, pole_fill_rows=p.pole_fill_rows,
                     mount_t_ambient=p.mount_t_ambient)
    for n in ("t", "u", "v", "w"):
        r = _rel(got[n], want[n])
        print(f"bc_T {n}: {r:.2e}")
        assert r <= 1e-12, f"bc_T {n}: {r:.3e}"
    # Shapiro (passes = 1) on u, v, w
    got = adjoint(m, lam, 3, False, LIN_SHAPIRO)
    for n in ("u", "v", "w"):
        want = ALIN.shapiro4_T(lam[n], g["topo"], p.shapiro_strength)
        r = _rel(got[n], want)
        print(f"shapiro4_T {n}: {r:.2e}")
        assert r <= 1e-12, f"shapiro4_T {n}: {r:.3e}"
    # column balance of v
    got = adjoint(m, lam, 3, False, LIN_BALANCE)
    want = ALIN.balance_v_T(lam["v"], g["topo"], g["rad"], p.dr)
    r = _rel(got["v"], want)
    print(f"balance_v_T: {r:.2e}")
    assert r <= 1e-12
    # the pressure pass (an even iteration), aux's incoming adjoint zero; the clamp mask of the
    # base state's source
    lam_p = dict(lam, aux_u=np.zeros(shape), aux_v=np.zeros(shape), aux_w=np.zeros(shape))
    base_aux = [m.download(n) for n in ("aux_u", "aux_v", "aux_w")]
    got = adjoint(m, lam_p, 2, False, LIN_PRESSURE)
    W, den, interior, _, _ = ALIN._press_weights(p, g)
    src = ALIN.pressure_source(p, g, base_aux)
    mask = (np.abs(src) <= p.p_dyn_cap * den).astype(float)
    lp, la = ALIN.pressure_T(lam["p_dyn"], p, g, p.press_sweeps, pass_mask=mask)
    for n, a, b in (("p_dyn", got["p_dyn"], lp), ("aux_u", got["aux_u"], la[0]),
                    ("aux_v", got["aux_v"], la[1]), ("aux_w", got["aux_w"], la[2])):
        r = _rel(a, b)
        print(f"pressure_T {n}: {r:.2e}")
        assert r <= 1e-12, f"pressure_T {n}: {r:.3e}"
    m.close()


def _iterate(m, x, it):
    for n in LIN_FIELDS:
        m.upload(n, x[n])
    m.step(it, False)
    return state(m)


@pytest.mark.parametrize("it", [2, 3], ids=["even", "odd"])
def test_tangent_linear_matches_differences(it):
    p, g, m = prepared((41, 61, 97), 85)
    x0 = state(m)
    sc = scales(x0)
    d = direction(m.shape, 30 + it, sc)
    tl = tlm(m, d, it, False)
    yp = _iterate(m, {n: x0[n] + EPS * d[n] for n in LIN_FIELDS}, it)
    ym = _iterate(m, {n: x0[n] - EPS * d[n] for n in LIN_FIELDS}, it)
    m.close()
    for n in LIN_FIELDS:
        fd = (yp[n] - ym[n]) / (2.0 * EPS)
        if not np.any(fd) and not np.any(tl[n]):
            continue
        r = _rel(tl[n], fd)
        print(f"iteration {it}, {n}: TL vs central difference rel L2 {r:.2e}")
        assert r <= 1e-6, f"{n}: {r:.3e}"


def test_gradient_of_k_iterations_matches_reference_differences(ref_required):
    """K = 3 dry iterations from the dry configuration's state, 8 directions on t, u, v, w."""
    import torch

    import baseline_state as BS
    from atjup_b200.autograd import iterations
    from helpers import dump_fields, dump_grid, dump_params, ref_dump
    K, NDIR = 3, 8
    d = ref_dump("--baseline", "dry", "--iter-fd", f"{NDIR}:{EPS}:{K}")
    assert np.array_equal(d["fd_zm0"], d["fd_zm0_again"])   # the reference's runs repeat exactly
    P, g = dump_params(d, env=BS.ENVS["dry"]), dump_grid(d)
    m = gpu_from(P, g, dump_fields(d))
    im, jm, km = m.shape
    the = g["the"]
    uref = AC.u_ref(the, P.u_0)
    x0 = state(m)
    x = [t.requires_grad_() for t in padded(m, [x0[n] for n in LIN_FIELDS])]
    out = iterations(m, x, K)
    zm = out[3][im - 2, :, : km - 1].mean(dim=1)
    th = torch.tensor(the, device="cuda")
    ur = torch.tensor(uref, device="cuda")
    J = (torch.sin(th) * (zm - ur) ** 2).sum()
    J.backward()
    grad = {n: x[q].grad[:, :, :km].cpu().numpy() for q, n in enumerate(LIN_FIELDS)}
    j0 = AC.loss_from_mean(d["fd_zm0"], the, uref)
    floor = 10.0 * np.finfo(float).eps * abs(j0) / (2.0 * EPS)
    worst = 0.0
    for k in range(NDIR):
        dk = AC.direction(k, m.shape)
        ad = dot(grad, dk, AC.FIELDS)
        jp = AC.loss_from_mean(d[f"fd_zmp_{k}"], the, uref)
        jm_ = AC.loss_from_mean(d[f"fd_zmm_{k}"], the, uref)
        fd = (jp - jm_) / (2.0 * EPS)
        rel = abs(ad - fd) / abs(fd)
        worst = max(worst, rel)
        print(f"direction {k}: adjoint {ad:.12e}  reference central difference {fd:.12e}  "
              f"rel {rel:.2e}")
        assert abs(ad - fd) <= 1e-6 * abs(fd) + floor, f"direction {k}: {rel:.3e}"
    m.close()
    print(f"K = {K}: J {j0:.6e}, rounding floor {floor:.1e}, worst relative difference {worst:.2e}")
