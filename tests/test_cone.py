"""The in-loop projection of the wind around the obstacle (projectAroundObstacle(in_loop = true),
InitValues_Jup.cpp:1595-1822, every ATJUP_CONE_PROJ_STRIDE iterations at cJupiterModel.cpp:1362).

* CPU: the kernel's schedule -- lexicographic SOR replayed as a pipelined anti-diagonal wavefront,
  with the snapshot it returns to when a sweep converges after later sweeps have started --
  gives plain lexicographic SOR's phi and sweep count bit for bit, on random boxes with solid,
  wall and near cells (a Python statement of the schedule, not of the kernel's code).
* GPU, against the reference: from the dry configuration's state before iteration 1 and after
  iterations 3 and 8 (the reference's own u, v, w at each), one call each on the same context, so
  the second and third are warm-started from the phi of the one before: v and w equal the
  reference's bit for bit, u is untouched, and the largest sweep count equals the one the
  reference printed.
* GPU, in the loop: the dry configuration with ATJUP_CONE_PROJ_STRIDE=5 over 20 iterations
  (projections at 5, 10, 15 and 20; the configuration's own stride, the reference's default 10,
  is in tests/test_baseline_configs.py), every field within the FP64 bar of 1e-10 relative L2.
* CPU, against the reference: the oracle's restatement (ora_cone_project) on the same three calls
  as the GPU test, bit for bit.
"""
import math
import random

import numpy as np
import pytest

from helpers import dump_fields, dump_grid, dump_params, gpu_from, ref_dump, rel_l2

OMEGA, TOL, MAXIT = 1.9, 1.0e-10, 40000
DTHE = DPHI = math.pi / 180.0


def _case(nj, nk, seed):
    """A box with a halo: solid flags (halo included), near flags, row sines, per-cell v, w and
    divergence source, and a warm-start phi (zero on the halo)."""
    rnd = random.Random(seed)
    solid = [[rnd.random() < 0.15 for _ in range(nk + 2)] for _ in range(nj + 2)]
    near = [[rnd.random() < 0.3 for _ in range(nk)] for _ in range(nj)]
    s = [0.55 + 0.45 * rnd.random() for _ in range(nj + 2)]
    cst = [[(rnd.gauss(0, 1e-3), rnd.gauss(0, 1e-3), rnd.gauss(0, 1e-4)) for _ in range(nk)]
           for _ in range(nj)]
    phi = [[0.0] * (nk + 2) for _ in range(nj + 2)]
    for x in range(1, nj + 1):
        for y in range(1, nk + 1):
            phi[x][y] = rnd.gauss(0, 1e-3) if rnd.random() < 0.5 else 0.0
    return solid, near, s, cst, phi


def _update(phi, case, a, b, div):
    """One cell's SOR update in the reference's order of operations
    (InitValues_Jup.cpp:1739-1758); None for a skipped cell, else (|change|, |phi|)."""
    solid, near, s, cst, _ = case
    x, y = a + 1, b + 1
    if solid[x][y]:
        return None
    sj = s[x]
    aN = 0.5 * (sj + s[x - 1]) / (DTHE * DTHE)
    aS = 0.5 * (sj + s[x + 1]) / (DTHE * DTHE)
    aL = 1.0 / (sj * DPHI * DPHI)
    vp, wp, g = cst[a][b]
    A = B = 0.0
    if div and near[a][b]:
        if not solid[x - 1][y]:
            A += aN
            B += aN * phi[x - 1][y]
        if not solid[x + 1][y]:
            A += aS
            B += aS * phi[x + 1][y]
        if not solid[x][y - 1]:
            A += aL
            B += aL * phi[x][y - 1]
        if not solid[x][y + 1]:
            A += aL
            B += aL * phi[x][y + 1]
        B += g
    else:
        if solid[x - 1][y]:
            B -= aN * DTHE * (-vp)
        else:
            A += aN
            B += aN * phi[x - 1][y]
        if solid[x + 1][y]:
            B -= aS * DTHE * (vp)
        else:
            A += aS
            B += aS * phi[x + 1][y]
        if solid[x][y - 1]:
            B -= aL * sj * DPHI * (-wp)
        else:
            A += aL
            B += aL * phi[x][y - 1]
        if solid[x][y + 1]:
            B -= aL * sj * DPHI * (wp)
        else:
            A += aL
            B += aL * phi[x][y + 1]
    if not (A > 0.0):
        return None
    p = phi[x][y]
    pn = p + OMEGA * (B / A - p)
    phi[x][y] = pn
    return abs(pn - p), abs(pn)


def _lexicographic(case, nj, nk, div):
    """The reference's loop (InitValues_Jup.cpp:1726-1762)."""
    phi = [r[:] for r in case[4]]
    for it in range(1, MAXIT + 1):
        dmax = pmax = 0.0
        for a in range(nj):
            for b in range(nk):
                r = _update(phi, case, a, b, div)
                if r:
                    dmax, pmax = max(dmax, r[0]), max(pmax, r[1])
        if dmax <= TOL * max(pmax, 1.0e-30):
            return phi, it
    return phi, MAXIT + 1


def _wavefront(case, nj, nk, div, snap_every):
    """The kernel's schedule: step tau updates diagonal tau - 2(t-1) of every sweep t in flight,
    folds each sweep's maxima into ring slot t % R, tests sweep t after step D + 2(t-1), and on
    convergence returns to the newest snapshot with no cell past that sweep and replays."""
    phi = [r[:] for r in case[4]]
    D = nj + nk - 2
    R = D // 2 + 2
    n_snap = (D + snap_every) // snap_every + 2
    ring = [[0.0, 0.0] for _ in range(R)]
    snaps = [[r[:] for r in phi]] + [None] * (n_snap - 1)
    tags = [-1] + [None] * (n_snap - 1)
    nxt = 1 % n_snap

    def step(tau, t_stop, reduce):
        t_hi = min(t_stop, tau // 2 + 1)
        t_lo = 1 if tau <= D else (tau - D + 1) // 2 + 1
        for t in range(t_lo, t_hi + 1):
            d = tau - 2 * (t - 1)
            dm = pm = 0.0
            for a in range(max(0, d - (nk - 1)), min(d, nj - 1) + 1):
                r = _update(phi, case, a, d - a, div)
                if r:
                    dm, pm = max(dm, r[0]), max(pm, r[1])
            if reduce:
                sl = ring[t % R]
                sl[:] = [dm, pm] if d == 0 else [max(sl[0], dm), max(sl[1], pm)]

    tau, t_conv = 0, 0
    while True:
        step(tau, MAXIT, True)
        if tau >= D and (tau - D) % 2 == 0:
            t = (tau - D) // 2 + 1
            if ring[t % R][0] <= TOL * max(ring[t % R][1], 1.0e-30):
                t_conv = t
                break
            if t == MAXIT:
                return phi, MAXIT + 1
        if tau % snap_every == snap_every - 1:
            snaps[nxt], tags[nxt] = [r[:] for r in phi], tau
            nxt = (nxt + 1) % n_snap
        tau += 1
    target = 2 * (t_conv - 1)
    best = max((x for x in range(n_snap) if tags[x] is not None and tags[x] <= target),
               key=lambda x: tags[x])
    phi[:] = [r[:] for r in snaps[best]]
    for tau in range(tags[best] + 1, D + 2 * (t_conv - 1) + 1):
        step(tau, t_conv, False)
    return phi, t_conv


@pytest.mark.parametrize("seed", range(8))
def test_wavefront_schedule_is_lexicographic_sor(seed):
    rnd = random.Random(1000 + seed)
    nj, nk = rnd.randint(1, 13), rnd.randint(1, 15)
    case = _case(nj, nk, seed)
    for div in (False, True):
        p0, i0 = _lexicographic(case, nj, nk, div)
        p1, i1 = _wavefront(case, nj, nk, div, snap_every=4 + seed)
        assert i0 == i1, f"sweeps {i0} vs {i1}"
        assert p0 == p1, "phi differs"


@pytest.mark.gpu
@pytest.mark.slow
def test_gpu_cone_projection_bit_exact(ref_required):
    import baseline_state as BS
    calls = (0, 3, 8)
    d = ref_dump("--baseline", "dry", "--iters", "8", "--cone-at", ",".join(map(str, calls)))
    P = dump_params(d, env=BS.DRY_ENV)
    m = gpu_from(P, dump_grid(d), dump_fields(d))
    try:
        for tag in calls:
            for n in ("u", "v", "w"):
                m.upload(n, d[f"cone{tag}_pre_{n}"])
            m.cone_project()
            levels, sweeps = m.cone_stats()
            assert levels.size > 0 and (sweeps[:, 1] > 0).all()
            assert int(sweeps.max()) == int(d[f"cone{tag}_itmax"]), (
                f"call after iteration {tag}: largest sweep count {sweeps.max()} vs the "
                f"reference's {int(d[f'cone{tag}_itmax'])}")
            for n in ("v", "w"):
                got, want = m.download(n), d[f"cone{tag}_post_{n}"]
                assert np.array_equal(got, want), (
                    f"call after iteration {tag}: {n} differs in {np.sum(got != want)} cells, "
                    f"largest {np.max(np.abs(got - want)):.3e}")
            assert np.array_equal(m.download("u"), d[f"cone{tag}_pre_u"])
            print(f"projection after iteration {tag}: {levels.size} levels, sweeps per solve "
                  f"{sweeps.min()}..{sweeps.max()}: bit-identical")
    finally:
        m.close()


@pytest.mark.gpu
@pytest.mark.slow
def test_gpu_dry_config_with_cone_projection(ref_required):
    import baseline_state as BS
    env = {**BS.DRY_ENV, "ATJUP_CONE_PROJ_STRIDE": "5"}
    d = ref_dump("--baseline", "dry", "--iters", "20", "--env", "ATJUP_CONE_PROJ_STRIDE=5")
    P = dump_params(d, env=env)
    assert P.cone_proj_stride == 5 and P.cone_proj_div == 3 and P.cone_proj_margin == 40
    m = gpu_from(P, dump_grid(d), dump_fields(d))
    try:
        for it in range(1, 21):
            m.step(it, it == 1)
        names = ("t", "u", "v", "w", "p_dyn", "p_hydro", "rho_mix")
        worst = {n: rel_l2(m.download(n), d["out_" + n]) for n in names}
        assert m.nonfinite_count() == 0
    finally:
        m.close()
    print("dry configuration with the projection every 5 iterations, 20 iterations vs reference:",
          {k: f"{v:.1e}" for k, v in worst.items()})
    for n in names:
        assert worst[n] <= 1e-10, f"{n}: relative L2 {worst[n]:.3e}"


@pytest.mark.slow
def test_oracle_cone_projection_bit_exact(ref_required):
    """The oracle's restatement (ora_cone_project) against the reference: the same three calls as
    the GPU test, the second and third warm-started, bit for bit, with the reference's sweeps."""
    import baseline_state as BS
    from helpers import oracle_from
    calls = (0, 3, 8)
    d = ref_dump("--baseline", "dry", "--iters", "8", "--cone-at", ",".join(map(str, calls)))
    P = dump_params(d, env=BS.DRY_ENV)
    o = oracle_from(P, dump_grid(d), dump_fields(d))
    for tag in calls:
        for n in ("u", "v", "w"):
            o.f[n][...] = d[f"cone{tag}_pre_{n}"]
        sweeps = o.cone_project()
        assert int(sweeps.max()) == int(d[f"cone{tag}_itmax"])
        for n in ("v", "w"):
            assert np.array_equal(o.f[n], d[f"cone{tag}_post_{n}"]), f"call after {tag}: {n}"
