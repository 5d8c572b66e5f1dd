"""Shared pieces of the RK4 tangent-linear / adjoint tests: seeded perturbation directions of
the dry state and the zonal-jet loss at the top level. Test infrastructure only.

The loss is the one of the dry adjoint configuration: J = sum_j sin(the_j) (<w>_phi(i_top, j) -
u_ref(the_j))^2 with the_j the colatitude, <w>_phi the mean over the km - 1 distinct meridians of
the zonal wind w at the last integrated level i_top = im - 2, and u_ref(the) = sum_{n=1..8} a_n
sin(n the) with a_n ~ U(-50, 150) m/s (seeded), divided by u_0 into model units."""
import numpy as np

FIELDS = ("t", "u", "v", "w")
# a direction is N(0, 1) in every cell of every field (model units, where t and w are of order 1):
# eps d with eps = 1e-6 is then a relative perturbation of 1e-6, large enough against the
# rounding of the loss and small enough for the central difference's truncation
UREF_SEED = 20261204
DIR_SEED = 20261205


def direction(k, shape, seed=DIR_SEED):
    rng = np.random.Generator(np.random.Philox(key=seed + k))
    return {f: rng.standard_normal(shape) for f in FIELDS}


def u_ref(the, u_0, seed=UREF_SEED):
    a = np.random.Generator(np.random.Philox(key=seed)).uniform(-50.0, 150.0, 8) / u_0
    n = np.arange(1, 9)
    return (a[None, :] * np.sin(n[None, :] * np.asarray(the)[:, None])).sum(axis=1)


def zonal_mean_top(w):
    im, jm, km = w.shape
    return w[im - 2, :, : km - 1].mean(axis=1)


def loss_from_mean(zm, the, uref):
    return float((np.sin(the) * (zm - uref) ** 2).sum())


def loss(w, the, uref):
    return loss_from_mean(zonal_mean_top(w), the, uref)


def loss_adjoint_w(w, the, uref):
    """dJ/dw (im, jm, km): nonzero on the top level's distinct meridians"""
    im, jm, km = w.shape
    g = np.zeros(w.shape)
    zm = zonal_mean_top(w)
    g[im - 2, :, : km - 1] = (2.0 * np.sin(the) * (zm - uref) / (km - 1))[:, None]
    return g
