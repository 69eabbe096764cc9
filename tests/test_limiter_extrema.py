"""The cell limiter's theta from nodal extrema equals the all-node minimum.

The reference takes theta = min(1, min over nodes of alpha(d)) with the
Venkatakrishnan / Barth-Jespersen ratio
alpha = (D^2 + 2 D d + eps^2) / (D^2 + 2 d^2 + D d + eps^2)
(src/solver.mojo:384-530, src/local_mesh_2d_gpu_limiter.mojo:74-153).  The
product's theta pass evaluates alpha only at each side's largest deviation,
read from the least / largest nodal value that the means pass keeps
(limiter.cuh).  This checks that rule against the all-node minimum on random
node sets in FP32 and FP64, bit for bit, with the same operation order as
the kernels; it runs on the CPU and touches no product code.
"""
import numpy as np
import pytest


def _alpha(D, da, eps2, dt):
    D2, d2, Dd = D * D, da * da, D * da
    return (D2 + dt(2) * Dd + eps2) / (D2 + dt(2) * d2 + Dd + eps2)


def _theta_all_nodes(u, own, lo, hi, eps2, dt):
    tiny = dt(1e-30)
    pD = np.maximum(hi - own, dt(0))
    nD = np.maximum(own - lo, dt(0))
    dl = (u - own[:, None]).astype(dt)
    da = np.abs(dl)
    D = np.where(dl > 0, pD[:, None], nD[:, None]).astype(dt)
    al = _alpha(D, da, eps2[:, None], dt).astype(dt)
    al = np.where(da <= tiny, dt(1), al)
    return np.minimum(dt(1), al.min(axis=1))


def _theta_extrema(u, own, lo, hi, eps2, dt):
    tiny = dt(1e-30)
    pD = np.maximum(hi - own, dt(0))
    nD = np.maximum(own - lo, dt(0))
    dp = (u.max(axis=1) - own).astype(dt)
    dn = (own - u.min(axis=1)).astype(dt)
    th = np.ones_like(own)
    ap = _alpha(pD, dp, eps2, dt).astype(dt)
    an = _alpha(nD, dn, eps2, dt).astype(dt)
    th = np.where((dp > tiny) & (ap < th), ap, th)
    th = np.where((dn > tiny) & (an < th), an, th)
    return th


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("NP", [3, 10, 21, 35, 56])
def test_theta_from_extrema_matches_all_nodes(dt, NP):
    rng = np.random.default_rng(1000 + NP)
    n = 20000
    scale = rng.choice([1e-3, 1e-1, 1.0, 10.0], size=n)
    u = (rng.standard_normal((n, NP)) * scale[:, None] + rng.standard_normal(n)[:, None]).astype(dt)
    own = u.mean(axis=1).astype(dt)
    spread = rng.choice([1e-3, 0.1, 1.0], size=n)
    nb = (own[:, None] + rng.standard_normal((n, 4)) * spread[:, None]).astype(dt)
    lo = np.minimum(own, nb.min(axis=1)).astype(dt)
    hi = np.maximum(own, nb.max(axis=1)).astype(dt)
    eps = rng.choice([0.0, 1e-2, 5e-2, 0.1], size=n).astype(dt)
    eps2 = (eps * eps).astype(dt)
    with np.errstate(invalid="ignore", divide="ignore"):
        a = _theta_all_nodes(u, own, lo, hi, eps2, dt)
        b = _theta_extrema(u, own, lo, hi, eps2, dt)
    assert (a < 1).mean() > 0.2  # the limiter is active on a good share of the sets
    np.testing.assert_array_equal(a, b)
