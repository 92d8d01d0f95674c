"""The articulated torsional/rolling friction block (wgsl.js:2655-2930: t1, t2, spin, roll1, roll2 on
the elliptic or pyramidal cone) checked against the problem it solves, not against a copy of its
code: the oracle's block (o_cone5.h, the same source as the CUDA solver's cone5.cuh, so GPU parity
alone cannot catch a mistake in it) must return the minimizer of the rows' quadratic model over
the cone, as computed here independently in float64.

Model: with the rows' 5x5 response H, velocity residual g at the current impulses lam and the
coefficients mu, the block minimizes f(x) = g.(x - lam) + 1/2 (x - lam).H.(x - lam) over the cone
{x : |x / mu| <= load} (elliptic) or {x : |x01 / mu01| + |x2 / mu2| + |x34 / mu34| <= load}
(pyramidal), with relaxation 1 and no creep. Checked: the analytic sticking case (interior
minimizer lam - H^-1 g), sliding on the ball (the trust-region solution and its KKT conditions),
and the pyramid's faces (the objective of an accelerated projected-gradient solve)."""
import numpy as np
import pytest

from oracle import oracle as orc


def _problem(rng, scale_g):
    A = rng.normal(size=(5, 5))
    H = A @ A.T / 5 + 0.2 * np.eye(5)
    H = (H + H.T) / 2
    mu = rng.uniform(0.3, 1.0, 5)
    load = float(rng.uniform(0.5, 2.0))
    y0 = rng.normal(size=5)
    y0 *= 0.5 * load / np.linalg.norm(y0)
    lam = (mu * y0).astype(np.float32)
    g = scale_g * rng.normal(size=5)
    return H.astype(np.float32), g.astype(np.float32), mu.astype(np.float32), lam, np.float32(load)


def _f(x, H, g, lam):
    d = np.asarray(x, np.float64) - np.asarray(lam, np.float64)
    return float(np.asarray(g, np.float64) @ d + 0.5 * d @ np.asarray(H, np.float64) @ d)


def _ball_solution(H, g, mu, lam, load):
    """Trust-region subproblem in y = x / mu, in float64: the unconstrained minimizer if inside the
    ball, else (Hy + nu I) y = Hy y0 - gy with |y| = load, nu by bisection."""
    H, g, mu, lam = (np.asarray(v, np.float64) for v in (H, g, mu, lam))
    D = np.diag(mu)
    Hy, gy, y0 = D @ H @ D, mu * g, lam / mu
    rhs = Hy @ y0 - gy
    y = np.linalg.solve(Hy, rhs)
    if np.linalg.norm(y) <= load:
        return mu * y, 0.0
    lo, hi = 0.0, 1.0
    while np.linalg.norm(np.linalg.solve(Hy + hi * np.eye(5), rhs)) > load:
        hi *= 2
    for _ in range(200):
        nu = 0.5 * (lo + hi)
        if np.linalg.norm(np.linalg.solve(Hy + nu * np.eye(5), rhs)) > load:
            lo = nu
        else:
            hi = nu
    return mu * np.linalg.solve(Hy + hi * np.eye(5), rhs), hi


def _group_l1_project(z, load):
    groups = [[0, 1], [2], [3, 4]]
    n = np.array([np.linalg.norm(z[gp]) for gp in groups])
    if n.sum() <= load:
        return z.copy()
    lo, hi = 0.0, n.max()
    for _ in range(60):
        th = 0.5 * (lo + hi)
        if np.maximum(n - th, 0).sum() > load:
            lo = th
        else:
            hi = th
    out = z.copy()
    for gp, ng in zip(groups, n):
        out[gp] = z[gp] * (max(ng - hi, 0.0) / ng if ng > 0 else 0.0)
    return out


def _pyramid_solution(H, g, mu, lam, load, iters=3000):
    """Accelerated projected gradient (FISTA) in y = x / mu over the group-l1 ball, float64."""
    H, g, mu, lam = (np.asarray(v, np.float64) for v in (H, g, mu, lam))
    D = np.diag(mu)
    Hy, gy, y0 = D @ H @ D, mu * g, lam / mu
    step = 1.0 / np.linalg.eigvalsh(Hy).max()
    y = _group_l1_project(y0, load)
    z, t = y.copy(), 1.0
    for _ in range(iters):
        y_new = _group_l1_project(z - step * (gy + Hy @ (z - y0)), load)
        t_new = 0.5 * (1 + np.sqrt(1 + 4 * t * t))
        z = y_new + ((t - 1) / t_new) * (y_new - y)
        y, t = y_new, t_new
    return mu * y


@pytest.mark.parametrize("seed", range(6))
def test_sticking_is_the_unconstrained_minimizer(seed, oracle_lib):
    rng = np.random.default_rng(100 + seed)
    H, g, mu, lam, load = _problem(rng, 1e-3)
    x = orc.cone5(H, g, mu, lam, load)
    want = lam.astype(np.float64) - np.linalg.solve(H.astype(np.float64), g.astype(np.float64))
    assert np.linalg.norm((want / mu)) < load
    np.testing.assert_allclose(x, want, rtol=0, atol=1e-5 * max(1.0, np.abs(want).max()))


@pytest.mark.parametrize("seed", range(12))
def test_sliding_on_the_ball_meets_kkt(seed, oracle_lib):
    rng = np.random.default_rng(200 + seed)
    H, g, mu, lam, load = _problem(rng, 20.0)
    x = orc.cone5(H, g, mu, lam, load).astype(np.float64)
    want, nu = _ball_solution(H, g, mu, lam, load)
    assert nu > 0, "the case must slide"
    y = x / mu
    assert abs(np.linalg.norm(y) - load) <= 1e-4 * load, "not on the cone's surface"
    # KKT in y: the gradient mu * (g + H (x - lam)) is -nu y with nu >= 0.
    grad = mu * (g.astype(np.float64) + H.astype(np.float64) @ (x - lam))
    nu_x = -(grad @ y) / (y @ y)
    assert nu_x > 0
    assert np.linalg.norm(grad + nu_x * y) <= 2e-3 * np.linalg.norm(grad)
    np.testing.assert_allclose(x, want, rtol=0, atol=2e-4 * np.abs(want).max())
    assert _f(x, H, g, lam) <= _f(want, H, g, lam) + 1e-5 * abs(_f(want, H, g, lam))


@pytest.mark.parametrize("seed", range(8))
def test_pyramid_faces_reach_the_minimum(seed, oracle_lib):
    rng = np.random.default_rng(300 + seed)
    H, g, mu, lam, load = _problem(rng, 20.0)
    x = orc.cone5(H, g, mu, lam, load, pyramidal=True).astype(np.float64)
    y = x / mu
    norm = np.linalg.norm(y[:2]) + abs(y[2]) + np.linalg.norm(y[3:])
    assert norm <= load * (1 + 1e-5), "outside the pyramid"
    want = _pyramid_solution(H, g, mu, lam, load)
    f_x, f_w = _f(x, H, g, lam), _f(want, H, g, lam)
    assert f_w < _f(lam, H, g, lam), "the case must move"
    assert f_x <= f_w + 1e-3 * abs(f_w), (f_x, f_w)
