"""The diffusion-step oracle (ins::diffusion, include/ins/diffusion.h)
against the reference and against the numerics it restates: the wall
weights equal the reference's own fd::discretization bit for bit (golden
fixture from the bridge); the operator I~ - lambda L is symmetric; the CG
solve agrees with a dense solve under both preconditioners; the reference's
Chebyshev preconditioner has the residual polynomial of a shifted,
scaled Chebyshev polynomial on the Gershgorin interval (which holds the
spectrum); and the reference's own diffusion test case (test/diffusion.cc:
a parabolic profile between Dirichlet walls under a constant force, the
discrete steady state) is left unchanged by a step."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_wall_weights_match_the_reference(oracle):
    g = np.load(os.path.join(HERE, "golden", "wall_weights.npz"))
    for (shift, res, la, lb, ua, ub), ref in zip(g["cases"], g["weights"]):
        lo = oracle.wall_weights((la, lb), 1 / res, shift)
        up = oracle.wall_weights((ua, ub), -1 / res, 1 - shift)
        assert np.array_equal(np.concatenate([lo, up]), ref)


def _grid(oracle, tag, comp, robin):
    # 1.6 x 0.8 x 0.8, x solid, y solid, z periodic
    g = oracle.geometry(3, [1.6, 0.8, 0.8], [1, 1, 0], tag=tag, refinement=8)
    return oracle.FluidGrid(g, comp, robin)


ROBIN = [((1.0, 0.0), (0.0, 1.0)), ((2.0, 0.5), (1.0, 0.0)), ((0.0, 0.0), (0.0, 0.0))]


@pytest.mark.parametrize("comp", [0, 1, 2])
def test_helmholtz_operator_is_symmetric(oracle, comp):
    fg = _grid(oracle, oracle.TAG_MAC, comp, ROBIN)
    rng = np.random.default_rng(comp)
    a, b = rng.normal(size=fg.size), rng.normal(size=fg.size)
    for op in (0, 2):
        ha = oracle.diffusion_apply(fg, op, a, lam=0.3)
        hb = oracle.diffusion_apply(fg, op, b, lam=0.3)
        assert abs(a @ hb - b @ ha) <= 1e-12 * np.abs(a) @ np.abs(hb)


def test_step_agrees_with_a_dense_solve(oracle):
    fg = _grid(oracle, oracle.TAG_MAC, 1, ROBIN)
    n = fg.size
    dt, mu, gamma = 2e-3, 1.5, 0.5
    lam = dt * mu / 2
    H = np.stack([oracle.diffusion_apply(fg, 2, e, lam=lam) for e in np.eye(n)], axis=1)
    L = np.stack([oracle.diffusion_apply(fg, 0, e) for e in np.eye(n)], axis=1)
    Id = np.stack([oracle.diffusion_apply(fg, 1, e) for e in np.eye(n)], axis=1)
    rng = np.random.default_rng(4)
    u, rhs, f = rng.normal(size=n), rng.normal(size=n), rng.normal(size=n)
    k = gamma * dt
    want = u + np.linalg.solve(H, k * (Id @ f) + k * mu * (L @ u + rhs))
    its = []
    for pc in (oracle.CHEBYSHEV, oracle.JACOBI):
        got, it = oracle.diffusion_step(fg, dt, mu, 1e-13, 1000, gamma, u, rhs, f, precond=pc)
        assert it > 0
        assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
        its.append(it)
    assert its[0] < its[1]          # the polynomial preconditioner needs fewer iterations
    # the Gershgorin interval holds the spectrum of the (symmetric) operator
    lo, hi = oracle.gershgorin(fg, lam)
    ev = np.linalg.eigvalsh((H + H.T) / 2)
    assert lo <= ev.min() + 1e-12 and ev.max() <= hi + 1e-12


def test_chebyshev_weights_give_the_chebyshev_residual_polynomial(oracle):
    """With p(z) = w3 - w2 z + w1 z^2 - w0 z^3 (the reference's Horner loop,
    algo/chebyshev.h:152-167), 1 - z p(z) = T4(s(z)) / T4(s(0)) with s the
    affine map of [lower, upper] onto [-1, 1] (algo/chebyshev.h:9-45)."""
    for lower, upper in ((1.0, 10.6), (0.3, 2.0), (2.5, 7.0)):
        w = oracle.chebyshev_weights(upper, lower)
        z = np.linspace(lower, upper, 101)
        p = w[3] - w[2] * z + w[1] * z ** 2 - w[0] * z ** 3
        s = (2 * z - (lower + upper)) / (upper - lower)
        s0 = -(lower + upper) / (upper - lower)
        T4 = lambda t: 8 * t ** 4 - 8 * t ** 2 + 1
        assert np.abs((1 - z * p) - T4(s) / T4(s0)).max() <= 1e-12


def test_parabolic_steady_state_is_kept(oracle):
    """test/diffusion.cc in 3-D: u = x (L - x) / 2 between Dirichlet walls in
    x (periodic y, z), force mu: the discrete Laplacian with its corrected
    identity is exact for this profile, so a step changes nothing."""
    g = oracle.geometry(3, [1.6, 0.8, 0.8], [1, 0, 0], tag=oracle.TAG_CENTERED, refinement=32)
    fg = oracle.FluidGrid(g, 0, [((1.0, 0.0), (1.0, 0.0))] * 3)
    P = fg.points
    x = (np.arange(P[0]) + fg.shift[0]) / fg.res
    u = np.tile(0.5 * x * (1.6 - x), P[1] * P[2])
    mu = 0.7
    out, _ = oracle.diffusion_step(fg, 1e-3, mu, 1e-11, 1000, 1.0, u, np.zeros_like(u), np.full_like(u, mu))
    assert np.abs(out - u).max() <= 1e-12 * np.abs(u).max()
