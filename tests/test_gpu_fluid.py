"""The diffusion step on the device (ibk_diffusion_*) against the oracle,
through the C ABI: the operators L, I~ and I~ - lambda L bit for bit (same
expressions, no contraction); a step within the solver's tolerance of the
oracle's (the sums of the CG reductions run in another order); the
reference's parabolic steady state kept; a solve that cannot converge in its
iteration budget reported, not hung."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROBIN = [((1.0, 0.0), (0.0, 1.0)), ((2.0, 0.5), (1.0, 0.0)), ((0.0, 0.0), (0.0, 0.0))]


def _plan(ibk, tag):
    dom = ibk.Domain(ibk.Dimension(1.6, ibk.SOLID), ibk.Dimension(0.8, ibk.SOLID), ibk.Dimension(0.8))
    return ibk.Plan(tag, dom, ibk.Bspline(3), ibk.FP64)


@pytest.mark.parametrize("comp", [0, 1, 2])
def test_operators_match_oracle_bit_for_bit(ibk, cuda, oracle, comp):
    import torch
    plan = _plan(ibk, ibk.Mac(8))
    fg = oracle.FluidGrid(oracle.geometry(3, [1.6, 0.8, 0.8], [1, 1, 0], tag=oracle.TAG_MAC, refinement=8),
                          comp, ROBIN)
    dt, mu = 2e-3, 1.5
    d = ibk.Diffusion(plan, comp, dt, mu, robin=ROBIN)
    assert d.size == fg.size
    u = np.random.default_rng(comp).normal(size=fg.size)
    U = torch.from_numpy(u).to(cuda)
    for op in (0, 1, 2):
        got = d.apply(op, U).cpu().numpy()
        want = oracle.diffusion_apply(fg, op, u, lam=dt * mu / 2)
        assert np.array_equal(got, want), op


@pytest.mark.parametrize("comp,gamma,pc", [(0, 0.5, 0), (1, 1.0, 0), (2, 0.5, 0), (0, 1.0, 1), (2, 0.5, 1)])
def test_step_matches_oracle(ibk, cuda, oracle, comp, gamma, pc):
    import torch
    plan = _plan(ibk, ibk.Mac(8))
    fg = oracle.FluidGrid(oracle.geometry(3, [1.6, 0.8, 0.8], [1, 1, 0], tag=oracle.TAG_MAC, refinement=8),
                          comp, ROBIN)
    dt, mu, tol = 2e-3, 1.5, 1e-12
    d = ibk.Diffusion(plan, comp, dt, mu, tolerance=tol, robin=ROBIN, preconditioner=pc)
    rng = np.random.default_rng(10 + comp)
    u, rhs, f = (rng.normal(size=fg.size) for _ in range(3))
    got = d.step(*(torch.from_numpy(a).to(cuda) for a in (u, rhs, f)), gamma=gamma).cpu().numpy()
    want, it = oracle.diffusion_step(fg, dt, mu, tol, 10000, gamma, u, rhs, f, precond=pc)
    assert d.iterations > 0 and abs(d.iterations - it) <= 2
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()


def test_parabolic_steady_state_is_kept(ibk, cuda):
    import torch
    dom = ibk.Domain(ibk.Dimension(1.6, ibk.SOLID), ibk.Dimension(0.8), ibk.Dimension(0.8))
    plan = ibk.Plan(ibk.Centered(32), dom, ibk.Bspline(3), ibk.FP64)
    info = plan.info
    P = [info.points[0][a] for a in range(3)]
    x = (np.arange(P[0]) + info.shift[0][0]) / info.resolution
    u = np.tile(0.5 * x * (1.6 - x), P[1] * P[2])
    mu = 0.7
    d = ibk.Diffusion(plan, 0, 1e-3, mu)
    U = torch.from_numpy(u).to(cuda)
    out = d.step(U, torch.zeros_like(U), torch.full_like(U, mu)).cpu().numpy()
    assert np.abs(out - u).max() <= 1e-12 * np.abs(u).max()


def test_budget_exhausted_is_reported(ibk, cuda):
    import torch
    plan = _plan(ibk, ibk.Mac(8))
    d = ibk.Diffusion(plan, 0, 2e-3, 1.5, tolerance=1e-30, max_iterations=2, robin=ROBIN)
    u = torch.randn(d.size, dtype=torch.float64, device=cuda)
    with pytest.raises(ibk.IbkError):
        d.step(u, u, u)
    # the device stays usable
    assert torch.isfinite(d.apply(2, u)).all()


# Grids whose sizes leave partial operator blocks on every axis (blocks of 32
# x 8 columns marching 16 planes): 40 x 25 x 35 faces, periodic or walled,
# and a two-dimensional grid.
EDGE_CASES = [(3, [4.0, 2.5, 3.5], [0, 0, 0]), (3, [4.0, 2.5, 3.5], [1, 0, 1]), (3, [4.0, 2.5, 3.5], [0, 1, 0]),
              (2, [4.0, 2.5], [0, 1])]
ROBIN_WALLS = [((1.0, 0.0), (0.0, 1.0)), ((2.0, 0.5), (1.0, 0.0)), ((1.0, 0.0), (1.0, 0.0))]


@pytest.mark.parametrize("case", range(len(EDGE_CASES)))
def test_operators_on_ragged_grids_match_oracle_bit_for_bit(ibk, cuda, oracle, case):
    import torch
    dims, lengths, solid = EDGE_CASES[case]
    dom = ibk.Domain(*[ibk.Dimension(l, ibk.SOLID if s else ibk.PERIODIC) for l, s in zip(lengths, solid)])
    plan = ibk.Plan(ibk.Mac(5), dom, ibk.Bspline(3), ibk.FP64)
    dt, mu = 2e-3, 1.5
    for comp in range(dims):
        fg = oracle.FluidGrid(oracle.geometry(dims, lengths, solid, tag=oracle.TAG_MAC, refinement=5), comp, ROBIN_WALLS)
        d = ibk.Diffusion(plan, comp, dt, mu, robin=ROBIN_WALLS)
        assert d.size == fg.size
        u = np.random.default_rng(100 + 10 * case + comp).normal(size=fg.size)
        U = torch.from_numpy(u).to(cuda)
        for op in (0, 1, 2):
            assert np.array_equal(d.apply(op, U).cpu().numpy(), oracle.diffusion_apply(fg, op, u, lam=dt * mu / 2)), \
                (comp, op)


@pytest.mark.parametrize("case", [1, 3])
def test_step_on_ragged_grids_matches_oracle(ibk, cuda, oracle, case):
    import torch
    dims, lengths, solid = EDGE_CASES[case]
    dom = ibk.Domain(*[ibk.Dimension(l, ibk.SOLID if s else ibk.PERIODIC) for l, s in zip(lengths, solid)])
    plan = ibk.Plan(ibk.Mac(5), dom, ibk.Bspline(3), ibk.FP64)
    fg = oracle.FluidGrid(oracle.geometry(dims, lengths, solid, tag=oracle.TAG_MAC, refinement=5), 0, ROBIN_WALLS)
    dt, mu, tol = 2e-3, 1.5, 1e-12
    d = ibk.Diffusion(plan, 0, dt, mu, tolerance=tol, robin=ROBIN_WALLS)
    rng = np.random.default_rng(40 + case)
    u, rhs, f = (rng.normal(size=fg.size) for _ in range(3))
    got = d.step(*(torch.from_numpy(a).to(cuda) for a in (u, rhs, f)), gamma=1.0).cpu().numpy()
    want, it = oracle.diffusion_step(fg, dt, mu, tol, 10000, 1.0, u, rhs, f)
    assert d.iterations > 0 and abs(d.iterations - it) <= 2
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()


def test_degenerate_wall_is_rejected(ibk, cuda):
    plan = _plan(ibk, ibk.Mac(8))
    bad = [((0.0, 0.0), (0.0, 1.0)), ((1.0, 0.0), (1.0, 0.0)), ((0.0, 0.0), (0.0, 0.0))]   # x lower wall: a = b = 0
    with pytest.raises(ibk.IbkError):
        ibk.Diffusion(plan, 0, 2e-3, 1.5, robin=bad)


@pytest.mark.parametrize("case", range(len(EDGE_CASES)))
def test_chebyshev_interval_and_weights_match_oracle(ibk, cuda, oracle, case):
    """The device's Gershgorin interval (a min / max over the rows, exact in
    any order) and the host's Chebyshev weights equal the oracle's bit for
    bit."""
    dims, lengths, solid = EDGE_CASES[case]
    dom = ibk.Domain(*[ibk.Dimension(l, ibk.SOLID if s else ibk.PERIODIC) for l, s in zip(lengths, solid)])
    plan = ibk.Plan(ibk.Mac(5), dom, ibk.Bspline(3), ibk.FP64)
    dt, mu = 2e-3, 1.5
    for comp in range(dims):
        fg = oracle.FluidGrid(oracle.geometry(dims, lengths, solid, tag=oracle.TAG_MAC, refinement=5), comp,
                              ROBIN_WALLS)
        (lo, hi), w = ibk.Diffusion(plan, comp, dt, mu, robin=ROBIN_WALLS).info()
        want = oracle.gershgorin(fg, dt * mu / 2)
        assert (lo, hi) == (want[0], want[1])
        assert np.array_equal(np.array(w), oracle.chebyshev_weights(hi, lo))
