"""The diffusion solve's oracle pinned to the reference's own solver code:
include/solvers/pcg.h and include/algo/chebyshev.h compiled on the host as
they are, over a shim linalg layer (host vectors, reductions as plain sums in
index order; oracle/ref_solver.cc, oracle/ref_shim_solver/), with the
oracle's matrix-free operator and Gershgorin interval: the reference's
Chebyshev-preconditioned CG gives the oracle's solution bit for bit in the
same number of iterations, and impl::chebw<4> the oracle's weights.  Skipped
where the reference tree (and so the bridge) is absent."""
import numpy as np
import pytest

ROBIN = [((1.0, 0.0), (0.0, 1.0)), ((2.0, 0.5), (1.0, 0.0)), ((1.0, 0.0), (1.0, 0.0))]


@pytest.fixture(scope="module")
def bridge(oracle):
    if oracle.ref_solver() is None:
        pytest.skip("reference tree not available here")
    return oracle


@pytest.mark.parametrize("interval", [(1.0, 10.6), (0.3, 2.0), (2.5, 7.0), (1e-3, 4.0)])
def test_chebyshev_weights_equal_the_reference(bridge, interval):
    lower, upper = interval
    assert np.array_equal(bridge.chebyshev_weights(upper, lower), bridge.ref_chebyshev_weights(upper, lower))


@pytest.mark.parametrize("case", [(3, [1.6, 0.8, 0.8], [1, 1, 0], 8, 0), (3, [4.0, 2.5, 3.5], [1, 0, 1], 5, 1),
                                  (2, [4.0, 2.5], [0, 1], 8, 0), (3, [4.0, 2.5, 3.5], [0, 0, 0], 5, 2)])
def test_chebyshev_pcg_equals_the_reference(bridge, case):
    dims, lengths, solid, refinement, comp = case
    fg = bridge.FluidGrid(bridge.geometry(dims, lengths, solid, tag=bridge.TAG_MAC, refinement=refinement), comp,
                          ROBIN)
    dt, mu, gamma, tol = 4e-3, 1.5, 1.0, 1e-12
    rng = np.random.default_rng(20 + comp)
    rhs = rng.normal(size=fg.size)
    zero = np.zeros(fg.size)
    # u = 0 and f = 0: the step's right-hand side is exactly (k mu) rhs, its
    # output exactly the solve's x
    out, it = bridge.diffusion_step(fg, dt, mu, tol, 10000, gamma, zero, rhs, zero)
    x, applications = bridge.ref_chebpcg(fg, dt * mu / 2, ((gamma * dt) * mu) * rhs, tol)
    assert it > 0 and applications == 3 + 4 * it      # three per preconditioner, one per iteration
    assert np.array_equal(out, x)
