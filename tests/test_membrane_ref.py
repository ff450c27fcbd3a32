"""The membrane-force oracle pinned to the reference's own force code:
include/forces/{skalak,neohookean,hookean,bending,dissipation,tether}.h and
tension1d (skalak1d, hookean1d) compiled on the host as they are, over shim
containers for the geometry and operators (oracle/ref_forces.cc,
oracle/ref_shim_forces/), fed the same geometry as the oracle: every force
equals the restatement bit for bit.  Skipped where the reference tree (and so
the bridge) is absent."""
import numpy as np
import pytest

import torus as T

A = np.array([[1.3, 0.2, 0.0], [0.0, 0.8, 0.1], [0.05, 0.0, 1.1]])
NU, NV, NC = 24, 12, 2


@pytest.fixture(scope="module")
def shapes(oracle):
    if oracle.ref_forces() is None:
        pytest.skip("reference tree not available here")
    w = T.weights(NU, NV)
    ops = T.operators(NU, NV)
    x0 = T.pack([T.shape(NU, NV, R=2.0, r=0.7) for _ in range(NC)])["position"]
    x1 = T.pack([T.shape(NU, NV, R=2.0, r=0.7, A=A, eps=0.03 * (i + 1)) for i in range(NC)])["position"]
    rest, cur = oracle.surface_geometry(ops, w, x0, NC), oracle.surface_geometry(ops, w, x1, NC)
    return w, ops, x0, x1, rest, cur


@pytest.mark.parametrize("law", [0, 1, 2])
def test_tension_equals_the_reference(oracle, shapes, law):
    _, _, _, _, rest, cur = shapes
    assert np.array_equal(oracle.membrane_tension(law, 2.5, 25.0, rest, cur),
                          oracle.ref_membrane_tension(law, 2.5, 25.0, rest, cur))
    # random (valid) geometry as well
    rng = np.random.default_rng(5 + law)
    n = 2000
    base = {k: rng.normal(size=3 * n) for k in ("tu", "tv", "tuu", "tuv", "tvv")}
    base["tu"] = (base["tu"].reshape(3, n) + np.array([[2.0], [0.0], [0.0]])).reshape(-1)
    base["tv"] = (base["tv"].reshape(3, n) + np.array([[0.0], [2.0], [0.0]])).reshape(-1)
    base["sigma"] = rng.uniform(0.5, 1.5, size=n)
    moved = {k: v + 0.1 * rng.normal(size=v.size) for k, v in base.items()}
    assert np.array_equal(oracle.membrane_tension(law, 2.5, 25.0, base, moved),
                          oracle.ref_membrane_tension(law, 2.5, 25.0, base, moved))


@pytest.mark.parametrize("preferred", [False, True])
def test_bending_equals_the_reference(oracle, shapes, preferred):
    w, ops, x0, x1, rest, cur = shapes
    dops = [None] + ops[1:]
    data_rest, data_cur = oracle.surface_geometry(dops, w, x0, NC), oracle.surface_geometry(dops, w, x1, NC)
    got = oracle.membrane_bending(dops, w, ops, 0.7, preferred, x0, x1, rest, cur, NC)
    assert np.array_equal(got, oracle.ref_membrane_bending(ops, 0.7, preferred, data_rest, data_cur, rest, cur, NC))


def test_dissipation_and_tether_equal_the_reference(oracle, shapes):
    _, ops, x0, x1, _, cur = shapes
    u = np.random.default_rng(1).normal(size=x1.size)
    assert np.array_equal(oracle.membrane_dissipation(ops, 0.7, u, cur, NC),
                          oracle.ref_membrane_dissipation(ops, 0.7, u, cur, NC))
    assert np.array_equal(oracle.membrane_tether(3.0, x0, x1), oracle.ref_membrane_tether(3.0, x0, x1))


@pytest.mark.parametrize("law", [0, 2])
def test_curve_tension_equals_the_reference(oracle, law):
    if oracle.ref_forces() is None:
        pytest.skip("reference tree not available here")
    n = 64
    ops, w = T.curve_operators(n), T.curve_weights(n)
    rest = oracle.curve_geometry(ops, w, T.curve_shape(n)["position"].reshape(-1), 1)
    cur = oracle.curve_geometry(ops, w, T.curve_shape(n, A=np.array([[1.2, 0.1], [-0.05, 0.9]]),
                                                        eps=0.05)["position"].reshape(-1), 1)
    assert np.array_equal(oracle.curve_tension(law, 2.5, 0.3, rest, cur),
                          oracle.ref_curve_tension(law, 2.5, 0.3, rest, cur))
