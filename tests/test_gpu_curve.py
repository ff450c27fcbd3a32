"""Curve forces for two-dimensional runs (bases::geometry<1>,
forces::tension1d with skalak1d / hookean1d) on the device against the
oracle, through the C ABI.  The tension kernel evaluates the reference's
expressions in its order without contraction and equals the oracle bit for
bit; the geometry's operator products are library GEMMs (summation order
differs: 1e-12 of each quantity's largest value)."""
import ctypes

import numpy as np
import pytest

import torus as T

pytestmark = pytest.mark.gpu

N = 64
MATS = [np.array([[1.2, 0.1], [-0.05, 0.9]]), np.diag([0.8, 1.25]), np.array([[1.0, 0.3], [0.0, 1.1]])]
SHEAR, BULK = 2.5, 0.3


def _to(d, dev):
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in d.items()}


def _pack(curves, key="position"):
    return np.stack([c[key] for c in curves], axis=1).reshape(-1)


@pytest.mark.parametrize("law", [0, 2])
def test_curve_tension_matches_oracle_bit_for_bit(ibk, cuda, oracle, law):
    rng = np.random.default_rng(29)
    n = 30000
    rest = {"tu": rng.normal(size=2 * n), "tuu": rng.normal(size=2 * n), "sigma": rng.uniform(0.5, 1.5, size=n)}
    rest["tu"] = (rest["tu"].reshape(2, n) + np.array([[3.0], [0.0]])).reshape(-1)
    cur = {k: rest[k] + 0.2 * rng.normal(size=rest[k].size) for k in ("tu", "tuu")}
    f = ibk.curve_tension(law, SHEAR, BULK, _to(rest, cuda), _to(cur, cuda)).cpu().numpy()
    assert np.array_equal(f, oracle.curve_tension(law, SHEAR, BULK, rest, cur))


def test_curve_geometry_and_tension_pipeline(ibk, cuda, oracle):
    import torch
    ops, w = T.curve_operators(N), T.curve_weights(N)
    nc = 3
    x0 = _pack([T.curve_shape(N, R=0.8) for _ in range(nc)])
    x1 = _pack([T.curve_shape(N, R=0.8, A=MATS[i], eps=0.03 * (i + 1)) for i in range(nc)])
    for first in (ops[0], None):
        o = [first] + ops[1:]
        plan = ibk.CurvePlan([None if m is None else torch.from_numpy(m).to(cuda) for m in o],
                             torch.from_numpy(w).to(cuda))
        rest, cur = plan.geometry(torch.from_numpy(x0).to(cuda), nc), plan.geometry(torch.from_numpy(x1).to(cuda), nc)
        r_ref, c_ref = oracle.curve_geometry(o, w, x0, nc), oracle.curve_geometry(o, w, x1, nc)
        for k in oracle.CURVE_FIELDS:
            got = cur[k].cpu().numpy()
            assert np.abs(got - c_ref[k]).max() <= 1e-12 * np.abs(c_ref[k]).max(), k
        # balance: near rounding for skalak1d; hookean1d's 1/sqrt(i) is
        # resolved to 1.7e-8 at 64 samples (1.3e-12 at 96, 3e-14 at 128)
        for law, tol in ((0, 1e-12), (2, 1e-7)):
            f = ibk.curve_tension(law, SHEAR, BULK, rest, cur).cpu().numpy()
            f_ref = oracle.curve_tension(law, SHEAR, BULK, r_ref, c_ref)
            assert np.abs(f - f_ref).max() <= 1e-10 * np.abs(f_ref).max()
            F = f.reshape(2, nc, N)
            X = x1.reshape(2, nc, N)
            for c in range(nc):
                scale = np.abs(F[:, c]).sum()
                assert np.abs(F[:, c].sum(axis=1)).max() <= tol * scale
                assert abs((X[0, c] * F[1, c] - X[1, c] * F[0, c]).sum()) <= tol * scale


def test_surface_forces_refuse_a_curve_plan(ibk, cuda):
    import torch
    ops, w = T.curve_operators(N), T.curve_weights(N)
    plan = ibk.CurvePlan([torch.from_numpy(m).to(cuda) for m in ops], torch.from_numpy(w).to(cuda))
    L = ibk.lib()
    s = ibk._Surface()
    buf = torch.zeros(16, dtype=torch.float64, device=cuda)
    assert L.ibk_membrane_dissipation(plan.handle, 1.0, 1, buf.data_ptr(), ctypes.byref(s), buf.data_ptr(),
                                      None) == 1
    assert L.ibk_membrane_bending(plan.handle, plan.handle, 1.0, 0, 1, None, buf.data_ptr(), None,
                                  ctypes.byref(s), buf.data_ptr(), None) == 1
