"""The curve-force oracle (bases::geometry<1> and forces::tension1d under the
skalak1d and hookean1d laws; include/bases/geometry.h, include/forces/
tension.h:120-205) against the mechanics it restates, on closed curves with
analytic geometry and exact Fourier differentiation: no force at rest, zero
total force and torque on a closed curve, the uniform inward pull
weight * stretch * phi(stretch^2) on a dilated circle, forces that rotate
with the curve.  Plus the library's argument checks (no device work)."""
import ctypes

import numpy as np
import pytest

import torus as T

N = 64
A = np.array([[1.2, 0.1], [-0.05, 0.9]])
SHEAR, BULK = 2.5, 0.3


def phi(law, i):
    if law == 0:
        return SHEAR * (i - 1) - BULK * i * (i * i - 1)
    return SHEAR * (1 - 1 / np.sqrt(i))


@pytest.fixture(scope="module")
def curves(oracle):
    ops, w = T.curve_operators(N), T.curve_weights(N)
    rest = oracle.curve_geometry(ops, w, T.curve_shape(N)["position"].reshape(-1), 1)
    cur = oracle.curve_geometry(ops, w, T.curve_shape(N, A=A, eps=0.05)["position"].reshape(-1), 1)
    return ops, w, rest, cur


def test_fourier_operators_reproduce_the_analytic_curve(oracle):
    exact = T.curve_shape(N, A=A, eps=0.05)
    ops, w = T.curve_operators(N), T.curve_weights(N)
    for first in (ops[0], None):
        g = oracle.curve_geometry([first] + ops[1:], w, exact["position"].reshape(-1), 1)
        for k in ("position", "tu", "tuu"):
            assert np.abs(g[k] - exact[k].reshape(-1)).max() <= 1e-11 * np.abs(exact[k]).max(), k
        t = exact["tu"]
        speed = np.sqrt((t * t).sum(axis=0))
        assert np.allclose(g["sigma"], w * speed, rtol=1e-13)
        assert np.allclose(g["normal"].reshape(2, -1), np.stack([t[1], -t[0]]) / speed, rtol=0, atol=1e-13)


@pytest.mark.parametrize("law", [0, 2])
def test_no_force_at_rest(oracle, curves, law):
    _, _, rest, _ = curves
    assert np.abs(oracle.curve_tension(law, SHEAR, BULK, rest, rest)).max() == 0.0


@pytest.mark.parametrize("law,tol", [(0, 1e-13), (2, 1e-9)])
def test_total_force_and_torque_vanish_on_a_closed_curve(oracle, curves, law, tol):
    _, _, rest, cur = curves
    F = oracle.curve_tension(law, SHEAR, BULK, rest, cur).reshape(2, -1)
    X = cur["position"].reshape(2, -1)
    scale = np.abs(F).sum()
    assert np.abs(F.sum(axis=1)).max() <= tol * scale
    assert abs((X[0] * F[1] - X[1] * F[0]).sum()) <= tol * scale


@pytest.mark.parametrize("law", [0, 2])
def test_dilated_circle_is_pulled_in_uniformly(oracle, curves, law):
    ops, w, rest, _ = curves
    lam = 1.3
    d = oracle.curve_geometry(ops, w, (lam * T.curve_shape(N)["position"]).reshape(-1), 1)
    F = oracle.curve_tension(law, SHEAR, BULK, rest, d).reshape(2, -1)
    X = d["position"].reshape(2, -1)
    r = np.sqrt((X * X).sum(axis=0))
    radial = (F * X).sum(axis=0) / r
    tangential = (X[0] * F[1] - X[1] * F[0]) / r
    expected = -w * lam * phi(law, lam * lam)
    assert np.abs(radial - expected).max() <= 1e-11 * np.abs(expected).max()
    assert np.abs(tangential).max() <= 1e-12 * np.abs(expected).max()


@pytest.mark.parametrize("law", [0, 2])
def test_curve_forces_rotate_with_the_curve(oracle, curves, law):
    _, _, rest, cur = curves
    c, s = np.cos(0.9), np.sin(0.9)
    Q = np.array([[c, -s], [s, c]])
    rot = {k: (Q @ cur[k].reshape(2, -1)).reshape(-1) for k in ("tu", "tuu")}
    f = oracle.curve_tension(law, SHEAR, BULK, rest, cur)
    fr = oracle.curve_tension(law, SHEAR, BULK, rest, rot)
    assert np.abs(fr - (Q @ f.reshape(2, -1)).reshape(-1)).max() <= 1e-12 * np.abs(f).max()


def test_curve_argument_checks(ibk):
    L = ibk.lib()
    h = ctypes.c_void_p()
    ops = (ctypes.c_void_p * 3)()
    assert L.ibk_curve_plan_create(0, 4, ops, None, ctypes.byref(h)) == 1
    assert L.ibk_curve_plan_create(4, 4, ops, ctypes.c_void_p(8), ctypes.byref(h)) == 1   # null derivatives
    s = ibk._Surface()
    assert L.ibk_curve_tension(1, 1.0, 1.0, 10, ctypes.byref(s), ctypes.byref(s), None, None) == 1   # no 1-D neo-Hookean
    assert L.ibk_curve_tension(0, 1.0, 1.0, 0, None, None, None, None) == 0
    assert L.ibk_curve_tension(2, 1.0, 1.0, 10, ctypes.byref(s), ctypes.byref(s), None, None) == 1
