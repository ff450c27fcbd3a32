"""The membrane-force oracle (surface geometry and hyperelastic tension,
include/bases/geometry.h, include/forces/tension.h) against the mechanics it
restates, on tori with analytic geometry: zero force at rest, zero total
force and torque on a closed surface (the force is the surface divergence
of a symmetric in-plane tension), forces that rotate with the shape, and
Fourier operators that reproduce the analytic derivatives.  Plus the
library's argument checks, which run before any device work."""
import ctypes

import numpy as np
import pytest

import torus as T

NU, NV = 48, 24
A = np.array([[1.3, 0.2, 0.0], [0.0, 0.8, 0.1], [0.05, 0.0, 1.1]])
SHEAR, BULK = 2.5, 25.0


def analytic(s, w):
    g = {k: s[k].reshape(-1) for k in T.KEYS}
    c = np.cross(s["tu"].T, s["tv"].T).T
    g["sigma"] = w * np.sqrt((c * c).sum(axis=0))
    return g


@pytest.fixture(scope="module")
def shapes():
    w = T.weights(NU, NV)
    return analytic(T.shape(NU, NV), w), analytic(T.shape(NU, NV, A=A, eps=0.05), w)


@pytest.mark.parametrize("law", [0, 1])
def test_zero_force_at_rest(oracle, shapes, law):
    rest, cur = shapes
    f_rest = oracle.membrane_tension(law, SHEAR, BULK, rest, rest)
    f = oracle.membrane_tension(law, SHEAR, BULK, rest, cur)
    assert np.abs(f_rest).max() <= 1e-14 * np.abs(f).max()


@pytest.mark.parametrize("law,tol", [(0, 1e-13), (1, 1e-7)])
def test_total_force_and_torque_vanish_on_a_closed_surface(oracle, shapes, law, tol):
    rest, cur = shapes
    f = oracle.membrane_tension(law, SHEAR, BULK, rest, cur)
    F, M = T.totals(f, cur["position"], NU * NV)
    scale = np.abs(f).sum()
    assert np.abs(F).max() <= tol * scale
    assert np.abs(M).max() <= tol * scale


@pytest.mark.parametrize("law", [0, 1])
def test_forces_rotate_with_the_shape(oracle, shapes, law):
    rest, cur = shapes
    c, s = np.cos(0.7), np.sin(0.7)
    Q = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]]) @ np.array([[1.0, 0, 0], [0, c, s], [0, -s, c]])
    rot = {k: (Q @ cur[k].reshape(3, -1)).reshape(-1) for k in T.KEYS}
    rot["sigma"] = cur["sigma"]
    f = oracle.membrane_tension(law, SHEAR, BULK, rest, cur)
    fr = oracle.membrane_tension(law, SHEAR, BULK, rest, rot)
    assert np.abs(fr - (Q @ f.reshape(3, -1)).reshape(-1)).max() <= 1e-12 * np.abs(f).max()


def test_fourier_operators_reproduce_the_analytic_geometry(oracle, shapes):
    _, cur = shapes
    w = T.weights(NU, NV)
    ops = T.operators(NU, NV)
    for first in (ops[0], None):          # evaluation matrix, or samples = data sites
        g = oracle.surface_geometry([first] + ops[1:], w, cur["position"], 1)
        for k in ("position", "tu", "tv", "tuu", "tuv", "tvv", "sigma"):
            assert np.abs(g[k] - cur[k]).max() <= 1e-10 * np.abs(cur[k]).max(), k
        n = g["normal"].reshape(3, -1)
        assert np.abs((n * n).sum(axis=0) - 1).max() < 1e-14


def test_membrane_argument_checks(ibk):
    """Rejected before any device work (status 1: invalid argument)."""
    L = ibk.lib()
    h = ctypes.c_void_p()
    ops = (ctypes.c_void_p * 6)()
    assert L.ibk_surface_plan_create(0, 4, ops, None, ctypes.byref(h)) == 1
    assert L.ibk_surface_plan_create(4, 4, None, None, ctypes.byref(h)) == 1
    assert L.ibk_surface_plan_destroy(None) == 0
    assert L.ibk_surface_geometry(None, 1, None, None, None) == 1
    s = ibk._Surface()
    assert L.ibk_membrane_tension(7, 1.0, 1.0, 10, ctypes.byref(s), ctypes.byref(s), None, None) == \
        1
    assert L.ibk_membrane_tension(0, 1.0, 1.0, 0, None, None, None, None) == 0
    assert L.ibk_membrane_tension(0, 1.0, 1.0, 10, ctypes.byref(s), ctypes.byref(s), None, None) == \
        1


def _bending(oracle, nu, nv, R, r, A=None, eps=0.0, preferred=False):
    w = T.weights(nu, nv)
    ops = T.operators(nu, nv)
    dops = [None] + ops[1:]
    x = T.shape(nu, nv, R=R, r=r, A=A, eps=eps)["position"].reshape(-1)
    x0 = T.shape(nu, nv, R=R, r=r)["position"].reshape(-1)
    g, g0 = oracle.surface_geometry(dops, w, x, 1), oracle.surface_geometry(dops, w, x0, 1)
    return oracle.membrane_bending(dops, w, ops, 1.0, preferred, x0, x, g0, g, 1), g


def test_no_bending_force_on_the_clifford_torus(oracle):
    """R/r = sqrt(2) solves the Willmore shape equation Lap H + 2H(H^2 - K) = 0."""
    f_clifford, _ = _bending(oracle, 64, 32, np.sqrt(2.0), 1.0)
    f_other, _ = _bending(oracle, 64, 32, 2.5, 1.0)
    assert np.abs(f_clifford).max() <= 1e-3 * np.abs(f_other).max()


def test_bending_at_the_preferred_shape_is_zero(oracle):
    f, _ = _bending(oracle, 48, 24, 2.5, 1.0, preferred=True)
    assert np.abs(f).max() == 0.0


def test_bending_force_and_torque_balance(oracle):
    f, g = _bending(oracle, 48, 24, 2.0, 0.7, A=np.diag([1.1, 0.9, 1.05]), eps=0.03)
    F, M = T.totals(f, g["position"], 48 * 24)
    scale = np.abs(f).sum()
    assert np.abs(F).max() <= 1e-10 * scale and np.abs(M).max() <= 1e-10 * scale
