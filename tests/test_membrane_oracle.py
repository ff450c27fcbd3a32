"""The membrane-force oracle (surface geometry, hyperelastic tension,
bending, viscous dissipation, tether and wall repulsion; include/bases/
geometry.h, include/forces/) against the mechanics it restates, on tori with
analytic geometry: zero force at rest, zero total force and torque on a
closed surface (the force is the surface divergence of a symmetric in-plane
tension), forces that rotate with the shape, a dissipation that vanishes
under rigid motion and whose power is -kappa/2 times the integral of
tr((g^-1 g')^2), and Fourier operators that reproduce the analytic
derivatives.  Plus the library's argument checks, which run before any
device work."""
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


def test_hookean_rest_state_is_a_uniform_tension(oracle, shapes):
    """The reference's Hookean law (hookean.h:19-30) has w1 = shear (1 -
    1/sqrt(I1)), not zero at I1 = 2: the rest shape carries the isotropic
    tension shear (1 - 1/sqrt(2)), whose force is normal to the surface."""
    rest, _ = shapes
    f = oracle.membrane_tension(2, SHEAR, BULK, rest, rest).reshape(3, -1)
    c = np.cross(rest["tu"].reshape(3, -1).T, rest["tv"].reshape(3, -1).T).T
    nrm = c / np.sqrt((c * c).sum(axis=0))
    tangential = f - (f * nrm).sum(axis=0) * nrm
    assert np.abs(f).max() > 0
    assert np.abs(tangential).max() <= 1e-10 * np.abs(f).max()


@pytest.mark.parametrize("law,tol", [(0, 1e-13), (1, 1e-7), (2, 1e-10)])
def test_total_force_and_torque_vanish_on_a_closed_surface(oracle, shapes, law, tol):
    rest, cur = shapes
    f = oracle.membrane_tension(law, SHEAR, BULK, rest, cur)
    F, M = T.totals(f, cur["position"], NU * NV)
    scale = np.abs(f).sum()
    assert np.abs(F).max() <= tol * scale
    assert np.abs(M).max() <= tol * scale


@pytest.mark.parametrize("law", [0, 1, 2])
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


# ---- viscous dissipation (include/forces/dissipation.h), tether, repelling
KAPPA = 0.7


def _velocity(phase):
    """A smooth velocity field on the (u, v) grid, [component][site]."""
    u, v = T.grid(NU, NV)
    return np.stack([np.sin(u + phase) * np.cos(v), np.cos(2 * u) + 0.3 * np.sin(v - phase),
                     np.sin(u - 2 * v)]).reshape(-1)


@pytest.fixture(scope="module")
def moving(oracle):
    ops = T.operators(NU, NV)
    x = T.shape(NU, NV, A=A, eps=0.05)["position"].reshape(-1)
    return ops, oracle.surface_geometry(ops, T.weights(NU, NV), x, 1)


def test_rigid_motion_dissipates_nothing(oracle, moving):
    ops, g = moving
    X = g["position"].reshape(3, -1)
    omega, a = np.array([0.3, -0.5, 0.8]), np.array([1.0, 2.0, -0.5])
    rigid = (a[:, None] + np.cross(omega, X.T).T).reshape(-1)
    f = oracle.membrane_dissipation(ops, KAPPA, _velocity(0.3), g, 1)
    fr = oracle.membrane_dissipation(ops, KAPPA, rigid, g, 1)
    assert np.abs(fr).max() <= 1e-12 * np.abs(f).max()


def test_dissipation_force_and_torque_balance(oracle, moving):
    ops, g = moving
    f = oracle.membrane_dissipation(ops, KAPPA, _velocity(0.3), g, 1)
    F, M = T.totals(f, g["position"], NU * NV)
    scale = np.abs(f).sum()
    # the product-rule expansion of the stress divergence is exact only to
    # the grid's accuracy (1e-7 here)
    assert np.abs(F).max() <= 1e-6 * scale and np.abs(M).max() <= 1e-6 * scale


def test_dissipated_power(oracle, moving):
    """sum f . u = -kappa/2 * integral of tr((g^-1 g')^2) dA <= 0, with g'_ij
    = t_i . u_j + u_i . t_j: the force is the divergence of the viscous stress
    kappa g^-1 g' g^-1."""
    ops, g = moving
    U = _velocity(0.3)
    f = oracle.membrane_dissipation(ops, KAPPA, U, g, 1)
    power = (f * U).sum()
    du = [(m @ U.reshape(3, -1).T) for m in ops[1:3]]
    t = [g["tu"].reshape(3, -1).T, g["tv"].reshape(3, -1).T]
    n = NU * NV
    G, Gd = np.zeros((n, 2, 2)), np.zeros((n, 2, 2))
    for i in range(2):
        for j in range(2):
            G[:, i, j] = (t[i] * t[j]).sum(axis=1)
            Gd[:, i, j] = (t[i] * du[j]).sum(axis=1) + (du[i] * t[j]).sum(axis=1)
    R = np.linalg.solve(G, Gd)
    expected = -0.5 * KAPPA * (g["sigma"] * np.einsum("nij,nji->n", R, R)).sum()
    assert power < 0
    assert abs(power - expected) <= 1e-5 * abs(expected)


def test_dissipation_is_linear_in_the_velocity(oracle, moving):
    ops, g = moving
    u1, u2 = _velocity(0.3), _velocity(1.1)
    f1 = oracle.membrane_dissipation(ops, KAPPA, u1, g, 1)
    f2 = oracle.membrane_dissipation(ops, KAPPA, u2, g, 1)
    assert np.array_equal(oracle.membrane_dissipation(ops, KAPPA, 2 * u1, g, 1), 2 * f1)
    f12 = oracle.membrane_dissipation(ops, KAPPA, u1 + u2, g, 1)
    assert np.abs(f12 - f1 - f2).max() <= 1e-13 * np.abs(f12).max()


def test_tether_and_repelling_formulas(oracle, moving):
    _, g = moving
    rng = np.random.default_rng(11)
    x0 = g["position"] + 0.01 * rng.normal(size=g["position"].size)
    assert np.array_equal(oracle.membrane_tether(3.0, x0, g["position"]), 3.0 * (x0 - g["position"]))
    # a wall at y = 1.2 with range 0.1: samples within 0.2 of it are pushed away (down)
    f = oracle.membrane_repelling(2.0, 1.2, 0.1, g["position"], g["sigma"]).reshape(3, -1)
    y = g["position"].reshape(3, -1)[1]
    r = np.abs(1.2 - y) / 0.1
    inside = r < 2
    fy = np.where(inside, -np.log(np.where(inside, r, 1.0) / 2) * np.exp(-4 / (4 - np.where(inside, r, 0.0) ** 2)), 0)
    assert inside.any() and (~inside).any()
    assert np.abs(f[1] - (-2.0 * fy * g["sigma"])).max() <= 1e-15 * np.abs(f[1]).max()
    assert (f[1][inside] < 0).all() and (f[1][~inside] == 0).all() and (f[0] == 0).all() and (f[2] == 0).all()


def test_more_membrane_argument_checks(ibk):
    L = ibk.lib()
    s = ibk._Surface()
    assert L.ibk_membrane_dissipation(None, 1.0, 1, None, None, None, None) == 1
    assert L.ibk_membrane_tether(1.0, 0, None, None, None, None) == 0
    assert L.ibk_membrane_tether(1.0, 5, ctypes.byref(s), ctypes.byref(s), None, None) == 1
    assert L.ibk_membrane_repelling(1.0, 1.6, 0.025, 0, None, None, None) == 0
    assert L.ibk_membrane_repelling(1.0, 1.6, 0.025, 5, ctypes.byref(s), None, None) == 1
    assert L.ibk_membrane_tension(2, 1.0, 1.0, 0, None, None, None, None) == 0
