"""Closed test surfaces for the membrane forces: tori with analytic tangents
and second derivatives, and exact Fourier differentiation operators on their
periodic (u, v) grid.

A torus has a regular periodic parameterisation, so sums over the trapezoid
grid are spectrally accurate: the total force and torque of a tension field
(the surface divergence of a symmetric in-plane stress) vanish on it to near
rounding, whatever the deformation.  Layout as the reference's shape
matrices: [component][shape][site], site index u fastest.
"""
import numpy as np


def grid(nu, nv):
    u = 2 * np.pi * np.arange(nu) / nu
    v = 2 * np.pi * np.arange(nv) / nv
    uu, vv = np.meshgrid(u, v, indexing="xy")      # (nv, nu): u fastest when flattened
    return uu.ravel(), vv.ravel()


def _rest(u, v, R, r):
    cu, su, cv, sv = np.cos(u), np.sin(u), np.cos(v), np.sin(v)
    rho = R + r * cv
    z = np.zeros_like(u)
    return {
        "position": np.stack([rho * cu, rho * su, r * sv]),
        "tu": np.stack([-rho * su, rho * cu, z]),
        "tv": np.stack([-r * sv * cu, -r * sv * su, r * cv]),
        "tuu": np.stack([-rho * cu, -rho * su, z]),
        "tuv": np.stack([r * sv * su, -r * sv * cu, z]),
        "tvv": np.stack([-r * cv * cu, -r * cv * su, -r * sv]),
    }


def _bump(u, v):
    """A smooth periodic displacement and its derivatives."""
    z = np.zeros_like(u)
    s2, c2 = np.sin(2 * u), np.cos(2 * u)
    suv, cuv = np.sin(u + v), np.cos(u + v)
    return {
        "position": np.stack([np.sin(v), c2, suv]),
        "tu": np.stack([z, -2 * s2, cuv]),
        "tv": np.stack([np.cos(v), z, cuv]),
        "tuu": np.stack([z, -4 * c2, -suv]),
        "tuv": np.stack([z, z, -suv]),
        "tvv": np.stack([-np.sin(v), z, -suv]),
    }


KEYS = ("position", "tu", "tv", "tuu", "tuv", "tvv")


def shape(nu, nv, R=1.0, r=0.4, A=None, eps=0.0):
    """Analytic geometry of A @ torus(R, r) + eps * bump: dict of (3, ns)
    arrays for the KEYS."""
    u, v = grid(nu, nv)
    g = _rest(u, v, R, r)
    A = np.eye(3) if A is None else np.asarray(A, dtype=np.float64)
    b = _bump(u, v)
    return {k: A @ g[k] + eps * b[k] for k in KEYS}


def pack(shapes, keys=KEYS):
    """Stack per-shape (3, ns) arrays into [component][shape][site] vectors."""
    return {k: np.stack([s[k] for s in shapes], axis=1).reshape(-1) for k in keys}


def weights(nu, nv):
    return np.full(nu * nv, (2 * np.pi / nu) * (2 * np.pi / nv))


def _d1(n):
    h = 2 * np.pi / n
    k = np.arange(n)
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            if i != j:
                D[i, j] = 0.5 * (-1.0) ** (i - j) / np.tan((i - j) * h / 2)
    return D


def _d2(n):
    h = 2 * np.pi / n
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            D[i, j] = (-np.pi ** 2 / (3 * h ** 2) - 1.0 / 6) if i == j else \
                -0.5 * (-1.0) ** (i - j) / np.sin((i - j) * h / 2) ** 2
    return D


def operators(nu, nv):
    """Fourier differentiation on the (u, v) grid (even nu, nv): evaluation
    (identity), d/du, d/dv, d2/du2, d2/dudv, d2/dv2 as dense (ns, ns) arrays;
    exact for trigonometric polynomials of degree below nu/2, nv/2."""
    Iu, Iv = np.eye(nu), np.eye(nv)
    Du, Dv, Duu, Dvv = _d1(nu), _d1(nv), _d2(nu), _d2(nv)
    return [np.kron(Iv, Iu), np.kron(Iv, Du), np.kron(Dv, Iu), np.kron(Iv, Duu), np.kron(Dv, Du), np.kron(Dvv, Iu)]


def totals(f, x, n):
    """Total force and torque of forces f at positions x ([component][site])."""
    F = f.reshape(3, n)
    X = x.reshape(3, n)
    return F.sum(axis=1), np.cross(X.T, F.T).sum(axis=0)


# ---- closed curves for the two-dimensional (curve) forces
def curve_shape(n, R=1.0, A=None, eps=0.0):
    """Analytic geometry of A @ circle(R) + eps * bump on n equispaced
    parameter values: dict of (2, n) arrays position, tu, tuu."""
    s = 2 * np.pi * np.arange(n) / n
    c, si = np.cos(s), np.sin(s)
    c3, s3 = np.cos(3 * s), np.sin(3 * s)
    g = {"position": np.stack([R * c, R * si]), "tu": np.stack([-R * si, R * c]),
         "tuu": np.stack([-R * c, -R * si])}
    b = {"position": np.stack([c3, s3 * c]),
         "tu": np.stack([-3 * s3, 3 * c3 * c - s3 * si]),
         "tuu": np.stack([-9 * c3, -9 * s3 * c - 3 * c3 * si - 3 * c3 * si - s3 * c])}
    A = np.eye(2) if A is None else np.asarray(A, dtype=np.float64)
    return {k: A @ g[k] + eps * b[k] for k in g}


def curve_weights(n):
    return np.full(n, 2 * np.pi / n)


def curve_operators(n):
    """Fourier evaluation (identity), d/ds and d2/ds2 on n equispaced points
    (even n): exact for trigonometric polynomials of degree below n/2."""
    return [np.eye(n), _d1(n), _d2(n)]
