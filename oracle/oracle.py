"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this
module, and only as the checker / CPU baseline.  It wraps

* ``libibk_oracle.so`` -- the plain-C restatement of sonwell/ib.cu's
  spread / interpolate (``ibk_oracle.c``), always buildable with gcc;
* ``_ref/libibref.so`` -- the reference's own host headers compiled from the
  reference tree (``ref_bridge.cc``); present only where that tree exists.

Array conventions follow the reference: positions and forces are ``dims x n``
column blocks (``x[d*n + p]``, include/ib/novel.h:127-128), grid components
are flat x-fastest vectors (include/ib/indexing.h:27-33).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libibk_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libibref.so")
REF_FORCES_PATH = os.path.join(HERE, "_ref", "libibref_forces.so")
REF_SOLVER_PATH = os.path.join(HERE, "_ref", "libibref_solver.so")

PERIODIC, SOLID = 0, 1
TAG_MAC, TAG_CENTERED = 0, 1
BSPLINE, PESKIN, ROMA, COSINE, HAT = 0, 1, 2, 3, 4
DELTA_NAMES = {"bspline": BSPLINE, "peskin": PESKIN, "roma": ROMA, "cosine": COSINE, "hat": HAT}

_lock = threading.Lock()
_lib = None
_ref = None
_ref_forces = None
_ref_solver = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class Geom(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_int),
        ("delta_kind", ctypes.c_int),
        ("delta_order", ctypes.c_int),
        ("meshwidths", ctypes.c_int),
        ("values", ctypes.c_int),
        ("pattern", ctypes.c_int),
        ("per_sweep", ctypes.c_int),
        ("sweeps", ctypes.c_int),
        ("unit", ctypes.c_double),
        ("resolution", ctypes.c_double),
        ("length", ctypes.c_double * 3),
        ("solid", ctypes.c_int * 3),
        ("cells", (ctypes.c_int * 3) * 3),
        ("points", (ctypes.c_int * 3) * 3),
        ("shift", (ctypes.c_double * 3) * 3),
        ("size", ctypes.c_longlong * 3),
    ]

    def comp_points(self, c):
        return [self.points[c][d] for d in range(self.dims)]

    def comp_shape(self, c):
        """numpy shape of component c (reversed: slowest dimension first)."""
        return tuple(reversed(self.comp_points(c)))


def build(force: bool = False) -> None:
    """Compile the oracle (and, where the reference tree exists, its bridge)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE, "libibk_oracle.so"], check=True)


def reference_root():
    """Location of the sonwell/ib.cu tree: the IBK_REFERENCE_ROOT environment
    variable, or None (no default location)."""
    return os.environ.get("IBK_REFERENCE_ROOT") or None


def build_ref(ref_root=None) -> bool:
    """Compile the bridge from the reference tree at ref_root (default:
    reference_root()); without a tree, report whether a bridge is built."""
    ref_root = ref_root or reference_root()
    if not ref_root or not os.path.isdir(os.path.join(ref_root, "include", "ib")):
        return os.path.exists(REF_PATH)
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_root}"], check=True)
    return os.path.exists(REF_PATH)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(LIB_PATH)
            L.ibo_geometry.argtypes = [ctypes.c_int, _dp, _ip, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.POINTER(Geom)]
            L.ibo_geometry.restype = ctypes.c_int
            L.ibo_phi.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
            L.ibo_phi.restype = ctypes.c_double
            L.ibo_sort_keys.argtypes = [ctypes.POINTER(Geom), ctypes.c_int, ctypes.c_int, _dp, _ip]
            L.ibo_stencil.argtypes = [ctypes.POINTER(Geom), ctypes.c_int, ctypes.c_int, _dp,
                                      _ip, _dp, _dp, _ip, _ip]
            L.ibo_spread.argtypes = [ctypes.POINTER(Geom), ctypes.c_int, _dp, _dp,
                                     ctypes.POINTER(_dp), ctypes.POINTER(_dp)]
            L.ibo_spread.restype = ctypes.c_int
            L.ibo_spread_mt.argtypes = [ctypes.POINTER(Geom), ctypes.c_int, _dp, _dp,
                                        ctypes.POINTER(_dp), ctypes.c_int]
            L.ibo_spread_mt.restype = ctypes.c_int
            L.ibo_interpolate.argtypes = [ctypes.POINTER(Geom), ctypes.c_int, _dp,
                                          ctypes.POINTER(_dp), _dp, _dp]
            L.ibo_interpolate_mt.argtypes = [ctypes.POINTER(Geom), ctypes.c_int, _dp,
                                             ctypes.POINTER(_dp), _dp, ctypes.c_int]
            L.ibo_max_threads.restype = ctypes.c_int
            L.ibo_surface_geometry.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_dp),
                                               _dp, _dp, ctypes.POINTER(_dp)]
            L.ibo_membrane_tension.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                               ctypes.POINTER(_dp), ctypes.POINTER(_dp), _dp]
            L.ibo_wall_weights.argtypes = [_dp, ctypes.c_double, ctypes.c_double, _dp]
            L.ibo_diffusion_apply.argtypes = [ctypes.c_int, _ip, _ip, _dp, ctypes.c_double, _dp, ctypes.c_double,
                                              ctypes.c_int, _dp, _dp]
            L.ibo_diffusion_step.argtypes = [ctypes.c_int, _ip, _ip, _dp, ctypes.c_double, _dp, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_int, _dp, _dp, _dp, _dp]
            L.ibo_diffusion_step.restype = ctypes.c_int
            L.ibo_gershgorin.argtypes = [ctypes.c_int, _ip, _ip, _dp, ctypes.c_double, _dp, ctypes.c_double, _dp]
            L.ibo_chebyshev_weights.argtypes = [ctypes.c_double, ctypes.c_double, _dp]
            L.ibo_membrane_bending.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_dp), _dp,
                                               ctypes.POINTER(_dp), ctypes.c_double, ctypes.c_int, _dp, _dp,
                                               ctypes.POINTER(_dp), ctypes.POINTER(_dp), _dp]
            L.ibo_membrane_dissipation.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_dp),
                                                   ctypes.c_double, _dp, ctypes.POINTER(_dp), _dp]
            L.ibo_curve_geometry.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_dp),
                                             _dp, _dp, ctypes.POINTER(_dp)]
            L.ibo_curve_tension.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                            ctypes.POINTER(_dp), ctypes.POINTER(_dp), _dp]
            L.ibo_membrane_tether.argtypes = [ctypes.c_double, ctypes.c_int, _dp, _dp, _dp]
            L.ibo_membrane_repelling.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                 _dp, _dp, _dp]
            _lib = L
    return _lib


def ref_forces():
    """The reference's own membrane-force code built on host shims
    (ref_forces.cc), or None where it cannot be built."""
    global _ref_forces
    if ref() is None or not os.path.exists(REF_FORCES_PATH):
        return None
    with _lock:
        if _ref_forces is None:
            R = ctypes.CDLL(REF_FORCES_PATH)
            R.ibref_membrane_tension.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                 ctypes.POINTER(_dp), ctypes.POINTER(_dp), _dp]
            R.ibref_membrane_bending.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_dp),
                                                 ctypes.c_double, ctypes.c_int, ctypes.POINTER(_dp),
                                                 ctypes.POINTER(_dp), ctypes.POINTER(_dp), ctypes.POINTER(_dp), _dp]
            R.ibref_membrane_dissipation.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_dp),
                                                     ctypes.c_double, _dp, ctypes.POINTER(_dp), _dp]
            R.ibref_membrane_tether.argtypes = [ctypes.c_double, ctypes.c_int, _dp, _dp, _dp]
            R.ibref_curve_tension.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                              ctypes.POINTER(_dp), ctypes.POINTER(_dp), _dp]
            _ref_forces = R
    return _ref_forces


def ref():
    """The reference-built bridge, or None where it cannot be built."""
    global _ref
    with _lock:
        if _ref is None:
            if not os.path.exists(REF_PATH):
                try:
                    build_ref()
                except Exception:
                    return None
            if not os.path.exists(REF_PATH):
                return None
            R = ctypes.CDLL(REF_PATH)
            R.ibref_stencil.argtypes = [ctypes.c_int, _dp, _ip, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        _dp, _ip, _ip, _dp, _dp, _ip, _ip, _dp]
            R.ibref_stencil.restype = ctypes.c_int
            R.ibref_phi.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
            R.ibref_phi.restype = ctypes.c_double
            R.ibref_domain_unit.argtypes = [ctypes.c_int, _dp]
            R.ibref_wall_weights.argtypes = [ctypes.c_double] * 7 + [_dp]
            R.ibref_domain_unit.restype = ctypes.c_double
            _ref = R
    return _ref


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def geometry(dims, length, solid, tag=TAG_MAC, refinement=16, delta="bspline", order=3) -> Geom:
    kind = DELTA_NAMES[delta] if isinstance(delta, str) else int(delta)
    L = np.zeros(3, np.float64)
    L[:dims] = length
    S = np.zeros(3, np.int32)
    S[:dims] = solid
    g = Geom()
    rc = lib().ibo_geometry(dims, _d(L), _i(S), tag, refinement, kind, order, ctypes.byref(g))
    if rc != 0:
        raise ValueError("unsupported geometry / delta")
    g._length = L
    g._solid = S
    g._tag = tag
    g._refinement = refinement
    return g


def _as_points(x, dims):
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    assert x.size % dims == 0
    return x, x.size // dims


def sort_keys(g: Geom, comp: int, x) -> np.ndarray:
    x, n = _as_points(x, g.dims)
    keys = np.empty(n, np.int32)
    lib().ibo_sort_keys(ctypes.byref(g), comp, n, _d(x), _i(keys))
    return keys


def stencil(g: Geom, comp: int, x):
    """(base[n,dims], delta[n,dims], weights[n,V], spread_idx[n,V], interp_idx[n,V])"""
    x, n = _as_points(x, g.dims)
    V = g.values
    base = np.empty((n, g.dims), np.int32)
    delta = np.empty((n, g.dims), np.float64)
    w = np.empty((n, V), np.float64)
    sidx = np.empty((n, V), np.int32)
    iidx = np.empty((n, V), np.int32)
    lib().ibo_stencil(ctypes.byref(g), comp, n, _d(x), _i(base), _d(delta), _d(w), _i(sidx), _i(iidx))
    return base, delta, w, sidx, iidx


def _ptr_array(arrs):
    P = (_dp * 3)()
    for c, a in enumerate(arrs):
        P[c] = _d(a)
    return P


def spread(g: Geom, x, f, fe=None, with_abs=False, threads=1):
    """Reference spread.  Returns list of flat component arrays (and abs sums)."""
    x, n = _as_points(x, g.dims)
    f = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
    if fe is None:
        fe = [np.zeros(int(g.size[c]), np.float64) for c in range(g.dims)]
    absum = [np.zeros(int(g.size[c]), np.float64) for c in range(g.dims)] if with_abs else None
    if threads == 1:
        rc = lib().ibo_spread(ctypes.byref(g), n, _d(x), _d(f), _ptr_array(fe),
                              _ptr_array(absum) if absum else None)
    else:
        rc = lib().ibo_spread_mt(ctypes.byref(g), n, _d(x), _d(f), _ptr_array(fe), threads)
    if rc != 0:
        raise MemoryError("oracle spread failed")
    return (fe, absum) if with_abs else fe


def interpolate(g: Geom, x, ue, with_abs=False, threads=1):
    x, n = _as_points(x, g.dims)
    ue = [np.ascontiguousarray(u, dtype=np.float64).reshape(-1) for u in ue]
    ul = np.zeros(g.dims * n, np.float64)
    ua = np.zeros(g.dims * n, np.float64) if with_abs else None
    if threads == 1:
        lib().ibo_interpolate(ctypes.byref(g), n, _d(x), _ptr_array(ue), _d(ul), _d(ua))
    else:
        lib().ibo_interpolate_mt(ctypes.byref(g), n, _d(x), _ptr_array(ue), _d(ul), threads)
    return (ul, ua) if with_abs else ul


def max_threads() -> int:
    return int(lib().ibo_max_threads())


SURFACE_FIELDS = ("position", "tu", "tv", "tuu", "tuv", "tvv", "normal", "sigma")


def surface_geometry(ops, weights, x, nc):
    """Surface geometry of nc shapes (include/bases/geometry.h:30-49, 95-119):
    ops = six (ns, nd) arrays (ops[0] None: samples are the data sites),
    weights (ns,), x 3*nd*nc positions [component][shape][site]; returns a
    dict of the SURFACE_FIELDS arrays."""
    weights = np.ascontiguousarray(weights, dtype=np.float64)
    ns = weights.size
    cm = [None if o is None else np.asfortranarray(o, dtype=np.float64) for o in ops]   # column-major
    x = np.ascontiguousarray(x, dtype=np.float64)
    m = ns * nc
    out = {k: np.zeros(m if k == "sigma" else 3 * m) for k in SURFACE_FIELDS}
    opp = (_dp * 6)(*[None if o is None else o.ctypes.data_as(_dp) for o in cm])
    outp = (_dp * 8)(*[_d(out[k]) for k in SURFACE_FIELDS])
    nd = cm[1].shape[1]
    lib().ibo_surface_geometry(ns, nd, nc, opp, _d(weights), _d(x), outp)
    return out


def membrane_tension(law, shear, bulk, rest, cur):
    """Tension force at every sample (include/forces/tension.h:71-112;
    law 0 Skalak, 1 neo-Hookean, 2 Hookean) from rest and current geometry
    dicts."""
    keep = [np.ascontiguousarray(rest[k], dtype=np.float64) for k in ("tu", "tv", "tuu", "tuv", "tvv", "sigma")]
    keep += [np.ascontiguousarray(cur[k], dtype=np.float64) for k in ("tu", "tv", "tuu", "tuv", "tvv")]
    n = keep[5].size
    f = np.zeros(3 * n)
    rp = (_dp * 6)(*[_d(a) for a in keep[:6]])
    cp = (_dp * 5)(*[_d(a) for a in keep[6:]])
    lib().ibo_membrane_tension(int(law), float(shear), float(bulk), n, rp, cp, _d(f))
    return f


def membrane_bending(data_ops, data_weights, sample_ops, modulus, preferred, x_rest, x_cur, rest, cur, nc):
    """Bending force at every sample (include/forces/bending.h:145-229):
    data_ops / sample_ops as for surface_geometry (the shape family's
    operators at its data sites and at its samples), rest / cur sample
    geometry dicts, positions 3*nd*nc; returns 3*ns*nc forces."""
    cmd = [None if o is None else np.asfortranarray(o, dtype=np.float64) for o in data_ops]
    cms = [None if o is None else np.asfortranarray(o, dtype=np.float64) for o in sample_ops]
    dw = np.ascontiguousarray(data_weights, dtype=np.float64)
    ns, nd = cms[1].shape
    keys = ("tu", "tv", "tuu", "tuv", "tvv", "normal")
    r = [np.ascontiguousarray(rest[k], dtype=np.float64) for k in keys]
    c = [np.ascontiguousarray(cur[k], dtype=np.float64) for k in keys + ("sigma",)]
    xr = np.ascontiguousarray(x_rest, dtype=np.float64)
    xc = np.ascontiguousarray(x_cur, dtype=np.float64)
    f = np.zeros(3 * ns * nc)
    dp = (_dp * 6)(*[None if o is None else o.ctypes.data_as(_dp) for o in cmd])
    sp = (_dp * 6)(*[None if o is None else o.ctypes.data_as(_dp) for o in cms])
    lib().ibo_membrane_bending(ns, nd, nc, dp, _d(dw), sp, float(modulus), int(bool(preferred)), _d(xr), _d(xc),
                               (_dp * 6)(*[_d(a) for a in r]), (_dp * 7)(*[_d(a) for a in c]), _d(f))
    return f


def membrane_dissipation(sample_ops, modulus, u, cur, nc):
    """Viscous dissipation at every sample (include/forces/dissipation.h:
    216-265): sample_ops as for surface_geometry, u the data-site velocity
    (3*nd*nc), cur the current sample geometry dict; returns 3*ns*nc forces."""
    cms = [None if o is None else np.asfortranarray(o, dtype=np.float64) for o in sample_ops]
    ns, nd = cms[1].shape
    c = [np.ascontiguousarray(cur[k], dtype=np.float64) for k in ("tu", "tv", "tuu", "tuv", "tvv", "sigma")]
    uu = np.ascontiguousarray(u, dtype=np.float64)
    f = np.zeros(3 * ns * nc)
    sp = (_dp * 6)(*[None if o is None else o.ctypes.data_as(_dp) for o in cms])
    lib().ibo_membrane_dissipation(ns, nd, nc, sp, float(modulus), _d(uu), (_dp * 6)(*[_d(a) for a in c]), _d(f))
    return f


CURVE_FIELDS = ("position", "tu", "tuu", "normal", "sigma")


def curve_geometry(ops, weights, x, nc):
    """Geometry of nc closed curves in a two-dimensional run
    (include/bases/geometry.h:74-124 with one tangent): ops = three (ns, nd)
    arrays (evaluation or None, d/ds, d2/ds2), x 2*nd*nc positions; returns
    a dict of the CURVE_FIELDS arrays."""
    weights = np.ascontiguousarray(weights, dtype=np.float64)
    ns = weights.size
    cm = [None if o is None else np.asfortranarray(o, dtype=np.float64) for o in ops]
    x = np.ascontiguousarray(x, dtype=np.float64)
    m = ns * nc
    out = {k: np.zeros(m if k == "sigma" else 2 * m) for k in CURVE_FIELDS}
    opp = (_dp * 3)(*[None if o is None else o.ctypes.data_as(_dp) for o in cm])
    outp = (_dp * 5)(*[_d(out[k]) for k in CURVE_FIELDS])
    lib().ibo_curve_geometry(ns, cm[1].shape[1], nc, opp, _d(weights), _d(x), outp)
    return out


def curve_tension(law, shear, bulk, rest, cur):
    """One-dimensional tension (include/forces/tension.h:160-200; law 0
    skalak1d, 2 hookean1d) from rest and current curve geometry dicts."""
    keep = [np.ascontiguousarray(rest[k], dtype=np.float64) for k in ("tu", "tuu", "sigma")]
    keep += [np.ascontiguousarray(cur[k], dtype=np.float64) for k in ("tu", "tuu")]
    n = keep[2].size
    f = np.zeros(2 * n)
    lib().ibo_curve_tension(int(law), float(shear), float(bulk), n, (_dp * 3)(*[_d(a) for a in keep[:3]]),
                            (_dp * 2)(*[_d(a) for a in keep[3:]]), _d(f))
    return f


def membrane_tether(modulus, x_rest, x_cur):
    """Tether force modulus (x_rest - x_cur) (include/forces/tether.h:14-22)."""
    xr = np.ascontiguousarray(x_rest, dtype=np.float64)
    xc = np.ascontiguousarray(x_cur, dtype=np.float64)
    f = np.zeros(xr.size)
    lib().ibo_membrane_tether(float(modulus), xr.size // 3, _d(xr), _d(xc), _d(f))
    return f


def membrane_repelling(modulus, height, range_, x, sigma):
    """Wall repulsion at every sample (include/forces/repelling.h:15-45)."""
    xx = np.ascontiguousarray(x, dtype=np.float64)
    s = np.ascontiguousarray(sigma, dtype=np.float64)
    f = np.zeros(xx.size)
    lib().ibo_membrane_repelling(float(modulus), float(height), float(range_), s.size, _d(xx), _d(s), _d(f))
    return f


def ref_stencil(g: Geom, comp: int, x):
    """Same outputs as :func:`stencil`, computed by the reference's headers,
    plus the geometry vector (unit, resolution, cells/points/shift per dim)."""
    R = ref()
    if R is None:
        return None
    x, n = _as_points(x, g.dims)
    V = g.values
    keys = np.empty(n, np.int32)
    base = np.empty((n, g.dims), np.int32)
    delta = np.empty((n, g.dims), np.float64)
    w = np.empty((n, V), np.float64)
    sidx = np.empty((n, V), np.int32)
    iidx = np.empty((n, V), np.int32)
    geo = np.zeros(2 + 3 * g.dims, np.float64)
    rc = R.ibref_stencil(g.dims, _d(g._length), _i(g._solid), g._tag, g._refinement,
                         g.delta_kind, g.delta_order, comp, n, _d(x), _i(keys), _i(base),
                         _d(delta), _d(w), _i(sidx), _i(iidx), _d(geo))
    if rc != 0:
        raise ValueError("reference bridge does not cover this configuration")
    return keys, base, delta, w, sidx, iidx, geo


class FluidGrid:
    """One component grid for the diffusion oracle: points, periodicity and
    shift per axis (from a Geom), the resolution, and the wall conditions
    robin[axis][side] = (a, b)."""

    def __init__(self, g, comp, robin):
        self.dims = g.dims
        self.points = np.array(g.comp_points(comp) + [1] * (3 - g.dims), dtype=np.int32)
        self.periodic = np.array([0 if g.solid[d] else 1 for d in range(g.dims)] + [1] * (3 - g.dims), dtype=np.int32)
        self.shift = np.array([g.shift[comp][d] for d in range(g.dims)] + [0.0] * (3 - g.dims))
        self.res = float(g.resolution)
        self.robin = np.ascontiguousarray(np.asarray(robin, dtype=np.float64).reshape(3, 2, 2))
        self.size = int(np.prod(self.points))


def wall_weights(p, h, s):
    """{interior, laplacian, boundary} ghost-point weights of one wall
    (include/fd/discretization.h:47-80)."""
    out = np.zeros(3)
    lib().ibo_wall_weights(_d(np.ascontiguousarray(p, dtype=np.float64)), float(h), float(s), _d(out))
    return out


def diffusion_apply(fg: FluidGrid, op, u, lam=0.0):
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(fg.size)
    lib().ibo_diffusion_apply(fg.dims, _i(fg.points), _i(fg.periodic), _d(fg.shift), fg.res, _d(fg.robin),
                              float(lam), int(op), _d(u), _d(out))
    return out


CHEBYSHEV, JACOBI = 0, 1


def diffusion_step(fg: FluidGrid, timestep, mu, tolerance, max_iterations, gamma, u, rhs, f, precond=CHEBYSHEV):
    """out = u + (I~ - lambda L)^-1 (k I~ f + k mu (L u + rhs)) and the
    iteration count (include/ins/diffusion.h:47-56), preconditioned as the
    reference does (CHEBYSHEV, include/solvers/chebpcg.h) or by JACOBI."""
    u, rhs, f = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, rhs, f))
    out = np.zeros(fg.size)
    it = lib().ibo_diffusion_step(fg.dims, _i(fg.points), _i(fg.periodic), _d(fg.shift), fg.res, _d(fg.robin),
                                  float(timestep), float(mu), float(tolerance), int(max_iterations), float(gamma),
                                  int(precond), _d(u), _d(rhs), _d(f), _d(out))
    return out, it


def gershgorin(fg: FluidGrid, lam):
    """Gershgorin interval (lower, upper) of I~ - lam L (include/algo/gershgorin.h)."""
    out = np.zeros(2)
    lib().ibo_gershgorin(fg.dims, _i(fg.points), _i(fg.periodic), _d(fg.shift), fg.res, _d(fg.robin), float(lam),
                         _d(out))
    return out


def chebyshev_weights(a, b):
    """The four weights of impl::chebw<4>(a, b) (include/algo/chebyshev.h)."""
    out = np.zeros(4)
    lib().ibo_chebyshev_weights(float(a), float(b), _d(out))
    return out


def ref_wall_weights(length, resolution, shift, lower, upper):
    """The reference's own wall weights (bridge): {interior, laplacian,
    boundary} of the lower and of the upper wall."""
    out = np.zeros(6)
    ref().ibref_wall_weights(float(length), float(resolution), float(shift), float(lower[0]), float(lower[1]),
                             float(upper[0]), float(upper[1]), _d(out))
    return out[:3], out[3:]



# ---- the reference's own membrane forces (ref_forces.cc), for pinning the restatement
_KEYS5 = ("tu", "tv", "tuu", "tuv", "tvv")


def _parr(arrays):
    keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in arrays]
    return keep, (_dp * len(keep))(*[None if a is None else _d(a) for a in keep])


def ref_membrane_tension(law, shear, bulk, rest, cur):
    R = ref_forces()
    kr, rp = _parr([rest[k] for k in _KEYS5] + [rest["sigma"]])
    kc, cp = _parr([cur[k] for k in _KEYS5])
    n = kr[5].size
    f = np.zeros(3 * n)
    R.ibref_membrane_tension(int(law), float(shear), float(bulk), n, rp, cp, _d(f))
    return f


def ref_membrane_bending(sample_ops, modulus, preferred, data_rest, data_cur, rest, cur, nc):
    """data_rest / data_cur: the data-site geometry dicts (tu .. tvv, normal,
    sigma) of the rest and current shapes; rest / cur: the sample ones."""
    R = ref_forces()
    cms = [None if o is None else np.asfortranarray(o, dtype=np.float64) for o in sample_ops]
    ns, nd = cms[1].shape
    keys = _KEYS5 + ("normal", "sigma")
    k1, a1 = _parr([data_rest[k] for k in keys])
    k2, a2 = _parr([data_cur[k] for k in keys])
    k3, a3 = _parr([rest[k] for k in keys])
    k4, a4 = _parr([cur[k] for k in keys])
    sp = (_dp * 6)(*[None if o is None else o.ctypes.data_as(_dp) for o in cms])
    f = np.zeros(3 * ns * nc)
    R.ibref_membrane_bending(ns, nd, nc, sp, float(modulus), int(bool(preferred)), a1, a2, a3, a4, _d(f))
    return f


def ref_membrane_dissipation(sample_ops, modulus, u, cur, nc):
    R = ref_forces()
    cms = [None if o is None else np.asfortranarray(o, dtype=np.float64) for o in sample_ops]
    ns, nd = cms[1].shape
    kc, cp = _parr([cur[k] for k in _KEYS5] + [cur["sigma"]])
    uu = np.ascontiguousarray(u, dtype=np.float64)
    sp = (_dp * 6)(*[None if o is None else o.ctypes.data_as(_dp) for o in cms])
    f = np.zeros(3 * ns * nc)
    R.ibref_membrane_dissipation(ns, nd, nc, sp, float(modulus), _d(uu), cp, _d(f))
    return f


def ref_membrane_tether(modulus, x_rest, x_cur):
    R = ref_forces()
    xr = np.ascontiguousarray(x_rest, dtype=np.float64)
    xc = np.ascontiguousarray(x_cur, dtype=np.float64)
    f = np.zeros(xr.size)
    R.ibref_membrane_tether(float(modulus), xr.size // 3, _d(xr), _d(xc), _d(f))
    return f


def ref_curve_tension(law, shear, bulk, rest, cur):
    R = ref_forces()
    kr, rp = _parr([rest["tu"], rest["tuu"], rest["sigma"]])
    kc, cp = _parr([cur["tu"], cur["tuu"]])
    n = kr[2].size
    f = np.zeros(2 * n)
    R.ibref_curve_tension(int(law), float(shear), float(bulk), n, rp, cp, _d(f))
    return f


# ---- the reference's own solver loop (ref_solver.cc), for pinning the diffusion solve
_APPLY = ctypes.CFUNCTYPE(None, _dp, _dp, ctypes.c_void_p)


def ref_solver():
    """solvers::pcg and algo::chebyshev built on host shims, or None."""
    global _ref_solver
    if ref() is None or not os.path.exists(REF_SOLVER_PATH):
        return None
    with _lock:
        if _ref_solver is None:
            R = ctypes.CDLL(REF_SOLVER_PATH)
            R.ibref_chebpcg.argtypes = [ctypes.c_int, _APPLY, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                        _dp, ctypes.c_double, _dp]
            R.ibref_chebpcg.restype = ctypes.c_longlong
            R.ibref_chebyshev_weights.argtypes = [ctypes.c_double, ctypes.c_double, _dp]
            _ref_solver = R
    return _ref_solver


def ref_chebyshev_weights(a, b):
    out = np.zeros(4)
    ref_solver().ibref_chebyshev_weights(float(a), float(b), _d(out))
    return out


def ref_chebpcg(fg: FluidGrid, lam, b, tolerance):
    """x = (I~ - lam L)^-1 b by the reference's pcg and Chebyshev
    preconditioner, the operator being the oracle's, on the oracle's
    Gershgorin interval; returns (x, operator applications)."""
    n = fg.size
    lower, upper = gershgorin(fg, lam)

    def apply(inp, out, ctx):
        src = np.ctypeslib.as_array(inp, shape=(n,))
        dst = np.ctypeslib.as_array(out, shape=(n,))
        dst[:] = diffusion_apply(fg, 2, src.copy(), lam=lam)

    cb = _APPLY(apply)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n)
    calls = ref_solver().ibref_chebpcg(n, cb, None, float(lower), float(upper), _d(bb), float(tolerance), _d(x))
    return x, int(calls)
