"""Membrane forces (tension, bending, dissipation, tether, repelling) on the
device against the oracle, through the C ABI.

The tension kernel evaluates the reference's expressions in its order
without contraction, so it matches the oracle bit for bit.  The surface
geometry's operator products are library GEMMs whose summation order differs
from the oracle's loop: they are held to 1e-11 of each quantity's largest
value with Fourier differentiation operators (entries up to N^2, sums with
cancellation) and 1e-12 with random ones, the normal and patch area alike.  The whole
pipeline (geometry of the rest and current shapes, then tension) keeps the
mechanics: total force and torque vanish on closed surfaces (to the
trapezoid rule's accuracy: near rounding for the Skalak law, 1e-6 for the
neo-Hookean law, whose 1/sqrt(I2) terms converge more slowly on the grid)."""
import numpy as np
import pytest

import torus as T

pytestmark = pytest.mark.gpu

NU, NV = 48, 24
SHEAR, BULK = 2.5, 25.0
MATS = [np.array([[1.3, 0.2, 0.0], [0.0, 0.8, 0.1], [0.05, 0.0, 1.1]]),
        np.diag([0.9, 1.2, 1.0]),
        np.array([[1.0, 0.0, 0.3], [0.1, 1.1, 0.0], [0.0, -0.2, 0.95]])]


def _to(d, dev):
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in d.items()}


def _host(d):
    return {k: v.cpu().numpy() for k, v in d.items()}


def _shapes(nc, cur=True):
    return [T.shape(NU, NV, A=MATS[i % len(MATS)] if cur else None, eps=0.02 * (i + 1) if cur else 0.0)
            for i in range(nc)]


def _analytic(shapes):
    g = T.pack(shapes)
    w = T.weights(NU, NV)
    g["sigma"] = np.concatenate([w * np.linalg.norm(np.cross(s["tu"].T, s["tv"].T), axis=1) for s in shapes])
    return g


@pytest.mark.parametrize("law", [0, 1, 2])
def test_tension_matches_oracle_bit_for_bit(ibk, cuda, oracle, law):
    rest, cur = _analytic(_shapes(3, cur=False)), _analytic(_shapes(3))
    f_ref = oracle.membrane_tension(law, SHEAR, BULK, rest, cur)
    f = ibk.membrane_tension(law, SHEAR, BULK, _to(rest, cuda), _to(cur, cuda)).cpu().numpy()
    assert np.array_equal(f, f_ref)
    # random (valid, non-degenerate) geometry as well
    rng = np.random.default_rng(3)
    n = 5000
    base = {k: rng.normal(size=3 * n) for k in ("tu", "tv", "tuu", "tuv", "tvv")}
    base["tu"] = (base["tu"].reshape(3, n) + np.array([[2.0], [0.0], [0.0]])).reshape(-1)
    base["tv"] = (base["tv"].reshape(3, n) + np.array([[0.0], [2.0], [0.0]])).reshape(-1)
    base["sigma"] = rng.uniform(0.5, 1.5, size=n)
    moved = {k: v + 0.1 * rng.normal(size=v.size) for k, v in base.items()}
    f_ref = oracle.membrane_tension(law, SHEAR, BULK, base, moved)
    f = ibk.membrane_tension(law, SHEAR, BULK, _to(base, cuda), _to(moved, cuda)).cpu().numpy()
    assert np.array_equal(f, f_ref)


def test_geometry_matches_oracle(ibk, cuda, oracle):
    import torch
    w = T.weights(NU, NV)
    ops = T.operators(NU, NV)
    shapes = _shapes(3)
    x = T.pack(shapes)["position"]
    for first in (ops[0], None):
        o = [first] + ops[1:]
        plan = ibk.SurfacePlan([None if m is None else torch.from_numpy(m).to(cuda) for m in o],
                               torch.from_numpy(w).to(cuda))
        g = _host(plan.geometry(torch.from_numpy(x).to(cuda), 3))
        ref = oracle.surface_geometry(o, w, x, 3)
        for k in oracle.SURFACE_FIELDS:
            assert np.abs(g[k] - ref[k]).max() <= 1e-11 * np.abs(ref[k]).max(), k
    # rectangular operators (more samples than data sites), several shapes
    rng = np.random.default_rng(5)
    ns, nd, nc = 300, 120, 4
    o = [rng.normal(size=(ns, nd)) / nd for _ in range(6)]
    wr = rng.uniform(0.5, 1.0, size=ns)
    xr = rng.normal(size=3 * nd * nc)
    plan = ibk.SurfacePlan([torch.from_numpy(m).to(cuda) for m in o], torch.from_numpy(wr).to(cuda))
    g = _host(plan.geometry(torch.from_numpy(xr).to(cuda), nc))
    ref = oracle.surface_geometry(o, wr, xr, nc)
    for k in oracle.SURFACE_FIELDS:
        assert np.abs(g[k] - ref[k]).max() <= 1e-12 * np.abs(ref[k]).max(), k


@pytest.mark.parametrize("law,tol", [(0, 1e-10), (1, 1e-6)])
def test_pipeline_keeps_force_and_torque_balance(ibk, cuda, oracle, law, tol):
    import torch
    w = T.weights(NU, NV)
    ops = [torch.from_numpy(m).to(cuda) for m in T.operators(NU, NV)]
    plan = ibk.SurfacePlan(ops, torch.from_numpy(w).to(cuda))
    nc = 3
    x0 = torch.from_numpy(T.pack(_shapes(nc, cur=False))["position"]).to(cuda)
    x1 = torch.from_numpy(T.pack(_shapes(nc))["position"]).to(cuda)
    rest, cur = plan.geometry(x0, nc), plan.geometry(x1, nc)
    f = ibk.membrane_tension(law, SHEAR, BULK, rest, cur).cpu().numpy()
    n = NU * NV
    pos = cur["position"].cpu().numpy().reshape(3, nc, n)
    F = f.reshape(3, nc, n)
    for c in range(nc):
        Fc, Mc = T.totals(F[:, c].reshape(-1), pos[:, c].reshape(-1), n)
        scale = np.abs(F[:, c]).sum()
        assert np.abs(Fc).max() <= tol * scale and np.abs(Mc).max() <= tol * scale
    # the same pipeline on the oracle
    on = [m.cpu().numpy() for m in ops]
    r = oracle.surface_geometry(on, w, x0.cpu().numpy(), nc)
    c_ = oracle.surface_geometry(on, w, x1.cpu().numpy(), nc)
    f_ref = oracle.membrane_tension(law, SHEAR, BULK, r, c_)
    assert np.abs(f - f_ref).max() <= 1e-9 * np.abs(f_ref).max()


@pytest.mark.parametrize("preferred", [False, True])
def test_bending_matches_oracle(ibk, cuda, oracle, preferred):
    import torch
    w = T.weights(NU, NV)
    ops = T.operators(NU, NV)
    dops = [None] + ops[1:]
    dev_ops = [None if m is None else torch.from_numpy(m).to(cuda) for m in dops]
    wt = torch.from_numpy(w).to(cuda)
    data_plan = ibk.SurfacePlan(dev_ops, wt)
    sample_plan = ibk.SurfacePlan([torch.from_numpy(m).to(cuda) for m in ops], wt)
    nc = 3
    x0 = T.pack([T.shape(NU, NV, R=2.0, r=0.7) for _ in range(nc)])["position"]
    x1 = T.pack([T.shape(NU, NV, R=2.0, r=0.7, A=MATS[i], eps=0.02 * (i + 1)) for i in range(nc)])["position"]
    X0, X1 = torch.from_numpy(x0).to(cuda), torch.from_numpy(x1).to(cuda)
    rest, cur = sample_plan.geometry(X0, nc), sample_plan.geometry(X1, nc)
    f = ibk.membrane_bending(data_plan, sample_plan, 1.0, preferred, X0, X1, rest, cur, nc).cpu().numpy()
    r, c = oracle.surface_geometry(ops, w, x0, nc), oracle.surface_geometry(ops, w, x1, nc)
    f_ref = oracle.membrane_bending(dops, w, ops, 1.0, preferred, x0, x1, r, c, nc)
    assert np.abs(f - f_ref).max() <= 1e-9 * np.abs(f_ref).max()
    if not preferred:
        n = NU * NV
        F = f.reshape(3, nc, n)
        pos = cur["position"].cpu().numpy().reshape(3, nc, n)
        for k in range(nc):
            Fc, Mc = T.totals(F[:, k].reshape(-1), pos[:, k].reshape(-1), n)
            scale = np.abs(F[:, k]).sum()
            # the grid's accuracy for the bending integrand on these sheared
            # tori at 48 x 24 (the oracle gives up to 2.7e-6, converging to
            # 1.5e-8 at 64 x 32)
            assert np.abs(Fc).max() <= 1e-5 * scale and np.abs(Mc).max() <= 1e-5 * scale


def test_no_bending_force_on_the_clifford_torus_gpu(ibk, cuda):
    import torch
    w = torch.from_numpy(T.weights(64, 32)).to(cuda)
    ops = [torch.from_numpy(m).to(cuda) for m in T.operators(64, 32)]
    data_plan = ibk.SurfacePlan([None] + ops[1:], w)
    sample_plan = ibk.SurfacePlan(ops, w)
    out = []
    for R in (np.sqrt(2.0), 2.5):
        x = torch.from_numpy(T.shape(64, 32, R=R, r=1.0)["position"].reshape(-1)).to(cuda)
        g = sample_plan.geometry(x, 1)
        out.append(ibk.membrane_bending(data_plan, sample_plan, 1.0, False, None, x, None, g, 1).abs().max().item())
    assert out[0] <= 1e-3 * out[1]


KAPPA = 0.7


def _velocity(nc, phase=0.3):
    u, v = T.grid(NU, NV)
    one = [np.stack([np.sin(u + phase + c) * np.cos(v), np.cos(2 * u) + 0.3 * np.sin(v - phase),
                     np.sin(u - 2 * v + c)]) for c in range(nc)]
    return np.stack(one, axis=1).reshape(-1)


def test_dissipation_kernel_matches_oracle_bit_for_bit(ibk, cuda, oracle):
    """Integer operators and velocities make every operator product exact
    whatever the GEMM's summation order, so the per-sample kernel sees the
    oracle's inputs and must give its bits."""
    import torch
    rng = np.random.default_rng(17)
    ns, nd, nc = 300, 40, 3
    ops = [rng.integers(-3, 4, size=(ns, nd)).astype(np.float64) for _ in range(6)]
    u = rng.integers(-5, 6, size=3 * nd * nc).astype(np.float64)
    n = ns * nc
    cur = {k: rng.normal(size=3 * n) for k in ("tu", "tv", "tuu", "tuv", "tvv")}
    cur["tu"] = (cur["tu"].reshape(3, n) + np.array([[2.0], [0.0], [0.0]])).reshape(-1)
    cur["tv"] = (cur["tv"].reshape(3, n) + np.array([[0.0], [2.0], [0.0]])).reshape(-1)
    cur["sigma"] = rng.uniform(0.5, 1.5, size=n)
    plan = ibk.SurfacePlan([torch.from_numpy(m).to(cuda) for m in ops],
                           torch.from_numpy(rng.uniform(0.5, 1.0, size=ns)).to(cuda))
    f = ibk.membrane_dissipation(plan, KAPPA, torch.from_numpy(u).to(cuda), _to(cur, cuda), nc).cpu().numpy()
    f_ref = oracle.membrane_dissipation(ops, KAPPA, u, cur, nc)
    assert np.array_equal(f, f_ref)


def test_dissipation_pipeline(ibk, cuda, oracle):
    """Geometry then dissipation on sheared tori: the oracle's forces (to the
    GEMMs' summation order), none under rigid motion, and zero total force
    and torque to the grid's accuracy."""
    import torch
    w = T.weights(NU, NV)
    ops = T.operators(NU, NV)
    plan = ibk.SurfacePlan([torch.from_numpy(m).to(cuda) for m in ops], torch.from_numpy(w).to(cuda))
    nc = 3
    x = T.pack(_shapes(nc))["position"]
    X = torch.from_numpy(x).to(cuda)
    cur = plan.geometry(X, nc)
    U = _velocity(nc)
    f = ibk.membrane_dissipation(plan, KAPPA, torch.from_numpy(U).to(cuda), cur, nc).cpu().numpy()
    g = oracle.surface_geometry(ops, w, x, nc)
    f_ref = oracle.membrane_dissipation(ops, KAPPA, U, g, nc)
    assert np.abs(f - f_ref).max() <= 1e-9 * np.abs(f_ref).max()
    n = NU * NV
    pos = x.reshape(3, nc, n)
    F = f.reshape(3, nc, n)
    for c in range(nc):
        Fc, Mc = T.totals(F[:, c].reshape(-1), pos[:, c].reshape(-1), n)
        scale = np.abs(F[:, c]).sum()
        # the grid's accuracy for the stress divergence on these sheared tori
        # at 48 x 24 (the oracle gives up to 1.5e-6, converging to 1.5e-8 at
        # 64 x 32 and 5e-13 at 96 x 48)
        assert np.abs(Fc).max() <= 1e-5 * scale and np.abs(Mc).max() <= 1e-5 * scale
    omega, a = np.array([0.3, -0.5, 0.8]), np.array([1.0, 2.0, -0.5])
    rigid = np.stack([a[:, None] + np.cross(omega, pos[:, c].T).T for c in range(nc)], axis=1).reshape(-1)
    fr = ibk.membrane_dissipation(plan, KAPPA, torch.from_numpy(rigid).to(cuda), cur, nc).cpu().numpy()
    assert np.abs(fr).max() <= 1e-11 * np.abs(f).max()


def test_tether_and_repelling_match_oracle(ibk, cuda, oracle):
    rng = np.random.default_rng(23)
    n = 20000
    rest = {"position": rng.normal(size=3 * n)}
    cur = {"position": rest["position"] + 0.05 * rng.normal(size=3 * n), "sigma": rng.uniform(0.5, 1.5, size=n)}
    f = ibk.membrane_tether(3.0, _to(rest, cuda), _to(cur, cuda)).cpu().numpy()
    assert np.array_equal(f, oracle.membrane_tether(3.0, rest["position"], cur["position"]))
    # a wall at y = 0.3 reaching 0.5 either side: about a third of the samples
    f = ibk.membrane_repelling(2.0, _to(cur, cuda), height=0.3, range_=0.25).cpu().numpy()
    f_ref = oracle.membrane_repelling(2.0, 0.3, 0.25, cur["position"], cur["sigma"])
    # the device's log and exp against the C library's: a few ulp apart
    assert np.abs(f - f_ref).max() <= 4e-15 * np.abs(f_ref).max()
    assert np.array_equal(f == 0, f_ref == 0)


def test_red_cell_force_set_balances(ibk, cuda):
    """The reference's red-cell forces (tension, bending, dissipation; summed
    as forces::combine does) on deformed, moving tori: zero total force and
    torque per shape to the grid's accuracy."""
    import torch
    w = torch.from_numpy(T.weights(NU, NV)).to(cuda)
    ops = [torch.from_numpy(m).to(cuda) for m in T.operators(NU, NV)]
    data_plan = ibk.SurfacePlan([None] + ops[1:], w)
    sample_plan = ibk.SurfacePlan(ops, w)
    nc = 3
    X0 = torch.from_numpy(T.pack([T.shape(NU, NV, R=2.0, r=0.7) for _ in range(nc)])["position"]).to(cuda)
    X1 = torch.from_numpy(T.pack([T.shape(NU, NV, R=2.0, r=0.7, A=MATS[i], eps=0.02 * (i + 1))
                                  for i in range(nc)])["position"]).to(cuda)
    rest, cur = sample_plan.geometry(X0, nc), sample_plan.geometry(X1, nc)
    U = torch.from_numpy(_velocity(nc)).to(cuda)
    f = (ibk.membrane_tension(ibk.SKALAK, SHEAR, BULK, rest, cur)
         + ibk.membrane_bending(data_plan, sample_plan, 0.05, False, X0, X1, rest, cur, nc)) \
        + ibk.membrane_dissipation(sample_plan, KAPPA, U, cur, nc)
    n = NU * NV
    F = f.cpu().numpy().reshape(3, nc, n)
    pos = X1.cpu().numpy().reshape(3, nc, n)
    for c in range(nc):
        Fc, Mc = T.totals(F[:, c].reshape(-1), pos[:, c].reshape(-1), n)
        scale = np.abs(F[:, c]).sum()
        assert np.abs(Fc).max() <= 1e-5 * scale and np.abs(Mc).max() <= 1e-5 * scale
