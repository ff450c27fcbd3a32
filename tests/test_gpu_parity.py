"""GPU parity of the CUDA operators against the oracle and the reference's
golden fixtures, through the C ABI.

Tolerances (FP64 path):
  * sort keys, stencil origins: bit-exact;
  * interpolate: bit-exact (same operation order as the reference), except
    the cosine delta, whose cos() comes from CUDA's libdevice and may differ
    from the host's libm in the last place: |err| <= 1e-13 * sum|w u|;
  * spread: differs from the reference only by summation order:
    |err| <= 1e-12 * sum|res w F| per face (faces nobody touches are 0).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")
SPREAD_TOL = 1e-12
COS_TOL = 1e-13
FP32C_TOL = 1e-5      # normwise: max|err| <= 1e-5 * max|reference| per component


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def dev(a, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


def plan_for(ibk, dims, L, solid, tag, ref, kind, order, precision=0):
    T = ibk.Mac if tag == 0 else ibk.Centered
    dom = ibk.Domain(*[ibk.Dimension(float(L[d]), int(solid[d])) for d in range(dims)])
    delta = ibk.DeltaFn()
    delta.kind, delta.order = int(kind), int(order)
    return ibk.Plan(T(int(ref)), dom, delta, precision)


def device_keys(plan, x, device):
    import torch
    n = x.size // plan.dims
    xd = dev(x, device)
    out = []
    for c in range(plan.dims):
        k = torch.empty(n, dtype=torch.int32, device=device)
        plan.sort_keys(c, n, xd, k)
        out.append(k.cpu().numpy())
    return out


def device_spread(plan, x, f, device, prefill=np.nan):
    import torch
    n = x.size // plan.dims
    fe = [torch.full((s,), prefill, dtype=torch.float64, device=device) for s in plan.sizes()]
    plan.spread(n, dev(x, device), dev(f, device), fe)
    torch.cuda.synchronize()
    plan.check()
    return [t.cpu().numpy() for t in fe]


def device_interp(plan, x, ue, device, prefill=np.nan):
    import torch
    n = x.size // plan.dims
    ul = torch.full((plan.dims * n,), prefill, dtype=torch.float64, device=device)
    plan.interpolate(n, dev(x, device), [dev(u, device) for u in ue], ul)
    torch.cuda.synchronize()
    plan.check()
    return ul.cpu().numpy()


def check_spread(got, want, absum, tol=SPREAD_TOL):
    for c in range(len(want)):
        err = np.abs(got[c] - want[c])
        bound = tol * absum[c]
        bad = ~(err <= bound)
        assert not bad.any(), (c, int(bad.sum()), float(err[bad].max()) if bad.any() else 0)


def check_interp(got, want, absum, exact=True, tol=COS_TOL):
    if exact:
        assert np.array_equal(got, want), float(np.abs(got - want).max())
    else:
        assert np.all(np.abs(got - want) <= tol * absum)


def golden_cases(z):
    return sorted({k.split("/")[0] for k in z.files})


def golden_plan(ibk, z, prefix):
    dims, tag, ref, kind, order = (int(v) for v in z[f"{prefix}/meta"])
    return plan_for(ibk, dims, z[f"{prefix}/length"], z[f"{prefix}/solid"], tag, ref, kind, order)


def test_plan_geometry_matches_reference(ibk, cuda, golden):
    for prefix in golden_cases(golden):
        plan = golden_plan(ibk, golden, prefix)
        for c in range(plan.dims):
            geo = golden[f"{prefix}/c{c}/geo"]
            assert plan.info.unit == geo[0] and plan.info.resolution == geo[1]
            for d in range(plan.dims):
                assert plan.info.cells[c][d] == geo[2 + 3 * d]
                assert plan.info.points[c][d] == geo[3 + 3 * d]
                assert plan.info.shift[c][d] == geo[4 + 3 * d]


def test_sort_keys_bit_exact_golden(ibk, cuda, golden):
    for prefix in golden_cases(golden):
        plan = golden_plan(ibk, golden, prefix)
        keys = device_keys(plan, golden[f"{prefix}/x"], cuda)
        for c in range(plan.dims):
            assert np.array_equal(keys[c], golden[f"{prefix}/c{c}/keys"]), (prefix, c)


def test_interpolate_fp64_golden(ibk, cuda, golden):
    for prefix in golden_cases(golden):
        plan = golden_plan(ibk, golden, prefix)
        ue = [golden[f"{prefix}/ue{c}"] for c in range(plan.dims)]
        ul = device_interp(plan, golden[f"{prefix}/x"], ue, cuda)
        exact = "cosine" not in prefix
        check_interp(ul, golden[f"{prefix}/ul"], golden[f"{prefix}/ul_abs"], exact)


def test_spread_fp64_golden(ibk, cuda, golden):
    for prefix in golden_cases(golden):
        plan = golden_plan(ibk, golden, prefix)
        fe = device_spread(plan, golden[f"{prefix}/x"], golden[f"{prefix}/f"], cuda)
        want = [golden[f"{prefix}/fe{c}"] for c in range(plan.dims)]
        absum = [golden[f"{prefix}/fe_abs{c}"] for c in range(plan.dims)]
        check_spread(fe, want, absum)


def _workload_case(ibk, oracle, w, device, precision=0):
    g = oracle.geometry(3, w.lengths, w.boundaries, oracle.TAG_MAC, w.refinement)
    plan = plan_for(ibk, 3, w.lengths, w.boundaries, 0, w.refinement, 0, 3, precision)
    from ib_cu_b200 import workloads as W
    ue = W.grid_velocity(w, [int(g.size[c]) for c in range(3)], [g.comp_points(c) for c in range(3)])
    return g, plan, ue


@pytest.mark.parametrize("name", ["single-rbc", "channel"])
def test_workload_parity_fp64(ibk, oracle, cuda, name):
    from ib_cu_b200 import workloads as W
    w = W.CONFIGS[name](seed=11)
    g, plan, ue = _workload_case(ibk, oracle, w, cuda)
    keys = device_keys(plan, w.x, cuda)
    for c in range(3):
        assert np.array_equal(keys[c], oracle.sort_keys(g, c, w.x))
    ul = device_interp(plan, w.x, ue, cuda)
    want_ul, ua = oracle.interpolate(g, w.x, ue, with_abs=True)
    check_interp(ul, want_ul, ua, exact=True)
    fe = device_spread(plan, w.x, w.f, cuda)
    want_fe, fa = oracle.spread(g, w.x, w.f, with_abs=True)
    check_spread(fe, want_fe, fa)


@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("delta", [("bspline", 1), ("bspline", 2), ("bspline", 3), ("bspline", 4),
                                   ("bspline", 5), ("peskin", 0), ("roma", 0), ("cosine", 0), ("hat", 0)])
def test_every_delta_fp64(ibk, oracle, cuda, dims, delta):
    rng = np.random.default_rng(100 + dims)
    L = [1.6, 0.8, 1.2][:dims]
    solid = [0, 1, 0][:dims]
    kind = oracle.DELTA_NAMES[delta[0]]
    g = oracle.geometry(dims, L, solid, oracle.TAG_MAC, 32, kind, delta[1])
    plan = plan_for(ibk, dims, L, solid, 0, 32, kind, delta[1])
    n = 2000
    x = np.concatenate([rng.uniform(-0.02, l + 0.02, n) for l in L])
    f = rng.normal(size=dims * n)
    ue = [rng.normal(size=int(g.size[c])) for c in range(dims)]
    ul = device_interp(plan, x, ue, cuda)
    want, ua = oracle.interpolate(g, x, ue, with_abs=True)
    check_interp(ul, want, ua, exact=(delta[0] != "cosine"))
    fe = device_spread(plan, x, f, cuda)
    want_fe, fa = oracle.spread(g, x, f, with_abs=True)
    check_spread(fe, want_fe, fa)


def test_zero_points_is_a_no_op(ibk, cuda):
    import torch
    plan = plan_for(ibk, 3, [1.6] * 3, [0, 0, 0], 0, 16, 0, 3)
    fe = [torch.full((s,), 5.0, dtype=torch.float64, device=cuda) for s in plan.sizes()]
    x = torch.zeros(3, dtype=torch.float64, device=cuda)
    plan.spread(0, x, x, fe)
    ul = torch.full((3,), 5.0, dtype=torch.float64, device=cuda)
    plan.interpolate(0, x, fe, ul)
    plan.spread(-1, x, x, fe)
    torch.cuda.synchronize()
    assert all(bool((t == 5.0).all()) for t in fe) and bool((ul == 5.0).all())


def test_overwrite_semantics(ibk, oracle, cuda):
    """Pre-filled outputs (NaN, garbage) give identical results."""
    rng = np.random.default_rng(9)
    plan = plan_for(ibk, 3, [1.6] * 3, [0, 0, 0], 0, 16, 0, 3)
    x = rng.uniform(0, 1.6, 3 * 64)
    f = rng.normal(size=3 * 64)
    ue = [rng.normal(size=s) for s in plan.sizes()]
    a = device_spread(plan, x, f, cuda, prefill=np.nan)
    b = device_spread(plan, x, f, cuda, prefill=1e30)
    for c in range(3):
        assert np.allclose(a[c], b[c], rtol=1e-13, atol=1e-300)
    u1 = device_interp(plan, x, ue, cuda, prefill=np.nan)
    u2 = device_interp(plan, x, ue, cuda, prefill=-7.0)
    assert np.array_equal(u1, u2)


def test_points_outside_walls_and_domain(ibk, oracle, cuda):
    """Points beyond solid walls clamp their origin (lossy, as in the
    reference); points outside a periodic box wrap."""
    rng = np.random.default_rng(10)
    L = [3.2, 1.6, 3.2]
    g = oracle.geometry(3, L, [0, 1, 0], oracle.TAG_MAC, 16)
    plan = plan_for(ibk, 3, L, [0, 1, 0], 0, 16, 0, 3)
    n = 500
    x = np.concatenate([rng.uniform(-3.0, 6.0, n), rng.uniform(-0.5, 2.1, n), rng.uniform(-3.0, 6.0, n)])
    f = rng.normal(size=3 * n)
    ue = [rng.normal(size=int(g.size[c])) for c in range(3)]
    keys = device_keys(plan, x, cuda)
    for c in range(3):
        assert np.array_equal(keys[c], oracle.sort_keys(g, c, x))
    ul = device_interp(plan, x, ue, cuda)
    want, ua = oracle.interpolate(g, x, ue, with_abs=True)
    check_interp(ul, want, ua)
    fe = device_spread(plan, x, f, cuda)
    want_fe, fa = oracle.spread(g, x, f, with_abs=True)
    check_spread(fe, want_fe, fa)


def test_reference_shaped_python_api(ibk, oracle, cuda):
    """Spread(tag, domain, delta)(n, x, fl) returns new grid vectors;
    Interpolate(...)(x, ue) returns a new point matrix (novel.h:236-250,
    interpolate.h:124-138)."""
    import torch
    dom = ibk.Domain(ibk.Dimension(1.0), ibk.Dimension(1.0), ibk.Dimension(1.0))
    spread = ibk.Spread(ibk.Mac(16), dom, ibk.Bspline(3))
    interp = ibk.Interpolate(ibk.Mac(16), dom, ibk.Bspline(3))
    x = torch.full((6,), 0.5, dtype=torch.float64, device=cuda)     # test/grid.cc
    fl = torch.ones(6, dtype=torch.float64, device=cuda)
    fe = spread(2, x, fl)
    u = [torch.ones(16 ** 3, dtype=torch.float64, device=cuda) for _ in range(3)]
    ul = interp(x, u)
    torch.cuda.synchronize()
    assert torch.allclose(ul, torch.ones_like(ul), atol=1e-15)
    for c in range(3):
        assert abs(float(fe[c].sum()) / 16 ** 3 - 2.0) < 1e-12


def normwise(got, want):
    """max |got - want| / max |want| (the accuracy metric of the FP32C form)."""
    return float(np.abs(got - want).max() / max(np.abs(want).max(), 1e-300))


@pytest.mark.parametrize("name", ["single-rbc", "channel"])
def test_workload_accuracy_fp32c(ibk, oracle, cuda, name):
    """FP32 weights and products with exact fixed-point sums (spread), FP32
    staged values and row sums with an FP64 total (interpolate), against
    the FP64 oracle."""
    from ib_cu_b200 import workloads as W
    w = W.CONFIGS[name](seed=12)
    g, plan, ue = _workload_case(ibk, oracle, w, cuda, precision=ibk.FP32C)
    ul = device_interp(plan, w.x, ue, cuda)
    want_ul = oracle.interpolate(g, w.x, ue)
    fe = device_spread(plan, w.x, w.f, cuda)
    want_fe = oracle.spread(g, w.x, w.f)
    n = w.n
    for c in range(3):
        e = normwise(ul[c * n:(c + 1) * n], want_ul[c * n:(c + 1) * n])
        assert e <= FP32C_TOL, ("interp", c, e)
        e = normwise(fe[c], want_fe[c])
        assert e <= FP32C_TOL, ("spread", c, e)
        # faces no stencil touches stay exactly zero
        assert np.all(fe[c][want_fe[c] == 0] == 0)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("lengths,solid,ref", [
    ([2.0, 1.0, 1.0], [0, 1, 0], 17),   # 34 x 17 x 17 cells: tiles 14+14+6, one, one
    ([2.0, 1.0, 1.0], [1, 0, 1], 9),    # 18 x 9 x 9: two tiles (14+4) along x
    ([1.0, 1.0, 1.0], [0, 0, 0], 33),   # 33^3: tiles 14+14+5 on every axis
    ([0.75, 0.5, 0.875], [0, 0, 0], 2), # 12 x 8 x 14: every axis a single wrapping tile
    # periodic axes cut into two tiles where the stencil width plus the tile
    # extent reaches the period (18 cells: 14+4, nodes wrapped one by one) and
    # where it stays one cell below it (19 cells: 14+5, one shift per axis)
    ([2.0, 1.0, 1.0], [0, 1, 0], 9),    # 18 x 9 x 9
    ([1.0, 1.0, 1.0], [0, 1, 0], 19),   # 19 x 19 x 19
])
def test_tile_decompositions(ibk, oracle, cuda, precision, lengths, solid, ref):
    rng = np.random.default_rng(21)
    g = oracle.geometry(3, lengths, solid, oracle.TAG_MAC, ref)
    plan = plan_for(ibk, 3, lengths, solid, 0, ref, 0, 3, precision)
    plan.set_tiles([16, 16, 16], [16, 16, 16])    # the decompositions listed above
    assert [plan.info.cells[0][d] for d in range(3)] == [g.cells[0][d] for d in range(3)]
    n = 3000
    x = np.concatenate([rng.uniform(-0.1, l + 0.1, n) for l in lengths])
    f = rng.normal(size=3 * n)
    ue = [rng.normal(size=int(g.size[c])) for c in range(3)]
    ul = device_interp(plan, x, ue, cuda)
    want, ua = oracle.interpolate(g, x, ue, with_abs=True)
    fe = device_spread(plan, x, f, cuda)
    want_fe, fa = oracle.spread(g, x, f, with_abs=True)
    if precision == 0:
        check_interp(ul, want, ua)
        check_spread(fe, want_fe, fa)
    else:
        for c in range(3):
            assert normwise(ul[c * n:(c + 1) * n], want[c * n:(c + 1) * n]) <= FP32C_TOL
            assert normwise(fe[c], want_fe[c]) <= FP32C_TOL


@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("delta", [("bspline", 2), ("bspline", 3), ("bspline", 5), ("peskin", 0),
                                   ("roma", 0), ("cosine", 0), ("hat", 0)])
def test_every_delta_fp32c(ibk, oracle, cuda, dims, delta):
    rng = np.random.default_rng(200 + dims)
    L = [1.6, 0.8, 1.2][:dims]
    solid = [0, 1, 0][:dims]
    kind = oracle.DELTA_NAMES[delta[0]]
    g = oracle.geometry(dims, L, solid, oracle.TAG_MAC, 32, kind, delta[1])
    plan = plan_for(ibk, dims, L, solid, 0, 32, kind, delta[1], ibk.FP32C)
    n = 2000
    x = np.concatenate([rng.uniform(0, l, n) for l in L])
    f = rng.normal(size=dims * n)
    ue = [rng.normal(size=int(g.size[c])) for c in range(dims)]
    ul = device_interp(plan, x, ue, cuda)
    want = oracle.interpolate(g, x, ue)
    fe = device_spread(plan, x, f, cuda)
    want_fe = oracle.spread(g, x, f)
    for c in range(dims):
        assert normwise(ul[c * n:(c + 1) * n], want[c * n:(c + 1) * n]) <= FP32C_TOL
        assert normwise(fe[c], want_fe[c]) <= FP32C_TOL


@pytest.mark.parametrize("seed", [0, 1])
def test_dense_tiles_fp32c_and_fp64(ibk, oracle, cuda, seed):
    """Tiles where one face receives more terms than a 32-bit fixed-point word
    holds (here about five points per cell on a 32^3 periodic grid, the
    density of the ensemble's smallest grids) take the folded FP32C form; both
    forms against the oracle, and the FP32C spread bit-identical run to run."""
    rng = np.random.default_rng(500 + seed)
    L = [0.8, 0.8, 0.8]                    # 32^3 cells at fd::mac{32}
    g = oracle.geometry(3, L, [0, 0, 0], oracle.TAG_MAC, 32)
    n = 160000
    # points crowded onto a few spherical shells, as cell surfaces are
    centres = rng.uniform(0.1, 0.7, size=(12, 3))
    which = rng.integers(0, len(centres), n)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    pts = centres[which] + 0.12 * v
    x = np.ascontiguousarray(pts.T.reshape(-1))
    f = rng.normal(size=3 * n)
    want_fe, fa = oracle.spread(g, x, f, with_abs=True)
    p64 = plan_for(ibk, 3, L, [0, 0, 0], 0, 32, 0, 3, ibk.FP64)
    check_spread(device_spread(p64, x, f, cuda), want_fe, fa)
    p32 = plan_for(ibk, 3, L, [0, 0, 0], 0, 32, 0, 3, ibk.FP32C)
    a = device_spread(p32, x, f, cuda)
    b = device_spread(p32, x, f, cuda)
    for c in range(3):
        assert normwise(a[c], want_fe[c]) <= FP32C_TOL
        assert np.array_equal(a[c], b[c])
