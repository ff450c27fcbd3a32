"""GPU test of ibk_interpolate_noalloc, the interpolation entry point for
callers that may not allocate device memory (it keeps its scratch in a fixed
array inside the library instead of plan buffers grown with cudaMalloc).

Two calls in a row (different grids and point sets, so the second call runs
on scratch the first one left behind) are each compared with the regular
plan-based ibk_interpolate: bit-exact in FP64, within the FP32C normwise
tolerance otherwise -- in 2-D and 3-D, on MAC and cell-centred grids, for
several deltas, and on a grid too small to tile (the per-point kernel).
Oversized calls (too many points, too many bins) are rejected before any
device work.  This file sorts last so a stop-at-first-failure run has already
run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP32C_TOL = 1e-5


def _abi_domain(ibk, dims, lengths, bounds):
    d = ibk._Domain()
    d.dims = dims
    for i in range(dims):
        d.length[i] = lengths[i]
        d.boundary[i] = bounds[i]
    return d


def _both(ibk, device, dims, lengths, bounds, tag, ref, delta, precision, n, seed):
    """(noalloc result, plan result) for one seeded case."""
    import torch
    rng = np.random.default_rng(seed)
    T = ibk.Mac if tag == ibk.TAG_MAC else ibk.Centered
    dom = ibk.Domain(*[ibk.Dimension(lengths[i], bounds[i]) for i in range(dims)])
    dl = ibk.DeltaFn()
    dl.kind, dl.order = delta
    plan = ibk.Plan(T(ref), dom, dl, precision)
    sizes = plan.sizes()
    x = np.concatenate([rng.uniform(-0.05, lengths[i] + 0.05, n) for i in range(dims)])
    xd = torch.from_numpy(x).to(device)
    ue = [torch.from_numpy(rng.normal(size=s)).to(device) for s in sizes]
    want = torch.full((dims * n,), np.nan, dtype=torch.float64, device=device)
    plan.interpolate(n, xd, ue, want)
    got = torch.full((dims * n,), np.nan, dtype=torch.float64, device=device)
    ptrs = (ctypes.c_void_p * 3)(*([u.data_ptr() for u in ue] + [0] * (3 - dims)))
    d = ibk._Delta()
    d.kind, d.order = delta
    stream = torch.cuda.current_stream().cuda_stream
    ibk.check(ibk.lib().ibk_interpolate_noalloc(
        ctypes.byref(_abi_domain(ibk, dims, lengths, bounds)), tag, ref, d, precision, n,
        xd.data_ptr(), ptrs, got.data_ptr(), stream))
    torch.cuda.synchronize()
    return got.cpu().numpy(), want.cpu().numpy()


def _compare(ibk, got, want, precision, dims, n):
    assert np.all(np.isfinite(got))
    if precision == ibk.FP64:
        assert np.array_equal(got, want)
    else:
        for c in range(dims):
            a, b = got[c * n:(c + 1) * n], want[c * n:(c + 1) * n]
            assert np.abs(a - b).max() <= FP32C_TOL * np.abs(b).max()


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_plan_entry_point_twice(ibk, cuda, precision):
    from ib_cu_b200 import workloads as W
    for w in (W.channel(seed=31), W.single_rbc(seed=32)):
        import torch
        dom = ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)])
        plan = ibk.Plan(ibk.Mac(w.refinement), dom, ibk.Bspline(3), precision)
        sizes = plan.sizes()
        ue_host = W.grid_velocity(w, sizes, [plan.info.comp_points(c) for c in range(3)])
        x = torch.from_numpy(w.x).to(cuda)
        ue = [torch.from_numpy(u).to(cuda) for u in ue_host]
        n = w.n
        want = torch.full((3 * n,), np.nan, dtype=torch.float64, device=cuda)
        plan.interpolate(n, x, ue, want)
        got = torch.full((3 * n,), np.nan, dtype=torch.float64, device=cuda)
        ptrs = (ctypes.c_void_p * 3)(*[u.data_ptr() for u in ue])
        d = ibk._Delta()
        d.kind, d.order = ibk.BSPLINE, 3
        ibk.check(ibk.lib().ibk_interpolate_noalloc(
            ctypes.byref(_abi_domain(ibk, 3, w.lengths, w.boundaries)), ibk.TAG_MAC, w.refinement, d,
            precision, n, x.data_ptr(), ptrs, got.data_ptr(), torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        _compare(ibk, got.cpu().numpy(), want.cpu().numpy(), precision, 3, n)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case", [
    # dims, lengths, boundaries, tag, refinement, delta, points
    (2, [1.6, 0.8], [0, 1], 0, 32, (0, 3), 3000),          # 2-D MAC, walls, bspline<3>
    (3, [0.8, 0.8, 0.8], [0, 0, 0], 1, 24, (0, 3), 4000),   # cell-centred grid
    (3, [1.2, 0.6, 0.9], [1, 0, 1], 0, 20, (1, 0), 4000),   # peskin (every-other ordering)
    (3, [1.0, 0.5, 1.0], [0, 1, 0], 0, 32, (2, 0), 4000),   # roma (3 points)
    (3, [0.4, 0.4, 0.4], [0, 0, 0], 0, 4, (0, 5), 500),     # 4 cells per axis < 6: per-point kernel
])
def test_noalloc_shapes_deltas_and_tags(ibk, cuda, precision, case):
    dims, lengths, bounds, tag, ref, delta, n = case
    for seed in (1, 2):   # two calls in a row on the shared scratch
        got, want = _both(ibk, cuda, dims, lengths, bounds, tag, ref, delta, precision, n, seed)
        _compare(ibk, got, want, precision, dims, n)


def test_noalloc_rejects_oversized_calls(ibk, cuda):
    from ib_cu_b200 import workloads as W
    w = W.channel(seed=33)
    delta = ibk._Delta()
    delta.kind, delta.order = ibk.BSPLINE, 3
    ptrs = (ctypes.c_void_p * 3)(1, 1, 1)
    lib = ibk.lib()
    status = lib.ibk_interpolate_noalloc(
        ctypes.byref(_abi_domain(ibk, 3, w.lengths, w.boundaries)), ibk.TAG_MAC, w.refinement, delta,
        ibk.FP64, (1 << 19) + 1, 1, ptrs, 1, None)
    assert status == 5   # IBK_ERR_CAPACITY, raised before any device work
    assert b"524288" in lib.ibk_last_error()
    # 512 x 256 x 512 cells: 32 x 16 x 32 tiles x 27 reach classes > 262144 bins
    status = lib.ibk_interpolate_noalloc(
        ctypes.byref(_abi_domain(ibk, 3, [12.8, 6.4, 12.8], [0, 1, 0])), ibk.TAG_MAC, 256, delta,
        ibk.FP64, 10, 1, ptrs, 1, None)
    assert status == 5
    assert b"262144" in lib.ibk_last_error()
