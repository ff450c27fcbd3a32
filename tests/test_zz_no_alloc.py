"""GPU test of ibk_interpolate_noalloc, the interpolation entry point for
callers that may not allocate device memory (it keeps its scratch in a fixed
array inside the library instead of plan buffers grown with cudaMalloc).

Two calls in a row (different grids and point sets, so the second call runs
on scratch the first one left behind) are each compared with the regular
plan-based ibk_interpolate: bit-exact in FP64, within the FP32C normwise
tolerance otherwise.  This file sorts last so a stop-at-first-failure run has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP32C_TOL = 1e-5


def _domain(ibk, w):
    d = ibk._Domain()
    d.dims = 3
    for i in range(3):
        d.length[i] = w.lengths[i]
        d.boundary[i] = w.boundaries[i]
    return d


def _run_both(ibk, w, precision, device):
    import torch
    from ib_cu_b200 import workloads as W
    dom = ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)])
    plan = ibk.Plan(ibk.Mac(w.refinement), dom, ibk.Bspline(3), precision)
    sizes = plan.sizes()
    ue_host = W.grid_velocity(w, sizes, [plan.info.comp_points(c) for c in range(3)])
    x = torch.from_numpy(w.x).to(device)
    ue = [torch.from_numpy(u).to(device) for u in ue_host]
    n = w.n
    want = torch.full((3 * n,), np.nan, dtype=torch.float64, device=device)
    plan.interpolate(n, x, ue, want)
    got = torch.full((3 * n,), np.nan, dtype=torch.float64, device=device)
    ptrs = (ctypes.c_void_p * 3)(*[u.data_ptr() for u in ue])
    delta = ibk._Delta()
    delta.kind, delta.order = ibk.BSPLINE, 3
    stream = torch.cuda.current_stream().cuda_stream
    ibk.check(ibk.lib().ibk_interpolate_noalloc(
        ctypes.byref(_domain(ibk, w)), ibk.TAG_MAC, w.refinement, delta, precision, n,
        x.data_ptr(), ptrs, got.data_ptr(), stream))
    torch.cuda.synchronize()
    return got.cpu().numpy(), want.cpu().numpy()


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_plan_entry_point_twice(ibk, cuda, precision):
    from ib_cu_b200 import workloads as W
    for w in (W.channel(seed=31), W.single_rbc(seed=32)):
        got, want = _run_both(ibk, w, precision, cuda)
        assert np.all(np.isfinite(got))
        if precision == ibk.FP64:
            assert np.array_equal(got, want)
        else:
            n = w.n
            for c in range(3):
                a, b = got[c * n:(c + 1) * n], want[c * n:(c + 1) * n]
                assert np.abs(a - b).max() <= FP32C_TOL * np.abs(b).max()


def test_noalloc_rejects_oversized_calls(ibk, cuda):
    from ib_cu_b200 import workloads as W
    w = W.channel(seed=33)
    delta = ibk._Delta()
    delta.kind, delta.order = ibk.BSPLINE, 3
    ptrs = (ctypes.c_void_p * 3)(1, 1, 1)
    status = ibk.lib().ibk_interpolate_noalloc(
        ctypes.byref(_domain(ibk, w)), ibk.TAG_MAC, w.refinement, delta, ibk.FP64,
        (1 << 19) + 1, 1, ptrs, 1, None)
    assert status == 5   # IBK_ERR_CAPACITY, raised before any device work
    assert b"524288" in ibk.lib().ibk_last_error()
