"""The GPU restatement of the reference's algorithm (baseline/ref_gpu, used
only to time the reference's own scheme on the same B200) agrees with the
library's FP64 path: spread to summation order (1e-12 of max|fe|),
interpolation bit for bit."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_algorithm_restatement_agrees(ibk, cuda):
    import subprocess
    import sys
    import torch
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "baseline", "ref_gpu")], check=True)
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    from ib_cu_b200 import workloads as W
    w = W.channel(seed=21)
    dom = ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)])
    plan = ibk.Plan(ibk.Mac(w.refinement), dom, ibk.Bspline(3), ibk.FP64)
    sizes = plan.sizes()
    x = torch.from_numpy(w.x).to(cuda)
    f = torch.from_numpy(w.f).to(cuda)
    gen = torch.Generator(device=cuda)
    gen.manual_seed(4)
    ue = [torch.randn(s, generator=gen, dtype=torch.float64, device=cuda) for s in sizes]
    r = bench.run_reference_gpu(ibk, w, plan.info, x, f, ue, steps=1)
    assert r is not None
    fe = [torch.empty(s, dtype=torch.float64, device=cuda) for s in sizes]
    plan.spread(w.n, x, f, fe)
    ul = torch.empty(3 * w.n, dtype=torch.float64, device=cuda)
    plan.interpolate(w.n, x, ue, ul)
    torch.cuda.synchronize()
    for a, b in zip(r["fe"], fe):
        assert float((a - b).abs().max()) <= 1e-12 * float(b.abs().max())
    assert torch.equal(r["ul"], ul)
