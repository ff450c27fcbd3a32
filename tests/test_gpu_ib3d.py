"""One step of the coupling in three dimensions, as test/ib-whole.cc composes
it for red cells: deformed, moving cells (tori with exact Fourier operators)
in a periodic 16 um box on a MAC grid of 64 cells per side; their red-cell
forces (Skalak tension, bending and dissipation, summed as forces::combine
does), the spread onto the grid (FP64 and FP32C), one implicit diffusion step
per velocity component (the reference's Chebyshev-preconditioned solve) and
the interpolation back, all on the device through the C ABI.  Checked
against laws that hold whatever the shape: balanced forces per cell; force
conserved by the spread; momentum k sum f kept by the diffusion step; spread
and interpolation adjoint (sum_p F . U = h^3 sum_j f . u, to rounding in
FP64 and within the FP32C contract of 1e-5)."""
import numpy as np
import pytest

import torus as T

pytestmark = pytest.mark.gpu

NU, NV, NC = 48, 24, 2
MATS = [np.array([[1.15, 0.1, 0.0], [0.0, 0.9, 0.05], [0.02, 0.0, 1.05]]), np.diag([0.95, 1.1, 1.0])]
CENTRES = [(0.5, 0.8, 0.8), (1.1, 0.8, 0.85)]


def _cells(scale, deformed):
    shapes = []
    for c in range(NC):
        s = T.shape(NU, NV, R=2.0, r=0.7, A=MATS[c] if deformed else None, eps=0.03 * (c + 1) if deformed else 0.0)
        shapes.append({k: s[k] * scale for k in T.KEYS})
    x = T.pack(shapes)["position"].reshape(3, NC, -1)
    for c in range(NC):
        x[:, c] += np.array(CENTRES[c])[:, None]
    return x.reshape(-1)


def test_red_cells_step(ibk, cuda):
    import torch
    scale = 0.1                          # torus R = 0.2 (2 um), r = 0.07
    w = torch.from_numpy(T.weights(NU, NV)).to(cuda)
    ops = [torch.from_numpy(m).to(cuda) for m in T.operators(NU, NV)]
    data_plan = ibk.SurfacePlan([None] + ops[1:], w)
    sample_plan = ibk.SurfacePlan(ops, w)
    x0 = torch.from_numpy(_cells(scale, False)).to(cuda)
    x1 = torch.from_numpy(_cells(scale, True)).to(cuda)
    rest, cur = sample_plan.geometry(x0, NC), sample_plan.geometry(x1, NC)
    u, v = T.grid(NU, NV)
    vel = np.stack([np.stack([0.1 * np.sin(u + c) * np.cos(v), 0.05 * np.cos(2 * u), 0.1 * np.sin(u - 2 * v)])
                    for c in range(NC)], axis=1).reshape(-1)
    U = torch.from_numpy(vel).to(cuda)
    f = (ibk.membrane_tension(ibk.SKALAK, 2.5e-3, 2.5e-1, rest, cur)
         + ibk.membrane_bending(data_plan, sample_plan, 2e-4, False, x0, x1, rest, cur, NC)) \
        + ibk.membrane_dissipation(sample_plan, 2.5e-3, U, cur, NC)
    n = NU * NV * NC
    x = cur["position"]

    dom = ibk.Domain(ibk.Dimension(1.6), ibk.Dimension(1.6), ibk.Dimension(1.6))
    dt, mu = 1e-4, 1.0
    for precision, tol in ((ibk.FP64, 1e-12), (ibk.FP32C, 1e-5)):
        plan = ibk.Plan(ibk.Mac(64), dom, ibk.Bspline(3), precision)
        h3 = 1.0 / plan.info.resolution ** 3
        mom = plan.force_moments(n, x, f)
        scale_f = f.abs().sum().item()
        # per-cell balance to the grid's accuracy; the pair's total too
        assert np.abs(mom[:3]).max() <= 1e-5 * scale_f
        fe = [torch.empty(s, dtype=torch.float64, device=cuda) for s in plan.sizes()]
        plan.spread(n, x, f, fe)
        totals = plan.grid_totals(fe)
        assert np.abs(totals - mom[:3]).max() <= tol * scale_f
        ue = []
        for c in range(3):
            d = ibk.Diffusion(plan, c, dt, mu, tolerance=1e-13)
            z = torch.zeros_like(fe[c])
            ue.append(d.step(z, z, fe[c], gamma=1.0))
            assert d.iterations > 0
            assert abs(ue[c].sum().item() - dt * fe[c].sum().item()) <= 1e-9 * dt * fe[c].abs().sum().item()
        ul = torch.empty(3 * n, dtype=torch.float64, device=cuda)
        plan.interpolate(n, x, ue, ul)
        point_power = (f * ul).sum().item()
        grid_power = h3 * sum((fe[c] * ue[c]).sum().item() for c in range(3))
        assert grid_power > 0
        assert abs(point_power - grid_power) <= tol * abs(grid_power)
        plan.close()
