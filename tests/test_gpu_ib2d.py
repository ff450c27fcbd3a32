"""One step of the coupling in a two-dimensional run, as test/ib-platelet1d.cc
composes it: a platelet outline (a closed curve, sheared from its rest
circle) in a periodic 16 um box on a MAC grid of 96 cells per side; its
one-dimensional Skalak tension (ibk_curve_*), the spread onto the grid, one
implicit diffusion step per velocity component, and the interpolation back
to the outline, all on the device through the C ABI.  Checked against laws
that hold whatever the shape: the tension's total force and torque vanish on
the closed curve; the spread conserves force (grid total = point total in a
periodic box); the diffusion step conserves momentum (sum of u = k sum of f on
a periodic grid); spread and interpolation are adjoint (sum_p F_p . U_p =
h^2 sum_j f_j u_j), and the force does positive work."""
import numpy as np
import pytest

import torus as T

pytestmark = pytest.mark.gpu

N = 64                      # samples on the outline (the data sites)
R = 0.18                    # 1.8 um rest radius (internal unit: 10 um)
CENTRE = (0.8, 0.8)
SHEAR = np.array([[1.1, 0.0], [0.0, 1.0 / 1.1]])   # bases::shear of the driver
E_SHEAR, E_BULK = 1e-3, 0.0                           # skalak1d{shear, bulk}


def _outline(A):
    s = T.curve_shape(N, R=R, A=A)
    return (s["position"] + np.array(CENTRE)[:, None]).reshape(-1)


def test_platelet_outline_step(ibk, cuda):
    import torch
    dom = ibk.Domain(ibk.Dimension(1.6), ibk.Dimension(1.6))
    plan = ibk.Plan(ibk.Mac(96), dom, ibk.Bspline(3), ibk.FP64)
    h2 = 1.0 / plan.info.resolution ** 2
    ops = [torch.from_numpy(m).to(cuda) for m in T.curve_operators(N)]
    outline = ibk.CurvePlan(ops, torch.from_numpy(T.curve_weights(N)).to(cuda))
    x0 = torch.from_numpy(_outline(None)).to(cuda)
    x1 = torch.from_numpy(_outline(SHEAR)).to(cuda)
    rest, cur = outline.geometry(x0, 1), outline.geometry(x1, 1)

    # tension of the sheared outline: balanced on the closed curve
    f = ibk.curve_tension(ibk.SKALAK, E_SHEAR, E_BULK, rest, cur)
    x = cur["position"]
    mom = plan.force_moments(N, x, f)
    scale = f.abs().sum().item()
    assert scale > 0
    assert np.abs(mom[:2]).max() <= 1e-11 * scale and abs(mom[5]) <= 1e-11 * scale

    # spread: force conserved on the periodic grid
    fe = [torch.empty(s, dtype=torch.float64, device=cuda) for s in plan.sizes()]
    plan.spread(N, x, f, fe)
    assert np.allclose(plan.grid_totals(fe), mom[:2], rtol=0, atol=1e-13 * scale)

    # one Crank-Nicolson diffusion step per component from rest: momentum k sum f
    dt, mu = 1e-4, 1.0
    u = []
    for c in range(2):
        d = ibk.Diffusion(plan, c, dt, mu, tolerance=1e-13)
        z = torch.zeros_like(fe[c])
        u.append(d.step(z, z, fe[c], gamma=1.0))
        assert d.iterations > 0
        assert abs(u[c].sum().item() - dt * fe[c].sum().item()) <= 1e-9 * dt * fe[c].abs().sum().item()

    # interpolation back to the outline: the adjoint of the spread
    ul = torch.empty(2 * N, dtype=torch.float64, device=cuda)
    plan.interpolate(N, x, u, ul)
    point_power = (f * ul).sum().item()
    grid_power = h2 * sum((fe[c] * u[c]).sum().item() for c in range(2))
    assert point_power > 0
    assert abs(point_power - grid_power) <= 1e-12 * abs(grid_power)
