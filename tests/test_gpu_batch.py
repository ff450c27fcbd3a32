"""GPU tests of batches (many grids per launch, persistent kernels) through
the C ABI, against single plans on the same inputs.

A batch instance must behave exactly like a plan of its own:
  * FP32C spread: bit-identical (the fixed-point sum is exact and
    order-independent, and the tiles are the same);
  * interpolation (both precisions): bit-identical (no cross-thread sums);
  * FP64 spread: equal up to summation order, |err| <= 1e-12 * max|fe|.
After autotuning, tile shapes may differ from the plan's, so FP32C results
are then held to the FP32C bar against the FP64 plan (normwise 1e-5).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP32C_TOL = 1e-5
FP64_SPREAD_TOL = 1e-12


def _instances(seed=5):
    from ib_cu_b200 import workloads as W
    rng = np.random.default_rng(seed)
    shapes = [(32, 3, False), (48, 2, False), (40, 4, True), (32, 1, False), (64, 5, False), (36, 2, True)]
    return [W.small_instance(rng, side, nc, walls, f"inst{i}") for i, (side, nc, walls) in enumerate(shapes)]


def _domain(ibk, w):
    return ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)])


def _dev(a, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


class Case:
    """Device arrays of one instance plus a plan for it."""

    def __init__(self, ibk, w, precision, device, seed):
        import torch
        from ib_cu_b200 import workloads as W
        self.w = w
        self.n = w.n
        self.plan = ibk.Plan(ibk.Mac(w.refinement), _domain(ibk, w), ibk.Bspline(3), precision)
        self.sizes = self.plan.sizes()
        rng = np.random.default_rng(seed)
        ue = W.grid_velocity(w, self.sizes, [self.plan.info.comp_points(c) for c in range(3)], rng)
        self.x = _dev(w.x, device)
        self.f = _dev(w.f, device)
        self.ue = [_dev(u, device) for u in ue]
        self.fe = [torch.full((s,), np.nan, dtype=torch.float64, device=device) for s in self.sizes]
        self.ul = torch.full((3 * self.n,), np.nan, dtype=torch.float64, device=device)
        xref = w.x + rng.normal(size=w.x.size) * 0.01 * w.lengths[0] / w.refinement
        self.xref = _dev(xref, device)
        self.xn = torch.full((3 * self.n,), np.nan, dtype=torch.float64, device=device)
        self.fs = torch.full((3 * self.n,), np.nan, dtype=torch.float64, device=device)

    def io(self, active=True):
        return {"n": self.n if active else 0, "x": self.x, "fl": self.f, "fe": self.fe, "ue": self.ue,
                "ul": self.ul, "xn": self.xn, "xref": self.xref, "fs": self.fs}

    def plan_spread(self, x=None, f=None):
        import torch
        fe = [torch.full((s,), np.nan, dtype=torch.float64, device=self.x.device) for s in self.sizes]
        self.plan.spread(self.n, self.x if x is None else x, self.f if f is None else f, fe)
        return [a.cpu().numpy() for a in fe]

    def plan_interp(self):
        import torch
        ul = torch.full((3 * self.n,), np.nan, dtype=torch.float64, device=self.x.device)
        self.plan.interpolate(self.n, self.x, self.ue, ul)
        return ul.cpu().numpy()


def _make(ibk, precision, device, seed=5, capacity_extra=0):
    ws = _instances(seed)
    cases = [Case(ibk, w, precision, device, seed + i) for i, w in enumerate(ws)]
    insts = [ibk.Instance(ibk.Mac(w.refinement), _domain(ibk, w)) for w in ws]
    cap = sum(c.n for c in cases) + capacity_extra
    batch = ibk.Batch(insts, ibk.Bspline(3), precision, max_points=cap)
    return batch, cases


def _check_spread(got, want, precision):
    for g, w in zip(got, want):
        assert np.all(np.isfinite(g))
        if precision == 1:
            assert np.array_equal(g, w)
        else:
            assert np.abs(g - w).max() <= FP64_SPREAD_TOL * max(np.abs(w).max(), 1e-300)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_single_plans(ibk, cuda, precision):
    import torch
    batch, cases = _make(ibk, precision, cuda)
    batch.bind([c.io() for c in cases])
    batch.run(ibk.OP_SPREAD)
    batch.run(ibk.OP_INTERPOLATE)
    torch.cuda.synchronize()
    batch.check()
    for c in cases:
        _check_spread([a.cpu().numpy() for a in c.fe], c.plan_spread(), precision)
        assert np.array_equal(c.ul.cpu().numpy(), c.plan_interp())


def test_idle_instance_is_untouched(ibk, cuda):
    import torch
    batch, cases = _make(ibk, 1, cuda)
    idle = 2
    batch.bind([c.io(active=(i != idle)) for i, c in enumerate(cases)])
    batch.run(ibk.OP_SPREAD)
    batch.run(ibk.OP_INTERPOLATE)
    torch.cuda.synchronize()
    assert all(torch.isnan(a).all().item() for a in cases[idle].fe)
    assert torch.isnan(cases[idle].ul).all().item()
    for i, c in enumerate(cases):
        if i != idle:
            _check_spread([a.cpu().numpy() for a in c.fe], c.plan_spread(), 1)


def test_graph_replay_with_new_bindings(ibk, cuda):
    """A captured graph reads the arrays bound at replay time."""
    import torch
    batch, cases = _make(ibk, 1, cuda)
    batch.bind([c.io() for c in cases])
    batch.capture(ibk.OP_SPREAD)
    batch.capture(ibk.OP_INTERPOLATE)
    before = batch.launch_count()
    batch.run(ibk.OP_SPREAD)
    batch.run(ibk.OP_INTERPOLATE)
    torch.cuda.synchronize()
    # four binning kernels per operator; FP32C spread: the one-pass and the
    # folded (dense tiles) kernel; interpolation: one kernel
    assert batch.launch_count() == before + (4 + 2) + (4 + 1)
    for c in cases:
        _check_spread([a.cpu().numpy() for a in c.fe], c.plan_spread(), 1)
        assert np.array_equal(c.ul.cpu().numpy(), c.plan_interp())
    # second binding: other point sets (halved counts, every other instance idle)
    for i, c in enumerate(cases):
        c.n = c.n // 2 if i % 2 == 0 else c.n
        for a in c.fe:
            a.fill_(np.nan)
        c.ul.fill_(np.nan)
        c.x = c.x.clone()
        c.x[: 3 * c.n].copy_(torch.cat([c.x[d * c.w.n: d * c.w.n + c.n] for d in range(3)]))
        c.f = c.f.clone()
        c.f[: 3 * c.n].copy_(torch.cat([c.f[d * c.w.n: d * c.w.n + c.n] for d in range(3)]))
    batch.bind([c.io(active=(i != 1)) for i, c in enumerate(cases)])
    batch.run(ibk.OP_SPREAD)
    batch.run(ibk.OP_INTERPOLATE)
    torch.cuda.synchronize()
    for i, c in enumerate(cases):
        if i == 1:
            continue
        _check_spread([a.cpu().numpy() for a in c.fe], c.plan_spread(), 1)
        got = c.ul.cpu().numpy()[: 3 * c.n]
        assert np.array_equal(got, c.plan_interp()[: 3 * c.n])


@pytest.mark.parametrize("precision", [0, 1])
def test_step_matches_composition(ibk, cuda, precision):
    """OP_STEP == interpolate, x + dt U, -k (xn - xref), spread(xn, fs)."""
    import torch
    batch, cases = _make(ibk, precision, cuda)
    dt, k = 1e-3, 1e-3             # internal units: 1 us, 1 pN/um
    batch.set_step(dt, k)
    batch.bind([c.io() for c in cases])
    batch.run(ibk.OP_STEP)
    torch.cuda.synchronize()
    batch.check()
    for c in cases:
        U = c.plan_interp()
        assert np.array_equal(c.ul.cpu().numpy(), U)
        x = c.w.x
        xn = x + dt * U                      # separate roundings, as the kernel
        xref = c.xref.cpu().numpy()
        fs = (-k) * (xn - xref)
        assert np.array_equal(c.xn.cpu().numpy(), xn)
        assert np.array_equal(c.fs.cpu().numpy(), fs)
        want = c.plan_spread(_dev(xn, cuda), _dev(fs, cuda))
        _check_spread([a.cpu().numpy() for a in c.fe], want, precision)


def test_member_alone_and_in_the_mix(ibk, cuda):
    """Each instance's step result is identical whether it runs alone or with
    every other instance (FP32C: exact fixed-point sums, no order effects)."""
    import torch
    batch, cases = _make(ibk, 1, cuda)
    batch.set_step(1e-3, 1e-3)
    batch.bind([c.io() for c in cases])
    batch.capture(ibk.OP_STEP)
    batch.run(ibk.OP_STEP)
    torch.cuda.synchronize()
    mixed = [([a.cpu().numpy() for a in c.fe], c.xn.cpu().numpy(), c.fs.cpu().numpy()) for c in cases]
    for i, c in enumerate(cases):
        for a in c.fe:
            a.fill_(np.nan)
        c.xn.fill_(np.nan)
        batch.bind([cc.io(active=(j == i)) for j, cc in enumerate(cases)])
        batch.run(ibk.OP_STEP)
        torch.cuda.synchronize()
        fe, xn, fs = mixed[i]
        for g, w in zip(c.fe, fe):
            assert np.array_equal(g.cpu().numpy(), w)
        assert np.array_equal(c.xn.cpu().numpy(), xn)
        assert np.array_equal(c.fs.cpu().numpy(), fs)


def test_tune_keeps_results_within_fp32c_bar(ibk, cuda):
    import torch
    batch, cases = _make(ibk, 1, cuda)
    batch.bind([c.io() for c in cases])
    cfg = batch.tune(ibk.OP_SPREAD)
    assert cfg == batch.config()
    cfg_i = batch.tune(ibk.OP_INTERPOLATE)
    assert cfg_i == batch.config()
    for c in cases:
        for a in c.fe:
            a.fill_(np.nan)
    batch.run(ibk.OP_SPREAD)
    batch.run(ibk.OP_INTERPOLATE)
    torch.cuda.synchronize()
    for c in cases:
        p64 = ibk.Plan(ibk.Mac(c.w.refinement), _domain(ibk, c.w), ibk.Bspline(3), ibk.FP64)
        ref = [torch.empty(s, dtype=torch.float64, device=cuda) for s in c.sizes]
        p64.spread(c.n, c.x, c.f, ref)
        for g, w in zip(c.fe, ref):
            g, w = g.cpu().numpy(), w.cpu().numpy()
            assert np.abs(g - w).max() <= FP32C_TOL * np.abs(w).max()
        u64 = torch.empty(3 * c.n, dtype=torch.float64, device=cuda)
        p64.interpolate(c.n, c.x, c.ue, u64)
        got, want = c.ul.cpu().numpy(), u64.cpu().numpy()
        for comp in range(3):
            a, b = got[comp * c.n:(comp + 1) * c.n], want[comp * c.n:(comp + 1) * c.n]
            assert np.abs(a - b).max() <= FP32C_TOL * np.abs(b).max()


def test_spread_threads_per_cta_keep_the_result(ibk, cuda):
    """512 threads per FP32C spread CTA sum the same exact fixed-point terms as
    256: the grids are identical bit for bit."""
    import torch
    batch, cases = _make(ibk, 1, cuda)
    batch.bind([c.io() for c in cases])
    out = []
    for threads in (256, 512):
        batch.configure(spread_threads=threads)
        assert batch.config()["spread_threads"] == threads
        for c in cases:
            for a in c.fe:
                a.fill_(np.nan)
        batch.run(ibk.OP_SPREAD)
        torch.cuda.synchronize()
        out.append([a.cpu().numpy().copy() for c in cases for a in c.fe])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
    with pytest.raises(ibk.IbkError):
        batch.configure(spread_threads=384)


def test_bind_beyond_capacity_is_rejected(ibk, cuda):
    batch, cases = _make(ibk, 1, cuda, capacity_extra=-1)
    with pytest.raises(ibk.IbkError) as e:
        batch.bind([c.io() for c in cases])
    assert e.value.status == 5


def test_ensemble_instances_against_oracle(ibk, oracle, cuda):
    """Eight instances of the 256-instance ensemble (cube grids from 32^3 to
    128^3, dense and sparse) in one batch against the oracle: FP64
    interpolation bit for bit and spread within 1e-12 * sum |res w F| per face
    (the oracle's spread of |F|: bspline<3> weights are non-negative); FP32C
    to the normwise bar."""
    import torch
    from ib_cu_b200 import workloads as W
    every = W.ensemble(seed=0, count=256)
    sides = [int(round(w.lengths[0] / 0.025)) for w in every]
    pick = []
    for side in (32, 48, 64, 96, 128):
        pick += [i for i, s in enumerate(sides) if s == side][:2 if side in (32, 64, 128) else 1]
    ws = [every[i] for i in pick]
    insts = [ibk.Instance(ibk.Mac(w.refinement), _domain(ibk, w)) for w in ws]
    total = sum(w.n for w in ws)
    for precision in (ibk.FP64, ibk.FP32C):
        batch = ibk.Batch(insts, ibk.Bspline(3), precision, max_points=total)
        rng = np.random.default_rng(3)
        io, ue_h = [], []
        for i, w in enumerate(ws):
            sizes = batch.sizes(i)
            ue_h.append([rng.normal(size=s) for s in sizes])
            io.append({"n": w.n, "x": _dev(w.x, cuda), "fl": _dev(w.f, cuda),
                       "fe": [torch.full((s,), np.nan, dtype=torch.float64, device=cuda) for s in sizes],
                       "ue": [_dev(u, cuda) for u in ue_h[-1]],
                       "ul": torch.full((3 * w.n,), np.nan, dtype=torch.float64, device=cuda)})
        batch.bind(io)
        batch.run(ibk.OP_SPREAD_INTERPOLATE)
        torch.cuda.synchronize()
        for i, w in enumerate(ws):
            g = oracle.geometry(3, w.lengths, w.boundaries, oracle.TAG_MAC, w.refinement)
            want_fe = oracle.spread(g, w.x, w.f, threads=oracle.max_threads())
            want_ul = oracle.interpolate(g, w.x, ue_h[i], threads=oracle.max_threads())
            got_ul = io[i]["ul"].cpu().numpy()
            if precision == ibk.FP64:
                absum = oracle.spread(g, w.x, np.abs(w.f), threads=oracle.max_threads())
                assert np.array_equal(got_ul, want_ul), i
                for c in range(3):
                    err = np.abs(io[i]["fe"][c].cpu().numpy() - want_fe[c])
                    assert np.all(err <= 1e-12 * absum[c] + 1e-300), (i, c)
            else:
                for c in range(3):
                    got = io[i]["fe"][c].cpu().numpy()
                    assert np.abs(got - want_fe[c]).max() <= FP32C_TOL * np.abs(want_fe[c]).max(), (i, c)
                    n = w.n
                    ref = want_ul[c * n:(c + 1) * n]
                    assert np.abs(got_ul[c * n:(c + 1) * n] - ref).max() <= FP32C_TOL * np.abs(ref).max(), (i, c)
        del batch, io
