"""GPU tests of the serving loop (continuous batching of coupled steps).

* Each member's state after its steps is bit-identical whether its requests
  ran packed with other members' requests (a mixed queue served on several
  slots) or one request per launch, alone (FP32C spread sums are exact and
  order-independent; interpolation has no cross-thread sums).
* One served step equals the composition of single-plan operators:
  x1 = x0 + dt * interp(x0), fs = -k (x1 - x0) (the rest shape is the
  admitted shape), fe = spread(x1, fs).
* Admission respects the HBM budget; retiring frees it.
* The Poisson load generator serves every request and reports latencies.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT, K = 1e-3, 1e-3      # internal units: 1 us, 1 pN/um


def _members(seed=11):
    from ib_cu_b200 import workloads as W
    rng = np.random.default_rng(seed)
    shapes = [(32, 2, False), (40, 3, True), (32, 1, False), (48, 2, False), (36, 2, True)]
    return [W.small_instance(rng, side, nc, walls, f"m{i}") for i, (side, nc, walls) in enumerate(shapes)]


def _domain(ibk, w):
    return ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)])


def _velocities(ibk, w, seed):
    from ib_cu_b200 import workloads as W
    plan = ibk.Plan(ibk.Mac(w.refinement), _domain(ibk, w), ibk.Bspline(3), ibk.FP32C)
    ue = W.grid_velocity(w, plan.sizes(), [plan.info.comp_points(c) for c in range(3)],
                         np.random.default_rng(seed))
    return plan, ue


def _server(ibk, ws, ues, slots, budget=150 * 10**9):
    insts = [ibk.Instance(ibk.Mac(w.refinement), _domain(ibk, w)) for w in ws]
    srv = ibk.Server(insts, ibk.Bspline(3), ibk.FP32C, slots=slots, dt=DT, k=K, hbm_budget=budget,
                     max_points=sum(w.n for w in ws))
    for i, (w, ue) in enumerate(zip(ws, ues)):
        srv.admit(i, w.x, ue)
    return srv


def test_member_results_alone_equal_in_the_mix(ibk, cuda):
    ws = _members()
    plans, ues = zip(*[_velocities(ibk, w, 100 + i) for i, w in enumerate(ws)])
    rng = np.random.default_rng(3)
    seq = [int(m) for m in rng.integers(0, len(ws), size=40)]
    counts = [seq.count(i) for i in range(len(ws))]
    mixed = _server(ibk, ws, ues, slots=3)
    for m in seq:                       # one burst: launches pack many members
        mixed.submit(m)
    mixed.drain()
    st = mixed.stats()
    assert st["requests"] == len(seq)
    assert st["launches"] < len(seq)    # requests were packed together
    alone = _server(ibk, ws, ues, slots=1)
    for i, c in enumerate(counts):
        for _ in range(c):
            alone.submit(i)
            alone.drain()               # every launch holds one member
    assert alone.stats()["launches"] == len(seq)
    for i, w in enumerate(ws):
        xa, fa = mixed.read(i, w.n, plans[i].sizes())
        xb, fb = alone.read(i, w.n, plans[i].sizes())
        assert np.array_equal(xa, xb)
        for a, b in zip(fa, fb):
            assert np.array_equal(a, b)
        if counts[i] > 0:
            assert not np.array_equal(xa, w.x)


def test_one_step_equals_plan_composition(ibk, cuda):
    import torch
    ws = _members()[:2]
    plans, ues = zip(*[_velocities(ibk, w, 200 + i) for i, w in enumerate(ws)])
    srv = _server(ibk, ws, ues, slots=2)
    srv.submit(0)
    srv.submit(1)
    srv.drain()
    for i, w in enumerate(ws):
        plan = plans[i]
        x0 = torch.from_numpy(w.x).to(cuda)
        ue = [torch.from_numpy(u).to(cuda) for u in ues[i]]
        U = torch.empty(3 * w.n, dtype=torch.float64, device=cuda)
        plan.interpolate(w.n, x0, ue, U)
        x1 = w.x + DT * U.cpu().numpy()
        fs = (-K) * (x1 - w.x)
        fe = [torch.empty(s, dtype=torch.float64, device=cuda) for s in plan.sizes()]
        plan.spread(w.n, torch.from_numpy(x1).to(cuda), torch.from_numpy(fs).to(cuda), fe)
        xs, fes = srv.read(i, w.n, plan.sizes())
        assert np.array_equal(xs, x1)
        for a, b in zip(fes, fe):
            assert np.array_equal(a, b.cpu().numpy())


def test_admission_respects_the_budget(ibk, cuda):
    ws = _members()[:3]
    plans, ues = zip(*[_velocities(ibk, w, 300 + i) for i, w in enumerate(ws)])

    def state_bytes(w, plan):
        return 4 * 3 * w.n * 8 + 2 * 8 * sum(plan.sizes())

    need = [state_bytes(w, p) for w, p in zip(ws, plans)]
    insts = [ibk.Instance(ibk.Mac(w.refinement), _domain(ibk, w)) for w in ws]
    srv = ibk.Server(insts, ibk.Bspline(3), ibk.FP32C, slots=1, dt=DT, k=K,
                     hbm_budget=need[0] + need[1], max_points=sum(w.n for w in ws))
    srv.admit(0, ws[0].x, ues[0])
    srv.admit(1, ws[1].x, ues[1])
    with pytest.raises(ibk.IbkError) as e:
        srv.admit(2, ws[2].x, ues[2])
    assert e.value.status == 5
    assert srv.stats()["admitted_bytes"] == need[0] + need[1]
    srv.submit(1)
    srv.retire(1)                     # waits for the step in flight
    if need[2] <= need[1]:
        srv.admit(2, ws[2].x, ues[2])
    with pytest.raises(ibk.IbkError):
        srv.submit(1)                 # retired members take no requests


def test_poisson_load_serves_every_request(ibk, cuda):
    ws = _members()
    ues = [_velocities(ibk, w, 400 + i)[1] for i, w in enumerate(ws)]
    srv = _server(ibk, ws, ues, slots=2)
    st = srv.run_poisson(rate=5000.0, requests=200, seed=7)
    assert st["requests"] == 200
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["launches"] >= 1 and st["wall_s"] > 0


def test_checkpoint_restores_a_member(ibk, cuda, tmp_path):
    """A member saved in the linalg::io format and admitted into another
    server continues bit for bit like the original."""
    ws = _members()[:2]
    plans, ues = zip(*[_velocities(ibk, w, 500 + i) for i, w in enumerate(ws)])
    a = _server(ibk, ws, ues, slots=2)
    for _ in range(3):
        a.submit(0)
        a.submit(1)
    a.drain()
    path = str(tmp_path / "member0.bin")
    a.save(0, path)
    objs = ibk.io_read(path)
    assert [o.shape for o in objs[:2]] == [(ws[0].n, 3), (ws[0].n, 3)]
    assert len(objs) == 2 + 2 * 3
    insts = [ibk.Instance(ibk.Mac(w.refinement), _domain(ibk, w)) for w in ws]
    b = ibk.Server(insts, ibk.Bspline(3), ibk.FP32C, slots=1, dt=DT, k=K, max_points=sum(w.n for w in ws))
    b.admit_from(0, path)
    for srv in (a, b):
        srv.submit(0)
        srv.drain()
    xa, fa = a.read(0, ws[0].n, plans[0].sizes())
    xb, fb = b.read(0, ws[0].n, plans[0].sizes())
    assert np.array_equal(xa, xb)
    for u, v in zip(fa, fb):
        assert np.array_equal(u, v)
