"""CPU tests of the oracle: pinned to the reference's own compiled headers
(via the committed golden fixtures, and via oracle/_ref where the reference
tree is present), plus the identities the reference's math implies."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def cases(golden):
    return sorted({k.split("/")[0] for k in golden.files})


def geom_of(O, z, prefix):
    dims, tag, ref, kind, order = (int(v) for v in z[f"{prefix}/meta"])
    L = z[f"{prefix}/length"]
    solid = z[f"{prefix}/solid"]
    return O.geometry(dims, list(L), list(solid), tag, ref, kind, order)


def test_golden_has_cases(golden):
    names = cases(golden)
    assert "grid_smoke" in names and "channel" in names
    assert sum(n.startswith("delta_") for n in names) == 18


def test_oracle_stencils_match_reference_fixtures(oracle, golden):
    """Keys, origins, offsets, weights and node indices: bit-exact with the
    values the reference's headers produced."""
    for prefix in cases(golden):
        g = geom_of(oracle, golden, prefix)
        x = golden[f"{prefix}/x"]
        for c in range(g.dims):
            keys = oracle.sort_keys(g, c, x)
            base, delta, w, sidx, iidx = oracle.stencil(g, c, x)
            geo = golden[f"{prefix}/c{c}/geo"]
            assert geo[0] == g.unit and geo[1] == g.resolution, prefix
            for d in range(g.dims):
                assert geo[2 + 3 * d] == g.cells[c][d]
                assert geo[3 + 3 * d] == g.points[c][d]
                assert geo[4 + 3 * d] == g.shift[c][d]
            assert np.array_equal(keys, golden[f"{prefix}/c{c}/keys"]), prefix
            assert np.array_equal(base, golden[f"{prefix}/c{c}/base"]), prefix
            assert np.array_equal(delta.view(np.uint64), golden[f"{prefix}/c{c}/delta"].view(np.uint64)), prefix
            assert np.array_equal(w.view(np.uint64), golden[f"{prefix}/c{c}/weights"].view(np.uint64)), prefix
            assert np.array_equal(sidx, golden[f"{prefix}/c{c}/sidx"]), prefix
            assert np.array_equal(iidx, golden[f"{prefix}/c{c}/iidx"]), prefix


def test_oracle_operators_match_fixtures(oracle, golden):
    for prefix in cases(golden):
        g = geom_of(oracle, golden, prefix)
        x = golden[f"{prefix}/x"]
        f = golden[f"{prefix}/f"]
        fe, fa = oracle.spread(g, x, f, with_abs=True)
        ue = [golden[f"{prefix}/ue{c}"] for c in range(g.dims)]
        ul, ua = oracle.interpolate(g, x, ue, with_abs=True)
        for c in range(g.dims):
            assert np.array_equal(fe[c], golden[f"{prefix}/fe{c}"]), prefix
            assert np.allclose(fa[c], golden[f"{prefix}/fe_abs{c}"], rtol=1e-14, atol=0)
        assert np.array_equal(ul, golden[f"{prefix}/ul"]), prefix


def test_grid_smoke_known_answer(oracle, golden):
    """test/grid.cc: two coincident points at the centre of a 16^3 periodic
    grid with unit force / unit velocity.  Interpolating a constant field
    gives the partition-of-unity sum; spreading unit forces conserves
    h^3 * sum(fe) = sum(F)."""
    ul = golden["grid_smoke/ul"]
    assert np.allclose(ul, 1.0, rtol=0, atol=1e-15)
    h3 = 1.0 / 16 ** 3
    for c in range(3):
        assert abs(golden[f"grid_smoke/fe{c}"].sum() * h3 - 2.0) < 1e-12


def test_oracle_matches_reference_bridge_random(oracle):
    """Wider random sweep against the reference build (skipped where the
    reference tree is absent, e.g. on the GPU host)."""
    if oracle.ref() is None:
        pytest.skip("reference tree not available here")
    rng = np.random.default_rng(7)
    for dims in (2, 3):
        for solid in ([0, 0, 0], [0, 1, 0], [1, 1, 1]):
            for delta, order in (("bspline", 3), ("peskin", 0), ("roma", 0), ("bspline", 2)):
                L = [3.2, 1.6, 3.2][:dims]
                g = oracle.geometry(dims, L, solid[:dims], oracle.TAG_MAC, 16, delta, order)
                x = np.concatenate([rng.uniform(-0.2, l + 0.2, 500) for l in L])
                for c in range(dims):
                    keys, base, dl, w, sidx, iidx, _ = oracle.ref_stencil(g, c, x)
                    b2, d2, w2, s2, i2 = oracle.stencil(g, c, x)
                    assert np.array_equal(keys, oracle.sort_keys(g, c, x))
                    assert np.array_equal(base, b2) and np.array_equal(sidx, s2) and np.array_equal(iidx, i2)
                    assert np.array_equal(dl.view(np.uint64), d2.view(np.uint64))
                    assert np.array_equal(w.view(np.uint64), w2.view(np.uint64))


def test_channel_geometry(oracle):
    """Channel 32x16x32 um with walls in y at fd::mac{64}: MAC component
    sizes u 128x64x128, v 128x63x128, w 128x64x128, 40 points per unit."""
    g = oracle.geometry(3, [3.2, 1.6, 3.2], [0, 1, 0], oracle.TAG_MAC, 64)
    assert g.resolution == 40.0
    assert [g.comp_points(c) for c in range(3)] == [[128, 64, 128], [128, 63, 128], [128, 64, 128]]
    assert [[g.shift[c][d] for d in range(3)] for c in range(3)] == [
        [0.0, 0.5, 0.5], [0.5, 1.0, 0.5], [0.5, 0.5, 0.0]]
    assert (g.per_sweep, g.sweeps) == (8, 8)


def _random_periodic(oracle, rng, n=400, delta="bspline", order=3):
    g = oracle.geometry(3, [1.6, 1.6, 1.6], [0, 0, 0], oracle.TAG_MAC, 16, delta, order)
    x = rng.uniform(0, 1.6, 3 * n)
    return g, x


def test_partition_of_unity(oracle):
    rng = np.random.default_rng(1)
    for delta, order in (("bspline", 3), ("peskin", 0), ("roma", 0), ("cosine", 0), ("hat", 0), ("bspline", 5)):
        g, x = _random_periodic(oracle, rng, 200, delta, order)
        for c in range(3):
            _, _, w, _, _ = oracle.stencil(g, c, x)
            assert np.allclose(w.sum(axis=1), 1.0, atol=5e-15), delta


def test_force_conservation_periodic(oracle):
    rng = np.random.default_rng(2)
    g, x = _random_periodic(oracle, rng)
    f = rng.normal(size=x.size)
    fe = oracle.spread(g, x, f)
    h3 = 1.0 / g.resolution ** 3
    n = x.size // 3
    for c in range(3):
        assert abs(fe[c].sum() * h3 - f[c * n:(c + 1) * n].sum()) < 1e-11


def test_adjointness_periodic(oracle):
    """h^3 <spread(F), u> = <F, interp(u)> on a periodic domain."""
    rng = np.random.default_rng(3)
    g, x = _random_periodic(oracle, rng)
    f = rng.normal(size=x.size)
    ue = [rng.normal(size=int(g.size[c])) for c in range(3)]
    fe = oracle.spread(g, x, f)
    ul = oracle.interpolate(g, x, ue)
    lhs = sum(float(fe[c] @ ue[c]) for c in range(3)) / g.resolution ** 3
    rhs = float(f @ ul)
    assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(rhs))


def test_translation_by_one_cell_permutes(oracle):
    rng = np.random.default_rng(4)
    g, x = _random_periodic(oracle, rng, 100)
    f = rng.normal(size=x.size)
    h = 1.0 / g.resolution
    n = x.size // 3
    x2 = x.copy()
    x2[:n] += h          # shift every point by one cell along x
    fe = oracle.spread(g, x, f)
    fe2 = oracle.spread(g, x2, f)
    for c in range(3):
        p = g.comp_shape(c)
        a = fe[c].reshape(p)
        b = fe2[c].reshape(p)
        assert np.allclose(np.roll(a, 1, axis=2), b, rtol=1e-9, atol=1e-9 * np.abs(a).max())


def test_spread_overwrites(oracle):
    rng = np.random.default_rng(5)
    g, x = _random_periodic(oracle, rng, 50)
    f = rng.normal(size=x.size)
    fe = oracle.spread(g, x, f)
    pre = [np.full(int(g.size[c]), 123.0) for c in range(3)]
    fe2 = oracle.spread(g, x, f, fe=pre)
    for c in range(3):
        assert np.array_equal(fe[c], fe2[c])


def test_walls_drop_in_spread_clamp_in_interp(oracle):
    """Near a wall, spread drops out-of-range stencil nodes (errors_negative)
    while interpolate clamps them (indexing::clamped)."""
    g = oracle.geometry(3, [3.2, 1.6, 3.2], [0, 1, 0], oracle.TAG_MAC, 64)
    x = np.array([1.0, 0.02, 1.0])  # y = 0.2 um above the lower wall
    for c in range(3):
        _, _, w, sidx, iidx = oracle.stencil(g, c, x)
        assert (iidx >= 0).all()
    # survey probe: u drops 16 and v drops 32 of 64 nodes at y = 0.2 um
    _, _, _, su, _ = oracle.stencil(g, 0, x)
    _, _, _, sv, _ = oracle.stencil(g, 1, x)
    assert (su < 0).sum() == 16 and (sv < 0).sum() == 32


def test_multithreaded_oracle_matches_serial(oracle):
    rng = np.random.default_rng(6)
    g = oracle.geometry(3, [3.2, 1.6, 3.2], [0, 1, 0], oracle.TAG_MAC, 16)
    n = 3000
    x = np.concatenate([rng.uniform(0, l, n) for l in (3.2, 1.6, 3.2)])
    f = rng.normal(size=3 * n)
    ue = [rng.normal(size=int(g.size[c])) for c in range(3)]
    fe, fa = oracle.spread(g, x, f, with_abs=True)
    fe2 = oracle.spread(g, x, f, threads=4)
    for c in range(3):
        assert np.all(np.abs(fe[c] - fe2[c]) <= 1e-13 * fa[c] + 1e-300)
    ul = oracle.interpolate(g, x, ue)
    ul2 = oracle.interpolate(g, x, ue, threads=4)
    assert np.array_equal(ul, ul2)
