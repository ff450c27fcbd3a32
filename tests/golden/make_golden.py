"""Generate tests/golden/golden.npz from the reference itself.

Run from the repository root where the sonwell/ib.cu tree is available:

    python tests/golden/make_golden.py --reference <path of the sonwell/ib.cu tree>

Stencil data (sort keys, stencil origins, fractional offsets, weights, spread
and interpolation node indices) come from ``oracle/_ref/libibref.so``: the
reference's own fd / indexing / delta headers compiled from its tree (see
oracle/ref_bridge.cc).  Operator outputs (spread / interpolate) come from the
plain-C oracle, whose index / weight core is checked against the same
bridge before anything is written.  The fixtures are small (a few hundred
points, 16^3..32^3 grids) so the CPU suite reads them in milliseconds.
"""
import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

DELTAS = [("bspline", 1), ("bspline", 2), ("bspline", 3), ("bspline", 4), ("bspline", 5),
          ("peskin", 0), ("roma", 0), ("cosine", 0), ("hat", 0)]


def edge_points(rng, L, solid, n_random, h):
    """Random points plus the awkward ones: exact grid nodes, half nodes,
    domain edges, -0.0, and (for walls) points on and beyond the walls."""
    dims = len(L)
    pts = [rng.uniform(-0.05 * np.asarray(L), 1.05 * np.asarray(L), size=(n_random, dims))]
    special = []
    for d in range(dims):
        for v in (0.0, -0.0, L[d], L[d] - 1e-17, 3 * h, 3.5 * h, L[d] - 0.5 * h, -h, L[d] + h, -3 * h):
            p = np.asarray(L) * 0.37
            p[d] = v
            special.append(p)
    pts.append(np.asarray(special))
    return np.concatenate(pts, axis=0)


def stencil_case(store, prefix, dims, L, solid, tag, ref, delta, order, x):
    g = O.geometry(dims, L, solid, tag, ref, delta, order)
    for c in range(dims):
        r = O.ref_stencil(g, c, x)
        keys, base, dl, w, sidx, iidx, geo = r
        # the C oracle must agree bit for bit before anything is stored
        b2, d2, w2, s2, i2 = O.stencil(g, c, x)
        k2 = O.sort_keys(g, c, x)
        assert np.array_equal(keys, k2) and np.array_equal(base, b2)
        assert np.array_equal(dl.view(np.uint64), d2.view(np.uint64))
        assert np.array_equal(w, w2) and np.array_equal(sidx, s2) and np.array_equal(iidx, i2)
        store[f"{prefix}/c{c}/keys"] = keys
        store[f"{prefix}/c{c}/base"] = base
        store[f"{prefix}/c{c}/delta"] = dl
        store[f"{prefix}/c{c}/weights"] = w
        store[f"{prefix}/c{c}/sidx"] = sidx
        store[f"{prefix}/c{c}/iidx"] = iidx
        store[f"{prefix}/c{c}/geo"] = geo
    store[f"{prefix}/x"] = x
    store[f"{prefix}/meta"] = np.array([dims, tag, ref, O.DELTA_NAMES[delta], order], np.int64)
    store[f"{prefix}/length"] = np.asarray(L, np.float64)
    store[f"{prefix}/solid"] = np.asarray(solid, np.int64)
    return g


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the sonwell/ib.cu tree")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz"))
    args = ap.parse_args()
    O.build()
    if not O.build_ref(args.reference) or O.ref() is None:
        sys.exit("reference bridge could not be built; fixtures need the reference tree")
    rng = np.random.default_rng(20261203)
    store = {}

    # 1. test/grid.cc: 10 um periodic cube, fd::mac{16}, two points at
    #    (5, 5, 5) um, unit forces, unit face velocities (test/grid.cc:28-57).
    L = [1.0, 1.0, 1.0]
    x = np.full(6, 0.5)
    g = stencil_case(store, "grid_smoke", 3, L, [0, 0, 0], O.TAG_MAC, 16, "bspline", 3, x)
    f = np.ones(6)
    fe, fa = O.spread(g, x, f, with_abs=True)
    ue = [np.ones(int(g.size[c])) for c in range(3)]
    ul, ua = O.interpolate(g, x, ue, with_abs=True)
    store["grid_smoke/f"] = f
    for c in range(3):
        store[f"grid_smoke/fe{c}"] = fe[c]
        store[f"grid_smoke/fe_abs{c}"] = fa[c]
        store[f"grid_smoke/ue{c}"] = ue[c]
    store["grid_smoke/ul"] = ul
    store["grid_smoke/ul_abs"] = ua

    # 2. walled channel 32 x 16 x 32 um at fd::mac{16} (32 x 16 x 32 cells),
    #    random points including ones on / beyond the walls.
    L = [3.2, 1.6, 3.2]
    solid = [0, 1, 0]
    gtmp = O.geometry(3, L, solid, O.TAG_MAC, 16)
    x = edge_points(rng, L, solid, 150, 1.0 / gtmp.resolution)
    x = np.ascontiguousarray(x.T).reshape(-1)
    g = stencil_case(store, "channel", 3, L, solid, O.TAG_MAC, 16, "bspline", 3, x)
    n = x.size // 3
    f = rng.normal(size=3 * n)
    ue = [rng.normal(size=int(g.size[c])) for c in range(3)]
    fe, fa = O.spread(g, x, f, with_abs=True)
    ul, ua = O.interpolate(g, x, ue, with_abs=True)
    store["channel/f"] = f
    for c in range(3):
        store[f"channel/fe{c}"] = fe[c]
        store[f"channel/fe_abs{c}"] = fa[c]
        store[f"channel/ue{c}"] = ue[c]
    store["channel/ul"] = ul
    store["channel/ul_abs"] = ua

    # 3. every delta, 2-D and 3-D, mixed boundaries and both grid tags.
    for dims in (2, 3):
        for i, (delta, order) in enumerate(DELTAS):
            L = [1.6, 0.8, 1.2][:dims]
            solid = [i % 2, (i + 1) % 2, i % 2][:dims]
            tag = O.TAG_MAC if i % 3 else O.TAG_CENTERED
            x = rng.uniform(-0.05, 1.0, size=(40, dims)) * np.asarray(L)
            x = np.ascontiguousarray(x.T).reshape(-1)
            prefix = f"delta_{dims}d_{delta}{order}"
            g = stencil_case(store, prefix, dims, L, solid, tag, 4, delta, order, x)
            nn = x.size // dims
            f = rng.normal(size=dims * nn)
            ue = [rng.normal(size=int(g.size[c])) for c in range(dims)]
            fe, fa = O.spread(g, x, f, with_abs=True)
            ul, ua = O.interpolate(g, x, ue, with_abs=True)
            store[f"{prefix}/f"] = f
            for c in range(dims):
                store[f"{prefix}/fe{c}"] = fe[c]
                store[f"{prefix}/fe_abs{c}"] = fa[c]
                store[f"{prefix}/ue{c}"] = ue[c]
            store[f"{prefix}/ul"] = ul
            store[f"{prefix}/ul_abs"] = ua

    np.savez_compressed(args.out, **store)
    print(f"wrote {args.out}: {len(store)} arrays, {os.path.getsize(args.out) / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
