"""Generate tests/golden/wall_weights.npz: the reference's own ghost-point
wall weights (fd::discretization over Robin walls) for a set of alignments,
resolutions and wall conditions, through the bridge compiled from the
reference tree (oracle/Makefile `ref`).

    python tests/golden/make_wall_weights.py --reference <sonwell/ib.cu tree>
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the sonwell/ib.cu tree")
    args = ap.parse_args()
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    if not O.build_ref(args.reference):
        raise SystemExit("bridge not built")
    walls = [((1.0, 0.0), (1.0, 0.0)), ((0.0, 1.0), (0.0, 1.0)), ((1.0, 0.0), (0.0, 1.0)),
             ((2.0, 0.3), (0.5, 1.5)), ((1.0, 0.25), (3.0, 1.0))]
    cases, out = [], []
    for shift in (0.0, 0.5, 0.25, 0.75):
        for res in (10.0, 37.5, 80.0):
            for lo, up in walls:
                l, u = O.ref_wall_weights(1.6, res, shift, lo, up)
                cases.append([shift, res, lo[0], lo[1], up[0], up[1]])
                out.append(np.concatenate([l, u]))
    np.savez(os.path.join(HERE, "wall_weights.npz"), cases=np.array(cases), weights=np.array(out))
    print(f"{len(cases)} cases written")


if __name__ == "__main__":
    main()
