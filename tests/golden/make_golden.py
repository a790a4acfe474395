"""Writes the golden fixtures of tests/golden/ from the reference's own code.

Run in a container that has the reference sources (it reads the reference's 8-point
sample src/samplepc.txt and runs the reference's check.cpp / grid.cu compiled by
oracle/Makefile). The fixtures it writes are committed; tests never read the reference.

  samplepc.json   the sample cloud parsed as util.cpp:101-135 does (double -> float),
                  rows of the README's two runs (radius r=2 K=50; knn r=10 K=5) from
                  the oracle, each accepted by the reference's sanityCheck*, plus
                  hand-checkable facts.
  ref_grid.json   the reference's calcSearchSize masks on seeded count grids, its
                  MortonCode3 codes and getWidthFromIter widths.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

# the reference checkout: RTNN_REFERENCE_DIR, the same variable oracle/Makefile reads
REF_DIR = os.environ.get("RTNN_REFERENCE_DIR", "/root/reference")
REF_SAMPLE = os.path.join(REF_DIR, "src", "samplepc.txt")


def read_reference_csv(path):
    """One 'x,y,z' line per point, parsed as double then cast to float (util.cpp:123-129)."""
    pts = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line:
                continue
            x, y, z = (float(t) for t in line.split(",")[:3])
            pts.append((x, y, z))
    return np.asarray(pts, dtype=np.float64).astype(np.float32)


def main():
    oracle.build()
    assert oracle.ref_available(), "oracle/_ref not built (reference sources missing?)"
    pts = read_reference_csv(REF_SAMPLE)
    runs = []
    for mode, r, k in (("radius", 2.0, 50), ("knn", 10.0, 5)):
        rows = oracle.bruteforce(pts, None, mode, r, k)
        ok, log = oracle.refcheck(pts, None, rows, mode, r, k)
        assert ok, log
        runs.append({"mode": mode, "radius": r, "k": k, "rows": rows.tolist(),
                     "reference_check": "passed"})
    sample = {"source": "src/samplepc.txt of the reference (8 points)",
              "points": pts.tolist(), "runs": runs}
    with open(os.path.join(HERE, "samplepc.json"), "w") as f:
        json.dump(sample, f, indent=1)

    rng = np.random.Generator(np.random.PCG64(7))
    grids = []
    for case in range(6):
        dz, dy, dx = (int(v) for v in rng.integers(3, 9, size=3))
        lam = float(rng.uniform(0.05, 3.0))
        counts = rng.poisson(lam, size=(dz, dy, dx)).astype(np.uint32)
        knn = int(rng.integers(1, 60))
        cells = []
        for _ in range(12):
            cx, cy, cz = int(rng.integers(0, dx)), int(rng.integers(0, dy)), int(rng.integers(0, dz))
            # cellSize 1, maxWidth 11: the mask is the first shell holding knn + 1
            # points, or 5 when the width (2*iter+2) would exceed 11 first
            mask = oracle.ref_calc_search_size(counts, cx, cy, cz, 1.0, 11.0, knn)
            cells.append({"cell": [cx, cy, cz], "mask": mask})
        grids.append({"counts_zyx": counts.tolist(), "knn": knn, "cell_size": 1.0,
                      "max_width": 11.0, "cells": cells})
    morton = []
    for _ in range(64):
        x, y, z = (int(v) for v in rng.integers(0, 1024, size=3))
        morton.append({"xyz": [x, y, z], "code": oracle.ref_morton3(x, y, z)})
    widths = [{"iter": it, "cell": c, "width": oracle.ref_width_from_iter(it, c)}
              for it in range(5) for c in (0.25, 0.5, 1.0)]
    with open(os.path.join(HERE, "ref_grid.json"), "w") as f:
        json.dump({"calc_search_size": grids, "morton3": morton, "width_from_iter": widths}, f)
    print("wrote", os.path.join(HERE, "samplepc.json"), os.path.join(HERE, "ref_grid.json"))


if __name__ == "__main__":
    main()
