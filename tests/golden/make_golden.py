#!/usr/bin/env python3
"""Generate the golden vectors of the grid-search parity tests from the REFERENCE itself.

Run where the reference checkout exists, naming it in CGS_REFERENCE_DIR:

    CGS_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py

The reference has no tests and no golden vectors; its only fixtures are the 6x6 images of
its examples (src/gpu/cudaGridSearch_example1.cu:51-71, repeated in cudaGridSearch_main.cu
and _main_mi.cu).  This script reads those arrays from the example source as text, builds
the examples' grids (example 1: 2-D translation, example 2: by-reference translation SAD,
example 3: raw-homography SAD with four collapsed axes), adds small synthetic pairs for
every 8-parameter reference functor, and evaluates every case with the reference's own
functor source built for the host (oracle/_ref/libcgs_ref.so, oracle/ref_harness.cu).
Outputs (costs, lowest-index argmin over the whole grid) go to tests/golden/*.npz with an
index in tests/golden/manifest.json.  Large grids store every k-th cost (stride) plus the
argmin of the full grid.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from cugridsearch_b200 import synthetic as S  # noqa: E402

REF = os.environ.get("CGS_REFERENCE_DIR", "")
if not REF:
    sys.exit("set CGS_REFERENCE_DIR to the reference checkout")


def example_images() -> dict[str, np.ndarray]:
    """imageA/B/C_data of the reference's example 1, parsed from its source text."""
    src = open(os.path.join(REF, "src", "gpu", "cudaGridSearch_example1.cu")).read()
    out = {}
    for name in ("imageA_data", "imageB_data", "imageC_data"):
        m = re.search(name + r"\s*\[\s*6\s*\*\s*6\s*\]\s*=\s*\{([^}]*)\}", src)
        vals = [float(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()]
        assert len(vals) == 36, name
        out[name[5]] = np.array(vals, dtype=np.float64).reshape(6, 6)  # pixel_precision = double
    return out


def run_case(name, mov, fix, cost, start, end, count, stride=1):
    M, F = O.Image(mov), O.Image(fix)
    g = O.make_grid(start, end, count)
    n = O.grid_num(g)
    full = O.ref_search(cost, g, M, F)
    fin = np.where(np.isfinite(full), full, np.inf)
    argmin = int(np.argmin(fin)) if np.isfinite(fin).any() else -1
    idx = np.arange(0, n, stride, dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), moving=M.arr, fixed=F.arr, indices=idx,
                        costs=full[idx].astype(np.float32), argmin=np.int64(argmin),
                        argmin_cost=np.float32(full[argmin] if argmin >= 0 else np.inf))
    return {"name": name, "cost": cost, "start": [float(v) for v in start], "end": [float(v) for v in end],
            "count": [float(v) for v in count], "grid_points": n, "stride": stride, "argmin": argmin,
            "pixel": str(M.arr.dtype), "moving_shape": list(M.arr.shape), "fixed_shape": list(F.arr.shape)}


def main():
    if not O.have_ref():
        sys.exit("the reference harness (oracle/_ref) is not available: run where the reference exists")
    imgs = example_images()
    A, B, Cc = imgs["A"], imgs["B"], imgs["C"]
    cases = []
    # example 1 (cudaGridSearch_example1.cu:97-100): A vs A, 1000 x 1000 translations over [-3, 3]^2
    cases.append(run_case("ex1_A_A_translation_sad", A, A, "SAD_SUM_T", [-3, -3], [3, 3], [1000, 1000], 97))
    # example 2 (cudaGridSearch_example2.cu:89-99, by-reference SAD): A vs C, 103 x 111 translations
    cases.append(run_case("ex2_A_C_translation_sad_byref", A, Cc, "SAD_SUM_T_REF", [-3, -3], [3, 3], [103, 111]))
    cases.append(run_case("ex2_B_C_translation_sad", B, Cc, "SAD_SUM_T", [-3, -3], [3, 3], [103, 111]))
    # example 3 (cudaGridSearch_example3.cu:90-104): raw H, axes 0,1,3,4 collapse to one sample
    cases.append(run_case("ex3_A_A_raw_h_sad", A, A, "SAD_AVG_H", [1, 0, -3, 0, 1, -3, 0, 0],
                          [1, 0, 3, 0, 1, 3, .1, .1], [10, 10, 100, 10, 10, 100, 10, 10], 97))
    # the 6x6 fixtures under the 8-parameter functors (values 0/1 scaled to 0/255)
    for cost in ("SAD_AVG", "SQD_REF", "NCC_REF", "SQD_ALT", "NCC_ALT", "MI_ALT"):
        lo = [-0.2, 0.8, 0.8, -0.1, -2, -2, -1e-3, -1e-3]
        hi = [0.2, 1.2, 1.2, 0.1, 2, 2, 1e-3, 1e-3]
        cases.append(run_case(f"ex_A_B_{cost.lower()}", 255 * B, 255 * A, cost, lo, hi, [3] * 8))
    # synthetic pairs: every 8-parameter functor, f32 / u8 / f64, 1 and 3 channels, ragged sizes
    for k, cost in enumerate(("SAD_AVG", "SQD_REF", "NCC_REF", "SQD_ALT", "NCC_ALT", "MI_ALT")):
        for j, (u8, ch, size, msize) in enumerate([(False, 1, 20, 17), (True, 1, 24, 24), (False, 3, 16, 19)]):
            p = S.small_pair(1000 + 10 * k + j, size=size, count=3, cost=cost, u8=u8, channels=ch, msize=msize)
            if cost == "MI_ALT":  # normalised parametrisation: translations in fractions of the image
                p.lo[4:6], p.hi[4:6] = -0.15, 0.15
            mov, fix = p.moving, p.fixed
            if j == 0 and cost in ("NCC_REF", "SAD_AVG"):
                mov, fix = mov.astype(np.float64), fix.astype(np.float64)
            cases.append(run_case(f"syn_{cost.lower()}_{j}", mov, fix, cost, list(p.lo), list(p.hi), list(p.count)))
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump({"generator": "tests/golden/make_golden.py", "reference_functors": "oracle/ref_harness.cu",
                   "cases": cases}, fh, indent=1)
    print(f"{len(cases)} golden cases written to {HERE}")


if __name__ == "__main__":
    main()
