"""Test infrastructure: times the reference's OWN GPU search on this GPU -- CudaGridSearcher::
search_by_value with calcNCC (the NCC single-pair configuration, 256x256 float, 6^8 grid) and
calcMIAlt (the MI configuration's images, 512x512 uint8, 5^8 grid) -- compiled unchanged for
sm_100a in oracle/_ref, and prints one JSON line per case.  The numbers are a reported
baseline, next to the reference's CPU path and this library's kernels.

Buffers are padded as the reference's kernel needs: its result write at index n (bound check
'>') and its bilinear taps one row past an image stay inside the allocations.

Usage (on a GPU box): python oracle/time_reference_gpu.py [--mi]
"""
import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    import torch
    import oracle as O
    from cugridsearch_b200 import synthetic as S
    ap = argparse.ArgumentParser()
    ap.add_argument("--mi", action="store_true", help="also time calcMIAlt on the MI configuration")
    a = ap.parse_args()
    if not O.have_ref():
        print(json.dumps({"impl": "reference-gpu", "unavailable": "reference harness not built"}))
        return 0
    L = O.ref()
    L.cgsref_gpu_search.restype = C.c_int
    L.cgsref_gpu_search.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                    C.POINTER(C.c_float)]
    dev = torch.device("cuda")
    cases = [("NCC_REF", 5, S.config1())]
    if a.mi:
        cases.append(("MI_ALT", 8, S.config2()))
    for name, code, pair in cases:
        def padded(img):
            h, w = img.shape[:2]
            t = torch.zeros((h + 1) * w + 1, dtype=torch.from_numpy(img).dtype, device=dev)
            t[: h * w] = torch.from_numpy(np.ascontiguousarray(img[:, :, 0])).reshape(-1).to(dev)
            return t
        mov, fix = padded(pair.moving), padded(pair.fixed)
        lo, hi, cnt = pair.grid_args()
        n = int(np.prod(cnt))
        res = torch.empty(n + 1, dtype=torch.float32, device=dev)
        f8 = lambda v: (C.c_float * 8)(*[float(x) for x in v])
        ms = C.c_float(0)
        for rep in range(2):  # the first run includes module loading
            rc = L.cgsref_gpu_search(code, f8(lo), f8(hi), f8(cnt), mov.data_ptr(), pair.moving.shape[0],
                                     pair.moving.shape[1], fix.data_ptr(), pair.fixed.shape[0], pair.fixed.shape[1],
                                     res.data_ptr(), C.byref(ms))
            if rc != 0:
                print(json.dumps({"impl": "reference-gpu", "cost": name, "error": rc}))
                break
        else:
            print(json.dumps({"impl": "reference-gpu", "cost": name, "grid_points": n,
                              "pixels": int(pair.fixed.shape[0] * pair.fixed.shape[1]),
                              "ms": float(ms.value), "evals_per_s": n / (ms.value / 1e3),
                              "code": "CudaGridSearcher::search_by_value, unchanged reference source, sm_100a"}),
                  flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
