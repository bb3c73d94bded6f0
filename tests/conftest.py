"""Test configuration: the `gpu` marker, shared fixtures and tolerance helpers.

Tests marked `gpu` need an sm_100 device and the built library; everything else runs on
the CPU (oracle pinning, host-side grid arithmetic, ABI loading, multi-process logic).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU and the built CUDA library")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def lib():
    from cugridsearch_b200 import build
    build.build()
    import cugridsearch_b200 as cgs
    return cgs.library()


# Per-point cost tolerance against the FP64 oracle (same samples, exact sums): the GPU sums
# in FP32 in a different order than the reference, so costs agree to a relative 1e-5 of the
# cost's natural scale.  `scale` is the magnitude below which the tolerance is absolute.
REL_TOL = 1e-5
COST_SCALE = {"SAD_AVG": 1.0, "SAD_AVG_H": 1.0, "SAD_SUM_T": 1.0, "SAD_SUM_T_REF": 1.0, "SQD_REF": 1e-3,
              "NCC_REF": 1.0, "SQD_ALT": 1e-3, "NCC_ALT": 1.0, "MI_ALT": 1.0, "ZNCC": 1.0, "MI": 1.0}


def close_costs(gpu, ref32, ref64, name, rel=REL_TOL):
    """Elementwise check |gpu - fp64| <= |ref32 - fp64| + rel * max(|fp64|, scale).

    NaN and +-inf must match exactly (the reference's sentinels and no-overlap NaN)."""
    gpu = np.asarray(gpu, np.float64)
    r32 = np.asarray(ref32, np.float64)
    r64 = np.asarray(ref64, np.float64)
    scale = COST_SCALE[name]
    special = ~np.isfinite(r64) | ~np.isfinite(r32)
    bad_special = special & ~((np.isnan(gpu) & np.isnan(r32)) | (gpu == r32))
    fin = ~special
    tol = np.abs(r32 - r64) + rel * np.maximum(np.abs(r64), scale)
    bad = fin & ~(np.abs(gpu - r64) <= tol)
    return bad | bad_special


def separated_argmin(costs32, costs64, name, rel=REL_TOL):
    """Lowest-index argmin of the reference costs and whether it is separated from the
    runner-up by more than the tolerance (only then must an argmin match exactly)."""
    c = np.where(np.isfinite(costs32), costs32, np.inf).astype(np.float64)
    if not np.isfinite(c).any():
        return -1, True, np.array([], dtype=np.int64)
    i = int(np.argmin(c))
    tol = 2 * (abs(float(costs32[i]) - float(costs64[i])) + rel * max(abs(float(costs64[i])), COST_SCALE[name]))
    near = np.flatnonzero(c <= c[i] + tol)
    return i, len(near) == 1, near
