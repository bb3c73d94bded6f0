"""The batched search (cgs_batch_* / cgs_search_batched) on the GPU.

A batch evaluates many pairs of uneven sizes, each with its own grid and cost: the persistent
kernel over the per-sample pairs' tasks, the multi-pair span kernel over the ZNCC pairs that
cgs_search runs on its span kernel, and cgs_search's own launches for MI pairs whose grids fill
the GPU (CGS_BATCH_SPAN_TASKS_PER_SM tasks per SM, default 4; the small MI grids here stay in the
persistent kernel unless a test sets it to 0).  Its per-pair results are checked against
cgs_search on the same pair (itself checked against the oracle in test_gpu_parity.py):
  * block_split = 0: costs bit-identical for every points-per-warp / warps-per-block plan
    (each point's pixels are summed in the same order whatever the plan; ZNCC pairs as
    cgs_search's span kernel, MI pairs as its per-sample and span kernels, which agree bit for bit);
  * block_split = 1: MI costs bit-identical (exact counts, same final sum), the others
    within the FP32 summation-order tolerance; argmins equal where separated;
  * ZNCC and MI pairs with per-sample decisions run in the persistent kernel, bit-identical to
    cgs_search with the same flag;
and the pairs' costs against the FP64 oracle directly on a small batch.  Also: graph replay
after the images change in place, the autotuner, per-pair time stamps, the one-shot entry.
"""
import numpy as np
import pytest

import oracle as O
from conftest import close_costs, separated_argmin
from cugridsearch_b200 import synthetic as S

pytestmark = pytest.mark.gpu

# (cost, size, moving size, values per axis); sizes uneven on purpose
SPECS = [
    ("SAD_AVG", 40, 40, 3),
    ("ZNCC", 56, 52, 3),
    ("MI", 48, 48, 3),
    ("NCC_REF", 36, 38, 3),
    ("SQD_REF", 28, 28, 3),
    ("ZNCC", 72, 72, 2),
    ("MI", 64, 60, 2),
    ("SAD_AVG", 24, 24, 4),
]


def _make(cuda, specs, seed=7):
    import torch
    import cugridsearch_b200 as cgs
    items = []
    for i, (cost, size, msize, count) in enumerate(specs):
        pr = S.small_pair(seed + i, size=size, count=count, cost=cost, msize=msize)
        mov_t = torch.from_numpy(pr.moving).to(cuda)
        fix_t = torch.from_numpy(pr.fixed).to(cuda)
        grid = cgs.CudaGrid.from_ranges(*pr.grid_args())
        n = grid.numElements()
        items.append(dict(pair=pr, cost=cost, mov=cgs.CudaImage(mov_t), fix=cgs.CudaImage(fix_t), grid=grid,
                          costs=torch.empty(n, dtype=torch.float32, device=cuda), result=cgs.result_buffer(cuda)))
    return items


def _single(cuda, items, per_sample=False):
    """cgs_search per pair: (costs, argmin) on the host, with the batch pairs' flags."""
    import torch
    import cugridsearch_b200 as cgs
    out = []
    for it in items:
        c = torch.empty(it["grid"].numElements(), dtype=torch.float32, device=cuda)
        r = cgs.search(it["cost"], it["mov"], it["fix"], it["grid"], costs=c, per_sample_decisions=per_sample)
        out.append((c.cpu().numpy(), r))
    return out


def _batch_pairs(items, per_sample=False):
    import cugridsearch_b200 as cgs
    return [cgs.BatchPair(it["cost"], it["mov"], it["fix"], it["grid"], it["result"], it["costs"],
                          per_sample_decisions=per_sample) for it in items]


def _read(items):
    import cugridsearch_b200 as cgs
    return [(it["costs"].cpu().numpy(), cgs.read_result(it["result"])) for it in items]


@pytest.fixture(scope="module")
def items(cuda, lib):
    return _make(cuda, SPECS)


@pytest.fixture(scope="module")
def reference(cuda, items):
    return _single(cuda, items)


PLANS = [(g, w, 0) for g in (1, 2, 4, 8) for w in (4, 8, 16)]


@pytest.mark.parametrize("g,w,bs", PLANS)
def test_batch_warp_split_bit_identical(cuda, items, reference, g, w, bs):
    import torch
    import cugridsearch_b200 as cgs
    plan = cgs.BatchPlan(g, w, bs)
    try:
        batch = cgs.Batch(_batch_pairs(items), plan)
    except cgs.CgsError as e:
        assert e.status == 2, e  # a plan that does not fit an SM is reported as unsupported
        pytest.skip(f"plan {plan} does not fit: {e}")
    with batch:
        batch.launch()
        torch.cuda.synchronize()
        got = _read(items)
    for (c_ref, r_ref), (c, r), it in zip(reference, got, items):
        np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32), err_msg=it["cost"])
        assert r.index == r_ref.index and r.valid == r_ref.valid and r.status == 0
        np.testing.assert_array_equal(r.params, r_ref.params)


@pytest.mark.parametrize("g,w", [(1, 16), (2, 8), (4, 4), (8, 4), (8, 8)])
def test_batch_block_split(cuda, items, reference, g, w):
    import torch
    import cugridsearch_b200 as cgs
    try:
        batch = cgs.Batch(_batch_pairs(items), cgs.BatchPlan(g, w, 1))
    except cgs.CgsError as e:
        assert e.status == 2, e
        pytest.skip(str(e))
    with batch:
        batch.launch()
        torch.cuda.synchronize()
        got = _read(items)
    for (c_ref, r_ref), (c, r), it in zip(reference, got, items):
        name = it["cost"]
        if name == "MI":
            np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32))
        else:
            fin = np.isfinite(c_ref)
            assert np.array_equal(np.isfinite(c), fin)
            scale = {"SQD_REF": 1e-3}.get(name, 1.0)
            tol = 2e-5 * np.maximum(np.abs(c_ref[fin]), scale)
            assert np.all(np.abs(c[fin] - c_ref[fin]) <= tol), name
        _, sep, near = separated_argmin(c_ref, c_ref.astype(np.float64), name)
        assert r.status == 0 and (r.index == r_ref.index or (not sep and r.index in set(near.tolist())))


def test_batch_against_oracle(cuda, lib):
    """Small batch, every pair's costs against the FP64 oracle (parity tolerance)."""
    import torch
    import cugridsearch_b200 as cgs
    specs = [("SAD_AVG", 20, 20, 2), ("ZNCC", 24, 22, 2), ("MI", 20, 20, 2), ("NCC_REF", 16, 18, 2)]
    its = _make(cuda, specs, seed=101)
    with cgs.Batch(_batch_pairs(its)) as b:
        b.launch()
        torch.cuda.synchronize()
        got = _read(its)
    for it, (c, r) in zip(its, got):
        pr, name = it["pair"], it["cost"]
        og = O.make_grid(*pr.grid_args())
        c32, c64 = O.search(name, og, O.Image(pr.moving), O.Image(pr.fixed))
        bad = close_costs(c, c32, c64, name)
        assert not bad.any(), (name, np.flatnonzero(bad)[:5])
        i, sep, near = separated_argmin(c32, c64, name)
        assert r.index == i or (not sep and r.index in set(near.tolist()))


def test_batch_graph_replay_follows_image_contents(cuda, items, reference):
    """The graph binds buffers, not contents: change a pair's images in place, relaunch."""
    import torch
    import cugridsearch_b200 as cgs
    with cgs.Batch(_batch_pairs(items)) as b:
        b.launch()
        b.launch()  # replays are serialised
        torch.cuda.synchronize()
        first = _read(items)
        for (c, r), (c_ref, _) in zip(first, reference):
            np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32))
        # swap in other images of the same shape for pair 1, then relaunch
        it = items[1]
        old_m, old_f = it["mov"].tensor.clone(), it["fix"].tensor.clone()
        other = S.small_pair(999, size=it["fix"].height(), count=3, cost=it["cost"], msize=it["mov"].height())
        it["mov"].tensor.copy_(torch.from_numpy(other.moving).to(cuda))
        it["fix"].tensor.copy_(torch.from_numpy(other.fixed).to(cuda))
        try:
            b.launch()
            torch.cuda.synchronize()
            c_new = it["costs"].cpu().numpy()
            c_chk = torch.empty_like(it["costs"])
            cgs.search(it["cost"], it["mov"], it["fix"], it["grid"], costs=c_chk)
            np.testing.assert_array_equal(c_new.view(np.uint32), c_chk.cpu().numpy().view(np.uint32))
            assert not np.array_equal(c_new, reference[1][0])
        finally:
            it["mov"].tensor.copy_(old_m)
            it["fix"].tensor.copy_(old_f)


def test_batch_autotune_and_times(cuda, items, reference):
    import torch
    import cugridsearch_b200 as cgs
    with cgs.Batch(_batch_pairs(items)) as b:
        best, table = b.autotune(sample_points=64)
        assert len(table) == 24
        ok = [t for t in table if t[2] == 0]
        assert ok and all(np.isfinite(t[1]) and t[1] > 0 for t in ok)
        assert best == min(ok, key=lambda t: t[1])[0] and b.plan == best
        b.launch()
        t0, t1 = b.pair_times()
        got = _read(items)
    for (c_ref, r_ref), (c, r) in zip(reference, got):
        if best.block_split == 0:
            np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32))
        assert r.status == 0
    assert np.all(t0 > 0) and np.all(t1 >= t0)


def test_search_batched_one_shot(cuda, items, reference):
    import ctypes as C
    import torch
    import cugridsearch_b200 as cgs
    from cugridsearch_b200 import _abi
    for it in items:
        it["costs"].fill_(-1.0)
    arr = (_abi.CgsPair * len(items))(*[p.to_c() for p in _batch_pairs(items)])
    plan = cgs.BatchPlan(4, 8, 0).to_c()
    s = torch.cuda.current_stream().cuda_stream
    _abi.check(cgs.library().cgs_search_batched(arr, len(items), C.byref(plan), s))
    for (c_ref, r_ref), (c, r) in zip(reference, _read(items)):
        np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32))
        assert r.index == r_ref.index


@pytest.mark.parametrize("g,w,bs", [(2, 16, 0), (4, 8, 0), (1, 16, 1)])
def test_batch_per_sample_pairs_in_the_persistent_kernel(cuda, items, g, w, bs):
    """With per-sample decisions the ZNCC and MI pairs run in the persistent kernel too: costs
    bit-identical to cgs_search with the same flag (block_split = 1: MI exactly, ZNCC within the
    summation-order tolerance)."""
    import torch
    import cugridsearch_b200 as cgs
    ref = _single(cuda, items, per_sample=True)
    try:
        batch = cgs.Batch(_batch_pairs(items, per_sample=True), cgs.BatchPlan(g, w, bs))
    except cgs.CgsError as e:
        assert e.status == 2, e
        pytest.skip(str(e))
    with batch:
        batch.launch()
        torch.cuda.synchronize()
        got = _read(items)
        t0, t1 = batch.pair_times()
    for (c_ref, r_ref), (c, r), it in zip(ref, got, items):
        if bs == 0 or it["cost"] == "MI":
            np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32), err_msg=it["cost"])
            assert r.index == r_ref.index
        else:
            fin = np.isfinite(c_ref)
            assert np.array_equal(np.isfinite(c), fin)
            scale = {"SQD_REF": 1e-3}.get(it["cost"], 1.0)
            assert np.all(np.abs(c[fin] - c_ref[fin]) <= 2e-5 * np.maximum(np.abs(c_ref[fin]), scale)), it["cost"]
        assert r.status == 0
    assert np.all(t0 > 0) and np.all(t1 >= t0)


def test_batch_span_pairs_follow_cgs_search(cuda, items, reference, monkeypatch):
    """The ZNCC pairs share one multi-pair span launch and get cgs_search's span-kernel costs bit
    for bit; with every span-eligible pair routed (CGS_BATCH_SPAN_TASKS_PER_SM=0) the MI pairs
    are searched by cgs_search's own launches, FP64 verification included.  The graph holds
    staging, the span staging step, the persistent kernel and the multi-pair span kernel, plus
    the routed pairs' launches."""
    import torch
    import cugridsearch_b200 as cgs
    with cgs.Batch(_batch_pairs(items)) as b0:
        assert b0.kernel_launches == 4
        b0.launch()
        torch.cuda.synchronize()
        got = _read(items)
        t0, t1 = b0.pair_times()
    for (c_ref, r_ref), (c, r), it in zip(reference, got, items):
        np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32), err_msg=it["cost"])
        assert r.index == r_ref.index and r.status == 0
    assert np.all(t0 > 0) and np.all(t1 >= t0)
    monkeypatch.setenv("CGS_BATCH_SPAN_TASKS_PER_SM", "0")
    with cgs.Batch(_batch_pairs(items)) as b:
        assert b.kernel_launches > 4 + 4 * sum(it["cost"] == "MI" for it in items)
        b.launch()
        torch.cuda.synchronize()
        got = _read(items)
        t0, t1 = b.pair_times()
    for (c_ref, r_ref), (c, r), it in zip(reference, got, items):
        np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32), err_msg=it["cost"])
        if it["cost"] != "MI":
            continue
        assert (r.index, r.valid, r.status, r.verified, r.index_fp64) == \
            (r_ref.index, r_ref.valid, r_ref.status, r_ref.verified, r_ref.index_fp64)
        assert r.cost_fp64 == r_ref.cost_fp64 and r.err_fp64 == r_ref.err_fp64
    assert np.all(t0 > 0) and np.all(t1 >= t0)


def test_batch_zncc_group_of_mixed_sizes(cuda, lib):
    """ZNCC pairs of different sizes share one multi-pair span launch (one shared-memory carve for
    the largest tile count, one window stage for all): each pair's costs and argmin equal
    cgs_search's bit for bit."""
    import torch
    import cugridsearch_b200 as cgs
    specs = [("ZNCC", 300, 280, 2), ("ZNCC", 64, 60, 3), ("ZNCC", 200, 210, 2), ("ZNCC", 130, 130, 2)]
    its = _make(cuda, specs, seed=211)
    ref = _single(cuda, its)
    with cgs.Batch(_batch_pairs(its)) as b:
        assert b.kernel_launches == 3  # staging, span staging, the multi-pair span kernel
        b.launch()
        torch.cuda.synchronize()
        got = _read(its)
    for (c_ref, r_ref), (c, r), it in zip(ref, got, its):
        np.testing.assert_array_equal(c.view(np.uint32), c_ref.view(np.uint32))
        assert r.index == r_ref.index and r.status == 0 and r.valid == r_ref.valid
