"""CPU tests of the learned proposal: the float64 reference network's gradients against finite
differences (so it can serve as the GPU kernels' gradient oracle), the window rule and grid
windows (cgs_proposal_window, cgs_grid_window: host functions of the library), the coarse probe
and corner errors."""
import numpy as np
import pytest
import torch

import oracle.proposal_ref as R


@pytest.fixture(scope="module")
def small_net():
    rng = np.random.default_rng(5)
    off, total = R.layout()
    p = np.zeros(total)
    for l in range(5):
        o, (co, kp) = off[f"w{l}"]
        w = rng.normal(0, np.sqrt(2.0 / (9 * R.CIN[l])), (co, kp))
        w[:, 9 * R.CIN[l]:] = 0
        p[o:o + co * kp] = w.ravel()
        o, (cb,) = off[f"b{l}"]
        p[o:o + cb] = rng.normal(0, 0.05, cb)
    for name, sd in (("fc1w", np.sqrt(2.0 / 256)), ("fc1b", 0.05), ("fc2w", 0.1), ("fc2b", 0.1)):
        o, sh = off[name]
        p[o:o + int(np.prod(sh))] = rng.normal(0, sd, int(np.prod(sh)))
    fixed = rng.uniform(0, 255, (2, 128, 128))
    moving = rng.uniform(0, 255, (2, 128, 128))
    labels = rng.uniform(-1, 1, (2, 8))
    return p, fixed, moving, labels


def test_reference_gradients_match_finite_differences(small_net):
    p, fixed, moving, labels = small_net
    _, L, g = R.loss_and_grads(p, fixed, moving, labels, bf16=False)
    x = R.net_input(fixed, moving, bf16=False)
    lab = torch.from_numpy(labels)
    off, _ = R.layout()
    rng = np.random.default_rng(1)
    picks = []
    for name in ("w0", "b0", "w2", "w4", "b4", "fc1w", "fc2w", "fc2b"):
        o, sh = off[name]
        n = int(np.prod(sh))
        idx = [i for i in rng.integers(0, n, 40) if name != "w0" or (i % sh[1]) < 18][:4]
        picks += [o + int(i) for i in idx]
    for i in picks:
        h = 1e-5
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = float(R.loss(R.forward(torch.from_numpy(pp), x, bf16=False), lab))
        lm = float(R.loss(R.forward(torch.from_numpy(pm), x, bf16=False), lab))
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_reference_padding_weights_have_zero_gradient(small_net):
    p, fixed, moving, labels = small_net
    _, _, g = R.loss_and_grads(p, fixed, moving, labels, bf16=True)
    off, _ = R.layout()
    o, (co, kp) = off["w0"]
    assert np.all(g[o:o + co * kp].reshape(co, kp)[:, 18:] == 0)


def _full():
    from cugridsearch_b200 import proposal as P
    return P.full_grid(256, 6)


def test_proposal_window_rule(lib):
    """Windows hold the proposed centre's nearest value, span the radius (clamped to
    [min_values, max_values]) and stay inside the grid."""
    from cugridsearch_b200 import proposal as P
    full = _full()
    rng = np.random.default_rng(3)
    n = 6
    for _ in range(200):
        out = np.concatenate([rng.uniform(-1.2, 1.2, 8), rng.uniform(-7, 5, 8)]).astype(np.float32)
        for mn, mx in ((1, 1), (1, 5), (3, 5), (3, 3), (5, 5)):
            first, cnt = P.proposal_window(full, out, mn, mx)
            assert np.all(cnt >= mn) and np.all(cnt <= mx) and np.all(cnt % 2 == 1)
            assert np.all(first >= 0) and np.all(first + cnt <= n)
            ic = np.floor((np.clip(out[:8], -1, 1) + 1) * 0.5 * (n - 1) + 0.5).astype(int)
            assert np.all((first <= ic) & (ic <= first + cnt - 1))
            w = np.floor(np.exp(np.clip(out[8:], -6, 4)) * 0.5 * (n - 1) + 0.5)
            want = np.clip(2 * w + 1, mn, mx)
            np.testing.assert_array_equal(cnt, want)


def test_grid_window_values_are_full_grid_values(lib):
    from cugridsearch_b200 import proposal as P
    full = _full()
    counts = [int(c) for c in full.getAxisSampleCounts()]
    inc = np.cumprod([1] + counts[:-1])
    rng = np.random.default_rng(8)
    for _ in range(20):
        cnt = rng.integers(1, 6, 8)
        first = np.array([rng.integers(0, 6 - c + 1) for c in cnt])
        g = P.grid_window(full, first, cnt)
        np.testing.assert_array_equal(g.getAxisSampleCounts(), cnt.astype(np.float32))
        winc = np.cumprod([1] + list(cnt[:-1]))
        for a in range(8):
            for j in range(cnt[a]):
                v = float(g.getGridPoint(int(j * winc[a]))[a])
                ref = float(full.getGridPoint(int((first[a] + j) * inc[a]))[a])
                assert abs(v - ref) <= 2e-6 * max(1.0, abs(ref)), (a, j, v, ref)
    with pytest.raises(Exception):
        P.grid_window(full, np.full(8, 4), np.full(8, 3))  # past the last value


def test_coarse_probe_is_full_grid_points(lib):
    from cugridsearch_b200 import proposal as P
    full = _full()
    probe = P.coarse_grid(full, 3)
    np.testing.assert_array_equal(probe.getAxisSampleCounts(), np.full(8, 3.0))
    counts = [int(c) for c in full.getAxisSampleCounts()]
    inc = np.cumprod([1] + counts[:-1])
    for a in range(8):
        for j, i in enumerate((0, 2, 4)):
            v = float(probe.getGridPoint(int(j * 3 ** a))[a])
            assert abs(v - float(full.getGridPoint(int(i * inc[a]))[a])) <= 2e-6 * max(1.0, abs(v))


def test_corner_error():
    from cugridsearch_b200 import proposal as P
    p = np.array([0.1, 1.0, 1.0, 0.0, 3.0, -2.0, 0.0, 0.0])
    assert P.corner_error(p, p)[0] == 0.0
    q = p.copy()
    q[4] += 1.0  # one pixel of translation moves every corner by one pixel
    assert abs(P.corner_error(p, q)[0] - 1.0) < 1e-9


def _oracle_batch_search(cost, fixed, moving, grids, device, dump=None):
    """serve()'s batch search, done by the CPU oracle (FP32 reference sums, lowest index)."""
    import oracle as O
    ps, cs, vs, pts, dumps = [], [], [], 0, {}
    for i, g in enumerate(grids):
        m = g.matrix()
        og = O.make_grid(m[0], m[1], m[3])
        c32, _ = O.search(cost, og, O.Image(moving[i].numpy()[:, :, None]), O.Image(fixed[i].numpy()[:, :, None]),
                          f64=False)
        c = np.where(np.isfinite(c32), c32, np.inf)
        k = int(np.argmin(c))
        ps.append(O.grid_point(og, k)[: g.g.dims].astype(np.float64))
        cs.append(float(c[k]))
        vs.append(bool(np.isfinite(c[k])))
        pts += g.numElements()
        if dump is not None and i in dump:
            dumps[i] = c32
    if dump is not None:
        return np.stack(ps), np.array(cs), np.array(vs), pts, dumps
    return np.stack(ps), np.array(cs), np.array(vs), pts


def test_serve_logic_with_oracle_search(lib, monkeypatch):
    """The serving logic (windows, walks, local-minimum check, probe, fallback) with the searches
    done by the oracle: aimed proposals return the full grid's argmins without a fallback, off-target
    ones walk or fall back and still return them, and the points evaluated are counted."""
    from cugridsearch_b200 import proposal as P
    from cugridsearch_b200 import synthetic as S
    monkeypatch.setattr(P, "_batch_search", _oracle_batch_search)
    pairs = [S.small_pair(500 + i, size=16, count=4, cost="ZNCC") for i in range(3)]
    fixed = torch.from_numpy(np.stack([p.fixed[:, :, 0] for p in pairs]))
    moving = torch.from_numpy(np.stack([p.moving[:, :, 0] for p in pairs]))
    from cugridsearch_b200 import CudaGrid
    full = CudaGrid.from_ranges(*pairs[0].grid_args())
    truth, tcost, _, _ = _oracle_batch_search("ZNCC", fixed, moving, [full] * 3, None)
    assert np.all(np.isfinite(tcost))
    lo, hi = full.matrix()[0], full.matrix()[1]

    class Net:
        def __init__(self, out):
            self.out = out

        def forward(self, f, m):
            return torch.from_numpy(self.out)

    u = P.to_units(truth, lo, hi)
    aimed = np.concatenate([u, np.full((3, 8), -5.0)], 1).astype(np.float32)
    r = P.serve(Net(aimed), fixed, moving, full, min_values=3, max_values=3, starts=1)
    assert not r.fallback.any()
    np.testing.assert_allclose(r.params, truth, atol=1e-6)
    # off by one lattice step on every axis: a walk (or the fallback) recovers the argmins
    step = 2.0 / 3.0
    off = np.concatenate([np.clip(u + step, -1, 1), np.full((3, 8), -5.0)], 1).astype(np.float32)
    r2 = P.serve(Net(off), fixed, moving, full, min_values=3, max_values=3, walks=3, starts=1)
    np.testing.assert_allclose(r2.costs, tcost, rtol=1e-6, atol=1e-7)
    assert r2.points > r.points  # the walks cost more than the aimed first pass
    # more starts (the probe's best points) still return the argmins
    r3 = P.serve(Net(off), fixed, moving, full, min_values=3, max_values=3, walks=3, starts=3)
    np.testing.assert_allclose(r3.costs, tcost, rtol=1e-6, atol=1e-7)


def test_refine_serve_logic_with_oracle_search(lib, monkeypatch):
    """The refinement serving (local grids around the proposal, coarse to fine levels, edge walks,
    coarse probe, fallback) with the searches done by the oracle: started at the full grid's
    argmin it never returns a worse cost; every level is one batch search over the pairs still
    refining; a proposal far from the argmin with a tiny radius ends above the probe's best and
    falls back to the full grid's answer; the points evaluated are counted."""
    from cugridsearch_b200 import proposal as P
    from cugridsearch_b200 import synthetic as S
    calls = []

    def counted(cost, fixed, moving, grids, device, dump=None):
        calls.append(len(grids))
        return _oracle_batch_search(cost, fixed, moving, grids, device, dump)

    monkeypatch.setattr(P, "_batch_search", counted)
    pairs = [S.small_pair(600 + i, size=16, count=4, cost="ZNCC") for i in range(3)]
    fixed = torch.from_numpy(np.stack([p.fixed[:, :, 0] for p in pairs]))
    moving = torch.from_numpy(np.stack([p.moving[:, :, 0] for p in pairs]))
    from cugridsearch_b200 import CudaGrid
    full = CudaGrid.from_ranges(*pairs[0].grid_args())
    truth, tcost, _, _ = _oracle_batch_search("ZNCC", fixed, moving, [full] * 3, None)
    assert np.all(np.isfinite(tcost))

    class Net:
        def __init__(self, out):
            self.out = out

        def forward(self, f, m):
            return torch.from_numpy(self.out)

    zero = np.zeros((3, 16), np.float32)
    # started at the argmin: the first local grid holds it, so no answer costs more
    calls.clear()
    r = P.refine_serve(Net(zero), fixed, moving, full, values=3, levels=2, walks=0, start=truth)
    assert np.all(r.costs <= tcost + 1e-7) and not r.fallback.any()
    assert calls[0] == 6  # three local grids and three coarse probes in one search
    assert len(calls) <= 3 and all(c <= 3 for c in calls[1:])  # then one search per level
    # the counted points are the grids actually searched
    assert r.points == 3 * 3 ** 8 + 3 * 3 ** 8 + sum(calls[1:]) * 3 ** 8
    # far off (a corner of the range, the smallest radius): the refined cost is above the probe's
    # best for at least one pair, which then takes the full grid's answer
    lo, hi = full.matrix()[0], full.matrix()[1]
    far = np.concatenate([np.full((3, 8), 0.999), np.full((3, 8), -12.0)], 1).astype(np.float32)
    calls.clear()
    r2 = P.refine_serve(Net(far), fixed, moving, full, values=3, levels=1, walks=0, min_half=1e-4)
    assert r2.fallback.any()
    fb = r2.fallback
    np.testing.assert_allclose(r2.costs[fb], tcost[fb], rtol=1e-6, atol=1e-7)
    assert calls[-1] == int(fb.sum())  # the fallback searches the full grid of those pairs only
    assert np.all(r2.params >= lo - 1e-6) and np.all(r2.params <= hi + 1e-6)


def test_batch_search_reads_every_pair_result(lib, monkeypatch):
    """_batch_search hands each pair a slot of one result block and reads all of them with one
    copy: a stand-in batch writes a distinct result through each pair's result pointer, and each
    comes back to its own pair."""
    import ctypes as C
    import cugridsearch_b200 as cgs
    from cugridsearch_b200 import _abi
    from cugridsearch_b200 import proposal as P

    class FakeBatch:
        def __init__(self, pairs, plan=None):
            self.pairs = pairs

        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

        def launch(self, stream=None):
            for i, bp in enumerate(self.pairs):
                r = _abi.CgsArgmin()
                r.cost, r.valid, r.index = -0.5 - i, 1, 1000 + i
                for a in range(8):
                    r.params[a] = float(i + a)
                addr = bp.result.data_ptr()
                assert addr % 8 == 0
                C.memmove(addr, C.addressof(r), C.sizeof(r))

    monkeypatch.setattr(cgs, "Batch", FakeBatch)
    monkeypatch.setattr(cgs, "CudaImage", lambda t: t)  # host tensors stand in for the images
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    full = P.full_grid(256, 6)
    n = 5
    img = torch.zeros((n, 4, 4))
    params, costs, valid, pts = P._batch_search("ZNCC", img, img, [full] * n, torch.device("cpu"))
    assert valid.all() and pts == n * full.numElements()
    np.testing.assert_array_equal(costs, -0.5 - np.arange(n))
    np.testing.assert_array_equal(params, np.arange(n)[:, None] + np.arange(8)[None, :])


def _refine_per_pair(net, n, full, search, values, levels, spread, min_half, walks):
    """The refinement serving's rules applied pair by pair (a restatement for the test): keep the
    best point, walk on an inner edge while walks are left, else halve while levels are left."""
    from cugridsearch_b200 import CudaGrid
    from cugridsearch_b200 import proposal as P
    d = 8
    lo, hi = full.matrix()[0].astype(np.float64), full.matrix()[1].astype(np.float64)
    out = net.forward(None, None).numpy().astype(np.float64)
    centre = P.from_units(np.clip(out[:, :d], -1, 1), lo, hi)
    half = np.clip(spread * np.exp(np.clip(out[:, 8:], -12, 4)), min_half, 1.0) * (hi - lo) / 2

    def local(c, h):
        a, b = np.maximum(lo, c - h), np.minimum(hi, c + h)
        return CudaGrid.from_ranges(list(a), list(np.where(b > a, b, a)),
                                    [values if b[k] > a[k] else 1 for k in range(d)])

    probe = P.coarse_grid(full, 3)
    grids = [local(centre[i], half[i]) for i in range(n)]
    p, c, v, pts = search(grids + [probe] * n)
    probe_cost = np.where(v[n:], c[n:], np.inf)
    params, costs = np.zeros((n, d)), np.full(n, np.inf)
    lev, wal = [levels] * n, [walks] * n
    active, cur = list(range(n)), (p[:n], c[:n], v[:n], grids)
    while True:
        nxt, ng = [], []
        for j, i in enumerate(active):
            cp, cc, cv, cg = cur[0][j], cur[1][j], cur[2][j], cur[3][j]
            if cv and cc < costs[i]:
                params[i], costs[i] = cp, cc
            if not cv or not np.isfinite(costs[i]):
                continue
            a = np.array(cg.g.start[:d], np.float64)
            r = np.array(cg.g.resolution[:d], np.float64)
            cnt = np.array(cg.g.count[:d]).astype(int)
            loc = np.where(cnt > 1, np.rint((params[i] - a) / np.where(r != 0, r, 1.0)), 0)
            edge = ((loc == 0) & (a > lo + 1e-9 * (hi - lo))) | \
                ((loc == cnt - 1) & (a + r * (cnt - 1) < hi - 1e-9 * (hi - lo)))
            if edge.any() and wal[i] > 0:
                wal[i] -= 1
            elif lev[i] > 0:
                lev[i] -= 1
                half[i] = half[i] / 2
            else:
                continue
            nxt.append(i)
            ng.append(local(params[i], half[i]))
        if not nxt:
            break
        p2, c2, v2, k = search(ng)
        pts += k
        active, cur = nxt, (p2, c2, v2, ng)
    fb = ~(costs <= probe_cost)
    if fb.any():
        pf, cf, _, k = search([full] * int(fb.sum()))
        pts += k
        params[fb], costs[fb] = pf, cf
    return params, costs, fb, pts


def test_refine_serve_decisions_match_the_per_pair_rules(lib, monkeypatch):
    """refine_serve takes its keep / walk / halve / stop decisions for all active pairs at once;
    on stand-in searches (deterministic in the grid, some results invalid) its answers, fallbacks
    and point counts equal the rules applied pair by pair."""
    from cugridsearch_b200 import proposal as P
    full = P.full_grid(256, 6)
    lo, hi = full.matrix()[0].astype(np.float64), full.matrix()[1].astype(np.float64)

    def stand_in(seed):
        tgt = lo + (hi - lo) * np.random.default_rng(seed).uniform(0.1, 0.9, 8)

        def search(grids):
            ps, cs, vs = [], [], []
            for g in grids:
                key = int(abs(np.sum(np.array(g.g.start[:8]) * 1.37 + np.array(g.g.end[:8]))) * 1e6) % (2 ** 32)
                rs = np.random.default_rng([seed, key])
                q = np.array(g.getGridPoint(int(rs.integers(0, g.numElements()))), np.float64)
                ps.append(q)
                cs.append(float(np.sum(((q - tgt) / (hi - lo)) ** 2)) + rs.uniform(0, 1e-3))
                vs.append(rs.random() > 0.05)
            return np.stack(ps), np.array(cs), np.array(vs), sum(g.numElements() for g in grids)
        return search

    class Net:
        def __init__(self, seed, n):
            r = np.random.default_rng(seed)
            self.out = np.concatenate([r.uniform(-1, 1, (n, 8)), r.uniform(-6, 1, (n, 8))], 1).astype(np.float32)

        def forward(self, f, m):
            return torch.from_numpy(self.out)

    fallbacks = 0
    for seed in range(24):
        n = 1 + seed % 7
        kw = dict(values=3, levels=1 + seed % 4, spread=2.0, min_half=0.02, walks=seed % 3)
        search = stand_in(seed)
        monkeypatch.setattr(P, "_batch_search", lambda cost, f, m, grids, dev, dump=None: search(grids))
        img = torch.zeros((n, 4, 4))
        r = P.refine_serve(Net(seed, n), img, img, full, **kw)
        p, c, fb, pts = _refine_per_pair(Net(seed, n), n, full, search, **kw)
        np.testing.assert_array_equal(r.params, p)
        np.testing.assert_array_equal(r.costs, c)
        np.testing.assert_array_equal(r.fallback, fb)
        assert r.points == pts
        fallbacks += int(fb.sum())
    assert fallbacks > 0  # the stand-in exercises the fallback too
