"""The learned proposal on the GPU.

* Forward outputs and gradients of the CUDA network (BF16 tensor-core convolutions, FP32
  accumulation) against the float64 torch reference that mirrors its BF16 rounding points
  (oracle/proposal_ref.py).  Tolerance: the reference sums in float64 and the GPU in FP32, and
  a BF16 rounding can land on the other side for a few elements, so each gradient tensor must
  agree to 2 % relative L2 with cosine similarity above 0.999; outputs to 1 % of their scale.
* One Adam step against a numpy restatement of Adam on the GPU's own gradients.
* The serving path (proposal windows, window walks, coarse probe, full-grid fallback): with
  proposals placed on the full grid's argmins it reproduces them exactly without a fallback;
  with blind proposals the fallback finds them anyway.
* A short training run: the trained network lowers the held-out loss and, served, evaluates
  fewer grid points than the full grid while agreeing with it.
* Coarse-to-fine refinement serving: started at the full grid's argmin it never loses it; with
  the committed trained network its answers cost no more than the full grid's and lie closer to
  the ground truth than the full grid's argmin, where an untrained network does not.
"""
import numpy as np
import pytest

import oracle.proposal_ref as R

pytestmark = pytest.mark.gpu


def _images(cuda, n, side, seed):
    from cugridsearch_b200 import synthetic as S
    f, m, gt = S.config4_batch(seed, n, cuda, side)
    return f, m, gt


@pytest.fixture(scope="module")
def net_and_batch(cuda, lib):
    import torch
    from cugridsearch_b200.proposal import ProposalNet
    net = ProposalNet(max_batch=64, seed=11)
    f, m, _ = _images(cuda, 6, 256, seed=41)
    rng = np.random.default_rng(2)
    labels = rng.uniform(-1, 1, (6, 8)).astype(np.float32)
    yield net, f, m, labels
    net.close()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_and_gradients_match_reference(cuda, net_and_batch):
    import torch
    net, f, m, labels = net_and_batch
    p = net.params()
    out = net.forward(f, m)
    loss = net.backward(torch.from_numpy(labels).to(cuda))
    g = net.grads()
    out_ref, loss_ref, g_ref = R.loss_and_grads(p.astype(np.float64), f.cpu().numpy(), m.cpu().numpy(), labels)
    o = out.cpu().numpy()
    assert np.max(np.abs(o - out_ref)) <= 1e-2 * max(1.0, np.max(np.abs(out_ref))), (o, out_ref)
    assert abs(float(loss.cpu()) - loss_ref) <= 1e-3 * max(1.0, abs(loss_ref))
    off, _ = R.layout()
    for name, (o0, sh) in off.items():
        n = int(np.prod(sh))
        a, b = g[o0:o0 + n].astype(np.float64), g_ref[o0:o0 + n]
        if np.linalg.norm(b) == 0:
            assert np.all(a == 0), name
            continue
        cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
        assert _rel(a, b) < 2e-2 and cos > 0.999, (name, _rel(a, b), cos)


def test_adam_step_matches_numpy(cuda, net_and_batch):
    import torch
    from cugridsearch_b200.proposal import ProposalNet
    net2 = ProposalNet(max_batch=16, seed=3)
    try:
        _, f, m, labels = net_and_batch
        p0 = net2.params().astype(np.float64)
        lr = 1e-3
        m1 = np.zeros_like(p0)
        m2 = np.zeros_like(p0)
        p = p0.copy()
        for t in (1, 2):
            net2.forward(f, m)
            net2.backward(torch.from_numpy(labels).to(cuda))
            g = net2.grads().astype(np.float64)
            net2.adam_step(lr)
            m1 = 0.9 * m1 + 0.1 * g
            m2 = 0.999 * m2 + 0.001 * g * g
            p = p - lr * (m1 / (1 - 0.9 ** t)) / (np.sqrt(m2 / (1 - 0.999 ** t)) + 1e-8)
        got = net2.params().astype(np.float64)
        assert np.max(np.abs(got - p)) <= 1e-6 + 1e-5 * np.max(np.abs(p0))
        assert not np.array_equal(got, p0)
    finally:
        net2.close()


def test_serving_reproduces_full_grid(cuda, lib):
    """Proposals on the argmins (narrow radius): the local grid holds them and they come back
    exactly.  Blind proposals (centre 0, narrow): the probe or the fallback finds them."""
    import torch
    from cugridsearch_b200 import proposal as P

    class Fixed:
        def __init__(self, out):
            self.out = out

        def forward(self, f, m):
            return torch.from_numpy(self.out)

    side, n = 128, 6
    f, m, _ = _images(cuda, n, side, seed=77)
    full = P.full_grid(side, 4)
    truth, tcost = P.grid_argmins(f, m, full)
    lo, hi = full.matrix()[0], full.matrix()[1]
    u = P.to_units(truth, lo, hi)
    aimed = np.concatenate([u, np.full((n, 8), -5.0)], 1).astype(np.float32)
    r = P.serve(Fixed(aimed), f, m, full, min_values=3, max_values=5)
    assert not r.fallback.any()
    np.testing.assert_allclose(r.params, truth, rtol=0, atol=1e-6)
    assert r.points < n * full.numElements()
    blind = np.concatenate([np.zeros((n, 8)), np.full((n, 8), -5.0)], 1).astype(np.float32)
    rb = P.serve(Fixed(blind), f, m, full, min_values=1, max_values=1)
    assert np.all(rb.costs <= tcost + 1e-5 * np.maximum(1, np.abs(tcost)))
    assert np.all(P.corner_error(rb.params, truth, side) < 0.5)


def test_training_gains_over_untrained(cuda, lib):
    """Train on grid-search labels of 768 small pairs; on 96 held-out pairs the trained network
    has a lower loss than the untrained one, and the served answers agree with the full grid
    while evaluating fewer grid points."""
    import torch
    from cugridsearch_b200 import proposal as P
    side = 128
    full = P.full_grid(side, 4)
    lo, hi = full.matrix()[0], full.matrix()[1]
    f, m, _ = _images(cuda, 864, side, seed=1234)
    truth, _ = P.grid_argmins(f, m, full)
    u = P.to_units(truth, lo, hi).astype(np.float32)
    tr, te = slice(0, 768), slice(768, 864)
    net = P.ProposalNet(max_batch=128, seed=5)
    try:
        lab_te = torch.from_numpy(u[te]).to(cuda)
        net.forward(f[te].contiguous(), m[te].contiguous())
        before = float(net.backward(lab_te).cpu())
        hist = P.train(net, f[tr].contiguous(), m[tr].contiguous(), u[tr], epochs=25, batch=128, lr=1e-3, seed=1)
        net.forward(f[te].contiguous(), m[te].contiguous())
        after = float(net.backward(lab_te).cpu())
        assert hist[-1] < hist[0] and after < before, (hist[0], hist[-1], before, after)
        r = P.serve(net, f[te].contiguous(), m[te].contiguous(), full, min_values=3, max_values=3)
        err = P.corner_error(r.params, truth[te], side)
        frac = r.points / (96 * full.numElements())
        print(f"held-out loss {before:.3f} -> {after:.3f}; fallback {r.fallback.mean():.3f}; "
              f"corner error mean {err.mean():.3f} px; points {frac:.3f} of the full grid")
        assert np.mean(err <= 0.5) >= 0.9
        assert frac < 1.0
    finally:
        net.close()


def test_refinement_from_the_argmin_never_loses_it(cuda, lib):
    """Coarse-to-fine local grids started at the full grid's argmin (narrow first range): every
    answer costs at most the argmin's cost (the start is the first grid's centre), and no pair
    falls back."""
    from cugridsearch_b200 import proposal as P

    class Blind:
        def forward(self, f, m):
            import torch
            return torch.zeros((f.shape[0], 16))

    side, n = 128, 6
    f, m, _ = _images(cuda, n, side, seed=91)
    full = P.full_grid(side, 4)
    truth, tcost = P.grid_argmins(f, m, full)
    r = P.refine_serve(Blind(), f, m, full, values=3, levels=3, min_half=0.01, walks=1, start=truth)
    assert not r.fallback.any()
    assert np.all(r.costs <= tcost + 1e-5 * np.maximum(1.0, np.abs(tcost))), (r.costs, tcost)
    assert r.points < n * full.numElements()
    assert r.d2h_bytes > 0


def test_trained_network_gains_in_refinement_serving(cuda, lib):
    """The committed network (models/proposal_net.npz, trained on 200,000 generated pairs) on 32
    held-out 256 px pairs, served by coarse-to-fine local grids: its answers cost no more than
    the full grid's argmin on nearly every pair and lie closer to the generator's ground truth
    than the full grid's argmin; an untrained network with the same serving lands far from the
    truth or falls back."""
    import os
    from cugridsearch_b200 import proposal as P
    ckpt = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "models", "proposal_net.npz")
    n = 32
    f, m, gt = P.config4_batch_cached(20261203 + 10 ** 7, n, cuda)
    full = P.full_grid(256, 6)
    truth, tcost = P.grid_argmins(f, m, full)
    kw = dict(values=3, levels=4, spread=2.0, min_half=0.02, walks=2)
    net = P.ProposalNet(max_batch=256)
    raw = P.ProposalNet(max_batch=256, seed=3)
    try:
        net.load(ckpt)
        r = P.refine_serve(net, f, m, full, **kw)
        r0 = P.refine_serve(raw, f, m, full, **kw)
    finally:
        net.close()
        raw.close()
    g = gt.numpy()
    e_trained = P.corner_error(r.params, g, 256).mean()
    e_full = P.corner_error(truth, g, 256).mean()
    e_raw = P.corner_error(r0.params, g, 256).mean()
    print(f"corner error vs ground truth: trained {e_trained:.2f} px, untrained {e_raw:.2f} px, "
          f"full grid {e_full:.2f} px; fallback {r.fallback.mean():.3f} / {r0.fallback.mean():.3f}")
    assert r.fallback.mean() <= 1.0 / n
    assert np.mean(r.costs <= tcost + 1e-6) >= 0.9
    assert e_trained < 0.5 * e_full
    assert e_trained < 0.5 * e_raw or r0.fallback.mean() > 0.25
