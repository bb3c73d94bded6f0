"""Test infrastructure: a torch float64 restatement of the proposal network of
``cugridsearch_b200/csrc/cgs_net.cu``, used only by the tests to check the CUDA forward pass
and gradients.  It is a floating-point model, so the reference is torch (float64 on the CPU)
rather than C: autograd supplies the gradients, and the places where the CUDA path rounds to
BF16 are mirrored:

* the input planes, the convolution weights and every convolution output (after ReLU) are
  rounded to BF16 in the forward pass (gradients pass straight through the rounding);
* the gradient w.r.t. each convolution's pre-activation (after the ReLU mask) is rounded to
  BF16 in the backward pass, as the CUDA path stores it;
* sums run in float64 here and in FP32 on the GPU: the tests compare with a tolerance.

With ``bf16=False`` no rounding happens and the model is a plain float64 network (used to
check the analytic gradients against finite differences).

Parameter layout (flat): per conv layer W[Cout][Kp] (k = (3 ky + kx) Cin + ci, Kp = 9 Cin
rounded up to 32, padding zero) and b[Cout]; fc1 W[128][256], b[128]; fc2 W[16][128], b[16].
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

CIN = [2, 32, 64, 128, 128]
COUT = [32, 64, 128, 128, 256]
FEAT, HID, OUT = 256, 128, 16
S_MIN, S_MAX = -6.0, 4.0


def kpad(l: int) -> int:
    return (9 * CIN[l] + 31) // 32 * 32


def layout():
    """Offsets of (w_l, b_l) for the conv layers, then fc1 w/b, fc2 w/b, and the total."""
    off, o = {}, 0
    for l in range(5):
        off[f"w{l}"] = (o, (COUT[l], kpad(l)))
        o += COUT[l] * kpad(l)
        off[f"b{l}"] = (o, (COUT[l],))
        o += COUT[l]
    for name, shape in (("fc1w", (HID, FEAT)), ("fc1b", (HID,)), ("fc2w", (OUT, HID)), ("fc2b", (OUT,))):
        off[name] = (o, shape)
        o += int(np.prod(shape))
    return off, o


def _bf16(t):
    return t.to(torch.bfloat16).to(t.dtype)


class _RoundST(torch.autograd.Function):
    """Forward: round to BF16; backward: identity."""

    @staticmethod
    def forward(ctx, x):
        return _bf16(x)

    @staticmethod
    def backward(ctx, g):
        return g


class _RoundGrad(torch.autograd.Function):
    """Forward: identity; backward: round the gradient to BF16."""

    @staticmethod
    def forward(ctx, x):
        return x.clone()

    @staticmethod
    def backward(ctx, g):
        return _bf16(g)


def unflatten(flat: torch.Tensor) -> dict:
    off, _ = layout()
    return {k: flat[o:o + int(np.prod(sh))].view(*sh) for k, (o, sh) in off.items()}


def net_input(fixed: np.ndarray, moving: np.ndarray, bf16: bool = True) -> torch.Tensor:
    """(n, 2, 128, 128) float64 input: box average to 128 and (v - 127.5) / 64."""
    f = torch.from_numpy(np.asarray(fixed, np.float64))
    m = torch.from_numpy(np.asarray(moving, np.float64))
    n, side = f.shape[0], f.shape[-1]
    s = side // 128
    x = torch.stack([f, m], 1).reshape(n, 2, 128, s, 128, s).mean(dim=(3, 5))
    x = (x - 127.5) / 64.0
    return _bf16(x) if bf16 else x


def forward(flat: torch.Tensor, x: torch.Tensor, bf16: bool = True) -> torch.Tensor:
    """The network's 16 outputs per pair (float64)."""
    P = unflatten(flat)
    a = x
    for l in range(5):
        w = P[f"w{l}"][:, : 9 * CIN[l]].reshape(COUT[l], 3, 3, CIN[l]).permute(0, 3, 1, 2)
        if bf16:
            w = _RoundST.apply(w)
        z = F.conv2d(a, w, P[f"b{l}"], stride=2, padding=1)
        if bf16:
            z = _RoundGrad.apply(z)
        a = F.relu(z)
        if bf16:
            a = _RoundST.apply(a)
    g = a.mean(dim=(2, 3))
    h = F.relu(g @ P["fc1w"].T + P["fc1b"])
    return h @ P["fc2w"].T + P["fc2b"]


def loss(out: torch.Tensor, labels: torch.Tensor) -> torch.Tensor:
    """Mean Laplace negative log-likelihood |c - y| e^-s + s, s clamped to [-6, 4]."""
    c, s = out[:, :8], torch.clamp(out[:, 8:], S_MIN, S_MAX)
    return ((c - labels).abs() * torch.exp(-s) + s).mean()


def loss_and_grads(params: np.ndarray, fixed: np.ndarray, moving: np.ndarray, labels: np.ndarray,
                   bf16: bool = True):
    """(outputs, loss, flat gradient) of the network at params on a batch."""
    flat = torch.tensor(np.asarray(params, np.float64), requires_grad=True)
    x = net_input(fixed, moving, bf16)
    out = forward(flat, x, bf16)
    L = loss(out, torch.from_numpy(np.asarray(labels, np.float64)))
    L.backward()
    return out.detach().numpy(), float(L.detach()), flat.grad.numpy()
