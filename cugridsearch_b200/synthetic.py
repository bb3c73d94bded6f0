"""Seeded synthetic image pairs and grids of the benchmark configurations.

No public dataset is used.  A fixed image is a sum of isotropic Gaussian blobs plus a
sinusoid texture; the moving image is the fixed image warped by a ground-truth homography
so that ``m(q) = f(H q)`` -- the convention the reference's functors sample with
(``calcNewCoordH`` maps a fixed pixel p to ``H^-1 p`` in the moving image,
src/gpu/cudaImageFunctions.cuh:277-285) -- then Gaussian noise (and, for the MI
configuration, a monotone gamma remap and 8-bit quantisation).

Parameter order is the reference's ``[theta, sx, sy, shear, tx, ty, kx, ky]``.  Grids
take ``count`` values from ``lo`` to ``hi`` inclusive (``start = lo``, ``end = hi``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

DEG = math.pi / 180.0
DEFAULT_SEED = 20261203


@dataclass
class Pair:
    fixed: np.ndarray            # (H, W, 1) float32 or uint8
    moving: np.ndarray
    gt: np.ndarray               # (8,) float32 ground-truth parameters
    lo: np.ndarray               # (8,) grid start
    hi: np.ndarray               # (8,) grid end
    count: np.ndarray            # (8,) samples per axis
    cost: str = "ZNCC"
    meta: dict = field(default_factory=dict)

    def grid_args(self):
        return [float(v) for v in self.lo], [float(v) for v in self.hi], [float(v) for v in self.count]


def homography(p, kind: str = "centred", cx: float = 0.0, cy: float = 0.0) -> np.ndarray:
    """3x3 homography (double) of parameter vector p.  ``centred`` is the reference's
    parametersToHomography (src/gpu/cudaImageFunctions.cuh:216-252); ``uncentred`` the
    one inlined in averageAbsoluteDifference (cudaErrorFunctions.cuh:42-57)."""
    th, sx, sy, sh, tx, ty, kx, ky = [float(v) for v in p]
    c, s = math.cos(th), math.sin(th)
    if kind == "uncentred":
        return np.array([[sx * c, sy * sh * c - sy * s, sx * tx],
                         [sx * s, sy * sh * s + sy * c, sy * ty],
                         [kx, ky, 1.0]])
    a2, a4 = cx * kx + 1, cx * ky
    a6 = c * a2 + a4 * s
    t5 = sh * a6 - s * a2 + a4 * c
    b2, b4 = cy * ky + 1, cy * kx
    b6 = s * b2 + b4 * c
    v5 = sh * b6 + c * b2 - b4 * s
    d3 = kx * c + ky * s
    e5 = sh * d3 + ky * c - kx * s
    H = np.array([[sx * a6, sy * t5, cx + tx * a2 - cx * sx * a6 - cy * sy * t5 + a4 * ty],
                  [sx * b6, sy * v5, cy + ty * b2 - cx * sx * b6 - cy * sy * v5 + b4 * tx],
                  [sx * d3, sy * e5, kx * tx + ky * ty - cy * sy * e5 - cx * sx * d3 + 1]])
    return H / H[2, 2]


def blob_image(rng: np.random.Generator, size: int, n_blobs: int, sigma: tuple[float, float],
               amp: tuple[float, float] = (40.0, 200.0), texture: float = 0.2) -> np.ndarray:
    """Sum of ``n_blobs`` Gaussian blobs (centres uniform, sigma and amplitude uniform) plus
    a sinusoid texture of relative amplitude ``texture`` (of the 255 full scale), clipped
    to [0, 255]."""
    yy, xx = np.mgrid[0:size, 0:size].astype(np.float64)
    img = np.zeros((size, size))
    for _ in range(n_blobs):
        cx, cy = rng.uniform(0, size, 2)
        sg = rng.uniform(*sigma)
        a = rng.uniform(*amp)
        img += a * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * sg * sg))
    lx, ly = rng.uniform(size / 12, size / 5, 2)
    ph = rng.uniform(0, 2 * math.pi, 2)
    img += texture * 255.0 * 0.5 * (1 + np.sin(2 * math.pi * xx / lx + ph[0]) * np.sin(2 * math.pi * yy / ly + ph[1]))
    return np.clip(img, 0, 255)


def warp(fixed: np.ndarray, H: np.ndarray) -> np.ndarray:
    """m(q) = f(H q) with bilinear interpolation, zero outside the fixed image."""
    h, w = fixed.shape
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    X = H[0, 0] * xx + H[0, 1] * yy + H[0, 2]
    Y = H[1, 0] * xx + H[1, 1] * yy + H[1, 2]
    Z = H[2, 0] * xx + H[2, 1] * yy + H[2, 2]
    x, y = X / Z, Y / Z
    x0, y0 = np.floor(x), np.floor(y)
    ax, ay = x - x0, y - y0
    out = np.zeros_like(fixed, dtype=np.float64)
    pad = np.zeros((h + 2, w + 2))
    pad[1:-1, 1:-1] = fixed
    ix, iy = x0.astype(np.int64) + 1, y0.astype(np.int64) + 1
    ok = (ix >= 0) & (iy >= 0) & (ix < w + 1) & (iy < h + 1)
    ixc, iyc = np.clip(ix, 0, w), np.clip(iy, 0, h)
    v = ((1 - ax) * (1 - ay) * pad[iyc, ixc] + ax * (1 - ay) * pad[iyc, ixc + 1] +
         (1 - ax) * ay * pad[iyc + 1, ixc] + ax * ay * pad[iyc + 1, ixc + 1])
    out[ok] = v[ok]
    return out


def _ranges(rot_deg, scale, shear, trans, persp):
    lo = np.array([-rot_deg * DEG, 1 - scale, 1 - scale, -shear, -trans, -trans, -persp, -persp], dtype=np.float32)
    hi = np.array([rot_deg * DEG, 1 + scale, 1 + scale, shear, trans, trans, persp, persp], dtype=np.float32)
    return lo, hi


def make_pair(seed: int, size: int, n_blobs: int, sigma: tuple[float, float], lo, hi, count, kind: str,
              noise: float = 2.0, u8: bool = False, gamma: tuple[float, float] | None = None,
              cost: str = "ZNCC", gt_in_grid: float = 1.0) -> Pair:
    rng = np.random.default_rng(seed)
    f = blob_image(rng, size, n_blobs, sigma)
    # ground truth drawn inside the middle gt_in_grid fraction of every range
    mid, half = (lo + hi) / 2.0, (hi - lo) / 2.0 * gt_in_grid
    gt = rng.uniform(mid - half, mid + half).astype(np.float32)
    H = homography(gt, kind, size / 2.0, size / 2.0)
    m = warp(f, H) + rng.normal(0.0, noise, f.shape)
    m = np.clip(m, 0, 255)
    meta = {"seed": seed, "kind": kind}
    if gamma is not None:
        g = float(rng.uniform(*gamma))
        m = 255.0 * (m / 255.0) ** g
        meta["gamma"] = g
    if u8:
        fixed = np.round(f).astype(np.uint8)[:, :, None]
        moving = np.round(np.clip(m, 0, 255)).astype(np.uint8)[:, :, None]
    else:
        fixed = f.astype(np.float32)[:, :, None]
        moving = m.astype(np.float32)[:, :, None]
    return Pair(fixed, moving, gt, np.asarray(lo, np.float32), np.asarray(hi, np.float32),
                np.asarray(count, np.float32), cost, meta)


def config0(seed: int = DEFAULT_SEED) -> Pair:
    """64x64 f32, 12 blobs (sigma 3-10), rotation +-10 deg, scale 0.9-1.1, shear +-0.05,
    translation +-6 px, perspective +-1e-4; 4 values per parameter; SAD over the overlap
    (the reference's averageAbsoluteDifference and its uncentred parametrisation)."""
    lo, hi = _ranges(10, 0.1, 0.05, 6, 1e-4)
    return make_pair(seed, 64, 12, (3, 10), lo, hi, [4] * 8, "uncentred", cost="SAD_AVG")


def config1(seed: int = DEFAULT_SEED) -> Pair:
    """256x256 f32, 40 blobs with sigma x4 (12-40), translation +-24 px, 6 values per
    parameter (1,679,616 points); zero-mean NCC."""
    lo, hi = _ranges(10, 0.1, 0.05, 24, 1e-4)
    return make_pair(seed, 256, 40, (12, 40), lo, hi, [6] * 8, "centred", cost="ZNCC")


def config2(seed: int = DEFAULT_SEED) -> Pair:
    """512x512 u8 (quantised generator, 40 blobs sigma 24-80), moving image gamma-remapped
    (gamma 0.6-1.6), 5 values per parameter (390,625 points), MI with 32 x 32 bins."""
    lo, hi = _ranges(10, 0.1, 0.05, 48, 1e-4)
    return make_pair(seed, 512, 40, (24, 80), lo, hi, [5] * 8, "centred", u8=True, gamma=(0.6, 1.6), cost="MI")


def config3_pairs(seed: int = DEFAULT_SEED, n: int = 64) -> list[Pair]:
    """64 pairs, square sizes log-uniform in [128, 1024], f32; costs cycle SAD / NCC / MI;
    translation range scaled to the size; 4-6 values per parameter.  Images follow the NCC
    pair's recipe scaled to the size (40 blobs, sigma 12-40 px at 256 px), so larger pairs are
    as textured as the benchmark pair rather than saturated."""
    rng = np.random.default_rng(seed)
    pairs = []
    costs = ["SAD_AVG", "ZNCC", "MI"]
    for i in range(n):
        size = int(round(math.exp(rng.uniform(math.log(128), math.log(1024)))))
        cnt = [int(rng.integers(4, 7)) for _ in range(8)]
        cost = costs[i % 3]
        lo, hi = _ranges(10, 0.1, 0.05, 24.0 * size / 256.0, 1e-4)
        kind = "uncentred" if cost == "SAD_AVG" else "centred"
        pairs.append(make_pair(seed + 1 + i, size, 40, (12.0 * size / 256.0, 40.0 * size / 256.0), lo, hi, cnt, kind,
                               cost=cost))
    return pairs


def config4(seed: int = DEFAULT_SEED) -> Pair:
    """256x256 f32 from the config-0 generator with rotation +-20 deg, translation +-32 px;
    full grid 6 values per parameter."""
    lo, hi = _ranges(20, 0.1, 0.05, 32, 1e-4)
    return make_pair(seed, 256, 40, (12, 40), lo, hi, [6] * 8, "centred", cost="ZNCC")


def small_pair(seed: int, size: int = 32, count: int = 3, cost: str = "ZNCC", u8: bool = False,
               channels: int = 1, kind: str | None = None, msize: int | None = None) -> Pair:
    """A small pair for parity tests (oracle-sized)."""
    kind = kind or ("uncentred" if cost == "SAD_AVG" else "centred")
    lo, hi = _ranges(8, 0.08, 0.05, size * 0.1, 2e-4 if size <= 64 else 1e-4)
    p = make_pair(seed, size, max(6, size // 6), (size / 16.0, size / 5.0), lo, hi, [count] * 8, kind, u8=u8,
                  cost=cost)
    if msize is not None and msize != size:
        rng = np.random.default_rng(seed + 7)
        src = p.moving[:, :, 0].astype(np.float64)
        yy, xx = np.mgrid[0:msize, 0:msize]
        m = src[np.clip(yy, 0, size - 1), np.clip(xx, 0, size - 1)] + rng.normal(0, 1, (msize, msize))
        m = np.clip(m, 0, 255)
        p.moving = (np.round(m).astype(np.uint8) if u8 else m.astype(np.float32))[:, :, None]
    if channels > 1:
        rng = np.random.default_rng(seed + 11)
        def extra(img):
            planes = [img[:, :, 0]]
            for c in range(1, channels):
                noise = rng.normal(0, 3.0, img.shape[:2])
                planes.append(np.clip(img[:, :, 0].astype(np.float64) * (1.0 - 0.2 * c) + noise, 0, 255))
            st = np.stack(planes, axis=-1)
            return np.round(st).astype(np.uint8) if u8 else st.astype(np.float32)
        p.fixed, p.moving = extra(p.fixed), extra(p.moving)
    return p


def config4_ranges(side: int = 256):
    """Grid ranges of the learned-proposal configuration for images of `side` pixels: rotation
    +-20 deg, scale 0.9-1.1, shear +-0.05, translation +-32 px and perspective +-1e-4 at 256 px
    (translation scales with the side, perspective inversely)."""
    f = side / 256.0
    return _ranges(20, 0.1, 0.05, 32 * f, 1e-4 / f)


def config4_batch(seed: int, n: int, device, side: int = 256, scene: bool = False):
    """n pairs of the learned-proposal configuration generated on the GPU with torch (training
    and evaluation data; same distribution as config4(), not the same numbers): 40 blobs with
    sigma 12-40 px (at 256 px) plus the sinusoid texture, the moving image m(q) = f(H q) for a
    ground-truth H drawn uniformly in the grid ranges (centred parametrisation), Gaussian noise
    sigma 2, clipped to [0, 255].  Returns (fixed, moving, gt) as float32 tensors of shapes
    (n, side, side), (n, side, side), (n, 8).

    scene=False: f is the fixed image, zero outside it, so the moving image is black where H q
    leaves the fixed image.  scene=True: f continues beyond the fixed image's edges as its
    mirror image (reflection padding by half a side), so every moving pixel sees content; the
    fixed images are the same."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(int(seed))
    u = lambda *shape: torch.rand(*shape, generator=g, dtype=torch.float64)
    f = side / 256.0
    lo, hi = config4_ranges(side)
    lo_t, hi_t = torch.tensor(lo, dtype=torch.float64), torch.tensor(hi, dtype=torch.float64)
    gt = (lo_t + (hi_t - lo_t) * u(n, 8)).float()
    cx, cy = u(n, 40) * side, u(n, 40) * side
    sg = (12 + 28 * u(n, 40)) * f
    amp = 40 + 160 * u(n, 40)
    lx, ly = side / 12 + (side / 5 - side / 12) * u(n), side / 12 + (side / 5 - side / 12) * u(n)
    ph = 2 * math.pi * u(n, 2)
    noise_seed = int(torch.randint(0, 2 ** 62, (1,), generator=g))
    dev = torch.device(device)
    yy, xx = torch.meshgrid(torch.arange(side, device=dev, dtype=torch.float32),
                            torch.arange(side, device=dev, dtype=torch.float32), indexing="ij")
    img = torch.zeros((n, side, side), device=dev, dtype=torch.float32)
    for b in range(40):
        c_x, c_y = cx[:, b].float().to(dev)[:, None, None], cy[:, b].float().to(dev)[:, None, None]
        s2 = (2 * sg[:, b] ** 2).float().to(dev)[:, None, None]
        img += amp[:, b].float().to(dev)[:, None, None] * torch.exp(-((xx - c_x) ** 2 + (yy - c_y) ** 2) / s2)
    tx = torch.sin(2 * math.pi * xx / lx.float().to(dev)[:, None, None] + ph[:, 0].float().to(dev)[:, None, None])
    ty = torch.sin(2 * math.pi * yy / ly.float().to(dev)[:, None, None] + ph[:, 1].float().to(dev)[:, None, None])
    img += 0.2 * 255.0 * 0.5 * (1 + tx * ty)
    fixed = img.clamp_(0, 255)
    margin = side // 2 if scene else 0
    cs = side + 2 * margin
    canvas = (torch.nn.functional.pad(fixed[:, None], (margin,) * 4, mode="reflect")[:, 0] if scene else fixed)
    H = torch.tensor(np.stack([homography(p, "centred", side / 2.0, side / 2.0) for p in gt.numpy()]),
                     dtype=torch.float32, device=dev)
    X = H[:, 0, 0, None, None] * xx + H[:, 0, 1, None, None] * yy + H[:, 0, 2, None, None]
    Y = H[:, 1, 0, None, None] * xx + H[:, 1, 1, None, None] * yy + H[:, 1, 2, None, None]
    Z = H[:, 2, 0, None, None] * xx + H[:, 2, 1, None, None] * yy + H[:, 2, 2, None, None]
    x, y = X / Z + margin, Y / Z + margin  # canvas coordinates
    x0, y0 = torch.floor(x), torch.floor(y)
    ax, ay = x - x0, y - y0
    pad = torch.nn.functional.pad(canvas, (1, 1, 1, 1))
    ix, iy = x0.long() + 1, y0.long() + 1
    ok = (ix >= 0) & (iy >= 0) & (ix < cs + 1) & (iy < cs + 1)
    ixc, iyc = ix.clamp(0, cs), iy.clamp(0, cs)
    flat = pad.reshape(n, -1)
    w2 = cs + 2

    def tap(dy, dx):
        return torch.gather(flat, 1, ((iyc + dy) * w2 + ixc + dx).reshape(n, -1)).reshape(n, side, side)

    m = ((1 - ax) * (1 - ay) * tap(0, 0) + ax * (1 - ay) * tap(0, 1) + (1 - ax) * ay * tap(1, 0) +
         ax * ay * tap(1, 1))
    m = torch.where(ok, m, torch.zeros_like(m))
    gn = torch.Generator(device=dev).manual_seed(noise_seed)
    m = (m + 2.0 * torch.randn(m.shape, generator=gn, device=dev)).clamp_(0, 255)
    return fixed.contiguous(), m.contiguous(), gt
