"""Seeded synthetic frame pairs with known ground-truth flow.

The reference ships four video clips without ground truth and needs OpenCV to
read them; here every workload is generated from a seed instead, with the
shapes and value distributions of the benchmark configurations:

* ``hs_pair``    320x240 blurred uniform noise, rigid motion (translation
                 (1.5, -0.75) px + 2 degree rotation about the centre).
* ``lk_pair``    640x480 4-octave value noise, smooth vortex (peak 8 px) and
                 N(0, 1) pixel noise.
* ``tvl1_pair``  1024x436 blurred noise, affine background (<= 4 px) and
                 0-3 discs of radius 80 moving independently (occlusions),
                 N(0, 2) pixel noise.

Flow convention (shared with the solvers): u is the displacement of a
frame-0 pixel into frame 1, so I1(x + u(x)) ~= I0(x).  Frames are float32 in
[0, 255]; ``quantize`` gives the uint8 bytes used for parity runs.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Pair:
    I0: np.ndarray            # float32 [h, w]
    I1: np.ndarray            # float32 [h, w]
    u: np.ndarray             # ground-truth flow, float32 [h, w]
    v: np.ndarray
    valid: np.ndarray         # bool [h, w]: not occluded, target inside the frame
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return self.I0.shape


def quantize(img: np.ndarray) -> np.ndarray:
    """Round half to even and clip to uint8."""
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def _blur(img: np.ndarray, sigma: float) -> np.ndarray:
    r = int(np.ceil(3 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-x * x / (2 * sigma * sigma))
    k /= k.sum()
    pad = np.pad(img.astype(np.float64), r, mode="reflect")
    tmp = np.zeros((pad.shape[0], img.shape[1]))
    for i, kv in enumerate(k):
        tmp += kv * pad[:, i:i + img.shape[1]]
    out = np.zeros(img.shape)
    for i, kv in enumerate(k):
        out += kv * tmp[i:i + img.shape[0], :]
    return out


def _stretch(img: np.ndarray, lo=0.0, hi=255.0) -> np.ndarray:
    a, b = img.min(), img.max()
    return (lo + (img - a) * (hi - lo) / max(b - a, 1e-12)).astype(np.float64)


def bilinear(img: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Sample img at float coordinates, clamp-to-edge."""
    h, w = img.shape
    x = np.clip(x, 0, w - 1)
    y = np.clip(y, 0, h - 1)
    x0 = np.floor(x).astype(np.int64)
    y0 = np.floor(y).astype(np.int64)
    x1 = np.minimum(x0 + 1, w - 1)
    y1 = np.minimum(y0 + 1, h - 1)
    fx = x - x0
    fy = y - y0
    top = img[y0, x0] * (1 - fx) + img[y0, x1] * fx
    bot = img[y1, x0] * (1 - fx) + img[y1, x1] * fx
    return top * (1 - fy) + bot * fy


def _invert(flow_fn, gx, gy, iters=8):
    """Solve x + u(x) = y for x by fixed-point iteration (smooth flows)."""
    x, y = gx.copy(), gy.copy()
    for _ in range(iters):
        u, v = flow_fn(x, y)
        x, y = gx - u, gy - v
    return x, y


def noise_texture(rng, h, w, sigma=2.0, margin=0):
    return _stretch(_blur(rng.uniform(0, 255, (h + 2 * margin, w + 2 * margin)), sigma))


def value_noise(rng, h, w, octaves=4, persistence=0.5, base_cell=32.0):
    out = np.zeros((h, w))
    amp, cell = 1.0, base_cell
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    for _ in range(octaves):
        gh, gw = int(np.ceil(h / cell)) + 2, int(np.ceil(w / cell)) + 2
        grid = rng.uniform(0, 1, (gh, gw))
        gx, gy = xx / cell, yy / cell
        x0, y0 = np.floor(gx).astype(int), np.floor(gy).astype(int)
        tx, ty = gx - x0, gy - y0
        sx, sy = tx * tx * (3 - 2 * tx), ty * ty * (3 - 2 * ty)
        a = grid[y0, x0] * (1 - sx) + grid[y0, x0 + 1] * sx
        b = grid[y0 + 1, x0] * (1 - sx) + grid[y0 + 1, x0 + 1] * sx
        out += amp * (a * (1 - sy) + b * sy)
        amp *= persistence
        cell /= 2
    return _stretch(out)


def hs_pair(seed=0, w=320, h=240, shift=(1.5, -0.75), angle_deg=2.0) -> Pair:
    """Config 0: blurred uniform noise, rigid motion about the centre."""
    rng = np.random.default_rng(seed)
    I0 = _stretch(_blur(rng.uniform(0, 255, (h, w)), 2.0))
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    th = np.deg2rad(angle_deg)
    c, s = np.cos(th), np.sin(th)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    # T(x) = R (x - c) + c + t; u = T(x) - x
    tx = c * (xx - cx) - s * (yy - cy) + cx + shift[0]
    ty = s * (xx - cx) + c * (yy - cy) + cy + shift[1]
    u, v = tx - xx, ty - yy
    # I1(y) = I0(T^-1 y)
    bx, by = xx - cx - shift[0], yy - cy - shift[1]
    sx = c * bx + s * by + cx
    sy = -s * bx + c * by + cy
    I1 = bilinear(I0, sx, sy)
    valid = (tx >= 0) & (tx <= w - 1) & (ty >= 0) & (ty <= h - 1)
    return Pair(I0.astype(np.float32), I1.astype(np.float32), u.astype(np.float32),
                v.astype(np.float32), valid, {"config": "hs", "seed": seed})


def lk_pair(seed=0, w=640, h=480, peak=8.0, noise=1.0) -> Pair:
    """Config 1: value noise, smooth vortex flow, N(0, noise) pixel noise."""
    rng = np.random.default_rng(seed)
    I0 = value_noise(rng, h, w)
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    sig = 0.25 * min(w, h)

    def flow(x, y):
        dx, dy = x - cx, y - cy
        r2 = dx * dx + dy * dy
        # tangential field; |u| peaks at r = sig with value `peak`
        g = peak * np.exp(0.5) / sig * np.exp(-r2 / (2 * sig * sig))
        return -dy * g, dx * g

    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    u, v = flow(xx, yy)
    sx, sy = _invert(flow, xx, yy)
    I1 = bilinear(I0, sx, sy) + rng.normal(0, noise, (h, w))
    I0n = I0 + 0.0
    valid = (xx + u >= 0) & (xx + u <= w - 1) & (yy + v >= 0) & (yy + v <= h - 1)
    return Pair(I0n.astype(np.float32), np.clip(I1, 0, 255).astype(np.float32),
                u.astype(np.float32), v.astype(np.float32), valid,
                {"config": "lk", "seed": seed})


def tvl1_pair(seed=0, w=1024, h=436, ndiscs=1, speed=None, radius=80.0, noise=2.0,
              bg_max=4.0) -> Pair:
    """Config 2 (and the warm-start training generator): affine background
    (|u| <= bg_max over the frame) plus `ndiscs` textured discs of `radius`
    px.  With ndiscs=1 and speed=None the disc moves (12, -5) px."""
    rng = np.random.default_rng(seed)
    m = 24
    bg = noise_texture(rng, h, w, 2.0, margin=m)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    # affine background: translation + small linear part, scaled to bg_max
    t = rng.uniform(-1, 1, 2)
    M = rng.uniform(-1, 1, (2, 2)) / max(w, h)
    ub = t[0] + M[0, 0] * (xx - cx) + M[0, 1] * (yy - cy)
    vb = t[1] + M[1, 0] * (xx - cx) + M[1, 1] * (yy - cy)
    mag = np.sqrt(ub * ub + vb * vb).max()
    k = bg_max * rng.uniform(0.5, 1.0) / max(mag, 1e-9)
    t, M = t * k, M * k

    def bg_flow(x, y):
        return (t[0] + M[0, 0] * (x - cx) + M[0, 1] * (y - cy),
                t[1] + M[1, 0] * (x - cx) + M[1, 1] * (y - cy))

    ub, vb = bg_flow(xx, yy)
    sx, sy = _invert(bg_flow, xx, yy)
    I0 = bg[m:m + h, m:m + w].copy()
    I1 = bilinear(bg, sx + m, sy + m)
    u, v = ub.copy(), vb.copy()
    occl = np.zeros((h, w), bool)
    discs = []
    for d in range(ndiscs):
        if speed is None and ndiscs == 1:
            dv = np.array([12.0, -5.0])
            c0 = np.array([w * 0.45, h * 0.5])
        else:
            sp = rng.uniform(0, speed if speed is not None else 16.0)
            a = rng.uniform(0, 2 * np.pi)
            dv = np.array([sp * np.cos(a), sp * np.sin(a)])
            c0 = np.array([rng.uniform(radius, w - radius), rng.uniform(radius, h - radius)])
        tex = noise_texture(rng, int(2 * radius + 4), int(2 * radius + 4), 2.0)
        discs.append((c0, dv, tex))
    # frame 0: discs painted in order over the background
    for c0, dv, tex in discs:
        inside0 = (xx - c0[0]) ** 2 + (yy - c0[1]) ** 2 <= radius * radius
        I0[inside0] = bilinear(tex, xx[inside0] - c0[0] + radius + 2,
                               yy[inside0] - c0[1] + radius + 2)
        u[inside0] = dv[0]
        v[inside0] = dv[1]
    # frame 1: discs at their moved centres
    for c0, dv, tex in discs:
        c1 = c0 + dv
        inside1 = (xx - c1[0]) ** 2 + (yy - c1[1]) ** 2 <= radius * radius
        I1[inside1] = bilinear(tex, xx[inside1] - c1[0] + radius + 2,
                               yy[inside1] - c1[1] + radius + 2)
    # occlusion: the destination of a frame-0 pixel is covered in frame 1 by a
    # disc that the pixel does not belong to
    tx, ty = xx + u, yy + v
    for c0, dv, tex in discs:
        c1 = c0 + dv
        cov = (tx - c1[0]) ** 2 + (ty - c1[1]) ** 2 <= radius * radius
        own = (np.abs(u - dv[0]) < 1e-9) & (np.abs(v - dv[1]) < 1e-9)
        occl |= cov & ~own
    I0 = I0 + rng.normal(0, noise, (h, w))
    I1 = I1 + rng.normal(0, noise, (h, w))
    valid = ~occl & (tx >= 0) & (tx <= w - 1) & (ty >= 0) & (ty <= h - 1)
    return Pair(np.clip(I0, 0, 255).astype(np.float32), np.clip(I1, 0, 255).astype(np.float32),
                u.astype(np.float32), v.astype(np.float32), valid,
                {"config": "tvl1", "seed": seed, "ndiscs": ndiscs})


BATCH_SIZES = [(320, 240), (640, 480), (1024, 436), (1280, 720), (1920, 1080)]


def batch_specs(n=256, seed=0):
    """Config 3: (solver, w, h, seed) for n pairs; sizes uniform over
    BATCH_SIZES, half HS and half TV-L1, in a shuffled order."""
    rng = np.random.default_rng(seed)
    solvers = np.array(["hs"] * (n // 2) + ["tvl1"] * (n - n // 2))
    rng.shuffle(solvers)
    out = []
    for i in range(n):
        w, h = BATCH_SIZES[rng.integers(len(BATCH_SIZES))]
        out.append((str(solvers[i]), int(w), int(h), int(rng.integers(1 << 31))))
    return out


def epe(u, v, gu, gv, mask=None, margin=0):
    """Mean end-point error over `mask` (all pixels if None), ignoring a
    border of `margin` pixels."""
    e = np.sqrt((u - gu) ** 2 + (v - gv) ** 2)
    m = np.ones(e.shape, bool) if mask is None else mask.copy()
    if margin:
        m[:margin, :] = False
        m[-margin:, :] = False
        m[:, :margin] = False
        m[:, -margin:] = False
    return float(e[m].mean()) if m.any() else float("nan")
