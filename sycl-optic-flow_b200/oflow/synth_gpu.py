"""Seeded synthetic pairs generated on the GPU with torch, for workloads too
large for the numpy generator (the 256-pair mixed batch, warm-start training
sets).  Same recipes as oflow.synth: blurred-noise texture, affine background
up to `bg_max` px, textured discs moving independently, Gaussian pixel noise,
uint8 frames.  Flow convention: I1(x + u(x)) = I0(x).

Data generation only: nothing here is on a solver's path.
"""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F


def _gauss_kernel(sigma: float, device):
    r = int(math.ceil(3 * sigma))
    x = torch.arange(-r, r + 1, device=device, dtype=torch.float32)
    k = torch.exp(-x * x / (2 * sigma * sigma))
    return k / k.sum(), r


def blur(img: torch.Tensor, sigma: float) -> torch.Tensor:
    """Separable Gaussian of [N, H, W] (reflect padding)."""
    k, r = _gauss_kernel(sigma, img.device)
    x = img[:, None]
    x = F.conv2d(F.pad(x, (r, r, 0, 0), mode="reflect"), k.view(1, 1, 1, -1))
    x = F.conv2d(F.pad(x, (0, 0, r, r), mode="reflect"), k.view(1, 1, -1, 1))
    return x[:, 0]


def _stretch(x: torch.Tensor) -> torch.Tensor:
    lo = x.amin(dim=(-2, -1), keepdim=True)
    hi = x.amax(dim=(-2, -1), keepdim=True)
    return (x - lo) * (255.0 / (hi - lo).clamp_min(1e-6))


def _sample(img: torch.Tensor, sx: torch.Tensor, sy: torch.Tensor) -> torch.Tensor:
    """Bilinear sample of [N, H, W] at pixel coordinates [N, h, w], clamp to edge."""
    N, H, W = img.shape
    gx = sx / max(W - 1, 1) * 2 - 1
    gy = sy / max(H - 1, 1) * 2 - 1
    grid = torch.stack([gx, gy], dim=-1)
    return F.grid_sample(img[:, None], grid, mode="bilinear", padding_mode="border",
                         align_corners=True)[:, 0]


def tvl1_pairs(n: int, w: int, h: int, seed: int, device="cuda", ndiscs_max: int = 1,
               speed_max: float | None = None, radius: float = 80.0, noise: float = 2.0,
               bg_max: float = 4.0):
    """n pairs of the TV-L1 workload.  ndiscs_max=1 with speed_max=None: one
    disc per pair moving (12, -5) px (the 1024x436 benchmark recipe); otherwise
    0..ndiscs_max discs with speeds uniform up to speed_max.  Returns
    (I0 u8 [n,h,w], I1 u8, u f32, v f32, valid bool)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    m = 24
    bg = _stretch(blur(torch.rand((n, h + 2 * m, w + 2 * m), generator=g, device=device) * 255, 2.0))
    yy, xx = torch.meshgrid(torch.arange(h, device=device, dtype=torch.float32),
                            torch.arange(w, device=device, dtype=torch.float32), indexing="ij")
    xx, yy = xx.expand(n, h, w), yy.expand(n, h, w)
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    t = torch.rand((n, 2, 1, 1), generator=g, device=device) * 2 - 1
    M = (torch.rand((n, 2, 2, 1, 1), generator=g, device=device) * 2 - 1) / max(w, h)
    ub = t[:, 0] + M[:, 0, 0] * (xx - cx) + M[:, 0, 1] * (yy - cy)
    vb = t[:, 1] + M[:, 1, 0] * (xx - cx) + M[:, 1, 1] * (yy - cy)
    mag = torch.sqrt(ub * ub + vb * vb).amax(dim=(-2, -1), keepdim=True)
    k = bg_max * (0.5 + 0.5 * torch.rand((n, 1, 1), generator=g, device=device)) / mag.clamp_min(1e-9)
    ub, vb = ub * k, vb * k
    # inverse of x -> x + (ub, vb)(x) by fixed point (smooth field)
    sx, sy = xx.clone(), yy.clone()
    for _ in range(6):
        fu = _sample(ub, sx, sy)
        fv = _sample(vb, sx, sy)
        sx, sy = xx - fu, yy - fv
    I0 = bg[:, m:m + h, m:m + w].clone()
    I1 = _sample(bg, sx + m, sy + m)
    u, v = ub.clone(), vb.clone()
    occl = torch.zeros((n, h, w), dtype=torch.bool, device=device)
    nd = torch.randint(0, ndiscs_max + 1, (n,), generator=g, device=device) \
        if (speed_max is not None or ndiscs_max != 1) else torch.ones(n, dtype=torch.long, device=device)
    D = int(nd.max().item()) if n else 0
    R = float(min(radius, 0.45 * min(w, h)))
    discs = []
    for d in range(D):
        active = (nd > d).view(n, 1, 1)
        if speed_max is None and ndiscs_max == 1:
            dv = torch.tensor([12.0, -5.0], device=device).expand(n, 2)
            c0 = torch.tensor([w * 0.45, h * 0.5], device=device).expand(n, 2)
        else:
            sp = torch.rand(n, generator=g, device=device) * (speed_max or 16.0)
            ang = torch.rand(n, generator=g, device=device) * 2 * math.pi
            dv = torch.stack([sp * torch.cos(ang), sp * torch.sin(ang)], dim=1)
            c0 = torch.stack([R + torch.rand(n, generator=g, device=device) * (w - 2 * R),
                              R + torch.rand(n, generator=g, device=device) * (h - 2 * R)], dim=1)
        tex = _stretch(blur(torch.rand((n, int(2 * R + 4), int(2 * R + 4)), generator=g,
                                       device=device) * 255, 2.0))
        discs.append((active, c0, dv, tex))
        dx = xx - c0[:, 0, None, None]
        dy = yy - c0[:, 1, None, None]
        inside0 = (dx * dx + dy * dy <= R * R) & active
        val = _sample(tex, dx + R + 2, dy + R + 2)
        I0 = torch.where(inside0, val, I0)
        u = torch.where(inside0, dv[:, 0, None, None].expand(n, h, w), u)
        v = torch.where(inside0, dv[:, 1, None, None].expand(n, h, w), v)
    for active, c0, dv, tex in discs:
        c1 = c0 + dv
        dx = xx - c1[:, 0, None, None]
        dy = yy - c1[:, 1, None, None]
        inside1 = (dx * dx + dy * dy <= R * R) & active
        I1 = torch.where(inside1, _sample(tex, dx + R + 2, dy + R + 2), I1)
    tx, ty = xx + u, yy + v
    for active, c0, dv, tex in discs:
        c1 = c0 + dv
        cov = ((tx - c1[:, 0, None, None]) ** 2 + (ty - c1[:, 1, None, None]) ** 2 <= R * R) & active
        own = ((u - dv[:, 0, None, None]).abs() < 1e-6) & ((v - dv[:, 1, None, None]).abs() < 1e-6)
        occl |= cov & ~own
    I0 = I0 + torch.randn((n, h, w), generator=g, device=device) * noise
    I1 = I1 + torch.randn((n, h, w), generator=g, device=device) * noise
    valid = ~occl & (tx >= 0) & (tx <= w - 1) & (ty >= 0) & (ty <= h - 1)
    q = lambda x: torch.clamp(torch.round(x), 0, 255).to(torch.uint8)
    return q(I0), q(I1), u, v, valid


def hs_pairs(n: int, w: int, h: int, seed: int, device="cuda", shift=(1.5, -0.75),
             angle_deg=2.0):
    """n pairs of the Horn-Schunck workload (blurred noise, rigid motion about
    the centre).  Returns (I0 f32 [n,h,w], I1 f32, u, v)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    I0 = _stretch(blur(torch.rand((n, h, w), generator=g, device=device) * 255, 2.0))
    yy, xx = torch.meshgrid(torch.arange(h, device=device, dtype=torch.float32),
                            torch.arange(w, device=device, dtype=torch.float32), indexing="ij")
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    th = math.radians(angle_deg)
    c, s = math.cos(th), math.sin(th)
    tx = c * (xx - cx) - s * (yy - cy) + cx + shift[0]
    ty = s * (xx - cx) + c * (yy - cy) + cy + shift[1]
    bx, by = xx - cx - shift[0], yy - cy - shift[1]
    sx = (c * bx + s * by + cx).expand(n, h, w)
    sy = (-s * bx + c * by + cy).expand(n, h, w)
    I1 = _sample(I0, sx, sy)
    return I0.contiguous(), I1.contiguous(), (tx - xx).expand(n, h, w), (ty - yy).expand(n, h, w)
