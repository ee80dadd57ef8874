"""Generates the golden fixtures in this directory.

TV-L1 fixtures come from the reference's own sequential TV-L1
(src/tvl1/sequential, compiled in place into oracle/_ref by
oracle/build_ref.sh), run single-threaded (OMP_NUM_THREADS=1) so its float
error sum has a fixed order.  The reference has no HS or LK CPU code and no
test vectors of its own; the HS/LK fixtures are outputs of the oracle
restatement, kept to catch regressions.

Run from the repository root:  OMP_NUM_THREADS=1 python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

os.environ.setdefault("OMP_NUM_THREADS", "1")
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "sycl-optic-flow_b200")]

import ctypes as C  # noqa: E402

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from oflow import synth  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def tvl1_cases(ref):
    cases = {}
    specs = [
        ("tvl1_97x61", dict(seed=11, w=97, h=61, radius=12.0), dict(nscales=100, max_iterations=50)),
        ("tvl1_160x96", dict(seed=12, w=160, h=96, radius=20.0), dict(nscales=3, max_iterations=20)),
        ("tvl1_128x64_w2", dict(seed=13, w=128, h=64, radius=15.0),
         dict(nscales=2, warps=2, max_iterations=300, epsilon=0.05)),
    ]
    for name, g, prm in specs:
        p = synth.tvl1_pair(**g)
        a, b = synth.quantize(p.I0), synth.quantize(p.I1)
        par = oracle.TVL1Params(**prm)
        u, v = oracle.ref_tvl1(a, b, par)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), I0=a, I1=b, u=u, v=v,
                            tau=par.tau, lambda_=par.lambda_, theta=par.theta,
                            nscales=par.nscales, zfactor=par.zfactor, warps=par.warps,
                            epsilon=par.epsilon, max_iterations=par.max_iterations)
        cases[name] = float(np.abs(u).mean())
    return cases


def blocks(ref):
    rng = np.random.default_rng(5)
    nx, ny = 37, 23
    img = f32(rng.uniform(0, 255, (ny, nx)))
    d = {"img": img}
    for tag, sigma in (("g08", 0.8), ("gz", float(np.float32(0.6 * np.sqrt(3.0))))):
        g = img.copy()
        assert ref.ref_lib().ref_gaussian(g, nx, ny, sigma) == 0
        d[tag] = g
    zo = np.zeros((12, 19), np.float32)
    assert ref.ref_lib().ref_zoom_out(img, zo, nx, ny, 0.5) == 0
    d["zoom_out"] = zo
    zi = np.zeros((ny, nx), np.float32)
    ref.ref_lib().ref_zoom_in(zo, zi, 19, 12, nx, ny)
    d["zoom_in"] = zi
    fu = f32(rng.uniform(-3, 3, (ny, nx)))
    fv = f32(rng.uniform(-3, 3, (ny, nx)))
    d["fu"], d["fv"] = fu, fv
    for bo in (0, 1):
        w = np.zeros_like(img)
        ref.ref_lib().ref_bicubic_warp(img, fu, fv, w, nx, ny, bo)
        d[f"warp{bo}"] = w
    dx, dy = np.zeros_like(img), np.zeros_like(img)
    ref.ref_lib().ref_centered_gradient(img, dx, dy, nx, ny)
    d["cgx"], d["cgy"] = dx, dy
    div = np.zeros_like(img)
    ref.ref_lib().ref_divergence(fu, fv, div, nx, ny)
    d["div"] = div
    gx, gy = np.zeros_like(img), np.zeros_like(img)
    ref.ref_lib().ref_forward_gradient(img, gx, gy, nx, ny)
    d["fgx"], d["fgy"] = gx, gy
    n0 = f32(rng.uniform(10, 120, (ny, nx)))
    n1 = f32(rng.uniform(5, 90, (ny, nx)))
    o0, o1 = np.zeros_like(n0), np.zeros_like(n1)
    ref.ref_lib().ref_normalize(n0, n1, o0, o1, nx * ny)
    d["n0"], d["n1"], d["nn0"], d["nn1"] = n0, n1, o0, o1
    # bicubic samples, including negative coordinates and mixed signs (the
    # stencil row above uses the x sign)
    pts = np.array([[3.25, 4.5], [-0.5, 2.25], [2.5, -0.75], [-1.5, -2.5], [0.0, 0.0],
                    [35.9, 21.9], [36.5, 22.5], [17.3, 11.7], [1.0, 20.99], [-0.25, 10.5]],
                   np.float32)
    for bo in (0, 1):
        d[f"at{bo}"] = np.array([ref.ref_lib().ref_bicubic_at(img, float(x), float(y), nx, ny, bo)
                                 for x, y in pts], np.float32)
    d["pts"] = pts
    # one pyramid level of dualTVL1 (tvl1.cpp:182-294) with the dual variables
    p = synth.tvl1_pair(seed=21, w=48, h=40, radius=8.0)
    I0, I1 = f32(p.I0), f32(p.I1)
    u1 = f32(rng.uniform(-1, 1, I0.shape))
    u2 = f32(rng.uniform(-1, 1, I0.shape))
    uo1, uo2 = u1.copy(), u2.copy()
    pp = np.zeros((4, 40, 48), np.float32)
    ref.ref_lib().ref_set_max_iterations(7)
    ref.ref_lib().ref_dual_tvl1(I0, I1, uo1, uo2, 48, 40, 0.25, 0.15, 0.3, 3, 0.01,
                                pp.ctypes.data_as(C.c_void_p))
    d.update(lvl_I0=I0, lvl_I1=I1, lvl_u1=u1, lvl_u2=u2, lvl_out1=uo1, lvl_out2=uo2, lvl_p=pp)
    np.savez_compressed(os.path.join(OUT, "tvl1_blocks.npz"), **d)


def hs_lk_cases():
    q = synth.hs_pair(seed=4, w=64, h=48)
    u, v = oracle.hs(q.I0, q.I1, 15.0, 1, 1, 50)
    u3, v3 = oracle.hs(q.I0, q.I1, 0.2, 3, 2, 20)
    np.savez_compressed(os.path.join(OUT, "hs_64x48.npz"), I0=q.I0, I1=q.I1, u=u, v=v, u3=u3, v3=v3)
    l = synth.lk_pair(seed=6, w=80, h=60)
    pu, pv = oracle.pyrlk(l.I0, l.I1, 3, 3, 3, 5)
    fr = [synth.quantize(l.I0), synth.quantize(l.I1)]
    su, sv = oracle.lk_ring(fr, 1, 3, 2, 5)
    np.savez_compressed(os.path.join(OUT, "lk_80x60.npz"), I0=l.I0, I1=l.I1, pu=pu, pv=pv,
                        f0=fr[0], f1=fr[1], su=su, sv=sv)


if __name__ == "__main__":
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref not built: run oracle/build_ref.sh first")
    print(tvl1_cases(oracle))
    blocks(oracle)
    hs_lk_cases()
    print("golden fixtures written to", OUT)
