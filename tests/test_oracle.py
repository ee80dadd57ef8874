"""The oracle, pinned: the C restatement against the reference's own sequential
TV-L1 (compiled in place, oracle/_ref) and against the golden fixtures made
from it, plus known-answer and quirk tests.  CPU only."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def params_of(d, oracle):
    return oracle.TVL1Params(float(d["tau"]), float(d["lambda_"]), float(d["theta"]),
                             int(d["nscales"]), float(d["zfactor"]), int(d["warps"]),
                             float(d["epsilon"]), int(d["max_iterations"]))


@pytest.mark.parametrize("name", ["tvl1_97x61.npz", "tvl1_160x96.npz", "tvl1_128x64_w2.npz"])
def test_restatement_matches_golden(orc, name):
    d = load(name)
    u, v = orc.tvl1(d["I0"].astype(np.float32), d["I1"].astype(np.float32), params_of(d, orc),
                    error_mode=0)
    assert np.array_equal(u, d["u"]) and np.array_equal(v, d["v"])


def test_building_blocks_match_golden(orc):
    d = load("tvl1_blocks.npz")
    L = orc.orc_lib()
    img = d["img"]
    ny, nx = img.shape
    for tag, sigma in (("g08", 0.8), ("gz", float(np.float32(0.6 * np.sqrt(3.0))))):
        g = img.copy()
        assert L.orc_gaussian(g, nx, ny, sigma) == 0
        assert np.array_equal(g, d[tag]), tag
    zo = np.zeros_like(d["zoom_out"])
    assert L.orc_zoom_out(img, zo, nx, ny, 0.5) == 0
    assert np.array_equal(zo, d["zoom_out"])
    zi = np.zeros_like(img)
    L.orc_zoom_in(d["zoom_out"], zi, zo.shape[1], zo.shape[0], nx, ny)
    assert np.array_equal(zi, d["zoom_in"])
    for bo in (0, 1):
        w = np.zeros_like(img)
        L.orc_bicubic_warp(img, d["fu"], d["fv"], w, nx, ny, bo)
        assert np.array_equal(w, d[f"warp{bo}"])
        at = np.array([L.orc_bicubic_at(img, float(x), float(y), nx, ny, bo) for x, y in d["pts"]],
                      np.float32)
        assert np.array_equal(at, d[f"at{bo}"])
    dx, dy = np.zeros_like(img), np.zeros_like(img)
    L.orc_centered_gradient(img, dx, dy, nx, ny)
    assert np.array_equal(dx, d["cgx"]) and np.array_equal(dy, d["cgy"])
    div = np.zeros_like(img)
    L.orc_divergence(d["fu"], d["fv"], div, nx, ny)
    assert np.array_equal(div, d["div"])
    gx, gy = np.zeros_like(img), np.zeros_like(img)
    L.orc_forward_gradient(img, gx, gy, nx, ny)
    assert np.array_equal(gx, d["fgx"]) and np.array_equal(gy, d["fgy"])
    n0, n1 = d["n0"].copy(), d["n1"].copy()
    L.orc_normalize(n0, n1, nx * ny)
    assert np.array_equal(n0, d["nn0"]) and np.array_equal(n1, d["nn1"])


def test_level_solve_and_dual_variables_match_golden(orc):
    d = load("tvl1_blocks.npz")
    prm = orc.TVL1Params(max_iterations=7, warps=3)
    u1, u2, p, its, _ = orc.dual_tvl1(d["lvl_I0"], d["lvl_I1"], d["lvl_u1"], d["lvl_u2"], prm, 0)
    assert np.array_equal(u1, d["lvl_out1"]) and np.array_equal(u2, d["lvl_out2"])
    assert np.array_equal(p, d["lvl_p"])


def test_restatement_bit_identical_to_reference(orc, ref):
    from oflow import synth
    for seed, (w, h) in enumerate([(64, 48), (131, 77), (200, 150)]):
        p = synth.tvl1_pair(seed=40 + seed, w=w, h=h, radius=min(w, h) / 5)
        a, b = synth.quantize(p.I0), synth.quantize(p.I1)
        prm = orc.TVL1Params(nscales=100, max_iterations=30)
        ur, vr = orc.ref_tvl1(a, b, prm)
        uo, vo = orc.tvl1(a.astype(np.float32), b.astype(np.float32), prm, error_mode=0)
        assert np.array_equal(ur, uo) and np.array_equal(vr, vo), (w, h)


def test_building_blocks_bit_identical_to_reference_random(orc, ref):
    rng = np.random.default_rng(9)
    L, R = orc.orc_lib(), ref.ref_lib()
    for nx, ny in [(16, 9), (33, 17), (64, 48), (97, 61)]:
        img = rng.uniform(-50, 300, (ny, nx)).astype(np.float32)
        for sigma in (0.8, 1.0392304, 2.0):
            a, b = img.copy(), img.copy()
            ra = L.orc_gaussian(a, nx, ny, sigma)
            rb = R.ref_gaussian(b, nx, ny, sigma) if orc.orc_lib().orc_gaussian_window(sigma) <= ny else ra
            if ra == 0 and rb == 0:
                assert np.array_equal(a, b), (nx, ny, sigma)
        fu = rng.uniform(-6, 6, (ny, nx)).astype(np.float32)
        fv = rng.uniform(-6, 6, (ny, nx)).astype(np.float32)
        for bo in (0, 1):
            wa, wb = np.zeros_like(img), np.zeros_like(img)
            L.orc_bicubic_warp(img, fu, fv, wa, nx, ny, bo)
            R.ref_bicubic_warp(img, fu, fv, wb, nx, ny, bo)
            assert np.array_equal(wa, wb)
        da, db = np.zeros_like(img), np.zeros_like(img)
        L.orc_divergence(fu, fv, da, nx, ny)
        R.ref_divergence(fu, fv, db, nx, ny)
        assert np.array_equal(da, db)
        for fn in ("centered_gradient", "forward_gradient"):
            xa, ya, xb, yb = (np.zeros_like(img) for _ in range(4))
            getattr(L, "orc_" + fn)(img, xa, ya, nx, ny)
            getattr(R, "ref_" + fn)(img, xb, yb, nx, ny)
            assert np.array_equal(xa, xb) and np.array_equal(ya, yb)


def test_dual_level_bit_identical_to_reference(orc, ref):
    from oflow import synth
    p = synth.tvl1_pair(seed=3, w=72, h=56, radius=10.0)
    I0, I1 = p.I0.astype(np.float32), p.I1.astype(np.float32)
    rng = np.random.default_rng(1)
    u1 = rng.uniform(-2, 2, I0.shape).astype(np.float32)
    u2 = rng.uniform(-2, 2, I0.shape).astype(np.float32)
    for iters in (1, 2, 5):
        ref.ref_lib().ref_set_max_iterations(iters)
        a1, a2 = u1.copy(), u2.copy()
        pr = np.zeros((4,) + I0.shape, np.float32)
        ref.ref_lib().ref_dual_tvl1(I0, I1, a1, a2, I0.shape[1], I0.shape[0], 0.25, 0.15, 0.3, 2,
                                    0.01, pr.ctypes.data_as(C.c_void_p))
        b1, b2, po, _, _ = orc.dual_tvl1(I0, I1, u1, u2, orc.TVL1Params(max_iterations=iters, warps=2))
        assert np.array_equal(a1, b1) and np.array_equal(a2, b2) and np.array_equal(pr, po), iters


def test_known_answer_constant_image_gives_zero_flow(orc):
    I = np.full((48, 64), 77.0, np.float32)
    u, v = orc.tvl1(I, I, orc.TVL1Params(nscales=3, max_iterations=20))
    assert np.all(u == 0) and np.all(v == 0)


def test_known_answer_integer_shift(orc):
    rng = np.random.default_rng(2)
    from oflow import synth
    big = synth._blur(rng.uniform(0, 255, (140, 180)), 2.0).astype(np.float32)
    I0 = big[10:130, 10:170]
    I1 = big[10:130, 8:168]  # I1(x + 2) = I0(x)
    u, v = orc.tvl1(synth.quantize(I0).astype(np.float32), synth.quantize(I1).astype(np.float32),
                    orc.TVL1Params(nscales=4, max_iterations=50))
    inner = (slice(12, -12), slice(12, -12))
    assert abs(float(np.median(u[inner])) - 2.0) < 0.05
    assert abs(float(np.median(v[inner]))) < 0.05


def test_bicubic_quirks(orc):
    """Negative coordinates truncate toward zero and step the stencil away from
    zero; the row above the sample uses the x sign (bicubic_interpolation.cpp:
    83-96); with border zeroing any clamped tap gives 0."""
    L = orc.orc_lib()
    img = np.arange(10 * 12, dtype=np.float32).reshape(10, 12) ** 1.3
    img = np.ascontiguousarray(img, np.float32)
    # x in (-1, 0): the stencil clamps -> zero with border_out
    assert L.orc_bicubic_at(img, -0.5, 4.5, 12, 10, 1) == 0.0
    # x in [0, 1): the tap at -1 clamps -> zero with border_out
    assert L.orc_bicubic_at(img, 0.5, 4.5, 12, 10, 1) == 0.0
    # interior sample with integer coordinates is the pixel itself
    assert L.orc_bicubic_at(img, 5.0, 4.0, 12, 10, 1) == img[4, 5]
    # mixed signs without border zeroing: the y stencil steps by sign(x)
    a = L.orc_bicubic_at(img, -0.5, 4.5, 12, 10, 0)
    b = L.orc_bicubic_at(img, 0.5, 4.5, 12, 10, 0)
    assert np.isfinite(a) and np.isfinite(b) and a != b


def test_scales_rule(orc):
    # tvl1.cpp:42-43: N = 1 + log(hypot(w,h)/16)/log(1/zfactor), capped
    assert orc.nscales(1024, 436, 100) == 7
    assert orc.nscales(1024, 436, 5) == 5
    assert orc.nscales(97, 61, 100) == 3


def test_hs_lk_oracle_golden(orc):
    d = load("hs_64x48.npz")
    u, v = orc.hs(d["I0"], d["I1"], 15.0, 1, 1, 50)
    assert np.array_equal(u, d["u"]) and np.array_equal(v, d["v"])
    u, v = orc.hs(d["I0"], d["I1"], 0.2, 3, 2, 20)
    assert np.array_equal(u, d["u3"]) and np.array_equal(v, d["v3"])
    e = load("lk_80x60.npz")
    u, v = orc.pyrlk(e["I0"], e["I1"], 3, 3, 3, 5)
    assert np.array_equal(u, e["pu"]) and np.array_equal(v, e["pv"])
    u, v = orc.lk_ring([e["f0"], e["f1"]], 1, 3, 2, 5)
    assert np.array_equal(u, e["su"]) and np.array_equal(v, e["sv"])


def test_hs_oracle_recovers_translation(orc):
    from oflow import synth
    q = synth.hs_pair(seed=0, w=160, h=120, shift=(0.6, -0.4), angle_deg=0.0)
    u, v = orc.hs(q.I0, q.I1, 15.0, 1, 1, 300)
    m = (slice(10, -10), slice(10, -10))
    assert abs(float(np.median(u[m])) - 0.6) < 0.1
    assert abs(float(np.median(v[m])) + 0.4) < 0.1


def test_lk_oracle_ring_order_and_borders(orc):
    """Newest frame in slot iframe % T; derivatives on the oldest; the border of
    width window//2 is zero."""
    rng = np.random.default_rng(4)
    from oflow import synth
    base = synth._blur(rng.uniform(0, 255, (60, 80)), 2.0)
    f_old = synth.quantize(base[:, 1:-1])
    f_new = synth.quantize(base[:, 0:-2])  # content moves right by one pixel
    u1, v1 = orc.lk_ring([f_new, f_old], 0, 3, 2, 5)  # newest in slot 0
    u2, v2 = orc.lk_ring([f_old, f_new], 1, 3, 2, 5)  # newest in slot 1
    assert np.array_equal(u1, u2) and np.array_equal(v1, v2)
    assert np.all(u1[:2] == 0) and np.all(u1[:, :2] == 0) and np.all(u1[-2:] == 0)
    assert float(np.median(u1[5:-5, 5:-5])) > 0.5


def test_flow_to_color_known_answers(orc):
    """flowToColor restatement (main.cpp:93-126): V = round(10|f|) capped at
    255, H = round(deg/2) with negative angles at 0, S = 255, hexcone BGR."""
    u = np.array([[1, 0, 0, -1, 3, 30, 0]], np.float32)
    v = np.array([[0, 1, -1, 0, 3, 0, 0]], np.float32)
    got = orc.flow_to_color(u, v)[0].tolist()
    assert got == [[0, 0, 10],      # 0 deg: red
                   [0, 10, 5],      # 90 deg: H 45, sector 1
                   [0, 0, 10],      # -90 deg saturates to H 0
                   [10, 10, 0],     # 180 deg: H 90, sector 3
                   [0, 31, 42],     # 45 deg: H 22 (22.5 rounds to even), |f| 4.24
                   [0, 0, 255],     # magnitude capped
                   [0, 0, 0]]       # zero flow
