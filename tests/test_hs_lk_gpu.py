"""Horn-Schunck and Lucas-Kanade on the GPU through the C ABI against the
oracle restatements (bit-identical by construction: same operation order, no
FMA) and the golden fixtures."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(a, b)


@pytest.mark.parametrize("alpha,L,nw,ns,w,h", [(15.0, 1, 1, 200, 320, 240), (0.2, 3, 2, 30, 320, 240),
                                               (5.0, 2, 3, 7, 131, 77), (1.0, 1, 1, 1, 33, 17)])
def test_hs_bit_identical_to_oracle(of, orc, ctx, alpha, L, nw, ns, w, h):
    from oflow import synth
    q = synth.hs_pair(seed=w + h, w=w, h=h)
    u, v = of.hs(q.I0, q.I1, of.HSParams(alpha, L, nw, ns), ctx)
    ou, ov = orc.hs(q.I0, q.I1, alpha, L, nw, ns)
    assert _same(u, ou) and _same(v, ov)


@pytest.mark.parametrize("cfg", range(6))
def test_hs_every_jacobi_config_bit_identical(of, orc, monkeypatch, cfg):
    """Each Jacobi configuration (tile shape, sweeps per launch), forced by
    OFLOW_HS_CFG, gives the oracle's bits: 37 sweeps exercise a partial last
    launch at every depth, the odd size ragged tiles."""
    from oflow import synth
    monkeypatch.setenv("OFLOW_HS_CFG", str(cfg))
    c = of.Context(0)
    q = synth.hs_pair(seed=5, w=203, h=117)
    u, v = of.hs(q.I0, q.I1, of.HSParams(3.0, 2, 2, 37), c)
    ou, ov = orc.hs(q.I0, q.I1, 3.0, 2, 2, 37)
    c.close()
    assert _same(u, ou) and _same(v, ov)


def test_hs_autotune_keeps_results_and_roundtrips(of, tmp_path):
    """The HS autotuner picks a configuration per level; the flow after tuning
    is identical; the choices are saved as "hs" lines and picked up by a fresh
    context."""
    from oflow import synth
    ctx = of.Context(0)
    qs = [synth.hs_pair(seed=s, w=240, h=160) for s in (7, 8)]
    pairs = [(q.I0, q.I1) for q in qs]
    prm = of.HSParams(15.0, 3, 1, 24)
    before = of.hs_batch(pairs, prm, ctx)
    cfg = of.hs_autotune(pairs, prm, ctx)
    assert len(cfg) == 3 and all(0 <= c < 6 for c in cfg)
    after = of.hs_batch(pairs, prm, ctx)
    for (u0, v0), (u1, v1) in zip(before, after):
        assert _same(u0, u1) and _same(v0, v1)
    path = str(tmp_path / "tune_hs.txt")
    ctx.save_tuning(path)
    lines = [l.split() for l in open(path) if not l.startswith("#")]
    assert len(lines) == 3 and all(l[0] == "hs" and l[3] == "2" for l in lines)
    assert sorted(int(l[4]) for l in lines) == sorted(cfg)
    ctx2 = of.Context(0)
    ctx2.load_tuning(path)
    again = of.hs_batch(pairs, prm, ctx2)
    for (u0, v0), (u1, v1) in zip(before, again):
        assert _same(u0, u1) and _same(v0, v1)
    ctx.close()
    ctx2.close()


def test_hs_1920x1080_against_oracle(of, orc, ctx):
    """The largest frame of the mixed batch workload with the HS parameters
    it uses (alpha 15, one level, one warp, 200 sweeps), and a 3-level
    pyramid at the same size: bit-identical to the oracle."""
    from oflow import synth
    q = synth.hs_pair(seed=33, w=1920, h=1080)
    for prm in (of.HSParams(15.0, 1, 1, 200), of.HSParams(0.2, 3, 2, 20)):
        u, v = of.hs(q.I0, q.I1, prm, ctx)
        ou, ov = orc.hs(q.I0, q.I1, prm.alpha, prm.nlevels, prm.nwarp, prm.nsolver)
        assert _same(u, ou) and _same(v, ov)


def test_hs_golden(of, ctx):
    d = dict(np.load(os.path.join(GOLDEN, "hs_64x48.npz")))
    u, v = of.hs(d["I0"], d["I1"], of.HSParams(15.0, 1, 1, 50), ctx)
    assert _same(u, d["u"]) and _same(v, d["v"])
    u, v = of.hs(d["I0"], d["I1"], of.HSParams(0.2, 3, 2, 20), ctx)
    assert _same(u, d["u3"]) and _same(v, d["v3"])


def test_hs_batch_and_compat(of, ctx):
    from oflow import synth
    qs = [synth.hs_pair(seed=s, w=160, h=120) for s in range(3)]
    res = of.hs_batch([(q.I0, q.I1) for q in qs], of.HSParams(15.0, 1, 1, 40), ctx)
    for q, (u, v) in zip(qs, res):
        su, sv = of.hs(q.I0, q.I1, of.HSParams(15.0, 1, 1, 40), ctx)
        assert _same(u, su) and _same(v, sv)
    # ComputeFlow with a stride (src/hs/cuda/flow.cuh:21-31)
    q = qs[0]
    stride = 192
    I0 = np.zeros((120, stride), np.float32)
    I1 = np.zeros((120, stride), np.float32)
    I0[:, :160], I1[:, :160] = q.I0, q.I1
    U = np.zeros((120, stride), np.float32)
    V = np.zeros((120, stride), np.float32)
    of.initFlow(1, stride, 160, 120)
    of.ComputeFlow(I0, I1, 160, 120, stride, 15.0, 1, 1, 40, U, V)
    of.deleteFlow_mem(1)
    assert _same(U[:, :160], res[0][0]) and _same(V[:, :160], res[0][1])


@pytest.mark.parametrize("spac,temp,window", [(3, 2, 5), (1, 1, 3), (5, 3, 7), (7, 5, 9), (9, 9, 5)])
def test_lk_single_step_bit_identical(of, orc, ctx, spac, temp, window):
    from oflow import synth
    rng = np.random.default_rng(spac * 10 + temp)
    base = synth.value_noise(rng, 70, 110)
    frames = [synth.quantize(base + rng.normal(0, 2, base.shape) + k) for k in range(temp)]
    for iframe in (0, temp - 1, 2 * temp + 1):
        u, v = of.lk(frames, iframe, of.LKParams(spac, temp, window), ctx)
        ou, ov = orc.lk_ring(frames, iframe, spac, temp, window)
        assert _same(u, ou) and _same(v, ov), iframe


def test_lk_golden_and_compat(of, ctx):
    d = dict(np.load(os.path.join(GOLDEN, "lk_80x60.npz")))
    u, v = of.lk([d["f0"], d["f1"]], 1, of.LKParams(3, 2, 5), ctx)
    assert _same(u, d["su"]) and _same(v, d["sv"])
    lk = of.LucasKanade(3, 2, 5, 80, 60)
    lk.copy_frames_circularbuffer_GPU_wrapper(d["f0"].ravel(), 2, 0, 80 * 60)
    lk.copy_frames_circularbuffer_GPU_wrapper(d["f1"].ravel(), 2, 1, 80 * 60)
    Vx = np.zeros(80 * 60, np.float32)
    Vy = np.zeros(80 * 60, np.float32)
    lk.lucas_kanade(Vx, Vy, 1)
    assert _same(Vx.reshape(60, 80), d["su"]) and _same(Vy.reshape(60, 80), d["sv"])


@pytest.mark.parametrize("levels,iters,window,w,h", [(3, 3, 5, 640, 480), (2, 1, 3, 97, 61),
                                                     (4, 2, 7, 320, 240)])
def test_pyrlk_bit_identical(of, orc, ctx, levels, iters, window, w, h):
    from oflow import synth
    l = synth.lk_pair(seed=w, w=w, h=h)
    u, v = of.pyrlk(l.I0, l.I1, of.LKParams(3, 2, window, levels, iters), ctx)
    ou, ov = orc.pyrlk(l.I0, l.I1, levels, iters, 3, window)
    assert _same(u, ou) and _same(v, ov)


def test_pyrlk_batch_matches_single_pairs(of, orc, ctx):
    """oflow_pyrlk_batch: pairs of two sizes (one plan per size) give each
    pair's oflow_pyrlk flow, which is the oracle's."""
    from oflow import synth
    pairs = [synth.lk_pair(seed=s, w=w, h=h) for s, (w, h) in
             enumerate([(160, 120), (97, 61), (160, 120), (160, 120), (97, 61)])]
    prm = of.LKParams(3, 2, 5, 3, 2)
    res = of.pyrlk_batch([(l.I0, l.I1) for l in pairs], prm, ctx)
    for l, (u, v) in zip(pairs, res):
        su, sv = of.pyrlk(l.I0, l.I1, prm, ctx)
        assert np.array_equal(u, su) and np.array_equal(v, sv)
        ou, ov = orc.pyrlk(l.I0, l.I1, 3, 2, 3, 5)
        assert _same(u, ou) and _same(v, ov)


@pytest.mark.parametrize("solver", ["hs", "pyrlk", "tvl1", "mixed"])
def test_device_frames_and_flows_in_place(of, ctx, solver):
    """Batches of device frames (uint8 with a row pitch, and float) and device
    flows with a row pitch: read and written in place through the plans'
    frame and output tables (HS, pyramidal LK, TV-L1, and a mixed batch of
    HS and TV-L1 jobs), bit-identical to the same pairs from host memory;
    padding of the pitched output rows is left untouched."""
    import torch
    from oflow import synth
    w, h = 97, 61
    gen = [synth.lk_pair(seed=50 + i, w=w, h=h) for i in range(3)]
    dev = torch.device("cuda", 0)
    host = [(synth.quantize(g.I0), synth.quantize(g.I1)) for g in gen]
    pitched = []
    for a, b in host:  # uint8 frames inside wider device rows
        pa = torch.zeros((h, w + 13), dtype=torch.uint8, device=dev)
        pb = torch.zeros((h, w + 13), dtype=torch.uint8, device=dev)
        pa[:, :w] = torch.from_numpy(a)
        pb[:, :w] = torch.from_numpy(b)
        pitched.append((pa[:, :w], pb[:, :w]))
    outs = [(torch.full((h, w + 5), 7.0, device=dev)[:, :w],
             torch.full((h, w + 5), 7.0, device=dev)[:, :w]) for _ in gen]
    run = None
    if solver == "hs":
        prm = of.HSParams(2.0, 2, 2, 30)
        run = lambda pairs, out=None: of.hs_batch(pairs, prm, ctx, out=out)
    elif solver == "pyrlk":
        prm = of.LKParams(3, 2, 5, 2, 2)
        run = lambda pairs, out=None: of.pyrlk_batch(pairs, prm, ctx, out=out)
    elif solver == "tvl1":
        prm = of.TVL1Params(nscales=3, max_iterations=10)
        run = lambda pairs, out=None: of.tvl1_batch(pairs, prm, ctx, out=out)
    else:
        tp, hp = of.TVL1Params(nscales=3, max_iterations=10), of.HSParams(2.0, 1, 1, 20)

        def run(pairs, out=None):
            jobs = [("tvl1" if i % 2 == 0 else "hs", a, b, tp if i % 2 == 0 else hp)
                    for i, (a, b) in enumerate(pairs)]
            return of.batch(jobs, ctx, out=out)
    ref = run(host)
    res = run(pitched, outs)
    torch.cuda.synchronize()
    for (ru, rv), (u, v) in zip(ref, res):
        assert np.array_equal(u.cpu().numpy(), ru) and np.array_equal(v.cpu().numpy(), rv)
    for (u, v) in outs:  # the padding columns of the output rows
        full_u = u.as_strided((h, w + 5), (w + 5, 1))
        assert torch.all(full_u[:, w:] == 7.0)
    # float frames on the device, contiguous flows
    fl = [(torch.from_numpy(a.astype(np.float32)).to(dev),
           torch.from_numpy(b.astype(np.float32)).to(dev)) for a, b in host]
    res2 = run(fl)
    for (ru, rv), (u, v) in zip(ref, res2):
        assert np.array_equal(u.cpu().numpy(), ru) and np.array_equal(v.cpu().numpy(), rv)


def test_pyrlk_golden_and_accuracy(of, ctx):
    from oflow import synth
    d = dict(np.load(os.path.join(GOLDEN, "lk_80x60.npz")))
    u, v = of.pyrlk(d["I0"], d["I1"], of.LKParams(3, 2, 5, 3, 3), ctx)
    assert _same(u, d["pu"]) and _same(v, d["pv"])
    l = synth.lk_pair(seed=0)
    u, v = of.pyrlk(l.I0, l.I1, of.LKParams(), ctx)
    assert synth.epe(u, v, l.u, l.v, l.valid, 8) < 1.0


def test_mixed_batch_matches_single_solves(of, ctx):
    """oflow_batch: HS and TV-L1 pairs of several sizes in one multi-branch
    graph give the same flows as solving each pair alone; the replayed graph
    (same composition) gives them again."""
    from oflow import synth
    tp = of.TVL1Params(nscales=3, max_iterations=10)
    hp = of.HSParams(15.0, 1, 1, 30)
    jobs = []
    for k, (w, h) in enumerate([(96, 64), (128, 96), (96, 64), (160, 120)]):
        p = synth.tvl1_pair(seed=80 + k, w=w, h=h, radius=12.0)
        jobs.append(("tvl1", synth.quantize(p.I0), synth.quantize(p.I1), tp))
        q = synth.hs_pair(seed=90 + k, w=w, h=h)
        jobs.append(("hs", q.I0, q.I1, hp))
    for _ in range(2):
        res = of.batch(jobs, ctx)
        for (solver, a, b, prm), (u, v) in zip(jobs, res):
            su, sv = (of.tvl1 if solver == "tvl1" else of.hs)(a, b, prm, ctx)
            assert _same(u, su) and _same(v, sv)
    # host buffers run each group on its own stream, device buffers as one
    # multi-branch graph: same flows
    import torch
    djobs = [(s_, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), p_) for s_, a, b, p_ in jobs]
    for _ in range(2):
        for (u, v), (du, dv) in zip(res, of.batch(djobs, ctx)):
            assert _same(u, du.cpu().numpy()) and _same(v, dv.cpu().numpy())
