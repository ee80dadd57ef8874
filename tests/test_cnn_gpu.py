"""The warm-start network's BF16 tensor-core convolution kernels against a
float64 CPU oracle (oracle/cnn_ref.py): forward, backward-data and
backward-weight (the gradient check), stride 1 and 2, with and without the
ReLU mask; then the network trains (loss falls) and the warm-started TV-L1
respects its energy judge."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 2e-3  # bf16 operands are exact in f32 products; f32 sums over <= 9*224 terms


def _bf16(t):
    import torch
    return t.to(torch.bfloat16)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-12))


@pytest.mark.parametrize("N,H,W,C,K,stride,relu", [(2, 9, 13, 16, 32, 1, True), (1, 12, 10, 32, 8, 2, False),
                                                   (2, 7, 11, 48, 64, 2, True), (1, 16, 16, 160, 64, 1, True),
                                                   (2, 13, 17, 224, 96, 1, True), (1, 11, 9, 96, 128, 2, True),
                                                   (3, 20, 30, 16, 32, 2, True)])
def test_conv_products_match_cpu_oracle(of, N, H, W, C, K, stride, relu):
    """Forward, backward-data and backward-weight on both tensor-core kernels
    (tcgen05 with the accumulator in tensor memory, and mma.sync), against
    the float64 oracle."""
    import torch
    from oracle import cnn_ref
    g = torch.Generator().manual_seed(N * 1000 + C + K)
    P, Q = cnn_ref.conv_out(H, stride), cnn_ref.conv_out(W, stride)
    x = _bf16(torch.randn((N, H, W, C), generator=g))
    w = _bf16(torch.randn((K, 3, 3, C), generator=g) * 0.1)
    b = torch.randn(K, generator=g) * 0.1
    xd, wd, bd = x.cuda(), w.cuda(), b.cuda()
    ref = cnn_ref.forward(x.float().numpy(), w.float().numpy(), b.numpy(), stride, relu)
    for mode in (0, 3):
        # forward, f32 output
        y = torch.full((N, P, Q, K), float("nan"), dtype=torch.float32, device="cuda")
        of.conv3x3(mode, N, H, W, C, K, stride, relu, True, xd, None, wd, y, bias=bd)
        assert _rel(y.cpu().numpy(), ref) < REL, mode
        # forward, bf16 output (what the network stores)
        yb = torch.full((N, P, Q, K), float("nan"), dtype=torch.bfloat16, device="cuda")
        of.conv3x3(mode, N, H, W, C, K, stride, relu, False, xd, None, wd, yb, bias=bd)
        assert _rel(yb.float().cpu().numpy(), ref) < 1e-2, mode
    # backward: gradients of sum(gout * y); gout is rounded to bf16 by the
    # kernels, so the oracle gets the same rounded values
    gout = torch.randn((N, P, Q, K), generator=g)
    gout_b = _bf16(gout).float()
    yact = yb if relu else None
    gx_ref, gw_ref, gb_ref = cnn_ref.backward(x.float().numpy(), w.float().numpy(), gout_b.numpy(),
                                              stride, yb.float().cpu().numpy() if relu else None)
    gx = torch.empty((N, H, W, C), dtype=torch.float32, device="cuda")
    if K % 8 == 0:  # mode 1: tcgen05, the backward-data product as a forward convolution
        of.conv3x3(1, N, H, W, C, K, stride, relu, True, gout.cuda(), yact, wd, gx)
        assert _rel(gx.cpu().numpy(), gx_ref) < REL
        gx.fill_(float("nan"))
    of.conv3x3(4, N, H, W, C, K, stride, relu, True, gout.cuda(), yact, wd, gx)  # mma.sync
    gw = torch.empty((K, 3, 3, C), dtype=torch.float32, device="cuda")
    gb = torch.empty(K, dtype=torch.float32, device="cuda")
    # mode 2: tcgen05 (MN-major operands, pixels split across CTAs); mode 5: mma.sync
    of.conv3x3(2, N, H, W, C, K, stride, relu, True, gout.cuda(), yact, xd, gw, gbias=gb)
    torch.cuda.synchronize()
    assert _rel(gw.cpu().numpy(), gw_ref) < REL
    gw.fill_(float("nan"))
    of.conv3x3(5, N, H, W, C, K, stride, relu, True, gout.cuda(), yact, xd, gw, gbias=gb)
    torch.cuda.synchronize()
    assert _rel(gx.cpu().numpy(), gx_ref) < REL
    assert _rel(gw.cpu().numpy(), gw_ref) < REL
    # the bias gradient sums the unrounded f32 gradient
    gb_ref_f = (gout.numpy() * ((yb.float().cpu().numpy() > 0) if relu else 1)).sum(axis=(0, 1, 2))
    assert _rel(gb.cpu().numpy(), gb_ref_f) < 1e-4


def _init_params(of, seed=0):
    """He-normal weights, zero biases; the last layer scaled down."""
    from oflow import warmstart
    return warmstart.init_params(seed)


def test_network_trains(of):
    import torch
    from oflow import synth_gpu
    net = of.WarmNet(128, 96, 4)
    assert (net.out_w, net.out_h) == (16, 12)
    net.set_params(_init_params(of, 1))
    a, b, u, v, _ = synth_gpu.tvl1_pairs(4, 128, 96, seed=5, radius=20.0)
    frames = torch.stack([a, b], dim=1).contiguous()
    # target: ground truth averaged over 8x8 blocks, in 1/8-scale pixels
    t = torch.stack([u, v], dim=1)
    tgt = (torch.nn.functional.avg_pool2d(t, 8, ceil_mode=True) / 8).permute(0, 2, 3, 1).contiguous()
    losses = [net.train_step(frames, tgt, 2e-3) for _ in range(60)]
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.5 * losses[0]
    pred = net.predict(frames)
    assert pred.shape == (4, 12, 16, 2)
    p = net.get_params()
    net2 = of.WarmNet(128, 96, 4)
    net2.set_params(p)
    assert torch.equal(net2.predict(frames), pred)


def test_warm_start_judge(of):
    """With the plain solve as judge, every returned flow is either the warm
    result (energy within 1%) or exactly the plain result."""
    import torch
    from oflow import synth
    pairs = []
    for s in range(2):
        p = synth.tvl1_pair(seed=300 + s, w=256, h=128, radius=25.0)
        pairs.append((synth.quantize(p.I0), synth.quantize(p.I1)))
    net = of.WarmNet(256, 128, 2)
    net.set_params(_init_params(of, 2))
    warm = of.TVL1Params(nscales=5, warps=2, max_iterations=20)
    plain = of.TVL1Params(nscales=5, max_iterations=50)
    res, info = of.tvl1_warm(pairs, net, warm, plain)
    warm_only, _ = of.tvl1_warm(pairs, net, warm, None)
    for (a, b), (u, v), (wu, wv), acc, ew, ep, er in zip(
            pairs, res, warm_only, info["accepted"], info["energy_warm"], info["energy_plain"],
            info["epe_vs_plain"]):
        assert np.isfinite(ew) and np.isfinite(ep) and ep > 0
        pu, pv = of.tvl1(a, b, plain)
        # the end-point criterion: sum |warm - plain| / sum |plain| (double)
        d = np.hypot(wu.astype(np.float64) - pu, wv.astype(np.float64) - pv).sum()
        m = np.hypot(pu.astype(np.float64), pv.astype(np.float64)).sum()
        assert abs(er - d / m) <= 1e-9 * max(1.0, d / m)
        assert acc == (ew <= 1.01 * ep and er <= 0.01)
        if acc:
            assert np.array_equal(u, wu) and np.array_equal(v, wv)
        else:
            assert np.array_equal(u, pu) and np.array_equal(v, pv)


def test_warm_start_per_scale_schedule(of):
    """A per-scale schedule: the uniform values given per scale reproduce the
    uniform solve bit for bit, and a mixed schedule respects every scale's
    warp count and iteration cap."""
    from oflow import synth
    pairs = []
    for s in range(2):
        p = synth.tvl1_pair(seed=310 + s, w=256, h=128, radius=25.0)
        pairs.append((synth.quantize(p.I0), synth.quantize(p.I1)))
    net = of.WarmNet(256, 128, 2)
    net.set_params(_init_params(of, 2))
    warm = of.TVL1Params(nscales=5, warps=3, max_iterations=20)
    r0, i0 = of.tvl1_warm(pairs, net, warm)
    r1, i1 = of.tvl1_warm(pairs, net, warm, warps_per_scale=[3, 3, 3, 3],
                          iters_per_scale=[20, 20, 20, 20])
    for (u0, v0), (u1, v1) in zip(r0, r1):
        assert np.array_equal(u0, u1) and np.array_equal(v0, v1)
    ws, its = [3, 1, 2, 1], [12, 5, 7, 3]
    _, i2 = of.tvl1_warm(pairs, net, warm, warps_per_scale=ws, iters_per_scale=its)
    for st in i2["stats"]:
        it = st["iterations"]  # [scale][warp]
        for s in range(4):
            assert np.all(it[s, :ws[s]] >= 1) and np.all(it[s, :ws[s]] <= its[s])
            assert np.all(it[s, ws[s]:] == 0)


def test_trained_network_gains_over_no_network(of):
    """What the trained network buys: the same reduced schedule (2 warps x 20
    iterations) on 1024x436 pairs of the benchmark generator, started three
    ways -- scale 3 from the trained network, scale 3 from zero flow (all
    network weights zero), and the plain pyramid from the coarsest scale.
    The trained start gives lower TV-L1 energy and lower EPE than both."""
    from oflow import synth, warmstart
    n = 8
    gen = [synth.tvl1_pair(seed=20_000 + i) for i in range(n)]
    pairs = [(synth.quantize(p.I0), synth.quantize(p.I1)) for p in gen]
    ctx = of.Context(0)
    net = of.WarmNet(1024, 436, n, ctx)
    params, _ = warmstart.load()
    reduced = of.TVL1Params(nscales=5, warps=2, max_iterations=20)

    def epe(res):
        return np.mean([synth.epe(u, v, p.u, p.v, p.valid, 8) for (u, v), p in zip(res, gen)])

    net.set_params(params)
    # the judge here is the plain pyramid with the same reduced schedule
    _, info_t = of.tvl1_warm(pairs, net, reduced, reduced, ctx)
    e_trained, e_plain = info_t["energy_warm"], info_t["energy_plain"]
    plain_res = of.tvl1_batch(pairs, reduced, ctx)
    net.set_params(np.zeros_like(params))
    res_z, info_z = of.tvl1_warm(pairs, net, reduced, None, ctx)
    e_zero = info_z["energy_warm"]
    # energies are of the warm results themselves (not of the judged choice)
    assert np.mean(e_trained) < np.mean(e_zero)
    assert np.mean(e_trained) < np.mean(e_plain)
    # EPE of the warm-started results (re-solved without the judge)
    net.set_params(params)
    res_t2, _ = of.tvl1_warm(pairs, net, reduced, None, ctx)
    assert epe(res_t2) < epe(res_z)
    assert epe(res_t2) < epe(plain_res)
    ctx.close()
