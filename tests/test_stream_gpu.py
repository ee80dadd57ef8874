"""Frame streams (oflow_stream_*, the reference's streaming TV-L1
runDualTVL1Multiscale(const float *) of src/tvl1/cuda/tvl1.cu:122-130): each
push pairs every lane's previous frame (zeros before the first) with its new
frame, and the flows equal the two-frame solves of the same pairs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _frames(seed, n, w, h):
    from oflow import synth
    out = []
    for k in range(n):
        p = synth.tvl1_pair(seed=seed + k, w=w, h=h, radius=min(w, h) / 5.0)
        out.append(synth.quantize(p.I0))
    return out


def test_tvl1_stream_lanes_equal_pair_solves(of):
    w, h = 97, 61
    prm = of.TVL1Params(nscales=4, max_iterations=20)
    lanes = [_frames(10, 3, w, h), _frames(20, 3, w, h)]
    ctx = of.Context(0)
    s = of.FrameStream(w, h, "tvl1", lanes=2, params=prm, ctx=ctx)
    prev = [np.zeros((h, w), np.uint8)] * 2
    for k in range(3):
        new = [lanes[0][k], lanes[1][k]]
        res, st = s.push(new, stats=True)
        for i in range(2):
            u, v, st1 = of.tvl1(prev[i], new[i], prm, ctx, stats=True)
            assert np.array_equal(res[i][0], u) and np.array_equal(res[i][1], v)
            assert np.array_equal(st[i]["iterations"], st1["iterations"])
        prev = new
    assert s.frames == 3
    s.close()
    ctx.close()


def test_hs_stream_and_async_device_pushes(of):
    import torch
    w, h = 80, 60
    prm = of.HSParams(alpha=15.0, nlevels=2, nwarp=2, nsolver=30)
    fr = _frames(30, 4, w, h)
    ctx = of.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    s = of.FrameStream(w, h, "hs", lanes=1, params=prm, ctx=ctx)
    dev = [torch.from_numpy(f).cuda() for f in fr]
    torch.cuda.synchronize()
    outs = [(torch.empty((h, w), device="cuda"), torch.empty((h, w), device="cuda")) for _ in fr]
    with torch.cuda.stream(stream):
        for k in range(4):  # returns after enqueueing: device frames, device outputs
            s.push([dev[k]], out=[outs[k]])
    stream.synchronize()
    ctx.set_stream(None)
    prev = np.zeros((h, w), np.uint8)
    for k in range(4):
        u, v = of.hs(prev, fr[k], prm, ctx)
        assert np.array_equal(outs[k][0].cpu().numpy(), u)
        assert np.array_equal(outs[k][1].cpu().numpy(), v)
        prev = fr[k]
    s.close()
    ctx.close()


def test_stream_rejects_wrong_frames(of):
    ctx = of.Context(0)
    s = of.FrameStream(32, 24, "tvl1", lanes=1, params=of.TVL1Params(nscales=2, max_iterations=5),
                       ctx=ctx)
    with pytest.raises(of.OflowError):
        s.push([np.zeros((24, 33), np.uint8)])
    with pytest.raises(of.OflowError):
        s.push([np.zeros((24, 32), np.float32)])
    with pytest.raises(ValueError):
        s.push([])
    s.close()
    ctx.close()


def test_objects_outlive_their_context(of):
    """A context destroyed before its network and stream leaves them inert:
    using them is an error status, destroying them is safe."""
    ctx = of.Context(0)
    s = of.FrameStream(32, 24, "tvl1", lanes=1, params=of.TVL1Params(nscales=2, max_iterations=5),
                       ctx=ctx)
    net = of.WarmNet(64, 48, 1, ctx)
    s.push([np.zeros((24, 32), np.uint8)])
    ctx.close()
    with pytest.raises(of.OflowError):
        s.push([np.zeros((24, 32), np.uint8)])
    with pytest.raises(of.OflowError):
        net.set_params(np.zeros(of.net_num_params(), np.float32))
    s.close()
    net.close()
