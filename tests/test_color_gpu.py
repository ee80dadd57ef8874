"""flowToColor (src/tvl1/sequential/main.cpp:93-126) on the GPU against the
oracle's restatement: bit-exact bytes for random flows (zero, signed zeros,
huge magnitudes, every octant), a solver's flow, host and device buffers,
pitched rows, widths that are not a multiple of 4 (the scalar edge path) and
more flows than one launch takes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _flows(seed, h, w):
    rng = np.random.default_rng(seed)
    u = (rng.standard_normal((h, w)) * rng.choice([0.05, 1, 8, 40], (h, w))).astype(np.float32)
    v = (rng.standard_normal((h, w)) * rng.choice([0.05, 1, 8, 40], (h, w))).astype(np.float32)
    u.flat[:8] = [0.0, -0.0, 0.0, -0.0, 1e30, -1e30, 3.0, -3.0]
    v.flat[:8] = [0.0, 0.0, -0.0, -0.0, 1.0, -1.0, 3.0, -3.0]
    return u, v


@pytest.mark.parametrize("h,w", [(61, 97), (48, 64), (7, 5), (436, 1024)])
def test_bit_identical_to_oracle_host_buffers(of, orc, h, w):
    u, v = _flows(h * w, h, w)
    got = of.flow_to_color(u, v)
    assert got.shape == (h, w, 3) and got.dtype == np.uint8
    assert np.array_equal(got, orc.flow_to_color(u, v))


def test_device_pitched_and_batched(of, orc):
    import torch
    h, w = 37, 53
    flows = [_flows(100 + i, h, w) for i in range(40)]  # two launches (32 per launch)
    want = [orc.flow_to_color(u, v) for u, v in flows]
    dev = [(torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()) for u, v in flows]
    got = of.flow_to_color_batch(dev)
    for g, e in zip(got, want):
        assert g.is_cuda and np.array_equal(g.cpu().numpy(), e)
    # pitched device output (rows of 3*w + 13 bytes) from pitched device flows
    base = torch.zeros((h, 3 * w + 13), dtype=torch.uint8, device="cuda")
    img = base[:, : 3 * w].view(h, w, 3)
    U = torch.zeros((h, w + 3), device="cuda")
    V = torch.zeros((h, w + 3), device="cuda")
    U[:, :w] = dev[0][0]
    V[:, :w] = dev[0][1]
    import ctypes as C
    from oflow.capi import BgrImage, Flow, lib
    f = Flow(C.cast(C.c_void_p(U.data_ptr()), C.POINTER(C.c_float)),
             C.cast(C.c_void_p(V.data_ptr()), C.POINTER(C.c_float)), w + 3, 1)
    o = BgrImage(img.data_ptr(), 3 * w + 13, 1)
    ctx = of.Context(0)
    assert lib().oflow_flow_to_color(ctx.handle, 1, w, h, C.byref(f), C.byref(o)) == 0
    torch.cuda.synchronize()
    assert np.array_equal(img.cpu().numpy(), want[0])
    assert int(base[:, 3 * w:].sum()) == 0  # bytes past each row untouched
    ctx.close()


def test_solver_flow_and_ppm(of, orc, tmp_path):
    from oflow import synth
    p = synth.tvl1_pair(seed=5, w=160, h=96, radius=25.0)
    u, v = of.tvl1(synth.quantize(p.I0), synth.quantize(p.I1),
                   of.TVL1Params(nscales=4, max_iterations=20))
    img = of.flow_to_color(u, v)
    assert np.array_equal(img, orc.flow_to_color(u, v))
    path = tmp_path / "flow.ppm"
    of.save_ppm(str(path), img)
    data = path.read_bytes()
    assert data.startswith(b"P6\n160 96\n255\n")
    rgb = np.frombuffer(data[len(b"P6\n160 96\n255\n"):], np.uint8).reshape(96, 160, 3)
    assert np.array_equal(rgb, img[:, :, ::-1])


def test_errors_are_status_codes(of):
    u = np.zeros((4, 4), np.float32)
    with pytest.raises(ValueError):
        of.flow_to_color_batch([(u, u), (np.zeros((5, 4), np.float32), u)])
