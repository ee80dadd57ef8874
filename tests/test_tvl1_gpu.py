"""TV-L1 on the GPU through the C ABI against the oracle and the reference.

Tolerances against the compiled reference: max |du|,|dv| <= 1e-3 px and |dEPE| <= 1e-4 px after
the full solve; per-iteration energy within 1e-5 relative.  Against the C
restatement with the same error-sum rounding (one rounding of a double sum)
the kernels are bit-identical, and that is asserted where it holds by
construction."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL_FLOW = 1e-3
TOL_EPE = 1e-4
TOL_ENERGY = 1e-5


def _pair(seed, w, h, **kw):
    from oflow import synth
    p = synth.tvl1_pair(seed=seed, w=w, h=h, radius=kw.pop("radius", min(w, h) / 5.0), **kw)
    return p, synth.quantize(p.I0), synth.quantize(p.I1)


def _oracle(orc, a, b, prm, mode=1):
    return orc.tvl1(a.astype(np.float32), b.astype(np.float32),
                    orc.TVL1Params(prm.tau, prm.lambda_, prm.theta, prm.nscales, prm.zfactor,
                                   prm.warps, prm.epsilon, prm.max_iterations),
                    error_mode=mode, trace=True)


@pytest.mark.parametrize("w,h,ns,mi", [(97, 61, 100, 50), (64, 48, 3, 10), (131, 77, 4, 30),
                                       (200, 150, 5, 50), (33, 17, 2, 5)])
def test_bit_identical_to_oracle(of, orc, ctx, w, h, ns, mi):
    _, a, b = _pair(w * h, w, h)
    prm = of.TVL1Params(nscales=ns, max_iterations=mi)
    u, v, st = of.tvl1(a, b, prm, ctx, stats=True)
    ou, ov, its, _ = _oracle(orc, a, b, prm)
    assert np.array_equal(st["iterations"], its)
    assert np.array_equal(u, ou) and np.array_equal(v, ov)


@pytest.mark.parametrize("zf,warps,eps", [(0.6, 3, 0.01), (0.75, 2, 0.0), (0.5, 1, 0.5)])
def test_other_parameters(of, orc, ctx, zf, warps, eps):
    _, a, b = _pair(17, 120, 90)
    prm = of.TVL1Params(nscales=4, zfactor=zf, warps=warps, epsilon=eps, max_iterations=15)
    u, v, st = of.tvl1(a, b, prm, ctx, stats=True)
    ou, ov, its, _ = _oracle(orc, a, b, prm)
    assert np.array_equal(st["iterations"], its)
    assert np.array_equal(u, ou) and np.array_equal(v, ov)


@pytest.mark.parametrize("name", ["tvl1_97x61.npz", "tvl1_160x96.npz", "tvl1_128x64_w2.npz"])
def test_golden_reference_outputs(of, ctx, name):
    d = dict(np.load(os.path.join(GOLDEN, name)))
    prm = of.TVL1Params(float(d["tau"]), float(d["lambda_"]), float(d["theta"]),
                        int(d["nscales"]), float(d["zfactor"]), int(d["warps"]),
                        float(d["epsilon"]), int(d["max_iterations"]))
    u, v = of.tvl1(d["I0"], d["I1"], prm, ctx)
    assert max(np.abs(u - d["u"]).max(), np.abs(v - d["v"]).max()) <= TOL_FLOW


def test_energy_per_iteration(of, orc, ctx):
    _, a, b = _pair(23, 128, 96)
    prm = of.TVL1Params(nscales=3, max_iterations=12)
    u, v, st, en = of.tvl1_energy_trace(a, b, prm, ctx)
    ou, ov, its, oen = _oracle(orc, a, b, prm)
    assert np.array_equal(np.isnan(en), np.isnan(oen))
    m = ~np.isnan(oen)
    assert m.sum() == its.sum()
    assert np.max(np.abs(en[m] - oen[m]) / np.abs(oen[m])) <= TOL_ENERGY
    assert np.array_equal(u, ou)


def test_stats_energy_is_final_energy(of, orc, ctx):
    _, a, b = _pair(29, 96, 64)
    prm = of.TVL1Params(nscales=3, max_iterations=8)
    _, _, st = of.tvl1(a, b, prm, ctx, stats=True)
    _, _, _, en = of.tvl1_energy_trace(a, b, prm, ctx)
    last = en[0, -1][~np.isnan(en[0, -1])][-1]
    assert abs(st["energy"] - last) <= TOL_ENERGY * abs(last)


def test_batch_equals_single_and_mixed_sizes(of, ctx):
    specs = [(31, 96, 64), (32, 96, 64), (33, 120, 80), (34, 96, 64), (35, 64, 64)]
    pairs = [_pair(s, w, h)[1:] for s, w, h in specs]
    prm = of.TVL1Params(nscales=3, max_iterations=20)
    batch, stats = of.tvl1_batch(pairs, prm, ctx, stats=True)
    for (a, b), (u, v), st in zip(pairs, batch, stats):
        su, sv, ss = of.tvl1(a, b, prm, ctx, stats=True)
        assert np.array_equal(u, su) and np.array_equal(v, sv)
        assert np.array_equal(st["iterations"], ss["iterations"])


def test_u8_and_f32_inputs_agree(of, ctx):
    _, a, b = _pair(41, 100, 70)
    prm = of.TVL1Params(nscales=3, max_iterations=10)
    u1, v1 = of.tvl1(a, b, prm, ctx)
    u2, v2 = of.tvl1(a.astype(np.float32), b.astype(np.float32), prm, ctx)
    assert np.array_equal(u1, u2) and np.array_equal(v1, v2)


def test_device_and_pitched_buffers(of, ctx):
    import torch
    _, a, b = _pair(43, 100, 70)
    prm = of.TVL1Params(nscales=3, max_iterations=10)
    u, v = of.tvl1(a, b, prm, ctx)
    # pitched host frames
    pa = np.zeros((70, 128), np.uint8)
    pb = np.zeros((70, 128), np.uint8)
    pa[:, :100], pb[:, :100] = a, b
    up, vp = of.tvl1(pa[:, :100], pb[:, :100], prm, ctx)
    assert np.array_equal(u, up) and np.array_equal(v, vp)
    # device frames, device (pitched) outputs
    da = torch.from_numpy(pa).cuda()[:, :100]
    db = torch.from_numpy(pb).cuda()[:, :100]
    ou = torch.zeros((70, 112), dtype=torch.float32, device="cuda")[:, :100]
    ov = torch.zeros((70, 112), dtype=torch.float32, device="cuda")[:, :100]
    of.tvl1(da, db, prm, ctx, out=(ou, ov))
    torch.cuda.synchronize()
    assert np.array_equal(ou.cpu().numpy(), u) and np.array_equal(ov.cpu().numpy(), v)


def test_device_frames_read_in_place_then_host_frames(of, orc, ctx):
    """Device frames (pitched u8 and f32) are read in place through the plan's
    frame table, with conversion and normalisation in the first blur; later
    calls on the same plan with host frames, and the autotuner, read their own
    staged copies, never the earlier device pointers."""
    import torch
    prm = of.TVL1Params(nscales=4, max_iterations=15)
    A = [_pair(500 + i, 90, 66)[1:] for i in range(2)]
    Bp = [_pair(600 + i, 90, 66)[1:] for i in range(2)]

    def pitched(img, dtype):
        t = torch.zeros((66, 96), dtype=dtype, device="cuda")
        t[:, :90] = torch.from_numpy(img).to(dtype).cuda()
        return t[:, :90]

    def check(pairs, res):
        for (a, b), (u, v) in zip(pairs, res):
            ou, ov, _, _ = _oracle(orc, a, b, prm)
            u = u.cpu().numpy() if hasattr(u, "cpu") else u
            v = v.cpu().numpy() if hasattr(v, "cpu") else v
            assert np.array_equal(u, ou) and np.array_equal(v, ov)

    check(A, of.tvl1_batch([(pitched(a, torch.uint8), pitched(b, torch.uint8)) for a, b in A], prm, ctx))
    check(Bp, of.tvl1_batch(Bp, prm, ctx))
    f32 = [(a.astype(np.float32), b.astype(np.float32)) for a, b in A]
    check(A, of.tvl1_batch([(pitched(a, torch.float32), pitched(b, torch.float32)) for a, b in f32],
                           prm, ctx))
    of.tvl1_autotune(Bp, prm, ctx)
    check(Bp, of.tvl1_batch(Bp, prm, ctx))


@pytest.mark.parametrize("chunks", ["1", "4"])
def test_host_batch_in_chunks_matches_device_batch(of, ctx, monkeypatch, chunks):
    """A batch with host frames and host flows runs as one plan with its copies
    around it (the default) or as up to four chunks on side streams
    (OFLOW_HOST_CHUNKS; copies of one chunk overlap the solves of the others);
    the flows and statistics equal those of the same batch solved as one plan
    from device frames, including a batch that does not split evenly."""
    import torch
    monkeypatch.setenv("OFLOW_HOST_CHUNKS", chunks)
    prm = of.TVL1Params(nscales=3, max_iterations=14)
    for n in (8, 13):
        pairs = [_pair(900 + i, 84, 60)[1:] for i in range(n)]
        host, st_h = of.tvl1_batch(pairs, prm, ctx, stats=True)
        dev = of.tvl1_batch([(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
                             for a, b in pairs], prm, ctx)
        _, st_d = of.tvl1_batch(pairs[:1], prm, ctx, stats=True)
        for (hu, hv), (du, dv) in zip(host, dev):
            assert np.array_equal(hu, du.cpu().numpy()) and np.array_equal(hv, dv.cpu().numpy())
        assert np.array_equal(st_h[0]["iterations"], st_d[0]["iterations"])
        assert all(s["energy"] > 0 for s in st_h)


@pytest.mark.parametrize("side_queue", ["0", "1", "4"])
def test_host_chunks_of_tiled_levels_match_device_batch(of, monkeypatch, side_queue):
    """Host frames and flows of tiled levels (256x128) in four chunks
    (OFLOW_HOST_CHUNKS=4): the chunks on side streams run one launch per
    block of iterations (the default), or the
    work queue on all or a quarter of the resident slots (OFLOW_SIDE_QUEUE);
    the flows equal the device batch solved as one plan."""
    import torch
    monkeypatch.setenv("OFLOW_HOST_CHUNKS", "4")
    monkeypatch.setenv("OFLOW_SIDE_QUEUE", side_queue)
    c = of.Context(0)
    prm = of.TVL1Params(nscales=3, max_iterations=20)
    pairs = [_pair(950 + i, 256, 128)[1:] for i in range(12)]
    host = of.tvl1_batch(pairs, prm, c)
    dev = of.tvl1_batch([(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
                         for a, b in pairs], prm, c)
    for (hu, hv), (du, dv) in zip(host, dev):
        assert np.array_equal(hu, du.cpu().numpy()) and np.array_equal(hv, dv.cpu().numpy())
    c.close()


@pytest.mark.parametrize("queue", [True, False])
def test_launch_count_of_the_schedule(of, monkeypatch, queue):
    """oflow_ctx_last_launches reports the captured schedule: per warp stage
    one warp launch and one persistent work-queue launch (k_tvl1_q) for the
    tiled levels; with the queue off (OFLOW_TB_QUEUE=0), for levels larger
    than 9216 pixels, ceil(50/4)+1 tiled inner-iteration launches (one for a
    re-run after a stop inside a launch that wrote no snapshots).  A smaller
    level runs its whole stage in one launch either way.  Plus the ingest,
    pyramid (one fused blur-and-decimate launch per level), gradient and
    column-coefficient, zoom and output launches."""
    if not queue:
        monkeypatch.setenv("OFLOW_TB_QUEUE", "0")
    ctx = of.Context(0)
    pairs = [_pair(700 + i, 128, 96)[1:] for i in range(3)]
    prm = of.TVL1Params(nscales=5, max_iterations=50)
    _, st = of.tvl1_batch(pairs, prm, ctx, stats=True)
    ns = st[0]["nscales"]
    sizes = [(128, 96)]
    for _ in range(ns - 1):
        w, h = sizes[-1]
        sizes.append((int(w * 0.5 + 0.5), int(h * 0.5 + 0.5)))
    per_stage = [1 + (1 if (w * h <= 9216 or queue) else 14) for w, h in sizes]
    expect = 5 * sum(per_stage)
    n = ctx.last_launches()
    # ingest 2, level-0 blur 1, pyramid ns-1, column coefficients ns, zooms ns-1, output 1
    # (the final energy runs on demand, when statistics are read)
    assert n == expect + 3 * ns + 2
    ctx.close()


def test_full_size_workload_against_oracle_and_reference(of, orc, ctx):
    """1024x436, 5 scales x 5 warps x 50 iterations (the benchmark workload)."""
    from oflow import synth
    p, a, b = _pair(0, 1024, 436, radius=80.0)
    prm = of.TVL1Params(nscales=5, max_iterations=50)
    u, v, st = of.tvl1(a, b, prm, ctx, stats=True)
    ou, ov, its, _ = _oracle(orc, a, b, prm, mode=1)
    assert np.array_equal(st["iterations"], its)
    assert np.array_equal(u, ou) and np.array_equal(v, ov)
    if orc.ref_available():
        ru, rv = orc.ref_tvl1(a, b, orc.TVL1Params(nscales=5, max_iterations=50))
        assert max(np.abs(u - ru).max(), np.abs(v - rv).max()) <= TOL_FLOW
        e_gpu = synth.epe(u, v, p.u, p.v, p.valid, 8)
        e_ref = synth.epe(ru, rv, p.u, p.v, p.valid, 8)
        assert abs(e_gpu - e_ref) <= TOL_EPE
    assert synth.epe(u, v, p.u, p.v, p.valid, 8) < 0.5


@pytest.mark.parametrize("cfg", [None, "3", "5"])
def test_repeated_full_size_solves_match_the_oracle(of, orc, monkeypatch, cfg):
    """Five solves of the 1024x436 pair, each on a fresh context (new plan,
    new graph, reused device memory), with the tile shapes the plan picks,
    with the smallest tile forced everywhere, and with the cluster kernel on
    every level whose band fits (the two coarsest): every solve equals the
    oracle.  Catches order-dependent faults that a single solve can miss."""
    if cfg:
        monkeypatch.setenv("OFLOW_TB_CFG", cfg)
    p, a, b = _pair(0, 1024, 436, radius=80.0)
    prm = of.TVL1Params(nscales=5, warps=1, max_iterations=50)
    ou, ov, its, _ = _oracle(orc, a, b, prm, mode=1)
    for _ in range(5):
        c = of.Context(0)
        u, v, st = of.tvl1(a, b, prm, c, stats=True)
        c.close()
        assert np.array_equal(st["iterations"], its)
        assert np.array_equal(u, ou) and np.array_equal(v, ov)


@pytest.mark.parametrize("env", [{"OFLOW_TB_QUEUE": "0"}, {"OFLOW_TB_PREDICT": "0"},
                                 {"OFLOW_TB_PREDICT": "1"}])
@pytest.mark.parametrize("w,h,ns", [(1024, 436, 5), (131, 77, 4), (333, 201, 5)])
def test_alternative_kernel_forms_match_the_oracle(of, orc, monkeypatch, env, w, h, ns):
    """The tiled stages as one launch per block of iterations (k_tvl1_tb),
    as the persistent work queue with full blocks of iterations, and with
    blocks sized to the predicted stop keeping their snapshots: the same bits
    as the oracle (the default form, blocks sized to the predicted stop
    without snapshots, is what every other test runs).  Odd widths take the
    plain region loads."""
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    _, a, b = _pair(w + h, w, h, radius=min(w, h) / 5.0)
    prm = of.TVL1Params(nscales=ns, warps=2, max_iterations=30)
    ou, ov, its, _ = _oracle(orc, a, b, prm, mode=1)
    c = of.Context(0)
    u, v, st = of.tvl1(a, b, prm, c, stats=True)
    c.close()
    assert np.array_equal(st["iterations"], its)
    assert np.array_equal(u, ou) and np.array_equal(v, ov)


def test_timeout_is_reported_and_the_context_recovers(of, orc, monkeypatch):
    """A kernel that gives up a bounded wait sets the plan's error flag; the
    call then returns OFLOW_ERR_TIMEOUT (3).  The flag is raised from the
    host here (OFLOW_INJECT_TIMEOUT), so no GPU wait runs out.  The next call
    on the same context, reusing the same plan and graph, equals the oracle."""
    _, a, b = _pair(41, 200, 150)
    prm = of.TVL1Params(nscales=4, max_iterations=30)
    ou, ov, its, _ = _oracle(orc, a, b, prm)
    c = of.Context(0)
    of.tvl1(a, b, prm, c)
    monkeypatch.setenv("OFLOW_INJECT_TIMEOUT", "1")
    with pytest.raises(of.OflowError) as e:
        of.tvl1(a, b, prm, c)
    assert e.value.status == 3
    monkeypatch.delenv("OFLOW_INJECT_TIMEOUT")
    for _ in range(2):
        u, v, st = of.tvl1(a, b, prm, c, stats=True)
        assert np.array_equal(st["iterations"], its)
        assert np.array_equal(u, ou) and np.array_equal(v, ov)
    c.close()


def test_known_answers_on_gpu(of, ctx):
    I = np.full((96, 128), 90, np.uint8)
    u, v = of.tvl1(I, I, of.TVL1Params(nscales=3, max_iterations=20), ctx)
    assert np.all(u == 0) and np.all(v == 0)
    from oflow import synth
    rng = np.random.default_rng(2)
    big = synth._blur(rng.uniform(0, 255, (160, 220)), 2.0)
    I0 = synth.quantize(big[10:150, 10:210])
    I1 = synth.quantize(big[10:150, 7:207])   # I1(x + 3) = I0(x)
    u, v = of.tvl1(I0, I1, of.TVL1Params(nscales=4, max_iterations=50), ctx)
    assert abs(float(np.median(u[16:-16, 16:-16])) - 3.0) < 0.05


def test_errors_are_status_codes(of, ctx):
    small = np.zeros((4, 4), np.uint8)
    with pytest.raises(of.OflowError) as e:
        of.tvl1(small, small, of.TVL1Params(), ctx)
    assert e.value.status == 1
    with pytest.raises(of.OflowError) as e:
        of.tvl1(np.zeros((32, 32), np.uint8), np.zeros((32, 40), np.uint8), of.TVL1Params(), ctx)
    assert e.value.status == 1
    # the context stays usable
    u, v = of.tvl1(np.zeros((32, 32), np.uint8), np.zeros((32, 32), np.uint8),
                   of.TVL1Params(nscales=2, max_iterations=3), ctx)
    assert np.all(u == 0)


def test_reference_class_mirror(of, orc):
    """TV_L1 with both reference call forms (sequential uint8 pair; streaming
    float frames paired with the previous call)."""
    _, a, b = _pair(51, 96, 64)
    t = of.TV_L1(96, 64, nscales=3, max_iterations=10)
    t.runDualTVL1Multiscale(a, b)
    U = t.getU().copy()
    u, v = of.tvl1(a, b, of.TVL1Params(nscales=3, max_iterations=10))
    assert np.array_equal(U[: 96 * 64], u.ravel()) and np.array_equal(U[96 * 64:], v.ravel())
    s = of.TV_L1(96, 64, nscales=3, max_iterations=10)
    s.runDualTVL1Multiscale(a.astype(np.float32).ravel())
    s.runDualTVL1Multiscale(b.astype(np.float32).ravel())
    assert np.array_equal(s.getU(), U)


def test_autotune_keeps_results_and_roundtrips(of, tmp_path):
    """The autotuner picks a configuration per scale; every configuration is
    exact, so the flow after tuning is identical; the table survives a
    save/load round trip into a fresh context."""
    ctx = of.Context(0)
    pairs = [_pair(s, 160, 120)[1:] for s in (61, 62)]
    prm = of.TVL1Params(nscales=3, max_iterations=12)
    before = of.tvl1_batch(pairs, prm, ctx)
    cfg = of.tvl1_autotune(pairs, prm, ctx)
    assert len(cfg) == 3 and all(0 <= c < 6 for c in cfg)  # 4, 5: whole level per block, per cluster
    after = of.tvl1_batch(pairs, prm, ctx)
    for (u0, v0), (u1, v1) in zip(before, after):
        assert np.array_equal(u0, u1) and np.array_equal(v0, v1)
    path = str(tmp_path / "tune.txt")
    ctx.save_tuning(path)
    lines = [l for l in open(path) if not l.startswith("#")]
    assert len(lines) == 3 and all(l.startswith("tvl1 ") for l in lines)
    ctx2 = of.Context(0)
    ctx2.load_tuning(path)
    again = of.tvl1_batch(pairs, prm, ctx2)
    for (u0, v0), (u1, v1) in zip(before, again):
        assert np.array_equal(u0, u1) and np.array_equal(v0, v1)
    bad = tmp_path / "bad.txt"
    bad.write_text("tvl1 1 2\n")
    with pytest.raises(of.OflowError):
        ctx2.load_tuning(str(bad))
    ctx.close()
    ctx2.close()


@pytest.mark.parametrize("w,h,seed", [(1920, 1080, 31), (1280, 720, 32)])
def test_largest_batch_sizes_against_oracle_and_reference(of, orc, ctx, w, h, seed):
    """The two largest frame sizes of the mixed batch workload (1920x1080,
    1280x720), 5 scales x 5 warps x 50 iterations: bit-identical to the
    oracle (flow and iteration counts), within the stated tolerances of the
    compiled reference."""
    from oflow import synth
    p, a, b = _pair(seed, w, h, radius=min(w, h) / 5.0)
    prm = of.TVL1Params(nscales=5, max_iterations=50)
    u, v, st = of.tvl1(a, b, prm, ctx, stats=True)
    ou, ov, its, _ = _oracle(orc, a, b, prm, mode=1)
    assert np.array_equal(st["iterations"], its)
    assert np.array_equal(u, ou) and np.array_equal(v, ov)
    if orc.ref_available():
        ru, rv = orc.ref_tvl1(a, b, orc.TVL1Params(nscales=5, max_iterations=50))
        assert max(np.abs(u - ru).max(), np.abs(v - rv).max()) <= TOL_FLOW
        assert abs(synth.epe(u, v, p.u, p.v, p.valid, 8) -
                   synth.epe(ru, rv, p.u, p.v, p.valid, 8)) <= TOL_EPE


def test_benchmark_pairs_against_reference(of, orc, ctx):
    """The first 8 pairs the benchmark solves (generator seeds 10000-10007 at
    1024x436), solved as one batch: each bit-identical to the oracle with the
    GPU's error-sum rounding; each within max |du|,|dv| <= 1e-3 px and
    |dEPE| <= 1e-4 px of the compiled reference.  The iteration counts per
    (scale, warp) are also compared with the oracle in the reference's own
    summation order (left to right in float): a stage whose count differs is
    a stopping-decision flip, printed, and the flow tolerances above still
    hold."""
    from oflow import synth
    seeds = list(range(10_000, 10_008))
    pairs = []
    for s in seeds:
        p = synth.tvl1_pair(seed=s, w=1024, h=436)
        pairs.append((p, synth.quantize(p.I0), synth.quantize(p.I1)))
    prm = of.TVL1Params(nscales=5, max_iterations=50)
    res, stats = of.tvl1_batch([(a, b) for _, a, b in pairs], prm, ctx, stats=True)
    flips = []
    for s, (p, a, b), (u, v), st in zip(seeds, pairs, res, stats):
        ou, ov, its, _ = _oracle(orc, a, b, prm, mode=1)
        assert np.array_equal(st["iterations"], its), s
        assert np.array_equal(u, ou) and np.array_equal(v, ov), s
        _, _, its0, _ = _oracle(orc, a, b, prm, mode=0)
        flips += [(s, int(k), int(w_), int(its[k, w_]), int(its0[k, w_]))
                  for k, w_ in zip(*np.nonzero(its != its0))]
        if orc.ref_available():
            ru, rv = orc.ref_tvl1(a, b, orc.TVL1Params(nscales=5, max_iterations=50))
            assert max(np.abs(u - ru).max(), np.abs(v - rv).max()) <= TOL_FLOW, s
            assert abs(synth.epe(u, v, p.u, p.v, p.valid, 8) -
                       synth.epe(ru, rv, p.u, p.v, p.valid, 8)) <= TOL_EPE, s
    print(f"iteration-count flips (seed, scale, warp, gpu, reference order): {flips}")
