"""Horn-Schunck and Lucas-Kanade pinned to the reference's own CUDA kernels.

oracle/build_ref.sh compiles, where they lie in the reference checkout and
unmodified, the reference's defect-free HS kernels (JacobiIteration<32,6>,
AddKernel, DownscaleKernel: src/hs/cuda/kernels/*.cuh) and its LK sources
(src/lk/cuda/lucaskanade.cu, kernels/kernels.cu) into oracle/_ref, twice:
with -fmad=false (the library's arithmetic contract) and with the reference's
own flags (-O3, contraction into fused multiply-adds).  These tests feed the
reference kernels and this library identical inputs:

* -fmad=false build: bit-identical results required.
* stock build: the only difference is the rounding of contracted a*b+c, so
  results agree within a few ulp; the bounds are written per test.

Steps whose reference kernels read outside their buffers (WarpingKernel,
ComputeDerivativesKernel, UpscaleKernel; the LK y-filter when ny < nx) are
never run; the HS pipeline takes the oracle's restatement of those steps
(deviations D-H1..D-H4), so the comparison of a whole HS solve is a
composition of reference kernels and documented deviations.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refg():
    import oracle
    if not (oracle.refg_available(False) and oracle.refg_available(True)):
        pytest.skip("reference HS/LK kernels (oracle/_ref) not built here")
    return oracle


def _align32(n):
    return (n + 31) // 32 * 32


def _hs_inputs(orc, w, h, seed):
    from oflow import synth
    q = synth.hs_pair(seed=seed, w=w, h=h)
    I1w = orc.hs_warp(q.I1, np.zeros_like(q.I0), np.zeros_like(q.I0))
    Ix, Iy, Iz = orc.hs_derivatives(q.I0, I1w)
    return q, Ix, Iy, Iz


# ------------------------------------------------------------------ HS steps
@pytest.mark.parametrize("w,h", [(320, 240), (131, 77), (64, 48), (203, 117), (9, 8)])
def test_hs_downscale_interior_equals_reference(refg, w, h):
    """DownscaleKernel (downscaleKernel.cuh:27-40) against the restatement:
    every pixel the reference writes (all but the last row and column) is the
    same; the restatement also writes those (D-H1)."""
    from oflow import synth
    src = synth.hs_pair(seed=w * h, w=w, h=h).I0
    ours = refg.hs_downscale(src)
    for stock in (False, True):
        ref = refg.refg_hs_downscale(src, stock=stock)
        assert np.isnan(ref[-1, :]).all() and np.isnan(ref[:, -1]).all()
        assert np.array_equal(ref[:-1, :-1], ours[:-1, :-1])


@pytest.mark.parametrize("w,h,alpha,sweeps", [(320, 240, 15.0, 200), (131, 77, 0.2, 37),
                                              (33, 17, 1.0, 1), (203, 117, 5.0, 64)])
def test_hs_jacobi_equals_reference(refg, w, h, alpha, sweeps):
    """JacobiIteration<32,6> (solverKernel.cuh:41-153), `sweeps` sweeps from
    zero with the buffer swap of flow.cu:186-193, against the restatement's
    sweeps: bit-identical for the -fmad=false build at the stride the
    reference's demo uses and at stride = width."""
    q, Ix, Iy, Iz = _hs_inputs(refg, w, h, seed=w + sweeps)
    du = np.zeros_like(Ix)
    dv = np.zeros_like(Ix)
    for _ in range(sweeps):
        du, dv = refg.hs_jacobi(du, dv, Ix, Iy, Iz, alpha)
    for stride in (w, _align32(w)):
        rdu, rdv = refg.refg_hs_jacobi(Ix, Iy, Iz, alpha, sweeps, stride=stride)
        assert np.array_equal(rdu, du) and np.array_equal(rdv, dv), stride
    # stock flags: contracted a*b+c round once instead of twice.  Each sweep
    # averages, so the difference stays at the level of a few ulp of the
    # field's magnitude.
    sdu, sdv = refg.refg_hs_jacobi(Ix, Iy, Iz, alpha, sweeps, stride=_align32(w), stock=True)
    scale = max(np.abs(du).max(), np.abs(dv).max(), 1e-30)
    tol = 64 * np.finfo(np.float32).eps * scale
    assert np.abs(sdu - du).max() <= tol and np.abs(sdv - dv).max() <= tol


def test_hs_add_equals_reference(refg):
    """AddKernel (addKernel.cuh:28-36): u + du, both builds."""
    rng = np.random.default_rng(4)
    a = rng.normal(0, 3, (77, 131)).astype(np.float32)
    b = rng.normal(0, 1e-3, (77, 131)).astype(np.float32)
    for stock in (False, True):
        assert np.array_equal(refg.refg_hs_add(a, b, stock=stock), a + b)


def _hs_with_reference_kernels(orc, I0, I1, alpha, L, nw, ns):
    """ComputeFlow's control flow (flow.cu:112-208) with the reference's own
    Downscale, SolveForUpdate and Add kernels (-fmad=false build) and the
    restatement for the steps whose reference kernels are defective: the last
    row and column of the downscale (D-H1), the warp (D-H2), the derivatives
    (D-H3) and the upscale (D-H4)."""
    P0, P1 = [None] * L, [None] * L
    P0[L - 1], P1[L - 1] = np.asarray(I0, np.float32), np.asarray(I1, np.float32)
    for l in range(L - 1, 0, -1):
        for P in (P0, P1):
            d = orc.refg_hs_downscale(P[l])
            r = orc.hs_downscale(P[l])
            d[-1, :], d[:, -1] = r[-1, :], r[:, -1]
            P[l - 1] = d
    u = np.zeros_like(P0[0])
    v = np.zeros_like(P0[0])
    for l in range(L):
        h, w = P0[l].shape
        for _ in range(nw):
            I1w = orc.hs_warp(P1[l], u, v)
            Ix, Iy, Iz = orc.hs_derivatives(P0[l], I1w)
            du, dv = orc.refg_hs_jacobi(Ix, Iy, Iz, alpha, ns, stride=_align32(w))
            u = orc.refg_hs_add(u, du)
            v = orc.refg_hs_add(v, dv)
        if l != L - 1:
            nh, nw_ = P0[l + 1].shape
            sx = np.float32(nw_) / np.float32(w)
            sy = np.float32(nh) / np.float32(h)
            u = orc.upscale(u, nw_, nh, float(sx))
            v = orc.upscale(v, nw_, nh, float(sy))
    return u, v


@pytest.mark.parametrize("alpha,L,nw,ns,w,h", [(15.0, 1, 1, 200, 320, 240),
                                               (0.2, 3, 2, 30, 320, 240),
                                               (5.0, 2, 3, 7, 131, 77)])
def test_hs_solve_equals_reference_kernels(of, refg, ctx, alpha, L, nw, ns, w, h):
    """A whole oflow_hs solve equals ComputeFlow run on the reference's own
    Downscale/Jacobi/Add kernels (with the documented deviations for the
    rest), bit for bit."""
    from oflow import synth
    q = synth.hs_pair(seed=w + h + L, w=w, h=h)
    u, v = of.hs(q.I0, q.I1, of.HSParams(alpha, L, nw, ns), ctx)
    ru, rv = _hs_with_reference_kernels(refg, q.I0, q.I1, alpha, L, nw, ns)
    assert np.array_equal(u, ru) and np.array_equal(v, rv)


@pytest.mark.parametrize("cfg", range(6))
def test_hs_every_jacobi_config_equals_reference_kernels(of, refg, monkeypatch, cfg):
    """Every Jacobi tiling of the library (tile shape, sweeps per launch)
    against the reference kernels: 37 sweeps, ragged tiles, two levels."""
    from oflow import synth
    monkeypatch.setenv("OFLOW_HS_CFG", str(cfg))
    c = of.Context(0)
    q = synth.hs_pair(seed=11, w=203, h=117)
    u, v = of.hs(q.I0, q.I1, of.HSParams(3.0, 2, 2, 37), c)
    c.close()
    ru, rv = _hs_with_reference_kernels(refg, q.I0, q.I1, 3.0, 2, 2, 37)
    assert np.array_equal(u, ru) and np.array_equal(v, rv)


# ------------------------------------------------------------------ LK steps
@pytest.mark.parametrize("spac", [1, 3, 5, 7, 9])
@pytest.mark.parametrize("temp", [1, 2, 3, 5, 7, 9])
def test_lk_filter_taps_equal_reference(refg, spac, temp):
    """getfilters (lucaskanade.cu:79-161): the same tap values."""
    fx, fy, ft = refg.refg_lk_filters(spac, temp)
    fs, ots = refg.lk_filters(spac, temp)
    assert np.array_equal(fx, fs) and np.array_equal(fy, fs) and np.array_equal(ft, ots)


def _ring(seed, w, h, temp):
    from oflow import synth
    rng = np.random.default_rng(seed)
    base = synth.value_noise(rng, h, w)
    return [synth.quantize(base + rng.normal(0, 2, base.shape) + 1.5 * k) for k in range(temp)]


@pytest.mark.parametrize("spac,temp,window,w,h", [(3, 2, 5, 110, 70), (1, 1, 3, 64, 80),
                                                  (5, 3, 7, 97, 61), (7, 5, 9, 120, 90),
                                                  (9, 9, 5, 70, 110)])
def test_lk_equals_reference_kernels(of, refg, ctx, spac, temp, window, w, h):
    """oflow_lk against the reference's temporal FIR, x-FIR and 1-step window
    solve (kernels.cu:14-30, 44-80, 134-181), with the y-FIR taken through the
    reference's x-FIR on the transposed frame (its own y-FIR reads past the
    frame when ny < nx; D-L1).  Flow and border zeros (D-L2) bit-identical."""
    frames = _ring(spac * 100 + temp, w, h, temp)
    for iframe in (0, temp - 1, 2 * temp + 1):
        u, v = of.lk(frames, iframe, of.LKParams(spac, temp, window), ctx)
        rVx, rVy, *_ = refg.refg_lk(frames, iframe, spac, temp, window)
        assert np.array_equal(u, rVx) and np.array_equal(v, rVy), iframe


@pytest.mark.parametrize("spac,temp,window,n", [(3, 2, 5, 96), (5, 3, 7, 80), (9, 9, 9, 64),
                                                (1, 2, 3, 48)])
def test_lk_class_equals_reference_class(of, refg, spac, temp, window, n):
    """The reference LucasKanade class itself (constructor, ring loads,
    lucas_kanade: lucaskanade.cu:5-77) on square frames, where its y-filter is
    in bounds and exact, against the library's LucasKanade shim driven the
    same way.  Interior bit-identical (the reference leaves the border
    unwritten); derivatives of the whole frame bit-identical to the
    parts-based run."""
    frames = _ring(n + window, n, n, temp)
    iframe = temp + 1
    rVx, rVy, rIx, rIy, rIt = refg.refg_lk(frames, iframe, spac, temp, window, whole_class=True)
    pVx, pVy, pIx, pIy, pIt = refg.refg_lk(frames, iframe, spac, temp, window)
    assert np.array_equal(rIx, pIx) and np.array_equal(rIy, pIy) and np.array_equal(rIt, pIt)
    lk = of.LucasKanade(spac, temp, window, n, n)
    for k in range(temp):
        lk.copy_frames_circularbuffer_GPU_wrapper(frames[k].ravel(), temp, k, n * n)
    Vx = np.zeros(n * n, np.float32)
    Vy = np.zeros(n * n, np.float32)
    lk.lucas_kanade(Vx, Vy, iframe)
    r = (window - 1) // 2
    inner = (slice(r, n - r), slice(r, n - r))
    Vx, Vy = Vx.reshape(n, n), Vy.reshape(n, n)
    assert np.array_equal(Vx[inner], rVx[inner]) and np.array_equal(Vy[inner], rVy[inner])


def test_lk_stock_build_within_ulps(refg):
    """The reference's own flags (FMA contraction): derivative planes within a
    few ulp of the -fmad=false build; the flow agrees closely except where the
    2x2 system is near singular, where last-bit differences of the window
    sums are amplified by 1/det."""
    frames = _ring(7, 96, 96, 3)
    a = refg.refg_lk(frames, 2, 5, 3, 7, whole_class=True)
    b = refg.refg_lk(frames, 2, 5, 3, 7, whole_class=True, stock=True)
    for x, y in zip(a[2:], b[2:]):
        tol = 8 * np.finfo(np.float32).eps * max(np.abs(x).max(), 1.0)
        assert np.abs(x - y).max() <= tol
    inner = (slice(3, -3), slice(3, -3))
    d = np.abs(a[0][inner] - b[0][inner])
    assert np.median(d) <= 1e-5 and np.quantile(d, 0.99) <= 1e-2
