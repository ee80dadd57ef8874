"""Synthetic workloads: determinism and the flow convention I1(x+u) = I0(x)."""
import numpy as np

from oflow import synth


def _residual(p, margin=6):
    h, w = p.I0.shape
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    warped = synth.bilinear(p.I1.astype(np.float64), xx + p.u, yy + p.v)
    m = p.valid.copy()
    m[:margin] = m[-margin:] = False
    m[:, :margin] = m[:, -margin:] = False
    return np.abs(warped - p.I0)[m]


def test_deterministic():
    a, b = synth.tvl1_pair(seed=7, w=128, h=64, radius=16), synth.tvl1_pair(seed=7, w=128, h=64, radius=16)
    assert np.array_equal(a.I0, b.I0) and np.array_equal(a.I1, b.I1) and np.array_equal(a.u, b.u)
    c = synth.tvl1_pair(seed=8, w=128, h=64, radius=16)
    assert not np.array_equal(a.I0, c.I0)


def test_hs_pair_convention():
    p = synth.hs_pair(seed=1)
    assert p.I0.shape == (240, 320)
    # two bilinear resamplings of blurred noise leave about one grey level
    assert float(np.median(_residual(p))) < 2.0
    flipped = synth.Pair(p.I0, p.I1, -p.u, -p.v, p.valid)
    assert float(np.median(_residual(flipped))) > 5 * float(np.median(_residual(p)))


def test_lk_pair_convention():
    p = synth.lk_pair(seed=1)
    assert p.I0.shape == (480, 640)
    mag = np.sqrt(p.u ** 2 + p.v ** 2)
    assert 7.5 < mag.max() <= 8.0 + 1e-3
    assert float(np.median(_residual(p))) < 2.0


def test_tvl1_pair_convention_and_occlusion():
    p = synth.tvl1_pair(seed=2)
    assert p.I0.shape == (436, 1024)
    inside = (np.abs(p.u - 12) < 1e-6) & (np.abs(p.v + 5) < 1e-6)
    assert inside.sum() > 0.9 * np.pi * 80 ** 2
    assert (~p.valid).sum() > 0  # occluded background exists
    assert float(np.median(_residual(p))) < 4.0  # N(0,2) noise on both frames


def test_batch_specs():
    s = synth.batch_specs(256, seed=0)
    assert len(s) == 256
    assert sum(1 for x in s if x[0] == "hs") == 128
    assert {(w, h) for _, w, h, _ in s} <= set(synth.BATCH_SIZES)


def test_epe():
    z = np.zeros((10, 10), np.float32)
    o = np.ones((10, 10), np.float32)
    assert synth.epe(o, z, z, z) == 1.0
    assert abs(synth.epe(o, o, z, z) - np.sqrt(2)) < 1e-6
