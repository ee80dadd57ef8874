"""Drop-in mirrors of the reference's solver entry points, over the C ABI.

Same names, argument meaning and output layout as the reference; the work
runs on the GPU through liboflow.so.  Errors raise OflowError (the reference
prints, terminates or exits instead).
"""
from __future__ import annotations

import numpy as np

from . import LKParams, HSParams, TVL1Params, hs as _hs, lk as _lk, tvl1 as _tvl1


class TV_L1:
    """src/tvl1/sequential/tvl1.hpp:10-17 and src/tvl1/cuda/tvl1.cuh:12-20.

    ``runDualTVL1Multiscale(I0, I1)`` takes two uint8 frames (sequential form);
    ``runDualTVL1Multiscale(I)`` takes one float frame and pairs it with the
    previous call's frame (CUDA/SYCL streaming form, src/tvl1/cuda/tvl1.cu:
    122-130; before the first frame the previous frame is all zeros).
    ``getU()`` returns the planar flow [u (w*h) | v (w*h)], valid until the next
    call.  ``max_iterations`` is the reference's compile-time MAX_ITERATIONS.
    """

    def __init__(self, width, height, tau=0.25, lambda_=0.15, theta=0.3, nscales=100,
                 zfactor=0.5, warps=5, epsilon=0.01, max_iterations=300, ctx=None):
        self._w, self._h = int(width), int(height)
        self.params = TVL1Params(tau, lambda_, theta, nscales, zfactor, warps, epsilon,
                                 max_iterations)
        self._ctx = ctx
        self._u = np.zeros(2 * self._w * self._h, np.float32)
        self._prev = None
        self.stats = None

    def runDualTVL1Multiscale(self, I0, I1=None):
        if I1 is None:
            cur = np.ascontiguousarray(np.asarray(I0, np.float32).reshape(self._h, self._w))
            prev = self._prev if self._prev is not None else np.zeros_like(cur)
            self._prev = cur
            a, b = prev, cur
        else:
            a = np.asarray(I0).reshape(self._h, self._w)
            b = np.asarray(I1).reshape(self._h, self._w)
        n = self._w * self._h
        u = self._u[:n].reshape(self._h, self._w)
        v = self._u[n:].reshape(self._h, self._w)
        _, _, self.stats = _tvl1(a, b, self.params, self._ctx, stats=True, out=(u, v))

    def getU(self):
        return self._u


def initFlow(nLevels, stride, width, height):
    """src/hs/cuda/flow.cu:46-72.  Device buffers live in the context's plan
    cache, so this only validates its arguments."""
    if stride < width or nLevels < 1:
        raise ValueError("initFlow: stride < width or nLevels < 1")


def deleteFlow_mem(nLevels):
    """src/hs/cuda/flow.cu:74-93 (buffers are released with the context)."""


def ComputeFlow(I0, I1, width, height, stride, alpha, nLevels, nWarpIters, nSolverIters, u, v,
                ctx=None):
    """src/hs/cuda/flow.cu:112-208: frames of `height` rows of `stride` floats;
    u, v (same layout) receive the flow."""
    a = np.asarray(I0, np.float32).reshape(height, stride)[:, :width]
    b = np.asarray(I1, np.float32).reshape(height, stride)[:, :width]
    uo = np.asarray(u).reshape(height, stride)
    vo = np.asarray(v).reshape(height, stride)
    ru, rv = _hs(np.ascontiguousarray(a), np.ascontiguousarray(b),
                 HSParams(alpha, nLevels, nWarpIters, nSolverIters), ctx)
    uo[:, :width] = ru
    vo[:, :width] = rv


class LucasKanade:
    """src/lk/cuda/lucaskanade.cuh:6-12: a ring of ``temp_filt_size`` uint8
    frames; ``copy_frames_circularbuffer_GPU_wrapper`` stores a frame in slot
    fr % T, ``lucas_kanade`` solves with the newest frame in slot iframe % T."""

    def __init__(self, spac_filt_size, temp_filt_size, window_size, nx, ny, ctx=None):
        self.params = LKParams(spac_filt_size, temp_filt_size, window_size)
        self.nx, self.ny = int(nx), int(ny)
        self._ring = [np.zeros((self.ny, self.nx), np.uint8) for _ in range(temp_filt_size)]
        self._ctx = ctx

    def copy_frames_circularbuffer_GPU_wrapper(self, frame, temp_size, fr, frame_size):
        if temp_size != self.params.temp or frame_size != self.nx * self.ny:
            raise ValueError("ring size or frame size does not match the object")
        self._ring[fr % temp_size] = np.ascontiguousarray(
            np.asarray(frame, np.uint8).reshape(self.ny, self.nx))

    def lucas_kanade(self, Vx, Vy, iframe):
        ru, rv = _lk(self._ring, iframe, self.params, self._ctx)
        np.asarray(Vx).reshape(self.ny, self.nx)[:] = ru
        np.asarray(Vy).reshape(self.ny, self.nx)[:] = rv
