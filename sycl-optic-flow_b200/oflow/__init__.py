"""oflow: dense optical flow (TV-L1, Horn-Schunck, Lucas-Kanade) on B200.

Python side of the C ABI in include/oflow.h (liboflow.so, sm_100a kernels).
There is no CPU fallback: importing works anywhere, but every solve needs the
built library and a CUDA device and raises otherwise.

Two layers:

* functions ``tvl1``, ``tvl1_batch``, ``hs``, ``hs_batch``, ``lk``,
  ``pyrlk`` taking numpy arrays (host) or CUDA torch tensors (device) and
  returning (u, v);
* classes mirroring the reference entry points: ``TV_L1``
  (src/tvl1/sequential/tvl1.hpp:10-17, src/tvl1/cuda/tvl1.cuh:12-20),
  ``initFlow`` / ``ComputeFlow`` / ``deleteFlow_mem`` (src/hs/cuda/flow.cuh:
  19-33) and ``LucasKanade`` (src/lk/cuda/lucaskanade.cuh:6-12).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from .capi import (LIB_PATH, SOLVER_HS, SOLVER_TVL1, BgrImage, Flow, StreamDesc, HsParams, Image, Job, LkParams,
                   MAX_SCALES, OflowError, Tvl1Params, Tvl1Profile, Tvl1Stats, lib, status_string)

__all__ = [
    "Context", "OflowError", "TVL1Params", "HSParams", "LKParams", "tvl1", "tvl1_batch",
    "tvl1_energy_trace", "hs", "hs_batch", "lk", "pyrlk", "pyrlk_batch", "TV_L1", "initFlow", "ComputeFlow",
    "deleteFlow_mem", "LucasKanade", "nscales", "LIB_PATH", "flow_to_color", "flow_to_color_batch",
    "save_ppm", "FrameStream",
]


@dataclass
class TVL1Params:
    """Defaults of src/tvl1/sequential/tvl1.hpp:6,12-14."""
    tau: float = 0.25
    lambda_: float = 0.15
    theta: float = 0.3
    nscales: int = 100
    zfactor: float = 0.5
    warps: int = 5
    epsilon: float = 0.01
    max_iterations: int = 300

    def c(self) -> Tvl1Params:
        return Tvl1Params(self.tau, self.lambda_, self.theta, self.nscales, self.zfactor,
                          self.warps, self.epsilon, self.max_iterations)


@dataclass
class HSParams:
    """Defaults of the reference demo (src/hs/cuda/main.cu:140-148)."""
    alpha: float = 0.2
    nlevels: int = 5
    nwarp: int = 3
    nsolver: int = 150

    def c(self) -> HsParams:
        return HsParams(self.alpha, self.nlevels, self.nwarp, self.nsolver)


@dataclass
class LKParams:
    """Defaults of the reference demo (src/lk/cuda/main.cu:132-134) plus the
    pyramid shape used by oflow_pyrlk."""
    spac: int = 3
    temp: int = 2
    window: int = 5
    levels: int = 3
    iters: int = 3

    def c(self) -> LkParams:
        return LkParams(self.spac, self.temp, self.window, self.levels, self.iters)


def _check(status, ctx=None):
    if status != 0:
        msg = status_string(status)
        if ctx is not None:
            detail = lib().oflow_ctx_last_error(ctx).decode()
            if detail:
                msg += ": " + detail
        raise OflowError(status, msg)


class Context:
    """One oflow context (device, stream, cached plans).  Use from one thread."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        _check(lib().oflow_ctx_create(device, C.byref(self._h)))
        self.device = device

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int | None):
        _check(lib().oflow_ctx_set_stream(self._h, C.c_void_p(stream_ptr or 0)), self._h)

    def trim(self):
        _check(lib().oflow_ctx_trim(self._h), self._h)

    def last_launches(self) -> int:
        """Kernel launches the last tvl1 / tvl1_batch call executed on the device."""
        n = C.c_longlong()
        _check(lib().oflow_ctx_last_launches(self.handle, C.byref(n)), self.handle)
        return n.value

    def save_tuning(self, path: str):
        _check(lib().oflow_ctx_save_tuning(self._h, os.fsencode(path)), self._h)

    def load_tuning(self, path: str):
        _check(lib().oflow_ctx_load_tuning(self._h, os.fsencode(path)), self._h)

    def close(self):
        if self._h:
            lib().oflow_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


# ------------------------------------------------------------------ marshalling
def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _image(x) -> tuple[Image, object]:
    """numpy (host) or torch CUDA tensor (device) -> oflow_image, keep-alive."""
    if _is_torch(x):
        import torch
        if x.dim() != 2:
            raise ValueError("frames must be 2-D")
        if x.dtype == torch.uint8:
            dt = 0
        elif x.dtype == torch.float32:
            dt = 1
        else:
            raise TypeError("frames must be uint8 or float32")
        if x.stride(1) != 1:
            x = x.contiguous()
        loc = 1 if x.is_cuda else 0
        return Image(C.c_void_p(x.data_ptr()), x.shape[1], x.shape[0], x.stride(0), dt, loc), x
    a = np.asarray(x)
    if a.ndim != 2:
        raise ValueError("frames must be 2-D")
    if a.dtype == np.uint8:
        dt = 0
    elif a.dtype == np.float32:
        dt = 1
    else:
        a = a.astype(np.float32)
        dt = 1
    a = np.ascontiguousarray(a)
    return Image(a.ctypes.data_as(C.c_void_p), a.shape[1], a.shape[0], a.shape[1], dt, 0), a


def _outputs(like, h, w, out=None):
    """Allocate (u, v) on the same side as `like` unless given."""
    if out is not None:
        u, v = out
    elif _is_torch(like) and like.is_cuda:
        import torch
        u = torch.empty((h, w), dtype=torch.float32, device=like.device)
        v = torch.empty((h, w), dtype=torch.float32, device=like.device)
    else:
        u = np.empty((h, w), np.float32)
        v = np.empty((h, w), np.float32)
    if _is_torch(u):
        f = Flow(C.cast(C.c_void_p(u.data_ptr()), C.POINTER(C.c_float)),
                 C.cast(C.c_void_p(v.data_ptr()), C.POINTER(C.c_float)), u.stride(0),
                 1 if u.is_cuda else 0)
    else:
        f = Flow(u.ctypes.data_as(C.POINTER(C.c_float)), v.ctypes.data_as(C.POINTER(C.c_float)),
                 u.shape[1], 0)
    return f, (u, v)


def _ctx(ctx):
    return (ctx or default_context()).handle


# ------------------------------------------------------------------ TV-L1
def nscales(width, height, params: TVL1Params | None = None) -> int:
    p = (params or TVL1Params()).c()
    return lib().oflow_tvl1_nscales(width, height, C.byref(p))


def _stats_dict(s: Tvl1Stats):
    its = np.ctypeslib.as_array(s.iterations)[: s.nscales * s.warps].reshape(s.nscales, s.warps)
    return {"nscales": s.nscales, "warps": s.warps, "iterations": its.copy(), "energy": s.energy}


def tvl1_batch(pairs, params: TVL1Params | None = None, ctx: Context | None = None,
               stats: bool = False, out=None):
    """Solve a list of (I0, I1) pairs in one schedule.  Returns a list of
    (u, v) (and a list of stats dicts if stats=True)."""
    p = (params or TVL1Params()).c()
    n = len(pairs)
    I0 = (Image * n)()
    I1 = (Image * n)()
    O = (Flow * n)()
    keep, res = [], []
    for i, (a, b) in enumerate(pairs):
        I0[i], ka = _image(a)
        I1[i], kb = _image(b)
        keep += [ka, kb]
        O[i], uv = _outputs(a, I0[i].height, I0[i].width, None if out is None else out[i])
        res.append(uv)
    st = (Tvl1Stats * n)() if stats else None
    h = _ctx(ctx)
    _check(lib().oflow_tvl1_batch(h, n, I0, I1, C.byref(p), O, st), h)
    if stats:
        return res, [_stats_dict(s) for s in st]
    return res


def tvl1_batch_profile(pairs, params: TVL1Params | None = None, ctx: Context | None = None,
                       out=None):
    """tvl1_batch (equal sizes) run eagerly with CUDA events around every warp
    and inner-iteration launch.  Returns (results, stats, profile dict)."""
    p = (params or TVL1Params()).c()
    n = len(pairs)
    I0 = (Image * n)()
    I1 = (Image * n)()
    O = (Flow * n)()
    keep, res = [], []
    for i, (a, b) in enumerate(pairs):
        I0[i], ka = _image(a)
        I1[i], kb = _image(b)
        keep += [ka, kb]
        O[i], uv = _outputs(a, I0[i].height, I0[i].width, None if out is None else out[i])
        res.append(uv)
    st = (Tvl1Stats * n)()
    pr = Tvl1Profile()
    h = _ctx(ctx)
    _check(lib().oflow_tvl1_batch_profile(h, n, I0, I1, C.byref(p), O, st, C.byref(pr)), h)
    prof = {k: getattr(pr, k) for k, _ in Tvl1Profile._fields_}
    prof["iter_ms_scale"] = list(pr.iter_ms_scale)
    return res, [_stats_dict(s) for s in st], prof


def tvl1_autotune(pairs, params: TVL1Params | None = None, ctx: Context | None = None):
    """Tune the blocked-iteration configuration per scale for this size and
    batch (see oflow_tvl1_autotune).  Returns the chosen config per scale."""
    p = (params or TVL1Params()).c()
    n = len(pairs)
    I0 = (Image * n)()
    I1 = (Image * n)()
    keep = []
    for i, (a, b) in enumerate(pairs):
        I0[i], ka = _image(a)
        I1[i], kb = _image(b)
        keep += [ka, kb]
    cfg = (C.c_int * 16)()
    h = _ctx(ctx)
    _check(lib().oflow_tvl1_autotune(h, n, I0, I1, C.byref(p), cfg), h)
    return [c for c in cfg if c >= 0]


def tvl1(I0, I1, params: TVL1Params | None = None, ctx: Context | None = None,
         stats: bool = False, out=None):
    r = tvl1_batch([(I0, I1)], params, ctx, stats, None if out is None else [out])
    if stats:
        return r[0][0][0], r[0][0][1], r[1][0]
    return r[0]


def tvl1_energy_trace(I0, I1, params: TVL1Params | None = None, ctx: Context | None = None):
    """Solve one pair and return (u, v, stats, energy[nscales, warps, max_iterations])
    with the energy after every inner iteration (NaN where a stage stopped)."""
    prm = params or TVL1Params()
    p = prm.c()
    a, ka = _image(I0)
    b, kb = _image(I1)
    f, (u, v) = _outputs(I0, a.height, a.width)
    ns = nscales(a.width, a.height, prm)
    en = np.full(ns * prm.warps * max(prm.max_iterations, 1), np.nan, np.float64)
    st = Tvl1Stats()
    h = _ctx(ctx)
    _check(lib().oflow_tvl1_energy_trace(h, C.byref(a), C.byref(b), C.byref(p), C.byref(f),
                                         C.byref(st), en.ctypes.data_as(C.POINTER(C.c_double))), h)
    return u, v, _stats_dict(st), en.reshape(ns, prm.warps, max(prm.max_iterations, 1))


# ------------------------------------------------------------------ Horn-Schunck
def hs_batch(pairs, params: HSParams | None = None, ctx: Context | None = None, out=None):
    p = (params or HSParams()).c()
    n = len(pairs)
    I0 = (Image * n)()
    I1 = (Image * n)()
    O = (Flow * n)()
    keep, res = [], []
    for i, (a, b) in enumerate(pairs):
        I0[i], ka = _image(a)
        I1[i], kb = _image(b)
        keep += [ka, kb]
        O[i], uv = _outputs(a, I0[i].height, I0[i].width, None if out is None else out[i])
        res.append(uv)
    h = _ctx(ctx)
    _check(lib().oflow_hs_batch(h, n, I0, I1, C.byref(p), O), h)
    return res


def hs(I0, I1, params: HSParams | None = None, ctx: Context | None = None, out=None):
    return hs_batch([(I0, I1)], params, ctx, None if out is None else [out])[0]


def hs_autotune(pairs, params: HSParams | None = None, ctx: Context | None = None):
    """Tune the Jacobi configuration (tile shape, sweeps per launch) per
    pyramid level for this size and batch (see oflow_hs_autotune).  Returns
    the chosen config per level, coarsest first."""
    p = (params or HSParams()).c()
    n = len(pairs)
    I0 = (Image * n)()
    I1 = (Image * n)()
    keep = []
    for i, (a, b) in enumerate(pairs):
        I0[i], ka = _image(a)
        I1[i], kb = _image(b)
        keep += [ka, kb]
    cfg = (C.c_int * 16)()
    h = _ctx(ctx)
    _check(lib().oflow_hs_autotune(h, n, I0, I1, C.byref(p), cfg), h)
    return [c for c in cfg if c >= 0]


# ------------------------------------------------------------------ mixed batches
def batch(jobs, ctx: Context | None = None, out=None):
    """Solve a mixed list of jobs ("tvl1" | "hs", I0, I1, params) as one
    schedule (oflow_batch).  Returns a list of (u, v)."""
    n = len(jobs)
    J = (Job * n)()
    keep, res = [], []
    for i, (solver, a, b, prm) in enumerate(jobs):
        ia, ka = _image(a)
        ib, kb = _image(b)
        f, uv = _outputs(a, ia.height, ia.width, None if out is None else out[i])
        cp = prm.c()
        keep += [ka, kb, cp]
        if solver == "tvl1":
            J[i] = Job(SOLVER_TVL1, ia, ib, C.pointer(cp), None, f)
        elif solver == "hs":
            J[i] = Job(SOLVER_HS, ia, ib, None, C.pointer(cp), f)
        else:
            raise ValueError("solver must be 'tvl1' or 'hs'")
        res.append(uv)
    h = _ctx(ctx)
    _check(lib().oflow_batch(h, n, J), h)
    return res


# ------------------------------------------------------------------ warm start
def net_num_params() -> int:
    return lib().oflow_net_num_params()


class WarmNet:
    """The warm-start network (oflow_net_*) for `batch` pairs of width x
    height.  Frames and targets are CUDA torch tensors."""

    def __init__(self, width: int, height: int, batch: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self._h = C.c_void_p()
        _check(lib().oflow_net_create(self.ctx.handle, width, height, batch, C.byref(self._h)),
               self.ctx.handle)
        ow, oh = C.c_int(), C.c_int()
        lib().oflow_net_out_size(self._h, C.byref(ow), C.byref(oh))
        self.width, self.height, self.batch = width, height, batch
        self.out_w, self.out_h = ow.value, oh.value

    @property
    def handle(self):
        return self._h

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, np.float32)
        if p.size != net_num_params():
            raise ValueError("wrong number of parameters")
        _check(lib().oflow_net_set_params(self._h, p.ctypes.data_as(C.c_void_p)), self.ctx.handle)

    def get_params(self) -> np.ndarray:
        p = np.empty(net_num_params(), np.float32)
        _check(lib().oflow_net_get_params(self._h, p.ctypes.data_as(C.c_void_p)), self.ctx.handle)
        return p

    def train_step(self, frames, target, lr: float) -> float:
        """frames: CUDA [batch, 2, h, w] uint8/float32; target: CUDA float32
        [batch, out_h, out_w, 2]."""
        import torch
        dt = 0 if frames.dtype == torch.uint8 else 1
        loss = C.c_double()
        _check(lib().oflow_net_train_step(self._h, C.c_void_p(frames.data_ptr()), dt,
                                          C.c_void_p(target.data_ptr()), lr, C.byref(loss)),
               self.ctx.handle)
        return loss.value

    def predict(self, frames):
        import torch
        dt = 0 if frames.dtype == torch.uint8 else 1
        out = torch.empty((self.batch, self.out_h, self.out_w, 2), dtype=torch.float32,
                          device=frames.device)
        _check(lib().oflow_net_predict(self._h, C.c_void_p(frames.data_ptr()), dt,
                                       C.c_void_p(out.data_ptr())), self.ctx.handle)
        return out

    def close(self):
        if self._h:
            lib().oflow_net_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tvl1_warm(pairs, net: WarmNet, warm: TVL1Params, plain: TVL1Params | None = None,
              ctx: Context | None = None, out=None, warps_per_scale=None, iters_per_scale=None):
    """Warm-started TV-L1 (oflow_tvl1_warm).  warps_per_scale /
    iters_per_scale: optional per-scale schedule (index 0 = finest).  Returns
    (results, info) with info = {energy_warm, energy_plain, epe_vs_plain,
    accepted} arrays and "stats", the warm solve's per-pair iteration dicts."""
    n = len(pairs)
    I0 = (Image * n)()
    I1 = (Image * n)()
    O = (Flow * n)()
    keep, res = [], []
    for i, (a, b) in enumerate(pairs):
        I0[i], ka = _image(a)
        I1[i], kb = _image(b)
        keep += [ka, kb]
        O[i], uv = _outputs(a, I0[i].height, I0[i].width, None if out is None else out[i])
        res.append(uv)
    ew = np.zeros(n, np.float64)
    ep = np.zeros(n, np.float64)
    er = np.zeros(n, np.float64)
    acc = np.zeros(n, np.int32)
    st = (Tvl1Stats * n)()
    wp = warm.c()
    pp = plain.c() if plain is not None else None

    def sched(a):
        if a is None:
            return None, None
        arr = np.zeros(MAX_SCALES, np.int32)
        arr[:len(a)] = a
        return arr, arr.ctypes.data_as(C.c_void_p)

    ws, wsp = sched(warps_per_scale)
    its, itp = sched(iters_per_scale)
    h = (ctx or net.ctx).handle
    _check(lib().oflow_tvl1_warm(h, net.handle, n, I0, I1, C.byref(wp), wsp, itp,
                                 C.byref(pp) if pp is not None else None, O,
                                 ew.ctypes.data_as(C.c_void_p), ep.ctypes.data_as(C.c_void_p),
                                 er.ctypes.data_as(C.c_void_p),
                                 acc.ctypes.data_as(C.c_void_p), st), h)
    return res, {"energy_warm": ew, "energy_plain": ep, "epe_vs_plain": er,
                 "accepted": acc.astype(bool), "stats": [_stats_dict(s) for s in st]}


def conv3x3(mode, N, H, W, C_, K, stride, relu, out_f32, a, y_act, b, out, bias=None, gbias=None):
    """oflow_conv3x3 on CUDA torch tensors (validation of the network kernels)."""
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    _check(lib().oflow_conv3x3(mode, N, H, W, C_, K, stride, int(relu), int(out_f32), ptr(a),
                               ptr(y_act), ptr(b), ptr(out), ptr(bias), ptr(gbias), None))


# ------------------------------------------------------------------ Lucas-Kanade
def lk(frames, iframe: int, params: LKParams | None = None, ctx: Context | None = None,
       out=None):
    """Single-step LK over a ring of `params.temp` uint8 frames (frames[k] = ring
    slot k, newest frame in slot iframe % temp)."""
    prm = params or LKParams()
    p = prm.c()
    T = prm.temp
    if len(frames) != T:
        raise ValueError("lk: need exactly `temp` ring frames")
    arr = (Image * T)()
    keep = []
    for k in range(T):
        arr[k], kk = _image(frames[k])
        keep.append(kk)
    f, uv = _outputs(frames[0], arr[0].height, arr[0].width, out)
    h = _ctx(ctx)
    _check(lib().oflow_lk(h, arr, iframe, C.byref(p), C.byref(f)), h)
    return uv


def pyrlk(I0, I1, params: LKParams | None = None, ctx: Context | None = None, out=None):
    p = (params or LKParams()).c()
    a, ka = _image(I0)
    b, kb = _image(I1)
    f, uv = _outputs(I0, a.height, a.width, out)
    h = _ctx(ctx)
    _check(lib().oflow_pyrlk(h, C.byref(a), C.byref(b), C.byref(p), C.byref(f)), h)
    return uv


def pyrlk_batch(pairs, params: LKParams | None = None, ctx: Context | None = None, out=None):
    """oflow_pyrlk_batch: pyramidal LK of many pairs in one call."""
    p = (params or LKParams()).c()
    n = len(pairs)
    I0 = (Image * n)()
    I1 = (Image * n)()
    O = (Flow * n)()
    keep, res = [], []
    for i, (a, b) in enumerate(pairs):
        I0[i], ka = _image(a)
        I1[i], kb = _image(b)
        keep += [ka, kb]
        O[i], uv = _outputs(a, I0[i].height, I0[i].width, None if out is None else out[i])
        res.append(uv)
    h = _ctx(ctx)
    _check(lib().oflow_pyrlk_batch(h, n, I0, I1, C.byref(p), O), h)
    return res


# ------------------------------------------------------------------ streams
class FrameStream:
    """oflow_stream_*: `lanes` videos of width x height; push() takes one new
    frame per lane, uploads it once and returns the flows of the pairs
    (previous frame, new frame); before a lane's first frame the previous
    frame is all zeros (the reference's streaming TV-L1)."""

    def __init__(self, width: int, height: int, solver: str = "tvl1", lanes: int = 1,
                 params=None, dtype: str = "u8", ctx: Context | None = None):
        self.ctx = ctx or default_context()
        d = StreamDesc()
        d.solver = {"tvl1": SOLVER_TVL1, "hs": SOLVER_HS}[solver]
        d.width, d.height, d.lanes = width, height, lanes
        d.dtype = {"u8": 0, "f32": 1}[dtype]
        d.tvl1 = (params if solver == "tvl1" and params is not None else TVL1Params()).c()
        d.hs = (params if solver == "hs" and params is not None else HSParams()).c()
        self.width, self.height, self.lanes, self.solver = width, height, lanes, solver
        self._h = C.c_void_p()
        _check(lib().oflow_stream_create(self.ctx.handle, C.byref(d), C.byref(self._h)),
               self.ctx.handle)

    @property
    def frames(self) -> int:
        return int(lib().oflow_stream_frames(self._h))

    def push(self, frames, out=None, stats: bool = False):
        """frames: list of `lanes` 2-D frames (numpy or torch).  Returns a list
        of (u, v) (and stats dicts for TV-L1 when stats=True)."""
        if len(frames) != self.lanes:
            raise ValueError("push: one frame per lane")
        I = (Image * self.lanes)()
        O = (Flow * self.lanes)()
        keep, res = [], []
        for i, f in enumerate(frames):
            I[i], k = _image(f)
            keep.append(k)
            O[i], uv = _outputs(f, self.height, self.width, None if out is None else out[i])
            res.append(uv)
        st = (Tvl1Stats * self.lanes)() if stats and self.solver == "tvl1" else None
        _check(lib().oflow_stream_push(self._h, I, O, st), self.ctx.handle)
        if st is not None:
            return res, [_stats_dict(x) for x in st]
        return res

    def close(self):
        if getattr(self, "_h", None):
            lib().oflow_stream_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ visualisation
def flow_to_color_batch(flows, ctx: Context | None = None, out=None):
    """oflow_flow_to_color on a list of (u, v) flows of one size: returns B, G, R
    images [h, w, 3] uint8 (torch CUDA tensors for CUDA flows, numpy otherwise)."""
    n = len(flows)
    if n == 0:
        return []
    F = (Flow * n)()
    O = (BgrImage * n)()
    keep, res = [], []
    h, w = flows[0][0].shape
    for i, (u, v) in enumerate(flows):
        if tuple(u.shape) != (h, w) or tuple(v.shape) != (h, w):
            raise ValueError("flow_to_color: flows must share one size")
        if _is_torch(u):
            if u.dtype != v.dtype or str(u.dtype) != "torch.float32":
                raise ValueError("flow_to_color: float32 flows")
            u, v = u.contiguous(), v.contiguous()
            keep += [u, v]
            F[i] = Flow(C.cast(C.c_void_p(u.data_ptr()), C.POINTER(C.c_float)),
                        C.cast(C.c_void_p(v.data_ptr()), C.POINTER(C.c_float)), w,
                        1 if u.is_cuda else 0)
            dev = u.is_cuda
        else:
            u = np.ascontiguousarray(u, np.float32)
            v = np.ascontiguousarray(v, np.float32)
            keep += [u, v]
            F[i] = Flow(u.ctypes.data_as(C.POINTER(C.c_float)), v.ctypes.data_as(C.POINTER(C.c_float)),
                        w, 0)
            dev = False
        if out is not None:
            img = out[i]
        elif dev:
            import torch
            img = torch.empty((h, w, 3), dtype=torch.uint8, device=u.device)
        else:
            img = np.empty((h, w, 3), np.uint8)
        if _is_torch(img):
            O[i] = BgrImage(img.data_ptr(), img.stride(0), 1 if img.is_cuda else 0)
        else:
            O[i] = BgrImage(img.ctypes.data, img.strides[0], 0)
        res.append(img)
    hd = _ctx(ctx)
    _check(lib().oflow_flow_to_color(hd, n, w, h, F, O), hd)
    return res


def flow_to_color(u, v, ctx: Context | None = None, out=None):
    """B, G, R image [h, w, 3] uint8 of one flow (the demos' flowToColor)."""
    return flow_to_color_batch([(u, v)], ctx, None if out is None else [out])[0]


def save_ppm(path: str, bgr) -> None:
    """Write a B, G, R byte image [h, w, 3] as a binary PPM (RGB) file."""
    a = bgr.cpu().numpy() if _is_torch(bgr) else np.asarray(bgr)
    h, w, _ = a.shape
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(np.ascontiguousarray(a[:, :, ::-1]).tobytes())


from .compat import TV_L1, ComputeFlow, LucasKanade, deleteFlow_mem, initFlow  # noqa: E402
