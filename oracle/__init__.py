"""CPU oracle for the optical-flow solvers -- TEST INFRASTRUCTURE ONLY.

Two libraries, both used only as the checker by tests/, the smoke check and
the CPU-baseline leg of bench.py (never by the product path):

* ``liboracle.so`` -- the C restatement in ``oracle.c`` (TV-L1, HS, LK).
* ``_ref/libtvl1_ref.so`` -- the reference's own sequential TV-L1
  (src/tvl1/sequential) compiled from its sources in place by
  ``build_ref.sh``.  Present only where the reference checkout was available
  at build time (it travels with the tree as a built file).
* ``_ref/libhslk_ref.so`` / ``_ref/libhslk_ref_stock.so`` -- the reference's
  Horn-Schunck and Lucas-Kanade CUDA kernels (src/hs/cuda/kernels,
  src/lk/cuda) behind ``ref_gpu_harness.cu``, built by ``build_ref.sh`` with
  -fmad=false and with the reference's own flags.  They need a GPU.

Arrays are numpy, row-major, C-contiguous float32 / uint8.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtvl1_ref.so")
REFG_SO = {False: os.path.join(HERE, "_ref", "libhslk_ref.so"),
           True: os.path.join(HERE, "_ref", "libhslk_ref_stock.so")}

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> None:
    """Compile liboracle.so (and _ref when the reference checkout is present)."""
    subprocess.check_call(["make", "-s", "-C", HERE])


class _Params(C.Structure):
    _fields_ = [("tau", C.c_float), ("lambda_", C.c_float), ("theta", C.c_float),
                ("nscales", C.c_int), ("zfactor", C.c_float), ("warps", C.c_int),
                ("epsilon", C.c_float), ("max_iterations", C.c_int),
                ("error_mode", C.c_int)]


class _Trace(C.Structure):
    _fields_ = [("iterations", C.c_void_p), ("energy", C.c_void_p)]


@dataclass
class TVL1Params:
    """Reference defaults (src/tvl1/sequential/tvl1.hpp:12-14) with the
    inner-iteration cap of the 1024x436 workload."""
    tau: float = 0.25
    lambda_: float = 0.15
    theta: float = 0.3
    nscales: int = 5
    zfactor: float = 0.5
    warps: int = 5
    epsilon: float = 0.01
    max_iterations: int = 50

    def c(self, error_mode: int = 0) -> _Params:
        return _Params(self.tau, self.lambda_, self.theta, self.nscales, self.zfactor,
                       self.warps, self.epsilon, self.max_iterations, error_mode)


_orc = None
_ref = None
_refg = {}


def orc_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = C.CDLL(ORACLE_SO)
        lib.orc_gaussian.argtypes = [_f32p, C.c_int, C.c_int, C.c_double]
        lib.orc_gaussian.restype = C.c_int
        lib.orc_gaussian_window.argtypes = [C.c_double]
        lib.orc_gaussian_window.restype = C.c_int
        lib.orc_bicubic_at.argtypes = [_f32p, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int]
        lib.orc_bicubic_at.restype = C.c_float
        lib.orc_bicubic_warp.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int]
        lib.orc_zoom_out.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_float]
        lib.orc_zoom_out.restype = C.c_int
        lib.orc_zoom_in.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.orc_zoom_size.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_float]
        lib.orc_centered_gradient.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int]
        lib.orc_divergence.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int]
        lib.orc_forward_gradient.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int]
        lib.orc_normalize.argtypes = [_f32p, _f32p, C.c_int]
        lib.orc_tvl1_nscales.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float]
        lib.orc_tvl1_nscales.restype = C.c_int
        lib.orc_dual_tvl1.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int,
                                      C.POINTER(_Params), C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_tvl1.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.POINTER(_Params), _f32p,
                                 _f32p, C.POINTER(_Trace)]
        lib.orc_tvl1.restype = C.c_int
        lib.orc_tvl1_energy.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int,
                                        C.c_float]
        lib.orc_tvl1_energy.restype = C.c_double
        lib.orc_hs.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                               C.c_int, _f32p, _f32p]
        lib.orc_hs.restype = C.c_int
        lib.orc_hs_downscale.argtypes = [_f32p, C.c_int, C.c_int, _f32p]
        lib.orc_hs_warp.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int, _f32p]
        lib.orc_hs_derivatives.argtypes = [_f32p, _f32p, C.c_int, C.c_int, _f32p, _f32p, _f32p]
        lib.orc_hs_jacobi.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int,
                                      C.c_float, _f32p, _f32p]
        lib.orc_upscale.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, _f32p]
        lib.orc_lk_filters.argtypes = [C.c_int, C.c_int, _f32p, _f32p]
        lib.orc_lk_filters.restype = C.c_int
        lib.orc_lk.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_int,
                               C.c_int, C.c_int, _f32p, _f32p]
        lib.orc_lk.restype = C.c_int
        lib.orc_lk_f32.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p]
        lib.orc_lk_f32.restype = C.c_int
        lib.orc_bilinear_warp.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int, _f32p]
        lib.orc_flow_to_color.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_void_p]
        lib.orc_flow_to_color.restype = None
        lib.orc_pyrlk.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_int, _f32p, _f32p]
        lib.orc_pyrlk.restype = C.c_int
        _orc = lib
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    """The reference's sequential TV-L1 (compiled in place).  Raises if absent."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        lib = C.CDLL(REF_SO)
        lib.ref_set_max_iterations.argtypes = [C.c_longlong]
        lib.ref_tvl1_nscales.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float]
        lib.ref_tvl1_nscales.restype = C.c_int
        lib.ref_tvl1_run.argtypes = [_u8p, _u8p, C.c_int, C.c_int, C.c_float, C.c_float,
                                     C.c_float, C.c_int, C.c_float, C.c_int, C.c_float,
                                     _f32p, _f32p]
        lib.ref_tvl1_run.restype = C.c_int
        lib.ref_tvl1_level.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_int),
                                       C.POINTER(C.c_int)]
        lib.ref_tvl1_level.restype = C.c_int
        lib.ref_dual_tvl1.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_float,
                                      C.c_float, C.c_float, C.c_int, C.c_float, C.c_void_p]
        lib.ref_normalize.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int]
        lib.ref_gaussian.argtypes = [_f32p, C.c_int, C.c_int, C.c_double]
        lib.ref_gaussian.restype = C.c_int
        lib.ref_zoom_out.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_float]
        lib.ref_zoom_out.restype = C.c_int
        lib.ref_zoom_in.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.ref_bicubic_at.argtypes = [_f32p, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int]
        lib.ref_bicubic_at.restype = C.c_float
        lib.ref_bicubic_warp.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int]
        lib.ref_centered_gradient.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int]
        lib.ref_divergence.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int]
        lib.ref_forward_gradient.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int]
        _ref = lib
    return _ref


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ---------------------------------------------------------------- restatement
def tvl1(I0, I1, params: TVL1Params | None = None, error_mode: int = 0,
         trace: bool = False):
    """Full multiscale TV-L1 on float frames.  Returns (u, v) or
    (u, v, iterations[nscales, warps], energy[nscales, warps, max_it])."""
    p = params or TVL1Params()
    I0 = _f32(I0)
    I1 = _f32(I1)
    h, w = I0.shape
    u = np.zeros_like(I0)
    v = np.zeros_like(I0)
    lib = orc_lib()
    ns = lib.orc_tvl1_nscales(w, h, p.nscales, p.zfactor)
    its = np.zeros((max(ns, 1), p.warps), np.int32)
    en = np.full((max(ns, 1), p.warps, p.max_iterations), np.nan, np.float64)
    tr = _Trace(its.ctypes.data, en.ctypes.data) if trace else _Trace(None, None)
    cp = p.c(error_mode)
    rc = lib.orc_tvl1(I0, I1, w, h, C.byref(cp), u, v, C.byref(tr))
    if rc < 0:
        raise ValueError("oracle tvl1: image too small for the pyramid")
    if trace:
        return u, v, its, en
    return u, v


def dual_tvl1(I0, I1, u1, u2, params: TVL1Params | None = None, error_mode: int = 0):
    """One level.  Returns (u1, u2, p[4,h,w], iterations[warps], energy[warps, max_it])."""
    p = params or TVL1Params()
    I0 = _f32(I0)
    I1 = _f32(I1)
    h, w = I0.shape
    u1 = _f32(u1).copy()
    u2 = _f32(u2).copy()
    pp = np.zeros((4, h, w), np.float32)
    its = np.zeros(p.warps, np.int32)
    en = np.full((p.warps, p.max_iterations), np.nan, np.float64)
    cp = p.c(error_mode)
    orc_lib().orc_dual_tvl1(I0, I1, u1, u2, w, h, C.byref(cp), pp.ctypes.data,
                            its.ctypes.data, en.ctypes.data)
    return u1, u2, pp, its, en


def nscales(w, h, n=5, zfactor=0.5):
    return orc_lib().orc_tvl1_nscales(w, h, n, zfactor)


def hs(I0, I1, alpha=15.0, nlevels=1, nwarp=1, nsolver=200):
    I0 = _f32(I0)
    I1 = _f32(I1)
    h, w = I0.shape
    u = np.zeros_like(I0)
    v = np.zeros_like(I0)
    if orc_lib().orc_hs(I0, I1, w, h, alpha, nlevels, nwarp, nsolver, u, v) != 0:
        raise ValueError("oracle hs: bad arguments")
    return u, v


def hs_downscale(src):
    """2x2 box to (h//2, w//2), every pixel (D-H1)."""
    src = _f32(src)
    h, w = src.shape
    out = np.zeros((h // 2, w // 2), np.float32)
    orc_lib().orc_hs_downscale(src, w, h, out)
    return out


def hs_warp(src, u, v):
    """Bilinear clamp-to-edge sample of src at (x+u, y+v) (D-H2)."""
    src = _f32(src)
    h, w = src.shape
    out = np.zeros_like(src)
    orc_lib().orc_hs_warp(src, _f32(u), _f32(v), w, h, out)
    return out


def hs_derivatives(I0, I1w):
    """(Ix, Iy, Iz) with clamped 5-tap stencils (D-H3)."""
    I0 = _f32(I0)
    h, w = I0.shape
    Ix, Iy, Iz = (np.zeros_like(I0) for _ in range(3))
    orc_lib().orc_hs_derivatives(I0, _f32(I1w), w, h, Ix, Iy, Iz)
    return Ix, Iy, Iz


def hs_jacobi(du0, dv0, Ix, Iy, Iz, alpha):
    """One Jacobi sweep; returns (du1, dv1)."""
    du0 = _f32(du0)
    h, w = du0.shape
    du1 = np.zeros_like(du0)
    dv1 = np.zeros_like(du0)
    orc_lib().orc_hs_jacobi(du0, _f32(dv0), _f32(Ix), _f32(Iy), _f32(Iz), w, h, alpha, du1, dv1)
    return du1, dv1


def upscale(src, nw, nh, scale):
    """Centre-aligned bilinear x2 upsample times `scale` (D-H4)."""
    src = _f32(src)
    h, w = src.shape
    out = np.zeros((nh, nw), np.float32)
    orc_lib().orc_upscale(src, w, h, nw, nh, scale, out)
    return out


def lk_filters(spac, temp):
    """(spatial taps, temporal taps) of the restatement."""
    fs = np.zeros(9, np.float32)
    ft = np.zeros(9, np.float32)
    if orc_lib().orc_lk_filters(spac, temp, fs, ft) != 0:
        raise ValueError("oracle lk_filters: size without a tap table")
    return fs[:spac], ft[:temp]


def lk_ring(frames, iframe, spac=3, temp=2, window=5):
    """Single-step LK over a ring of `temp` uint8 frames (slot k = frames[k])."""
    fr = [np.ascontiguousarray(f, dtype=np.uint8) for f in frames]
    h, w = fr[0].shape
    ptrs = (C.c_void_p * len(fr))(*[f.ctypes.data for f in fr])
    u = np.zeros((h, w), np.float32)
    v = np.zeros((h, w), np.float32)
    if orc_lib().orc_lk(ptrs, w, h, spac, temp, window, iframe, u, v) != 0:
        raise ValueError("oracle lk: bad arguments")
    return u, v


def lk(I0, I1, spac=3, window=5):
    I0 = _f32(I0)
    I1 = _f32(I1)
    h, w = I0.shape
    u = np.zeros_like(I0)
    v = np.zeros_like(I0)
    if orc_lib().orc_lk_f32(I0, I1, w, h, spac, window, u, v) != 0:
        raise ValueError("oracle lk: bad arguments")
    return u, v


def pyrlk(I0, I1, levels=3, iters=3, spac=3, window=5):
    I0 = _f32(I0)
    I1 = _f32(I1)
    h, w = I0.shape
    u = np.zeros_like(I0)
    v = np.zeros_like(I0)
    if orc_lib().orc_pyrlk(I0, I1, w, h, levels, iters, spac, window, u, v) != 0:
        raise ValueError("oracle pyrlk: bad arguments")
    return u, v


# ---------------------------------------------------------------- reference
def ref_tvl1(I0_u8, I1_u8, params: TVL1Params | None = None):
    """The reference's runDualTVL1Multiscale on uint8 frames (OpenMP threads per
    OMP_NUM_THREADS).  Returns (u, v)."""
    p = params or TVL1Params()
    a = np.ascontiguousarray(I0_u8, dtype=np.uint8)
    b = np.ascontiguousarray(I1_u8, dtype=np.uint8)
    h, w = a.shape
    u = np.zeros((h, w), np.float32)
    v = np.zeros((h, w), np.float32)
    lib = ref_lib()
    lib.ref_set_max_iterations(p.max_iterations)
    rc = lib.ref_tvl1_run(a, b, w, h, p.tau, p.lambda_, p.theta, p.nscales, p.zfactor,
                          p.warps, p.epsilon, u, v)
    if rc < 0:
        raise ValueError("reference tvl1: image too small for the pyramid")
    return u, v


def flow_to_color(u, v):
    """BGR bytes [h, w, 3] of a flow by orc_flow_to_color."""
    u = _f32(u)
    v = _f32(v)
    h, w = u.shape
    out = np.zeros((h, w, 3), np.uint8)
    orc_lib().orc_flow_to_color(u, v, w, h, out.ctypes.data_as(C.c_void_p))
    return out


# ------------------------------------------------- reference HS/LK CUDA kernels
def refg_available(stock: bool = False) -> bool:
    return os.path.exists(REFG_SO[stock])


def refg_lib(stock: bool = False):
    """The reference's HS/LK CUDA kernels behind ref_gpu_harness.cu.
    stock=False: built with -fmad=false; stock=True: the reference's flags."""
    if stock not in _refg:
        path = REFG_SO[stock]
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        lib.refg_device_count.restype = C.c_int
        lib.refg_hs_downscale.argtypes = [_f32p, C.c_int, C.c_int, _f32p]
        lib.refg_hs_jacobi.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_float,
                                       C.c_int, _f32p, _f32p]
        lib.refg_hs_add.argtypes = [_f32p, _f32p, C.c_int, _f32p]
        lib.refg_lk_filters.argtypes = [C.c_int, C.c_int, _f32p, _f32p, _f32p]
        for fn in (lib.refg_lk_class, lib.refg_lk_parts):
            fn.argtypes = [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                           _f32p, _f32p, _f32p, _f32p, _f32p]
        for fn in (lib.refg_hs_downscale, lib.refg_hs_jacobi, lib.refg_hs_add,
                   lib.refg_lk_filters, lib.refg_lk_class, lib.refg_lk_parts):
            fn.restype = C.c_int
        _refg[stock] = lib
    return _refg[stock]


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference {what}: status {rc}")


def refg_hs_downscale(src, stock=False):
    """DownscaleKernel output (h//2, w//2); the last row and column, which the
    kernel does not write, are NaN."""
    src = _f32(src)
    h, w = src.shape
    out = np.full((h // 2, w // 2), np.nan, np.float32)
    _check(refg_lib(stock).refg_hs_downscale(src, w, h, out), "Downscale")
    return out


def refg_hs_jacobi(Ix, Iy, Iz, alpha, nsweeps, stride=None, stock=False):
    """nsweeps JacobiIteration<32,6> sweeps from zero; returns (du, dv)."""
    Ix, Iy, Iz = _f32(Ix), _f32(Iy), _f32(Iz)
    h, w = Ix.shape
    du = np.zeros_like(Ix)
    dv = np.zeros_like(Ix)
    _check(refg_lib(stock).refg_hs_jacobi(Ix, Iy, Iz, w, h, stride or w, alpha, nsweeps, du, dv),
           "SolveForUpdate")
    return du, dv


def refg_hs_add(a, b, stock=False):
    a, b = _f32(a), _f32(b)
    out = np.zeros_like(a)
    _check(refg_lib(stock).refg_hs_add(a.ravel(), b.ravel(), a.size, out.ravel()), "Add")
    return out


def refg_lk_filters(spac, temp, stock=False):
    fx = np.zeros(9, np.float32)
    fy = np.zeros(9, np.float32)
    ft = np.zeros(9, np.float32)
    _check(refg_lib(stock).refg_lk_filters(spac, temp, fx, fy, ft), "getfilters")
    return fx[:spac], fy[:spac], ft[:temp]


def refg_lk(frames, iframe, spac=3, temp=2, window=5, whole_class=False, stock=False):
    """The reference LK on a ring of `temp` uint8 frames (slot k = frames[k]).
    whole_class=True runs LucasKanade::lucas_kanade (square frames only);
    otherwise the kernel wrappers with the y-filter taken through the x-filter
    on the transposed frame.  Returns (Vx, Vy, Ix, Iy, It)."""
    ring = np.ascontiguousarray(np.stack([np.asarray(f, np.uint8) for f in frames]))
    _, h, w = ring.shape
    outs = [np.zeros((h, w), np.float32) for _ in range(5)]
    fn = refg_lib(stock).refg_lk_class if whole_class else refg_lib(stock).refg_lk_parts
    _check(fn(ring.ravel(), w, h, spac, temp, window, iframe, *outs), "lucas_kanade")
    return tuple(outs)
