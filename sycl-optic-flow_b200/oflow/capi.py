"""ctypes declarations of include/oflow.h and the loader of liboflow.so.

The library is built in-tree (``make -C sycl-optic-flow_b200``) and loaded
from there; there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("OFLOW_LIB", os.path.join(os.path.dirname(HERE), "liboflow.so"))

MAX_SCALES = 16
MAX_WARPS = 32


class OflowError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class Image(C.Structure):
    _fields_ = [("data", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("pitch", C.c_int), ("dtype", C.c_int), ("location", C.c_int)]


class Flow(C.Structure):
    _fields_ = [("u", C.POINTER(C.c_float)), ("v", C.POINTER(C.c_float)),
                ("pitch", C.c_int), ("location", C.c_int)]


class BgrImage(C.Structure):
    _fields_ = [("data", C.c_void_p), ("pitch", C.c_int), ("location", C.c_int)]


class Tvl1Params(C.Structure):
    _fields_ = [("tau", C.c_float), ("lambda_", C.c_float), ("theta", C.c_float),
                ("nscales", C.c_int), ("zfactor", C.c_float), ("warps", C.c_int),
                ("epsilon", C.c_float), ("max_iterations", C.c_int)]


class Tvl1Stats(C.Structure):
    _fields_ = [("nscales", C.c_int), ("warps", C.c_int),
                ("iterations", C.c_int * (MAX_SCALES * MAX_WARPS)), ("energy", C.c_double)]


class Tvl1Profile(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("iter_ms", C.c_double), ("warp_ms", C.c_double),
                ("iter_launches", C.c_int), ("warp_launches", C.c_int), ("launches", C.c_int),
                ("iter_ms_scale", C.c_double * MAX_SCALES)]


class HsParams(C.Structure):
    _fields_ = [("alpha", C.c_float), ("nlevels", C.c_int), ("nwarp", C.c_int),
                ("nsolver", C.c_int)]


class StreamDesc(C.Structure):
    _fields_ = [("solver", C.c_int), ("width", C.c_int), ("height", C.c_int), ("dtype", C.c_int),
                ("lanes", C.c_int), ("tvl1", Tvl1Params), ("hs", HsParams)]


class LkParams(C.Structure):
    _fields_ = [("spac", C.c_int), ("temp", C.c_int), ("window", C.c_int), ("levels", C.c_int),
                ("iters", C.c_int)]


class Job(C.Structure):
    _fields_ = [("solver", C.c_int), ("I0", Image), ("I1", Image),
                ("tvl1", C.POINTER(Tvl1Params)), ("hs", C.POINTER(HsParams)), ("out", Flow)]


SOLVER_TVL1, SOLVER_HS = 0, 1

# every entry point of include/oflow.h: name -> (restype, argtypes)
_VP, _I = C.c_void_p, C.c_int
SIGNATURES = {
    "oflow_abi_version": (_I, []),
    "oflow_status_string": (C.c_char_p, [_I]),
    "oflow_ctx_create": (_I, [_I, C.POINTER(C.c_void_p)]),
    "oflow_ctx_destroy": (_I, [_VP]),
    "oflow_ctx_set_stream": (_I, [_VP, _VP]),
    "oflow_ctx_trim": (_I, [_VP]),
    "oflow_ctx_last_error": (C.c_char_p, [_VP]),
    "oflow_tvl1_default_params": (None, [C.POINTER(Tvl1Params)]),
    "oflow_tvl1_nscales": (_I, [_I, _I, C.POINTER(Tvl1Params)]),
    "oflow_tvl1": (_I, [_VP, C.POINTER(Image), C.POINTER(Image), C.POINTER(Tvl1Params),
                        C.POINTER(Flow), C.POINTER(Tvl1Stats)]),
    "oflow_tvl1_batch": (_I, [_VP, _I, C.POINTER(Image), C.POINTER(Image),
                              C.POINTER(Tvl1Params), C.POINTER(Flow), C.POINTER(Tvl1Stats)]),
    "oflow_tvl1_energy_trace": (_I, [_VP, C.POINTER(Image), C.POINTER(Image),
                                     C.POINTER(Tvl1Params), C.POINTER(Flow),
                                     C.POINTER(Tvl1Stats), C.POINTER(C.c_double)]),
    "oflow_tvl1_batch_profile": (_I, [_VP, _I, C.POINTER(Image), C.POINTER(Image),
                                      C.POINTER(Tvl1Params), C.POINTER(Flow),
                                      C.POINTER(Tvl1Stats), C.POINTER(Tvl1Profile)]),
    "oflow_tvl1_autotune": (_I, [_VP, _I, C.POINTER(Image), C.POINTER(Image),
                                 C.POINTER(Tvl1Params), C.POINTER(C.c_int)]),
    "oflow_ctx_save_tuning": (_I, [_VP, C.c_char_p]),
    "oflow_ctx_load_tuning": (_I, [_VP, C.c_char_p]),
    "oflow_hs_default_params": (None, [C.POINTER(HsParams)]),
    "oflow_hs": (_I, [_VP, C.POINTER(Image), C.POINTER(Image), C.POINTER(HsParams),
                      C.POINTER(Flow)]),
    "oflow_hs_batch": (_I, [_VP, _I, C.POINTER(Image), C.POINTER(Image), C.POINTER(HsParams),
                            C.POINTER(Flow)]),
    "oflow_hs_autotune": (_I, [_VP, _I, C.POINTER(Image), C.POINTER(Image),
                               C.POINTER(HsParams), C.POINTER(C.c_int)]),
    "oflow_hs_noalloc": (_I, [_VP, _VP, _I, _I, _I, C.POINTER(HsParams), _VP, _VP, _I, _VP]),
    "oflow_batch": (_I, [_VP, _I, C.POINTER(Job)]),
    "oflow_net_num_params": (_I, []),
    "oflow_net_create": (_I, [_VP, _I, _I, _I, C.POINTER(C.c_void_p)]),
    "oflow_net_destroy": (_I, [_VP]),
    "oflow_net_out_size": (_I, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "oflow_net_set_params": (_I, [_VP, _VP]),
    "oflow_net_get_params": (_I, [_VP, _VP]),
    "oflow_net_train_step": (_I, [_VP, _VP, _I, _VP, C.c_float, C.POINTER(C.c_double)]),
    "oflow_net_predict": (_I, [_VP, _VP, _I, _VP]),
    "oflow_tvl1_warm": (_I, [_VP, _VP, _I, C.POINTER(Image), C.POINTER(Image),
                             C.POINTER(Tvl1Params), _VP, _VP, C.POINTER(Tvl1Params),
                             C.POINTER(Flow), _VP, _VP, _VP, _VP, C.POINTER(Tvl1Stats)]),
    "oflow_stream_create": (_I, [_VP, C.POINTER(StreamDesc), C.POINTER(_VP)]),
    "oflow_stream_destroy": (_I, [_VP]),
    "oflow_stream_push": (_I, [_VP, C.POINTER(Image), C.POINTER(Flow), C.POINTER(Tvl1Stats)]),
    "oflow_stream_frames": (C.c_longlong, [_VP]),
    "oflow_ctx_last_launches": (_I, [_VP, C.POINTER(C.c_longlong)]),
    "oflow_selftest_math": (_I, [_I, C.c_uint32, C.c_uint32, C.c_ulonglong,
                                 C.POINTER(C.c_ulonglong)]),
    "oflow_flow_to_color": (_I, [_VP, _I, _I, _I, C.POINTER(Flow), C.POINTER(BgrImage)]),
    "oflow_conv3x3": (_I, [_I, _I, _I, _I, _I, _I, _I, _I, _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "oflow_lk_default_params": (None, [C.POINTER(LkParams)]),
    "oflow_lk": (_I, [_VP, C.POINTER(Image), _I, C.POINTER(LkParams), C.POINTER(Flow)]),
    "oflow_pyrlk": (_I, [_VP, C.POINTER(Image), C.POINTER(Image), C.POINTER(LkParams),
                         C.POINTER(Flow)]),
    "oflow_pyrlk_batch": (_I, [_VP, _I, C.POINTER(Image), C.POINTER(Image),
                               C.POINTER(LkParams), C.POINTER(Flow)]),
}

_lib = None


def lib():
    """Load liboflow.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"liboflow.so not built (expected at {LIB_PATH}); "
                          "run `make -C sycl-optic-flow_b200`")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def status_string(s: int) -> str:
    return lib().oflow_status_string(s).decode()
