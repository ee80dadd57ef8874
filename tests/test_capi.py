"""The C-ABI library: loads, exports every entry point of include/oflow.h, and
rejects bad arguments with status codes.  No compute calls (CPU only)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(oflow_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol(of):
    lib = C.CDLL(of.LIB_PATH)
    names = header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(of):
    assert set(header_functions()) <= set(of.capi.SIGNATURES)


def test_abi_version_and_status_strings(of):
    L = of.capi.lib()
    assert L.oflow_abi_version() == 1
    for s, txt in [(0, "ok"), (1, "bad argument"), (4, "no CUDA device"), (5, "out of memory")]:
        assert L.oflow_status_string(s).decode() == txt


def test_default_params_match_reference(of):
    L = of.capi.lib()
    p = of.capi.Tvl1Params()
    L.oflow_tvl1_default_params(C.byref(p))
    # src/tvl1/sequential/tvl1.hpp:6,12-14
    assert (round(p.tau, 6), round(p.lambda_, 6), round(p.theta, 6)) == (0.25, 0.15, 0.3)
    assert (p.nscales, p.zfactor, p.warps, p.max_iterations) == (100, 0.5, 5, 300)
    assert abs(p.epsilon - 0.01) < 1e-9
    h = of.capi.HsParams()
    L.oflow_hs_default_params(C.byref(h))
    assert (h.nlevels, h.nwarp, h.nsolver) == (5, 3, 150)
    k = of.capi.LkParams()
    L.oflow_lk_default_params(C.byref(k))
    assert (k.spac, k.temp, k.window) == (3, 2, 5)


def test_nscales_rule(of):
    assert of.nscales(1024, 436) == 7
    assert of.nscales(1024, 436, of.TVL1Params(nscales=5)) == 5
    L = of.capi.lib()
    p = of.capi.Tvl1Params()
    L.oflow_tvl1_default_params(C.byref(p))
    p.zfactor = 1.5
    assert L.oflow_tvl1_nscales(64, 64, C.byref(p)) == -1


def test_bad_arguments_return_status(of):
    L = of.capi.lib()
    assert L.oflow_ctx_create(0, None) == 1
    assert L.oflow_ctx_destroy(None) == 1
    assert L.oflow_ctx_set_stream(None, None) == 1
    p = of.capi.Tvl1Params()
    L.oflow_tvl1_default_params(C.byref(p))
    img = of.capi.Image()
    fl = of.capi.Flow()
    assert L.oflow_tvl1(None, C.byref(img), C.byref(img), C.byref(p), C.byref(fl), None) == 1
    assert L.oflow_tvl1_batch(None, 0, None, None, C.byref(p), None, None) == 1


def test_context_without_device_reports_no_device(of):
    try:
        import torch
        have = torch.cuda.is_available()
    except Exception:
        have = False
    L = of.capi.lib()
    h = C.c_void_p()
    rc = L.oflow_ctx_create(0, C.byref(h))
    if have:
        assert rc == 0
        assert L.oflow_ctx_destroy(h) == 0
    else:
        assert rc == 4 and not h.value


def test_solver_without_library_path_fails_loudly(tmp_path):
    """No fallback: a missing library is an error, not a CPU path."""
    import subprocess
    import sys
    code = ("import sys; sys.path[:0]=[%r,%r]; import os; os.environ['OFLOW_LIB']='%s';"
            "import oflow, numpy as np\n"
            "try:\n    oflow.tvl1(np.zeros((16,16),np.uint8), np.zeros((16,16),np.uint8))\n"
            "except OSError as e:\n    print('raised', e)\n") % (
        ROOT, os.path.join(ROOT, "sycl-optic-flow_b200"), tmp_path / "missing.so")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         env={**os.environ, "OFLOW_LIB": str(tmp_path / "missing.so")})
    assert "raised" in out.stdout, out.stderr
