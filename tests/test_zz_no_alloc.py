"""oflow_hs_noalloc, the Horn-Schunck entry point for callers that cannot
allocate device memory (real-time loops, fixed memory budgets): called
through the C ABI on device buffers, twice in a row, it must give the same flow
as the regular oflow_hs entry point, allocate nothing between calls, and reject
frames beyond its static scratch.  Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(of, I0, I1, params, u, v, stream=0):
    L = of.capi.lib()
    h, w = I0.shape
    p = params.c()
    return L.oflow_hs_noalloc(C.c_void_p(I0.data_ptr()), C.c_void_p(I1.data_ptr()), w, h, 0,
                              C.byref(p), C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()), 0,
                              C.c_void_p(stream))


def test_noalloc_matches_hs_on_two_calls(of):
    import torch
    from oflow import synth
    cases = [(synth.hs_pair(seed=5), of.HSParams(15.0, 1, 1, 200)),
             (synth.hs_pair(seed=6, w=160, h=120), of.HSParams(0.2, 3, 2, 30))]
    free_after_first = None
    for k, (q, prm) in enumerate(cases):
        I0 = torch.from_numpy(q.I0).cuda()
        I1 = torch.from_numpy(q.I1).cuda()
        u = torch.full_like(I0, float("nan"))
        v = torch.full_like(I0, float("nan"))
        torch.cuda.synchronize()
        if k == 1:
            free_before = torch.cuda.mem_get_info()[0]
        assert _call(of, I0, I1, prm, u, v, torch.cuda.current_stream().cuda_stream) == 0
        torch.cuda.synchronize()
        if k == 1:
            assert torch.cuda.mem_get_info()[0] == free_before  # nothing allocated
        ru, rv = of.hs(q.I0, q.I1, prm)
        tol = 0.0  # the HS parity tests require identical results
        assert np.abs(u.cpu().numpy() - ru).max() <= tol
        assert np.abs(v.cpu().numpy() - rv).max() <= tol


def test_noalloc_rejects_frames_beyond_capacity(of):
    import torch
    big = torch.zeros((1080, 1920), dtype=torch.float32, device="cuda")
    u = torch.empty_like(big)
    v = torch.empty_like(big)
    assert _call(of, big, big, of.HSParams(15.0, 1, 1, 10), u, v) == 1
