"""The C++ drop-in shims (include/oflow_compat.hpp): a program written against
the reference's class and function names compiles and links against
liboflow.so; on a GPU it produces the same flow as the C ABI."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

PROGRAM = r'''
#include "oflow_compat.hpp"
#include <cstdio>
#include <cstdlib>
#include <vector>
int main(int argc, char **argv) {
    const int w = 96, h = 64;
    std::vector<uint8_t> I0(w * h), I1(w * h);
    FILE *f = fopen(argv[1], "rb");
    if (!f || fread(I0.data(), 1, w * h, f) != (size_t)(w * h) ||
        fread(I1.data(), 1, w * h, f) != (size_t)(w * h)) return 3;
    fclose(f);
    try {
        TV_L1 t(w, h, 0.25, 0.15, 0.3, 3, 0.5, 5, 0.01, 10);
        t.runDualTVL1Multiscale(I0.data(), I1.data());
        FILE *o = fopen(argv[2], "wb");
        fwrite(t.getU(), sizeof(float), 2 * w * h, o);
        fclose(o);
        std::vector<float> a(w * h), b(w * h), u(w * h), v(w * h);
        for (int i = 0; i < w * h; i++) { a[i] = I0[i]; b[i] = I1[i]; }
        initFlow(1, w, w, h);
        ComputeFlow(a.data(), b.data(), w, h, w, 15.0f, 1, 1, 40, u.data(), v.data());
        deleteFlow_mem(1);
        LucasKanade lk(3, 2, 5, w, h);
        lk.copy_frames_circularbuffer_GPU_wrapper(I0.data(), 2, 0, w * h);
        lk.copy_frames_circularbuffer_GPU_wrapper(I1.data(), 2, 1, w * h);
        lk.lucas_kanade(u.data(), v.data(), 1);
        o = fopen(argv[3], "wb");
        fwrite(u.data(), sizeof(float), w * h, o);
        fclose(o);
        // streaming form: the second frame pairs with the first (tvl1.cu:122-130)
        TV_L1 s(w, h, 0.25, 0.15, 0.3, 3, 0.5, 5, 0.01, 10);
        s.runDualTVL1Multiscale(a.data());
        s.runDualTVL1Multiscale(b.data());
        std::vector<unsigned char> bgr(3 * w * h);
        flowToColor(w, h, s.getU(), bgr.data());
        o = fopen(argv[4], "wb");
        fwrite(s.getU(), sizeof(float), 2 * w * h, o);
        fwrite(bgr.data(), 1, 3 * w * h, o);
        fclose(o);
    } catch (const oflow::compat_error &e) {
        printf("compat_error %d %s\n", (int)e.status, e.what());
        return 2;
    }
    return 0;
}
'''


def _build(tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    src = tmp_path / "prog.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "prog"
    subprocess.check_call([cxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src),
                           "-L", PKG, "-loflow", "-Wl,-rpath," + PKG, "-o", str(exe)])
    return exe


def test_compat_program_compiles_and_reports_errors_without_device(tmp_path, of):
    exe = _build(tmp_path)
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("device present: covered by the GPU test")
    except Exception:
        pass
    (tmp_path / "in.bin").write_bytes(bytes(96 * 64 * 2))
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "u.bin"),
                        str(tmp_path / "l.bin"), str(tmp_path / "s.bin")], capture_output=True,
                       text=True)
    assert r.returncode == 2 and "compat_error 4" in r.stdout


@pytest.mark.gpu
def test_compat_program_matches_c_abi(tmp_path, of):
    from oflow import synth
    exe = _build(tmp_path)
    p = synth.tvl1_pair(seed=77, w=96, h=64, radius=12.0)
    a, b = synth.quantize(p.I0), synth.quantize(p.I1)
    (tmp_path / "in.bin").write_bytes(a.tobytes() + b.tobytes())
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "u.bin"),
                        str(tmp_path / "l.bin"), str(tmp_path / "s.bin")], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    U = np.fromfile(tmp_path / "u.bin", np.float32)
    u, v = of.tvl1(a, b, of.TVL1Params(nscales=3, max_iterations=10))
    assert np.array_equal(U, np.concatenate([u.ravel(), v.ravel()]))
    L = np.fromfile(tmp_path / "l.bin", np.float32).reshape(64, 96)
    lu, _ = of.lk([a, b], 1, of.LKParams(3, 2, 5))
    assert np.array_equal(L, lu)
    S = np.fromfile(tmp_path / "s.bin", np.uint8)
    su = S[: 2 * 96 * 64 * 4].view(np.float32)
    fu, fv = of.tvl1(a.astype(np.float32), b.astype(np.float32),
                     of.TVL1Params(nscales=3, max_iterations=10))
    assert np.array_equal(su, np.concatenate([fu.ravel(), fv.ravel()]))
    img = S[2 * 96 * 64 * 4:].reshape(64, 96, 3)
    assert np.array_equal(img, of.flow_to_color(fu, fv))
