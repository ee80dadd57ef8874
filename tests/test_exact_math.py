"""The exact fast forms of csrc/exact_math.cuh, compiled for the host, against
the functions they stand for: hypot_ref ((float)sqrt((double)a^2 +
(double)b^2)) against this host's hypotf, which the reference's std::hypot
calls, on random operands and on Pythagorean triples whose hypotenuse is
exactly a float rounding midpoint; and the Markstein division against IEEE
p / g on random operands over the whole exponent range, signed zeros and the
TH step's range of g."""
import os
import shutil
import subprocess

import pytest

from conftest import PKG

PROGRAM = r'''
#include "exact_math.cuh"
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
using namespace oflow;

static uint32_t bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static bool same(float a, float b) { return bits(a) == bits(b) || (a != a && b != b); }

int main(int argc, char **argv) {
    const long n = atol(argv[1]);
    std::mt19937_64 rng(20240611);
    std::uniform_real_distribution<double> unit(1.0, 2.0);
    long bad_h = 0, bad_d = 0, mids = 0, cases = 0;
    auto rnd = [&](int emin, int emax) {
        const int e = emin + (int)(rng() % (uint64_t)(emax - emin + 1));
        const float m = (float)unit(rng);
        const float v = ldexpf(m, e);
        return (rng() & 1) ? -v : v;
    };
    for (long i = 0; i < n; i++) {
        const float a = rnd(-140, 70), b = rnd(-140, 70);
        cases++;
        if (!same(hypot_ref(a, b), hypotf(a, b))) bad_h++;
    }
    // primitive triples m^2-n^2, 2mn, m^2+n^2 with an odd 25-bit hypotenuse:
    // sqrt(a^2+b^2) lies exactly halfway between two floats, where double then
    // single rounding and single rounding part ways
    for (long i = 0; i < n; i++) {
        const uint64_t m = 2900 + rng() % 2900, k = 1 + rng() % (m - 1);
        if (((m ^ k) & 1) == 0) continue;
        const uint64_t c = m * m + k * k, a = m * m - k * k, b = 2 * m * k;
        if (c < (1u << 24) || c >= (1u << 25) || a >= (1u << 24)) continue;
        const int sc = (int)(rng() % 40) - 20;
        const float fa = ldexpf((float)a, sc), fb = ldexpf((float)b, sc);
        mids++;
        for (float x : {fa, nextafterf(fa, 0.0f)}) {
            cases++;
            if (!same(hypot_ref(x, fb), hypotf(x, fb))) bad_h++;
        }
    }
    // Markstein division for the dual update's g >= 1, p of any size and sign
    for (long i = 0; i < n; i++) {
        const float g = 1.0f + ldexpf((float)unit(rng), (int)(rng() % 20) - 10);
        float p = rnd(-140, 20);
        if (i % 97 == 0) p = 0.0f;
        if (i % 89 == 0) p = -0.0f;
        const float y = 1.0f / g;
        if (!same(div_by_rcp(p, g, y), p / g)) bad_d++;
        if (markstein_safe(p) && !same(markstein(p, g, y), p / g)) bad_d++;
    }
    // the TH step's quotient -rho/grad: g over the whole refined-reciprocal range
    for (long i = 0; i < n; i++) {
        const float g = ldexpf((float)unit(rng), (int)(rng() % 64) - 40);
        const float p = rnd(-99, 30);
        const float y = 1.0f / g;
        if (rcp_in_range(g) && markstein_safe(p) && !same(markstein(p, g, y), p / g)) bad_d++;
    }
    printf("%ld %ld %ld %ld\n", bad_h, bad_d, mids, cases);
    return 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_exact_fast_forms_equal_plain_expressions(tmp_path):
    src = tmp_path / "exact.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "exact"
    cuda_inc = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/include"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math",
                           "-I", os.path.join(PKG, "csrc"), "-I", cuda_inc, str(src), "-o",
                           str(exe), "-lm"])
    out = subprocess.run([str(exe), "300000"], capture_output=True, text=True, check=True)
    bad_h, bad_d, mids, cases = map(int, out.stdout.split())
    assert mids > 1000 and cases > 300_000
    assert (bad_h, bad_d) == (0, 0)
