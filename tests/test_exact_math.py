"""The exact fast forms of csrc/exact_math.cuh, compiled for the host, against
the plain expressions they replace: hypot_fast / hypot2_fast against glibc's
hypotf formula (float)sqrt((double)a^2 + (double)b^2), and the Markstein
division against IEEE p / g.  Random operands over the whole exponent range,
the tiny range where low-order product terms would be subnormal, and
Pythagorean triples whose hypotenuse is exactly a float rounding midpoint
(where double-then-single rounding and single rounding part ways)."""
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
    long bad_h = 0, bad_h2 = 0, bad_d = 0, mids = 0, cases = 0;
    auto rnd = [&](int emin, int emax) {
        const int e = emin + (int)(rng() % (uint64_t)(emax - emin + 1));
        const float m = (float)unit(rng);
        const float v = ldexpf(m, e);
        return (rng() & 1) ? -v : v;
    };
    auto check_h = [&](float a, float b) {
        cases++;
        if (!same(hypot_fast(a, b), hypot_ref(a, b))) bad_h++;
    };
    auto check_h2 = [&](float a1, float b1, float a2, float b2) {
        float h1, h2;
        hypot2_fast(a1, b1, a2, b2, h1, h2);
        if (!same(h1, hypot_ref(a1, b1)) || !same(h2, hypot_ref(a2, b2))) bad_h2++;
    };
    for (long i = 0; i < n; i++) {
        const float a = rnd(-140, 70), b = rnd(-140, 70);
        check_h(a, b);
        const float c = rnd(-30, 10), d = c * (float)unit(rng);  // similar magnitudes
        check_h(c, d);
        const float t = rnd(-62, -44), s = rnd(-75, -44);  // low terms near subnormal
        check_h(t, s);
        check_h2(a, b, t, s);
        check_h2(c, d, 0.0f, t);
    }
    const float sp[] = {0.0f, -0.0f, 1.0f, 3.0f, 4.0f, 1e-45f, 1e-38f, 3e38f, INFINITY, -INFINITY, NAN};
    for (float a : sp)
        for (float b : sp) {
            check_h(a, b);
            check_h2(a, b, b, a);
        }
    // primitive triples m^2-n^2, 2mn, m^2+n^2 with an odd 25-bit hypotenuse:
    // sqrt(a^2+b^2) lies exactly halfway between two floats
    for (long i = 0; i < n; i++) {
        const uint64_t m = 2900 + rng() % 2900, k = 1 + rng() % (m - 1);
        if (((m ^ k) & 1) == 0) continue;
        const uint64_t c = m * m + k * k, a = m * m - k * k, b = 2 * m * k;
        if (c < (1u << 24) || c >= (1u << 25) || a >= (1u << 24)) continue;
        const int sc = (int)(rng() % 40) - 20;
        const float fa = ldexpf((float)a, sc), fb = ldexpf((float)b, sc);
        mids++;
        check_h(fa, fb);
        check_h(fb, -fa);
        check_h(nextafterf(fa, 0.0f), fb);
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
    printf("%ld %ld %ld %ld %ld\n", bad_h, bad_h2, bad_d, mids, cases);
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
    bad_h, bad_h2, bad_d, mids, cases = map(int, out.stdout.split())
    assert mids > 1000 and cases > 1_000_000
    assert (bad_h, bad_h2, bad_d) == (0, 0, 0)
