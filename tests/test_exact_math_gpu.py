"""The hardware-estimate refinements behind the TV-L1 kernels' exact fast
forms, checked on the device (the host cannot reproduce the estimate
instructions): every positive normal float for the square root, every float
of the reciprocal's range, and 2^28 seeded operand pairs each for the hypot
and the Markstein quotient.  Any mismatch would change the flow's bits."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _count(of, which, lo, hi, seed=0):
    n = C.c_ulonglong(0)
    assert of.capi.lib().oflow_selftest_math(which, lo, hi, seed, C.byref(n)) == 0
    return n.value


def _bits(f):
    import struct
    return struct.unpack("<I", struct.pack("<f", f))[0]


def test_sqrt_near_within_one_ulp_for_every_normal_float(of):
    assert _count(of, 0, 0x00800000, 0x7F800000) == 0


def test_refined_reciprocal_correctly_rounded_over_its_range(of):
    assert _count(of, 1, _bits(2.0 ** -40), _bits(2.0 ** 24)) == 0


@pytest.mark.parametrize("seed", [1, 2])
def test_fast_hypot_equals_double_formula(of, seed):
    assert _count(of, 2, 0, 1 << 28, seed) == 0


@pytest.mark.parametrize("seed", [3, 4])
def test_markstein_from_refined_reciprocal_equals_ieee_division(of, seed):
    assert _count(of, 3, 0, 1 << 28, seed) == 0
