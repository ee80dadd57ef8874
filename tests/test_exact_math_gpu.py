"""The hardware-estimate refinement behind the TV-L1 kernels' exact fast
division, checked on the device (the host cannot reproduce the estimate
instruction): every float of the refined reciprocal's range, and 2^28
seeded operand pairs twice for the Markstein quotient built on it.  Any
mismatch would change the flow's bits."""
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


def test_refined_reciprocal_correctly_rounded_over_its_range(of):
    assert _count(of, 1, _bits(2.0 ** -40), _bits(2.0 ** 24)) == 0


@pytest.mark.parametrize("seed", [3, 4])
def test_markstein_from_refined_reciprocal_equals_ieee_division(of, seed):
    assert _count(of, 3, 0, 1 << 28, seed) == 0
