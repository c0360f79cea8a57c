"""The correctly rounded reciprocals of the FP32 reference-rounding stage
kernel, checked on the GPU against the IEEE quotient for every float input.

The kernel replaces two divisions of the reference's WENO weights
(GPUonly.cuh:111-118) by branch-free Newton-Raphson sequences: the double
reciprocal 1/(10 (beta+eps)^2) and the float reciprocal of the weights' sum.
Bit-identical results for all 2^32 float bit patterns are what keeps the
kernel bit-identical to the oracle whatever the state."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which,what", [(0, "double reciprocal of 10 x^2"), (1, "float reciprocal")])
def test_reciprocal_is_correctly_rounded_for_every_float(mpcf, which, what):
    bad = ctypes.c_ulonglong()
    first = (ctypes.c_uint * 8)()
    rc = mpcf.lib().mpcf_selftest_ieee(which, 0, ctypes.byref(bad), first)
    assert rc == 0, mpcf.lib().mpcf_last_error()
    assert bad.value == 0, (what, bad.value, [hex(v) for v in first[:min(8, bad.value)]])
