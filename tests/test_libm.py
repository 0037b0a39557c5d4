"""The restated glibc expf / log1pf of the device Forward (protlocus_b200/csrc/
glibc_mathf.cuh), built for the host, against the host's own libm: every result
bit-equal.  rc_logsum (recheck.c:260-265) calls log1pf(expf(mn - mx)) with
mn - mx in [-50, 0], so expf is swept densely over [-50, 0] and log1pf over
[0, 1]; both are also swept sparsely over every float (infinities, NaN,
overflow, underflow, subnormals).  Exhaustive runs over all 4.28e9 floats gave
0 mismatches for both; the device build is checked over the full Forward range
in tests/test_gpu_forward.py.  The branch-free forms rc_logsum uses on the device
(gl_expf_rng, gl_log1pf_unit) equal the host libm on every float of [-50, 50] and
[0, 1] (exhaustive runs, 0 mismatches); the sweeps below repeat that densely.
"""
import ctypes as C
import os
import struct

import pytest

LIB = os.path.join(os.path.dirname(__file__), "..", "oracle", "_build", "liblmcheck.so")

pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="oracle/_build/liblmcheck.so not built")


def _lib():
    lib = C.CDLL(LIB)
    lib.lm_mismatch.restype = C.c_int64
    lib.lm_mismatch.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32)]
    return lib


def _bits(f):
    return struct.unpack("<I", struct.pack("<f", f))[0]


@pytest.mark.parametrize("fn,lo,hi,stride", [
    (0, 0x80000000, _bits(-50.0) + 1, 7),   # expf over the Forward's [-50, -0]
    (1, 0x00000000, _bits(1.0) + 1, 7),     # log1pf over [0, 1]
    (0, 0x00000000, 0xffffffff, 4099),      # every float range, sparsely
    (1, 0x00000000, 0xffffffff, 4099),
    (0, _bits(-0.4), _bits(-0.5) + 1, 1),   # a dense window of each, every pattern
    (1, _bits(0.40), _bits(0.45) + 1, 1),   # around log1pf's 0.41422 branch
    (2, 0x80000000, _bits(-50.0) + 1, 7),   # the branch-free forms on rc_logsum's ranges
    (3, 0x00000000, _bits(1.0) + 1, 7),
    (3, _bits(0.40), _bits(0.45) + 1, 1),
    (3, _bits(0.99), _bits(1.0) + 1, 1),    # |f| < 2^-20 near 1 + x = 2
])
def test_restated_libm_equals_host(fn, lo, hi, stride):
    bad = C.c_uint32()
    n = _lib().lm_mismatch(fn, lo, hi, stride, C.byref(bad))
    assert n == 0, f"{n} mismatches, first at bit pattern {bad.value:#010x}"
