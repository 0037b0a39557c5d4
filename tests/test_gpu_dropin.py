"""The reference's own GPU test program (test/test_gpu.c), linked against this
library in place of the reference's GPU objects, passes on the device.

oracle/Makefile's `dropin` target builds oracle/_ref/test_gpu_dropin from the
reference sources where they lie (nasw-sse.c, nasw-tab.c, kalloc.c, kthread.c,
hmm.c, test/test_gpu.c) and links libplgpu.so for ns_gpu_*, ns_ext_batch_* and
mp_hmm_dp_score_gpu*.  Its asserts cover the global DP's tile boundaries, the
32-bit route, 32 concurrent threads, 129 asynchronous requests, the HMM DP and
a 42-request extension sweep, each compared with the reference CPU code.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_gpu_dropin")


@pytest.mark.skipif(not os.path.exists(BIN), reason="oracle/_ref/test_gpu_dropin not built (needs the reference tree)")
def test_reference_gpu_test_program():
    env = dict(os.environ, NS_GPU_TEST_REQUIRED="1")
    p = subprocess.run([BIN], capture_output=True, text=True, timeout=600, env=env)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    assert "[SKIP]" not in p.stderr and "FAIL" not in p.stderr, p.stderr[-2000:]
