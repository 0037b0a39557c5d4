"""The C-ABI library loads and exports every symbol include/plgpu.h declares (CPU only;
no compute calls)."""
import ctypes as C
import os
import subprocess

import pytest

from protlocus_b200 import lib as L
from protlocus_b200.abi import NsOpt, NsRst, SpliceJob, SpliceResult

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_declared_symbols():
    lib = L.load()
    names = L.declared_symbols()
    assert "ns_gpu_submit" in names and "pl_splice_batch_device" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "plgpu.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(ns_opt_t), sizeof(ns_rst_t),'
                   ' sizeof(pl_splice_job_t), sizeof(pl_splice_result_t), offsetof(ns_opt_t, sc),'
                   ' offsetof(ns_opt_t, codon)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    want = [C.sizeof(NsOpt), C.sizeof(NsRst), C.sizeof(SpliceJob), C.sizeof(SpliceResult),
            NsOpt.sc.offset, NsOpt.codon.offset]
    assert [int(x) for x in out] == want


def test_no_device_is_an_error_not_a_fallback():
    """Without a GPU the entry points refuse: ns_gpu_init() returns 0 with a message."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = L.load()
    assert lib.ns_gpu_init(0) == 0
    assert lib.ns_gpu_error().decode() != "none"
    assert lib.ns_gpu_submit(None, b"ATG", 3, b"M", 1, None, None) is None
