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


RECORDS = [("GaplessCandidate", "ns_gpu_gapless_candidate_t"), ("GaplessAnchor", "ns_gpu_gapless_anchor_t"),
           ("SpliceJob", "pl_splice_job_t"), ("SpliceResult", "pl_splice_result_t"), ("ExtJob", "pl_ext_job_t"),
           ("ExtResult", "pl_ext_result_t"), ("ExtraJob", "pl_extra_job_t"), ("Feat", "pl_feat_t"),
           ("ExtraResult", "pl_extra_result_t"), ("PsJob", "pl_ps_job_t"), ("ChainOpt", "pl_chain_opt_t")]


def test_every_record_field_offset_matches_c(tmp_path):
    """sizeof and the offset of every field of each public record, as gcc lays them out
    from include/plgpu.h, equal the ctypes mirrors the Python layer passes."""
    from protlocus_b200 import abi
    lines, want = [], []
    for py, c in RECORDS:
        cls = getattr(abi, py)
        lines.append(f'printf("%zu\\n", sizeof({c}));')
        want.append(C.sizeof(cls))
        for name, _ in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({c}, {name}));')
            want.append(getattr(cls, name).offset)
    src = tmp_path / "off.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "plgpu.h"\nint main(void){\n' +
                   "\n".join(lines) + "\nreturn 0;}\n")
    exe = tmp_path / "off"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert out == want


def test_no_device_is_an_error_not_a_fallback():
    """Without a GPU the entry points refuse: ns_gpu_init() returns 0 with a message."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = L.load()
    assert lib.ns_gpu_init(0) == 0
    assert lib.ns_gpu_error().decode() != "none"
    assert lib.ns_gpu_submit(None, b"ATG", 3, b"M", 1, None, None) is None


def test_fault_hook_and_span_checks_without_a_device():
    """The fault-injection hook validates its site; with no device the extension batch object is
    refused (NULL) rather than run on the CPU."""
    lib = L.load()
    assert lib.pl_debug_fault(3, 0) == 0 and lib.pl_debug_fault(-1, 0) == 0
    for site in (0, 1, 2):
        assert lib.pl_debug_fault(site, -1) == 1
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        assert not lib.ns_ext_batch_init(None)


def test_band_cells_closed_form_matches_the_row_sum():
    """pl_ps_band_cells (the prescreen's cell count, summed in closed form) equals the sum of
    the clipped band widths row by row, over bands, diagonals far left / right of the ORF and
    tiny matrices."""
    import numpy as np
    lib = L.load()
    rng = np.random.default_rng(5)
    cases = [(1, 1, 0, 1), (5, 3, -10, 2), (5, 3, 10, 2), (0, 7, 0, 3), (7, 0, 0, 3), (9, 4, 2, 0), (9, 4, 2, -1)]
    cases += [(int(rng.integers(0, 300)), int(rng.integers(0, 500)), int(rng.integers(-400, 600)),
               int(rng.choice([1, 2, 8, 32, 64, 0, -3, 700]))) for _ in range(3000)]
    for L_, n, d, b in cases:
        want = 0
        for i in range(L_):
            lo, hi = (i + d - b, i + d + b) if b > 0 else (0, n - 1)
            lo, hi = max(lo, 0), min(hi, n - 1)
            want += max(0, hi - lo + 1)
        assert lib.pl_ps_band_cells(L_, n, d, b) == want, (L_, n, d, b)
