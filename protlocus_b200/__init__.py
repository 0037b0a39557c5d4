"""protlocus_b200 -- B200-native (sm_100a) alignment hot path of ProtLocus.

The product is the C-ABI shared library ``protlocus_b200/libplgpu.so`` built
from ``protlocus_b200/csrc``; this package is the Python host mirror of its
interface (ctypes) plus the synthetic workload generators used by the
benchmark.
"""
from .abi import Options, NsOpt, NsRst  # noqa: F401
