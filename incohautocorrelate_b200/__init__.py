"""B200-native pair-correlation path of IncohAutoCorrelate.

The product is libiac_b200.so (hand-written sm_100a CUDA kernels behind the C
ABI in include/iac_b200.h) and the C++ drop-in classes under cpp/.  This Python
package only binds the C ABI (capi) and generates the seeded synthetic
workloads (workloads) that the tests and the benchmark feed through it.
"""
from . import capi  # noqa: F401

__all__ = ["capi"]
