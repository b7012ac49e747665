"""cie_b200 -- B200 (sm_100a) backend for the kelofm/cie linear-solve hot path.

The CUDA kernels and the C-ABI live in libciecu.so (include/ciecu*.h); this
package is the Python mirror of the reference's operator API on top of it.
The library is loaded on first use (cie_b200.load()); a missing build fails
loudly -- there is no CPU fallback.
"""
from ._lib import CiecuError, Statistics, load  # noqa: F401

__all__ = ["CiecuError", "Statistics", "load"]
