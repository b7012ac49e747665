"""cie_b200 -- B200 (sm_100a) backend for the kelofm/cie linear-solve hot path.

The CUDA kernels and the C-ABI live in libciecu.so (include/ciecu*.h); this
package is the Python mirror of the reference's operator API on top of it.
Importing it loads the library and fails loudly if it has not been built.
"""
from . import _lib

_lib.load()

from ._lib import CiecuError, Statistics  # noqa: E402

__all__ = ["CiecuError", "Statistics"]
