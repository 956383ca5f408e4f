"""B200 (sm_100a) implementation of InductionEq's time-stepping path.

The product is the C-ABI shared library ``_lib/libinductioneq_b200.so`` (include/*.h);
``lib`` binds it with ctypes and ``induction_eq`` mirrors the reference's MATLAB host
driver on top of it.
"""
from .lib import Context, IeqError, load  # noqa: F401

__all__ = ["Context", "IeqError", "load"]
