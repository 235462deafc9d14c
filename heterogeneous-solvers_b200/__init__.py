"""B200-native blocked SPD solve path for Gaussian-process kernel matrices.

Host-side mirror of TimThuering/Heterogeneous-Solvers' operator and solver
interface over the C ABI of libhs_b200.so (include/hs_b200.h).  The package
directory name is not a Python identifier; load it with ``load_package()``
from the repository root helpers, or import it as ``hs_b200`` after
registering it (tests/conftest.py, bench.py and __graft_entry__.py do so).
"""
from ._lib import HSError, NoConvergenceError, NotSPDError, LIB_PATH, load as load_library  # noqa: F401
from .core import *  # noqa: F401,F403
from .core import __all__ as _core_all

__all__ = list(_core_all) + ["load_library", "LIB_PATH"]
