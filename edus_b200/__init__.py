"""edus_b200 — B200-native k-space density-matrix propagation (EDUS drop-in).

Python mirror of the C ABI in include/edus_b200.h. The compute path is the
in-tree libedus_b200.so (sm_100a kernels + C++ host); this module only loads
it with ctypes. There is no CPU fallback: every call that needs the library
raises if it is missing.
"""
from .lib import (  # noqa: F401
    EdusError,
    Problem,
    Context,
    Batch,
    Server,
    load_library,
    parse_input,
    default_params,
    library_path,
    coulomb_generate,
)
from . import abi  # noqa: F401

__all__ = ["EdusError", "Problem", "Context", "Batch", "Server", "load_library", "parse_input", "default_params", "abi", "library_path", "coulomb_generate"]
