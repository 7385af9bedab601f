"""hfgpu: Python binding of libhfg (the B200 Fock-build library).

The product is the CUDA library hf-rs_b200/libhfg.so with the C ABI of
include/hfg.h; this package loads it through ctypes for tests, the
benchmark and Python callers.  There is no CPU fallback: if the library is
missing or no CUDA device is present, the calls raise.
"""
from .lib import Context, HfgError, JKOptions, load_library, library_path  # noqa: F401
from .basis import CartesianBasis  # noqa: F401
from .clusters import water_cluster  # noqa: F401
