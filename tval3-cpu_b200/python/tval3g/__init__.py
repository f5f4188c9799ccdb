"""tval3g: TVAL3 total-variation reconstruction on NVIDIA B200 (sm_100a).

The solver core is libtval3g.so (C ABI, include/tval3g.h); ``capi`` binds it,
``workloads`` generates seeded synthetic problems.
"""
from . import capi, workloads  # noqa: F401
