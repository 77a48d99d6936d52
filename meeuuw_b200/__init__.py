"""meeuuw_b200: B200 (sm_100a) implementation of meeuuw's per-timestep hot path.

The CUDA kernels live in ``libmeeuuw_b200.so`` (C ABI in ``include/meeuuw_b200.h``); this
package holds the host side: ctypes bindings (``_lib``), tensor-level ops (``ops``), the Stokes
solver driver, the timestep driver, and drop-in modules with the reference's function names
(``meeuuw_b200/dropin``).
"""
__version__ = "0.1.0"
