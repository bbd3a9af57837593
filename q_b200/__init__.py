"""q_b200 -- a B200 (sm_100a) engine for the MD step of Q's qdyn.

Host-side Python over libqb's C ABI (include/qb.h).  The in-tree CUDA library
is loaded on first use of the API (not on `import q_b200.build`), and loading
fails loudly if it has not been built.
"""
__version__ = "0.1.0"

_API = {"FP64", "MIXED", "Batch", "System", "append_energy", "device_count", "maxwell", "write_restart",
        "peak_tflops"}
_LIB = {"E_NAMES", "EQ_NAMES", "QB_NE", "QB_NEQ", "QBError"}


def __getattr__(name):
    if name in _API:
        from . import api
        return getattr(api, name)
    if name in _LIB:
        from . import _lib
        return getattr(_lib, name)
    raise AttributeError(name)
