"""q_b200 -- a B200 (sm_100a) engine for the MD step of Q's qdyn.

Host-side Python over libqb's C ABI (include/qb.h).  Importing the package
loads the in-tree CUDA library and fails loudly if it has not been built.
"""
from .api import FP64, MIXED, Batch, System, append_energy, device_count, maxwell, write_restart  # noqa: F401
from ._lib import E_NAMES, EQ_NAMES, QB_NE, QB_NEQ, QBError  # noqa: F401

__version__ = "0.1.0"
