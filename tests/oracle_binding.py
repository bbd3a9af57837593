"""ctypes binding of the CPU oracle (oracle/qoracle.c) for the tests.

The oracle is the checker: tests run it beside the product on the same
prepared system and compare.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from q_b200._lib import QB_NE, QB_NEQ, SysView

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(REPO, "oracle", "_build", "libqoracle.so")


class Oracle:
    def __init__(self, lib: C.CDLL):
        self.lib = lib

    def create(self, system, history: int = 4096) -> "OracleRun":
        return OracleRun(self.lib, system, history)


class OracleRun:
    """md_run of one system on the CPU oracle."""

    def __init__(self, lib, system, history):
        self.lib = lib
        self.system = system          # keeps the view's memory alive
        self.view = system.view
        self.S = self.view.nstates
        self.N = self.view.natom
        self.st = lib.qo_create(C.byref(self.view), history)

    def run(self, n: int) -> int:
        return self.lib.qo_run(self.st, n)

    def final_energy(self) -> None:
        self.lib.qo_final_energy(self.st)

    def energy_vectors(self):
        E = np.zeros(QB_NE)
        EQ = np.zeros(max(self.S, 1) * QB_NEQ)
        self.lib.qo_energies(self.st, E.ctypes.data_as(C.POINTER(C.c_double)),
                             EQ.ctypes.data_as(C.POINTER(C.c_double)))
        return E, EQ[:self.S * QB_NEQ].reshape(self.S, QB_NEQ)

    def _vec(self, fn):
        out = np.zeros(3 * self.N)
        fn(self.st, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def gradient(self):
        return self._vec(self.lib.qo_gradient)

    def coords(self):
        return self._vec(self.lib.qo_coords)

    def velocities(self):
        return self._vec(self.lib.qo_velocities)

    def temperature(self):
        out = np.zeros(5)
        self.lib.qo_temperature(self.st, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def theta_corr(self):
        n = self.view.nwpolr_shell
        out = np.zeros(max(n, 1), dtype=np.float32)
        self.lib.qo_theta_corr(self.st, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out[:n]

    def history(self, kind: int = 0):
        n = self.lib.qo_history(self.st, kind, None, None, None)
        steps = np.zeros(max(n, 1), dtype=np.int32)
        E = np.zeros((max(n, 1), QB_NE))
        EQ = np.zeros((max(n, 1), max(self.S, 1), QB_NEQ))
        self.lib.qo_history(self.st, kind, steps.ctypes.data_as(C.POINTER(C.c_int)),
                            E.ctypes.data_as(C.POINTER(C.c_double)), EQ.ctypes.data_as(C.POINTER(C.c_double)))
        return steps[:n], E[:n], EQ[:n, :self.S]

    def offdiag(self, kind: int = 0):
        """[records, noffd] r_kl of each record's off-diagonal functions."""
        c = self.lib.qo_history(self.st, kind, None, None, None)
        n = self.view.noffd
        out = np.zeros(max(c * n, 1))
        self.lib.qo_offdiag(self.st, kind, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out[:c * n].reshape(c, n)

    def box(self):
        """Periodic box: edge lengths and centre (6 values)."""
        out = np.zeros(6)
        self.lib.qo_box(self.st, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def volume_moves(self):
        t, a = C.c_longlong(), C.c_longlong()
        self.lib.qo_volume_moves(self.st, C.byref(t), C.byref(a))
        return t.value, a.value

    def list_counts(self):
        out = (C.c_int * 5)()
        self.lib.qo_list_counts(self.st, out)
        return list(out)

    def __del__(self):
        try:
            self.lib.qo_destroy(self.st)
        except Exception:
            pass


def load_oracle() -> Oracle:
    lib = C.CDLL(ORACLE_SO)
    vp, dp = C.c_void_p, C.POINTER(C.c_double)
    lib.qo_create.restype = vp
    lib.qo_create.argtypes = [C.POINTER(SysView), C.c_int]
    lib.qo_destroy.argtypes = [vp]
    lib.qo_run.argtypes = [vp, C.c_int]
    lib.qo_final_energy.argtypes = [vp]
    lib.qo_energies.argtypes = [vp, dp, dp]
    for f in ("qo_gradient", "qo_coords", "qo_velocities", "qo_temperature"):
        getattr(lib, f).argtypes = [vp, dp]
    lib.qo_theta_corr.argtypes = [vp, C.POINTER(C.c_float)]
    lib.qo_history.argtypes = [vp, C.c_int, C.POINTER(C.c_int), dp, dp]
    lib.qo_offdiag.argtypes = [vp, C.c_int, dp]
    lib.qo_list_counts.argtypes = [vp, C.POINTER(C.c_int)]
    lib.qo_status.argtypes = [vp]
    lib.qo_box.argtypes = [vp, dp]
    lib.qo_volume_moves.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    return Oracle(lib)
