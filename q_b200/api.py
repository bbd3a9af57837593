"""Python host API over libqb (the QligFEP-side driver of the engine).

    sys = System.open("md.inp")                # parse + qdyn set-up (host only)
    batch = Batch([sys1, sys2, ...])           # upload to the GPU
    batch.run(1000)                            # md_run steps for every system
    E, EQ = batch.energies(0)

Energies are returned as dicts keyed by the names of the reference's energy
types (nrgy.f90:43-58).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import E_NAMES, EQ_NAMES, QB_NE, QB_NEQ, Options, SysView, check, lib

FP64 = 0
MIXED = 1
MAX_STATES = 10                                  # QB_MAX_STATES
HIST_REC = 1 + QB_NE + MAX_STATES * QB_NEQ + MAX_STATES   # QB_HIST_REC

Tuning = _lib._struct_from_header(_lib.os.path.join(_lib.INCLUDE, "qb.h"), "qb_tuning")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class System:
    """One prepared system (qb_open)."""

    def __init__(self, handle: C.c_void_p, path: str):
        self._h = handle
        self.path = path
        self.view = SysView()
        check(lib.qb_get_view(self._h, C.byref(self.view)))

    @classmethod
    def open(cls, inp_path: str, lambdas: Sequence[float] | None = None, seed: int = -1) -> "System":
        h = C.c_void_p()
        if lambdas is None and seed < 0:
            check(lib.qb_open(inp_path.encode(), None, C.byref(h)))
        else:
            lam = np.ascontiguousarray(lambdas if lambdas is not None else [], dtype=np.float64)
            check(lib.qb_open_override(inp_path.encode(), None, _dp(lam) if lam.size else None,
                                       int(lam.size), int(seed), C.byref(h)))
        return cls(h, inp_path)

    @property
    def natom(self) -> int:
        return self.view.natom

    @property
    def nstates(self) -> int:
        return self.view.nstates

    def array(self, name: str, n: int | None = None, dtype=None) -> np.ndarray:
        """Copy of a pointer field of the view (n elements)."""
        ptr = getattr(self.view, name)
        if n is None:
            n = 3 * self.natom
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

    def close(self) -> None:
        if self._h:
            lib.qb_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Systems stepped together on one GPU (qb_batch_*)."""

    def __init__(self, systems: Sequence[System], precision: int = FP64, device: int = 0):
        self.systems = list(systems)
        arr = (C.c_void_p * len(self.systems))(*[s._h for s in self.systems])
        opt = Options(precision=precision, device=device, verbose=0)
        self._b = C.c_void_p()
        check(lib.qb_batch_create(arr, len(self.systems), C.byref(opt), C.byref(self._b)))

    def run(self, nsteps: int) -> None:
        check(lib.qb_batch_run(self._b, int(nsteps)))

    def run_timed(self, nsteps: int) -> tuple[float, int]:
        """Run nsteps; return (device milliseconds, kernel launches)."""
        ms = C.c_double()
        n = C.c_longlong()
        check(lib.qb_batch_run_timed(self._b, int(nsteps), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def final_energy(self) -> None:
        check(lib.qb_batch_final_energy(self._b))

    def evaluate(self, energies: bool = True) -> None:
        """Lists and gradient at the current coordinates as a step that
        records energies (True) or one that does not (False: the mixed
        engine's packed FP32 water-water forces, no water-water energy)."""
        check(lib.qb_batch_evaluate(self._b, 1 if energies else 0))

    def fep(self, systems, rt: float, nskip: int = 0, **kw):
        """qfep's analysis of these systems' energy-file records, in window
        order (q_b200.fep.params for the keyword arguments)."""
        from .fep import batch_fep, params
        return batch_fep(self, systems, params(rt, nskip, **kw))

    def energies(self, sys: int) -> tuple[dict, list[dict]]:
        E = np.zeros(QB_NE)
        S = self.systems[sys].nstates
        EQ = np.zeros(max(S, 1) * QB_NEQ)
        check(lib.qb_batch_energies(self._b, sys, _dp(E), _dp(EQ)))
        return (dict(zip(E_NAMES, E.tolist())),
                [dict(zip(EQ_NAMES, EQ[k * QB_NEQ:(k + 1) * QB_NEQ].tolist())) for k in range(S)])

    def energy_vectors(self, sys: int) -> tuple[np.ndarray, np.ndarray]:
        E = np.zeros(QB_NE)
        S = self.systems[sys].nstates
        EQ = np.zeros(max(S, 1) * QB_NEQ)
        check(lib.qb_batch_energies(self._b, sys, _dp(E), _dp(EQ)))
        return E, EQ[:S * QB_NEQ].reshape(S, QB_NEQ)

    def temperature(self, sys: int) -> np.ndarray:
        t = np.zeros(5)
        check(lib.qb_batch_temperature(self._b, sys, _dp(t)))
        return t

    def _vec(self, fn, sys: int) -> np.ndarray:
        out = np.zeros(3 * self.systems[sys].natom)
        check(fn(self._b, sys, _dp(out)))
        return out

    def gradient(self, sys: int) -> np.ndarray:
        return self._vec(lib.qb_batch_gradient, sys)

    def coords(self, sys: int) -> np.ndarray:
        return self._vec(lib.qb_batch_get_coords, sys)

    def velocities(self, sys: int) -> np.ndarray:
        return self._vec(lib.qb_batch_get_velocities, sys)

    def set_coords(self, sys: int, x: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        check(lib.qb_batch_set_coords(self._b, sys, _dp(x)))

    def set_velocities(self, sys: int, v: np.ndarray) -> None:
        v = np.ascontiguousarray(v, dtype=np.float64)
        check(lib.qb_batch_set_velocities(self._b, sys, _dp(v)))

    # every system at once: one copy per call through the batch's pinned staging
    @property
    def natom_total(self) -> int:
        return sum(s.natom for s in self.systems)

    def coords_all(self, out: np.ndarray | None = None) -> np.ndarray:
        """Every system's coordinates, x y z per atom; `out` may be a
        page-locked buffer (copied into at full link speed)."""
        if out is None:
            out = np.zeros(3 * self.natom_total)
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == 3 * self.natom_total
        check(lib.qb_batch_get_coords_all(self._b, _dp(out)))
        return out

    def velocities_all(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros(3 * self.natom_total)
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == 3 * self.natom_total
        check(lib.qb_batch_get_velocities_all(self._b, _dp(out)))
        return out

    def set_coords_all(self, x: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.size == 3 * self.natom_total
        check(lib.qb_batch_set_coords_all(self._b, _dp(x)))

    def set_velocities_all(self, v: np.ndarray) -> None:
        v = np.ascontiguousarray(v, dtype=np.float64)
        assert v.size == 3 * self.natom_total
        check(lib.qb_batch_set_velocities_all(self._b, _dp(v)))

    def history_all(self, kind: int = 0, max_records: int | None = None, with_bytes: bool = False,
                    out: np.ndarray | None = None):
        """(counts[nsys], records[nsys, m, QB_HIST_REC]) of every system in
        two device copies; a record is step, E[QB_NE], EQ[QB_MAX_STATES,
        QB_NEQ], r_kl[QB_MAX_STATES].  With max_records None the counts are
        queried first (one more copy).  with_bytes adds the bytes the call
        copied from the device.  `out` (float64, C order, at least nsys x
        max_records x QB_HIST_REC values, e.g. a page-locked buffer) receives
        the records instead of a new array."""
        n = len(self.systems)
        counts = np.zeros(n, dtype=np.int32)
        ip = counts.ctypes.data_as(C.POINTER(C.c_int))
        nb = C.c_size_t(0)
        total = 0
        if max_records is None:
            check(lib.qb_batch_history_all(self._b, kind, 0, ip, None, C.byref(nb)))
            total += nb.value
            max_records = int(counts.max(initial=0))
        m = max(int(max_records), 1)
        if out is None:
            rec = np.zeros((n, m, HIST_REC))
        else:
            assert out.dtype == np.float64 and out.flags.c_contiguous and out.size >= n * m * HIST_REC
            rec = out.reshape(-1)[:n * m * HIST_REC].reshape(n, m, HIST_REC)
        check(lib.qb_batch_history_all(self._b, kind, m, ip, _dp(rec), C.byref(nb)))
        total += nb.value
        m = int(counts.max(initial=0))
        out = (counts, rec[:, :m])
        return out + (total,) if with_bytes else out

    def step_count(self) -> int:
        n = C.c_longlong()
        check(lib.qb_batch_step_count(self._b, C.byref(n)))
        return n.value

    def box(self, sys: int) -> np.ndarray:
        """Periodic box of system `sys`: edge lengths, then centre."""
        out = np.zeros(6)
        check(lib.qb_batch_box(self._b, sys, _dp(out), None, None))
        return out

    def volume_moves(self, sys: int) -> tuple[int, int]:
        """Monte Carlo volume moves (tried, accepted) of a constant-pressure run."""
        t, a = C.c_longlong(), C.c_longlong()
        check(lib.qb_batch_box(self._b, sys, _dp(np.zeros(6)), C.byref(t), C.byref(a)))
        return t.value, a.value

    def theta_corr(self, sys: int, n: int = 4) -> np.ndarray:
        out = np.zeros(n, dtype=np.float32)
        check(lib.qb_batch_get_theta_corr(self._b, sys, out.ctypes.data_as(C.POINTER(C.c_float)), n))
        return out

    def history(self, sys: int, kind: int = 0):
        """(steps, E[n, QB_NE], EQ[n, S, QB_NEQ]) recorded during run()."""
        cnt = C.c_int()
        check(lib.qb_batch_history(self._b, sys, kind, C.byref(cnt), None, None, None))
        n = cnt.value
        S = self.systems[sys].nstates
        steps = np.zeros(max(n, 1), dtype=np.int32)
        E = np.zeros((max(n, 1), QB_NE))
        EQ = np.zeros((max(n, 1), max(S, 1), QB_NEQ))
        check(lib.qb_batch_history(self._b, sys, kind, C.byref(cnt),
                                   steps.ctypes.data_as(C.POINTER(C.c_int)), _dp(E), _dp(EQ)))
        return steps[:n], E[:n], EQ[:n, :S]

    def offdiag(self, sys: int, kind: int = 0) -> np.ndarray:
        """[n, noffd, 2] (Hij, r_kl) of the records history() returns, for the
        system's EVB off-diagonal functions (offdiag, md.f90:12911)."""
        cnt = C.c_int()
        check(lib.qb_batch_offdiag(self._b, sys, kind, C.byref(cnt), None))
        n, m = cnt.value, self.systems[sys].view.noffd
        out = np.zeros(max(n * m * 2, 1))
        check(lib.qb_batch_offdiag(self._b, sys, kind, C.byref(cnt), _dp(out)))
        return out[:n * m * 2].reshape(n, m, 2)

    def clear_history(self) -> None:
        check(lib.qb_batch_clear_history(self._b))

    def set_profiling(self, on: bool) -> None:
        check(lib.qb_batch_set_profiling(self._b, 1 if on else 0))

    def profile(self) -> dict:
        n = 64
        names = C.create_string_buffer(8192)
        ms = np.zeros(n)
        launches = np.zeros(n, dtype=np.int64)
        nk = C.c_int()
        check(lib.qb_batch_profile(self._b, names, len(names), _dp(ms),
                                   launches.ctypes.data_as(C.POINTER(C.c_longlong)), n, C.byref(nk)))
        keys = names.value.decode().split("\n")[:nk.value]
        return {k: (float(ms[i]), int(launches[i])) for i, k in enumerate(keys)}

    def workload(self) -> np.ndarray:
        """Work totals of the last run: ww molecule pairs, pw, pp, qp, qw pairs,
        atoms, SHAKE constraints, charge groups, mean SHAKE iterations per
        molecule and step, most iterations of one molecule."""
        out = np.zeros(10)
        check(lib.qb_batch_workload(self._b, _dp(out), 10))
        return out

    def tuning(self) -> dict:
        """The step kernels' run-time choices (qb_tuning)."""
        t = Tuning()
        check(lib.qb_batch_get_tuning(self._b, C.addressof(t)))
        return {name: getattr(t, name) for name, _ in t._fields_}

    def set_tuning(self, **kw) -> None:
        t = Tuning()
        check(lib.qb_batch_get_tuning(self._b, C.addressof(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        check(lib.qb_batch_set_tuning(self._b, C.addressof(t)))

    def autotune(self, steps_per_trial: int = 100) -> dict:
        """Time candidate settings on real MD steps and keep the fastest
        (the steps advance every system; their energy records are cleared)."""
        t = Tuning()
        check(lib.qb_batch_autotune(self._b, steps_per_trial, C.addressof(t)))
        return {name: getattr(t, name) for name, _ in t._fields_}

    def status(self, sys: int) -> int:
        st = C.c_int()
        check(lib.qb_batch_status(self._b, sys, C.byref(st)))
        return st.value

    def close(self) -> None:
        if self._b:
            lib.qb_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_count() -> int:
    n = C.c_int()
    lib.qb_device_count(C.byref(n))
    return n.value


def peak_tflops(precision: int = FP64, device: int = 0) -> float:
    """Measured CUDA-core FMA throughput (TFLOP/s)."""
    t = C.c_double()
    check(lib.qb_peak_flops(device, precision, C.byref(t)))
    return t.value


def write_restart(path: str, x: np.ndarray, v: np.ndarray, theta_corr: np.ndarray | None = None,
                  box: np.ndarray | None = None) -> None:
    """qdyn's restart file; box: a periodic box's edge lengths and centre
    (6 values), written as its two trailing records."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    ns = 0 if theta_corr is None else int(theta_corr.size)
    tc = None if theta_corr is None else np.ascontiguousarray(theta_corr, dtype=np.float32)
    tcp = tc.ctypes.data_as(C.POINTER(C.c_float)) if tc is not None else None
    if box is None:
        check(lib.qb_write_re(path.encode(), x.size // 3, _dp(x), _dp(v), ns, tcp))
    else:
        b6 = np.ascontiguousarray(box, dtype=np.float64)
        check(lib.qb_write_re_box(path.encode(), x.size // 3, _dp(x), _dp(v), ns, tcp, _dp(b6)))


def append_energy(path: str, EQ: np.ndarray, offd=None) -> None:
    """One energy-file frame; offd = (ij[noffd, 2] state numbers, hr[noffd, 2]
    of Hij and r_kl) fills its off-diagonal record."""
    EQ = np.ascontiguousarray(EQ, dtype=np.float64)
    ns = EQ.shape[0] if EQ.ndim == 2 else 0
    if offd is None or len(offd[0]) == 0:
        check(lib.qb_append_en(path.encode(), ns, _dp(EQ)))
        return
    ij = np.ascontiguousarray(offd[0], dtype=np.int32)
    hr = np.ascontiguousarray(offd[1], dtype=np.float64)
    check(lib.qb_append_en_offd(path.encode(), ns, _dp(EQ), ij.shape[0], ij.ctypes.data_as(C.POINTER(C.c_int)),
                                _dp(hr)))


def maxwell(seed: int, temperature: float, mass: np.ndarray) -> np.ndarray:
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    out = np.zeros(3 * mass.size)
    check(lib.qb_maxwell(int(seed), float(temperature), mass.size, _dp(mass), _dp(out)))
    return out
