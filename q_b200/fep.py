"""Free-energy analysis of per-state energy series on the GPU (include/qb_fep.h).

The analysis is qfep's (src/q6/qfep.f90:200-762): per pair of adjacent lambda
windows Zwanzig forward and reverse, thermodynamic integration, overlap
sampling and BAR, plus the energy-gap binned reaction free energies.  It runs
on energy series held on the host (`analyze`, e.g. read from .en files with
`read_en`) or on a batch's own records in place (`Batch.fep`).
"""
from __future__ import annotations

import ctypes as C
import os
import struct
from dataclasses import dataclass

import numpy as np

from ._lib import INCLUDE, QB_NEQ, _struct_from_header, check, lib

FepParams = _struct_from_header(os.path.join(INCLUDE, "qb_fep.h"), "qb_fep_params")
FepResultC = _struct_from_header(os.path.join(INCLUDE, "qb_fep.h"), "qb_fep_result")
MAX_STATES = 4
BAR_MAX_ITER = 1000
PART2_W = 9
PART3_W = 8


@dataclass
class FepResult:
    """qfep's results; per-window arrays use qfep's indexing 0..nfiles+1
    (entry i belongs to window i, 1-based)."""
    lam: np.ndarray
    npts: np.ndarray
    avEQ: np.ndarray
    dgf: np.ndarray
    dgfsum: np.ndarray
    dgr: np.ndarray
    dgrsum: np.ndarray
    dG: np.ndarray
    dgti: np.ndarray
    dgtisum: np.ndarray
    dglu: np.ndarray
    dglusum: np.ndarray
    dgbar: np.ndarray
    dgbarsum: np.ndarray
    bar_iterations: np.ndarray
    gap_range: np.ndarray
    part2: np.ndarray        # (nfiles, nbins+2, 9)
    part3: np.ndarray        # (nbins+2, 8)

    @property
    def dG_bar(self) -> float:
        """Total BAR free energy over all windows."""
        return float(self.dgbarsum[len(self.npts)])


def params(rt: float, nskip: int, *, gas: int = 0, nbins: int = 20, nmin: int = 5, alfa=(), coeff=(1.0, -1.0),
           evb=()):
    """qfep's input; evb = [(i, j, A, mu, eta, rxy0)] (states 1-based) are its
    off-diagonal elements Hij(r_xy) (qfep.f90:163-172)."""
    p = FepParams()
    p.rt = float(rt)
    p.nskip = int(nskip)
    p.gas = int(gas)
    p.nbins = int(nbins)
    p.nmin = int(nmin)
    for k in range(MAX_STATES):
        p.alfa[k] = 0.0
        p.coeff[k] = 0.0
    for k, a in enumerate(alfa):
        if k + 1 < MAX_STATES:
            p.alfa[k + 1] = float(a)
    for k, c in enumerate(coeff[:MAX_STATES]):
        p.coeff[k] = float(c)
    p.nnoffd = len(evb)
    for i, j, A, mu, eta, r0 in evb:
        if not (1 <= i <= MAX_STATES and 1 <= j <= MAX_STATES):
            raise ValueError("off-diagonal element states out of range: %d %d" % (i, j))
        k = (i - 1) * MAX_STATES + (j - 1)
        p.evb_A[k], p.evb_mu[k], p.evb_eta[k], p.evb_rxy0[k] = float(A), float(mu), float(eta), float(r0)
    return p


def _buffers(nfiles: int, nstates: int, nbins: int):
    nb = nbins + 2
    arrs = {
        "lambda": np.zeros(nfiles * nstates), "npts": np.zeros(nfiles, dtype=np.int32),
        "avEQ": np.zeros(nfiles * nstates * QB_NEQ),
        "dgf": np.zeros(nfiles + 2), "dgfsum": np.zeros(nfiles + 2), "dgr": np.zeros(nfiles + 2),
        "dgrsum": np.zeros(nfiles + 2), "dG": np.zeros(nfiles + 2), "dgti": np.zeros(nfiles + 2),
        "dgtisum": np.zeros(nfiles + 2), "dglu": np.zeros(nfiles + 2), "dglusum": np.zeros(nfiles + 2),
        "dgbar": np.zeros(nfiles + 2), "dgbarsum": np.zeros(nfiles + 2),
        "bar_iterations": np.zeros(nfiles + 2, dtype=np.int32), "gap_range": np.zeros(2),
        "part2": np.zeros(nfiles * nb * PART2_W), "part3": np.zeros(nb * PART3_W),
    }
    r = FepResultC()
    for name, a in arrs.items():
        ct = C.c_int if a.dtype == np.int32 else C.c_double
        setattr(r, name, a.ctypes.data_as(C.POINTER(ct)))
    return r, arrs


def _result(arrs, nfiles: int, nstates: int, nbins: int) -> FepResult:
    nb = nbins + 2
    return FepResult(arrs["lambda"].reshape(nfiles, nstates), arrs["npts"].astype(int),
                     arrs["avEQ"].reshape(nfiles, nstates, QB_NEQ), arrs["dgf"], arrs["dgfsum"], arrs["dgr"],
                     arrs["dgrsum"], arrs["dG"], arrs["dgti"], arrs["dgtisum"], arrs["dglu"], arrs["dglusum"],
                     arrs["dgbar"], arrs["dgbarsum"], arrs["bar_iterations"].astype(int), arrs["gap_range"],
                     arrs["part2"].reshape(nfiles, nb, PART2_W), arrs["part3"].reshape(nb, PART3_W))


def analyze(series, p, device: int = 0, rxy=None) -> FepResult:
    """series: one array (npts, nstates, 15) per lambda window, in window
    order; with EVB elements in p, rxy gives each window's r_xy per record."""
    series = [np.ascontiguousarray(s, dtype=np.float64) for s in series]
    nfiles, nstates = len(series), series[0].shape[1]
    E = np.ascontiguousarray(np.concatenate([s.reshape(-1) for s in series]))
    npts = np.array([s.shape[0] for s in series], dtype=np.int32)
    if p.nnoffd > 0:
        if rxy is None or len(rxy) != nfiles or any(len(x) != n for x, n in zip(rxy, npts)):
            raise ValueError("EVB analysis needs r_xy for every record of every window")
        R = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64) for x in rxy]))
        p.rxy = R.ctypes.data_as(C.POINTER(C.c_double))
    r, arrs = _buffers(nfiles, nstates, p.nbins)
    check(lib.qb_fep_analyze(E.ctypes.data_as(C.POINTER(C.c_double)), npts.ctypes.data_as(C.POINTER(C.c_int)),
                             nfiles, nstates, C.addressof(p), int(device), C.addressof(r)))
    return _result(arrs, nfiles, nstates, p.nbins)


def batch_fep(batch, systems, p) -> FepResult:
    """The analysis of a batch's energy-file records, systems in window order."""
    sys_ = np.array(list(systems), dtype=np.int32)
    nstates = int(batch.systems[int(sys_[0])].nstates)
    r, arrs = _buffers(len(sys_), nstates, p.nbins)
    check(lib.qb_batch_fep(batch._b, sys_.ctypes.data_as(C.POINTER(C.c_int)), len(sys_), C.addressof(p),
                           C.addressof(r)))
    return _result(arrs, len(sys_), nstates, p.nbins)


def read_en(path: str, nstates: int) -> np.ndarray:
    """Records of a qdyn energy file (nrgy.f90:94-119, gfortran sequential
    unformatted): per frame one record (int, 15 doubles) per state and one
    off-diagonal record.  Returns (frames, nstates, 15); a trailing partial
    frame is dropped, as get_ene stops at the end of file."""
    raw = open(path, "rb").read()
    recs = []
    pos = 0
    while pos + 4 <= len(raw):
        (n,) = struct.unpack_from("<i", raw, pos)
        if n < 0 or pos + 8 + n > len(raw):
            break
        recs.append(raw[pos + 4:pos + 4 + n])
        pos += 8 + n
    frames = []
    k = 0
    # a frame counts once its off-diagonal record is read too (get_ene)
    while k + nstates + 1 <= len(recs):
        block = recs[k:k + nstates]
        if any(len(b) != 4 + 8 * QB_NEQ for b in block):
            break
        frames.append([np.frombuffer(b, dtype="<f8", offset=4, count=QB_NEQ) for b in block])
        k += nstates + 1
    return np.array(frames, dtype=np.float64).reshape(len(frames), nstates, QB_NEQ)


def read_offdiag(path: str, nstates: int) -> np.ndarray:
    """The off-diagonal record of every frame of a qdyn energy file
    (nrgy.f90:60-65): (frames, noffd, 4) of state i, state j, Hij, r_kl."""
    raw = open(path, "rb").read()
    recs, pos = [], 0
    while pos + 4 <= len(raw):
        (n,) = struct.unpack_from("<i", raw, pos)
        if n < 0 or pos + 8 + n > len(raw):
            break
        recs.append(raw[pos + 4:pos + 4 + n])
        pos += 8 + n
    out = []
    for k in range(nstates, len(recs), nstates + 1):
        r = recs[k]
        out.append([struct.unpack_from("<iidd", r, 24 * m) for m in range(len(r) // 24)])
    n = min((len(o) for o in out), default=0)
    return np.array([o[:n] for o in out], dtype=np.float64).reshape(len(out), n, 4)
