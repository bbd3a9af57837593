"""One perturbation's free energy from its lambda windows and replicas, all
stepped together in one batch on the GPU, analysed in place.

QligFEP runs a perturbation as a chain of qdyn processes, one window after
another (src/QligFEP/INPUTS/run.sh:109-123), then qfep on the energy files
(qligfep.py:906 write_qfep).  Here every window of every replica is one system
of a single batch: they equilibrate and sample together from the same
prepared start (each replica with its own Maxwell seed), their per-state
energy records stay on the device, and qfep's analysis (qb_batch_fep) runs on
them where they lie, BAR per replica.

`dg_versus_plain` measures the engine against the plain FP64 engine run one
system per launch: the batched mixed-precision perturbation's BAR free energy
and device seconds, a dense-window FP64 run of the same perturbation as the
judge of its error, and the plain engine's device seconds for the same
windows, replicas and steps (its per-step time measured on this GPU for one
window, times the system-steps: every window has the same atoms and lists).
"""
from __future__ import annotations

import os
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import asdict, dataclass, field

import numpy as np

from .api import FP64, MIXED, Batch, System


@dataclass
class PerturbationResult:
    dG: list                    # BAR free energy of each replica (kcal/mol)
    dG_mean: float
    dG_sem: float               # standard error over replicas (0 for one)
    gpu_seconds: float          # device time of all MD steps (CUDA events)
    analysis_seconds: float     # wall time of the free-energy analysis
    steps: int                  # MD steps per window (equilibration + production)
    windows: int
    replicas: int
    records_per_window: int
    precision: str = "mixed"
    bar: list = field(default_factory=list)   # per replica: per-window-pair BAR values


def open_systems(inp: str, lambdas, seeds, threads: int | None = None) -> list:
    """System.open of every (seed, lambda) pair, seeds outermost, on a thread
    pool (opening is host-only and the library releases the interpreter)."""
    jobs = [(tuple(l), int(s)) for s in seeds for l in lambdas]
    threads = threads or min(len(jobs), os.cpu_count() or 1)
    if threads <= 1:
        return [System.open(inp, lambdas=l, seed=s) for l, s in jobs]
    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(lambda j: System.open(inp, lambdas=j[0], seed=j[1]), jobs))


def run_perturbation(inp: str, lambdas, replicas: int = 1, *, steps_eq: int = 1000, steps_prod: int = 5000,
                     precision: int = MIXED, device: int = 0, rt: float = 0.592, seed0: int = 1,
                     nskip: int = 0) -> PerturbationResult:
    """Every (replica, window) of the perturbation in one batch: steps_eq
    equilibration steps whose records are dropped, then steps_prod production
    steps whose energy records (the input's energy interval) feed BAR.
    Replica r uses Maxwell seed seed0 + r for all its windows."""
    lambdas = [tuple(l) for l in lambdas]
    nw = len(lambdas)
    systems = open_systems(inp, lambdas, range(seed0, seed0 + replicas))
    batch = Batch(systems, precision=precision, device=device)
    try:
        gpu_ms = 0.0
        if steps_eq:
            ms, _ = batch.run_timed(steps_eq)
            gpu_ms += ms
        batch.clear_history()
        ms, _ = batch.run_timed(steps_prod)
        gpu_ms += ms
        dgs, bars = [], []
        t0 = time.perf_counter()
        nrec = 0
        for r in range(replicas):
            res = batch.fep(list(range(r * nw, (r + 1) * nw)), rt, nskip, nbins=10, nmin=1)
            dgs.append(res.dG_bar)
            bars.append([float(x) for x in res.dgbar[1:nw]])
            nrec = int(res.npts[0])
        ta = time.perf_counter() - t0
    finally:
        batch.close()
        for s in systems:
            s.close()
    sem = float(np.std(dgs, ddof=1) / np.sqrt(len(dgs))) if len(dgs) > 1 else 0.0
    return PerturbationResult(dgs, float(np.mean(dgs)), sem, gpu_ms / 1e3, ta, steps_eq + steps_prod, nw, replicas,
                              nrec, "fp64" if precision == FP64 else "mixed", bars)


def time_single_window(inp: str, lam, steps: int, *, precision: int = FP64, device: int = 0,
                       seed: int = 1, warmup: int = 50) -> float:
    """Device seconds per MD step of one window run alone (one system per
    launch, one CUDA graph replay per step): the plain engine a perturbation
    would otherwise run window after window."""
    s = System.open(inp, lambdas=tuple(lam), seed=seed)
    b = Batch([s], precision=precision, device=device)
    try:
        b.run(warmup)
        ms, _ = b.run_timed(steps)
    finally:
        b.close()
        s.close()
    return ms / 1e3 / steps


def dg_versus_plain(inp: str, *, windows: int = 21, replicas: int = 16, ref_windows: int = 41,
                    ref_replicas: int = 16, steps_eq: int = 1000, steps_prod: int = 10000, plain_steps: int = 1000,
                    rt: float = 0.592, device: int = 0, seed0: int = 1) -> dict:
    """The batched mixed-precision perturbation (uniform windows) against the
    dense-window FP64 reference and the plain FP64 one-system-per-launch
    engine; all times are device seconds on this GPU."""
    from .synth import window_lambdas
    prod = run_perturbation(inp, window_lambdas(windows), replicas, steps_eq=steps_eq, steps_prod=steps_prod,
                            precision=MIXED, device=device, rt=rt, seed0=seed0)
    ref = run_perturbation(inp, window_lambdas(ref_windows), ref_replicas, steps_eq=steps_eq, steps_prod=steps_prod,
                           precision=FP64, device=device, rt=rt, seed0=seed0 + 10000)
    plain_step = time_single_window(inp, (0.5, 0.5), plain_steps, precision=FP64, device=device)
    system_steps = windows * replicas * (steps_eq + steps_prod)
    plain_s = plain_step * system_steps
    diff = prod.dG_mean - ref.dG_mean
    diff_sem = float(np.hypot(prod.dG_sem, ref.dG_sem))
    return {
        "perturbation": {"windows": windows, "replicas": replicas, "steps_eq": steps_eq, "steps_prod": steps_prod},
        "batched_mixed": {k: v for k, v in asdict(prod).items() if k != "bar"},
        "reference_fp64_dense": {k: v for k, v in asdict(ref).items() if k != "bar"},
        "plain_fp64_one_system_per_launch": {"s_per_step": plain_step, "system_steps": system_steps,
                                             "gpu_seconds": plain_s},
        "dG_error": diff, "dG_error_sem": diff_sem, "within_0.1": bool(abs(diff) <= 0.1),
        "gpu_seconds_ratio_plain_over_batched": plain_s / prod.gpu_seconds,
    }
