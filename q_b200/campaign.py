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
                     nskip: int = 0, starts=None) -> PerturbationResult:
    """Every (replica, window) of the perturbation in one batch: steps_eq
    equilibration steps whose records are dropped, then steps_prod production
    steps whose energy records (the input's energy interval) feed BAR.
    Replica r uses Maxwell seed seed0 + r for all its windows, or, with
    starts (one .inp per replica, e.g. Equilibrated.inputs), starts every
    window from that replica's equilibrated restart: the windows run in
    parallel where QligFEP chains them one after another
    (INPUTS/run.sh:109-123)."""
    lambdas = [tuple(l) for l in lambdas]
    nw = len(lambdas)
    if starts is not None:
        replicas = len(starts)
        jobs = [(p, l) for p in starts for l in lambdas]
        with ThreadPoolExecutor(min(len(jobs), os.cpu_count() or 1)) as ex:
            systems = list(ex.map(lambda j: System.open(j[0], lambdas=j[1]), jobs))
    else:
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
        # warm-up as long as the timed run: its record capacity and step
        # graphs are in place before timing
        b.run(max(warmup, steps))
        b.clear_history()
        ms, _ = b.run_timed(steps)
    finally:
        b.close()
        s.close()
    return ms / 1e3 / steps


@dataclass
class Stage:
    """One equilibration stage: steps of stepsize fs at temperature K with the
    bath coupling (fs); restraint > 0 holds the solute atoms in a sequence
    restraint of that force constant (kcal/mol/A^2)."""
    steps: int
    stepsize: float
    temperature: float
    bath: float
    shake_hydrogens: bool
    restraint: float


# QligFEP's 2 fs heating schedule (INPUTS/eq1-5.inp with qligfep.py:107-123,
# 607-640): 0.1 fs at 1 K, then 50, 150, 275 K with the ligand restraint
# 10, 10, 5, 2.5, then the run temperature without it.
QLIGFEP_EQ_2FS = [
    Stage(10000, 0.1, 1.0, 0.2, False, 10.0),
    Stage(5000, 2.0, 50.0, 2.0, True, 10.0),
    Stage(5000, 2.0, 150.0, 2.0, True, 5.0),
    Stage(5000, 2.0, 275.0, 2.0, True, 2.5),
    Stage(50000, 2.0, 298.0, 10.0, True, 0.0),
]


@dataclass
class Equilibrated:
    restarts: list            # per replica: the .re after the last stage
    inputs: list              # per replica: an .inp that starts from it
    temperatures: list        # per stage: mean temperature of the replicas after the stage
    gpu_seconds: float


def equilibrate(inp: str, seeds, stages=QLIGFEP_EQ_2FS, *, lambdas=None, steps_scale: float = 1.0,
                restrain: tuple | None = None, precision: int = FP64, device: int = 0,
                tag: str = "eq") -> Equilibrated:
    """The heating protocol for every replica at once: stage k of all
    replicas is one batch, each system restarting from its own .re of stage
    k-1 (coordinates, velocities, water polarisation corrections), as qdyn
    chains eq1.re -> eq2 -> ... -> eq5.re.  Stage inputs are derived from
    `inp` (only the stage's keys change); the first stage draws Maxwell
    velocities at its temperature with each replica's seed.  `restrain`
    = (first, last) 1-based solute atoms held by the stages' restraint (default
    all solute atoms).  Returns, per replica, the last .re and an .inp that
    starts from it (for run_perturbation's windows)."""
    from .api import write_restart
    from .inputs import derive_inp
    seeds = [int(s) for s in seeds]
    probe = System.open(inp)
    nsol = probe.view.nat_solute
    probe.close()
    first, last = restrain or (1, nsol)
    lam = " ".join("%g" % x for x in lambdas) if lambdas is not None else None
    restarts = [None] * len(seeds)
    temps, gpu_ms = [], 0.0
    for k, st in enumerate(stages):
        steps = max(1, int(round(st.steps * steps_scale)))
        specs = []
        for r, seed in enumerate(seeds):
            md = {"steps": steps, "stepsize": st.stepsize, "temperature": st.temperature, "bath_coupling": st.bath,
                  "shake_hydrogens": "on" if st.shake_hydrogens else "off", "separate_scaling": "on"}
            drop = {"md": [], "files": ["trajectory", "energy"]}
            files = {"final": "%s%d_r%d.re" % (tag, k + 1, r)}
            if restarts[r] is None:
                md.update({"random_seed": seed, "initial_temperature": st.temperature})
                drop["files"].append("restart")
            else:
                drop["md"] += ["random_seed", "initial_temperature"]
                files["restart"] = os.path.basename(restarts[r])
            rows = {"sequence_restraints": ["%d %d %g 0 0" % (first, last, st.restraint)] if st.restraint > 0 else None,
                    "intervals": ["non_bond 25", "output %d" % max(steps, 1), "energy 0", "trajectory 0"]}
            if lam is not None:
                rows["lambdas"] = [lam]
            specs.append(derive_inp(inp, "%s%d_r%d.inp" % (tag, k + 1, r), set_keys={"md": md, "files": files},
                                    drop_keys=drop, set_rows=rows))
        systems = [System.open(p) for p in specs]
        batch = Batch(systems, precision=precision, device=device)
        try:
            ms, _ = batch.run_timed(steps)
            gpu_ms += ms
            d = os.path.dirname(os.path.abspath(inp))
            ts = []
            for r in range(len(seeds)):
                tc = batch.theta_corr(r, systems[r].view.nwpolr_shell) if systems[r].view.nwpolr_shell > 0 else None
                restarts[r] = os.path.join(d, "%s%d_r%d.re" % (tag, k + 1, r))
                write_restart(restarts[r], batch.coords(r), batch.velocities(r), tc)
                ts.append(float(batch.temperature(r)[0]))
            temps.append(float(np.mean(ts)))
        finally:
            batch.close()
            for s in systems:
                s.close()
    outs = []
    for r in range(len(seeds)):
        outs.append(derive_inp(inp, "%s_start_r%d.inp" % (tag, r),
                               set_keys={"files": {"restart": os.path.basename(restarts[r])}},
                               drop_keys={"md": ["random_seed", "initial_temperature"]}))
    return Equilibrated(restarts, outs, temps, gpu_ms / 1e3)


def dg_versus_plain(inp: str, *, windows: int = 21, replicas: int = 16, ref_windows: int = 41,
                    ref_replicas: int = 16, steps_eq: int = 1000, steps_prod: int = 10000, plain_steps: int = 1000,
                    rt: float = 0.592, device: int = 0, seed0: int = 1, placement=None) -> dict:
    """The batched mixed-precision perturbation against the dense-window FP64
    reference and the plain FP64 one-system-per-launch engine; all times are
    device seconds on this GPU.

    Without a placement model the product runs `windows` uniform windows.
    With one (lambda_placement.Placement) it runs the 5-window pilot (its
    device time counted), asks the network for the windows, and runs those.
    The plain engine runs the conventional protocol either way: `windows`
    uniform windows x the same replicas and steps, one system per launch (its
    per-step time measured here, times the system-steps)."""
    from .synth import window_lambdas
    pilot_s, placed = 0.0, None
    lams = window_lambdas(windows)
    if placement is not None:
        from . import lambda_placement as L
        pilot = L.sample([(inp, np.array(L.PILOT_U))], replicas=1, steps_eq=500, steps_prod=2000, device=device,
                         seed0=seed0 + 20000, bar=False)[0]
        pilot_s = pilot.gpu_seconds
        placed = placement.predict(L.pilot_features(pilot.dU[0]), device)[0]
        lams = L.windows_of(placed)
    prod = run_perturbation(inp, lams, replicas, steps_eq=steps_eq, steps_prod=steps_prod,
                            precision=MIXED, device=device, rt=rt, seed0=seed0)
    ref = run_perturbation(inp, window_lambdas(ref_windows), ref_replicas, steps_eq=steps_eq, steps_prod=steps_prod,
                           precision=FP64, device=device, rt=rt, seed0=seed0 + 10000)
    plain_step = time_single_window(inp, (0.5, 0.5), plain_steps, precision=FP64, device=device)
    system_steps = windows * replicas * (steps_eq + steps_prod)
    plain_s = plain_step * system_steps
    prod_s = prod.gpu_seconds + pilot_s
    diff = prod.dG_mean - ref.dG_mean
    diff_sem = float(np.hypot(prod.dG_sem, ref.dG_sem))
    return {
        "perturbation": {"windows": len(lams), "replicas": replicas, "steps_eq": steps_eq, "steps_prod": steps_prod,
                         "placement": "learned (5-window pilot + network)" if placement is not None else "uniform",
                         "lambda_2": [float(u) for u in (placed if placed is not None else
                                                         np.linspace(0.0, 1.0, windows))]},
        "batched_mixed": {k: v for k, v in asdict(prod).items() if k != "bar"},
        "pilot_gpu_seconds": pilot_s,
        "reference_fp64_dense": {k: v for k, v in asdict(ref).items() if k != "bar"},
        "plain_fp64_one_system_per_launch": {"windows": windows, "s_per_step": plain_step,
                                             "system_steps": system_steps, "gpu_seconds": plain_s},
        "dG_error": diff, "dG_error_sem": diff_sem, "within_0.1": bool(abs(diff) <= 0.1),
        "within_0.1_at_2_sem": bool(abs(diff) + 2.0 * diff_sem <= 0.1),
        "gpu_seconds_ratio_plain_over_batched": plain_s / prod_s,
    }


def dg_study(inp: str, *, replicas: int = 512, ref_replicas: int = 256, windows: int = 21, ref_windows: int = 41,
             steps_eq: int = 1000, steps_prod: int = 10000, device: int = 0, placement=None,
             max_systems: int = 4096) -> dict:
    """One dense FP64 reference judging two products of the same perturbation:
    the learned placement (pilot + network windows) and `windows` uniform
    windows, each batched in mixed precision with `replicas` replicas (split
    into batches of at most max_systems systems; device seconds summed).  With
    these replica counts the standard error of each product's error falls to
    ~0.05 kcal/mol.  Also the plain FP64 engine's device seconds for the
    uniform protocol one system per launch."""
    from .synth import window_lambdas

    def run(lams, reps, precision, seed0):
        per = max(1, max_systems // len(lams))
        dgs, gpu = [], 0.0
        for first in range(0, reps, per):
            n = min(per, reps - first)
            r = run_perturbation(inp, lams, n, steps_eq=steps_eq, steps_prod=steps_prod, precision=precision,
                                 device=device, seed0=seed0 + first)
            dgs += r.dG
            gpu += r.gpu_seconds
        return {"dG_mean": float(np.mean(dgs)), "dG_sem": float(np.std(dgs, ddof=1) / np.sqrt(len(dgs))),
                "gpu_seconds": gpu, "replicas": reps, "windows": len(lams)}

    ref = run(window_lambdas(ref_windows), ref_replicas, FP64, 100001)
    out = {"reference_fp64_dense": ref, "products": {}}
    pilot_s = 0.0
    if placement is not None:
        from . import lambda_placement as L
        pilot = L.sample([(inp, np.array(L.PILOT_U))], replicas=1, steps_eq=500, steps_prod=2000, device=device,
                         seed0=200001, bar=False)[0]
        pilot_s = pilot.gpu_seconds
        u = placement.predict(L.pilot_features(pilot.dU[0]), device)[0]
        p = run(L.windows_of(u), replicas, MIXED, 1)
        p["gpu_seconds"] += pilot_s
        p["lambda_2"] = [float(x) for x in u]
        out["products"]["learned"] = p
    out["products"]["uniform_%d" % windows] = run(window_lambdas(windows), replicas, MIXED, 1)
    plain_step = time_single_window(inp, (0.5, 0.5), 1000, precision=FP64, device=device)
    plain_s = plain_step * windows * replicas * (steps_eq + steps_prod)
    out["plain_fp64_one_system_per_launch"] = {"windows": windows, "s_per_step": plain_step, "gpu_seconds": plain_s}
    for name, p in out["products"].items():
        p["dG_error"] = p["dG_mean"] - ref["dG_mean"]
        p["dG_error_sem"] = float(np.hypot(p["dG_sem"], ref["dG_sem"]))
        p["within_0.1"] = bool(abs(p["dG_error"]) <= 0.1)
        p["gpu_seconds_ratio_plain_over_product"] = plain_s / p["gpu_seconds"]
    return out


def main(argv=None) -> int:
    """python -m q_b200.campaign dg-study <dir> [--replicas R] [--ref-replicas R]
    [--placement model.npz]: the perturbation of the synthetic FEP solute
    (its 8 Q atoms from state 1 to state 2), as the bench's dG check but at
    replica counts that bring the error's standard error near 0.05 kcal/mol."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("command", choices=["dg-study"])
    ap.add_argument("root")
    ap.add_argument("--replicas", type=int, default=512)
    ap.add_argument("--ref-replicas", type=int, default=256)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--placement", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                                         "placement_model.npz"))
    a = ap.parse_args(argv)
    from . import synth
    from .lambda_placement import Placement
    g = synth.fep_solute(os.path.join(a.root, "c1"), seed=1234, steps=a.steps)
    model = Placement.load(a.placement) if a.placement else None
    t0 = time.perf_counter()
    r = dg_study(g.inp, replicas=a.replicas, ref_replicas=a.ref_replicas, steps_prod=a.steps, placement=model)
    r["wall_s"] = time.perf_counter() - t0
    print(json.dumps(r, indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
