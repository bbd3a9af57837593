#!/usr/bin/env python
"""Throughput of the batched Q MD step on B200 (one JSON line on stdout).

Workload (one GPU): the batched FEP configuration -- 21 uniform lambda windows
x 4 seeded replicas of the 56-atom, 8-Q-atom FEP solute in a 20 A TIP3P sphere
(2 fs, SHAKE on X-H bonds and water, 10 A cut-offs + LRF) plus 16 TIP3P spheres
with radii drawn from {15, 20, 25} A (1 fs), all stepped together in one batch.
Synthetic, seeded inputs of those shapes (q_b200/synth.py).

A step is one MD step of every system.  `value` is the aggregate simulated
ns/day over all systems and ranks with the state resident in HBM, timed with
CUDA events on the engine's stream around exactly --steps steps; the timed
steps start on a pair-list rebuild step, so they hold the rebuilds (and the
energy-recording steps) of their share of list cycles (counted in the line).
`e2e` is the same metric through the C ABI with host buffers: coordinates and
velocities of every system uploaded, the steps run, the energy records and
coordinates read back, all inside the timed region, one copy per direction
through the batch's page-locked staging.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl qb|reference]
                    [--precision fp64|mixed]

At one GPU the line also carries single-system lines of the three plain
configurations (per_config: the 15 A water sphere, the FEP solute in 20 A, the
protein-ligand sphere in 25 A; FP64, one system per batch) and the second half
of the metric (`dG`, `gpu_s_per_dG`): the perturbation's BAR free energy from
21 uniform windows x --dg-replicas replicas in one mixed-precision batch, its
device seconds, the plain FP64 engine's device seconds for the same windows,
replicas and steps run one system per launch, and the error against a dense
41-window FP64 run of the same perturbation.

Under torchrun each rank runs its own copy of the batch (weak scaling); time is
the maximum over ranks.  `--impl reference` runs the reference's algorithm on
the host cores: the CPU oracle (the restatement of Q's Fortran step, which
cannot be compiled here) steps the same batch, every system in its own process
spread over all cores by cost, wall-clocked as the slowest worker.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "aggregate ns/day (batched λ-windows) & GPU-s per ΔG at ≤0.1 kcal/mol vs plain"
WORKLOAD = ("21 lambda windows x 4 replicas of the 56-atom 8-Q-atom FEP solute in a 20 A TIP3P sphere "
            "(2 fs) + 16 TIP3P spheres R in {15,20,25} A (1 fs), one batch")
FLOP_WW = 229        # per SPC/TIP3P molecule pair (1 LJ+Coulomb, 8 Coulomb)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="qb", choices=["qb", "reference"])
    p.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    p.add_argument("--windows", type=int, default=21)
    p.add_argument("--replicas", type=int, default=4)
    p.add_argument("--spheres", type=int, default=16)
    p.add_argument("--equil", type=int, default=100, help="untimed equilibration steps (in addition to warm-up)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the single-system lines of the plain configs")
    p.add_argument("--no-autotune", action="store_true", help="keep the default tile sizes and streams")
    p.add_argument("--dg-replicas", type=int, default=32,
                   help="replicas of the batched mixed-precision perturbation for the GPU-s per dG comparison "
                        "(0 skips it; runs at one GPU only)")
    p.add_argument("--dg-ref-replicas", type=int, default=32, help="replicas of the dense FP64 reference")
    p.add_argument("--dg-ref-windows", type=int, default=41)
    p.add_argument("--dg-equil", type=int, default=1000)
    p.add_argument("--dg-steps", type=int, default=10000, help="production steps per window")
    p.add_argument("--dg-placement", default="learned", choices=["learned", "uniform"],
                   help="learned: the 5-window pilot and the trained network place the product's windows "
                        "(q_b200/data/placement_model.npz); uniform: --windows uniform windows")
    return p.parse_args()


def workload_files(root: str, rank: int, args):
    """Generate (or reuse) the Q input files of the batch; returns a list of
    (inp, lambdas, seed, dt_fs)."""
    import numpy as np

    from q_b200 import synth
    from q_b200.synth import window_lambdas
    os.makedirs(root, exist_ok=True)
    c1 = synth.fep_solute(os.path.join(root, "c1"), seed=1234, steps=10000)
    systems = []
    for r in range(args.replicas):
        for lam in window_lambdas(args.windows):
            systems.append((c1.inp, lam, 1 + r + 1000 * rank, 2.0))
    rr = np.random.default_rng(4321 + rank)
    for k in range(args.spheres):
        R = float(rr.choice([15.0, 20.0, 25.0]))
        g = synth.water_sphere(os.path.join(root, "sph%02d" % k), radius=R, seed=1234 + 100 + k, steps=10000,
                               name="sph%02d" % k)
        systems.append((g.inp, None, 1 + k + 1000 * rank, 1.0))
    return systems


def config_files(root: str):
    """The plain single-system configurations (the three spheres and a
    periodic box at constant pressure): (name, inp, lambdas, dt_fs,
    description)."""
    from q_b200 import synth
    c0 = synth.water_sphere(os.path.join(root, "cfg_c0"), radius=15.0, seed=1234, steps=1000, name="c0")
    c1 = synth.fep_solute(os.path.join(root, "cfg_c1"), seed=1234, steps=5000)
    c2 = synth.polymer_sphere(os.path.join(root, "cfg_c2"), seed=1234, steps=5000)
    bx = synth.fep_box(os.path.join(root, "cfg_box"), edge=30.0, seed=1234, steps=5000, constant_pressure=True,
                       volume_change=25)
    return [("c0_water_sphere_15A", c0.inp, None, 1.0, "TIP3P sphere R 15 A, 1 fs, LRF, SHAKE, restraints"),
            ("c1_fep_solute_20A", c1.inp, (0.5, 0.5), 2.0,
             "56-atom solute, 8 two-state Q atoms (soft-core), lambda 0.5, 20 A TIP3P sphere, 2 fs"),
            ("c2_protein_ligand_25A", c2.inp, (0.5, 0.5), 2.0,
             "3000-atom polymer around the FEP solute, 25 A sphere, atoms beyond 23 A restrained, Q cut-off 99"),
            ("box_fep_solute_30A_npt", bx.inp, (0.5, 0.5), 2.0,
             "the FEP solute in a 30 A periodic TIP3P box, nearest images, LRF to 14 A, molecules put back "
             "in the box, Monte Carlo volume moves every 25 steps, 2 fs")]


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, which: str):
        setattr(self, which, time.time())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, margin: float = 0.3):
        """Samples that arrived while the timed steps ran (t0..t1), widened by
        `margin` seconds on either side, during which the GPU ran the same
        steps (a timed region of a few ms falls between two samples)."""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", 1e300)
        for ts, l in self.lines:
            if not (t0 - margin <= ts <= t1 + margin):
                continue
            f = [x.strip() for x in l.split(",")]
            if len(f) < 10:
                continue
            try:
                sm.append(float(f[2]))
                smax = float(f[3])
            except ValueError:
                continue
            for n, v in zip(names, f[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- step plans

def step_kinds(views, start: int, k: int) -> tuple[int, int]:
    """(pair-list rebuild steps, energy-evaluating steps) among steps
    start..start+k-1 of a run call: rebuilds where any system's non_bond
    interval divides the step, energies where any system records an output
    or energy-file record, and on the call's last step."""
    rebuild = energy = 0
    for i in range(k):
        s = start + i
        if any(s % v.NBcycle == 0 for v in views):
            rebuild += 1
        if i == k - 1 or any((v.iout_cycle > 0 and s % v.iout_cycle == 0) or
                             (v.iene_cycle > 0 and s > 0 and s % v.iene_cycle == 0) for v in views):
            energy += 1
    return rebuild, energy


def align_to_rebuild(batch, views) -> int:
    """Run the few steps up to the next pair-list rebuild; returns them."""
    nb = min(v.NBcycle for v in views)
    extra = (-batch.step_count()) % nb
    if extra:
        batch.run(extra)
    return extra


def prime_cycle_graphs(batch, views) -> None:
    """Untimed: replay every list-cycle pattern once so that the timed runs
    find their CUDA graphs captured.  A cycle's graph depends on which of its
    steps record energies (the phase of the step count against the output
    and energy-file intervals) and on whether it ends a run; one aligned run
    over twice the period of these intervals, then one single-cycle run at
    each phase, meets each pattern."""
    nb = min(v.NBcycle for v in views)
    period = nb
    for v in views:
        for c in (v.iout_cycle, v.iene_cycle):
            if c > 0:
                period = period * c // math.gcd(period, c)
    if period > 40 * nb:
        return
    align_to_rebuild(batch, views)
    batch.run(2 * period)
    for _ in range(period // nb):
        batch.run(nb)


def pair_interactions(w) -> float:
    """Atom-pair interactions of one step from the list totals: 9 per water-
    water molecule pair (md.f90:8276), solute-water and solute-solute atom
    pairs, Q-solute pairs x states, Q-water pairs x states x 3 sites."""
    return 9.0 * w[0] + w[1] + w[2] + w[3] + 3.0 * w[4]


# --------------------------------------------------------------- CPU side

def _oracle_worker(job, out):
    """The CPU oracle on some systems (spawned process, one thread): warm-up
    steps, a barrier, then the timed steps; puts (seconds, natoms) on out."""
    specs, steps, warm, barrier = job
    sys.path.insert(0, REPO)
    from q_b200 import System
    from tests.oracle_binding import load_oracle
    lib = load_oracle()
    runs = []
    natoms = 0
    for inp, lam, seed in specs:
        s = System.open(inp, lambdas=lam, seed=seed)
        runs.append((s, lib.create(s)))
        natoms += s.natom
    for _, o in runs:
        if warm:
            o.run(warm)
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    for _, o in runs:
        o.run(steps)
    out.put((time.perf_counter() - t0, natoms))


def oracle_batch(systems, steps: int, warm: int, workers: int):
    """The oracle stepping every system of the batch `steps` steps, systems
    spread over `workers` processes by atom count (one thread each); wall
    time is the slowest worker's, timed after a common barrier."""
    from q_b200 import System
    from q_b200.dist import shard
    natom = []
    for inp, lam, seed, dt in systems:
        s = System.open(inp, lambdas=lam, seed=seed)
        natom.append(s.natom)
        s.close()
    workers = max(1, min(workers, len(systems)))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(workers)
    q = ctx.Queue()
    procs = []
    for r in range(workers):
        mine = shard(len(systems), r, workers, natom)
        job = ([(systems[i][0], systems[i][1], systems[i][2]) for i in mine], steps, warm, barrier)
        procs.append(ctx.Process(target=_oracle_worker, args=(job, q)))
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    return max(r[0] for r in res), sum(r[1] for r in res)


def cpu_sample(systems, budget_steps: int = 25):
    """The oracle on one core over a bounded sample: one system of each shape
    (the FEP window and one water sphere per size), one pair-list cycle each,
    scaled to the batch by the shape counts.  Returns (ns/day, description)."""
    shapes = {}
    for inp, lam, seed, dt in systems:
        key = (lam is None, inp if lam is not None else os.path.getsize(inp.replace(".inp", ".top")) // 20000)
        if key not in shapes:
            shapes[key] = [inp, lam, seed, dt, 0]
        shapes[key][4] += 1
    per_step, sim_fs = 0.0, 0.0
    for inp, lam, seed, dt, cnt in shapes.values():
        sec, _ = oracle_batch([(inp, lam, seed, dt)], budget_steps, 0, 1)
        per_step += cnt * sec / budget_steps
        sim_fs += cnt * dt
    ns_day = sim_fs * 1e-6 / per_step * 86400
    desc = ("CPU oracle (C, FP64), one thread, on %d representative systems x %d steps (one pair-list cycle), "
            "scaled to the %d-system batch by shape counts" % (len(shapes), budget_steps, len(systems)))
    return ns_day, desc


def run_reference(args, rank, world):
    """--impl reference: the CPU oracle steps the actual batch on every host core."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    root = os.path.join(tempfile.gettempdir(), "qb_bench_inputs")
    systems = workload_files(root, 0, args)
    steps = args.steps
    # warm-up rounded up to whole pair-list cycles: the timed steps start on a
    # rebuild step, as the GPU arm's do
    nb = 25
    warm = -(-max(args.warmup, 0) // nb) * nb
    sec, natoms = oracle_batch(systems, steps, warm, threads)
    sim_ns = sum(dt for _, _, _, dt in systems) * steps * 1e-6
    value = sim_ns / sec * 86400.0
    sample = ("measured: CPU oracle (C, FP64 restatement of qdyn's step; Fortran qdyn cannot be compiled on this "
              "image) stepping all %d systems (%d atoms) of the batch for %d steps after %d warm-up steps (the "
              "timed steps start on a pair-list rebuild, non_bond 25), one process per core on %d cores, systems "
              "spread by atom count, wall time of the slowest process" % (len(systems), natoms, steps, warm, threads))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "ms_per_step": sec / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "systems": len(systems), "atoms": natoms},
        "cpu_baseline": {"value": value, "unit": "ns/day", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU side

def per_config_lines(root: str, device: int, steps: int = 200):
    """ns/day, pair interactions/s and the top kernel of each plain single-
    system configuration (FP64, one system per batch), beside the oracle on
    one core for one pair-list cycle of the same system."""
    from q_b200 import FP64, Batch, System
    from q_b200.api import peak_tflops
    out = {}
    peak64 = peak_tflops(FP64, device)
    for name, inp, lam, dt, desc in config_files(root):
        s = System.open(inp, lambdas=lam, seed=11)
        b = Batch([s], precision=FP64, device=device)
        b.run(50)
        # record capacity and graphs of the timed run first (growing the
        # records inside it would drop and recapture the step graphs)
        b.run(steps)
        b.clear_history()
        prime_cycle_graphs(b, [s.view])
        b.clear_history()
        align_to_rebuild(b, [s.view])
        # the same steps untimed right before the timed ones: a single system
        # runs for milliseconds, within the GPU's clock ramp after the host
        # pauses of the preparation
        nb = s.view.NBcycle
        b.run(-(-steps // nb) * nb)
        b.clear_history()
        start = b.step_count()
        ms, launches = b.run_timed(steps)
        rebuild, energy = step_kinds([s.view], start, steps)
        w = b.workload()
        b.set_profiling(True)
        b.run(steps)
        prof = b.profile()
        b.set_profiling(False)
        tot = sum(v[0] for v in prof.values()) or 1.0
        top = max(prof.items(), key=lambda kv: kv[1][0])
        ww = prof.get("nb_ww", (0.0, 1))
        ww_ms = ww[0] / max(ww[1], 1)
        per_step = ms / steps
        line = {"description": desc, "precision": "fp64", "atoms": s.natom, "dt_fs": dt,
                "ns_per_day": dt * 1e-6 / (per_step * 1e-3) * 86400.0, "ms_per_step": per_step,
                "pair_interactions_per_s": pair_interactions(w) / (per_step * 1e-3),
                "pair_interactions_per_step": pair_interactions(w), "steps": steps,
                "rebuild_steps_in_timed_region": rebuild, "energy_steps_in_timed_region": energy,
                "gpu_launches": launches,
                "top_kernel": top[0], "top_kernel_share": top[1][0] / tot,
                "kernels_ms_per_step": {k: round(v[0] / steps, 5) for k, v in
                                        sorted(prof.items(), key=lambda kv: -kv[1][0])[:6]}}
        if w[0] > 0 and ww_ms > 0:
            ach = FLOP_WW * w[0] / (ww_ms * 1e-3) / 1e12
            line["roofline_nb_ww"] = {"bound": "fp64", "achieved": ach, "peak": peak64, "unit": "TFLOP/s",
                                      "frac": ach / peak64, "launch_ms": ww_ms,
                                      "peak_source": "measured FP64 FMA loop (qb_peak_flops)"}
        b.close()
        sec, _ = oracle_batch([(inp, lam, 11, dt)], 25, 0, 1)
        line["cpu_oracle_1core_ns_per_day"] = dt * 1e-6 / (sec / 25) * 86400.0
        out[name] = line
        s.close()
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_
        dist = dist_
        if args.impl == "qb":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.destroy_process_group()
        return

    import numpy as np
    import torch

    from q_b200 import FP64, MIXED, Batch, System
    from q_b200.api import peak_tflops
    from q_b200.dist import max_over_ranks

    dev = "cuda:%d" % local
    prec = FP64 if args.precision == "fp64" else MIXED
    root = os.path.join(tempfile.gettempdir(), "qb_bench_inputs_r%d" % rank)
    t0 = time.perf_counter()
    specs = workload_files(root, rank, args)
    systems = [System.open(inp, lambdas=lam, seed=seed) for inp, lam, seed, dt in specs]
    views = [s.view for s in systems]
    setup_s = time.perf_counter() - t0
    dts = np.array([dt for _, _, _, dt in specs])
    natoms = sum(s.natom for s in systems)
    batch = Batch(systems, precision=prec, device=local)
    # untimed equilibration from the lattice start, the autotuner (its trial
    # steps are equilibration too), then warm-up
    batch.run(args.equil)
    tuning = batch.autotune(50) if not args.no_autotune else batch.tuning()
    batch.run(max(args.warmup, 3))
    # the energy-record capacity of a timed run (growing it would drop the
    # step graphs), then every list-cycle graph captured
    batch.run(max(args.steps, 1))
    batch.clear_history()
    prime_cycle_graphs(batch, views)
    batch.clear_history()

    def barrier():
        if dist:
            dist.barrier()

    barrier()
    torch.cuda.synchronize(local)
    with ClockSampler(local) as clk:
        # keep the GPU stepping until the sampler reports (nvidia-smi takes a
        # moment to start), then time; a few more steps after the timed ones
        # keep it under the same load for the samples just after them
        t_wait = time.time()
        batch.run(20)
        while len(clk.lines) < 3 and time.time() - t_wait < 5.0:
            batch.run(25)
        align_to_rebuild(batch, views)
        # no record growth inside the timed region (it would drop the graphs)
        batch.clear_history()
        start = batch.step_count()
        clk.mark("t0")
        ms, launches = batch.run_timed(args.steps)
        clk.mark("t1")
        t_after = time.time()
        while time.time() - t_after < 0.3:
            batch.run(25)
        batch.clear_history()
    barrier()
    rebuild, energy = step_kinds(views, start, args.steps)
    elapsed = max_over_ranks(ms / 1e3, dev)
    sim_ns = float(dts.sum()) * args.steps * 1e-6 * world
    value = sim_ns / elapsed * 86400.0
    w = batch.workload()
    pairs_step = pair_interactions(w)

    # whole pair-list cycles, for comparison with the K-step figure
    ncyc = 4 * min(v.NBcycle for v in views)
    align_to_rebuild(batch, views)
    batch.clear_history()
    ms_cyc, _ = batch.run_timed(ncyc)
    ms_cyc = max_over_ranks(ms_cyc, dev)

    # per-kernel device times: a separate profiled pass (one kernel at a time,
    # one stream) over the same step kinds
    align_to_rebuild(batch, views)
    batch.set_profiling(True)
    batch.run(args.steps)
    prof = batch.profile()
    batch.set_profiling(False)
    tot = sum(v[0] for v in prof.values()) or 1.0
    top = max(prof.items(), key=lambda kv: kv[1][0])
    kname = "nb_ww_x2" if "nb_ww_x2" in prof else "nb_ww"
    kk = prof.get(kname, (0.0, 1))
    k_ms = kk[0] / max(kk[1], 1)
    ww_flop = FLOP_WW * w[0]
    peak = peak_tflops(FP64 if prec == FP64 else MIXED, local)
    traffic = None
    try:
        tj = json.load(open(os.path.join(REPO, "profiles", "traffic.json")))
        traffic = tj.get(kname, {}).get("bytes_per_launch")
    except (OSError, ValueError):
        pass
    achieved = ww_flop / (k_ms * 1e-3) / 1e12 if k_ms > 0 else 0.0

    # end to end through the C ABI with host buffers: every system's
    # coordinates and velocities up, the steps, every system's records and
    # coordinates down; three repetitions, the median reported
    # the host buffers page-locked (torch's pinned allocator), as a serving
    # host keeps them
    def pinned(n):
        return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()

    x0, v0, xout = pinned(3 * natoms), pinned(3 * natoms), pinned(3 * natoms)
    batch.coords_all(x0)
    batch.velocities_all(v0)
    h2d = 2 * 24 * natoms                   # coordinates and velocities, x y z per atom
    # records a run of --steps steps can hold: output and energy-file intervals
    max_rec = [args.steps // max(1, min(v.iout_cycle for v in views)) + 2,
               args.steps // max(1, min(v.iene_cycle for v in views)) + 2]
    from q_b200.api import HIST_REC
    recbuf = [pinned(len(views) * m * HIST_REC) for m in max_rec]
    reps = []
    for _ in range(3):
        barrier()
        t0 = time.perf_counter()
        batch.set_coords_all(x0)
        batch.set_velocities_all(v0)
        t1 = time.perf_counter()
        batch.run(args.steps)
        t2 = time.perf_counter()
        d2h = 0
        for kind in (0, 1):
            counts, rec, nbytes = batch.history_all(kind, max_records=max_rec[kind], with_bytes=True,
                                                    out=recbuf[kind])
            d2h += nbytes
        batch.coords_all(xout)
        d2h += 24 * natoms                  # x y z per atom
        batch.clear_history()
        t3 = time.perf_counter()
        reps.append((t3 - t0, t1 - t0, t2 - t1, t3 - t2))
    reps.sort()
    te, e2e_up, e2e_run, e2e_down = reps[1]
    te = max_over_ranks(te, dev)
    e2e = sim_ns / te * 86400.0

    cpu = None
    per_config = None
    if rank == 0 and world == 1:
        if not args.no_cpu_baseline:
            ns_1core, desc = cpu_sample(specs)
            cpu = {"value": ns_1core, "unit": "ns/day", "cores": 1, "kind": "port", "sample": desc}
        if not args.no_configs:
            per_config = per_config_lines(root, local)

    line = {
        "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == FP64 else ("f32 water-water forces (packed FP32x2) on non-recording steps; f64 "
                                             "energies, water-water pairs on recording steps, Q terms, LRF "
                                             "expansion, SHAKE, update"),
        "data": "synthetic (seeded generator of the benchmark shapes)",
        "config": {"workload": WORKLOAD, "systems": len(systems), "atoms": natoms,
                   "precision": args.precision, "equilibration_steps": args.equil,
                   "l2": "per-step working set (coordinates, velocities, gradients, pair lists) exceeds the 126 MB L2",
                   "parallelism": "replicas only (%d GPU, whole systems per GPU)" % world,
                   "c1_charges": "solute charges with hydrogens at +0.10 +- 0.04 and heavy atoms N(0, 0.35) "
                                 "balancing to net 0 (the config's N(0, 0.3) on every atom bound water H to "
                                 "solute H and failed SHAKE; see DESIGN)",
                   "setup_s": round(setup_s, 2),
                   "tuning": {k: (round(v, 5) if isinstance(v, float) else v) for k, v in tuning.items()}},
        "timed_region": {"first_step": start, "rebuild_steps_in_timed_region": rebuild,
                         "energy_steps_in_timed_region": energy,
                         "ms_per_step_whole_list_cycles": ms_cyc / ncyc, "whole_cycle_steps": ncyc},
        "pair_interactions_per_s": pairs_step * args.steps * world / elapsed,
        "pair_interactions_per_step": pairs_step,
        "roofline": {"kernel": kname + " (water-water SPC forces)", "bound": "fp64" if prec == FP64 else "fp32",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "peak_source": "measured FMA loop (qb_peak_flops) on this GPU, of measured",
                     "flop_per_launch": ww_flop, "flop_basis": "229 FLOP x unique water-water molecule pairs",
                     "launch_ms": k_ms, "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/traffic.json",
                     "share_of_step": kk[0] / tot,
                     "top_kernel": top[0], "top_kernel_share": top[1][0] / tot},
        "kernels_ms_per_step": {k: round(v[0] / args.steps, 5) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
        "workload_per_step": {"ww_molecule_pairs": w[0], "pw_pairs": w[1], "pp_pairs": w[2],
                              "qp_pairs_x_states": w[3], "qw_pairs_x_states": w[4],
                              "shake_iterations_mean": round(float(w[8]), 3), "shake_iterations_max": int(w[9])},
        "e2e": {"value": e2e, "unit": "ns/day", "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps, "repetitions": 3, "statistic": "median",
                "phases_s": {"upload": round(e2e_up, 4), "run": round(e2e_run, 4), "read_back": round(e2e_down, 4)}},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if cpu:
        line["cpu_baseline"] = cpu
    if per_config:
        line["per_config"] = per_config
    batch.close()
    if rank == 0 and world == 1 and args.dg_replicas > 0:
        # second half of the metric: device seconds per dG, batched mixed
        # precision against the plain FP64 engine one system per launch,
        # the dG error judged by a dense-window FP64 run
        from q_b200.campaign import dg_versus_plain
        placement = None
        if args.dg_placement == "learned":
            from q_b200.lambda_placement import Placement
            placement = Placement.load(os.path.join(REPO, "q_b200", "data", "placement_model.npz"))
        t0 = time.perf_counter()
        dg = dg_versus_plain(specs[0][0], windows=args.windows, replicas=args.dg_replicas,
                             ref_windows=args.dg_ref_windows, ref_replicas=args.dg_ref_replicas,
                             steps_eq=args.dg_equil, steps_prod=args.dg_steps, device=local, placement=placement)
        dg["wall_s"] = round(time.perf_counter() - t0, 1)
        line["dG"] = dg
        line["gpu_s_per_dG"] = {"batched_mixed": dg["batched_mixed"]["gpu_seconds"],
                                "plain_fp64": dg["plain_fp64_one_system_per_launch"]["gpu_seconds"],
                                "ratio": dg["gpu_seconds_ratio_plain_over_batched"],
                                "dG_error_vs_fp64_dense": dg["dG_error"], "dG_error_sem": dg["dG_error_sem"],
                                "placement": dg["perturbation"]["placement"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
