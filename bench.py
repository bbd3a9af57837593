#!/usr/bin/env python
"""Throughput of the batched Q MD step on B200 (one JSON line on stdout).

Workload (one GPU): the batched FEP configuration -- 21 uniform lambda windows
x 4 seeded replicas of the 56-atom, 8-Q-atom FEP solute in a 20 A TIP3P sphere
(2 fs, SHAKE on X-H and water, 10 A cut-offs + LRF) plus 16 TIP3P spheres with
radii drawn from {15, 20, 25} A (1 fs), all stepped together in one batch.
Synthetic, seeded inputs of those shapes (q_b200/synth.py).

A step is one MD step of every system.  `value` is the aggregate simulated
ns/day over all systems and ranks with the state resident in HBM, timed with
CUDA events on the engine's stream; `e2e` is the same metric through the C ABI
with host buffers: coordinates and velocities uploaded, the steps run, energy
records and final coordinates read back, all inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl qb|reference]
                    [--precision fp64|mixed]

At one GPU the line also carries the second half of the metric (`dG`,
`gpu_s_per_dG`): the perturbation's BAR free energy from 21 uniform windows x
--dg-replicas replicas in one mixed-precision batch, its device seconds, the
plain FP64 engine's device seconds for the same windows, replicas and steps
run one system per launch (its per-step time measured here), and the error
against a dense 41-window FP64 run of the same perturbation.

Under torchrun each rank runs its own copy of the batch (weak scaling); time is
the maximum over ranks.  `--impl reference` times the CPU oracle (the
restatement of Q's Fortran step, which cannot be compiled here) on a bounded
sample of the same workload with every host core.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
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
FLOP_LJC = 37        # per LJ+Coulomb atom pair


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
    p.add_argument("--no-autotune", action="store_true", help="keep the default tile sizes and streams")
    p.add_argument("--dg-replicas", type=int, default=16,
                   help="replicas of the batched mixed-precision perturbation for the GPU-s per dG comparison "
                        "(0 skips it; runs at one GPU only)")
    p.add_argument("--dg-ref-replicas", type=int, default=16, help="replicas of the dense FP64 reference")
    p.add_argument("--dg-ref-windows", type=int, default=41)
    p.add_argument("--dg-equil", type=int, default=1000)
    p.add_argument("--dg-steps", type=int, default=10000, help="production steps per window")
    return p.parse_args()


def workload_files(root: str, rank: int, args):
    """Generate (or reuse) the Q input files of the batch; returns a list of
    (inp, lambdas, seed, dt_fs)."""
    from q_b200 import synth
    from q_b200.synth import window_lambdas
    os.makedirs(root, exist_ok=True)
    c1 = synth.fep_solute(os.path.join(root, "c1"), seed=1234, steps=10000)
    systems = []
    for r in range(args.replicas):
        for lam in window_lambdas(args.windows):
            systems.append((c1.inp, lam, 1 + r + 1000 * rank, 2.0))
    rng_radii = [15.0, 20.0, 25.0]
    import numpy as np
    rr = np.random.default_rng(4321 + rank)
    for k in range(args.spheres):
        R = float(rr.choice(rng_radii))
        g = synth.water_sphere(os.path.join(root, "sph%02d" % k), radius=R, seed=1234 + 100 + k, steps=10000,
                               name="sph%02d" % k)
        systems.append((g.inp, None, 1 + k + 1000 * rank, 1.0))
    return systems


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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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

    def summary(self):
        """Samples that arrived while the timed steps ran (t0..t1)."""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", 1e300)
        for ts, l in self.lines:
            if not (t0 <= ts <= t1 + 0.15):
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


def _oracle_worker(job):
    """CPU oracle on one system for a bounded number of steps (spawned process)."""
    inp, lam, seed, steps, equil = job
    sys.path.insert(0, REPO)
    from q_b200 import System
    from tests.oracle_binding import load_oracle
    s = System.open(inp, lambdas=lam, seed=seed)
    o = load_oracle().create(s)
    if equil:
        o.run(equil)
    t0 = time.perf_counter()
    o.run(steps)
    return time.perf_counter() - t0, s.natom


def cpu_sample(systems, threads: int, budget_steps: int = 25):
    """Time the oracle on a sample: one system of each shape (the FEP window
    and one water sphere per radius), one full pair-list cycle (25 steps) each,
    extrapolated to the whole batch.  Returns (ns/day on one core, wall
    seconds, description)."""
    shapes = {}
    for inp, lam, seed, dt in systems:
        key = open(inp).read().split("topology", 1)[0] if lam is None else inp
        natom_key = os.path.getsize(os.path.join(os.path.dirname(inp), [l.split()[1] for l in open(inp)
                                                                        if l.startswith("topology")][0]))
        key = (lam is None, natom_key // 20000)
        if key not in shapes:
            shapes[key] = [inp, lam, seed, dt, 0]
        shapes[key][4] += 1
    jobs = [(inp, lam, seed, budget_steps, 0) for inp, lam, seed, dt, cnt in shapes.values()]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(max(1, min(threads, len(jobs)))) as pool:
        res = pool.map(_oracle_worker, jobs)
    wall = time.perf_counter() - t0
    per_step = 0.0
    sim_fs = 0.0
    for (inp, lam, seed, dt, cnt), (sec, natom) in zip(shapes.values(), res):
        per_step += cnt * sec / budget_steps
        sim_fs += cnt * dt
    ns_day_1core = sim_fs * 1e-6 / per_step * 86400
    desc = ("CPU oracle (C, FP64) on %d representative systems x %d steps (one pair-list cycle), "
            "extrapolated to the %d-system batch" % (len(jobs), budget_steps, len(systems)))
    return ns_day_1core, wall, desc


def run_reference(args, rank, world):
    """--impl reference: the CPU oracle over a bounded sample with every host core."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    root = os.path.join(tempfile.gettempdir(), "qb_bench_inputs")
    systems = workload_files(root, 0, args)
    per_step_steps = 25
    # each timed step: a bounded sample of the batch spread over the cores;
    # throughput scaled to the whole batch on `threads` cores
    ns_1core, wall, desc = cpu_sample(systems, threads, budget_steps=per_step_steps)
    value = ns_1core * threads
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "systems": len(systems)},
        "cpu_baseline": {"value": value, "unit": "ns/day", "cores": threads, "kind": "port",
                         "sample": desc + "; Fortran qdyn cannot be compiled on this image (no Fortran compiler)"},
        "e2e": {"value": value, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_
        import datetime
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
    from q_b200 import FP64, MIXED, Batch, System
    from q_b200.api import peak_tflops

    prec = FP64 if args.precision == "fp64" else MIXED
    root = os.path.join(tempfile.gettempdir(), "qb_bench_inputs_r%d" % rank)
    t0 = time.perf_counter()
    specs = workload_files(root, rank, args)
    systems = [System.open(inp, lambdas=lam, seed=seed) for inp, lam, seed, dt in specs]
    setup_s = time.perf_counter() - t0
    dts = np.array([dt for _, _, _, dt in specs])
    natoms = sum(s.natom for s in systems)
    batch = Batch(systems, precision=prec, device=local)
    # untimed equilibration from the lattice start, the autotuner (its trial
    # steps are equilibration too), then warm-up
    batch.run(args.equil)
    tuning = batch.autotune(50) if not args.no_autotune else batch.tuning()
    batch.run(max(args.warmup, 3))
    batch.clear_history()

    def barrier():
        if dist:
            dist.barrier()

    import torch
    barrier()
    torch.cuda.synchronize(local) if torch.cuda.is_available() else None
    with ClockSampler(local) as clk:
        batch.run(max(args.warmup, 3) + 20)      # the sampler starts while the GPU is busy
        clk.mark("t0")
        ms, launches = batch.run_timed(args.steps)
        clk.mark("t1")
    barrier()
    elapsed = ms / 1e3
    if dist:
        t = torch.tensor([elapsed], device="cuda:%d" % local, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    sim_ns = float(dts.sum()) * args.steps * 1e-6 * world
    value = sim_ns / elapsed * 86400.0

    # workload totals of the current lists, for the roofline
    w = batch.workload()
    ww_pairs, pw_pairs, pp_pairs = w[0], w[1], w[2]

    # per-kernel device times (separate profiled pass of the same length)
    batch.set_profiling(True)
    batch.run(args.steps)
    prof = batch.profile()
    batch.set_profiling(False)
    tot = sum(v[0] for v in prof.values())
    top = max(prof.items(), key=lambda kv: kv[1][0])
    ww = prof.get("nb_ww", (0.0, 1))
    ww_ms = ww[0] / max(ww[1], 1)
    ww_flop = FLOP_WW * ww_pairs
    peak = peak_tflops(FP64 if prec == FP64 else MIXED, local)
    traffic = None
    try:
        tj = json.load(open(os.path.join(REPO, "profiles", "traffic.json")))
        traffic = tj.get(args.precision, {}).get("bytes_per_launch")
    except (OSError, ValueError):
        pass
    achieved = ww_flop / (ww_ms * 1e-3) / 1e12 if ww_ms > 0 else 0.0

    # end to end through the C ABI with host buffers: three repetitions, the
    # median reported, with its upload / run / read-back split
    xs = [batch.coords(k) for k in range(len(systems))]
    vs = [batch.velocities(k) for k in range(len(systems))]
    h2d = sum(x.nbytes + v.nbytes for x, v in zip(xs, vs))
    reps = []
    for _ in range(3):
        barrier()
        t0 = time.perf_counter()
        for k in range(len(systems)):
            batch.set_coords(k, xs[k])
            batch.set_velocities(k, vs[k])
        t1 = time.perf_counter()
        batch.run(args.steps)
        t2 = time.perf_counter()
        d2h = 0
        for k in range(len(systems)):
            st, E, EQ = batch.history(k, 0)
            x = batch.coords(k)
            d2h += E.nbytes + EQ.nbytes + st.nbytes + x.nbytes
        batch.clear_history()
        t3 = time.perf_counter()
        reps.append((t3 - t0, t1 - t0, t2 - t1, t3 - t2))
    reps.sort()
    te, e2e_up, e2e_run, e2e_down = reps[1]
    if dist:
        t = torch.tensor([te], device="cuda:%d" % local, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        te = float(t.item())
    e2e = sim_ns / te * 86400.0

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = 1
        ns_1core, wall, desc = cpu_sample(specs, threads=1, budget_steps=25)
        cpu = {"value": ns_1core, "unit": "ns/day", "cores": threads, "kind": "port",
               "sample": desc + "; single thread"}

    line = {
        "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == FP64 else "f32 pair math + f64 accumulation/LRF/SHAKE/update",
        "data": "synthetic (seeded generator of the benchmark shapes)",
        "config": {"workload": WORKLOAD, "systems": len(systems), "atoms": natoms,
                   "precision": args.precision, "equilibration_steps": args.equil,
                   "l2": "per-step working set (coordinates, velocities, gradients, pair lists) exceeds the 126 MB L2",
                   "parallelism": "replicas only (%d GPU, whole systems per GPU)" % world,
                   "setup_s": round(setup_s, 2),
                   "tuning": {k: (round(v, 5) if isinstance(v, float) else v) for k, v in tuning.items()}},
        "roofline": {"kernel": "nb_ww (water-water SPC pair kernel)", "bound": "fp64" if prec == FP64 else "fp32",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "peak_source": "measured FMA loop (qb_peak_flops) on this GPU",
                     "flop_per_launch": ww_flop, "launch_ms": ww_ms, "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/traffic.json",
                     "share_of_step": ww[0] / tot if tot else None,
                     "top_kernel": top[0], "top_kernel_share": top[1][0] / tot if tot else None},
        "kernels_ms_per_step": {k: round(v[0] / args.steps, 5) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
        "workload_per_step": {"ww_molecule_pairs": ww_pairs, "pw_pairs": pw_pairs, "pp_pairs": pp_pairs,
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
    batch.close()
    if rank == 0 and world == 1 and args.dg_replicas > 0:
        # second half of the metric: device seconds per dG, batched mixed
        # precision against the plain FP64 engine one system per launch,
        # the dG error judged by a dense-window FP64 run
        from q_b200.campaign import dg_versus_plain
        t0 = time.perf_counter()
        dg = dg_versus_plain(specs[0][0], windows=args.windows, replicas=args.dg_replicas,
                             ref_windows=args.dg_ref_windows, ref_replicas=args.dg_ref_replicas,
                             steps_eq=args.dg_equil, steps_prod=args.dg_steps, device=local)
        dg["wall_s"] = round(time.perf_counter() - t0, 1)
        line["dG"] = dg
        line["gpu_s_per_dG"] = {"batched_mixed": dg["batched_mixed"]["gpu_seconds"],
                                "plain_fp64": dg["plain_fp64_one_system_per_launch"]["gpu_seconds"],
                                "ratio": dg["gpu_seconds_ratio_plain_over_batched"],
                                "dG_error_vs_fp64_dense": dg["dG_error"], "dG_error_sem": dg["dG_error_sem"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
