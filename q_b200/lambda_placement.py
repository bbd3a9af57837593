"""Learned placement of lambda windows for a perturbation.

QligFEP spaces a perturbation's windows by a fixed schedule (get_lambdas,
src/QligFEP/qligfep.py:414-445: sigmoidal by default, or linear).  Here a
coarse pilot run of the perturbation (5 windows, one short replica, on the
batched engine) is summarised in 12 features, and a small network run on the
tensor cores (q_b200/mlp.py) maps them to the spacing of 12 windows.

Windows are written as u = weight of state 2 (window (1 - u, u)), from u = 0
to u = 1.  With linear coupling V(u) = (1 - u) V1 + u V2 the energy
difference between two windows is (u' - u) * dU, dU = V2 - V1 sampled at u.
The BAR variance of a narrow interval grows as ((u' - u) sigma(u))^2, sigma(u)
the standard deviation of dU at u, so the summed variance is smallest when
every interval carries the same increment of the thermodynamic length
L(u) = integral of sigma.  The training target of a perturbation is that
spacing, computed from a dense 21-window profile of sigma, written as the
centred logarithms of its 11 spacings (softmax gives the spacings back).  The
pilot already gives sigma at 5 points, whose interpolated length spacing is
the placement without a network; the network's 11 outputs are a correction
to that spacing's logarithms, and its output layer starts at zero, so an
untrained or strongly regularised network returns the pilot spacing.
Uniform spacing is the fallback when no model is given.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass, field

import numpy as np

from .api import FP64, MIXED, Batch

KT = 0.592                                  # kcal/mol at 298 K
PILOT_U = (0.0, 0.25, 0.5, 0.75, 1.0)
DENSE_U = tuple(k / 20 for k in range(21))
N_PLACED = 12                               # windows placed by the network
N_FEATURES = 12


# ------------------------------------------------------------------ schedules

def uniform(n: int) -> np.ndarray:
    return np.linspace(0.0, 1.0, n)


def qligfep_schedule(windows: int, sampling: str = "sigmoidal") -> np.ndarray:
    """QligFEP's get_lambdas (qligfep.py:414-445) with sigmoid(t, k) =
    k t / (k - t + 1) (functions.py:7), as values of u ascending.  The
    sigmoidal schedule has 2*(windows//2) + 1 windows, denser at both ends;
    values are rounded to 3 decimals as the reference formats them."""
    k = {"sigmoidal": -1.1, "linear": 1000.0, "exponential": -1.1, "reverse_exponential": 1.1}[sampling]

    def sig(t):
        return k * t / (k - t + 1.0)

    if sampling == "sigmoidal":
        step = int(windows / 2)
        hi = [round(0.5 * (sig(i / step) + 1.0), 3) for i in range(step + 1)]
        lo = [round(0.5 * (-sig(i / step) + 1.0), 3) for i in range(step + 1)][1:]
        lam1 = list(reversed(lo)) + hi              # ascending lambda_1
    else:
        lam1 = [round(sig(i / windows), 3) for i in range(windows + 1)]
    lam1 = lam1[::-1]                               # descending, as QligFEP writes them
    return np.array([1.0 - l for l in lam1])       # u = 1 - lambda_1, ascending


def windows_of(u) -> list[tuple[float, float]]:
    return [(1.0 - float(x), float(x)) for x in u]


def length_spacing(u_profile, sigma, n: int = N_PLACED) -> np.ndarray:
    """n windows (u from 0 to 1) at equal increments of the thermodynamic
    length of the piecewise-linear sigma(u) profile."""
    u_profile = np.asarray(u_profile, dtype=np.float64)
    s = np.maximum(np.asarray(sigma, dtype=np.float64), 1e-3 * KT)
    seg = 0.5 * (s[1:] + s[:-1]) * np.diff(u_profile)
    L = np.concatenate([[0.0], np.cumsum(seg)])
    targets = np.linspace(0.0, L[-1], n)
    out = np.empty(n)
    for i, Lt in enumerate(targets):
        j = min(np.searchsorted(L, Lt, side="right") - 1, len(seg) - 1)
        j = max(j, 0)
        # inside segment j, L grows quadratically when sigma is linear in u
        u0, h = u_profile[j], u_profile[j + 1] - u_profile[j]
        a = 0.5 * (s[j + 1] - s[j]) / h
        b = s[j]
        c = -(Lt - L[j])
        if abs(a) < 1e-12:
            du = -c / b
        else:
            du = (-b + np.sqrt(max(b * b - 4 * a * c, 0.0))) / (2 * a)
        out[i] = u0 + min(max(du, 0.0), h)
    out[0], out[-1] = 0.0, 1.0
    return np.maximum.accumulate(out)


def spacing_logits(u) -> np.ndarray:
    """Centred log-spacings of a schedule (the network's target)."""
    g = np.maximum(np.diff(np.asarray(u, dtype=np.float64)), 1e-6)
    lg = np.log(g)
    return lg - lg.mean()


def positions_from_logits(y) -> np.ndarray:
    y = np.asarray(y, dtype=np.float64)
    g = np.exp(y - y.max())
    g /= g.sum()
    u = np.concatenate([[0.0], np.cumsum(g)])
    u[-1] = 1.0
    return u


# ------------------------------------------------------------------ features

def _logmeanexp(a):
    m = a.max()
    return m + np.log(np.mean(np.exp(a - m)))


def pilot_features(dU, u=PILOT_U, kT: float = KT) -> np.ndarray:
    """12 features of a pilot: dU[w] = series of V2 - V1 at pilot window w.
    0-4: log sigma_w, centred; 5-9: <dU>_w, centred, over (mean sigma + kT);
    10: mean log(sigma/kT) / 3; 11: mean forward/reverse Zwanzig hysteresis
    of the pilot intervals, |dGf - dGr| / (|dGf| + |dGr| + kT)."""
    dU = [np.asarray(d, dtype=np.float64) for d in dU]
    m = np.array([d.mean() for d in dU])
    s = np.array([max(d.std(), 1e-3 * kT) for d in dU])
    ls = np.log(s / kT)
    f = np.empty(N_FEATURES)
    f[0:5] = ls - ls.mean()
    f[5:10] = (m - m.mean()) / (s.mean() + kT)
    f[10] = ls.mean() / 3.0
    hyst = []
    for k in range(len(u) - 1):
        du = u[k + 1] - u[k]
        dgf = -kT * _logmeanexp(-du * dU[k] / kT)
        dgr = kT * _logmeanexp(du * dU[k + 1] / kT)
        hyst.append(abs(dgf - dgr) / (abs(dgf) + abs(dgr) + kT))
    f[11] = float(np.mean(hyst))
    return f


# ------------------------------------------------------------------ model

@dataclass
class Placement:
    """The trained network and its feature normalisation."""
    params: np.ndarray
    fmean: np.ndarray
    fstd: np.ndarray
    loss: np.ndarray = field(default_factory=lambda: np.zeros(0))
    selection: dict = field(default_factory=dict)

    def predict_logits(self, features, device: int = 0) -> np.ndarray:
        from . import mlp
        F = np.atleast_2d(features)
        x = (F - self.fmean) / self.fstd
        base = np.array([spacing_logits(pilot_spacing(f)) for f in F])
        return base + mlp.forward(self.params, x.astype(np.float32), device).astype(np.float64)

    def predict(self, features, device: int = 0) -> list[np.ndarray]:
        return [positions_from_logits(y) for y in self.predict_logits(features, device)]

    def save(self, path: str) -> None:
        np.savez(path, params=self.params, fmean=self.fmean, fstd=self.fstd, loss=self.loss)

    @classmethod
    def load(cls, path: str) -> "Placement":
        d = np.load(path)
        return cls(d["params"], d["fmean"], d["fstd"], d["loss"])


def fit(features, targets, iters: int | None = None, lr: float = 2e-3, weight_decay: float = 0.0, seed: int = 0,
        device: int = 0, val_frac: float = 0.2, grid_iters=(50, 100, 200, 400, 800, 1600, 3200),
        grid_decay=(0.0, 0.01, 0.1)) -> Placement:
    """Train the network (full-batch AdamW on the tensor cores).  With iters
    None the number of steps and the weight decay are chosen on a held-back
    validation fraction of the samples (smallest validation error over the
    grid), then the network is trained on all samples with that choice."""
    from . import mlp
    X = np.asarray(features, dtype=np.float64)
    base = np.array([spacing_logits(pilot_spacing(f)) for f in X])
    T = (np.asarray(targets, dtype=np.float64) - base).astype(np.float32)     # correction to the pilot spacing
    fmean, fstd = X.mean(0), X.std(0) + 1e-6
    Xn = ((X - fmean) / fstd).astype(np.float32)
    selection = {}
    if iters is None:
        perm = np.random.default_rng(seed).permutation(len(X))
        nv = max(1, int(round(val_frac * len(X))))
        va, tr = perm[:nv], perm[nv:]
        table = []
        for wd in grid_decay:
            for it in grid_iters:
                p, _ = mlp.train(mlp.init(seed, True), Xn[tr], T[tr], it, lr=lr, weight_decay=wd, device=device)
                err = float(np.mean((mlp.forward(p, Xn[va], device) - T[va]) ** 2))
                table.append((err, it, wd))
        err, iters, weight_decay = min(table)
        selection = {"validation_mse": err, "iters": iters, "weight_decay": weight_decay,
                     "validation_mse_pilot": float(np.mean(T[va] ** 2)),
                     "grid": [{"iters": it, "weight_decay": wd, "validation_mse": e} for e, it, wd in table]}
    p, hist = mlp.train(mlp.init(seed, True), Xn, T, iters, lr=lr, weight_decay=weight_decay, device=device)
    return Placement(p, fmean, fstd, hist, selection)


def pilot_spacing(features, n: int = N_PLACED) -> np.ndarray:
    """The length spacing of the pilot's own 5-point sigma profile (the
    features hold it exactly: sigma_w = kT exp(f_w + 3 f_10)): the placement a
    pilot gives without the network."""
    f = np.asarray(features, dtype=np.float64)
    return length_spacing(PILOT_U, KT * np.exp(f[0:5] + 3.0 * f[10]), n)


def place(features, model: Placement | None = None, device: int = 0) -> np.ndarray:
    """The schedule for one perturbation: the model's, or uniform without one."""
    if model is None:
        return uniform(N_PLACED)
    return model.predict(features, device)[0]


def structured_profiles(n: int, seed: int = 0, samples: int = 200):
    """Pilot features and exact targets of n synthetic sigma(u) profiles with
    structure the pilot under-resolves: a level in [0.5, 10] kcal/mol, a tilt,
    and a Gaussian bump (height 0-6x, centre anywhere, width 0.05-0.3); the
    pilot sees `samples` normal draws of dU at each of its 5 windows.  A
    controlled benchmark of what the network adds to the pilot spacing."""
    rng = np.random.default_rng(seed)
    U = np.array(DENSE_U)
    F, T = np.empty((n, N_FEATURES)), np.empty((n, N_PLACED - 1))
    for i in range(n):
        level, tilt = rng.uniform(0.5, 10.0), rng.uniform(-0.8, 0.8)
        a, c, w = rng.uniform(0.0, 6.0), rng.uniform(0.0, 1.0), rng.uniform(0.05, 0.3)
        slope = level * 5.0 * rng.uniform(-1.0, 1.0)

        def sigma(u):
            return level * (1.0 + tilt * (u - 0.5) + a * np.exp(-((u - c) / w) ** 2))

        F[i] = pilot_features([rng.normal(slope * (1.0 - u), sigma(u), samples) for u in PILOT_U])
        T[i] = spacing_logits(length_spacing(U, sigma(U)))
    return F, T


# ------------------------------------------------------------------ sampling

@dataclass
class Perturbation:
    name: str
    inp: str
    qatoms: list
    charge_scale: float
    eps_scale: float


def make_perturbations(root: str, n: int, seed: int = 0, solute_seed: int = 1234, steps: int = 10000):
    """n random perturbations of the synthetic FEP solute: 4-12 of its heavy
    atoms become Q-atoms, state 2 scales their charges by c in [0, 1] and
    their epsilon by e in [0.3, 1] (soft-core in state 2).  One shared
    topology."""
    from . import synth
    base = synth.fep_solute(os.path.join(root, "solute"), seed=solute_seed, steps=steps)
    kinds = synth.solute_parameters(solute_seed)[0]
    heavy = [i for i, k in enumerate(kinds) if k >= 0]
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nq = int(rng.integers(4, 13))
        qatoms = sorted(int(a) for a in rng.choice(heavy, nq, replace=False))
        c, e = float(rng.uniform(0.0, 1.0)), float(rng.uniform(0.3, 1.0))
        g = synth.perturbation(base, "pert%04d" % i, qatoms, c, e, seed=solute_seed, steps=steps)
        out.append(Perturbation("pert%04d" % i, g.inp, qatoms, c, e))
    return base, out


@dataclass
class WindowRun:
    dU: list                 # per replica: per window the V2 - V1 series of the production records
    dG: list                 # per replica: BAR free energy over the windows
    gpu_seconds: float       # this job's share of the device time


def sample(jobs, *, replicas: int = 1, steps_eq: int = 500, steps_prod: int = 2000, precision: int = MIXED,
           seed0: int = 1, rt: float = KT, device: int = 0, max_systems: int = 2400, bar: bool = True):
    """Run every (job, replica, window) as one system, jobs = [(inp, u), ...],
    in batches of at most max_systems; returns one WindowRun per job.  Each
    job's device time is its systems' share of its batch's time (all systems
    of a batch step together)."""
    per_job = [len(u) * replicas for _, u in jobs]
    results = [None] * len(jobs)
    start = 0
    while start < len(jobs):
        stop, nsys = start, 0
        while stop < len(jobs) and (nsys == 0 or nsys + per_job[stop] <= max_systems):
            nsys += per_job[stop]
            stop += 1
        specs = []
        for j in range(start, stop):
            inp, u = jobs[j]
            for r in range(replicas):
                for w in windows_of(u):
                    specs.append((inp, w, seed0 + r))
        systems = _open(specs)
        batch = Batch(systems, precision=precision, device=device)
        try:
            ms = 0.0
            if steps_eq:
                ms += batch.run_timed(steps_eq)[0]
            batch.clear_history()
            ms += batch.run_timed(steps_prod)[0]
            k = 0
            for j in range(start, stop):
                nw = len(jobs[j][1])
                dU, dG = [], []
                for r in range(replicas):
                    series = []
                    for w in range(nw):
                        _, _, EQ = batch.history(k + w, 1)
                        series.append(EQ[:, 1, 1] - EQ[:, 0, 1])       # total of state 2 - state 1
                    dU.append(series)
                    if bar:
                        dG.append(batch.fep(list(range(k, k + nw)), rt, 0, nbins=10, nmin=1).dG_bar)
                    k += nw
                results[j] = WindowRun(dU, dG, ms / 1e3 * per_job[j] / nsys)
        finally:
            batch.close()
            for s in systems:
                s.close()
        start = stop
    return results


def _open(specs):
    from concurrent.futures import ThreadPoolExecutor
    from .api import System
    with ThreadPoolExecutor(min(len(specs), os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda sp: System.open(sp[0], lambdas=sp[1], seed=sp[2]), specs))


def training_data(perts, *, steps_eq: int = 500, steps_prod: int = 2000, device: int = 0) -> dict:
    """Pilot features and dense-profile targets of every perturbation (one
    replica each; pilot and dense profile from independent seeds)."""
    t0 = time.perf_counter()
    pilot = sample([(p.inp, np.array(PILOT_U)) for p in perts], steps_eq=steps_eq, steps_prod=steps_prod,
                   seed0=1, device=device, bar=False)
    dense = sample([(p.inp, np.array(DENSE_U)) for p in perts], steps_eq=steps_eq, steps_prod=steps_prod,
                   seed0=101, device=device, bar=False)
    F = np.array([pilot_features(r.dU[0]) for r in pilot])
    S = np.array([[max(np.std(d), 1e-3 * KT) for d in r.dU[0]] for r in dense])
    T = np.array([spacing_logits(length_spacing(DENSE_U, s)) for s in S])
    return {"features": F, "targets": T, "sigma_dense": S,
            "pilot_gpu_s": np.array([r.gpu_seconds for r in pilot]),
            "dense_gpu_s": np.array([r.gpu_seconds for r in dense]),
            "wall_s": time.perf_counter() - t0}


def evaluate(perts, features, model: Placement, *, replicas: int = 4, ref_replicas: int = 4, steps_eq: int = 1000,
             steps_prod: int = 5000, ref_windows: int = 41, device: int = 0) -> dict:
    """Free energies of held-out perturbations with each schedule (batched
    mixed precision) against a dense uniform FP64 reference.  Methods: the
    network's 12 windows, uniform 12, QligFEP sigmoidal 13, uniform 21; the
    pilot-interpolated length spacing (12) as the method without a network
    that uses the same pilot."""
    predicted = model.predict(features, device)
    methods = {
        "learned_12": predicted,
        "uniform_12": [uniform(12)] * len(perts),
        "qligfep_sigmoidal_13": [qligfep_schedule(12)] * len(perts),
        "uniform_21": [uniform(21)] * len(perts),
        "pilot_length_12": [pilot_spacing(f) for f in features],
    }
    out = {"methods": {}, "perturbations": [p.name for p in perts]}
    runs = {}
    for name, scheds in methods.items():
        runs[name] = sample([(p.inp, u) for p, u in zip(perts, scheds)], replicas=replicas, steps_eq=steps_eq,
                            steps_prod=steps_prod, seed0=1001, device=device)
    ref = sample([(p.inp, uniform(ref_windows)) for p in perts], replicas=ref_replicas, steps_eq=steps_eq,
                 steps_prod=steps_prod, precision=FP64, seed0=5001, device=device)
    ref_dG = np.array([np.mean(r.dG) for r in ref])
    ref_sem = np.array([np.std(r.dG, ddof=1) / np.sqrt(len(r.dG)) for r in ref])
    out["reference"] = {"windows": ref_windows, "replicas": ref_replicas, "dG": ref_dG.tolist(),
                        "sem": ref_sem.tolist(), "gpu_s": float(sum(r.gpu_seconds for r in ref))}
    for name, rs in runs.items():
        dG = np.array([np.mean(r.dG) for r in rs])
        sem = np.array([np.std(r.dG, ddof=1) / np.sqrt(len(r.dG)) for r in rs])
        err = dG - ref_dG
        out["methods"][name] = {
            "windows": int(len(methods[name][0])), "dG": dG.tolist(), "sem": sem.tolist(),
            "rms_error": float(np.sqrt(np.mean(err ** 2))), "mean_abs_error": float(np.mean(np.abs(err))),
            "rms_sem": float(np.sqrt(np.mean(sem ** 2))), "gpu_s": float(sum(r.gpu_seconds for r in rs)),
        }
    return out


# ------------------------------------------------------------------ study

def study(root: str, *, n_train: int = 200, n_test: int = 50, seed: int = 0, iters: int | None = None,
          replicas: int = 4, ref_replicas: int = 4, steps_eq: int = 1000, steps_prod: int = 5000,
          device: int = 0, data_file: str | None = None, run_dG: bool = True) -> dict:
    """Generate n_train + n_test perturbations, their pilot features and
    dense-profile targets, train the network on the first n_train, and
    evaluate every schedule on the held-out n_test against the dense FP64
    reference."""
    t0 = time.perf_counter()
    _, perts = make_perturbations(root, n_train + n_test, seed=seed)
    data_path = os.path.join(root, "placement_data.npz")
    if data_file and os.path.exists(data_file):
        d = np.load(data_file)
        data = {k: d[k] for k in d.files}
        data["wall_s"] = float(data["wall_s"])
    else:
        data = training_data(perts, device=device)
    np.savez(data_path, **data)
    F, T = data["features"], data["targets"]
    model = fit(F[:n_train], T[:n_train], iters=iters, device=device)
    model.save(os.path.join(root, "placement_model.npz"))
    Ft, Tt = F[n_train:], T[n_train:]
    pred = model.predict_logits(Ft, device)
    Fs, Ts = structured_profiles(2400, seed=seed + 1)
    ms = fit(Fs[:2000], Ts[:2000], device=device)
    ps = ms.predict_logits(Fs[2000:], device)
    structured = {"learned": float(np.mean((ps - Ts[2000:]) ** 2)),
                  "pilot_length": float(np.mean((np.array([spacing_logits(pilot_spacing(f)) for f in Fs[2000:]])
                                                 - Ts[2000:]) ** 2)),
                  "uniform": float(np.mean(Ts[2000:] ** 2)),
                  "selection": {k: v for k, v in ms.selection.items() if k != "grid"}}
    target_mse = {
        "structured_profiles_held_out": structured,
        "learned": float(np.mean((pred - Tt) ** 2)),
        "pilot_length": float(np.mean((np.array([spacing_logits(pilot_spacing(f)) for f in Ft]) - Tt) ** 2)),
        "uniform": float(np.mean(Tt ** 2)),
        "train_final_loss": float(model.loss[-1]),
    }
    target_mse["selection"] = {k: v for k, v in model.selection.items() if k != "grid"}
    ev = evaluate(perts[n_train:], Ft, model, replicas=replicas, ref_replicas=ref_replicas, steps_eq=steps_eq,
                  steps_prod=steps_prod, device=device) if run_dG else {"methods": {}, "reference": {}}
    ev["target_mse_held_out"] = target_mse
    ev["selection_grid"] = model.selection.get("grid", [])
    ev["data"] = {"n_train": n_train, "n_test": n_test, "pilot_gpu_s_mean": float(data["pilot_gpu_s"].mean()),
                  "dense_gpu_s_mean": float(data["dense_gpu_s"].mean()), "generation_wall_s": data["wall_s"]}
    ev["protocol"] = {"steps_eq": steps_eq, "steps_prod": steps_prod, "replicas": replicas,
                      "ref_replicas": ref_replicas, "iters": iters}
    ev["wall_s"] = time.perf_counter() - t0
    return ev


def main(argv=None) -> int:
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train and evaluate the lambda-placement network")
    ap.add_argument("root")
    ap.add_argument("--out", default=None)
    ap.add_argument("--train", type=int, default=200)
    ap.add_argument("--test", type=int, default=50)
    ap.add_argument("--replicas", type=int, default=4)
    ap.add_argument("--ref-replicas", type=int, default=4)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--iters", type=int, default=None, help="Adam steps (default: chosen on a validation split)")
    ap.add_argument("--data", default=None, help="reuse features/targets saved by an earlier study (npz)")
    ap.add_argument("--no-dG", action="store_true", help="stop after training (no free-energy evaluation)")
    a = ap.parse_args(argv)
    r = study(a.root, n_train=a.train, n_test=a.test, replicas=a.replicas, ref_replicas=a.ref_replicas,
              steps_prod=a.steps, iters=a.iters, data_file=a.data, run_dG=not a.no_dG)
    summary = {k: r[k] for k in ("target_mse_held_out", "data", "protocol", "wall_s")}
    summary["reference"] = {k: r["reference"][k] for k in ("windows", "replicas", "gpu_s") if k in r["reference"]}
    summary["methods"] = {m: {k: v for k, v in d.items() if k not in ("dG", "sem")} for m, d in r["methods"].items()}
    print(json.dumps(summary, indent=1))
    if a.out:
        json.dump(r, open(a.out, "w"), indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
