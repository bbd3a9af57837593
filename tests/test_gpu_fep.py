"""Free-energy analysis on the GPU (qb_fep_analyze, qb_batch_fep) against the
qfep restatement (oracle/qfep_oracle.py), and the qfep drop-in end to end.
Results agree to summation order: the GPU reduces in a tree, qfep in
sequence."""
import io
import os

import numpy as np
import pytest

from oracle.qfep_oracle import FepInput
from oracle.qfep_oracle import analyze as oracle_analyze

pytestmark = pytest.mark.gpu
TOL = 1e-9


def random_series(nf, n, ns, seed, spread=0.8):
    rng = np.random.default_rng(seed)
    out = []
    lams = np.linspace(0.0, 1.0, nf)
    for k in range(nf):
        e = rng.normal(0.0, spread, (n + k, ns, 15))    # uneven lengths
        w = np.zeros(ns)
        w[0], w[-1] = 1.0 - lams[k], lams[k]
        e[:, :, 0] = w
        out.append(e)
    return out


def compare(r, o, nf):
    for name in ("dgf", "dgfsum", "dgr", "dgrsum", "dG", "dgti", "dgtisum", "dglu", "dglusum", "dgbar", "dgbarsum"):
        a, b = getattr(r, name), getattr(o, name)
        assert np.allclose(a, b, rtol=TOL, atol=TOL), (name, a, b)
    assert np.allclose(r.avEQ[:, :, 1:], o.avEQ[:, :, 1:], rtol=1e-12, atol=1e-12)
    assert np.allclose(r.gap_range, [o.gapmin, o.gapmax], rtol=1e-12, atol=1e-12)
    assert list(r.bar_iterations[1:nf]) == list(o.bar_iterations)
    rows = [(f, ib) for f in range(nf) for ib in range(r.part2.shape[1]) if r.part2[f, ib, 7]]
    assert len(rows) == len(o.part2)
    for (f, ib), orow in zip(rows, o.part2):
        assert (f, ib) == (orow[0], orow[1])
        assert np.allclose(r.part2[f, ib, :5], [orow[2], orow[3], orow[4], orow[5], orow[6]], rtol=TOL, atol=TOL)
        assert np.allclose(r.part2[f, ib, 5:7], [orow[7], orow[8]], rtol=TOL, atol=TOL)
    prow = [ib for ib in range(r.part3.shape[0]) if r.part3[ib, 7]]
    assert prow == [x[0] for x in o.part3]
    for ib, orow in zip(prow, o.part3):
        assert np.allclose(r.part3[ib, :4], [orow[1], orow[2], orow[3], orow[4]], rtol=TOL, atol=TOL)
        assert np.allclose(r.part3[ib, 4:7], [orow[5], orow[6], orow[7]], rtol=TOL, atol=TOL)


@pytest.mark.parametrize("ns,gas,nskip", [(2, 0, 5), (2, 1, 0), (3, 0, 10), (4, 0, 3)])
def test_analysis_matches_oracle(ns, gas, nskip):
    from q_b200.fep import analyze, params
    nf = 6
    S = random_series(nf, 300, ns, seed=ns * 10 + gas)
    alfa = [0.7 * k for k in range(1, ns)]
    coeff = [1.0] + [0.0] * (ns - 2) + [-1.0]
    r = analyze(S, params(0.592, nskip, gas=gas, nbins=12, nmin=4, alfa=alfa, coeff=coeff))
    o = oracle_analyze(FepInput(S, 0.592, nskip, gas=gas, nbins=12, nmin=4, alfa=alfa, coeff=coeff))
    compare(r, o, nf)


EVB = {2: [(1, 2, 12.0, 0.4, 0.05, 1.8)],
       3: [(1, 2, 12.0, 0.4, 0.05, 1.8), (3, 1, 6.0, 0.8, 0.0, 2.2), (2, 3, 4.0, 0.2, 0.1, 2.0)],
       4: [(1, 2, 12.0, 0.4, 0.05, 1.8), (2, 3, 4.0, 0.2, 0.1, 2.0), (4, 3, 9.0, 0.6, 0.0, 2.5)]}


@pytest.mark.parametrize("ns", [2, 3, 4])
def test_evb_analysis_matches_oracle(ns):
    """EVB ground state from Hij(r_xy) (qfep.f90:286-318): the 2 x 2 closed
    form with the c1^2, c2^2 weights, or the lowest eigenvalue for more
    states; bin averages of c1^2, c2^2 and r_xy in Parts 2 and 3."""
    from q_b200.fep import analyze, params
    nf = 5
    S = random_series(nf, 250, ns, seed=40 + ns, spread=2.0)
    rng = np.random.default_rng(ns)
    rxy = [rng.uniform(1.5, 3.0, s.shape[0]) for s in S]
    coeff = [1.0] + [0.0] * (ns - 2) + [-1.0]
    r = analyze(S, params(0.592, 4, nbins=10, nmin=3, coeff=coeff, evb=EVB[ns]), rxy=rxy)
    o = oracle_analyze(FepInput(S, 0.592, 4, nbins=10, nmin=3, coeff=coeff, evb=EVB[ns], rxy=rxy))
    compare(r, o, nf)
    if ns == 2:
        assert np.any(r.part2[:, :, 5] > 0.01) and np.any(r.part3[:, 6] > 1.5)


def test_invalid_input_is_refused():
    from q_b200 import QBError
    from q_b200.fep import analyze, params
    S = random_series(3, 20, 2, seed=1)
    with pytest.raises(QBError):
        analyze(S, params(0.592, 50))           # more points skipped than recorded
    with pytest.raises(QBError):
        analyze(S[:1], params(0.592, 0))        # one window


def test_qfep_driver_end_to_end(tmp_path):
    from q_b200 import append_energy
    from q_b200.qfep import fmt_f, run
    nf = 5
    S = random_series(nf, 200, 2, seed=7, spread=0.5)
    names = []
    for k, s in enumerate(S):
        p = str(tmp_path / ("md_%d.en" % k))
        for frame in s:
            append_energy(p, frame)
        names.append(p)
    text = "%d\n2 0\n0.592 20\n10\n5\n0.0\n0\n1 -1\n%s\n" % (nf, "\n".join(names))
    out = io.StringIO()
    assert run(io.StringIO(text), out) == 0
    report = out.getvalue()
    o = oracle_analyze(FepInput(S, 0.592, 20, nbins=10, nmin=5, alfa=[0.0], coeff=[1.0, -1.0]))
    # Part 6 rows as QligFEP reads them (lambda, dG, sum(dG))
    part6 = report.split("# Part 6: BAR Bennet:")[1].splitlines()[2:2 + nf]
    for i, line in enumerate(part6, start=1):
        lam, dg, tot = line.split()
        assert lam == fmt_f(1.0 - (i - 1) / (nf - 1), 8, 6).strip()
        assert abs(float(tot) - o.dgbarsum[i]) < 1.5e-3
    assert "# Part 1: Free energy perturbation summary:" in report
    assert report.count("--> Name of file number") == nf


def test_batch_records_analysed_in_place(tmp_path):
    """Three lambda windows of the FEP system: the analysis of the batch's own
    records on the device equals the analysis of the same records copied out."""
    from q_b200 import MIXED, Batch, System, synth
    from q_b200.fep import analyze, params
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, steps=200)
    lams = [(1.0, 0.0), (0.5, 0.5), (0.0, 1.0)]
    systems = [System.open(g.inp, lambdas=l, seed=11) for l in lams]
    b = Batch(systems, precision=MIXED)
    b.run(60)
    p = params(0.592, 1, nbins=4, nmin=1)
    r = b.fep([0, 1, 2], 0.592, 1, nbins=4, nmin=1)
    series = []
    for k in range(3):
        _, _, EQ = b.history(k, 1)
        series.append(EQ[:, :2, :])
    h = analyze(series, p)
    for name in ("dgf", "dgr", "dgbar", "dgbarsum", "dglu", "dgti"):
        assert np.allclose(getattr(r, name), getattr(h, name), rtol=1e-12, atol=1e-12), name
    assert list(r.npts) == [s.shape[0] for s in series] and r.npts[0] >= 5


def test_perturbation_campaign(tmp_path):
    """Windows x replicas of one perturbation in one batch: equilibration
    records dropped, production records analysed per replica, device time
    measured; the plain engine's per-step time for one window."""
    from q_b200 import MIXED, synth
    from q_b200.campaign import run_perturbation, time_single_window
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, steps=1000)
    r = run_perturbation(g.inp, synth.window_lambdas(3), replicas=2, steps_eq=20, steps_prod=100,
                         precision=MIXED, seed0=5)
    assert (r.windows, r.replicas, r.steps) == (3, 2, 120)
    assert r.records_per_window == 10            # energy interval 10, records after the equilibration only
    assert len(r.dG) == 2 and all(np.isfinite(r.dG)) and r.dG[0] != r.dG[1]
    assert abs(r.dG_mean - np.mean(r.dG)) < 1e-12 and r.dG_sem > 0
    assert all(len(b) == 2 for b in r.bar)
    assert all(abs(sum(b) - d) < 1e-9 for b, d in zip(r.bar, r.dG))
    assert r.gpu_seconds > 0
    assert 0 < time_single_window(g.inp, (0.5, 0.5), 20, warmup=5) < 0.1
