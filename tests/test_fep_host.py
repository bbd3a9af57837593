"""Free-energy analysis, host side (no GPU): the qfep restatement (oracle)
on analytic cases, the energy-file reader against libqb's writer, qfep's
input reading and its Fortran number editing."""
import io
import math

import numpy as np
import pytest

from oracle.qfep_oracle import FepInput, analyze


def gaussian_windows(nf=11, n=3000, mu=2.0, s2=0.5, rt=0.592, seed=1):
    """Two states coupled linearly, U(l) = (1-l) U1 + l U2, with dU = U2 - U1
    Gaussian N(mu, s2) at l = 0.  At window l it is N(mu - l s2/kT, s2) and
    dG = mu - s2/(2 kT) exactly."""
    rng = np.random.default_rng(seed)
    out = []
    for l in np.linspace(0.0, 1.0, nf):
        e = np.zeros((n, 2, 15))
        e[:, 0, 0], e[:, 1, 0] = 1.0 - l, l
        u1 = rng.normal(0.0, 1.0, n)
        du = rng.normal(mu - l * s2 / rt, math.sqrt(s2), n)
        e[:, 0, 1], e[:, 1, 1] = u1, u1 + du
        out.append(e)
    return out, mu - s2 / (2 * rt)


def test_estimators_on_gaussian_perturbation():
    rt = 0.592
    E, exact = gaussian_windows(rt=rt)
    r = analyze(FepInput(E, rt, 100, nbins=10, nmin=10, alfa=[0.0], coeff=[1.0, -1.0]))
    nf = len(E)
    for est in (r.dgfsum[nf], -r.dgrsum[1], r.dgbarsum[nf], r.dglusum[nf], r.dG[nf]):
        assert abs(est - exact) < 0.05, (est, exact)
    # TI: trapezoid of <U2 - U1> over the step of lambda(1), lambda(i-1) - lambda(i)
    assert abs(r.dgtisum[nf] - exact) < 0.05
    assert all(1 <= k < 100 for k in r.bar_iterations)


def test_identical_windows_give_zero_and_alpha_shifts_gap():
    rng = np.random.default_rng(3)
    e = np.zeros((500, 2, 15))
    e[:, :, 0] = 0.5
    e[:, :, 1] = rng.normal(0, 1, (500, 2))
    r = analyze(FepInput([e, e.copy()], 0.6, 0, nbins=5, nmin=1, alfa=[0.0], coeff=[1.0, -1.0]))
    assert r.dgfsum[2] == pytest.approx(0.0, abs=1e-12) and r.dgbarsum[2] == pytest.approx(0.0, abs=1e-9)
    r2 = analyze(FepInput([e, e.copy()], 0.6, 0, nbins=5, nmin=1, alfa=[3.0], coeff=[1.0, -1.0]))
    assert r2.gapmin == pytest.approx(r.gapmin - 3.0) and r2.gapmax == pytest.approx(r.gapmax - 3.0)


def test_part0_uses_single_precision_scale():
    e = np.zeros((7, 1, 15))
    e[:, 0, 1] = 1.0
    r = analyze(FepInput([e, e], 0.6, 0, nbins=2, nmin=1))
    k = float(np.float32(1.0) / np.float32(7))
    assert r.avEQ[0, 0, 1] == 7.0 * k and r.avEQ[0, 0, 1] != 1.0


def test_energy_file_reader_round_trip(tmp_path):
    from q_b200 import append_energy
    from q_b200.fep import read_en
    path = str(tmp_path / "w.en")
    rng = np.random.default_rng(0)
    frames = rng.normal(size=(6, 2, 15))
    for k in range(6):
        append_energy(path, frames[k])
    got = read_en(path, 2)
    assert got.shape == (6, 2, 15) and np.array_equal(got, frames)
    # a frame without its off-diagonal record is not counted (get_ene)
    raw = open(path, "rb").read()
    open(path, "wb").write(raw[:-8])
    assert read_en(path, 2).shape[0] == 5


def test_fortran_number_editing():
    from q_b200.qfep import fmt_f, fmt_i
    assert fmt_f(1.0, 8, 6) == "1.000000"
    assert fmt_f(-0.123, 8, 6) == "-.123000"
    assert fmt_f(-1.5, 9, 3) == "   -1.500"
    assert fmt_f(1e9, 9, 3) == "*" * 9
    assert fmt_f(-math.inf, 9, 3) == "-Infinity" and fmt_f(math.nan, 9, 3) == "      NaN"
    assert fmt_i(123456, 4) == "****" and fmt_i(5, 4) == "   5"


def test_qfep_input_records():
    from q_b200.qfep import _Input
    text = "3\n2  0\n0.592  50\n\n50\n10\n0\n0\n1 0\n!ENERGY_FILES\na.en\nb.en\nc.en\n"
    inp = _Input(io.StringIO(text))
    assert inp.values(1) == ["3"] and inp.values(2) == ["2", "0"]
    assert inp.record().split() == ["0.592", "50"]
    assert inp.values(1) == ["50"] and inp.values(1) == ["10"]
    assert inp.values(1) == ["0"] and inp.values(1) == ["0"] and inp.values(2) == ["1", "0"]
    assert [inp.values(1)[0] for _ in range(3)] == ["a.en", "b.en", "c.en"]


def test_mlp_oracle_gradient_is_exact():
    """The network oracle's analytic gradient against central differences."""
    from oracle import mlp_oracle as M
    p = M.init(1)
    rng = np.random.default_rng(2)
    x, t = rng.normal(size=(40, M.IN)), rng.normal(size=(40, M.OUT))
    L, g = M.loss_grad(p, x, t)
    h = 1e-6
    for k in rng.choice(M.NPARAM, 60, replace=False):
        e = np.zeros(M.NPARAM)
        e[k] = h
        num = (M.loss_grad(p + e, x, t)[0] - M.loss_grad(p - e, x, t)[0]) / (2 * h)
        assert abs(num - g[k]) < 1e-7 * max(1.0, abs(g[k]))
    # the BF16 rounding used by the oracle: ties to even, exact on BF16 values
    v = np.array([1.0, 1.00390625, 1.005859375, -3.0e-3], dtype=np.float32)
    assert list(M.bf16(v)) == [1.0, 1.0, 1.0078125, float(np.float32(-0.0030059814453125))]


def test_qligfep_schedule_matches_reference_golden():
    """QligFEP's get_lambdas restated, against schedules produced by the
    reference's own function (tests/golden/make_lambda_golden.py)."""
    import json
    import os
    from q_b200 import lambda_placement as L
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "qligfep_lambdas.json")))
    for sampling, table in g.items():
        for w, lam in table.items():
            ref = np.array([1.0 - float(x) for x in lam])
            assert np.allclose(L.qligfep_schedule(int(w), sampling), ref, atol=1e-12), (sampling, w)


def test_length_spacing_and_features():
    from q_b200 import lambda_placement as L
    # constant sigma: uniform; sigma 4x larger on the upper half: 4x denser there
    assert np.allclose(L.length_spacing(L.DENSE_U, np.ones(21)), np.linspace(0, 1, 12))
    sig = np.where(np.array(L.DENSE_U) < 0.5, 1.0, 4.0)
    u = L.length_spacing(L.DENSE_U, sig)
    gaps = np.diff(u)
    assert u[0] == 0.0 and u[-1] == 1.0 and np.all(gaps > 0)
    assert gaps[0] / gaps[-1] > 3.5
    # logits round trip
    assert np.allclose(L.positions_from_logits(L.spacing_logits(u)), u, atol=1e-9)
    # the features carry the pilot's sigma profile exactly
    rng = np.random.default_rng(0)
    sd = (8.0, 6.0, 4.0, 3.0, 2.0)
    dU = [rng.normal(m, s, 400) for m, s in zip((50, 30, 15, 5, 0), sd)]
    f = L.pilot_features(dU)
    assert f.shape == (12,) and np.all(np.isfinite(f)) and 0 <= f[11] < 1
    assert np.allclose(L.KT * np.exp(f[0:5] + 3 * f[10]), [np.std(d) for d in dU])
    pu = L.pilot_spacing(f)
    assert np.all(np.diff(pu) > 0) and np.diff(pu)[0] < np.diff(pu)[-1]   # denser where sigma is large


def test_reference_python_estimators_on_constant_windows():
    """The reference's own Python estimators (src/Qgpu/calc.py, run unchanged
    by tests/golden/make_qfep_golden.py) against the qfep restatement.  They
    are not qfep: they pair record ipt with record ipt + 1 of one series,
    divide by the record count instead of the pairs used, take exp(-dv) in
    both halves of overlap sampling, and define BAR's dv as V(l1) - V(l2).
    On windows whose every record is the same, those differences reduce to
    exact identities, checked here: Zwanzig forward and reverse differ from
    qfep's by -kT ln((n - 1)/n), BAR is qfep's with the opposite sign, and
    overlap sampling is 0 where qfep's is the energy difference.  On other
    series the two differ by design (the golden file holds such cases, which
    are not compared)."""
    import json
    import os
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "qgpu_calc_estimators.json")))
    ncmp = 0
    for c in d["cases"]:
        if not c["constant"]:
            continue
        kT, l1, l2 = c["kT"], np.array(c["l1"]), np.array(c["l2"])
        row = np.array(c["series"][0])
        n = len(c["series"])
        files = []
        for lam in (l1, l2):
            e = np.zeros((n, 2, 15))
            e[:, :, 0] = lam
            e[:, :, 1] = row
            files.append(e)
        r = analyze(FepInput(files, kT, 0, nbins=4, nmin=1, alfa=[0.0], coeff=[1.0, -1.0]))
        shift = -kT * math.log((n - 1) / n)
        assert abs(c["EXPfwd"] - (r.dgf[1] + shift)) < 1e-10
        assert abs(c["EXPbwd"] - (r.dgr[2] + shift)) < 1e-10
        assert abs(c["BAR"] + r.dgbar[1]) < 2e-3          # both iterate to |change| <= 0.001
        assert c["overlap_sampling"] == 0.0
        assert abs(r.dglu[1] - float((l2 - l1) @ row)) < 1e-10
        ncmp += 1
    assert ncmp == 4
