"""EVB off-diagonal functions on the GPU: r_kl recorded with every output and
energy-file record (offdiag, md.f90:12911) against the oracle, and the qdyn
drop-in writing them into the energy file's off-diagonal record and the
log."""
import io
import os

import numpy as np
import pytest

from q_b200 import FP64, Batch, System, synth
from q_b200.fep import read_en, read_offdiag
from q_b200.inputs import derive_inp, inp_sections

pytestmark = pytest.mark.gpu

OFFD = [(1, 2, 1, 2, 50.0, 0.5), (2, 1, 3, 5, 20.0, 1.0)]


@pytest.fixture(scope="module")
def evb(tmp_path_factory):
    root = tmp_path_factory.mktemp("evb")
    g = synth.fep_solute(str(root), off_diagonals=OFFD, lambdas=(0.6, 0.4))
    return derive_inp(g.inp, "evb30.inp", set_keys={"md": {"steps": 30}, "intervals": {"output": 5, "energy": 5}})


def test_offdiag_records_match_oracle(evb, oracle):
    s = System.open(evb)
    b = Batch([s], precision=FP64)
    b.run(30)
    o = oracle.create(s)
    o.run(30)
    A = np.array([f[4] for f in OFFD])
    mu = np.array([f[5] for f in OFFD])
    for kind, n in ((0, 6), (1, 5)):
        od = b.offdiag(0, kind)
        r = o.offdiag(kind)
        assert od.shape == (n, 2, 2) and r.shape == (n, 2)
        assert np.max(np.abs(od[:, :, 1] - r)) < 1e-9
        assert np.allclose(od[:, :, 0], A * np.exp(-mu * od[:, :, 1]), rtol=1e-14, atol=0)
    # the values of the last step's force evaluation (kind 2)
    last = b.offdiag(0, 2)
    assert last.shape == (1, 2, 2) and np.all(last[0, :, 1] > 1.0)


def test_qdyn_writes_off_diagonal_records(evb):
    from q_b200 import qdyn
    out = io.StringIO()
    assert qdyn.run(evb, out=out) == 0
    log = out.getvalue()
    files = dict(l.split()[:2] for l in inp_sections(evb)["files"])
    en = os.path.join(os.path.dirname(evb), files["energy"])
    EQ = read_en(en, 2)
    od = read_offdiag(en, 2)
    assert EQ.shape[0] == 5 and od.shape == (5, 2, 4)
    assert np.array_equal(od[:, :, :2], np.tile([[1, 2], [2, 1]], (5, 1, 1)))
    A = np.array([f[4] for f in OFFD])
    mu = np.array([f[5] for f in OFFD])
    assert np.allclose(od[:, :, 2], A * np.exp(-mu * od[:, :, 3]), rtol=1e-14, atol=0)
    assert np.all((od[:, 0, 3] > 1.2) & (od[:, 0, 3] < 1.8))     # Q atoms 1-2 are bonded
    # one line per function in each of the 6 summaries and the final one
    assert log.count("H( 1, 2) =") == 7 and log.count("H( 2, 1) =") == 7
    assert "dist. between Q-atoms   1   2 =" in log


def test_batch_evb_analysis_in_place(tmp_path):
    """Three windows of the EVB system: qfep's EVB analysis of the batch's
    own records on the device (r_xy read from the record ring) equals the
    analysis of the same records and distances copied out."""
    from q_b200 import MIXED
    from q_b200.fep import analyze, params
    g = synth.fep_solute(str(tmp_path / "c1"), off_diagonals=OFFD, steps=200)
    inp = derive_inp(g.inp, "w.inp", set_keys={"intervals": {"energy": 2}})
    systems = [System.open(inp, lambdas=l, seed=11) for l in [(1.0, 0.0), (0.5, 0.5), (0.0, 1.0)]]
    b = Batch(systems, precision=MIXED)
    b.run(60)
    evb = [(1, 2, 30.0, 0.6, 0.0, 1.45)]
    r = b.fep([0, 1, 2], 0.592, 1, nbins=4, nmin=1, evb=evb)
    series = [b.history(k, 1)[2] for k in range(3)]
    rxy = [b.offdiag(k, 1)[:, 0, 1] for k in range(3)]
    assert all(x.shape[0] == 29 for x in rxy)
    h = analyze(series, params(0.592, 1, nbins=4, nmin=1, evb=evb), rxy=rxy)
    for name in ("dG", "dgbarsum", "dgtisum"):
        assert np.allclose(getattr(r, name), getattr(h, name), rtol=1e-12, atol=1e-12)
    assert np.allclose(r.part2, h.part2, rtol=1e-9, atol=1e-9)
    assert np.allclose(r.part3, h.part3, rtol=1e-9, atol=1e-9)
    assert np.any(r.part3[:, 6] > 1.2)                 # <r_xy> of the bonded Q atoms 1-2


def test_qfep_driver_reads_off_diagonal_records(tmp_path):
    """The qfep drop-in with EVB elements: r_xy from each energy file's
    off-diagonal records, Parts 2 and 3 with the c1^2, c2^2 and r_xy columns,
    against the oracle; a file without enough off-diagonal elements stops it
    as get_ene does."""
    from oracle.qfep_oracle import FepInput
    from oracle.qfep_oracle import analyze as oracle_analyze
    from q_b200 import append_energy
    from q_b200.qfep import run
    rng = np.random.default_rng(3)
    nf, names, S, R = 4, [], [], []
    for k in range(nf):
        e = rng.normal(0.0, 2.0, (120, 2, 15))
        e[:, :, 0] = [1.0 - k / (nf - 1), k / (nf - 1)]
        rx = rng.uniform(1.5, 3.0, 120)
        p = str(tmp_path / ("evb_%d.en" % k))
        for m in range(120):
            append_energy(p, e[m], (np.array([[1, 2]]), np.array([[10.0 * np.exp(-rx[m]), rx[m]]])))
        names.append(p)
        S.append(e)
        R.append(rx)
    text = "%d\n2 0\n0.592 5\n8\n3\n0.0\n1\n1 2 12.0 0.4 0.05 1.8\n1 -1\n%s\n" % (nf, "\n".join(names))
    out = io.StringIO()
    assert run(io.StringIO(text), out) == 0, out.getvalue()[-500:]
    rep = out.getvalue()
    assert "#   1   2    12.00     0.40     0.05     1.80" in rep
    o = oracle_analyze(FepInput(S, 0.592, 5, nbins=8, nmin=3, alfa=[0.0], coeff=[1.0, -1.0],
                                evb=[(1, 2, 12.0, 0.4, 0.05, 1.8)], rxy=R))
    part3 = rep.split("# Part 3: Bin-averaged summary:")[1].split("# Part 4")[0].splitlines()[2:]
    rows = [l.split() for l in part3 if l.strip()]
    assert len(rows) == len(o.part3)
    for row, orow in zip(rows, o.part3):
        assert int(row[0]) == orow[0]
        assert abs(float(row[5]) - orow[5]) < 1.5e-3 and abs(float(row[7]) - orow[7]) < 1.5e-3
    # two elements asked for, one stored
    bad = io.StringIO()
    text2 = "%d\n2 0\n0.592 5\n8\n3\n0.0\n2\n1 2 12.0 0.4 0.05 1.8\n2 1 1.0 0.1 0.0 2.0\n1 -1\n%s\n" % (
        nf, "\n".join(names))
    assert run(io.StringIO(text2), bad) == 1
    assert "Maybe there are less than 2 off-diagonal elements?" in bad.getvalue()


def test_morse_couplings_match_oracle(tmp_path, oracle):
    """EVB Morse couplings on the GPU (qangle, qurey_bradley, qtorsion,
    qimproper with couplings to a Morse bond that exists in state 1 only):
    an AMBER and a CHARMM system in one batch against the oracle over 20
    steps, the couplings' gradient on the bond atoms included."""
    from tests.test_gpu_parity import G_TOL, _worst_atoms, assert_energies, grad_err
    gens = [synth.fep_solute(str(tmp_path / ("ff%d" % ff)), ff_type=ff, q_bonded=True, morse_couplings=True)
            for ff in (2, 3)]
    systems = [System.open(g.inp, lambdas=(0.5, 0.5), seed=9) for g in gens]
    assert all(s.view.qang_cpl[0] == 0 and s.view.qimp_cpl_flag[0] == 1 for s in systems)
    b = Batch(systems, precision=FP64)
    b.run(20)
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.run(20)
        sg, Eg, EQg = b.history(k, 0)
        so, Eo, EQo = o.history(0)
        assert list(sg) == list(so)
        for m in range(len(sg)):
            assert_energies(Eg[m], EQg[m], Eo[m], EQo[m])
        err = grad_err(b.gradient(k), o.gradient())
        assert err < G_TOL, (k, err, _worst_atoms(b.gradient(k), o.gradient()))
