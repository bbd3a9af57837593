"""The CPU oracle against the reference's own known answers (CPU only).

Pins (tests/golden/make_golden.py says where each comes from):
  * test/q6/test1/eval_test.sh:67 -- the initial Q-surr line of eq1.log,
    "Q-surr. 1 1.0000 3.12 139.43", and the 10-seed bounds of
    qsurr_benchmark.en for the next two summaries (step 50 and FINAL of eq1);
  * test/3.shake/p-p/benzene Q5_data/eq1.log -- the step-0 and FINAL energy
    summaries and the initial temperature of a 1-step benzene run;
  * the same log's Maxwell velocities for random_seed 112 at 1 K.
"""
import os

import numpy as np
import pytest

from q_b200 import E_NAMES, System, maxwell

E = {n: i for i, n in enumerate(E_NAMES)}
QP_EL, QP_VDW, QW_EL, QW_VDW = 10, 11, 12, 13


def qsurr(EQ, st=0):
    return EQ[st, QP_EL] + EQ[st, QW_EL], EQ[st, QP_VDW] + EQ[st, QW_VDW]


def fmt2(x):
    return float("%.2f" % x)


def test_test1_initial_qsurr_exact(golden, oracle):
    sys_ = System.open(str(golden / "test1" / "eq1.inp"))
    run = oracle.create(sys_)
    run.run(1)
    steps, Eh, EQh = run.history(0)
    assert steps[0] == 0
    el, vdw = qsurr(EQh[0])
    line = "Q-surr. 1 %6.4f %9.2f %9.2f" % (EQh[0, 0, 0], el, vdw)
    assert line.split() == "Q-surr. 1 1.0000 3.12 139.43".split()


def test_test1_trajectory_within_seed_bounds(golden, oracle):
    """eq1 (100 steps of 0.1 fs at 0.1 K, LRF, solvent SHAKE, radial and
    polarisation restraints): the step-50 and FINAL Q-surr energies against the
    benchmark's mean +/- 1 sd over 10 seeds, allowing 3 sd."""
    sys_ = System.open(str(golden / "test1" / "eq1.inp"))
    bounds = np.loadtxt(str(golden / "test1" / "qsurr_bounds.txt"))
    run = oracle.create(sys_)
    assert run.run(100) == 0
    steps, Eh, EQh = run.history(0)
    assert list(steps) == [0, 50]
    run.final_energy()
    _, EQf = run.energy_vectors()
    values = [qsurr(EQh[1]), qsurr(EQf)]
    for (el, vdw), row in zip(values, bounds[1:3]):
        for val, lo, hi in ((el, row[1], row[2]), (vdw, row[3], row[4])):
            mid, sd = 0.5 * (lo + hi), max(0.5 * (hi - lo), 0.005)
            assert abs(val - mid) <= 3 * sd + 0.005, (val, lo, hi)


def _summary(E_):
    return [fmt2(E_[E["pp_el"]]), fmt2(E_[E["pp_vdw"]]), fmt2(E_[E["p_bond"]]),
            fmt2(E_[E["potential"]] + E_[E["kinetic"]]), fmt2(E_[E["potential"]]), fmt2(E_[E["kinetic"]])]


def test_benzene_energy_summaries(golden, oracle):
    sys_ = System.open(str(golden / "benzene" / "eq1.inp"))
    run = oracle.create(sys_)
    T0 = run.temperature()
    assert "%.2f %.2f" % (T0[0], T0[1]) == "1.04 1.04"      # "Initial temperatures are : Ttot = 1.04 Tfree = 1.04"
    run.run(1)
    steps, Eh, _ = run.history(0)
    # eq1.log: solute 1.92 6.04 0.86 ... SUM 8.87 8.82 0.05
    assert _summary(Eh[0]) == [1.92, 6.04, 0.86, 8.87, 8.82, 0.05]
    run.final_energy()
    Ef, _ = run.energy_vectors()
    # eq1.log FINAL: solute 1.92 6.00 0.80 ... SUM 8.78 8.73 0.05
    assert _summary(Ef) == [1.92, 6.00, 0.80, 8.78, 8.73, 0.05]


def test_benzene_maxwell_velocities_bit_exact(golden):
    sys_ = System.open(str(golden / "benzene" / "eq1.inp"))
    mass = sys_.array("mass", sys_.natom)
    v = maxwell(112, 1.0, mass)
    ref = []
    for line in open(str(golden / "benzene" / "velocities.csv")).read().split("\n")[2:]:
        if ";" in line:
            ref += [float(t) for t in line.split(";")]
    assert np.array_equal(v, np.array(ref))


def read_fortran_re(path):
    """qdyn's restart (write_xfin, md.f90:15452-15470), read here without the
    library: gfortran unformatted sequential records of (int32 nat3, nat3
    doubles) for x and v, each framed by int32 byte counts."""
    raw = open(path, "rb").read()
    recs, off = [], 0
    while off < len(raw):
        n = int(np.frombuffer(raw, "<i4", 1, off)[0])
        body = raw[off + 4:off + 4 + n]
        assert int(np.frombuffer(raw, "<i4", 1, off + 4 + n)[0]) == n
        recs.append(body)
        off += n + 8
    out = []
    for body in recs[:2]:
        nat3 = int(np.frombuffer(body, "<i4", 1, 0)[0])
        out.append(np.frombuffer(body, "<f8", nat3, 4).copy())
    return raw, out[0], out[1], len(recs)


def test_fortran_restart_read_and_written_byte_for_byte(golden, tmp_path):
    """The restart file Fortran qdyn wrote for the 1-step benzene run: the
    library's reader takes exactly its values, and the library's writer
    reproduces the file byte for byte."""
    from q_b200.api import write_restart
    from q_b200.inputs import derive_inp
    raw, x, v, nrec = read_fortran_re(str(golden / "benzene" / "eq1.re"))
    assert len(raw) == 600 and nrec == 2 and x.size == v.size == 36
    inp = derive_inp(str(golden / "benzene" / "eq1.inp"), "from_re.inp",
                     set_keys={"files": {"restart": "eq1.re"}},
                     drop_keys={"md": ["random_seed", "initial_temperature"]})
    s = System.open(inp)
    n = 3 * s.natom
    assert np.array_equal(np.ctypeslib.as_array(s.view.x0, shape=(n,)), x)
    assert np.array_equal(np.ctypeslib.as_array(s.view.v0, shape=(n,)), v)
    out = str(tmp_path / "again.re")
    write_restart(out, x, v)
    assert open(out, "rb").read() == raw


# Fortran's step and the restatement differ in the last bits of single-
# precision intermediates (FP32 inverse masses and charges, gfortran's own
# contraction of d*winv*dt): 5e-8 relative on velocities of ~0.03 A/fs-units
RE_V_RTOL = 1e-7


def test_oracle_step_matches_fortran_restart(golden, oracle):
    """The oracle's one MD step of the benzene run (Maxwell velocities of
    seed 112 at 1 K, leap-frog, Berendsen) against the coordinates and
    velocities Fortran qdyn wrote after that step."""
    _, x, v, _ = read_fortran_re(str(golden / "benzene" / "eq1.re"))
    s = System.open(str(golden / "benzene" / "eq1.inp"))
    run = oracle.create(s)
    run.run(1)
    assert np.max(np.abs(run.coords() - x)) < 1e-9
    np.testing.assert_allclose(run.velocities(), v, rtol=RE_V_RTOL, atol=1e-12 + RE_V_RTOL * np.abs(v).max())
