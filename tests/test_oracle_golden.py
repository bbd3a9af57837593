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
