"""Regenerate the golden fixtures of tests/golden from the reference tree.

    python tests/golden/make_golden.py /path/to/reference

The fixtures are the reference's own test inputs and known answers, copied
(gzip-compressed) so that the tests can run where the reference is absent:

  test1/        test/q6/test1: ligand in a 20 A TIP3P sphere.  The topology is
                prep/originals/lig_w.top.bak.original, the one the benchmark
                bounds of qsurr_benchmark.en were generated with (the
                regenerated prep/lig_w.top gives Q-surr 3.58 instead of 3.12
                at step 0).  eq1.inp is copied with its file paths pointed at
                the fixture names.  qsurr_bounds.txt holds the first lines of
                qsurr_benchmark.en (step, el lower/upper, vdW lower/upper).
  benzene/      test/3.shake/p-p/benzene/testfiles.tar.gz: benzene in vacuum.
                eq1.log was produced with solute SHAKE off (its header prints
                "SHAKE all solute bonds = off"), so the fixture input sets
                shake_solute off.  velocities.csv holds the Maxwell velocities
                the log prints for random_seed 112 at 1 K; eq1.re is the
                restart qdyn wrote after the run's one step (600 bytes).
  data/         test/data/topology and test/data/inputs: topologies and FEP
                files of the reference's Q6-vs-QGPU comparison harness
                (test/runTEST.py); its interaction-class cases (p-p, q-p,
                q-p-w, q-q, w-p, w-q, w-w) are GPU-vs-oracle parity cases.
"""
from __future__ import annotations

import gzip
import os
import shutil
import sys
import tarfile

HERE = os.path.dirname(os.path.abspath(__file__))


def gz_copy(src: str, dst: str) -> None:
    # mtime 0: the same input gives the same bytes
    with open(src, "rb") as f, open(dst + ".gz", "wb") as raw, \
            gzip.GzipFile(fileobj=raw, mode="wb", compresslevel=9, mtime=0) as g:
        g.write(f.read())


def main(ref: str) -> None:
    t1 = os.path.join(ref, "test/q6/test1")
    out = os.path.join(HERE, "test1")
    os.makedirs(out, exist_ok=True)
    gz_copy(os.path.join(t1, "prep/originals/lig_w.top.bak.original"), os.path.join(out, "lig_w.top"))
    shutil.copy(os.path.join(t1, "prep/lig_w.fep"), os.path.join(out, "lig_w.fep"))
    inp = open(os.path.join(t1, "eq1.inp")).read()
    inp = inp.replace("prep/lig_w.top", "lig_w.top").replace("prep/lig_w.fep", "lig_w.fep")
    open(os.path.join(out, "eq1.inp"), "w").write(inp)
    lines = [l for l in open(os.path.join(t1, "qsurr_benchmark.en")) if l.strip() and not l.startswith("#")]
    with open(os.path.join(out, "qsurr_bounds.txt"), "w") as f:
        f.write("# first lines of test/q6/test1/qsurr_benchmark.en: step el_lo el_hi vdw_lo vdw_hi\n")
        f.writelines(lines[:4])

    out = os.path.join(HERE, "benzene")
    os.makedirs(out, exist_ok=True)
    tmp = os.path.join(HERE, "_tmp_benzene")
    with tarfile.open(os.path.join(ref, "test/3.shake/p-p/benzene/testfiles.tar.gz")) as tf:
        tf.extractall(tmp, filter="data")
    q5 = os.path.join(tmp, "Q5_data")
    gz_copy(os.path.join(q5, "benzene-vacuum.top"), os.path.join(out, "benzene-vacuum.top"))
    inp = open(os.path.join(q5, "eq1.inp")).read()
    inp = "\n".join("shake_solute              off" if l.startswith("shake_solute") else l
                    for l in inp.split("\n"))
    open(os.path.join(out, "eq1.inp"), "w").write(inp)
    shutil.copy(os.path.join(q5, "velocities.csv"), os.path.join(out, "velocities.csv"))
    shutil.copy(os.path.join(q5, "eq1.log"), os.path.join(out, "eq1.log"))
    # the restart qdyn wrote at the end of that run (write_xfin, md.f90:15452):
    # coordinates and velocities after the one step, gfortran record markers
    shutil.copy(os.path.join(q5, "eq1.re"), os.path.join(out, "eq1.re"))
    shutil.rmtree(tmp)

    out = os.path.join(HERE, "data")
    os.makedirs(out, exist_ok=True)
    for name in ["ala_wat.top", "benzene-water.top", "benzene-vacuum.top", "dualtop_vacuum.top", "water.top",
                 "Na-benzene-vacuum.top", "Na-benzene-water.top"]:
        gz_copy(os.path.join(ref, "test/data/topology", name), os.path.join(out, name))
    for name in ["FEP_benzene.fep", "FEP_Na.fep", "dualtop.fep"]:
        shutil.copy(os.path.join(ref, "test/data/inputs", name), os.path.join(out, name))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(sys.argv[1])
