"""Drop-in replacement of the `qfep` program (src/q6/qfep.f90):

    python -m q_b200.qfep < qfep.inp > qfep.out

Reads qfep's input (qfep.f90:87-172: number of files; states and predefined
off-diagonal elements; kT, points to skip and the optional gas mode; gap bins;
minimum points per bin; alpha of states 2..n; the off-diagonal elements;
the linear combination defining the gap; the energy file names), reads the
energy files (nrgy.f90:94-119), runs the analysis on the GPU (libqb,
qb_fep_analyze) and prints the report in qfep's layout (Parts 0-6), which
QligFEP's readers parse (src/QligFEP/IO.py:316, 380).

EVB couplings are outside this path: input with predefined or parametrised
off-diagonal elements is refused.  Lines starting with '!' are skipped.
"""
from __future__ import annotations

import math
import sys


PROGRAM_VERSION = "6.0.1"


def fmt_f(x: float, w: int, d: int) -> str:
    """Fortran Fw.d editing as gfortran writes it: right-justified, the
    leading zero dropped when the field is too narrow, asterisks when the
    number does not fit, Infinity/NaN spelled out."""
    if math.isnan(x):
        s = "NaN"
    elif math.isinf(x):
        if x > 0:
            s = "Infinity" if w >= 8 else "Inf"
        else:
            s = "-Infinity" if w >= 9 else "-Inf"
    else:
        s = "%.*f" % (d, x)
        if len(s) > w:
            if s.startswith("0."):
                s = s[1:]
            elif s.startswith("-0."):
                s = "-" + s[2:]
    if len(s) > w:
        return "*" * w
    return s.rjust(w)


def fmt_i(n: int, w: int) -> str:
    s = "%d" % n
    return "*" * w if len(s) > w else s.rjust(w)


class _Input:
    """One list-directed read per call, as Fortran's read(*,*): a read takes
    the next non-blank record and as many items as it needs."""

    def __init__(self, stream):
        self.lines = [l.rstrip("\n") for l in stream]
        self.k = 0

    def record(self) -> str:
        while self.k < len(self.lines):
            line = self.lines[self.k]
            self.k += 1
            if line.strip() and not line.lstrip().startswith("!"):
                return line
        raise EOFError("qfep input ended early")

    def values(self, n: int) -> list[str]:
        out: list[str] = []
        while len(out) < n:
            out += self.record().replace(",", " ").split()
        return out[:n]


def run(stdin=sys.stdin, out=sys.stdout, device: int = 0) -> int:
    from .fep import analyze, params, read_en, read_offdiag

    w = out.write
    w("-" * 80 + "\n")
    w("Welcome to qfep version: %s (libqb, GPU)\n" % PROGRAM_VERSION)
    w(" \n")
    w("-" * 80 + "\n")
    inp = _Input(stdin)
    w("--> Number of energy files: ")
    nfiles = int(inp.values(1)[0])
    w("# Number of files                                  =%s\n" % fmt_i(nfiles, 6))
    w("--> No. of states, no. of predefined off-diag elements: ")
    v = inp.values(2)
    nstates, noffd = int(v[0]), int(v[1])
    w("# Number of states     =%s\n" % fmt_i(nstates, 6))
    w("# Number of off-diagonal elements                                              =%s\n" % fmt_i(noffd, 6))
    w("--> Give kT & num. of pts to skip & calculation mode: ")
    items = inp.record().replace(",", " ").split()
    if len(items) < 2:
        w("num. correct arguments for KT, data points to skip or calculation mode\n")
        return 1
    rt, nskip = float(items[0]), int(float(items[1]))
    gas = int(float(items[2])) if len(items) >= 3 else 0
    w("# kT                     =%s\n" % fmt_f(rt, 6, 3))
    w("# Number of data points to skip                                                =%s\n" % fmt_i(nskip, 6))
    w("# Only QQ interactions will be considered                                      =%s\n" % fmt_i(gas, 6))
    w("--> Give number of gap-bins: ")
    nbins = int(inp.values(1)[0])
    w("# Number of gap-bins                              =%s\n" % fmt_i(nbins, 6))
    w("--> Give minimum # pts/bin: ")
    nmin = int(inp.values(1)[0])
    w("# Minimum number of points per bin                 =%s\n" % fmt_i(nmin, 6))
    alfa = []
    for st in range(2, nstates + 1):
        w("--> Give alpha for state %s" % fmt_i(st, 2))
        a = float(inp.values(1)[0])
        alfa.append(a)
        w("# Alpha for state %s              =%s\n" % (fmt_i(st, 2), fmt_f(a, 6, 2)))
    if noffd != 0:
        # qfep reads no off-diagonal values in this mode (nnoffd is never set), so its result is undefined
        w("\n>>>>> ERROR: predefined off-diagonal elements (EVB) are not supported; give them as functions\n")
        return 1
    w("--> Number of off-diagonal elements: ")
    nnoffd = int(inp.values(1)[0])
    w("# Number of off-diagonal elements         =%s\n" % fmt_i(nnoffd, 6))
    if nnoffd > 0:
        w("#   i   j   A(i,j)  mu(i,j) eta(i,j) rxy0(i,j)\n")
    evb = []
    for _ in range(nnoffd):
        w("--> i, j, A_ij, mu_ij, eta_ij, r_xy0: ")
        v = inp.values(6)
        i, j, A, mu, eta, r0 = int(v[0]), int(v[1]), float(v[2]), float(v[3]), float(v[4]), float(v[5])
        if not (1 <= i <= nstates and 1 <= j <= nstates):
            w("\n>>>>> ERROR: off-diagonal element states out of range\n")
            return 1
        evb.append((i, j, A, mu, eta, r0))
        w("#" + fmt_i(i, 4) + fmt_i(j, 4) + "".join(fmt_f(x, 9, 2) for x in (A, mu, eta, r0)) + "\n")
    w("--> linear combination of states defining reaction coord: ")
    coeff = [float(x) for x in inp.values(nstates)]
    w("# Linear combination coefficients=%s\n" % "".join(fmt_f(c, 8, 2) for c in coeff))

    w("\n\n")
    w("# Part 0: Average energies for all states in all files\n")
    w("# file             state   pts   lambda    EQtot   EQbond  EQang   EQtor   EQimp    EQel   EQvdW  Eel_qq"
      "  EvdW_qq Eel_qp  EvdW_qp Eel_qw EvdW_qw Eqrstr\n")
    names, series, rxy = [], [], []
    for f in range(nfiles):
        name = inp.values(1)[0]
        try:
            s = read_en(name, nstates)
        except OSError:
            for g in range(f):
                w("--> Name of file number%s: \n" % fmt_i(g + 1, 4))
            w("--> Name of file number%s: \n" % fmt_i(f + 1, 4))
            w(">>>>> ERROR: Failed to open energy file %s\nqfep terminated abnormally: Failed to open energy file.\n"
              % name)
            return 1
        if s.shape[0] <= nskip:
            w(">>>>> ERROR: number of data sets in %s is less than number of points to skip!\n" % name)
            w("qfep terminated abnormally: Too few data points in file.\n")
            return 1
        if nnoffd > 0:
            od = read_offdiag(name, nstates)[:s.shape[0]]
            if od.shape[1] < nnoffd:
                w("ERROR: Unexpected end-of-file in first record of %s\n" % name)
                w("while reading off-diagonal elements.\n")
                w("Maybe there are less than %d off-diagonal elements?\n" % nnoffd)
                w("qfep terminated abnormally: Failed to read off-diagonals.\n")
                return 1
            rxy.append(od[:, 0, 3])
        names.append(name)
        series.append(s)
    if nfiles < 2:
        w(">>>>> ERROR: at least two energy files are needed\n")
        return 1
    r = analyze(series, params(rt, nskip, gas=gas, nbins=nbins, nmin=nmin, alfa=alfa, coeff=coeff, evb=evb), device,
                rxy=rxy if nnoffd > 0 else None)

    # each file's prompt, then its Part 0 rows: (a,t23,i2,1x,i6,1x,f8.6,14f8.2)
    for f in range(nfiles):
        w("--> Name of file number%s: \n" % fmt_i(f + 1, 4))
        for st in range(nstates):
            a = r.avEQ[f, st]
            w(names[f][:22].ljust(22) + fmt_i(st + 1, 2) + " " + fmt_i(int(r.npts[f]) - nskip, 6) + " "
              + fmt_f(r.lam[f, st], 8, 6) + "".join(fmt_f(x, 8, 2) for x in a[1:15]) + "\n")

    def row23(lam, *vals):
        return "   " + fmt_f(lam, 8, 6) + "".join(fmt_f(x, 9, 3) for x in vals)

    w("\n\n")
    w("# Part 1: Free energy perturbation summary:\n")
    w("# lambda(1)      dGf sum(dGf)      dGr sum(dGr)     <dG>\n")
    for i in range(1, nfiles + 1):
        w(row23(r.lam[i - 1, 0], r.dgf[i - 1], r.dgfsum[i], r.dgr[i + 1], r.dgrsum[i], r.dG[i]) + "\n")
    w("\n")
    w("# Min energy-gap is: %s\n" % fmt_f(r.gap_range[0], 9, 2))
    w("# Max energy-gap is: %s\n" % fmt_f(r.gap_range[1], 9, 2))
    w("\n\n")
    w("# Part 2: Reaction free energy summary:\n")
    w("# Lambda(1)  bin Energy gap      dGa     dGb     dGg    # pts    c1**2    c2**2\n")
    for f in range(nfiles):
        for ib in range(1, nbins + 1):
            p = r.part2[f, ib]
            if p[7] == 0.0:
                continue
            w("   " + fmt_f(r.lam[f, 0], 8, 6) + fmt_i(ib, 5) + "  " + "".join(fmt_f(x, 9, 2) for x in p[0:4])
              + "  " + fmt_i(int(p[4]), 5) + fmt_f(p[5], 9, 3) + fmt_f(p[6], 9, 3) + "\n")
    w("\n\n")
    w("# Part 3: Bin-averaged summary:\n")
    w("# bin  energy gap  <dGg> <dGg norm> pts  <c1**2> <c2**2> <r_xy>\n")
    for ib in range(1, nbins + 1):
        p = r.part3[ib]
        if p[7] == 0.0:
            continue
        w(fmt_i(ib, 4) + " " + "".join(fmt_f(x, 9, 2) for x in p[0:3]) + "  " + fmt_i(int(p[3]), 5)
          + "".join(fmt_f(x, 8, 3) for x in p[4:7]) + "\n")
    w("\n\n")
    w("# Part 4: Termodynamic integration:\n")
    w("# lambda(1)      dGti    sum(dGti) \n")
    for i in range(1, nfiles + 1):
        w(row23(r.lam[i - 1, 0], r.dgti[i - 1], r.dgtisum[i]) + "\n")
    w("\n\n")
    w("# Part 5: Overlap sampling Lu et al:\n")
    w("# lambda(1)      dG    sum(dG) \n")
    for i in range(1, nfiles + 1):
        w(row23(r.lam[i - 1, 0], r.dglu[i - 1], r.dglusum[i]) + "\n")
    w("\n\n")
    w("# Part 6: BAR Bennet:\n")
    w("# lambda(1)      dG    sum(dG) \n")
    for i in range(1, nfiles + 1):
        w(row23(r.lam[i - 1, 0], r.dgbar[i - 1], r.dgbarsum[i]) + "\n")
    bad = [i for i in range(1, nfiles) if r.bar_iterations[i] < 0]
    if bad:
        w("# BAR did not reach |change| <= 0.001 within 1000 iterations for window pairs: %s\n"
          % " ".join("%d-%d" % (i, i + 1) for i in bad))
    return 0


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    for a in argv:
        if a in ("-v", "--version"):
            print("qfep version %s" % PROGRAM_VERSION)
            return 0
        if a in ("-h", "--help"):
            print("usage:\npython -m q_b200.qfep < inputfile.inp > outputfile.out")
            return 0
    return run()


if __name__ == "__main__":
    sys.exit(main())
