"""CPU restatement of qfep's free-energy analysis (src/q6/qfep.f90), as test
infrastructure: the reference for the CUDA implementation in libqb
(qb_fep_analyze) and for the qfep-compatible driver.  Nothing in the product
imports this module.

Parity is pinned by restatement only: the reference ships no stored qfep output
and no Fortran compiler exists here.  The restatement follows the reference
loop by loop, in its order of summation, including its quirks:

* Part 0 averages are scaled by a single-precision 1./(npts-nskip)
  (qfep.f90:357, the `real` argument of scale_ene, nrgy.f90:193-215);
* alpha(1) is forced to 0 and added to every state's total (qfep.f90:264-266);
* BAR's sample-size ratios are single-precision quotients (qfep.f90:534-535);
* the 2-state ground state uses the closed form even with no coupling
  (qfep.f90:300-306); more states take the smallest diagonal element (the
  Householder/QL eigenvalues of a diagonal matrix), or with EVB elements the
  lowest eigenvalue of the matrix built from its lower triangle (tred2 reads
  no other part), here from numpy's symmetric eigensolver;
* EVB elements Hij(r) take the parameters of (i, j), or of (j, i) where
  A(i, j) is 0, at the first off-diagonal distance of each record, and only
  that first distance is averaged per bin (qfep.f90:274-299, 643-644);
* bin indices use int() truncation and may reach nbins+1 (qfep.f90:628);
* Part 3's minimum runs over every bin of the fixed-size array, so it is
  never above zero (qfep.f90:735);
* Parts 1/4/5/6 print dG(ifile-1) beside lambda(ifile) (qfep.f90:596-762).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# q_energies components, nrgy.f90:32-41 (the order of one .en record)
NEQ = 15
I_LAMBDA, I_TOTAL, I_BOND, I_ANGLE, I_TORSION, I_IMPROPER = 0, 1, 2, 3, 4, 5
I_QX_EL, I_QX_VDW, I_QQ_EL, I_QQ_VDW, I_QP_EL, I_QP_VDW, I_QW_EL, I_QW_VDW, I_RESTRAINT = range(6, 15)


@dataclass
class FepInput:
    """One qfep run: per file the records [npts][nstates][15] of q_energies."""
    energies: list            # list of arrays (npts, nstates, 15)
    rt: float
    nskip: int
    gas: int = 0
    nbins: int = 20
    nmin: int = 5
    alfa: list = field(default_factory=list)     # alpha of states 2..n (state 1 is 0)
    coeff: list = field(default_factory=list)    # linear combination defining the gap
    evb: list = field(default_factory=list)      # [(i, j, A, mu, eta, rxy0)], states 1-based
    rxy: list = field(default_factory=list)      # per file, r_xy of every record (EVB)


@dataclass
class FepResult:
    lam: np.ndarray          # (nfiles, nstates)
    npts: np.ndarray         # (nfiles,)
    avEQ: np.ndarray         # (nfiles, nstates, 15), Part 0
    dgf: np.ndarray
    dgfsum: np.ndarray
    dgr: np.ndarray
    dgrsum: np.ndarray
    dG: np.ndarray           # arrays indexed 0..nfiles+1 as in qfep
    dgti: np.ndarray
    dgtisum: np.ndarray
    dglu: np.ndarray
    dglusum: np.ndarray
    dgbar: np.ndarray
    dgbarsum: np.ndarray
    gapmin: float
    gapmax: float
    part2: list              # (ifile, ibin, gap centre, dGv1, dGv2, dGg, npts, c1, c2)
    part3: list              # (ibin, gap centre, <dGg>, <dGg norm>, pts, c1, c2, r)
    bar_iterations: list


def _bin(gap: float, gapmin: float, xint: float, nbins: int) -> int:
    """int((gap - gapmin)/xint) + 1 (qfep.f90:628); a degenerate range (all
    gaps equal: 0/0) goes to bin 1 and the index stays within 0..nbins+1,
    where qfep's result is undefined."""
    with np.errstate(all="ignore"):
        q = np.float64(gap - gapmin) / np.float64(xint)
    k = int(q) if math.isfinite(q) else (nbins + 1 if q > 0 else 0)
    return min(max(k + 1, 0), nbins + 1)


def analyze(inp: FepInput) -> FepResult:
    nfiles = len(inp.energies)
    ns = inp.energies[0].shape[1]
    rt, nskip = float(inp.rt), int(inp.nskip)
    alfa = np.zeros(ns)
    for k, a in enumerate(inp.alfa[: ns - 1]):
        alfa[k + 1] = a
    coeff = np.zeros(ns)
    coeff[: len(inp.coeff)] = inp.coeff[:ns]

    lam = np.zeros((nfiles, ns))
    npts = np.zeros(nfiles, dtype=int)
    avEQ = np.zeros((nfiles, ns, NEQ))
    V, VG, GAP, C1, C2, RX = [], [], [], [], [], []
    A, mu, eta, r0 = (np.zeros((4, 4)) for _ in range(4))
    for i, j, a, m, e, r in inp.evb:
        A[i - 1, j - 1], mu[i - 1, j - 1], eta[i - 1, j - 1], r0[i - 1, j - 1] = a, m, e, r
    nnoffd = len(inp.evb)

    def hij(i, j, r):      # qfep.f90:289-297, 0-based states
        if A[i, j] == 0.0:
            i, j = j, i
        return A[i, j] * math.exp(-mu[i, j] * (r - r0[i, j])) * math.exp(-eta[i, j] * (r - r0[i, j]) ** 2)
    gapmin, gapmax = 999.0, -999.0
    for f, raw in enumerate(inp.energies):
        eq = np.array(raw, dtype=np.float64)
        n = eq.shape[0]
        lam[f] = eq[0, :, I_LAMBDA]
        if inp.gas > 0:        # qfep.f90:257-263
            eq[:, :, I_TOTAL] = (eq[:, :, I_BOND] + eq[:, :, I_ANGLE] + eq[:, :, I_TORSION] + eq[:, :, I_IMPROPER]
                                 + eq[:, :, I_QQ_EL] + eq[:, :, I_QQ_VDW] + eq[:, :, I_RESTRAINT])
        acc = np.zeros((ns, NEQ))
        v = np.zeros((n, ns))
        vg = np.zeros(n)
        gap = np.zeros(n)
        c1, c2 = np.zeros(n), np.zeros(n)
        rx = np.array(inp.rxy[f], dtype=np.float64) if nnoffd > 0 else np.zeros(n)
        for ipt in range(n):
            if ipt + 1 > nskip:
                acc += eq[ipt]
            tot = eq[ipt, :, I_TOTAL] + alfa
            v[ipt] = tot
            if ns == 2:
                h = hij(0, 1, rx[ipt]) if nnoffd > 0 else 0.0
                vg[ipt] = 0.5 * (tot[0] + tot[1]) - 0.5 * math.sqrt((tot[0] - tot[1]) ** 2 + 4.0 * h ** 2)
                if nnoffd > 0:
                    c1[ipt] = 1.0 / (1.0 + ((vg[ipt] - tot[0]) / h) ** 2)
                    c2[ipt] = 1 - c1[ipt]
            elif nnoffd > 0:
                m = np.diag(tot)
                for i in range(ns):
                    for j in range(i):
                        m[i, j] = m[j, i] = hij(i, j, rx[ipt])
                vg[ipt] = float(np.min(np.linalg.eigvalsh(m)))
            else:
                vg[ipt] = float(np.min(tot))
            g = 0.0
            for st in range(ns):
                g = g + tot[st] * coeff[st]
            gap[ipt] = g
            if ipt + 1 > nskip:
                gapmin = min(gapmin, g) if g < gapmin else gapmin
                gapmax = g if g > gapmax else gapmax
        npts[f] = n
        if n <= nskip:
            raise ValueError("number of data sets in file %d is less than number of points to skip" % (f + 1))
        k = float(np.float32(1.0) / np.float32(n - nskip))
        avEQ[f] = acc * k
        V.append(v)
        VG.append(vg)
        GAP.append(gap)
        C1.append(c1)
        C2.append(c2)
        RX.append(rx)

    z = lambda: np.zeros(nfiles + 2)
    dgf, dgfsum, dgr, dgrsum, dG = z(), z(), z(), z(), z()
    dgti, dgtisum, dglu, dglusum, dgbar, dgbarsum = z(), z(), z(), z(), z(), z()
    part2, part3, bar_its = [], [], []
    if nfiles > 1:
        # Zwanzig forward (qfep.f90:392-421); arrays are 1-based in the reference
        for i in range(1, nfiles):
            s = 0.0
            for ipt in range(nskip, npts[i - 1]):
                v1 = 0.0
                v2 = 0.0
                for st in range(ns):
                    v1 = v1 + lam[i - 1, st] * V[i - 1][ipt, st]
                    v2 = v2 + lam[i, st] * V[i - 1][ipt, st]
                s = s + math.exp(-(v2 - v1) / rt)
            s = s / float(npts[i - 1] - nskip)
            dgf[i] = -rt * math.log(s)
            dgfsum[i + 1] = dgfsum[i] + dgf[i]
        # Zwanzig reverse (qfep.f90:424-445)
        for i in range(nfiles, 1, -1):
            s = 0.0
            for ipt in range(nskip, npts[i - 1]):
                v1 = 0.0
                v2 = 0.0
                for st in range(ns):
                    v1 = v1 + lam[i - 1, st] * V[i - 1][ipt, st]
                    v2 = v2 + lam[i - 2, st] * V[i - 1][ipt, st]
                s = s + math.exp(-(v2 - v1) / rt)
            s = s / float(npts[i - 1] - nskip)
            dgr[i] = -rt * math.log(s)
            dgrsum[i - 1] = dgrsum[i] + dgr[i]
        # TI between states 1 and 2 (qfep.f90:448-478); needs two states
        for i in range(1, nfiles + 1 if ns >= 2 else 1):
            s = 0.0
            for ipt in range(nskip, npts[i - 1]):
                s = s + (V[i - 1][ipt, 1] - V[i - 1][ipt, 0])
            dgti[i] = s / float(npts[i - 1] - nskip)
        for i in range(2, nfiles + 1):
            dlam = lam[i - 2, 0] - lam[i - 1, 0]
            dgtisum[i] = dgtisum[i - 1] + (0.5 * (dgti[i - 1] + dgti[i]) * dlam)
        # overlap sampling, Lu et al. (qfep.f90:481-521)
        for i in range(1, nfiles):
            s = 0.0
            for ipt in range(nskip, npts[i - 1]):
                v1 = v2 = 0.0
                for st in range(ns):
                    v1 = v1 + lam[i - 1, st] * V[i - 1][ipt, st]
                    v2 = v2 + lam[i, st] * V[i - 1][ipt, st]
                s = s + math.exp(-((v2 - v1) / 2) / rt)
            sumf = s / float(npts[i - 1] - nskip)
            s = 0.0
            for ipt in range(nskip, npts[i]):
                v1 = v2 = 0.0
                for st in range(ns):
                    v1 = v1 + lam[i - 1, st] * V[i][ipt, st]
                    v2 = v2 + lam[i, st] * V[i][ipt, st]
                s = s + math.exp(((v2 - v1) / 2) / rt)
            sumb = s / float(npts[i] - nskip)
            dglu[i] = -rt * math.log(sumf / sumb)
            dglusum[i + 1] = dglusum[i] + dglu[i]
        # BAR, iterated from the overlap estimate (qfep.f90:524-578)
        for i in range(1, nfiles):
            konst = dglu[i]
            fel = 1.0
            its = 0
            nf, nr = npts[i - 1] - nskip, npts[i] - nskip
            # real(n)/real(m): a single-precision quotient (qfep.f90:534-535)
            nfnr = float(np.float32(nf) / np.float32(nr))
            nrnf = float(np.float32(nr) / np.float32(nf))
            while fel > 0.001:
                s = 0.0
                for ipt in range(nskip, npts[i - 1]):
                    v1 = v2 = 0.0
                    for st in range(ns):
                        v1 = v1 + lam[i - 1, st] * V[i - 1][ipt, st]
                        v2 = v2 + lam[i, st] * V[i - 1][ipt, st]
                    s = s + 1 / (1 + (nfnr * math.exp(((v2 - v1) - konst) / rt)))
                sumf = s / float(nf)
                s = 0.0
                for ipt in range(nskip, npts[i]):
                    v1 = v2 = 0.0
                    for st in range(ns):
                        v1 = v1 + lam[i - 1, st] * V[i][ipt, st]
                        v2 = v2 + lam[i, st] * V[i][ipt, st]
                    s = s + 1 / (1 + (nrnf * math.exp((-(v2 - v1) + konst) / rt)))
                sumb = s / float(nr)
                dgbar[i] = -rt * math.log((sumf / sumb) * math.exp(-konst / rt) * nfnr)
                fel = abs(konst - dgbar[i])
                konst = dgbar[i]
                its += 1
            bar_its.append(its)
            dgbarsum[i + 1] = dgbarsum[i] + dgbar[i]
        # mean of forward and reverse (qfep.f90:586-589)
        for i in range(2, nfiles + 1):
            dG[i] = dG[i - 1] + 0.5 * (dgf[i - 1] - dgr[i])

        # Part 2: reaction free energy by energy-gap bins (qfep.f90:611-710)
        nbins = int(inp.nbins)
        xint = (gapmax - gapmin) / float(nbins)
        nb = nbins + 2
        binsum = np.zeros((nb, 4))
        ptsum = np.zeros(nb, dtype=int)
        for f in range(nfiles):
            avdvv = np.zeros((ns, nb))
            avdvg = np.zeros(nb)
            avc1 = np.zeros(nb)
            avc2 = np.zeros(nb)
            avr = np.zeros(nb)
            sumv = np.zeros((ns, nb))
            sumg = np.zeros(nb)
            nbinpts = np.zeros(nb, dtype=int)
            for ipt in range(nskip, npts[f]):
                ib = _bin(GAP[f][ipt], gapmin, xint, nbins)
                veff = 0.0
                for st in range(ns):
                    veff = veff + lam[f, st] * V[f][ipt, st]
                avdvv[:, ib] += V[f][ipt] - veff
                avdvg[ib] += VG[f][ipt] - veff
                avc1[ib] += C1[f][ipt]
                avc2[ib] += C2[f][ipt]
                if nnoffd > 0:
                    avr[ib] += RX[f][ipt]
                nbinpts[ib] += 1
            for ib in range(1, nbins + 1):
                if nbinpts[ib] != 0:
                    rn = float(np.float32(nbinpts[ib]))      # /real(nbinpts)
                    avc1[ib] /= rn
                    avc2[ib] /= rn
                    avr[ib] /= rn
                    avdvv[:, ib] /= nbinpts[ib]
                    avdvg[ib] /= nbinpts[ib]
            for ipt in range(nskip, npts[f]):
                ib = _bin(GAP[f][ipt], gapmin, xint, nbins)
                veff = 0.0
                for st in range(ns):
                    veff = veff + lam[f, st] * V[f][ipt, st]
                for st in range(ns):
                    sumv[st, ib] += math.exp(-(V[f][ipt, st] - veff - avdvv[st, ib]) / rt)
                sumg[ib] += math.exp(-(VG[f][ipt] - veff - avdvg[ib]) / rt)
            for ib in range(1, nbins + 1):
                if nbinpts[ib] >= inp.nmin:
                    binsum[ib, 1] += avc1[ib] * nbinpts[ib]
                    binsum[ib, 2] += avc2[ib] * nbinpts[ib]
                    binsum[ib, 3] += avr[ib] * nbinpts[ib]
                    sv = sumv[:, ib] / float(nbinpts[ib])
                    sg = sumg[ib] / float(nbinpts[ib])
                    ptsum[ib] += nbinpts[ib]
                    sumv2 = np.array([-rt * math.log(sv[st]) + avdvv[st, ib] for st in range(ns)])
                    sumg2 = -rt * math.log(sg) + avdvg[ib]
                    dGv = dG[f + 1] + sumv2
                    dGg = dG[f + 1] + sumg2
                    binsum[ib, 0] += dGg * nbinpts[ib]
                    part2.append((f, ib, gapmin + ib * xint - xint / 2.0, float(dGv[0]),
                                  float(dGv[1]) if ns > 1 else 0.0, float(dGg), int(nbinpts[ib]),
                                  float(avc1[ib]), float(avc2[ib])))
        for ib in range(1, nbins + 1):
            if ptsum[ib] >= inp.nmin:
                binsum[ib] /= float(ptsum[ib])
        mn = min(0.0, float(np.min(binsum[1:nbins + 1, 0])))
        for ib in range(1, nbins + 1):
            if ptsum[ib] >= inp.nmin:
                part3.append((ib, gapmin + ib * xint - xint / 2.0, float(binsum[ib, 0]), float(binsum[ib, 0] - mn),
                              int(ptsum[ib]), float(binsum[ib, 1]), float(binsum[ib, 2]), float(binsum[ib, 3])))
    return FepResult(lam, npts, avEQ, dgf, dgfsum, dgr, dgrsum, dG, dgti, dgtisum, dglu, dglusum, dgbar, dgbarsum,
                     gapmin, gapmax, part2, part3, bar_its)
