"""Set-up tables pinned independently of the library's own readers.

The oracle consumes the library's prepared system (qb_sysview), so a mistake
in parsing or in the set-up tables would reach both sides of every GPU-vs-
oracle test.  These tests re-derive two of those tables straight from the
input files' text, with their own small parsers and numpy, and compare them
with the view:

* the soft-core table sc_lookup (qatom.f90:1556-1685): both LJ combination
  rules, with softcore_use_max_potential on and off, alphas non-zero in both
  states and zero for some atoms, so every branch of the table is taken;
* the Q-atom connectivity qconn (make_qconn / find_bonded, md.f90:7312-7405):
  a breadth-first search over the solute bond graph of each state (topology
  bonds not redefined by a Q bond, plus the Q bonds present in that state),
  with the special exclusions of [excluded_pairs] set to 0.
"""
from __future__ import annotations

import math
import re
from collections import deque

import numpy as np
import pytest

from q_b200 import System, synth


# ------------------------------------------------------------ text readers

def read_top(path):
    """The few topology blocks the tables need, read from the .top text."""
    lines = open(path).read().split("\n")
    out = {}

    def ints_after(k, n):
        vals = []
        while len(vals) < n:
            k += 1
            vals += [int(t) for t in lines[k].split()]
        return vals, k

    def floats_after(k, n):
        vals = []
        while len(vals) < n:
            k += 1
            vals += [float(t) for t in lines[k].split()]
        return vals, k

    for k, l in enumerate(lines):
        if "= Total no. of atoms, no. of solute atoms" in l:
            out["natom"], out["nsol"] = (int(t) for t in l.split("=")[0].split())
        elif "= No. of bonds, no. of solute bonds" in l:
            nb, nbs = (int(t) for t in l.split("=")[0].split())
            v, _ = ints_after(k, 3 * nb)
            out["bonds"] = [tuple(v[3 * b:3 * b + 3]) for b in range(nbs)]
        elif "= No. of atom types" in l and "natyps" not in out and ":" not in l.split("=")[1][:15]:
            out["natyps"] = int(l.split("=")[0])
        elif "= vdW combination rule" in l:
            out["rule"] = int(l.split("=")[0])
        elif l.startswith(("sqrt (Aii) normal:", "R*ii normal:")):
            # sqrt(A) under the geometric rule, R* under the arithmetic one
            out["a1"], _ = floats_after(k, out["natyps"])
        elif l.startswith(("sqrt (Bii) normal:", "epsilon ii normal:")):
            out["b1"], _ = floats_after(k, out["natyps"])
    return out


def read_fep(path):
    """Sections of a FEP file: name -> list of token lists (comments dropped)."""
    sec, cur = {}, None
    for raw in open(path).read().split("\n"):
        l = re.split(r"[!#]", raw)[0].strip()
        if not l:
            continue
        m = re.match(r"\[(.+)\]", l)
        if m:
            cur = m.group(1).strip().lower()
            sec.setdefault(cur, [])
        elif cur:
            sec[cur].append(l.split())
    return sec


def fep_key(sec, key, default=False):
    for toks in sec.get("fep", []):
        if toks[0].lower() == key:
            return toks[1].lower() in ("on", "1", "yes", "true")
    return default


# ----------------------------------------------------------- sc_lookup

def sc_lookup_statement(top, sec):
    """qatom_load_fep's soft-core table (qatom.f90:1604-1680) in numpy, with
    the topology's epsilons square-rooted for the arithmetic rule before the
    table is made (topology, md.f90:14747-14752) and the Q types' epsilons
    not yet (get_fep takes them at md.f90:1519-1523)."""
    S = int(next(t[1] for t in sec["fep"] if t[0].lower() == "states"))
    nq = len(sec["atoms"])
    qtype = {t[0]: (float(t[1]), float(t[2])) for t in sec["atom_types"]}
    qiac = np.array([[t[1 + s] for s in range(S)] for t in sorted(sec["change_atoms"], key=lambda t: int(t[0]))])
    alpha = np.zeros((nq, S))
    for t in sec.get("softcore", []):
        alpha[int(t[0]) - 1] = [float(v) for v in t[1:1 + S]]
    maxpot = fep_key(sec, "softcore_use_max_potential")
    nat = top["natyps"]
    aj_top = np.array(top["a1"])
    bj_top = np.array(top["b1"])
    arith = top["rule"] == 2
    if arith:
        bj_top = np.sqrt(np.abs(bj_top))
    sc = np.zeros((nq, nat + nq, S))
    for s in range(S):
        aq = np.array([qtype[qiac[i, s]][0] for i in range(nq)])
        bq = np.array([qtype[qiac[i, s]][1] for i in range(nq)])
        for i in range(nq):
            am = alpha[i, s]
            # Q atom against the topology's atom types
            if not maxpot:
                sc[i, :nat, s] = am
            elif am != 0:
                if arith:
                    sc[i, :nat, s] = ((-2 * math.sqrt(bq[i]) * bj_top
                                       + 2 * np.sqrt(bq[i] * bj_top ** 2 + am * math.sqrt(bq[i]) * bj_top))
                                      * (aq[i] + aj_top) ** 6 / (2 * am))
                else:
                    sc[i, :nat, s] = (-bq[i] * bj_top + np.sqrt((bq[i] * bj_top) ** 2 + 4 * am * aq[i] * aj_top)) / (2 * am)
            # Q atom against Q atoms
            for j in range(nq):
                a2 = alpha[j, s]
                if not (am > 1e-6 or a2 > 1e-6):
                    continue
                if maxpot:
                    t = min(am, a2)
                    if am == 0 or a2 == 0:
                        t = max(am, a2)
                    if arith:
                        p = bq[i] * bq[j]
                        sc[i, nat + j, s] = ((-2 * math.sqrt(p) + 2 * math.sqrt(p + t * math.sqrt(p)))
                                             * (aq[i] + aq[j]) ** 6 / (2 * t))
                    else:
                        sc[i, nat + j, s] = (-bq[i] * bq[j] + math.sqrt((bq[i] * bq[j]) ** 2 + 4 * t * aq[i] * aq[j])) / (2 * t)
                else:
                    sc[i, nat + j, s] = max(am, a2)
    return sc


def rewrite_fep(path, maxpot, alphas):
    """Set softcore_use_max_potential and the [softcore] alphas of a FEP file."""
    text = open(path).read()
    text = text.replace("[FEP]\n", "[FEP]\nsoftcore_use_max_potential %s\n" % ("on" if maxpot else "off"), 1)
    head, tail = text.split("[softcore]\n", 1)
    rest = tail.split("\n\n", 1)
    body = "\n".join("%d %s" % (k + 1, " ".join("%g" % a for a in row)) for k, row in enumerate(alphas))
    text = head + "[softcore]\n" + body + "\n" + ("\n" + rest[1] if len(rest) > 1 else "")
    open(path, "w").write(text)


@pytest.mark.parametrize("rule", [1, 2])
@pytest.mark.parametrize("maxpot", [False, True])
def test_sc_lookup_matches_statement_from_file_text(tmp_path, rule, maxpot):
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, vdw_rule=rule)
    # per (Q atom, state): some zeros, different non-zero values in both states
    alphas = [(0.0, 20.0), (5.0, 0.0), (12.5, 30.0), (0.0, 0.0), (7.0, 7.0), (2.5, 40.0), (0.0, 15.0), (9.0, 1.0)]
    rewrite_fep(g.fep, maxpot, alphas)
    sys_ = System.open(g.inp)
    v = sys_.view
    top, sec = read_top(g.top), read_fep(g.fep)
    ref = sc_lookup_statement(top, sec)
    nq, S, nat = v.nqat, v.nstates, top["natyps"]
    assert (nq, S, nat) == (8, 2, v.natyps)
    got = np.ctypeslib.as_array(v.sc_lookup, shape=(nq * (nat + nq) * S,)).reshape(nq, nat + nq, S)
    assert np.any(ref != 0)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)


# ---------------------------------------------------------------- qconn

def qconn_statement(top, sec, nq, S):
    """qconn[state, atom, q]: 1 for the Q atom itself, 2/3/4 for atoms one,
    two or three bonds away in that state's bond graph, 9 beyond, 0 for the
    special exclusions of [excluded_pairs]."""
    nsol = top["nsol"]
    qseq = [int(t[1]) - 1 for t in sorted(sec["atoms"], key=lambda t: int(t[0]))]
    qbonds = [(int(t[0]) - 1, int(t[1]) - 1, [int(c) for c in t[2:2 + S]]) for t in sec.get("change_bonds", [])]
    redefined = {frozenset((i, j)) for i, j, _ in qbonds}
    base = [(i - 1, j - 1) for i, j, _ in top["bonds"] if frozenset((i - 1, j - 1)) not in redefined]
    qc = np.full((S, nsol, nq), 9, dtype=np.int8)
    for s in range(S):
        adj = [[] for _ in range(nsol)]
        for i, j in base + [(i, j) for i, j, c in qbonds if c[s] > 0]:
            adj[i].append(j)
            adj[j].append(i)
        for q, a in enumerate(qseq):
            dist = {a: 0}
            dq = deque([a])
            while dq:
                u = dq.popleft()
                if dist[u] == 3:
                    continue
                for w in adj[u]:
                    if w not in dist:
                        dist[w] = dist[u] + 1
                        dq.append(w)
            for atom, d in dist.items():
                qc[s, atom, q] = d + 1
    iqatom = {a: q for q, a in enumerate(qseq)}
    for t in sec.get("excluded_pairs", []):
        i, j = int(t[0]) - 1, int(t[1]) - 1
        for s in range(S):
            if int(t[2 + s]) == 1:
                if i in iqatom:
                    qc[s, j, iqatom[i]] = 0
                if j in iqatom:
                    qc[s, i, iqatom[j]] = 0
    return qc


def test_qconn_matches_bond_graph_search(tmp_path):
    # Q bonds redefine the topology bonds among the Q atoms; the first is a
    # Morse bond present in state 1 and absent in state 2, so the two states'
    # graphs differ
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, q_bonded=True, morse_couplings=True)
    sec0 = read_fep(g.fep)
    assert any(int(t[3]) == 0 for t in sec0["change_bonds"])
    top = read_top(g.top)
    nsol = top["nsol"]
    qseq = [int(t[1]) - 1 for t in sec0["atoms"]]
    nonq = [a for a in range(nsol) if a not in qseq]
    # special exclusions: a Q-nonQ pair (all states, as md.f90:1627-1633
    # requires when a non-Q atom is involved) and a Q-Q pair in state 2 only
    with open(g.fep, "a") as f:
        f.write("\n[excluded_pairs]\n%d %d 1 1\n%d %d 0 1\n" % (qseq[0] + 1, nonq[-1] + 1, qseq[2] + 1, qseq[5] + 1))
    sys_ = System.open(g.inp)
    v = sys_.view
    nq, S = v.nqat, v.nstates
    sec = read_fep(g.fep)
    ref = qconn_statement(top, sec, nq, S)
    got = np.ctypeslib.as_array(v.qconn, shape=(S * nsol * nq,)).reshape(S, nsol, nq)
    # the broken bond changes some connectivities between the states
    assert np.any(ref[0] != ref[1])
    assert (ref == 0).sum() >= 3
    np.testing.assert_array_equal(got, ref)
