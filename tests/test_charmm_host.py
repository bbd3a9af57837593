"""CHARMM topologies (ff_type 3) on the host: the optional Urey-Bradley
columns of the topology's angle codes and of the FEP file's angle_types, the
CHARMM rule for impropers a Q improper replaces, and the oracle's
urey_bradley (md.f90:904) against a numpy statement of the same term."""
import numpy as np
import pytest

from q_b200 import E_NAMES, EQ_NAMES, System, synth


def _ptr(p, n):
    return np.array([p[k] for k in range(n)])


@pytest.fixture(scope="module")
def charmm(tmp_path_factory):
    root = tmp_path_factory.mktemp("charmm")
    return {(ff, ub): synth.fep_solute(str(root / ("ff%d_%g" % (ff, ub))), ff_type=ff, q_bonded=True, ub_fk=ub)
            for ff, ub in ((3, 25.0), (3, 0.0), (2, 25.0))}


def test_urey_bradley_columns_parsed(charmm):
    s = System.open(charmm[(3, 25.0)].inp)
    v = s.view
    assert v.ff_type == 3
    na, nas = v.nangles, v.nangles_solute
    ufk, ur0 = _ptr(v.ang_ureyfk, na), _ptr(v.ang_ureyr0, na)
    assert np.all(ufk[:nas] == 25.0) and np.all(ur0[:nas] > 2.0)
    assert np.all(ufk[nas:] == 0.0)                       # the water angle has none
    S = v.nstates
    qfk = _ptr(v.qang_ureyfk, v.nqangle * S).reshape(-1, S)
    assert np.all(qfk[:, 0] == 25.0) and np.all(qfk[:, 1] == 12.5)
    # the same columns under AMBER are read and ignored (urey_bradley runs for CHARMM only)
    s2 = System.open(charmm[(2, 25.0)].inp)       # the view reads the System's memory: keep it
    w = s2.view
    assert not np.any(_ptr(w.ang_ureyfk, w.nangles)) and not np.any(_ptr(w.qang_ureyfk, w.nqangle * S))


@pytest.mark.parametrize("ff", [3, 2])
@pytest.mark.parametrize("swap", [False, True])
def test_improper_removal_rules(charmm, ff, swap):
    """md.f90:1571-1598: under CHARMM a topology improper goes when one of
    its ends is an end of a Q improper and both its centre atoms are among
    that Q improper's atoms; under the other force fields when its centre
    pair is the Q improper's.  With the Q impropers' last two atoms swapped
    the two rules part: CHARMM still removes the topology's impropers, the
    centre-pair rule keeps them."""
    from q_b200.inputs import derive_inp, inp_sections
    g = charmm[(ff, 25.0)]
    inp = g.inp
    if swap:
        fep_lines = open(g.fep).read().split("\n")
        k0 = fep_lines.index("[change_impropers]")
        for k in range(k0 + 1, len(fep_lines)):
            t = fep_lines[k].split()
            if len(t) < 6:
                break
            fep_lines[k] = " ".join([t[0], t[1], t[3], t[2]] + t[4:])
        fep2 = g.fep.replace(".fep", "_swap.fep")
        open(fep2, "w").write("\n".join(fep_lines))
        inp = derive_inp(g.inp, "swap.inp", set_keys={"files": {"fep": fep2.split("/")[-1]}})
    fep = inp_sections(fep2 if swap else g.fep)
    qimp = [tuple(int(t) - 1 for t in r.split()[:4]) for r in fep["change_impropers"]]
    top = open(g.top).read().split("\n")
    k = next(i for i, l in enumerate(top) if "No. of impropers" in l)
    nimp = int(top[k].split()[0])
    vals = " ".join(top[k + 1:k + 1 + (nimp + 1) // 2]).split()
    imps = [tuple(int(t) - 1 for t in vals[5 * m:5 * m + 4]) for m in range(nimp)]

    def removed(im, q):
        if ff == 3:
            ends = im[0] in (q[0], q[3]) or im[3] in (q[0], q[3])
            return ends and im[1] in q and im[2] in q
        return (im[1], im[2]) in ((q[1], q[2]), (q[2], q[1]))

    keep = [im for im in imps if not any(removed(im, q) for q in qimp)]
    s = System.open(inp)
    v = s.view
    got = [tuple(int(a) for a in t) for t in zip(*(_ptr(p, v.nimps) for p in (v.imp_i, v.imp_j, v.imp_k, v.imp_l)))]
    # shrink_topology fills a removed slot from the end of the list: compare as sets
    assert sorted(got) == sorted(keep)
    assert len(keep) == (nimp if (swap and ff == 2) else nimp - len(qimp))


def _ub_numpy(v, x):
    """Energy (solute, solvent) and gradient of k (|x_k - x_i| - r0)^2 over
    the view's angles."""
    na = v.nangles
    i, k = _ptr(v.ang_i, na), _ptr(v.ang_k, na)
    fk, r0 = _ptr(v.ang_ureyfk, na), _ptr(v.ang_ureyr0, na)
    rik = x[k] - x[i]
    d = np.linalg.norm(rik, axis=1)
    e = np.where(fk > 0, fk * (d - r0) ** 2, 0.0)
    g = np.zeros_like(x)
    du = np.where(fk > 0, 2 * fk * (d - r0) / d, 0.0)[:, None] * rik
    np.add.at(g, k, du)
    np.add.at(g, i, -du)
    return e[:v.nangles_solute].sum(), e[v.nangles_solute:].sum(), g


def test_oracle_urey_bradley_matches_numpy(charmm, oracle):
    """Same coordinates, UB constant 25 against 0: the difference in the
    oracle's angle energies and gradient is the Urey-Bradley term alone."""
    runs = {}
    for ub in (25.0, 0.0):
        s = System.open(charmm[(3, ub)].inp, lambdas=(0.3, 0.7))
        o = oracle.create(s)
        o.final_energy()
        E, EQ = o.energy_vectors()
        runs[ub] = (s, E, EQ, o.gradient().reshape(-1, 3), o.coords().reshape(-1, 3))
    s, E1, EQ1, g1, x = runs[25.0]
    _, E0, EQ0, g0, x0 = runs[0.0]
    assert np.array_equal(x, x0)
    ep, ew, g = _ub_numpy(s.view, x)
    names = list(E_NAMES)
    assert abs((E1[names.index("p_angle")] - E0[names.index("p_angle")]) - ep) < 1e-9
    assert abs(E1[names.index("w_angle")] - E0[names.index("w_angle")]) < 1e-12 and ew == 0.0
    # Q-angle Urey-Bradley: energy in the state's angle term, no gradient
    # (qurey_bradley computes du and never applies it, md.f90:14034)
    v = s.view
    S, na = v.nstates, v.nqangle
    qi, qk = _ptr(v.qang_i, na), _ptr(v.qang_k, na)
    d = np.linalg.norm(x[qk] - x[qi], axis=1)
    fk = _ptr(v.qang_ureyfk, na * S).reshape(na, S)
    r0 = _ptr(v.qang_ureyr0, na * S).reshape(na, S)
    on = _ptr(v.qang_on, na * S).reshape(na, S)
    eq = (np.where(on > 0, fk * (d[:, None] - r0) ** 2, 0.0)).sum(axis=0)
    ka = list(EQ_NAMES).index("angle")
    assert np.allclose(EQ1[:, ka] - EQ0[:, ka], eq, atol=1e-9, rtol=0)
    assert np.max(np.abs((g1 - g0) - g)) < 1e-9
