"""Q-Q pair options on the host: [soft_pairs] (exponential repulsion between
two Q atoms) and qq_use_library_charges, under both LJ combination rules.
The oracle's Q-Q energies are checked against a numpy statement of
nonbond_qq / nonbon2_qq and their _lib_charges variants (md.f90:10763,
10872, 9385, 9494), summed over the pair list the view holds."""
import numpy as np
import pytest

from q_b200 import EQ_NAMES, System, synth


def _arr(p, n):
    return np.array([p[k] for k in range(n)])


def qq_numpy(v, x):
    """(qq_el, qq_vdw) per state from the view's nbqq lists."""
    S, nq = v.nstates, v.nqat
    arith, lib = v.ivdw_rule == 2, bool(v.qq_use_library_charges)
    ncol = v.natyps + nq
    crg = _arr(v.crg, v.natom).astype(np.float64)
    qcrg = _arr(v.qcrg, nq * S).astype(np.float64)
    qiac = _arr(v.qiac, nq * S)
    qa, qb = _arr(v.qavdw, 3 * v.nqlib), _arr(v.qbvdw, 3 * v.nqlib)
    iqseq = _arr(v.iqseq, nq)
    cnt, off = _arr(v.nbqq_count, S), _arr(v.nbqq_off, S)
    out = np.zeros((S, 2))
    for st in range(S):
        for p in range(off[st], off[st] + cnt[st]):
            iq, j, jq, lj, el = v.nbqq_iq[p], v.nbqq_j[p], v.nbqq_jq[p], v.nbqq_ljcod[p], v.nbqq_el_scale[p]
            if jq < 0:
                continue
            assert v.qvdw_flag
            i = iqseq[iq]
            qi = crg[i] if lib else qcrg[iq * S + st]
            qj = crg[j] if lib else qcrg[jq * S + st]
            d = np.linalg.norm(x[j] - x[i])
            Vel = qi * qj / d * el * (v.el14_scale if lj == 3 else 1.0)
            ti, tj = qiac[iq * S + st], qiac[jq * S + st]
            ai, aj = qa[3 * ti + lj - 1], qa[3 * tj + lj - 1]
            bi, bj = qb[3 * ti + lj - 1], qb[3 * tj + lj - 1]
            if lj == 2:
                V = ai * aj * np.exp(-bi * bj * d)
            else:
                r6 = 1.0 / (d ** 6 + v.sc_lookup[(iq * ncol + v.natyps + jq) * S + st])
                if arith:
                    s6 = (ai + aj) ** 6
                    V = bi * bj * s6 * s6 * r6 * r6 - 2.0 * bi * bj * s6 * r6
                else:
                    V = ai * aj * r6 * r6 - bi * bj * r6
            out[st] += (Vel, V)
    return out


@pytest.fixture(scope="module")
def qq_systems(tmp_path_factory):
    root = tmp_path_factory.mktemp("qq")
    return {(rule, lib): synth.fep_solute(str(root / ("r%d_%d" % (rule, lib))), vdw_rule=rule, soft_pairs=3,
                                          library_charges=bool(lib))
            for rule in (1, 2) for lib in (0, 1)}


@pytest.mark.parametrize("rule", [1, 2])
@pytest.mark.parametrize("lib", [0, 1])
def test_oracle_qq_energies_match_numpy(qq_systems, oracle, rule, lib):
    s = System.open(qq_systems[(rule, lib)].inp, lambdas=(0.4, 0.6))
    v = s.view
    assert v.qq_use_library_charges == lib and v.ivdw_rule == rule
    ljc = [v.nbqq_ljcod[p] for p in range(sum(_arr(v.nbqq_count, v.nstates)))]
    assert ljc.count(2) == 3 * v.nstates                   # the soft pairs, in every state
    o = oracle.create(s)
    o.final_energy()
    _, EQ = o.energy_vectors()
    want = qq_numpy(v, o.coords().reshape(-1, 3))
    k_el, k_vdw = list(EQ_NAMES).index("qq_el"), list(EQ_NAMES).index("qq_vdw")
    assert np.allclose(EQ[:, k_el], want[:, 0], atol=1e-9, rtol=1e-12)
    assert np.allclose(EQ[:, k_vdw], want[:, 1], atol=1e-9, rtol=1e-12)


def test_library_charges_make_qq_electrostatics_state_independent(qq_systems, oracle):
    """With library charges the Q-Q electrostatics of both states use the
    topology charges: state 2's zeroed charges no longer switch them off."""
    E = {}
    for lib in (0, 1):
        s = System.open(qq_systems[(1, lib)].inp, lambdas=(0.4, 0.6))
        o = oracle.create(s)
        o.final_energy()
        E[lib] = o.energy_vectors()[1][:, list(EQ_NAMES).index("qq_el")]
    assert E[0][1] == 0.0 and E[0][0] != 0.0               # state 2 charges are zero
    assert E[1][0] == pytest.approx(E[1][1], rel=1e-12)    # same charges, same pair list


@pytest.mark.parametrize("rule", [1, 2])
def test_library_charges_on_q_neighbour_pairs(qq_systems, oracle, rule):
    """Q-atom to bonded-neighbour pairs of the Q-Q list keep the Q atom's
    state charge under the geometric rule (nonbond_qq_lib_charges) but take
    its topology charge under the arithmetic one (nonbon2_qq_lib_charges sets
    qi = crg(i) for every pair): the qp_el difference between library and
    state charges is exactly those pairs' charge change."""
    runs = {}
    for lib in (0, 1):
        s = System.open(qq_systems[(rule, lib)].inp, lambdas=(0.4, 0.6))
        o = oracle.create(s)
        o.final_energy()
        runs[lib] = (s, o.energy_vectors()[1], o.coords().reshape(-1, 3))
    s, EQ1, x = runs[1]
    EQ0, x0 = runs[0][1], runs[0][2]
    assert np.array_equal(x, x0)
    v = s.view
    S = v.nstates
    crg = _arr(v.crg, v.natom).astype(np.float64)
    qcrg = _arr(v.qcrg, v.nqat * S).astype(np.float64)
    iqseq = _arr(v.iqseq, v.nqat)
    want = np.zeros(S)
    for st in range(S):
        for p in range(v.nbqq_off[st], v.nbqq_off[st] + v.nbqq_count[st]):
            iq, j, jq, lj, el = v.nbqq_iq[p], v.nbqq_j[p], v.nbqq_jq[p], v.nbqq_ljcod[p], v.nbqq_el_scale[p]
            if jq >= 0 or rule == 1:
                continue
            i = iqseq[iq]
            d = np.linalg.norm(x[j] - x[i])
            want[st] += (crg[i] - qcrg[iq * S + st]) * crg[j] / d * el * (v.el14_scale if lj == 3 else 1.0)
    k = list(EQ_NAMES).index("qp_el")
    assert np.allclose(EQ1[:, k] - EQ0[:, k], want, atol=1e-9, rtol=1e-12)
    if rule == 2:
        assert np.any(np.abs(want) > 1e-3)
