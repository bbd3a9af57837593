"""EVB off-diagonal functions on the host: the FEP file's [off_diagonals]
(qatom.f90:1515-1555), their checks, and the off-diagonal record qdyn adds
to every energy-file frame (nrgy.f90:60-65, 116)."""
import numpy as np
import pytest

from q_b200 import EQ_NAMES, QBError, System, append_energy, synth
from q_b200.fep import read_en, read_offdiag

OFFD = [(1, 2, 1, 2, 50.0, 0.5), (2, 1, 3, 5, 20.0, 1.0)]


def test_off_diagonals_parsed(tmp_path):
    g = synth.fep_solute(str(tmp_path / "evb"), off_diagonals=OFFD)
    s = System.open(g.inp)
    v = s.view
    assert v.noffd == 2
    got = [(v.offd_i[k], v.offd_j[k], v.offd_k[k] + 1, v.offd_l[k] + 1, v.offd_A[k], v.offd_mu[k]) for k in range(2)]
    assert got == OFFD


@pytest.mark.parametrize("bad", [(1, 1, 1, 2, 50.0, 0.5), (1, 3, 1, 2, 50.0, 0.5), (1, 2, 1, 9, 50.0, 0.5)])
def test_invalid_off_diagonals_are_refused(tmp_path, bad):
    """Equal or out-of-range states and Q atoms beyond the FEP file's atoms
    stop qatom_load_fep (qatom.f90:1539-1553)."""
    g = synth.fep_solute(str(tmp_path / "evb"), off_diagonals=[bad])
    with pytest.raises(QBError) as e:
        System.open(g.inp)
    assert e.value.code == 3 and "off_diagonals" in str(e.value)     # QB_ERR_PARSE


def test_energy_frame_with_off_diagonal_record(tmp_path):
    """Per frame: one record per state, then noffd x (int32 i, int32 j,
    real8 Hij, real8 r_kl) in one record; frames without functions keep the
    empty record."""
    path = str(tmp_path / "x.en")
    EQ = np.arange(2 * len(EQ_NAMES), dtype=np.float64).reshape(2, -1)
    ij = np.array([[1, 2], [2, 1]])
    hr = np.array([[12.5, 1.44], [3.25, 2.7]])
    append_energy(path, EQ, (ij, hr))
    append_energy(path, EQ + 1, (ij, hr * 2))
    raw = open(path, "rb").read()
    assert len(raw) == 2 * (2 * (8 + 4 + 8 * len(EQ_NAMES)) + 8 + 48)
    assert np.array_equal(read_en(path, 2), np.stack([EQ, EQ + 1]))
    od = read_offdiag(path, 2)
    assert od.shape == (2, 2, 4)
    assert np.array_equal(od[1], np.column_stack([ij, hr * 2]))
    append_energy(str(tmp_path / "y.en"), EQ)
    assert read_offdiag(str(tmp_path / "y.en"), 2).shape == (1, 0, 4)


def test_oracle_two_state_evb_is_the_secular_determinant():
    """The 2-state closed form of qfep (qfep.f90:310-316) is the lower
    eigenvalue of [[E1, H12], [H12, E2]], and c1^2 is the squared first
    component of its eigenvector: the restatement against numpy."""
    from oracle.qfep_oracle import FepInput
    from oracle.qfep_oracle import analyze as oracle_analyze
    rng = np.random.default_rng(5)
    S = []
    for k in range(2):
        e = rng.normal(0.0, 3.0, (40, 2, 15))
        e[:, :, 0] = [1.0 - k, float(k)]
        S.append(e)
    rxy = [rng.uniform(1.5, 3.0, 40) for _ in S]
    evb = [(2, 1, 15.0, 0.5, 0.02, 2.0)]        # given as (2, 1): A(1, 2) is 0
    o = oracle_analyze(FepInput(S, 0.592, 0, nbins=4, nmin=1, coeff=[1.0, -1.0], evb=evb, rxy=rxy))
    assert o.part2, "no bins"
    e = S[0][:, :, 1]
    h = 15.0 * np.exp(-0.5 * (rxy[0] - 2.0)) * np.exp(-0.02 * (rxy[0] - 2.0) ** 2)
    for k in range(40):
        w, v = np.linalg.eigh(np.array([[e[k, 0], h[k]], [h[k], e[k, 1]]]))
        vg = 0.5 * (e[k, 0] + e[k, 1]) - 0.5 * np.sqrt((e[k, 0] - e[k, 1]) ** 2 + 4 * h[k] ** 2)
        assert abs(vg - w[0]) < 1e-10
        c1 = 1.0 / (1.0 + ((vg - e[k, 0]) / h[k]) ** 2)
        assert abs(c1 - v[0, 0] ** 2) < 1e-10


def _strip_couplings(path):
    """The FEP file without its coupling sections (same bonds and terms)."""
    out, skip = [], False
    for line in open(path).read().split("\n"):
        if line.startswith("["):
            skip = line.strip() in ("[angle_couplings]", "[torsion_couplings]", "[improper_couplings]")
        if not skip:
            out.append(line)
    twin = path.replace(".fep", "_plain.fep")
    open(twin, "w").write("\n".join(out))
    return twin


def _dihedral(x, i, j, k, l):
    rji, rjk, rkl = x[i] - x[j], x[k] - x[j], x[l] - x[k]
    nj, nk = np.cross(rji, rjk), -np.cross(rjk, rkl)
    phi = np.arccos(np.clip(nj @ nk / np.linalg.norm(nj) / np.linalg.norm(nk), -1, 1))
    return -phi if rjk @ np.cross(nj, nk) < 0 else phi


def test_oracle_morse_couplings_match_numpy(tmp_path, oracle):
    """Q angles, torsions and impropers coupled to a Morse bond (qangle,
    qtorsion, qimproper with EVB couplings): against the same system without
    the coupling sections, each coupled term's energy is scaled by
    gamma = EMorseD of the bond, or 1 - EMorseD for a flagged improper; in
    state 2 the bond is absent and EMorseD keeps state 1's value."""
    from q_b200.inputs import derive_inp, inp_sections
    g = synth.fep_solute(str(tmp_path / "c"), q_bonded=True, morse_couplings=True)
    twin = derive_inp(g.inp, "plain.inp", set_keys={"files": {"fep": _strip_couplings(g.fep).split("/")[-1]}})
    res = {}
    for name, inp in (("cpl", g.inp), ("plain", twin)):
        s = System.open(inp, lambdas=(0.5, 0.5))
        o = oracle.create(s)
        o.final_energy()
        res[name] = (s, o.energy_vectors()[1], o.coords().reshape(-1, 3))
    s, EQc, x = res["cpl"]
    EQp = res["plain"][1]
    v = s.view
    S = v.nstates
    assert v.nqangle and [v.qang_cpl[k] for k in range(v.nqangle)].count(0) >= 1
    b = 0                                            # the coupled bond: Morse in state 1 only
    i, j = v.qbnd_i[b], v.qbnd_j[b]
    r = np.linalg.norm(x[j] - x[i])
    db = r - v.qbnd_r0[b * S + 0]
    fe = np.exp(-v.qbnd_amz[b * S + 0] * db)
    emorse = -(fe * fe - 2 * fe) if db > 0 else 1.0
    want = {"angle": np.zeros(S), "torsion": np.zeros(S), "improper": np.zeros(S)}
    for a in range(v.nqangle):
        if v.qang_cpl[a] != b:
            continue
        ia, ja, ka = v.qang_i[a], v.qang_j[a], v.qang_k[a]
        u, w = x[ia] - x[ja], x[ka] - x[ja]
        ang = np.arccos(np.clip(u @ w / np.linalg.norm(u) / np.linalg.norm(w), -1, 1))
        for st in range(S):
            if v.qang_on[a * S + st]:
                ae = 0.5 * v.qang_fk[a * S + st] * (ang - v.qang_th0[a * S + st]) ** 2
                want["angle"][st] += ae * (emorse - 1.0)
    for t in range(v.nqtor):
        if v.qtor_cpl[t] != b:
            continue
        phi = _dihedral(x, v.qtor_i[t], v.qtor_j[t], v.qtor_k[t], v.qtor_l[t])
        for st in range(S):
            if v.qtor_on[t * S + st]:
                pe = v.qtor_fk[t * S + st] * (1 + np.cos(v.qtor_rmult[t * S + st] * phi - v.qtor_deltor[t * S + st]))
                want["torsion"][st] += pe * (emorse - 1.0)
    for t in range(v.nqimp):
        if v.qimp_cpl[t] != b:
            continue
        phi = _dihedral(x, v.qimp_i[t], v.qimp_j[t], v.qimp_k[t], v.qimp_l[t])
        g_ = 1.0 - emorse if v.qimp_cpl_flag[t] == 1 else emorse
        for st in range(S):
            if v.qimp_on[t * S + st]:
                arg = phi - v.qimp_imp0[t * S + st]
                arg -= 2 * np.pi * np.round(arg / (2 * np.pi))
                want["improper"][st] += 0.5 * v.qimp_fk[t * S + st] * arg * arg * (g_ - 1.0)
    for term, want_d in want.items():
        k = list(EQ_NAMES).index(term)
        assert np.allclose(EQc[:, k] - EQp[:, k], want_d, atol=1e-9, rtol=1e-9), term


def test_coupling_refusals(tmp_path):
    """A coupling to a bond that is harmonic in some state stops
    qatom_load_fep (bond_harmonic_in_any_state, qatom.f90:1423); a coupled
    term present in a state before its bond is would read EMorseD of a
    previous step, and is refused."""
    g = synth.fep_solute(str(tmp_path / "c"), q_bonded=True, morse_couplings=True)
    txt = open(g.fep).read()
    # bond 1 harmonic in state 1: the coupling is refused as qatom does
    bad1 = txt.replace("[change_bonds]\n1 2 1 0", "[change_bonds]\n1 2 3 0")
    open(g.fep, "w").write(bad1)
    with pytest.raises(QBError) as e:
        System.open(g.inp)
    assert e.value.code == 3 and "harmonic" in str(e.value)
    # the bond only in state 2, its coupled angles in both
    bad2 = txt.replace("[change_bonds]\n1 2 1 0", "[change_bonds]\n1 2 0 1")
    open(g.fep, "w").write(bad2)
    with pytest.raises(QBError) as e:
        System.open(g.inp)
    assert e.value.code == 4 and "previous step" in str(e.value)
