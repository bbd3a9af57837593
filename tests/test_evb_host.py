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
