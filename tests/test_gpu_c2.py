"""The protein-ligand sphere (3000-atom polymer around the FEP ligand in a
25 A sphere, atoms beyond 23 A excluded and restrained, Q cut-off 99) and the
p_restrain family, GPU engine against the oracle.

These are the systems where nonbond_pp (md.f90:10387), fix_shell
(md.f90:1414) and p_restrain (md.f90:12940) carry weight."""
import numpy as np
import pytest

from q_b200 import E_NAMES, FP64, MIXED, Batch, System

from tests.test_gpu_parity import E_TOL, G_TOL, assert_energies, grad_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2(tmp_path_factory):
    from q_b200 import synth
    return synth.polymer_sphere(str(tmp_path_factory.mktemp("c2") / "c2"), seed=1234)


def test_c2_trajectory_matches_oracle(c2, oracle):
    """Step 0 (output record), the energy records of steps 10 and 20, and the
    post-loop evaluation after 25 steps: every term within 1e-3 kcal/mol,
    gradients within 1e-4.  The excluded atoms' fix_shell restraint and the
    ~2e5 solute-solute pairs are part of every record."""
    s = System.open(c2.inp, seed=11)
    v = s.view
    nexcl = int(np.ctypeslib.as_array(v.excl, shape=(v.natom,)).sum())
    assert nexcl > 500 and v.nat_solute > 3000
    b = Batch([s], precision=FP64)
    b.run(25)
    o = oracle.create(s)
    o.run(25)
    for kind in (0, 1):
        sg, Eg, EQg = b.history(0, kind)
        so, Eo, EQo = o.history(kind)
        assert list(sg) == list(so) and len(sg) > 0
        for r in range(len(sg)):
            assert_energies(Eg[r], EQg[r], Eo[r], EQo[r])
    # the excluded atoms have moved off their restraint positions by step 20
    E = dict(zip(E_NAMES, b.history(0, 1)[1][-1]))
    assert E["rst_fix"] > 1e-2 and abs(E["pp_vdw"]) > 1.0
    w = b.workload()
    assert w[2] > 1e5          # solute-solute pairs
    b.final_energy()
    o.final_energy()
    Eg, EQg = b.energy_vectors(0)
    Eo, EQo = o.energy_vectors()
    assert_energies(Eg, EQg, Eo, EQo)
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL


def test_c2_mixed_precision_single_point(c2, oracle):
    """The benchmarked engine on the same system: energies of a recording
    step and the packed FP32 force path against the oracle."""
    s = System.open(c2.inp, seed=11)
    b = Batch([s], precision=MIXED)
    b.evaluate(energies=True)
    o = oracle.create(s)
    o.final_energy()
    Eg, EQg = b.energy_vectors(0)
    Eo, EQo = o.energy_vectors()
    assert_energies(Eg, EQg, Eo, EQo)
    b.evaluate(energies=False)
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL


def test_p_restrain_terms_match_oracle(tmp_path, oracle):
    """Sequence restraints (to the topology coordinates, centre of geometry
    and of mass, with and without hydrogens), atom position restraints,
    per-state distance and angle restraints, and wall restraints on the FEP
    solute (p_restrain, md.f90:12940-13276), against the oracle over 20 steps:
    rst_protein and the per-state restraint energies are non-zero."""
    from q_b200 import synth
    from q_b200.inputs import derive_inp
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234)
    inp = derive_inp(g.inp, "rst.inp", set_rows={
        "sequence_restraints": ["1 10 5.0 0 0", "11 30 2.0 1 1", "31 56 1.0 1 2"],
        "atom_restraints": ["12 0.5 -0.3 0.2 4.0 4.0 2.0 0", "40 -1.0 0.5 0.0 3.0 3.0 3.0 1"],
        "distance_restraints": ["1 9 1.0 2.0 10.0 0", "2 20 2.5 3.0 8.0 1", "5 33 1.5 2.5 6.0 2"],
        "angle_restraints": ["1 2 3 100.0 20.0 0", "4 5 6 120.0 15.0 2"],
        "wall_restraints": ["1 56 4.0 5.0 0.5 1.0 1", "1 10 1.5 10.0 0.5 2.0 0"],
    })
    systems = [System.open(inp, lambdas=lam, seed=7) for lam in ((0.5, 0.5), (0.8, 0.2))]
    b = Batch(systems, precision=FP64)
    b.run(20)
    runs = []
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.run(20)
        runs.append(o)
        for kind in (0, 1):
            sg, Eg, EQg = b.history(k, kind)
            so, Eo, EQo = o.history(kind)
            assert list(sg) == list(so)
            for r in range(len(sg)):
                assert_energies(Eg[r], EQg[r], Eo[r], EQo[r])
        E = dict(zip(E_NAMES, b.history(k, 0)[1][0]))
        assert abs(E["rst_protein"]) > 1e-3
        EQ = b.history(k, 0)[2][0]
        assert np.max(np.abs(EQ[:, -1])) > 1e-6      # per-state restraint energy
    # the post-loop evaluation at the coordinates both reached
    b.final_energy()
    for k, o in enumerate(runs):
        o.final_energy()
        Eg, EQg = b.energy_vectors(k)
        Eo, EQo = o.energy_vectors()
        assert_energies(Eg, EQg, Eo, EQo)
        assert grad_err(b.gradient(k), o.gradient()) < G_TOL
