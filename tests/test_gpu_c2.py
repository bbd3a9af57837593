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


def test_any_atom_cutoffs_match_oracle(tmp_path, oracle):
    """Charge-group cut-offs on any atom pair (iuse_switch_atom 0 in the
    topology): nbpplis2_lrf, nbpwlis2_lrf and nbqplis2 (md.f90:4926, 6477,
    7664) and the LRF windows they imply, on the FEP solute in water.  Two
    lambda windows over 50 steps (two list rebuilds) against the oracle; the
    mixed-precision engine at one point.  The lists differ from the
    switch-atom ones on this system, so the test separates the two modes."""
    from q_b200 import synth
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, switch_atoms=0)
    systems = [System.open(g.inp, lambdas=lam, seed=5) for lam in ((0.5, 0.5), (0.9, 0.1))]
    assert systems[0].view.iuse_switch_atom == 0
    b = Batch(systems, precision=FP64)
    b.run(50)
    runs = []
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.run(50)
        runs.append(o)
        for kind in (0, 1):
            sg, Eg, EQg = b.history(k, kind)
            so, Eo, EQo = o.history(kind)
            assert list(sg) == list(so)
            for r in range(len(sg)):
                assert_energies(Eg[r], EQg[r], Eo[r], EQo[r])
    b.final_energy()
    for k, o in enumerate(runs):
        o.final_energy()
        Eg, EQg = b.energy_vectors(k)
        Eo, EQo = o.energy_vectors()
        assert_energies(Eg, EQg, Eo, EQo)
        assert grad_err(b.gradient(k), o.gradient()) < G_TOL
    # the switch-atom lists of the same coordinates are different
    w_any = b.workload()
    g1 = synth.fep_solute(str(tmp_path / "c1s"), seed=1234, switch_atoms=1)
    b1 = Batch([System.open(g1.inp, lambdas=(0.5, 0.5), seed=5)], precision=FP64)
    b1.run(1)
    b0 = Batch([System.open(g.inp, lambdas=(0.5, 0.5), seed=5)], precision=FP64)
    b0.run(1)
    assert b0.workload()[1] != b1.workload()[1]
    # mixed precision on the any-atom lists
    s = System.open(g.inp, lambdas=(0.5, 0.5), seed=5)
    bm = Batch([s], precision=MIXED)
    bm.evaluate(energies=True)
    o = oracle.create(s)
    o.final_energy()
    Eg, EQg = bm.energy_vectors(0)
    Eo, EQo = o.energy_vectors()
    assert_energies(Eg, EQg, Eo, EQo)
    bm.evaluate(energies=False)
    assert grad_err(bm.gradient(0), o.gradient()) < G_TOL


def test_c2_runs_its_list_cycles(c2):
    """The protein-ligand sphere runs stably under the engine: 300 mixed-
    precision steps (twelve list rebuilds) without a SHAKE failure or a
    non-finite energy, the temperature settling below 700 K."""
    s = System.open(c2.inp, seed=11)
    b = Batch([s], precision=MIXED)
    b.run(300)
    assert b.status(0) == 0
    assert b.temperature(0)[0] < 700.0
