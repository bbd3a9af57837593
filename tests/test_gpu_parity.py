"""GPU engine (libqb, through its C ABI) against the CPU oracle.

Both run the same prepared system.  Tolerances follow the parity bar of this
path: every energy term and per-state energy within 1e-3 kcal/mol, gradients
within 1e-4 relative (per atom, relative to the larger of the atom's gradient
norm and 1% of the RMS gradient), in FP64.
"""
import numpy as np
import pytest

from q_b200 import FP64, MIXED, Batch, E_NAMES, System

pytestmark = pytest.mark.gpu

E_TOL = 1e-3
G_TOL = 1e-4


def grad_err(g, ref):
    g = g.reshape(-1, 3)
    ref = ref.reshape(-1, 3)
    nrm = np.linalg.norm(ref, axis=1)
    floor = 0.01 * np.sqrt(np.mean(nrm ** 2)) + 1e-12
    return float(np.max(np.linalg.norm(g - ref, axis=1) / np.maximum(nrm, floor)))


def energy_diffs(Eg, EQg, Eo, EQo):
    out = {n: abs(a - b) for n, a, b in zip(E_NAMES, Eg, Eo)}
    if EQo.size:
        out["EQ"] = float(np.max(np.abs(EQg - EQo)))
    return out


def assert_energies(Eg, EQg, Eo, EQo, tol=E_TOL):
    d = energy_diffs(Eg, EQg, Eo, EQo)
    bad = {k: v for k, v in d.items() if v > tol}
    assert not bad, bad


def single_point(oracle, inp):
    sys_ = System.open(inp)
    b = Batch([sys_], precision=FP64)
    b.run(1)
    o = oracle.create(sys_)
    o.run(1)
    return sys_, b, o


@pytest.mark.parametrize("case", ["test1", "benzene"])
def test_step0_energies_and_gradient(golden, oracle, case):
    inp = str(golden / case / "eq1.inp")
    sys_, b, o = single_point(oracle, inp)
    # energies of step 0 are the first output record of both engines
    _, Eg, EQg = b.history(0, 0)
    _, Eo, EQo = o.history(0)
    assert_energies(Eg[0], EQg[0], Eo[0], EQo[0])


@pytest.mark.parametrize("case", ["test1", "benzene"])
def test_gradient_single_point(golden, oracle, case):
    inp = str(golden / case / "eq1.inp")
    sys_ = System.open(inp)
    b = Batch([sys_], precision=FP64)
    b.final_energy()          # lists + potential at the starting coordinates
    o = oracle.create(sys_)
    o.final_energy()
    Eg, EQg = b.energy_vectors(0)
    Eo, EQo = o.energy_vectors()
    assert_energies(Eg, EQg, Eo, EQo)
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL


def test_test1_trajectory_matches_oracle(golden, oracle):
    """100 steps of eq1 (LRF, SHAKE, restraints, watpol): output records at
    steps 0 and 50 and the FINAL energies."""
    inp = str(golden / "test1" / "eq1.inp")
    sys_ = System.open(inp)
    b = Batch([sys_], precision=FP64)
    o = oracle.create(sys_)
    b.run(100)
    o.run(100)
    sg, Eg, EQg = b.history(0, 0)
    so, Eo, EQo = o.history(0)
    assert list(sg) == list(so) == [0, 50]
    for k in range(2):
        assert_energies(Eg[k], EQg[k], Eo[k], EQo[k])
    b.final_energy()
    o.final_energy()
    Eg, EQg = b.energy_vectors(0)
    Eo, EQo = o.energy_vectors()
    assert_energies(Eg, EQg, Eo, EQo)
    x_err = np.max(np.abs(b.coords(0) - o.coords()))
    assert x_err < 1e-6


def test_batch_of_systems_is_independent(golden, oracle):
    """A batch of different systems gives each system its own-run results."""
    a = System.open(str(golden / "test1" / "eq1.inp"))
    c = System.open(str(golden / "benzene" / "eq1.inp"))
    b = Batch([a, c, a], precision=FP64)
    b.run(3)
    o = oracle.create(a)
    o.run(3)
    _, Eo, EQo = o.history(0)
    for s in (0, 2):
        _, Eg, EQg = b.history(s, 0)
        assert_energies(Eg[0], EQg[0], Eo[0], EQo[0])
    assert np.max(np.abs(b.coords(0) - b.coords(2))) < 1e-9


@pytest.fixture(scope="module")
def synthetic(tmp_path_factory):
    from q_b200 import synth
    root = tmp_path_factory.mktemp("synth")
    return {"c0": synth.water_sphere(str(root / "c0"), radius=15.0, seed=1234),
            "c1": synth.fep_solute(str(root / "c1"), seed=1234),
            # more waters than one shared-memory chunk of the water-water kernel
            "c0_r25": synth.water_sphere(str(root / "c0_r25"), radius=25.0, seed=99),
            # more waters than one mixed-precision chunk
            "c0_r27": synth.water_sphere(str(root / "c0_r27"), radius=27.0, seed=7)}


@pytest.mark.parametrize("case", ["c0", "c1", "c0_r25"])
def test_synthetic_single_point(synthetic, oracle, case):
    """Benchmark-shaped systems: water sphere (LRF, restraints, watpol) and the
    8-Q-atom two-state soft-core FEP solute; energies and gradient."""
    sys_ = System.open(synthetic[case].inp)
    b = Batch([sys_], precision=FP64)
    b.final_energy()
    o = oracle.create(sys_)
    o.final_energy()
    Eg, EQg = b.energy_vectors(0)
    Eo, EQo = o.energy_vectors()
    assert_energies(Eg, EQg, Eo, EQo)
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL


def test_synthetic_windows_trajectory(synthetic, oracle):
    """Three lambda windows of the FEP system in one batch, 50 steps (two list
    rebuilds), each against its own oracle run."""
    inp = synthetic["c1"].inp
    lams = [(1.0, 0.0), (0.5, 0.5), (0.0, 1.0)]
    systems = [System.open(inp, lambdas=l, seed=7) for l in lams]
    b = Batch(systems, precision=FP64)
    b.run(50)
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.run(50)
        sg, Eg, EQg = b.history(k, 0)
        so, Eo, EQo = o.history(0)
        assert list(sg) == list(so)
        for r in range(len(sg)):
            assert_energies(Eg[r], EQg[r], Eo[r], EQo[r])
        # trajectories separate slowly from summation-order differences (1e-16)
        assert np.max(np.abs(b.coords(k) - o.coords())) < 1e-4


@pytest.mark.parametrize("case", ["c1", "c0_r25", "c0_r27"])
def test_mixed_precision_error_vs_fp64(synthetic, case):
    """The mixed-precision engine against the FP64 engine on the same
    coordinates, at the parity bar: the energies of a recording step (FP64
    water-water pairs, FP32 LRF multipole sums) within 1e-3 kcal/mol per term,
    and the gradient of a non-recording step (packed FP32 water-water forces)
    within 1e-4 relative."""
    sys_ = System.open(synthetic[case].inp)
    b64 = Batch([sys_], precision=FP64)
    b32 = Batch([sys_], precision=MIXED)
    b64.final_energy()
    b32.evaluate(energies=True)
    E64, EQ64 = b64.energy_vectors(0)
    E32, EQ32 = b32.energy_vectors(0)
    assert_energies(E32, EQ32, E64, EQ64)
    assert np.max(np.abs(EQ32 - EQ64), initial=0.0) < 1e-6
    b32.evaluate(energies=False)
    assert grad_err(b32.gradient(0), b64.gradient(0)) < G_TOL


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_water_pass_threads(synthetic, precision):
    """The water pass with a thread per water or per water atom: the same
    per-atom terms in the same order, so the same records (packed FP32 ones
    too), energies and forces, to the rounding of the atomic sums."""
    sys_ = System.open(synthetic["c1"].inp)
    out = []
    for per_atom in (0, 1):
        b = Batch([sys_], precision=precision)
        b.set_tuning(water_pass_per_atom=per_atom)
        assert b.tuning()["water_pass_per_atom"] == per_atom
        b.evaluate(energies=True)
        E, EQ = b.energy_vectors(0)
        b.evaluate(energies=False)
        out.append((E, EQ, b.gradient(0)))
    (E0, Q0, g0), (E1, Q1, g1) = out
    assert np.max(np.abs(E0 - E1)) < 1e-8 and np.max(np.abs(Q0 - Q1), initial=0.0) < 1e-8
    assert np.max(np.abs(g0 - g1)) < 1e-9


def _restart_copy(tmp_path, inp, name, x, v, theta):
    """A copy of `inp` that starts from coordinates x and velocities v (and the
    polarisation restraint's theta corrections) through a restart file."""
    import os
    from q_b200.api import write_restart
    from q_b200.inputs import derive_inp
    re_path = os.path.join(os.path.dirname(inp), name + ".re")
    write_restart(re_path, x, v, theta)
    return derive_inp(inp, name + ".inp", set_keys={"files": {"restart": name + ".re"}},
                      drop_keys={"md": ["random_seed", "initial_temperature"]})


def test_mixed_engine_matches_oracle_on_bench_shapes(synthetic, oracle, tmp_path):
    """The benchmarked mixed-precision engine against the oracle on the bench's
    own shapes in one batch: two lambda windows of the FEP solute and water
    spheres of 15, 25 and 27 A (one of them beyond one staging chunk).  At
    step 0 every energy record matches; then after 50 mixed-precision steps
    (two list rebuilds) each system's state is handed to the oracle through a
    restart file and both evaluate the same coordinates: energies within
    1e-3 kcal/mol (recording step) and gradients within 1e-4 (the packed FP32
    force path).  Trajectories themselves are not compared: FP32 forces make
    them separate from an FP64 trajectory by ~1e-5 A within tens of steps."""
    specs = [(synthetic["c1"].inp, (1.0, 0.0), 3), (synthetic["c1"].inp, (0.3, 0.7), 4),
             (synthetic["c0"].inp, None, 5), (synthetic["c0_r25"].inp, None, 6), (synthetic["c0_r27"].inp, None, 7)]
    systems = [System.open(inp, lambdas=lam, seed=seed) for inp, lam, seed in specs]
    b = Batch(systems, precision=MIXED)
    b.run(50)
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.run(1)
        sg, Eg, EQg = b.history(k, 0)
        so, Eo, EQo = o.history(0)
        assert sg[0] == so[0] == 0
        assert_energies(Eg[0], EQg[0], Eo[0], EQo[0])
        assert b.status(k) == 0
    states = [(b.coords(k), b.velocities(k), b.theta_corr(k, s.view.nwpolr_shell)) for k, s in enumerate(systems)]
    for k, (s, (inp, lam, seed)) in enumerate(zip(systems, specs)):
        x, v, th = states[k]
        again = System.open(_restart_copy(tmp_path, inp, "bench_shape_%d" % k, x, v, th), lambdas=lam)
        bb = Batch([again], precision=MIXED)
        bb.evaluate(energies=True)
        o = oracle.create(again)
        o.final_energy()
        Eg, EQg = bb.energy_vectors(0)
        Eo, EQo = o.energy_vectors()
        assert_energies(Eg, EQg, Eo, EQo)
        bb.evaluate(energies=False)
        assert grad_err(bb.gradient(0), o.gradient()) < G_TOL


def test_mixed_sizes_in_one_batch(synthetic, oracle):
    """Small and large spheres and the FEP system in one batch (one staging
    chunk size for all): each system matches its own oracle run."""
    names = ["c0", "c0_r25", "c1"]
    systems = [System.open(synthetic[n].inp) for n in names]
    b = Batch(systems, precision=FP64)
    b.final_energy()
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.final_energy()
        Eg, EQg = b.energy_vectors(k)
        Eo, EQo = o.energy_vectors()
        assert_energies(Eg, EQg, Eo, EQo)
        assert grad_err(b.gradient(k), o.gradient()) < G_TOL


def test_graph_replay_matches_direct_launches(synthetic, monkeypatch):
    """Steps replayed from captured CUDA graphs (the default) against the same
    kernels launched one by one: same records, same coordinates (to FP64
    atomic-order noise)."""
    inp = synthetic["c1"].inp
    runs = []
    for env in (None, "1"):
        if env:
            monkeypatch.setenv("QB_NO_GRAPHS", env)
        s = System.open(inp, lambdas=(0.5, 0.5), seed=3)
        b = Batch([s], precision=FP64)
        b.run(60)          # crosses two list rebuilds
        steps, E, EQ = b.history(0, 0)
        runs.append((steps, E, EQ, b.coords(0)))
    (s0, E0, Q0, x0), (s1, E1, Q1, x1) = runs
    assert list(s0) == list(s1)
    assert np.max(np.abs(E0 - E1)) < 1e-6 and np.max(np.abs(Q0 - Q1)) < 1e-6
    assert np.max(np.abs(x0 - x1)) < 1e-8


@pytest.mark.parametrize("kicked", ["water", "solute"])
def test_failed_system_stops_at_its_step(synthetic, kicked):
    """A system whose constraints fail stops where md_run stops (md.f90:14533
    'shake failure'): the error names the failing step, the system's
    positions stay those of that step (start = x - v*dt), its records stop,
    and the other systems of the batch carry on.  The failure is made by a
    40 A kick on one hydrogen, which no SHAKE sweep can absorb in 1000
    iterations (rigid-water kernel for a water hydrogen, the block-per-molecule
    kernel for a solute hydrogen)."""
    from q_b200 import QBError
    inp = synthetic["c1"].inp
    systems = [System.open(inp, lambdas=(0.5, 0.5), seed=3 + k) for k in range(2)]
    b = Batch(systems, precision=FP64)
    b.run(10)
    nsol = 56
    atom = nsol + 1 if kicked == "water" else nsol - 1   # first water's H1 / last solute hydrogen
    x10 = b.coords(1)
    v = b.velocities(1).reshape(-1, 3)
    v[atom] = (1000.0, 0.0, 0.0)
    b.set_velocities(1, v.reshape(-1))
    with pytest.raises(QBError) as err:
        b.run(20)
    assert err.value.code == 5 and "system 1 " in str(err.value) and "at step 10" in str(err.value)
    assert b.status(0) == 0 and b.status(1) == 5
    dt = systems[1].view.dt
    start = b.coords(1) - b.velocities(1) * dt
    assert np.max(np.abs(start - x10)) < 1e-9
    assert list(b.history(0, 1)[0]) == [10, 20]
    assert len(b.history(1, 1)[0]) == 0


def test_perturbations_with_different_q_atoms_in_one_batch(tmp_path, oracle):
    """Systems of one batch may carry different Q-atom sets (4 and 11 atoms,
    other charge and epsilon scalings): each matches the oracle."""
    from q_b200 import synth
    base = synth.fep_solute(str(tmp_path / "c1"), seed=1234)
    a = synth.perturbation(base, "pa", [0, 3, 9, 30], 0.3, 0.8)
    b = synth.perturbation(base, "pb", [1, 2, 4, 5, 6, 7, 8, 10, 12, 14, 16], 0.9, 0.35)
    sa = System.open(a.inp, lambdas=(0.7, 0.3), seed=2)
    sb = System.open(b.inp, lambdas=(0.2, 0.8), seed=3)
    batch = Batch([sa, sb, sa], precision=FP64)
    batch.final_energy()
    for k, s in ((0, sa), (1, sb), (2, sa)):
        o = oracle.create(s)
        o.final_energy()
        Eg, EQg = batch.energy_vectors(k)
        Eo, EQo = o.energy_vectors()
        assert_energies(Eg, EQg, Eo, EQo)
        assert grad_err(batch.gradient(k), o.gradient()) < G_TOL


def test_tuning_changes_only_rounding(synthetic, oracle):
    """The run-time choices of the step kernels (LRF tiles per block, water
    chunk, waters per water-water block, the water pass's threads, side
    streams) change only the order of atomic sums: two copies of
    a batch, one with other settings, give the same records and coordinates
    to rounding; out-of-range settings are refused; after autotuning the
    batch still matches the oracle."""
    from q_b200 import QBError
    inp = synthetic["c1"].inp
    runs = []
    for setting in (None, dict(lrf_tiles_per_block=1, ww_chunk=256, side_streams=0, ww_waters_per_block=32,
                               water_pass_per_atom=0)):
        s = System.open(inp, lambdas=(0.4, 0.6), seed=5)
        b = Batch([s], precision=FP64)
        t = b.tuning()
        assert t["ww_chunk_min"] <= 256 <= t["ww_chunk_max"] and t["ww_chunk"] == t["ww_chunk_max"]
        if setting:
            b.set_tuning(**setting)
            t = b.tuning()
            assert (t["lrf_tiles_per_block"], t["ww_chunk"], t["side_streams"], t["ww_waters_per_block"],
                    t["water_pass_per_atom"]) == (1, 256, 0, 32, 0)
        b.run(60)          # crosses two list rebuilds
        runs.append((b.history(0, 0), b.coords(0)))
    ((s0, E0, Q0), x0), ((s1, E1, Q1), x1) = runs
    assert list(s0) == list(s1)
    assert np.max(np.abs(E0 - E1)) < 1e-6 and np.max(np.abs(Q0 - Q1)) < 1e-6
    assert np.max(np.abs(x0 - x1)) < 1e-8
    with pytest.raises(QBError):
        b.set_tuning(ww_chunk=100)
    with pytest.raises(QBError):
        b.set_tuning(lrf_tiles_per_block=0)
    with pytest.raises(QBError):
        b.set_tuning(ww_waters_per_block=48)
    with pytest.raises(QBError):
        b.set_tuning(ww_waters_per_block=288)
    s = System.open(inp, lambdas=(0.4, 0.6), seed=5)
    b = Batch([s, s], precision=FP64)
    r = b.autotune(50)
    assert r["trials"] >= 3 and r["ms_per_step"] <= r["ms_per_step_before"]
    assert r["ww_chunk_min"] <= r["ww_chunk"] <= r["ww_chunk_max"] and r["lrf_tiles_per_block"] >= 1
    # the chosen setting, applied to a fresh batch, matches the oracle
    b = Batch([s], precision=FP64)
    b.set_tuning(**{k: r[k] for k in ("lrf_tiles_per_block", "ww_chunk", "side_streams", "ww_waters_per_block",
                                      "water_pass_per_atom")})
    b.final_energy()
    o = oracle.create(s)
    o.final_energy()
    Eg, EQg = b.energy_vectors(0)
    Eo, EQo = o.energy_vectors()
    assert_energies(Eg, EQg, Eo, EQo)
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL


@pytest.fixture(scope="module")
def arithmetic(tmp_path_factory):
    """The water sphere and FEP solute written with the arithmetic LJ rule
    (R*, epsilon) and, beside them, with the geometric rule: the same sigma
    and epsilon either way."""
    from q_b200 import synth
    root = tmp_path_factory.mktemp("arith")
    out = {}
    for rule in (1, 2):
        out[("c0", rule)] = synth.water_sphere(str(root / ("c0_%d" % rule)), radius=15.0, seed=1234, vdw_rule=rule)
        out[("c1", rule)] = synth.fep_solute(str(root / ("c1_%d" % rule)), seed=1234, vdw_rule=rule)
    return out


@pytest.mark.parametrize("case", ["c0", "c1"])
def test_arithmetic_rule_matches_oracle(arithmetic, oracle, case):
    """nonbon2_* (md.f90:8972-10230): every LJ term with R*_i + R*_j and
    sqrt(eps_i) sqrt(eps_j), soft-core Q-atom terms included, over 20 steps."""
    s = System.open(arithmetic[(case, 2)].inp, lambdas=(0.3, 0.7) if case == "c1" else None, seed=3)
    assert s.view.ivdw_rule == 2
    b = Batch([s], precision=FP64)
    b.run(20)
    o = oracle.create(s)
    o.run(20)
    sg, Eg, EQg = b.history(0, 0)
    so, Eo, EQo = o.history(0)
    assert list(sg) == list(so)
    for k in range(len(sg)):
        assert_energies(Eg[k], EQg[k], Eo[k], EQo[k])
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL


def test_arithmetic_rule_equals_geometric_for_like_pairs(arithmetic):
    """Between atoms of one type both rules give the same pair potential
    (sigma_ij = sigma either way): the water sphere's O-O van der Waals energy
    agrees between its arithmetic and geometric topologies to the precision
    the geometric one prints sqrt(A), sqrt(B) with (2 decimals).  (Unlike types
    differ by construction: arithmetic means of R* against geometric means of
    sigma.)"""
    E = {}
    for rule in (1, 2):
        s = System.open(arithmetic[("c0", rule)].inp)
        b = Batch([s], precision=FP64)
        b.final_energy()
        E[rule] = b.energy_vectors(0)[0]
    k = list(E_NAMES).index("ww_vdw")
    assert abs(E[2][k] - E[1][k]) <= 2e-3 * abs(E[1][k])
    k = list(E_NAMES).index("ww_el")
    assert abs(E[2][k] - E[1][k]) < 1e-9          # same charges; sums differ only in atomic order


@pytest.fixture(scope="module")
def charmm_pair(tmp_path_factory):
    """The FEP solute as a CHARMM topology (Urey-Bradley 1-3 terms,
    harmonic impropers) and as its AMBER twin, both with the bonded terms
    among the Q atoms redefined per state in the FEP file (Q bonds, one of
    them Morse in state 2; Q angles, with Urey-Bradley columns under CHARMM;
    Q torsions; Q impropers)."""
    from q_b200 import synth
    root = tmp_path_factory.mktemp("charmm")
    return {ff: synth.fep_solute(str(root / ("ff%d" % ff)), seed=1234, ff_type=ff, q_bonded=True)
            for ff in (3, 2)}


def _worst_atoms(g, ref, n=5):
    d = np.linalg.norm((g - ref).reshape(-1, 3), axis=1)
    return [(int(a), float(d[a])) for a in np.argsort(-d)[:n]]


def test_charmm_and_q_bonded_match_oracle(charmm_pair, oracle):
    """urey_bradley (md.f90:904), qurey_bradley (13992, energy only),
    qbond with Morse and harmonic types (14060), qangle (13896), qtorsion
    (14262), qimproper (14117) and the CHARMM improper set: a CHARMM system
    and an AMBER one in one batch, each against the oracle at step 0 and
    over 20 steps of dynamics."""
    systems = [System.open(charmm_pair[ff].inp, lambdas=(0.3, 0.7), seed=3) for ff in (3, 2)]
    assert [s.view.ff_type for s in systems] == [3, 2]
    assert all(s.view.nqbond and s.view.nqangle and s.view.nqtor and s.view.nqimp for s in systems)
    b = Batch(systems, precision=FP64)
    b.final_energy()
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.final_energy()
        Eo, EQo = o.energy_vectors()
        Eg, EQg = b.energy_vectors(k)
        assert_energies(Eg, EQg, Eo, EQo)
        err = grad_err(b.gradient(k), o.gradient())
        assert err < G_TOL, (s.view.ff_type, err, _worst_atoms(b.gradient(k), o.gradient()))
    b = Batch(systems, precision=FP64)
    b.run(20)
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.run(20)
        sg, Eg, EQg = b.history(k, 0)
        so, Eo, EQo = o.history(0)
        assert list(sg) == list(so)
        for m in range(len(sg)):
            assert_energies(Eg[m], EQg[m], Eo[m], EQo[m])
        assert grad_err(b.gradient(k), o.gradient()) < G_TOL


@pytest.fixture(scope="module")
def qq_options(tmp_path_factory):
    from q_b200 import synth
    root = tmp_path_factory.mktemp("qqopt")
    return [synth.fep_solute(str(root / ("r%d_%d" % (rule, lib))), vdw_rule=rule, soft_pairs=3, library_charges=bool(lib))
            for rule in (1, 2) for lib in (0, 1)]


def test_soft_pairs_and_library_charges_match_oracle(qq_options, oracle):
    """Q-Q soft pairs (A_i A_j exp(-B_i B_j r), nonbond_qq / nonbon2_qq) and
    qq_use_library_charges (nonbond_qq_lib_charges, nonbon2_qq_lib_charges)
    under both combination rules: four systems in one batch, 20 steps."""
    systems = [System.open(g.inp, lambdas=(0.4, 0.6), seed=5) for g in qq_options]
    assert [(s.view.ivdw_rule, s.view.qq_use_library_charges) for s in systems] == [(1, 0), (1, 1), (2, 0), (2, 1)]
    b = Batch(systems, precision=FP64)
    b.run(20)
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.run(20)
        sg, Eg, EQg = b.history(k, 0)
        so, Eo, EQo = o.history(0)
        assert list(sg) == list(so)
        for m in range(len(sg)):
            assert_energies(Eg[m], EQg[m], Eo[m], EQo[m])
        err = grad_err(b.gradient(k), o.gradient())
        assert err < G_TOL, (k, err, _worst_atoms(b.gradient(k), o.gradient()))


@pytest.fixture(scope="module")
def h_lj(tmp_path_factory):
    """Water with Lennard-Jones on its hydrogens: under the arithmetic rule
    (nonbon2_ww, nonbon2_qw) and as geometric-rule 3-atom solvent
    (nonbond_3atomsolvent, nonbond_qw_3atom), a water sphere and the FEP
    solute of each, and a plain SPC sphere."""
    from q_b200 import synth
    root = tmp_path_factory.mktemp("hlj")
    h = synth.TIP3P_H_LJ
    return {
        "w_arith": synth.water_sphere(str(root / "wa"), radius=14.0, vdw_rule=2, water_h_lj=h),
        "w_3atom": synth.water_sphere(str(root / "w3"), radius=14.0, solvent_type=1, water_h_lj=h),
        "q_arith": synth.fep_solute(str(root / "qa"), vdw_rule=2, water_h_lj=h),
        "q_3atom": synth.fep_solute(str(root / "q3"), solvent_type=1, water_h_lj=h),
        "w_spc": synth.water_sphere(str(root / "ws"), radius=12.0),
    }


def test_water_hydrogen_lj_matches_oracle(h_lj, oracle):
    """O-H and H-H Lennard-Jones in the water-water and Q-water terms (with
    the hydrogens' own soft-core shift), five systems in one batch over 20
    steps; the SPC sphere in that batch shows the variant leaves systems
    without hydrogen LJ as they were."""
    names = ["w_arith", "w_3atom", "q_arith", "q_3atom", "w_spc"]
    systems = [System.open(h_lj[n].inp, lambdas=(0.4, 0.6) if n.startswith("q") else None, seed=7) for n in names]
    assert [s.view.ww_hlj for s in systems] == [1, 1, 1, 1, 0]
    b = Batch(systems, precision=FP64)
    b.run(20)
    for k, s in enumerate(systems):
        o = oracle.create(s)
        o.run(20)
        sg, Eg, EQg = b.history(k, 0)
        so, Eo, EQo = o.history(0)
        assert list(sg) == list(so)
        for m in range(len(sg)):
            assert_energies(Eg[m], EQg[m], Eo[m], EQo[m])
        err = grad_err(b.gradient(k), o.gradient())
        assert err < G_TOL, (names[k], err, _worst_atoms(b.gradient(k), o.gradient()))


def test_water_hydrogen_lj_mixed_precision(h_lj):
    """The FP32 water-water variant with hydrogen LJ against FP64, as for
    SPC water: within the mixed path's stated energy budget."""
    s = System.open(h_lj["w_arith"].inp)
    b64 = Batch([s], precision=FP64)
    b32 = Batch([s], precision=MIXED)
    b64.final_energy()
    b32.evaluate(energies=True)
    e = dict(zip(E_NAMES, np.abs(b32.energy_vectors(0)[0] - b64.energy_vectors(0)[0])))
    assert max(e.values()) < E_TOL, e
    # the FP32 variant with hydrogen LJ serves the steps that record no energies
    b32.evaluate(energies=False)
    assert grad_err(b32.gradient(0), b64.gradient(0)) < G_TOL


def test_engine_step_matches_fortran_restart(golden):
    """The GPU engine's one MD step of the benzene run against the restart
    Fortran qdyn wrote after it (test/3.shake/p-p/benzene, Q5_data/eq1.re),
    the pin of the oracle's step in tests/test_oracle_golden.py."""
    from tests.test_oracle_golden import RE_V_RTOL, read_fortran_re
    _, x, v, _ = read_fortran_re(str(golden / "benzene" / "eq1.re"))
    s = System.open(str(golden / "benzene" / "eq1.inp"))
    b = Batch([s], precision=FP64)
    b.run(1)
    assert np.max(np.abs(b.coords(0) - x)) < 1e-9
    np.testing.assert_allclose(b.velocities(0), v, rtol=RE_V_RTOL, atol=1e-12 + RE_V_RTOL * np.abs(v).max())
