"""Periodic box (use_PBC) on the host: the set-up read from the files, the
restart file's box records, the box's cut-off checks, and the oracle's
nearest-image terms against an independent numpy restatement, under whole
molecule lattice shifts, put_back_in_box and Monte Carlo volume moves.

The reference ships no periodic-box test case or golden vector; the oracle's
box path is the sphere path (pinned against the reference's own tests) with
the nearest image of md.f90's *_box routines, so these tests pin the image
handling itself.
"""
import os

import numpy as np
import pytest

from q_b200 import QBError, System, synth, write_restart

EDGE = 30.0


@pytest.fixture(scope="module")
def box_inputs(tmp_path_factory):
    root = tmp_path_factory.mktemp("pbc")
    return {
        "nvt": synth.fep_box(str(root / "nvt"), edge=EDGE, seed=1234),
        "nolrf": synth.fep_box(str(root / "nolrf"), edge=EDGE, seed=1234, lrf=None),
        "npt": synth.fep_box(str(root / "npt"), edge=EDGE, seed=1234, constant_pressure=True, volume_change=10,
                             max_volume_displ=400.0),
    }


def _inp_with(g, tmp_path, name, **changes):
    """A copy of g's .inp beside its files with lines replaced."""
    txt = open(g.inp).read()
    for a, b in changes.items():
        txt = txt.replace(a, b)
    p = os.path.join(os.path.dirname(g.inp), name + ".inp")
    with open(p, "w") as f:
        f.write(txt)
    return p


def test_box_setup_from_files(box_inputs):
    g = box_inputs["npt"]
    s = System.open(g.inp)
    v = s.view
    assert v.use_pbc == 1
    assert list(v.boxlength) == [EDGE] * 3 and list(v.boxcenter) == [0.0] * 3
    assert v.constant_pressure == 1 and v.ivolume_cycle == 10 and v.pressure_seed == 3781
    assert v.max_vol_displ == 400.0
    # 1 bar in kcal/mol/A^3 with the reference's single-precision factor (md.f90:2619)
    assert v.pressure == float(np.float32(1.43836e-5))
    assert v.put_solute_back_in_box == 1 and v.put_solvent_back_in_box == 1 and v.rigid_box_center == 0
    assert v.qswitch == v.iqseq[0]
    # no excluded atoms, shell or polarisation in a box
    assert v.nexats == 0 and v.nshellats == 0 and v.nwpolr_shell == 0
    assert not any(v.excl[i] for i in range(v.natom))
    # molecule masses (md.f90:13861-13882)
    for m in (0, 1, v.nmol - 1):
        a, b = v.istart_mol[m], v.istart_mol[m + 1]
        tot = 0.0
        for j in range(a, b):   # in atom order (Python's sum() compensates)
            tot += v.type_mass[v.iac[j]]
        assert v.mol_mass_inv[m] == 1.0 / tot
    for j in (0, v.nat_solute, v.natom - 1):
        assert v.mass_box[j] == float(np.float32(1.0) / np.float32(v.winv[j]))


def test_box_restart_records_round_trip(box_inputs, tmp_path):
    g = box_inputs["nvt"]
    s = System.open(g.inp)
    v = s.view
    n3 = 3 * v.natom
    x = np.array([v.x0[k] for k in range(n3)])
    vel = np.zeros(n3)
    box = np.array([31.0, 30.5, 30.25, 0.5, -0.25, 0.125])
    re = os.path.join(os.path.dirname(g.inp), "with_box.re")
    write_restart(re, x, vel, None, box)
    raw = open(re, "rb").read()
    # records: (nat3, x), (nat3, v), (3 doubles), (3 doubles)
    assert len(raw) == 2 * (8 + 4 + 8 * n3) + 2 * (8 + 24)
    inp = _inp_with(g, tmp_path, "restarted", **{"random_seed 1\n": "", "initial_temperature 298\n": "",
                                                  "final pbc.re": "final pbc.re\nrestart with_box.re"})
    s2 = System.open(inp)
    v2 = s2.view
    assert list(v2.boxlength) == list(box[:3]) and list(v2.boxcenter) == list(box[3:])


def test_box_too_small_for_the_cut_offs(box_inputs, tmp_path):
    g = box_inputs["nvt"]
    txt = open(g.top).read().replace("  30.000  30.000  30.000 = Size of box", "  19.000  30.000  30.000 = Size of box")
    top = os.path.join(os.path.dirname(g.top), "small.top")
    open(top, "w").write(txt)
    inp = _inp_with(g, tmp_path, "small", **{"topology pbc.top": "topology small.top"})
    with pytest.raises(QBError) as e:
        System.open(inp)
    assert e.value.code == 3 and "Solute-solute cut-off radii too large" in str(e.value)


def _nearest_image_ww(x, ns, nwat, L, rc, qo, qh, A, B):
    """Water-water energies of nonbond_ww_spc_box: molecule pairs with O-O
    nearest image within rc, each molecule pair at the image of its O-O
    vector, 9 Coulomb terms and O-O Lennard-Jones."""
    O = x[ns::3][:nwat]
    el = vdw = 0.0
    q = np.array([qo, qh, qh])
    for i in range(nwat):
        d = O - O[i]
        t = L * np.round(d / L)
        r2 = np.sum((d - t) ** 2, axis=1)
        js = [j for j in range(nwat) if j != i and r2[j] <= rc * rc]
        for j in js:
            if j < i:
                continue
            xi = x[ns + 3 * i: ns + 3 * i + 3]
            xj = x[ns + 3 * j: ns + 3 * j + 3] - t[j]
            for a in range(3):
                for b in range(3):
                    r = np.linalg.norm(xj[b] - xi[a])
                    el += float(np.float32(q[a]) * np.float32(q[b])) / r
                    if a == 0 and b == 0:
                        vdw += A / r ** 12 - B / r ** 6
    return el, vdw


def test_oracle_nearest_image_water_energies(box_inputs, oracle):
    """The oracle's water-water energies at the first step against a numpy
    nearest-image restatement (no LRF)."""
    g = box_inputs["nolrf"]
    s = System.open(g.inp)
    v = s.view
    o = oracle.create(s)
    o.final_energy()
    E, _ = o.energy_vectors()
    x = o.coords().reshape(-1, 3)
    el, vdw = _nearest_image_ww(x, v.nat_solute, v.nwat, EDGE, v.Rcww, v.crg_ow, v.crg_hw, v.A_OO, v.B_OO)
    from q_b200 import E_NAMES
    e = dict(zip(E_NAMES, E))
    assert abs(e["ww_el"] - el) < 1e-6 * abs(el)
    assert abs(e["ww_vdw"] - vdw) < 1e-6 * max(1.0, abs(vdw))


def test_oracle_energy_is_invariant_under_lattice_shifts(box_inputs, oracle):
    """Moving whole molecules by box vectors changes no energy and no force
    (LRF included): every pair takes its nearest image."""
    g = box_inputs["nvt"]
    s = System.open(g.inp)
    v = s.view
    a = oracle.create(s)
    a.final_energy()
    Ea, _ = a.energy_vectors()
    ga = a.gradient()
    x = a.coords().reshape(-1, 3).copy()
    rng = np.random.default_rng(5)
    starts = [v.istart_mol[m] for m in range(v.nmol + 1)]
    for m in range(v.nmol):
        shift = EDGE * rng.integers(-1, 2, size=3)
        x[starts[m]:starts[m + 1]] += shift
    b = oracle.create(s)
    b.lib.qo_set_coords(b.st, np.ascontiguousarray(x.reshape(-1)).ctypes.data_as(
        __import__("ctypes").POINTER(__import__("ctypes").c_double)))
    b.final_energy()
    Eb, _ = b.energy_vectors()
    gb = b.gradient()
    assert np.max(np.abs(Ea - Eb)) < 1e-8 * max(1.0, np.max(np.abs(Ea)))
    assert np.max(np.abs(ga - gb)) < 1e-8 * max(1.0, np.max(np.abs(ga)))


def test_oracle_puts_molecules_back_in_the_box(box_inputs, oracle, tmp_path):
    """put_back_in_box at the first list step: the box centre becomes the
    solute's mean position and every molecule whose centre of mass lies
    beyond half an edge moves by one edge length along that axis (one per
    call: a molecule two edges out comes one edge closer)."""
    g = box_inputs["nvt"]
    s = System.open(g.inp)
    v = s.view
    x = np.array([v.x0[k] for k in range(3 * v.natom)]).reshape(-1, 3)
    x[v.istart_mol[5]:v.istart_mol[6]] += np.array([EDGE, 0, 0])
    x[v.istart_mol[9]:v.istart_mol[10]] -= np.array([0, 2 * EDGE, 0])
    re = os.path.join(os.path.dirname(g.inp), "displaced.re")
    write_restart(re, x.reshape(-1), np.zeros(x.size), None, np.array([EDGE] * 3 + [0.0] * 3))
    inp = _inp_with(g, tmp_path, "displaced", **{"random_seed 1\n": "", "initial_temperature 298\n": "",
                                                  "final pbc.re": "final pbc.re\nrestart displaced.re"})
    s2 = System.open(inp)
    o = oracle.create(s2)
    assert o.run(1) == 0
    box = o.box()
    xs = o.coords().reshape(-1, 3)
    c = xs[:v.nat_solute].mean(axis=0)
    assert np.allclose(box[3:], c, atol=0.1)
    mass = np.array([s2.view.mass_box[j] for j in range(v.natom)])
    for m in range(v.nmol):
        a, b = v.istart_mol[m], v.istart_mol[m + 1]
        cm = (xs[a:b] * mass[a:b, None]).sum(axis=0) / mass[a:b].sum()
        d = cm - box[3:]
        if m == 9:
            assert -1.5 * EDGE - 0.2 <= d[1] <= -0.5 * EDGE + 0.2
            d[1] += EDGE
        assert np.all(np.abs(d) <= EDGE / 2 + 0.2), m


def test_oracle_volume_moves(box_inputs, oracle):
    """Constant pressure: a volume move after steps 10 and 20; the box scales
    by the cube root of the volume ratio when accepted; the run is
    deterministic (randm's sequence)."""
    g = box_inputs["npt"]
    s = System.open(g.inp)
    runs = []
    for _ in range(2):
        o = oracle.create(s)
        assert o.run(25) == 0
        runs.append((o.box(), o.volume_moves(), o.coords()))
    (b0, m0, x0), (b1, m1, x1) = runs
    assert m0 == (2, m0[1]) and m0 == m1
    assert np.array_equal(b0, b1) and np.array_equal(x0, x1)
    if m0[1] > 0:
        assert not np.allclose(b0[:3], EDGE)
    assert np.allclose(b0[0], b0[1]) and np.allclose(b0[1], b0[2])
