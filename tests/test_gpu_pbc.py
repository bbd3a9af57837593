"""Periodic box (use_PBC) on the GPU engine against the CPU oracle: the
nearest-image lists and pair terms (nbpplist_box ... nonbond_ww_spc_box,
md.f90:5307-12100), LRF in the box, put_back_in_box at the list steps and
Monte Carlo volume moves (MC_volume, md.f90:15615).

Tolerances as the sphere's parity tests: every energy term within 1e-3
kcal/mol, FP64 gradients within 1e-4 relative per atom.
"""
import os

import numpy as np
import pytest

from q_b200 import FP64, MIXED, Batch, System, synth, write_restart

from test_gpu_parity import G_TOL, assert_energies, grad_err

pytestmark = pytest.mark.gpu

EDGE = 30.0


@pytest.fixture(scope="module")
def boxes(tmp_path_factory):
    root = tmp_path_factory.mktemp("pbc_gpu")
    return {
        "nvt": synth.fep_box(str(root / "nvt"), edge=EDGE, seed=1234),
        "nolrf": synth.fep_box(str(root / "nolrf"), edge=EDGE, seed=77, lrf=None),
        "npt": synth.fep_box(str(root / "npt"), edge=EDGE, seed=1234, constant_pressure=True, volume_change=10,
                             max_volume_displ=400.0),
        "rst": synth.fep_box(str(root / "rst"), edge=EDGE, seed=1234,
                             distance_restraints=["1 20 2.0 4.0 5.0 0", "3 40 1.0 2.0 5.0 0"]),
        # restraints reaching water atoms (atoms 100 and 301: waters after the
        # 56 solute atoms), whose gradient the water pass stores first
        "rst_water": synth.fep_box(str(root / "rst_water"), edge=EDGE, seed=1234,
                                   distance_restraints=["1 100 2.0 4.0 5.0 0", "5 301 1.0 2.0 5.0 0"]),
    }


@pytest.mark.parametrize("case", ["nvt", "nolrf", "rst", "rst_water"])
def test_box_single_point(boxes, oracle, case):
    """Lists and potential at the starting coordinates: energies and gradient."""
    s = System.open(boxes[case].inp)
    b = Batch([s], precision=FP64)
    b.final_energy()
    o = oracle.create(s)
    o.final_energy()
    Eg, EQg = b.energy_vectors(0)
    Eo, EQo = o.energy_vectors()
    assert_energies(Eg, EQg, Eo, EQo)
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL
    if case.startswith("rst"):
        # the same coordinates through the mixed engine's force path
        m = Batch([s], precision=MIXED)
        m.evaluate(energies=False)
        assert grad_err(m.gradient(0), o.gradient()) < G_TOL


def test_box_single_point_after_lattice_shifts(boxes, oracle):
    """Whole molecules moved by box vectors: the engine's nearest images give
    the oracle's energies and forces of the unshifted system."""
    s = System.open(boxes["nvt"].inp)
    v = s.view
    o = oracle.create(s)
    o.final_energy()
    Eo, EQo = o.energy_vectors()
    x = np.array([v.x0[k] for k in range(3 * v.natom)]).reshape(-1, 3)
    rng = np.random.default_rng(11)
    for m in range(v.nmol):
        x[v.istart_mol[m]:v.istart_mol[m + 1]] += EDGE * rng.integers(-1, 2, size=3)
    b = Batch([s], precision=FP64)
    b.set_coords(0, x.reshape(-1))
    b.final_energy()
    Eg, EQg = b.energy_vectors(0)
    assert_energies(Eg, EQg, Eo, EQo)
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL


def test_box_trajectory_fp64(boxes, oracle):
    """100 steps (lists every 25 with molecules put back in the box, LRF,
    SHAKE): the output records, final energies, coordinates and box."""
    s = System.open(boxes["nvt"].inp)
    b = Batch([s], precision=FP64)
    o = oracle.create(s)
    b.run(100)
    assert o.run(100) == 0
    sg, Eg, EQg = b.history(0, 0)
    so, Eo, EQo = o.history(0)
    assert list(sg) == list(so)
    for k in range(len(sg)):
        assert_energies(Eg[k], EQg[k], Eo[k], EQo[k])
    assert np.max(np.abs(b.coords(0) - o.coords())) < 1e-6
    assert np.max(np.abs(b.box(0) - o.box())) < 1e-9


def test_box_trajectory_mixed(boxes, oracle):
    """The mixed-precision engine in the box: 50 steps (two list rebuilds
    with molecules put back) stay near the FP64 oracle's trajectory; at the
    coordinates they reach, its recording-step energies (FP64 water-water)
    match the oracle within 1e-3 kcal/mol and its packed FP32 forces within
    1e-4 relative."""
    import ctypes as C
    s = System.open(boxes["nvt"].inp)
    b = Batch([s], precision=MIXED)
    o = oracle.create(s)
    b.run(50)
    assert o.run(50) == 0
    assert np.max(np.abs(b.coords(0) - o.coords())) < 2e-3
    x = np.ascontiguousarray(b.coords(0))
    p = oracle.create(s)
    p.lib.qo_set_coords(p.st, x.ctypes.data_as(C.POINTER(C.c_double)))
    p.final_energy()
    Eo, EQo = p.energy_vectors()
    b.evaluate(energies=True)
    Eg, EQg = b.energy_vectors(0)
    # the potential terms (kinetic energy: the engine's last step against the
    # oracle's starting velocities)
    Eg[1] = Eo[1]
    assert_energies(Eg, EQg, Eo, EQo)
    b.evaluate(energies=False)
    assert grad_err(b.gradient(0), p.gradient()) < G_TOL


def test_box_volume_moves(boxes, oracle):
    """Constant pressure: volume moves after steps 10, 20 and 30 with the
    oracle's random numbers, acceptances and boxes; the recorded energies of
    those steps are the accepted configuration's."""
    s = System.open(boxes["npt"].inp)
    b = Batch([s], precision=FP64)
    o = oracle.create(s)
    b.run(35)
    assert o.run(35) == 0
    assert b.volume_moves(0) == o.volume_moves() == (3, o.volume_moves()[1])
    assert np.max(np.abs(b.box(0) - o.box())) < 1e-9
    for kind in (0, 1):
        sg, Eg, EQg = b.history(0, kind)
        so, Eo, EQo = o.history(kind)
        assert list(sg) == list(so)
        for k in range(len(sg)):
            assert_energies(Eg[k], EQg[k], Eo[k], EQo[k])
    assert np.max(np.abs(b.coords(0) - o.coords())) < 1e-6


def test_box_batch_mixes_sizes_and_sphere(boxes, oracle, golden):
    """A batch of a periodic box, the same box at constant pressure and a
    sphere system: each as its own oracle run."""
    a = System.open(boxes["nvt"].inp)
    c = System.open(str(golden / "test1" / "eq1.inp"))
    d = System.open(boxes["npt"].inp)
    b = Batch([a, c, d], precision=FP64)
    b.run(20)
    for k, sys_ in ((0, a), (1, c), (2, d)):
        o = oracle.create(sys_)
        assert o.run(20) == 0
        _, Eg, EQg = b.history(k, 0)
        _, Eo, EQo = o.history(0)
        assert_energies(Eg[-1], EQg[-1], Eo[-1], EQo[-1])
        assert np.max(np.abs(b.coords(k) - o.coords())) < 1e-6


def test_box_restart_written_with_box(boxes, tmp_path):
    """The drop-in qdyn's final restart carries the box records; reading it
    back gives the same box."""
    from q_b200 import qdyn
    g = boxes["npt"]
    txt = open(g.inp).read().replace("steps 1000", "steps 30")
    inp = os.path.join(os.path.dirname(g.inp), "short.inp")
    open(inp, "w").write(txt.replace("final pbc.re", "final short.re"))
    with open(tmp_path / "log", "w") as out:
        assert qdyn.run(inp, out) == 0
    log = open(tmp_path / "log").read()
    assert "VOLUME CHANGE SUMMARY" in log and "terminated normally" in log
    raw = open(os.path.join(os.path.dirname(g.inp), "short.re"), "rb").read()
    box = np.frombuffer(raw[-32 - 28:-32 - 4], dtype=np.float64)
    assert np.all(box > 25.0)
