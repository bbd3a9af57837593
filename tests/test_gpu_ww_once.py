"""The mixed engine's packed water-water forces with every molecule pair
evaluated once (qb_tuning.ww_pairs_once 1: the second water's terms summed in
FP32 in shared memory; 2: in 32-bit fixed point), against the FP64 engine on
the same coordinates at the gradient bar (1e-4 relative per atom): one and
several staging chunks, a close contact whose terms leave the fixed-point
range, the periodic box, and lists rebuilt during a run.
"""
import numpy as np
import pytest

from q_b200 import FP64, MIXED, Batch, QBError, System, synth

from test_gpu_parity import G_TOL, grad_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spheres(tmp_path_factory):
    root = tmp_path_factory.mktemp("ww_once")
    return {"c0": synth.water_sphere(str(root / "c0"), radius=15.0, seed=1234),
            "c1": synth.fep_solute(str(root / "c1"), seed=1234),
            "c0_r27": synth.water_sphere(str(root / "c0_r27"), radius=27.0, seed=7),
            "box": synth.fep_box(str(root / "box"), edge=30.0, seed=1234)}


def _fp64_gradient(s, x=None):
    b = Batch([s], precision=FP64)
    if x is not None:
        b.set_coords(0, x)
    b.final_energy()
    return b.gradient(0)


def _mixed_gradient(s, once, x=None, **tuning):
    b = Batch([s], precision=MIXED)
    b.set_tuning(ww_pairs_once=once, **tuning)
    assert b.tuning()["ww_pairs_once"] == once
    if x is not None:
        b.set_coords(0, x)
    b.evaluate(energies=False)
    return b.gradient(0)


@pytest.mark.parametrize("once", [1, 2])
@pytest.mark.parametrize("case", ["c1", "c0_r27"])
def test_pairs_once_gradient(spheres, case, once):
    """c1: one staging chunk; the 27 A sphere (about 2,700 waters) in chunks
    of 1,024 waters."""
    s = System.open(spheres[case].inp)
    tuning = {"ww_chunk": 1024} if case == "c0_r27" else {}
    g64 = _fp64_gradient(s)
    g_once = _mixed_gradient(s, once, **tuning)
    g_both = _mixed_gradient(s, 0, **tuning)
    assert grad_err(g_once, g64) < G_TOL
    assert grad_err(g_once, g_both) < G_TOL


def test_close_contact_leaves_fixed_point_range(spheres):
    """Two waters 2 A apart (O-O Lennard-Jones alone ~850 kcal/mol/A, above
    the fixed-point accumulator's per-term limit): the terms on the second
    water go to the FP64 gradient directly, and both accumulations still
    match the FP64 engine."""
    s = System.open(spheres["c0"].inp)
    v = s.view
    x = np.array([v.x0[k] for k in range(3 * v.natom)]).reshape(-1, 3)
    ns, nw = v.nat_solute, v.nwat
    O = x[ns::3][:nw]
    i = nw // 2
    d = np.linalg.norm(O - O[i], axis=1)
    d[: i + 1] = np.inf
    j = int(np.argmin(d))                  # the nearest water above i
    u = (O[j] - O[i]) / d[j]
    x[ns + 3 * j: ns + 3 * j + 3] += O[i] + 2.0 * u - O[j]
    x = x.reshape(-1)
    g64 = _fp64_gradient(s, x)
    for once in (2, 1):
        assert grad_err(_mixed_gradient(s, once, x), g64) < G_TOL


def test_pairs_once_in_the_box(spheres):
    """Nearest images in the periodic box (the kernel's BOX form)."""
    s = System.open(spheres["box"].inp)
    g64 = _fp64_gradient(s)
    for once in (1, 2):
        assert grad_err(_mixed_gradient(s, once), g64) < G_TOL


def test_pairs_once_after_list_rebuilds(spheres):
    """30 mixed steps (a rebuild at step 25 moves the split points of the
    lists) with each pair once and from both sides: the trajectories stay
    within FP32 rounding of each other (a pair lost or doubled after the
    rebuild would move atoms by ~1e-2 A in five steps), and at the
    coordinates reached the two forms give the same forces (the water
    polarisation shells are then the run's own, not a fresh set-up's)."""
    s = System.open(spheres["c1"].inp)
    runs = []
    for once in (2, 0):
        b = Batch([s], precision=MIXED)
        b.set_tuning(ww_pairs_once=once)
        b.run(30)
        assert b.status(0) == 0
        runs.append(b)
    b2, b0 = runs
    assert np.max(np.abs(b2.coords(0) - b0.coords(0))) < 1e-4
    b2.evaluate(energies=False)
    g2 = b2.gradient(0)
    b2.set_tuning(ww_pairs_once=0)
    b2.evaluate(energies=False)
    assert grad_err(g2, b2.gradient(0)) < G_TOL


def test_pairs_once_settings_checked(spheres):
    s = System.open(spheres["c0_r27"].inp)
    b = Batch([s], precision=MIXED)
    with pytest.raises(QBError):
        b.set_tuning(ww_pairs_once=3)
    # the largest chunk's records and accumulator exceed the staging memory
    t = b.tuning()
    with pytest.raises(QBError):
        b.set_tuning(ww_pairs_once=1, ww_chunk=t["ww_chunk_max"])
    b.set_tuning(ww_pairs_once=1, ww_chunk=1024)
    assert b.tuning()["ww_pairs_once"] == 1
