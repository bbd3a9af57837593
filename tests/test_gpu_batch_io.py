"""Batched host copies of the C ABI (qb_batch_*_all, qb_batch_history_all)
against the per-system calls they replace on the end-to-end path."""
import numpy as np
import pytest

from q_b200 import MIXED, Batch, System

pytestmark = pytest.mark.gpu


def test_all_system_copies_match_per_system_calls(tmp_path):
    from q_b200 import synth
    a = synth.water_sphere(str(tmp_path / "a"), radius=15.0, seed=3)
    c = synth.fep_solute(str(tmp_path / "c"), seed=1234)
    systems = [System.open(a.inp, seed=5), System.open(c.inp, lambdas=(0.5, 0.5), seed=6),
               System.open(a.inp, seed=7)]
    b = Batch(systems, precision=MIXED)
    b.run(30)
    x_all, v_all = b.coords_all(), b.velocities_all()
    off = np.cumsum([0] + [3 * s.natom for s in systems])
    for k in range(len(systems)):
        assert np.array_equal(x_all[off[k]:off[k + 1]], b.coords(k))
        assert np.array_equal(v_all[off[k]:off[k + 1]], b.velocities(k))
    for kind in (0, 1):
        counts, rec = b.history_all(kind)
        for k, s in enumerate(systems):
            steps, E, EQ = b.history(k, kind)
            assert counts[k] == len(steps)
            assert np.array_equal(rec[k, :counts[k], 0].astype(int), steps)
            assert np.array_equal(rec[k, :counts[k], 1:1 + E.shape[1]], E)
    # setting every system at once equals setting them one by one
    b2 = Batch(systems, precision=MIXED)
    b2.set_coords_all(x_all)
    b2.set_velocities_all(v_all)
    b2.run(5)
    b3 = Batch(systems, precision=MIXED)
    for k in range(len(systems)):
        b3.set_coords(k, x_all[off[k]:off[k + 1]])
        b3.set_velocities(k, v_all[off[k]:off[k + 1]])
    b3.run(5)
    assert np.max(np.abs(b2.coords_all() - b3.coords_all())) < 1e-9
    assert b2.step_count() == 5 and b.step_count() == 30
