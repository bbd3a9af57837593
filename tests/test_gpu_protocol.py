"""The qdyn drop-in end to end (energy file, restart, trajectory) and the
batched heating protocol feeding parallel windows."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_qdyn_dropin_writes_trajectory_energy_and_restart(tmp_path):
    from q_b200 import synth
    from q_b200.fep import read_en
    from q_b200.trajectory import read_dcd
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, steps=50)
    inp = str(tmp_path / "c1" / "md.inp")
    synth.write_inp(inp, g.top, g.fep, steps=50, stepsize=2.0, lambdas=(0.5, 0.5), shake_hydrogens=True,
                    output=10, energy=10, trajectory=10, trajectory_atoms=["not excluded"])
    r = subprocess.run([sys.executable, "-m", "q_b200.qdyn", inp], cwd=REPO, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "terminated normally" in r.stdout and "Coordinates for" in r.stdout
    h, frames = read_dcd(str(tmp_path / "c1" / "md.dcd"))
    assert h["frames"] == 5 and frames.shape[0] == 5 and h["mask_rows"] == ["not excluded"]
    # energies only inside the loop, at istep = 10, 20, 30, 40 of 0..49 (md.f90:4155): 4 records
    assert read_en(str(tmp_path / "c1" / "md.en"), 2).shape[0] == 4
    # the last frame is the final coordinates (after step 50), as in the restart
    from q_b200.inputs import derive_inp
    from q_b200 import System
    q = derive_inp(inp, "again.inp", set_keys={"files": {"restart": "md.re"}},
                   drop_keys={"md": ["random_seed", "initial_temperature"]})
    s = System.open(q)
    x = s.array("x0", 3 * s.natom).reshape(-1, 3)
    excl = np.array(s.view.excl[:s.natom], bool)
    assert np.array_equal(frames[-1], x[~excl].astype(np.float32))


def test_heating_protocol_then_parallel_windows(tmp_path):
    from q_b200 import synth
    from q_b200.campaign import QLIGFEP_EQ_2FS, equilibrate, run_perturbation
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, steps=100)
    eq = equilibrate(g.inp, seeds=(11, 12), stages=QLIGFEP_EQ_2FS, lambdas=(1.0, 0.0), steps_scale=0.01)
    assert len(eq.restarts) == 2 and all(os.path.exists(p) for p in eq.restarts)
    assert len(eq.temperatures) == 5
    assert eq.temperatures[0] < 60.0 and 200.0 < eq.temperatures[-1] < 400.0
    r = run_perturbation(g.inp, synth.window_lambdas(3), steps_eq=20, steps_prod=100, starts=eq.inputs)
    assert r.replicas == 2 and len(r.dG) == 2 and np.all(np.isfinite(r.dG))
