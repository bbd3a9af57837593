"""The interaction-class cases of the reference's Q6-vs-QGPU comparison
harness (test/runTEST.py): topology, sphere radius and FEP file per case, and
the qdyn input the harness writes for them (1 fs, 1 K, seed 112, LRF off,
99 A cut-offs, lists every step, lambda 1/0)."""
import os

CASES = {
    "p-p": ("benzene-vacuum.top", 20, None),
    "q-p_benzene": ("Na-benzene-vacuum.top", 20, "FEP_benzene.fep"),
    "q-p_Na": ("Na-benzene-vacuum.top", 20, "FEP_Na.fep"),
    "q-p-w_benzene": ("Na-benzene-water.top", 20, "FEP_benzene.fep"),
    "q-p-w_Na": ("Na-benzene-water.top", 20, "FEP_Na.fep"),
    "q-q": ("benzene-vacuum.top", 20, "FEP_benzene.fep"),
    "w-p": ("benzene-water.top", 20, None),
    "w-q": ("benzene-water.top", 20, "FEP_benzene.fep"),
    "w-w": ("water.top", 20, None),
    "dualtop": ("dualtop_vacuum.top", 20, "dualtop.fep"),
}


def write_case(datadir: str, case: str, steps: int = 10, shake: bool = False) -> str:
    """Write the harness's eq1 input for `case` into datadir (beside the
    unpacked fixtures) and return its path."""
    top, radius, fep = CASES[case]
    sh = "on" if shake else "off"
    L = ["[MD]", "steps %d" % steps, "stepsize 1", "temperature 1", "bath_coupling 1", "random_seed 112",
         "initial_temperature 1", "shake_solvent %s" % sh, "shake_hydrogens %s" % sh, "shake_solute %s" % sh,
         "lrf off", "", "[cut-offs]", "solute_solvent 99.0", "solute_solute 99.0", "solvent_solvent 99.0",
         "q_atom 99.0", "lrf 99.0", "", "[sphere]", "shell_force 10.0", "shell_radius %d" % radius, "",
         "[solvent]", "radial_force 60.0", "polarisation on", "polarisation_force 20.0", "charge_correction off", "",
         "[intervals]", "output 1", "non_bond 1", "", "[files]", "topology %s" % top, "final %s.re" % case]
    if fep:
        L += ["fep %s" % fep, "", "[lambdas]", "1.000 0.000"]
    path = os.path.join(datadir, "%s%s.inp" % (case, "_shake" if shake else ""))
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")
    return path
