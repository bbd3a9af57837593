"""The reference's own interaction-class test matrix (test/runTEST.py: p-p,
q-p, q-p-w, q-q, w-p, w-q, w-w, and the dual-topology FEP), run on the GPU
and on the oracle from the same input: 10 steps of 1 fs at 1 K with lists
every step and 99 A cut-offs, with and without SHAKE.  Every energy record,
the gradient and the coordinates after the last step must agree."""
import numpy as np
import pytest

from q_b200 import FP64, Batch, System

from tests.reference_cases import CASES, write_case
from tests.test_gpu_parity import G_TOL, assert_energies, grad_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shake", [False, True], ids=["noshake", "shake"])
@pytest.mark.parametrize("case", list(CASES))
def test_reference_case(golden, oracle, case, shake):
    inp = write_case(str(golden / "data"), case, steps=10, shake=shake)
    s = System.open(inp)
    b = Batch([s], precision=FP64)
    b.run(10)
    o = oracle.create(s)
    o.run(10)
    sg, Eg, EQg = b.history(0, 0)
    so, Eo, EQo = o.history(0)
    assert list(sg) == list(so) and len(sg) == 10
    for k in range(len(sg)):
        assert_energies(Eg[k], EQg[k], Eo[k], EQo[k])
    assert grad_err(b.gradient(0), o.gradient()) < G_TOL
    # coordinates to 1e-7 A: the polarisation restraint takes a single-precision
    # acos (as qdyn does), whose CUDA and glibc values may differ by one ulp
    assert np.max(np.abs(b.coords(0) - o.coords())) < 1e-7
