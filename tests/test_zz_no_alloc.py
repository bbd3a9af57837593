"""The allocation-free water-water entry point (qb_ww_energy_static).

Hosts that cannot let a library call cudaMalloc (device memory handed out only
from the host's own pool, or allocation forbidden on the calling thread) use
this entry point: it computes the water-water energy and gradient on buffers
the caller owns and keeps its neighbour-list scratch in a fixed device array
inside the library.  The test compares it, through the C ABI, with the batch
engine (qb_batch_*) on a water sphere whose only interactions are water-water
terms, for two calls in a row on two different coordinate sets.  It lives in
its own file, collected last, and passes alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_TOL = 1e-3   # kcal/mol, as the other parity tests
G_TOL = 1e-4   # relative, as the other parity tests

PURE_WW_INP = """[MD]
steps 20
stepsize 1
temperature 298
bath_coupling 100
random_seed 11
initial_temperature 298
shake_solvent on
lrf off

[cut-offs]
solvent_solvent 10

[solvent]
radial_force 0
morse_depth 0
polarization off

[intervals]
non_bond 10
output 10

[files]
topology %s
final pure.re
"""


def test_static_entry_point_matches_batch_engine(tmp_path):
    torch = pytest.importorskip("torch")
    from q_b200 import FP64, Batch, E_NAMES, System, synth
    from q_b200._lib import check, lib

    g = synth.water_sphere(str(tmp_path), radius=15.0, seed=99)
    inp = tmp_path / "pure.inp"
    inp.write_text(PURE_WW_INP % g.top)
    sys_ = System.open(str(inp))
    v = sys_.view
    nwat, ns = v.nwat, v.nat_solute
    assert v.nwpolr_shell == 0 and not v.use_LRF

    b = Batch([sys_], precision=FP64)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    grad = torch.empty(9 * nwat, dtype=torch.float64, device=dev)
    energy = torch.empty(2, dtype=torch.float64, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)

    for call in range(2):
        if call == 1:
            b.run(10)          # a second coordinate set
        b.final_energy()
        E, _ = b.energy_vectors(0)
        e = dict(zip(E_NAMES, E))
        # the batch system has water-water terms only
        others = {k: val for k, val in e.items()
                  if k not in ("ww_el", "ww_vdw", "potential", "kinetic") and abs(val) > 1e-12}
        assert not others, others
        x = torch.tensor(b.coords(0)[3 * ns:], dtype=torch.float64, device=dev)
        rc = lib.qb_ww_energy_static(C.c_void_p(x.data_ptr()), nwat, v.crg_ow, v.crg_hw, v.A_OO, v.B_OO,
                                     v.Rcww, None, C.c_void_p(grad.data_ptr()), C.c_void_p(energy.data_ptr()),
                                     C.c_void_p(status.data_ptr()), C.c_void_p(stream.cuda_stream))
        check(rc)
        torch.cuda.synchronize(dev)
        assert int(status.item()) == 0
        el, vdw = energy.cpu().numpy()
        assert abs(el - e["ww_el"]) < E_TOL
        assert abs(vdw - e["ww_vdw"]) < E_TOL
        g_static = grad.cpu().numpy().reshape(-1, 3)
        g_batch = b.gradient(0)[3 * ns:].reshape(-1, 3)
        nrm = np.linalg.norm(g_batch, axis=1)
        floor = 0.01 * np.sqrt(np.mean(nrm ** 2))
        err = np.max(np.linalg.norm(g_static - g_batch, axis=1) / np.maximum(nrm, floor))
        assert err < G_TOL


def ww_reference(x, excl, qo, qh, A, B, rc):
    """numpy FP64 statement of nonbond_ww_spc (src/q6/md.f90:11823) over every
    pair of non-excluded waters whose O-O distance is within rc: energies
    (el, vdw) and the gradient dU/dx, waters as O,H,H."""
    w = x.reshape(-1, 3, 3)
    keep = ~excl.astype(bool)
    n = len(w)
    i, j = np.triu_indices(n, 1)
    ok = keep[i] & keep[j] & (np.linalg.norm(w[j, 0] - w[i, 0], axis=1) <= rc)
    i, j = i[ok], j[ok]
    q = np.array([qo, qh, qh], dtype=np.float32)
    g = np.zeros_like(w)
    el = vdw = 0.0
    for a in range(3):
        for b in range(3):
            d = w[j, b] - w[i, a]
            r2 = np.einsum("ij,ij->i", d, d)
            rinv = 1.0 / np.sqrt(r2)
            vel = float(np.float32(q[a] * q[b])) * rinv
            dv = -vel * rinv ** 2
            el += vel.sum()
            if a == 0 and b == 0:
                r6 = rinv ** 6
                va, vb = A * r6 * r6, B * r6
                vdw += (va - vb).sum()
                dv = dv + rinv ** 2 * (-12.0 * va + 6.0 * vb)
            f = dv[:, None] * d
            np.add.at(g[:, a], i, -f)
            np.add.at(g[:, b], j, f)
    return el, vdw, g.reshape(-1)


def test_static_entry_point_excluded_waters_and_overflow(tmp_path):
    """Waters flagged in `excl` take part in no pair: checked against a numpy
    FP64 statement of the water-water terms on the same coordinates.  A water
    with more neighbours than the fixed list row holds sets
    QB_ERR_LIST_OVERFLOW in the status word."""
    torch = pytest.importorskip("torch")
    from q_b200 import System, synth
    from q_b200._lib import check, lib

    g = synth.water_sphere(str(tmp_path), radius=15.0, seed=7)
    inp = tmp_path / "pure.inp"
    inp.write_text(PURE_WW_INP % g.top)
    sys_ = System.open(str(inp))
    v = sys_.view
    nwat, ns = v.nwat, v.nat_solute
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    xh = np.ctypeslib.as_array(v.xtop, shape=(3 * v.natom,))[3 * ns:].copy()
    rng = np.random.default_rng(5)
    excl = (rng.random(nwat) < 0.2).astype(np.uint8)
    x = torch.tensor(xh, dtype=torch.float64, device=dev)
    ex = torch.tensor(excl, dtype=torch.uint8, device=dev)
    grad = torch.empty(9 * nwat, dtype=torch.float64, device=dev)
    energy = torch.empty(2, dtype=torch.float64, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)

    def call(xd, n, rc, exd):
        check(lib.qb_ww_energy_static(C.c_void_p(xd.data_ptr()), n, v.crg_ow, v.crg_hw, v.A_OO, v.B_OO, rc,
                                      C.c_void_p(exd.data_ptr()) if exd is not None else None,
                                      C.c_void_p(grad.data_ptr()), C.c_void_p(energy.data_ptr()),
                                      C.c_void_p(status.data_ptr()), C.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize(dev)
        return int(status.item()), energy.cpu().numpy().copy(), grad.cpu().numpy()[:9 * n].copy()

    st, e, gr = call(x, nwat, v.Rcww, ex)
    assert st == 0
    el, vdw, gref = ww_reference(xh, excl, v.crg_ow, v.crg_hw, v.A_OO, v.B_OO, v.Rcww)
    assert abs(e[0] - el) < E_TOL and abs(e[1] - vdw) < E_TOL
    gs, gb = gr.reshape(-1, 3), gref.reshape(-1, 3)
    nrm = np.linalg.norm(gb, axis=1)
    floor = 0.01 * np.sqrt(np.mean(nrm ** 2))
    assert np.max(np.linalg.norm(gs - gb, axis=1) / np.maximum(nrm, floor)) < G_TOL
    assert not np.any(gs.reshape(-1, 9)[excl.astype(bool)])

    # every water of a 15 A sphere lies within 40 A of every other: rows of
    # nwat - 1 > QB_STATIC_WW_MAX_NEIGHBOURS entries
    assert nwat - 1 > 192
    st, _, _ = call(x, nwat, 40.0, None)
    assert st == 7   # QB_ERR_LIST_OVERFLOW
    # the next call starts from a cleared status word
    st, e2, _ = call(x, nwat, v.Rcww, ex)
    assert st == 0 and abs(e2[0] - el) < E_TOL


def test_static_entry_point_rejects_oversized_systems():
    from q_b200._lib import lib
    rc = lib.qb_ww_energy_static(None, 10 ** 6, 0.0, 0.0, 0.0, 0.0, 10.0, None, None, None, None, None)
    assert rc == 1   # QB_ERR_ARG
