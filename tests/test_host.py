"""Host-side logic of libqb, no GPU needed: the C ABI loads and exports what
its headers declare, the Q file readers and writers, error paths, the
synthetic generator, the qdyn log layout and the multi-rank helpers."""
import os
import struct

import numpy as np
import pytest

from q_b200 import QBError, System, append_energy, synth, write_restart
from q_b200._lib import exported_symbols, lib


def test_library_exports_every_declared_symbol():
    names = exported_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    import ctypes as C
    buf = C.create_string_buffer(64)
    assert lib.qb_version(buf, 64) == 0 and b"sm_100a" in buf.value


def test_test1_topology_and_setup(golden):
    s = System.open(str(golden / "test1" / "eq1.inp"))
    v = s.view
    assert (v.natom, v.nat_solute, v.nwat) == (3397, 46, 1117)
    assert (v.ncgp, v.ncgp_solute, v.natyps) == (1150, 33, 93)
    assert (v.nqat, v.nstates) == (46, 1)
    assert v.ff_type == 2 and v.iuse_switch_atom == 1
    # [cut_offs] is not the section name qdyn reads: defaults apply
    assert (v.Rcpp, v.Rcww, v.Rcpw, v.Rcq, v.RcLRF) == (10.0, 10.0, 10.0, 99.0, 99.0)
    assert v.use_LRF == 1 and v.NBcycle == 25 and v.iout_cycle == 50
    assert abs(v.dt - 0.020462 * 0.1) < 1e-15
    # solvent SHAKE: 3 constraints per water, the water angles removed
    assert v.shake_constraints == 3 * 1117 and v.nangles == v.nangles_solute
    assert v.Ndegf == 3 * 3397 - 3 * 1117
    # sequence restraint "1 46 0.5 0 1": to the geometric centre
    assert v.nrstr_seq == 1 and v.rseq_to_center[0] == 1 and v.rseq_fk[0] == 0.5
    # rexcl_i = 16 A (absolute), shell force 20
    assert v.rexcl_i == 16.0 and v.fk_pshell == 20.0
    # charges are stored scaled by sqrt(332) in single precision
    q = s.array("crg", v.natom)
    assert q.dtype == np.float32
    assert abs(q[v.nat_solute] - np.float32(-0.834 * np.sqrt(332.0))) < 1e-5
    assert v.nwpolr_shell == 3


def test_benzene_topology(golden):
    v = System.open(str(golden / "benzene" / "eq1.inp")).view
    assert (v.natom, v.nat_solute, v.nwat, v.nstates) == (12, 12, 0, 0)
    assert v.nbonds == 12 and v.nangles == 18 and v.nimps == 6


def test_restart_round_trip(tmp_path, golden):
    s = System.open(str(golden / "benzene" / "eq1.inp"))
    x = s.array("x0") + 0.01
    v = np.arange(x.size, dtype=np.float64) * 1e-3
    re = tmp_path / "in.re"
    write_restart(str(re), x, v)
    # gfortran records: (int32 nat3, 36 doubles) twice, each with 4-byte markers
    raw = re.read_bytes()
    assert len(raw) == 2 * (4 + 4 + 8 * 36 + 4)
    assert struct.unpack("<ii", raw[:8]) == (4 + 8 * 36, 36)
    inp = (golden / "benzene" / "eq1.inp").read_text()
    inp = inp.replace("initial_temperature       1", "").replace("final ", "restart in.re\nfinal ")
    inp = inp.replace("topology                  benzene-vacuum.top",
                      "topology                  %s" % (golden / "benzene" / "benzene-vacuum.top"))
    (tmp_path / "re.inp").write_text(inp)
    s2 = System.open(str(tmp_path / "re.inp"))
    assert np.array_equal(s2.array("x0"), x)
    assert np.array_equal(s2.array("v0"), v)


def test_energy_file_records(tmp_path):
    path = tmp_path / "x.en"
    EQ = np.arange(2 * 15, dtype=np.float64).reshape(2, 15)
    append_energy(str(path), EQ)
    append_energy(str(path), EQ + 1)
    raw = path.read_bytes()
    frame = 2 * (4 + 4 + 120 + 4) + 8
    assert len(raw) == 2 * frame
    n, st = struct.unpack("<ii", raw[:8])
    assert (n, st) == (124, 1)
    vals = struct.unpack("<15d", raw[8:128])
    assert vals == tuple(EQ[0])
    # the off-diagonal record of an empty list is a zero-length record
    assert struct.unpack("<ii", raw[frame - 8:frame]) == (0, 0)


def test_error_paths(tmp_path, golden):
    with pytest.raises(QBError) as e:
        System.open(str(tmp_path / "missing.inp"))
    assert e.value.code == 2
    # a periodic-box input with a sphere topology (md.f90:14752-14755)
    txt0 = (golden / "benzene" / "eq1.inp").read_text()
    txt0 = txt0.replace("benzene-vacuum.top", str(golden / "benzene" / "benzene-vacuum.top"))
    (tmp_path / "pbc.inp").write_text("[PBC]\nrigid_box_center off\n" + txt0)
    with pytest.raises(QBError) as e:
        System.open(str(tmp_path / "pbc.inp"))
    assert e.value.code == 3 and "same boundary" in str(e.value)
    txt = (golden / "benzene" / "eq1.inp").read_text().replace("stepsize                  1", "stepsize x")
    (tmp_path / "b.inp").write_text(txt.replace("benzene-vacuum.top", str(golden / "benzene" / "benzene-vacuum.top")))
    with pytest.raises(QBError) as e:
        System.open(str(tmp_path / "b.inp"))
    assert e.value.code == 3
    # truncated restart file
    (tmp_path / "t.re").write_bytes(b"\x00" * 10)
    txt = (golden / "benzene" / "eq1.inp").read_text()
    txt = txt.replace("initial_temperature       1", "").replace("final ", "restart t.re\nfinal ")
    txt = txt.replace("benzene-vacuum.top", str(golden / "benzene" / "benzene-vacuum.top"))
    (tmp_path / "r.inp").write_text(txt)
    with pytest.raises(QBError) as e:
        System.open(str(tmp_path / "r.inp"))
    assert e.value.code == 3


def test_synthetic_systems_parse(tmp_path):
    g0 = synth.water_sphere(str(tmp_path / "c0"), radius=15.0, seed=1234)
    v0 = System.open(g0.inp).view
    assert v0.nat_solute == 0 and 440 <= v0.nwat <= 500
    g1 = synth.fep_solute(str(tmp_path / "c1"), seed=1234)
    s1 = System.open(g1.inp)
    v1 = s1.view
    assert v1.nat_solute == 56 and v1.nqat == 8 and v1.nstates == 2
    assert 1000 <= v1.nwat <= 1130
    assert v1.qvdw_flag == 1
    q = s1.array("crg", v1.natom)[:56] / np.sqrt(332.0)
    assert abs(q.sum()) < 1e-3
    qc = s1.array("qcrg", 16).reshape(8, 2)
    assert np.all(qc[:, 1] == 0.0)
    s2 = System.open(g1.inp, lambdas=(0.25, 0.75), seed=5)   # the view lives as long as s2
    lam = getattr(s2.view, "lambda")
    assert (lam[0], lam[1]) == (0.25, 0.75)


def test_threaded_open_matches_sequential(tmp_path):
    """Windows and replicas opened on a thread pool (the perturbation
    campaign's path) are the systems sequential opens give, and a topology
    edited on disk is read again rather than served from the parse cache."""
    from q_b200.campaign import open_systems
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, steps=100)
    lams = synth.window_lambdas(5)
    seq = [System.open(g.inp, lambdas=l, seed=s) for s in (3, 4) for l in lams]
    par = open_systems(g.inp, lams, (3, 4), threads=4)
    assert len(par) == len(seq) == 10
    for a, b in zip(seq, par):
        assert tuple(a.array("lambda", a.nstates)) == tuple(b.array("lambda", b.nstates))
        assert np.array_equal(a.array("x0", 3 * a.natom), b.array("x0", 3 * b.natom))
        assert np.array_equal(a.array("v0", 3 * a.natom), b.array("v0", 3 * b.natom))
    # velocities differ between replicas, not between windows of one replica
    assert np.array_equal(par[0].array("v0", 30), par[4].array("v0", 30))
    assert not np.array_equal(par[0].array("v0", 30), par[5].array("v0", 30))
    # same path, new content: the charge of solute atom 10 (not a Q-atom) changed
    top = open(g.top).read().split("\n")
    k = next(i for i, l in enumerate(top) if "No. of atomic charges" in l)
    row = top[k + 2].split()
    row[0] = "%7.4f" % (float(row[0]) + 0.5)
    top[k + 2] = " ".join(row)
    import time as _t
    _t.sleep(0.01)
    open(g.top, "w").write("\n".join(top))
    c = System.open(g.inp, lambdas=lams[0], seed=3)
    dq = (c.array("crg", 11)[10] - seq[0].array("crg", 11)[10]) / np.sqrt(332.0716)
    assert abs(dq - 0.5) < 1e-3


def test_qdyn_log_layout():
    from q_b200.qdyn import write_out
    E = np.zeros(29)
    EQ = np.zeros((1, 15))
    EQ[0, 0] = 1.0
    EQ[0, 12], EQ[0, 13] = 3.1214, 139.4273
    text = write_out(E, EQ, 0, 1, 1117, True, 46, 46)
    assert "Energy summary at step      0" in text
    line = [l for l in text.split("\n") if l.startswith("Q-surr.")][0]
    assert line == "Q-surr. 1 1.0000      3.12    139.43"


# atoms x steps of a campaign's systems: 84 windows of one size, spheres of three
SHARD_COSTS = [3161 * 2] * 84 + [1392, 3423, 6500, 1392, 6500, 3423, 3423, 6500, 1392, 6500, 6500, 1392, 3423,
                                 3423, 1392, 6500]


def _gloo_worker(rank, world, port, out):
    import datetime

    import numpy as np
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from q_b200.dist import gather_series, max_over_ranks, shard, sum_over_ranks
    mine = shard(100, rank, world)
    t = max_over_ranks(1.0 + rank)
    n = sum_over_ranks(len(mine))
    owned = shard(len(SHARD_COSTS), rank, world, SHARD_COSTS)
    load = sum(SHARD_COSTS[i] for i in owned)
    # each rank's energy series of its systems (ragged lengths), gathered everywhere
    series = {i: np.full((3 + i % 4, 2), float(i)) for i in owned}
    allser = gather_series(series)
    out.put((rank, mine[:3], t, n, owned, load, {k: v.shape for k, v in allser.items()},
             all(np.all(v == k) for k, v in allser.items())))
    dist.destroy_process_group()


def test_multi_rank_helpers_gloo():
    import socket

    import torch.multiprocessing as tmp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res[0][:4] == (0, [0, 2, 4], 2.0, 100.0)
    assert res[1][:4] == (1, [1, 3, 5], 2.0, 100.0)
    # cost-balanced shards: disjoint, complete, loads within the LPT bound
    o0, o1 = res[0][4], res[1][4]
    assert sorted(o0 + o1) == list(range(len(SHARD_COSTS))) and not set(o0) & set(o1)
    loads = [res[0][5], res[1][5]]
    assert max(loads) <= 4 / 3 * sum(SHARD_COSTS) / 2 and max(loads) - min(loads) <= max(SHARD_COSTS)
    # every rank received every system's series with its own shape and values
    for r in res:
        assert r[6] == {i: (3 + i % 4, 2) for i in range(len(SHARD_COSTS))} and r[7]


def test_cost_shard_single_process():
    from q_b200.dist import shard
    costs = [5, 1, 1, 1, 1, 1]
    assert shard(6, 0, 2, costs) == [0] and shard(6, 1, 2, costs) == [1, 2, 3, 4, 5]
    assert shard(3, 0, 1, [1, 2, 3]) == [0, 1, 2]


def test_derived_inputs_and_restart(tmp_path):
    """An .inp derived with new keys, dropped keys and replaced rows opens
    like any input; a derived input that restarts from a written .re starts
    from its coordinates and velocities."""
    from q_b200.inputs import derive_inp, inp_sections
    g = synth.fep_solute(str(tmp_path / "c1"), seed=1234, steps=100)
    p = derive_inp(g.inp, "d1.inp", set_keys={"md": {"temperature": 150, "separate_scaling": "on"},
                                              "intervals": {"energy": 0}},
                   drop_keys={"files": ["energy"]},
                   set_rows={"sequence_restraints": ["1 56 5 0 0"], "lambdas": ["0.3 0.7"]})
    sec = inp_sections(p)
    md = dict(l.split(None, 1) for l in sec["md"])
    assert md["temperature"] == "150" and md["separate_scaling"] == "on" and md["steps"] == "100"
    assert not any(l.startswith("energy") for l in sec["files"])
    assert sec["sequence_restraints"] == ["1 56 5 0 0"] and sec["lambdas"] == ["0.3 0.7"]
    s = System.open(p)
    assert s.view.nrstr_seq == 1 and abs(s.view.Temp0 - 150.0) < 1e-12
    lam = getattr(s.view, "lambda")
    assert (lam[0], lam[1]) == (0.3, 0.7)
    x = s.array("x0", 3 * s.natom) + 0.01
    v = s.array("v0", 3 * s.natom) * 0.5
    write_restart(str(tmp_path / "c1" / "start.re"), x, v)
    q = derive_inp(g.inp, "d2.inp", set_keys={"files": {"restart": "start.re"}},
                   drop_keys={"md": ["random_seed", "initial_temperature"]})
    r = System.open(q)
    assert np.array_equal(r.array("x0", 3 * r.natom), x)


def test_dcd_layout_and_mask(tmp_path, golden):
    """The trajectory file has trj.f90's records; the mask follows mask.f90."""
    from q_b200.trajectory import DcdWriter, atom_mask, frame_steps, read_dcd
    s1 = System.open(str(golden / "test1" / "eq1.inp"))    # the view's arrays live as long as s1
    v = s1.view
    n, ns = v.natom, v.nat_solute
    excl = np.array(v.excl[:n], bool)
    heavy = np.array(v.heavy[:n], bool)
    assert atom_mask(v, []).sum() == n
    assert atom_mask(v, ["not excluded"]).sum() == n - excl.sum()
    assert np.array_equal(atom_mask(v, ["solute heavy"]), (np.arange(n) < ns) & heavy)
    assert np.array_equal(atom_mask(v, ["1 10", "not solute"]), (np.arange(n) < 10) | (np.arange(n) >= ns))
    assert atom_mask(v, ["5"]).sum() == 1 and atom_mask(v, ["5"])[4]
    with pytest.raises(ValueError):
        atom_mask(v, ["residue 1 2"])
    assert frame_steps(100, 10) == [11, 21, 31, 41, 51, 61, 71, 81, 91, 100]
    assert frame_steps(95, 10) == [11, 21, 31, 41, 51, 61, 71, 81, 91]
    m = atom_mask(v, ["not excluded"])
    path = str(tmp_path / "t.dcd")
    w = DcdWriter(path, m, frames=2, interval=10, steps=20, degf=v.Ndegfree, topology="lig_w.top",
                  mask_rows=["not excluded"])
    rng = np.random.default_rng(0)
    xs = [rng.normal(size=3 * n) for _ in range(2)]
    for x in xs:
        w.write(x)
    w.close()
    raw = open(path, "rb").read()
    assert raw[:8] == struct.pack("<i", 84) + b"CORD"
    assert struct.unpack_from("<i", raw, 88)[0] == 84                  # end marker of the header record
    assert struct.unpack_from("<i", raw, 92)[0] == 4 + 3 * 80          # title record: count + 3 rows
    h, fr = read_dcd(path)
    assert (h["frames"], h["steps_before"], h["interval"], h["steps"], h["degf"]) == (2, 10, 10, 20, v.Ndegfree)
    assert h["title"] == "Q DCD trajectory version 6.0.1" and h["topology"] == "lig_w.top"
    assert h["mask_rows"] == ["not excluded"] and h["atoms"] == m.sum()
    assert fr.shape == (2, m.sum(), 3)
    assert np.array_equal(fr[1], xs[1].reshape(-1, 3)[m].astype(np.float32))


def test_reference_cases_open(golden):
    """Every case of the reference's comparison harness reads and prepares:
    benzene, Na+ and benzene in water, water alone, the dual-topology FEP."""
    from tests.reference_cases import CASES, write_case
    sizes = {}
    for case in CASES:
        for shake in (False, True):
            s = System.open(write_case(str(golden / "data"), case, shake=shake))
            v = s.view
            sizes[case] = (v.natom, v.nqat)
            assert (v.shake_constraints > 0) == shake
    assert sizes["w-w"] == (3423, 0) and sizes["q-p-w_Na"] == (3418, 1) and sizes["dualtop"] == (98, 98)
