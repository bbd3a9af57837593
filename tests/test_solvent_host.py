"""Water whose hydrogens carry Lennard-Jones, on the host: which routines
take it (nonbon2_ww/nonbon2_qw under the arithmetic rule, the 3-atom
solvent's nonbond_3atomsolvent/nonbond_qw_3atom under the geometric one; the
SPC routines take O-O only), the O-H and H-H products set-up hands the
engine, and the solvent forms that are refused."""
import math

import pytest

from q_b200 import QBError, System, synth


def _products(rule, o, h):
    """(A, B) of two (sigma, epsilon) atoms under Q's rules: geometric
    sqrt(A_i A_j), sqrt(B_i B_j); arithmetic with R* = 2^(1/6) sigma / 2 and
    epsilon (md.f90 nonbon2_*)."""
    if rule == 1:
        a = [math.sqrt(4 * e * s ** 12) for s, e in (o, h)]
        b = [math.sqrt(4 * e * s ** 6) for s, e in (o, h)]
        return a[0] * a[1], b[0] * b[1]
    rs = [2 ** (1 / 6) * s / 2 for s, e in (o, h)]
    e = math.sqrt(o[1] * h[1])
    r6 = (rs[0] + rs[1]) ** 6
    return e * r6 * r6, 2 * e * r6


@pytest.mark.parametrize("rule,solvent,hlj", [(2, 0, True), (1, 1, True), (1, 0, False)])
def test_hydrogen_lj_products(tmp_path, rule, solvent, hlj):
    g = synth.water_sphere(str(tmp_path / "w"), radius=10.0, vdw_rule=rule, solvent_type=solvent,
                           water_h_lj=synth.TIP3P_H_LJ)
    s = System.open(g.inp)
    v = s.view
    assert v.ww_hlj == int(hlj)
    if not hlj:                     # SPC water under the geometric rule: O-O only
        assert v.A_OH == v.B_OH == v.A_HH == v.B_HH == 0.0
        return
    o, h = (synth.SIG_O, synth.EPS_O), synth.TIP3P_H_LJ
    tol = 1e-3 if rule == 2 else 1e-2  # the topology prints R*/epsilon to 5 decimals, sqrt(A) to 2 or 7
    for (A, B), (a, b) in (((v.A_OH, v.B_OH), _products(rule, o, h)), ((v.A_HH, v.B_HH), _products(rule, h, h))):
        assert A == pytest.approx(a, rel=tol) and B == pytest.approx(b, rel=tol)


def test_general_solvent_is_refused(tmp_path):
    """solvent_type 2 (mixed or non-3-atomic solvent) stops qdyn
    (md.f90:13802-13804), and is refused here."""
    g = synth.water_sphere(str(tmp_path / "w"), radius=8.0, solvent_type=2)
    with pytest.raises(QBError) as e:
        System.open(g.inp)
    assert e.value.code == 4 and "solvent_type 2" in str(e.value)


def test_three_atom_solvent_with_unlike_light_sites_is_refused(tmp_path):
    """The 3-atom routines read each site's own charge; the engine's water
    kernels take the two light sites as one hydrogen with -1/2 the first
    site's charge, so a solvent that breaks this is refused."""
    g = synth.water_sphere(str(tmp_path / "w"), radius=8.0, solvent_type=1)
    top = open(g.top).read().split("\n")
    k = next(i for i, l in enumerate(top) if "No. of atomic charges" in l)
    vals = top[k + 1].split()
    vals[1] = "%7.4f" % (float(vals[1]) + 0.01)     # the first water's first hydrogen
    top[k + 1] = " ".join(vals)
    open(g.top, "w").write("\n".join(top))
    with pytest.raises(QBError) as e:
        System.open(g.inp)
    assert e.value.code == 4 and "light sites" in str(e.value)
