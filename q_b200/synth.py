"""Seeded synthetic Q systems of the benchmark shapes, written as Q files.

The generator writes the Q topology format of topo_save (src/q6/topo.f90:1082,
same records and column formats), FEP files in the [section] format read by
qatom_load_fep (qatom.f90:874) and qdyn .inp files (md.f90:2528), so the engine
reads them through the same readers as any Q input.

Shapes (one generator per configuration):
  water_sphere(R)   TIP3P on a cubic lattice at 0.0334 / A^3 inside radius R,
                    seeded random orientations (config 0: R = 15).
  fep_solute(...)   a 32-heavy-atom random tree with hydrogens up to 56 atoms,
                    net-zero charges (hydrogens +0.10 +- 0.04, heavy atoms
                    ~N(0, 0.35) absorbing the balance), LJ from a 6-type
                    table, harmonic bonds/angles, periodic torsions (n=1..3),
                    periodic impropers on 3-connected centres, 8 Q-atoms with
                    two states (state 2: charge 0, epsilon x 0.5, soft-core),
                    solvated in a TIP3P sphere (config 1: R = 20).
  polymer_sphere()  a 3000-atom self-avoiding polymer walk (1.5 A steps,
                    non-bonded atoms >= 2.5 A apart) around the config-1 solute
                    in a 25 A sphere, charge groups of 10-15 atoms with net
                    charge -1/0/+1, atoms beyond 23 A excluded (restrained at
                    200 kcal/mol/A^2), remaining volume filled with water
                    (config 2).
Everything is deterministic in the seed (1234 + system id by default).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

DENSITY = 0.0334          # molecules / A^3
R_OH, ANG_HOH = 0.9572, 104.52
Q_O, Q_H = -0.834, 0.417
SIG_O, EPS_O = 3.15061, 0.1521
# the 6-type LJ table: sigma 3.0-3.5 A, epsilon 0.05-0.2 kcal/mol
TYPE_TABLE = [(3.00, 0.050, 12.011), (3.10, 0.080, 12.011), (3.20, 0.110, 14.007),
              (3.30, 0.140, 15.999), (3.40, 0.170, 12.011), (3.50, 0.200, 32.060)]
SIG_H, EPS_H, M_H = 2.50, 0.030, 1.008


def lj_sqrt(sigma: float, eps: float) -> tuple[float, float]:
    """Q's geometric-rule sqrt(A), sqrt(B) with A = 4 eps sigma^12, B = 4 eps sigma^6."""
    return 2.0 * math.sqrt(eps) * sigma ** 6, 2.0 * math.sqrt(eps) * sigma ** 3


@dataclass
class AtomType:
    name: str
    mass: float
    sigma: float
    eps: float

    def columns(self, vdw_rule: int = 1):
        """(a, b) for LJ codes normal, polar, 1-4 (1-4 at half epsilon):
        geometric rule sqrt(A), sqrt(B); arithmetic rule R* = 2^(1/6) sigma / 2
        and epsilon."""
        if vdw_rule == 2:
            rs = 2.0 ** (1.0 / 6.0) * self.sigma / 2.0
            return [(rs, self.eps), (rs, self.eps), (rs, self.eps / 2.0)]
        a, b = lj_sqrt(self.sigma, self.eps)
        return [(a, b), (a, b), (a / math.sqrt(2.0), b / math.sqrt(2.0))]


@dataclass
class Topology:
    """Atoms and terms of a Q topology; indices are 0-based here."""
    title: str = "synthetic"
    x: list = field(default_factory=list)
    iac: list = field(default_factory=list)
    crg: list = field(default_factory=list)
    types: list = field(default_factory=list)
    bonds: list = field(default_factory=list)        # (i, j, code)
    bond_lib: list = field(default_factory=list)     # (fk, b0)
    angles: list = field(default_factory=list)       # (i, j, k, code)
    angle_lib: list = field(default_factory=list)    # (fk, th0_deg[, urey_fk, urey_r0])
    tors: list = field(default_factory=list)         # (i, j, k, l, code)
    tor_lib: list = field(default_factory=list)      # (fk, rmult, delta_deg, paths)
    imps: list = field(default_factory=list)
    imp_lib: list = field(default_factory=list)      # (fk, imp0_deg)
    cgps: list = field(default_factory=list)         # (switch, [atoms])
    mol_starts: list = field(default_factory=list)
    res_starts: list = field(default_factory=list)
    res_names: list = field(default_factory=list)
    nat_solute: int = 0
    switch_atoms: int = 1       # 1: charge-group cut-offs on switch atoms; 0: on any atom pair (the *lis2 lists)
    nbonds_solute: int = 0
    nangles_solute: int = 0
    ntors_solute: int = 0
    nimps_solute: int = 0
    ncgp_solute: int = 0
    excl14: tuple = ((), ())                         # (exclusion pairs, 1-4 pairs) of solute atoms
    rexcl_o: float = 20.0
    rwat: float = 20.0
    excl: list = field(default_factory=list)
    vdw_rule: int = 1                                # 1 geometric, 2 arithmetic
    ff_type: int = 2                                 # 1 GROMOS, 2 AMBER, 3 CHARMM (Urey-Bradley, harmonic impropers)
    solvent_type: int = 0                            # 0 SPC-type water, 1 3-atom solvent (LJ on every site)
    water_h_lj: tuple = (0.0, 0.0)                   # sigma, epsilon of the water hydrogens
    box: tuple | None = None                         # periodic box: (edge lengths, centre)

    # ----------------------------------------------------------- writer
    def write(self, path: str) -> None:
        n = len(self.x)
        ns = self.nat_solute
        L = []
        L.append("Q topology file")
        L.append("TITLE      %s" % self.title)
        L.append("DATE       synthetic")
        L.append("VERSION     6.01")
        L.append("FORCEFIELD synthetic-geometric")
        L.append("FF_TYPE    %d" % self.ff_type)
        L.append("PRM_FILE   none")
        L.append("END        of header")
        L.append("%8d%8d = Total no. of atoms, no. of solute atoms. Coordinates: (2*3 per line)" % (n, ns))
        flat = [c for p in self.x for c in p]
        for k in range(0, len(flat), 6):
            L.append(" ".join("%9.3f" % v for v in flat[k:k + 6]))
        L.append("%8d = No. of integer atom codes. iac's: " % n)
        for k in range(0, n, 16):
            L.append(" ".join("%4d" % (t + 1) for t in self.iac[k:k + 16]))
        L.append("%8d%8d = No. of bonds, no. of solute bonds. i - j - icode: (5 per line)"
                 % (len(self.bonds), self.nbonds_solute))
        for k in range(0, len(self.bonds), 5):
            L.append(" ".join("%5d %5d %3d" % (i + 1, j + 1, c) for i, j, c in self.bonds[k:k + 5]))
        L.append("%8d = No. of bond codes. Parameters: " % len(self.bond_lib))
        for k, (fk, b0) in enumerate(self.bond_lib):
            L.append("%5d%9.3f %10.4f" % (k + 1, fk, b0))
        L.append("%8d%8d = No. of angles, no. of solute angles. i - j - k - icode: (3 per line)"
                 % (len(self.angles), self.nangles_solute))
        for k in range(0, len(self.angles), 3):
            L.append(" ".join("%5d %5d %5d %3d" % (i + 1, j + 1, kk + 1, c) for i, j, kk, c in self.angles[k:k + 3]))
        L.append("%8d = No. of angle codes. Parameters:" % len(self.angle_lib))
        for k, a in enumerate(self.angle_lib):
            fk, th, ufk, ur0 = (tuple(a) + (0.0, 0.0))[:4]
            L.append("%5d%9.3f %9.3f %9.3f %11.5f" % (k + 1, fk, th, ufk, ur0))
        L.append("%8d%8d = No. of torsions, solute torsions. i - j - k - l - icode: (2 per line)"
                 % (len(self.tors), self.ntors_solute))
        for k in range(0, len(self.tors), 2):
            L.append(" ".join("%5d %5d %5d %5d %3d" % (a + 1, b + 1, c + 1, d + 1, e)
                              for a, b, c, d, e in self.tors[k:k + 2]))
        L.append("%8d = No. of torsion codes. Parameters:" % len(self.tor_lib))
        for k, (fk, rm, dl, pa) in enumerate(self.tor_lib):
            L.append("%5d%9.3f %9.3f %9.3f %5d" % (k + 1, fk, rm, dl, pa))
        L.append("%8d%8d = No. of impropers, solute impr. i - j - k - l - icode: (2 per line)"
                 % (len(self.imps), self.nimps_solute))
        for k in range(0, len(self.imps), 2):
            L.append(" ".join("%5d %5d %5d %5d %3d" % (a + 1, b + 1, c + 1, d + 1, e)
                              for a, b, c, d, e in self.imps[k:k + 2]))
        L.append("%8d%8d = No. of improper codes, type (1=harmonic,2=periodic). Parameters:"
                 % (len(self.imp_lib), 2 if self.ff_type == 2 else 1))
        for k, (fk, i0) in enumerate(self.imp_lib):
            L.append("%5d%10.3f %10.3f" % (k + 1, fk, i0))
        L.append("%8d = No. of atomic charges" % n)
        for k in range(0, n, 10):
            L.append(" ".join("%7.4f" % q for q in self.crg[k:k + 10]))
        L.append("%8d%8d%8d = No. of charge groups, no of solvent cgps, switch atoms flag. nat_cgp, iswitch / atom list: "
                 % (len(self.cgps), self.ncgp_solute, self.switch_atoms))
        for sw, atoms in self.cgps:
            L.append("%5d %5d" % (len(atoms), sw + 1))
            for k in range(0, len(atoms), 13):
                L.append(" ".join("%5d" % (a + 1) for a in atoms[k:k + 13]))
        nt = len(self.types)
        L.append("%8d = No. of atom types" % nt)
        L.append("%8d = vdW combination rule (1 = Geom. / 2 = Arit.)" % self.vdw_rule)
        L.append("%8.5f%9.4f = Electrostatic 1-4 scaling factor and  Coulomb constant" % (0.5, 332.0))
        L.append("Masses: ")
        for k in range(0, nt, 10):
            L.append(" ".join("%7.3f" % t.mass for t in self.types[k:k + 10]))
        cols = [t.columns(self.vdw_rule) for t in self.types]
        names = ("Aii", "Bii") if self.vdw_rule == 1 else ("R*ii", "epsilon ii")
        def fmt(v):   # geometric: 2 decimals, more for small non-zero values (light atoms' sqrt(A))
            if self.vdw_rule == 2:
                return "%10.5f" % v
            return "%8.2f" % v if v == 0 or abs(v) >= 1 else "%10.7f" % v
        for c, label in enumerate(["normal", "polar", "1-4"]):
            for ab, nm in ((0, names[0]), (1, names[1])):
                L.append(("sqrt (%s) %s:" if self.vdw_rule == 1 else "%s %s:") % (nm, label))
                vals = [cols[t][c][ab] for t in range(nt)]
                for k in range(0, nt, 8):
                    L.append(" ".join(fmt(v) for v in vals[k:k + 8]))
        L.append("%8d = No. of type-2 vdW interactions. pairs: " % 0)
        ex_pairs, p14_pairs = self.excl14
        for pairs, label in ((p14_pairs, "1-4 neighbours"), (ex_pairs, "exclusions")):
            bits = np.zeros((ns, 25), dtype=np.int8)
            longp = []
            for i, j in pairs:
                a, b = min(i, j), max(i, j)
                if b - a <= 25:
                    bits[a, b - a - 1] = 1
                else:
                    longp.append((a, b))
            digits = "".join(str(v) for v in bits.reshape(-1))
            L.append("%8d = No. of %s. list (range=max_nbr_range): " % (len(pairs) - len(longp), label))
            for k in range(0, len(digits), 80):
                L.append(digits[k:k + 80])
            L.append("%8d = No. of long %s (>max_nbr_range). pairlist: " % (len(longp), label))
            for a, b in longp:
                L.append("%5d %5d" % (a + 1, b + 1))
        nres = len(self.res_starts)
        L.append("%8d%8d = No. of residues, No of solute residues. start atoms: " % (nres, 1 if ns else 0))
        for k in range(0, nres, 13):
            L.append(" ".join("%5d" % (a + 1) for a in self.res_starts[k:k + 13]))
        L.append("Sequence: ")
        for k in range(0, nres, 16):
            L.append(" ".join("%-4s" % nm for nm in self.res_names[k:k + 16]))
        L.append("%8d = No. of separate molecules. start atoms:" % len(self.mol_starts))
        for k in range(0, len(self.mol_starts), 13):
            L.append(" ".join("%5d" % (a + 1) for a in self.mol_starts[k:k + 13]))
        L.append("%8d = No. of atom types:" % nt)
        for k in range(0, nt, 8):
            L.append(" ".join("%-8s" % t.name for t in self.types[k:k + 8]))
        L.append("%8d = No. of SYBYL atom types:" % nt)
        for k in range(0, nt, 13):
            L.append(" ".join("%-5s" % "" for _ in self.types[k:k + 13]))
        L.append("%8d = solvent type (0=SPC,1=3-atom,2=general)" % self.solvent_type)
        if self.box is not None:
            # periodic box (topo.f90:1027-1034): no excluded atoms follow
            lengths, centre = self.box
            L.append("%8s = kind of boundary" % "PBC")
            L.append("%8.3f%8.3f%8.3f = Size of box, x y z" % tuple(lengths))
            L.append("%8.3f%8.3f%8.3f = Center coordinate of box" % tuple(centre))
            with open(path, "w") as f:
                f.write("\n".join(L) + "\n")
            return
        L.append("%8.3f%8.3f = Exclusion, solvent radii" % (self.rexcl_o, self.rwat))
        L.append("%8.3f%8.3f%8.3f = Solute center" % (0.0, 0.0, 0.0))
        L.append("%8.3f%8.3f%8.3f = Solvent center" % (0.0, 0.0, 0.0))
        excl = self.excl or [False] * n
        nexwat = sum(1 for k in range(ns, n, 3) if excl[k])
        L.append("%8d%8d = No. of excluded atoms (incl. water), no. of excluded waters" % (sum(excl), nexwat))
        s = "".join("T" if e else "F" for e in excl)
        for k in range(0, n, 80):
            L.append(s[k:k + 80])
        with open(path, "w") as f:
            f.write("\n".join(L) + "\n")


# ------------------------------------------------------------- geometry

def _rot(rng) -> np.ndarray:
    """Uniform random rotation (random unit quaternion)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _water_template() -> np.ndarray:
    h = math.radians(ANG_HOH / 2)
    return np.array([[0, 0, 0], [R_OH * math.sin(h), R_OH * math.cos(h), 0],
                     [-R_OH * math.sin(h), R_OH * math.cos(h), 0]])


def lattice_waters(radius: float, rng, avoid: np.ndarray | None = None, r_o: float = 2.8,
                   inner: float = 0.0) -> list[np.ndarray]:
    """TIP3P waters on a cubic lattice at DENSITY, O within `radius` of the
    origin (and beyond `inner`), seeded random orientations; waters with O
    within r_o of an `avoid` atom are dropped."""
    a = (1.0 / DENSITY) ** (1.0 / 3.0)
    n = int(math.ceil(radius / a)) + 1
    g = (np.arange(-n, n + 1) + 0.5) * a
    P = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T
    r = np.linalg.norm(P, axis=1)
    P = P[(r <= radius) & (r >= inner)]
    P = P[np.lexsort((P[:, 2], P[:, 1], P[:, 0]))]
    if avoid is not None and len(avoid):
        from scipy.spatial import cKDTree
        d, _ = cKDTree(avoid).query(P)
        P = P[d >= r_o]
    t = _water_template()
    return [p + t @ _rot(rng).T for p in P]


def _add_waters(top: Topology, waters: list[np.ndarray], excl_radius: float | None = None) -> None:
    types = {t.name: i for i, t in enumerate(top.types)}
    if "OW" not in types:
        top.types.append(AtomType("OW", 15.999, SIG_O, EPS_O))
        top.types.append(AtomType("HW", 1.008, *top.water_h_lj))
        types = {t.name: i for i, t in enumerate(top.types)}
    ow, hw = types["OW"], types["HW"]
    top.bond_lib.append((1106.0, R_OH))
    cb_oh = len(top.bond_lib)
    hh = 2 * R_OH * math.sin(math.radians(ANG_HOH / 2))
    top.bond_lib.append((0.0, hh))
    cb_hh = len(top.bond_lib)
    top.angle_lib.append((200.0, ANG_HOH))
    ca = len(top.angle_lib)
    for w in waters:
        o = len(top.x)
        top.mol_starts.append(o)
        top.res_starts.append(o)
        top.res_names.append("HOH")
        for k in range(3):
            top.x.append(tuple(float(c) for c in w[k]))
        top.iac += [ow, hw, hw]
        top.crg += [Q_O, Q_H, Q_H]
        top.bonds += [(o, o + 1, cb_oh), (o, o + 2, cb_oh), (o + 1, o + 2, cb_hh)]
        top.angles.append((o + 1, o, o + 2, ca))
        top.cgps.append((o, [o, o + 1, o + 2]))
        if excl_radius is not None:
            out = float(np.linalg.norm(w[0])) > excl_radius
            top.excl += [out] * 3


def _finish_solute_lists(top: Topology, bonds: list[tuple[int, int]], n: int) -> None:
    """1-2/1-3 exclusions and 1-4 pairs from the bond graph of solute atoms."""
    nb = [set() for _ in range(n)]
    for i, j in bonds:
        nb[i].add(j)
        nb[j].add(i)
    ex, p14 = set(), set()
    for i in range(n):
        for j in nb[i]:
            ex.add((min(i, j), max(i, j)))
            for k in nb[j]:
                if k != i:
                    ex.add((min(i, k), max(i, k)))
    for i in range(n):
        for j in nb[i]:
            for k in nb[j]:
                if k == i:
                    continue
                for l in nb[k]:
                    if l in (i, j):
                        continue
                    p = (min(i, l), max(i, l))
                    if p not in ex:
                        p14.add(p)
    top.excl14 = (sorted(ex), sorted(p14))


def dihedral_deg(xi, xj, xk, xl) -> float:
    """The dihedral i-j-k-l in degrees with Q's sign convention (md.f90
    torsion/improper: normals rji x rjk and rkl x rjk, signed by rjk)."""
    rji, rjk, rkl = xi - xj, xk - xj, xl - xk
    nj, nk = np.cross(rji, rjk), -np.cross(rjk, rkl)
    c = float(nj @ nk / (np.linalg.norm(nj) * np.linalg.norm(nk)))
    phi = math.degrees(math.acos(max(-1.0, min(1.0, c))))
    return -phi if float(rjk @ np.cross(nj, nk)) < 0 else phi


def charmm_terms(top: Topology, ub_fk: float = 25.0, imp_fk: float = 20.0) -> None:
    """Turn a solute's terms into CHARMM ones: every solute angle gets a
    Urey-Bradley 1-3 term whose r0 is 3% longer than the 1-3 distance of the
    generated geometry, and the impropers become harmonic about the
    geometry's own improper angle."""
    top.ff_type = 3
    X = np.asarray(top.x, dtype=float)
    for i, j, k, c in top.angles[:top.nangles_solute]:
        fk, th = top.angle_lib[c - 1][:2]
        r13 = float(np.linalg.norm(X[k] - X[i]))
        top.angle_lib[c - 1] = (fk, th, ub_fk, round(1.03 * r13, 4))
    for i, j, k, l, c in top.imps[:top.nimps_solute]:
        top.imp_lib[c - 1] = (imp_fk, round(dihedral_deg(X[i], X[j], X[k], X[l]), 3))


def _angle(a, b, c) -> float:
    u, v = a - b, c - b
    return math.degrees(math.acos(max(-1.0, min(1.0, float(u @ v / (np.linalg.norm(u) * np.linalg.norm(v)))))))


def random_tree_solute(rng, n_heavy: int = 32, n_total: int = 56):
    """Heavy-atom tree with hydrogens; returns coordinates, element kinds
    (type index or -1 for H), bonds.  Bond angles stay within 105-150 degrees
    (hydrogens 100-150): the angle terms take the generated geometry as their
    equilibrium, and a harmonic angle close to linear has a cusp at 180
    degrees (its force flips direction there) that feeds energy into the
    bend until the constraints of a neighbouring hydrogen fail."""
    X = [np.zeros(3)]
    bonds = []
    deg = [0]
    while len(X) < n_heavy:
        for _ in range(2000):
            p = int(rng.integers(len(X)))
            if deg[p] >= 3:
                continue
            u = rng.normal(size=3)
            u /= np.linalg.norm(u)
            c = X[p] + u * rng.uniform(1.40, 1.54)
            d = np.linalg.norm(np.array(X) - c, axis=1)
            d[p] = 99
            if d.min() < 2.5:
                continue
            if any(not 105 <= _angle(X[q], X[p], c) <= 150
                   for (a, b) in bonds for q in ((b,) if a == p else (a,) if b == p else ())):
                continue
            X.append(c)
            deg.append(1)
            deg[p] += 1
            bonds.append((p, len(X) - 1))
            break
        else:
            raise RuntimeError("tree growth failed")
    kinds = [int(rng.integers(len(TYPE_TABLE))) for _ in range(n_heavy)]
    # hydrogens on heavy atoms with free valence, leaves first
    order = sorted(range(n_heavy), key=lambda i: (deg[i], i))
    need = n_total - n_heavy
    while need > 0:
        placed = False
        for p in order:
            if need == 0:
                break
            if deg[p] >= 4:
                continue
            for _ in range(500):
                u = rng.normal(size=3)
                u /= np.linalg.norm(u)
                c = X[p] + u * 1.09
                d = np.linalg.norm(np.array(X) - c, axis=1)
                d[p] = 99
                if d.min() < 2.0:
                    continue
                nbrs = [b if a == p else a for a, b in bonds if p in (a, b)]
                if any(not 100 <= _angle(X[q], X[p], c) <= 150 for q in nbrs):
                    continue
                X.append(c)
                kinds.append(-1)
                deg.append(1)
                deg[p] += 1
                bonds.append((p, len(X) - 1))
                need -= 1
                placed = True
                break
        if not placed:
            raise RuntimeError("hydrogen placement failed")
    X = np.array(X)
    return X - X.mean(axis=0), kinds, bonds


def _solute_terms(top: Topology, X: np.ndarray, bonds, rng, offset: int = 0, heavy_fk=600.0) -> None:
    n = len(X)
    nb = [[] for _ in range(n)]
    for i, j in bonds:
        nb[i].append(j)
        nb[j].append(i)
    for i, j in bonds:
        b0 = float(np.linalg.norm(X[i] - X[j]))
        fk = 700.0 if b0 < 1.2 else heavy_fk
        top.bond_lib.append((fk, round(b0, 4)))
        top.bonds.append((offset + i, offset + j, len(top.bond_lib)))
    for j in range(n):
        for a in range(len(nb[j])):
            for b in range(a + 1, len(nb[j])):
                i, k = nb[j][a], nb[j][b]
                top.angle_lib.append((70.0, round(_angle(X[i], X[j], X[k]), 3)))
                top.angles.append((offset + i, offset + j, offset + k, len(top.angle_lib)))
    for j, k in bonds:
        for i in nb[j]:
            if i == k:
                continue
            for l in nb[k]:
                if l == j or l == i:
                    continue
                nmul = int(rng.integers(1, 4))
                top.tor_lib.append((round(float(rng.uniform(0.2, 1.5)), 3), float(nmul),
                                    float(rng.choice([0.0, 180.0])), 1))
                top.tors.append((offset + i, offset + j, offset + k, offset + l, len(top.tor_lib)))
    for j in range(n):
        if len(nb[j]) == 3:
            i, k, l = nb[j]
            top.imp_lib.append((1.1, 180.0))
            top.imps.append((offset + i, offset + j, offset + k, offset + l, len(top.imp_lib)))


def _tree_types(kinds) -> tuple[list[AtomType], list[int]]:
    types = [AtomType("H", M_H, SIG_H, EPS_H)] + [AtomType("T%d" % (k + 1), m, s, e)
                                                  for k, (s, e, m) in enumerate(TYPE_TABLE)]
    return types, [0 if k < 0 else k + 1 for k in kinds]


def _net_zero_charges(rng, n: int, sd: float = 0.3, total: float = 0.0) -> list[float]:
    q = rng.normal(0.0, sd, size=n)
    q = q - q.mean() + total / n
    q = np.round(q, 4)
    q[-1] = round(total - float(q[:-1].sum()), 4)
    return [float(v) for v in q]


def _solute_charges(rng, kinds) -> list[float]:
    """Net-zero partial charges of a tree solute in force-field ranges:
    hydrogens +0.10 +- 0.04 (within 0..0.20), heavy atoms 0.35 sigma (within
    +-0.70) shifted to cancel the total.  A hydrogen never carries a negative
    charge: water hydrogens have no Lennard-Jones repulsion, and a negative
    hydrogen binds them at about 1.2 A until a collision breaks the water's
    constraints.  Draws the same random numbers as _net_zero_charges(rng, n)."""
    z = rng.normal(0.0, 1.0, size=len(kinds))
    hyd = np.array([k < 0 for k in kinds])
    q = np.where(hyd, np.clip(0.10 + 0.04 * z, 0.0, 0.20), np.clip(0.35 * z, -0.70, 0.70))
    heavy = np.flatnonzero(~hyd)
    q[heavy] -= q.sum() / len(heavy)
    q = np.round(q, 4)
    q[heavy[-1]] = round(-float(q.sum() - q[heavy[-1]]), 4)
    return [float(v) for v in q]


# -------------------------------------------------------------- systems

@dataclass
class Generated:
    inp: str
    top: str
    fep: str | None
    natom: int
    nwat: int


def write_inp(path: str, top: str, fep: str | None, *, steps: int, stepsize: float, temp: float = 298.0,
              seed: int = 1, lambdas=None, shake_hydrogens: bool = False, bath: float = 100.0,
              output: int = 100, energy: int = 10, non_bond: int = 25, shell_radius: float | None = None,
              shell_force: float = 10.0, q_cutoff: float = 99.0, energy_file: str | None = None,
              trajectory: int = 0, trajectory_atoms=None, restart: str | None = None,
              sequence_restraints=None, separate_scaling: bool = False,
              initial_temperature: float | None = None, pbc: dict | None = None, lrf_cutoff: float = 99.0,
              volume_change: int | None = None, distance_restraints=None, lrf: bool = True) -> None:
    """A qdyn .inp (md.f90:2528-3262 sections).  With restart, coordinates
    and velocities come from that .re and no seed or initial temperature is
    written; trajectory > 0 adds the .dcd file and its [trajectory_atoms]
    rows; sequence_restraints are rows "first last force_k to_centre heavy",
    distance_restraints rows "i j d1 d2 force_k state".  pbc: the [PBC]
    section's keys and values (md.f90:2583-2656), volume_change the
    [intervals] key of constant pressure."""
    name = os.path.splitext(os.path.basename(path))[0]
    L = []
    if pbc is not None:
        L += ["[PBC]"] + ["%s %s" % (k, v) for k, v in pbc.items()] + [""]
    L += ["[MD]", "steps %d" % steps, "stepsize %g" % stepsize, "temperature %g" % temp, "bath_coupling %g" % bath]
    if restart is None:
        t0 = temp if initial_temperature is None else initial_temperature
        L += ["random_seed %d" % seed, "initial_temperature %g" % t0]
    L += ["shake_solvent on", "shake_solute off", "shake_hydrogens %s" % ("on" if shake_hydrogens else "off"),
          "lrf %s" % ("on" if lrf else "off")]
    if separate_scaling:
        L.append("separate_scaling on")
    L += ["", "[cut-offs]", "solute_solute 10", "solvent_solvent 10", "solute_solvent 10",
         "q_atom %g" % q_cutoff, "lrf %g" % lrf_cutoff, "", "[sphere]"]
    if shell_radius is not None:
        L.append("shell_radius %g" % shell_radius)
    L += ["shell_force %g" % shell_force, "", "[solvent]", "radial_force 60.0", "polarization on",
          "polarization_force 20.0", "", "[intervals]", "non_bond %d" % non_bond, "output %d" % output,
          "energy %d" % energy, "trajectory %d" % trajectory]
    if volume_change is not None:
        L.append("volume_change %d" % volume_change)
    L += ["", "[files]", "topology %s" % os.path.basename(top), "final %s.re" % name]
    if restart:
        L.append("restart %s" % os.path.basename(restart))
    if energy > 0:
        L.append("energy %s" % (energy_file or name + ".en"))
    if trajectory > 0:
        L.append("trajectory %s.dcd" % name)
    if fep:
        L.append("fep %s" % os.path.basename(fep))
    if trajectory > 0 and trajectory_atoms:
        L += ["", "[trajectory_atoms]"] + list(trajectory_atoms)
    if fep:
        L += ["", "[lambdas]", " ".join("%g" % x for x in lambdas)]
    if sequence_restraints:
        L += ["", "[sequence_restraints]"] + list(sequence_restraints)
    if distance_restraints:
        L += ["", "[distance_restraints]"] + list(distance_restraints)
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


# water hydrogens with Lennard-Jones (sigma, epsilon), as CHARMM's TIP3P has them
TIP3P_H_LJ = (0.4, 0.046)


def water_sphere(outdir: str, radius: float = 15.0, seed: int = 1234, steps: int = 1000, name: str = "c0",
                 stepsize: float = 1.0, vdw_rule: int = 1, water_h_lj=(0.0, 0.0), solvent_type: int = 0) -> Generated:
    """Config 0: TIP3P sphere, 1 fs, energies every 10 steps.  water_h_lj
    gives the hydrogens LJ; solvent_type 1 writes the water as 3-atom
    solvent."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    top = Topology(title="water_sphere_%g" % radius, rexcl_o=radius, rwat=radius, vdw_rule=vdw_rule,
                   water_h_lj=tuple(water_h_lj), solvent_type=solvent_type)
    _add_waters(top, lattice_waters(radius, rng))
    top.excl = [False] * len(top.x)
    tp = os.path.join(outdir, name + ".top")
    top.write(tp)
    inp = os.path.join(outdir, name + ".inp")
    write_inp(inp, tp, None, steps=steps, stepsize=stepsize, seed=seed % 100000 + 1, energy=10)
    return Generated(inp, tp, None, len(top.x), (len(top.x)) // 3)


def _q_bonded(top: Topology, qatoms: list[int], couplings: bool = False) -> list[str]:
    """FEP sections redefining the topology's bonds, angles, torsions and
    impropers that lie wholly among the Q atoms: state 1 keeps the topology's
    parameters, state 2 changes them (the first bond becomes a Morse bond of
    the same curvature, the last torsion is absent).  Impropers centred on a
    Q atom are redefined too, harmonic
    about the geometry's own improper angle in both states; under CHARMM the
    angle types carry the topology's Urey-Bradley columns, halved in state 2.
    With couplings, the first bond is a Morse bond in state 1 and absent in
    state 2 (a bond that breaks), and the angles, torsions and impropers
    holding both its atoms are coupled to it (EVB Morse couplings; the first
    improper coupling with gamma = 1 - EMorseD)."""
    qs = set(qatoms)
    X = np.asarray(top.x, dtype=float)
    L = []
    bonds = [(i, j, c) for i, j, c in top.bonds[:top.nbonds_solute] if i in qs and j in qs]
    if bonds:
        L += ["[bond_types]"]
        for n, (i, j, c) in enumerate(bonds):
            fk, b0 = top.bond_lib[c - 1]
            if n == 0 and couplings:
                L.append("%d %8.3f %6.3f %8.4f" % (2 * n + 1, fk / 8.0, 2.0, b0))
            else:
                L.append("%d %8.2f %8.4f" % (2 * n + 1, fk, b0))
            if n == 0:
                amz = 2.0
                L.append("%d %8.3f %6.3f %8.4f" % (2 * n + 2, fk / (2 * amz * amz), amz, b0 + 0.03))
            else:
                L.append("%d %8.2f %8.4f" % (2 * n + 2, 0.8 * fk, b0 + 0.02))
        L += ["", "[change_bonds]"]
        L += ["%d %d %d %d" % (i + 1, j + 1, 2 * n + 1, 0 if (n == 0 and couplings) else 2 * n + 2)
              for n, (i, j, c) in enumerate(bonds)]
        L += [""]
    angles = [(i, j, k, c) for i, j, k, c in top.angles[:top.nangles_solute] if i in qs and j in qs and k in qs]
    if angles:
        L += ["[angle_types]"]
        for n, (i, j, k, c) in enumerate(angles):
            fk, th, ufk, ur0 = (tuple(top.angle_lib[c - 1]) + (0.0, 0.0))[:4]
            for st, (f, t, u, r) in enumerate(((fk, th, ufk, ur0), (0.7 * fk, th + 4.0, 0.5 * ufk, ur0 + 0.05))):
                row = "%d %8.3f %8.3f" % (2 * n + 1 + st, f, t)
                L.append(row + (" %8.3f %8.4f" % (u, r) if top.ff_type == 3 else ""))
        L += ["", "[change_angles]"]
        L += ["%d %d %d %d %d" % (i + 1, j + 1, k + 1, 2 * n + 1, 2 * n + 2) for n, (i, j, k, c) in enumerate(angles)]
        L += [""]
    tors = [t for t in top.tors[:top.ntors_solute] if all(a in qs for a in t[:4])]
    if tors:
        L += ["[torsion_types]"]
        for n, (i, j, k, l, c) in enumerate(tors):
            fk, rm, dl, pa = top.tor_lib[c - 1]
            L.append("%d %8.3f %6.1f %8.2f" % (2 * n + 1, fk / pa, rm, dl))
            L.append("%d %8.3f %6.1f %8.2f" % (2 * n + 2, 0.5 * fk / pa, rm, dl))
        L += ["", "[change_torsions]"]
        L += ["%d %d %d %d %d %d" % (i + 1, j + 1, k + 1, l + 1, 2 * n + 1, 0 if n == len(tors) - 1 else 2 * n + 2)
              for n, (i, j, k, l, c) in enumerate(tors)]
        L += [""]
    imps = [t for t in top.imps[:top.nimps_solute] if t[1] in qs]
    if imps:
        L += ["[improper_types]"]
        for n, (i, j, k, l, c) in enumerate(imps):
            phi = round(dihedral_deg(X[i], X[j], X[k], X[l]), 3)
            L += ["%d %8.3f %8.3f" % (2 * n + 1, 15.0, phi), "%d %8.3f %8.3f" % (2 * n + 2, 25.0, phi)]
        L += ["", "[change_impropers]"]
        L += ["%d %d %d %d %d %d" % (i + 1, j + 1, k + 1, l + 1, 2 * n + 1, 2 * n + 2)
              for n, (i, j, k, l, c) in enumerate(imps)]
        L += [""]
    if couplings and bonds:
        a, b = bonds[0][0], bonds[0][1]
        hold = lambda t: a in t and b in t
        ca = [n + 1 for n, t in enumerate(angles) if hold(t[:3])]
        ct = [n + 1 for n, t in enumerate(tors) if hold(t[:4])]
        ci = [n + 1 for n, t in enumerate(imps) if hold(t[:4])]
        if ca:
            L += ["[angle_couplings]"] + ["%d 1" % n for n in ca] + [""]
        if ct:
            L += ["[torsion_couplings]"] + ["%d 1" % n for n in ct] + [""]
        if ci:
            L += ["[improper_couplings]"] + ["%d 1%s" % (n, " 1" if k == 0 else "") for k, n in enumerate(ci)] + [""]
    return L


def _fep_file(path: str, types: list[AtomType], iac: list[int], q: list[float], qatoms: list[int],
              alpha: float = 20.0, charge_scale: float = 0.0, eps_scale: float = 0.5, vdw_rule: int = 1,
              top: Topology | None = None, soft_pairs=(), library_charges: bool = False, off_diagonals=(),
              couplings: bool = False) -> None:
    """Two-state FEP file: state 2 scales the Q-atoms' charges by
    charge_scale and their epsilon by eps_scale, soft-core alpha in state 2.
    Given the topology, the bonded terms among the Q atoms are redefined too
    (_q_bonded).  soft_pairs (Q-atom index pairs, 0-based) interact by
    exponential repulsion A_i A_j exp(-B_i B_j r) instead of LJ, with the Q
    types' second parameter pair set for it; library_charges turns on
    qq_use_library_charges; off_diagonals = [(state_i, state_j, qatom_k,
    qatom_l, A, mu)] (1-based) are EVB off-diagonal functions."""
    L = ["[FEP]", "states 2"] + (["qq_use_library_charges on"] if library_charges else []) + ["", "[atoms]"]
    L += ["%d %d" % (k + 1, a + 1) for k, a in enumerate(qatoms)]
    L += ["", "[change_charges]"]
    L += ["%d %8.4f %8.4f" % (k + 1, q[a], round(q[a] * charge_scale, 4)) for k, a in enumerate(qatoms)]
    L += ["", "[atom_types]"]
    names = []
    for k, a in enumerate(qatoms):
        t = types[iac[a]]
        for st, scale in ((1, 1.0), (2, eps_scale)):
            nm = "Q%d_%d" % (k + 1, st)
            ea, eb = ((31.62, 1.87) if st == 1 else (25.0, 1.87)) if soft_pairs else (0.0, 0.0)
            if vdw_rule == 2:   # R*, epsilon (not square-rooted: the engine does it), 1-4 at half epsilon
                rs = 2.0 ** (1.0 / 6.0) * t.sigma / 2.0
                e = t.eps * scale
                L.append("%-8s %9.5f %9.5f %6.2f %6.2f %9.5f %9.5f %8.4f" % (nm, rs, e, ea, eb, rs, e / 2.0, t.mass))
            else:
                aa, bb = lj_sqrt(t.sigma, t.eps * scale)
                L.append("%-8s %9.2f %8.2f %6.2f %6.2f %9.2f %8.2f %8.4f"
                         % (nm, aa, bb, ea, eb, aa / math.sqrt(2), bb / math.sqrt(2), t.mass))
        names.append(("Q%d_1" % (k + 1), "Q%d_2" % (k + 1)))
    L += ["", "[change_atoms]"]
    L += ["%d %s %s" % (k + 1, a, b) for k, (a, b) in enumerate(names)]
    L += ["", "[softcore]"]
    L += ["%d %g %g" % (k + 1, 0.0, alpha) for k in range(len(qatoms))]
    if soft_pairs:
        L += ["", "[soft_pairs]"] + ["%d %d" % (a + 1, b + 1) for a, b in soft_pairs]
    if off_diagonals:
        L += ["", "[off_diagonals]"] + ["%d %d %d %d %g %g" % tuple(o) for o in off_diagonals]
    if top is not None:
        L += [""] + _q_bonded(top, qatoms, couplings)
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def solute_parameters(seed: int = 1234):
    """(kinds, types, iac, charges) of the tree solute fep_solute(seed=seed)
    builds: the same random draws in the same order."""
    rng = np.random.default_rng(seed)
    X, kinds, bonds = random_tree_solute(rng)
    types, iac = _tree_types(kinds)
    return kinds, types, iac, _solute_charges(rng, kinds)


def perturbation(base: Generated, name: str, qatoms, charge_scale: float, eps_scale: float,
                 seed: int = 1234, steps: int = 5000, run_seed: int = 1, lambdas=(1.0, 0.0)) -> Generated:
    """Another perturbation of fep_solute's system (same topology `base`, its
    files written beside it): the given solute atoms become two-state Q-atoms
    whose state 2 carries charge_scale x their charge and eps_scale x their
    epsilon (soft-core in state 2)."""
    outdir = os.path.dirname(base.top)
    kinds, types, iac, crg = solute_parameters(seed)
    fp = os.path.join(outdir, name + ".fep")
    _fep_file(fp, types, iac, crg, [int(a) for a in qatoms], charge_scale=charge_scale, eps_scale=eps_scale)
    inp = os.path.join(outdir, name + ".inp")
    write_inp(inp, base.top, fp, steps=steps, stepsize=2.0, seed=run_seed, lambdas=lambdas, shake_hydrogens=True)
    return Generated(inp, base.top, fp, base.natom, base.nwat)


def fep_solute(outdir: str, radius: float = 20.0, seed: int = 1234, steps: int = 5000, name: str = "c1",
               lambdas=(0.5, 0.5), run_seed: int = 1, vdw_rule: int = 1, ff_type: int = 2,
               q_bonded: bool = False, ub_fk: float = 25.0, soft_pairs: int = 0,
               library_charges: bool = False, water_h_lj=(0.0, 0.0), solvent_type: int = 0,
               off_diagonals=(), morse_couplings: bool = False, switch_atoms: int = 1) -> Generated:
    """Config 1: 56-atom solute with 8 two-state Q-atoms in a TIP3P sphere,
    2 fs with SHAKE on X-H bonds and water.  ff_type 3 writes it as a CHARMM
    topology (charmm_terms, Urey-Bradley constant ub_fk); q_bonded redefines the bonded terms among the
    Q atoms in the FEP file.  soft_pairs > 0 makes that many Q-atom pairs
    beyond 1-4 soft pairs; library_charges sets qq_use_library_charges.
    water_h_lj and solvent_type as for water_sphere; off_diagonals as for
    _fep_file; morse_couplings (with q_bonded) couples the Q terms of the
    first Q bond to it (_q_bonded)."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    X, kinds, bonds = random_tree_solute(rng)
    types, iac = _tree_types(kinds)
    n = len(X)
    top = Topology(title="fep_solute", rexcl_o=radius, rwat=radius, types=types, vdw_rule=vdw_rule,
                   water_h_lj=tuple(water_h_lj), solvent_type=solvent_type, switch_atoms=switch_atoms)
    top.x = [tuple(float(c) for c in p) for p in X]
    top.iac = iac
    top.crg = _solute_charges(rng, kinds)
    _solute_terms(top, X, bonds, rng)
    top.nat_solute = n
    top.nbonds_solute, top.nangles_solute = len(top.bonds), len(top.angles)
    top.ntors_solute, top.nimps_solute = len(top.tors), len(top.imps)
    nb = [[] for _ in range(n)]
    for i, j in bonds:
        nb[i].append(j)
        nb[j].append(i)
    for i in range(n):
        if kinds[i] >= 0:
            top.cgps.append((i, [i] + sorted(j for j in nb[i] if kinds[j] < 0)))
    top.ncgp_solute = len(top.cgps)
    top.mol_starts = [0]
    top.res_starts, top.res_names = [0], ["LIG"]
    _finish_solute_lists(top, bonds, n)
    waters = lattice_waters(radius, rng, avoid=X)
    _add_waters(top, waters)
    top.excl = [False] * len(top.x)
    if ff_type == 3:
        charmm_terms(top, ub_fk=ub_fk)
    tp = os.path.join(outdir, name + ".top")
    top.write(tp)
    fp = os.path.join(outdir, name + ".fep")
    heavy = [i for i in range(n) if kinds[i] >= 0]
    qat = heavy[:8]
    near = {tuple(sorted(p)) for p in list(top.excl14[0]) + list(top.excl14[1])}
    far = [(a, b) for a in range(len(qat)) for b in range(a + 1, len(qat)) if tuple(sorted((qat[a], qat[b]))) not in near]
    _fep_file(fp, types, iac, top.crg, qat, vdw_rule=vdw_rule, top=top if q_bonded else None,
              soft_pairs=far[:soft_pairs], library_charges=library_charges, off_diagonals=off_diagonals,
              couplings=morse_couplings)
    inp = os.path.join(outdir, name + ".inp")
    write_inp(inp, tp, fp, steps=steps, stepsize=2.0, seed=run_seed, lambdas=lambdas, shake_hydrogens=True)
    return Generated(inp, tp, fp, len(top.x), len(waters))


def box_waters(edge: float, rng, avoid: np.ndarray | None = None, r_o: float = 2.8) -> list[np.ndarray]:
    """TIP3P waters filling a cubic periodic box of the given edge, centred on
    the origin: a lattice of n^3 sites (n = edge * DENSITY^(1/3), rounded) that
    tiles the box, seeded random orientations; waters with O within r_o of an
    `avoid` atom (nearest image) are dropped."""
    n = max(2, int(round(edge * DENSITY ** (1.0 / 3.0))))
    a = edge / n
    g = (np.arange(n) + 0.5) * a - edge / 2
    P = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T
    if avoid is not None and len(avoid):
        from scipy.spatial import cKDTree
        d, _ = cKDTree(np.mod(avoid + edge / 2, edge), boxsize=edge).query(np.mod(P + edge / 2, edge))
        P = P[d >= r_o]
    t = _water_template()
    return [p + t @ _rot(rng).T for p in P]


def fep_box(outdir: str, edge: float = 30.0, seed: int = 1234, steps: int = 1000, name: str = "pbc",
            lambdas=(0.5, 0.5), run_seed: int = 1, constant_pressure: bool = False, volume_change: int = 10,
            max_volume_displ: float = 300.0, pressure_seed: int = 3781, put_back: bool = True,
            rigid_box_center: bool = False, lrf: float | None = 14.0, q_cutoff: float = 12.0,
            distance_restraints=None) -> Generated:
    """The FEP solute of fep_solute (56 atoms, 8 two-state Q-atoms) in a
    cubic periodic box of TIP3P water (use_PBC): 2 fs, SHAKE on X-H bonds and
    water, 10 A cut-offs, Q-atom cut-off q_cutoff around the first Q atom
    (the FEP file's [PBC] switching_atom), LRF to `lrf` A (None: no LRF).  constant_pressure
    adds Monte Carlo volume moves every volume_change steps (MC_volume);
    put_back puts solute and solvent back in the box at the list steps."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    X, kinds, bonds = random_tree_solute(rng)
    types, iac = _tree_types(kinds)
    n = len(X)
    top = Topology(title="fep_box", types=types, box=((edge, edge, edge), (0.0, 0.0, 0.0)))
    top.x = [tuple(float(c) for c in p) for p in X]
    top.iac = iac
    top.crg = _solute_charges(rng, kinds)
    _solute_terms(top, X, bonds, rng)
    top.nat_solute = n
    top.nbonds_solute, top.nangles_solute = len(top.bonds), len(top.angles)
    top.ntors_solute, top.nimps_solute = len(top.tors), len(top.imps)
    nb = [[] for _ in range(n)]
    for i, j in bonds:
        nb[i].append(j)
        nb[j].append(i)
    for i in range(n):
        if kinds[i] >= 0:
            top.cgps.append((i, [i] + sorted(j for j in nb[i] if kinds[j] < 0)))
    top.ncgp_solute = len(top.cgps)
    top.mol_starts = [0]
    top.res_starts, top.res_names = [0], ["LIG"]
    _finish_solute_lists(top, bonds, n)
    waters = box_waters(edge, rng, avoid=X)
    _add_waters(top, waters)
    tp = os.path.join(outdir, name + ".top")
    top.write(tp)
    fp = os.path.join(outdir, name + ".fep")
    heavy = [i for i in range(n) if kinds[i] >= 0]
    qat = heavy[:8]
    _fep_file(fp, types, iac, top.crg, qat)
    with open(fp, "a") as f:
        f.write("\n[PBC]\nswitching_atom %d\n" % (qat[0] + 1))
    pbc = {"rigid_box_center": "on" if rigid_box_center else "off",
           "constant_pressure": "on" if constant_pressure else "off",
           "put_solvent_back_in_box": "on" if put_back else "off",
           "put_solute_back_in_box": "on" if put_back else "off"}
    if constant_pressure:
        pbc.update({"max_volume_displ": "%g" % max_volume_displ, "pressure_seed": "%d" % pressure_seed,
                    "pressure": "1.0"})
    inp = os.path.join(outdir, name + ".inp")
    write_inp(inp, tp, fp, steps=steps, stepsize=2.0, seed=run_seed, lambdas=lambdas, shake_hydrogens=True,
              pbc=pbc, lrf_cutoff=lrf or 0.0, q_cutoff=q_cutoff,
              volume_change=volume_change if constant_pressure else None,
              distance_restraints=distance_restraints, lrf=lrf is not None)
    return Generated(inp, tp, fp, len(top.x), len(waters))


def _relax_chains(X: np.ndarray, n_fixed: int, chains, radius: float, target: float = 3.0, iters: int = 400,
                  bond: float = 1.5) -> np.ndarray:
    """Spread a grown set of chains apart before the system is written: atoms
    of non-bonded pairs (not 1-2 or 1-3 along a chain) closer than `target`
    are pushed apart, chain bonds kept at `bond`, chain angles kept within
    100-150 degrees (1-3 distances), every atom within radius - 0.5; the first
    n_fixed atoms (the ligand) do not move.  A random walk packed at 2.5 A
    starts with thousands of kcal/mol of steric strain, which 2 fs dynamics
    turns into heat and the polymer cannot survive; relaxed, it can."""
    from scipy.spatial import cKDTree
    X = X.copy()
    n = len(X)
    cid = np.full(n, -1)
    pos = np.zeros(n, dtype=int)
    for c, ch in enumerate(chains):
        cid[ch] = c
        pos[ch] = np.arange(len(ch))
    b = np.array([(a, b) for ch in chains for a, b in zip(ch[:-1], ch[1:])], dtype=int).reshape(-1, 2)
    a13 = np.array([(a, c) for ch in chains for a, c in zip(ch[:-2], ch[2:])], dtype=int).reshape(-1, 2)
    lo13, hi13 = 2 * bond * np.sin(np.radians(50.0)), 2 * bond * np.sin(np.radians(75.0))
    mobile = np.ones(n, dtype=bool)
    mobile[:n_fixed] = False
    for _ in range(iters):
        pr = cKDTree(X).query_pairs(target, output_type="ndarray")
        if len(pr):
            i, j = pr[:, 0], pr[:, 1]
            near = (cid[i] == cid[j]) & (cid[i] >= 0) & (np.abs(pos[i] - pos[j]) <= 2)
            i, j = i[~near], j[~near]
            d = X[j] - X[i]
            r = np.linalg.norm(d, axis=1)[:, None]
            push = 0.25 * (target - r) / np.maximum(r, 1e-6) * d
            disp = np.zeros_like(X)
            np.add.at(disp, i, -push)
            np.add.at(disp, j, push)
            disp[~mobile] = 0.0
            step = np.linalg.norm(disp, axis=1)[:, None]
            X += disp * np.minimum(1.0, 0.2 / np.maximum(step, 1e-12))
        for pairs, lo, hi in ((b, bond, bond), (a13, lo13, hi13)):
            for half in (0, 1):            # alternate pairs: no atom moved twice per pass
                p = pairs[half::2] if len(pairs) else pairs
                if not len(p):
                    continue
                d = X[p[:, 1]] - X[p[:, 0]]
                r = np.linalg.norm(d, axis=1)
                goal = np.clip(r, lo, hi)
                corr = ((r - goal) / np.maximum(r, 1e-9))[:, None] * d
                w0 = mobile[p[:, 0]].astype(float)
                w1 = mobile[p[:, 1]].astype(float)
                tot = np.maximum(w0 + w1, 1.0)[:, None]
                X[p[:, 0]] += corr * (w0[:, None] / tot)
                X[p[:, 1]] -= corr * (w1[:, None] / tot)
        rr = np.linalg.norm(X, axis=1)
        out = (rr > radius - 0.5) & mobile
        X[out] *= ((radius - 0.5) / rr[out])[:, None]
    return X


def polymer_sphere(outdir: str, radius: float = 25.0, seed: int = 1234, steps: int = 5000, name: str = "c2",
                   n_polymer: int = 3000, restrain_beyond: float = 23.0, lambdas=(0.5, 0.5),
                   min_dist: float = 2.5, charge_sd: float = 0.3, max_angle: float = 150.0,
                   angle_fk: float = 60.0, shell_radius: float | None = None, relax: bool = True,
                   switch_atoms: int = 0) -> Generated:
    """Config 2: 3000-atom polymer walk around the config-1 solute (ligand) in
    a 25 A sphere; atoms beyond 23 A are excluded and restrained; waters fill
    the remaining volume.

    The chains are spread apart after growth (_relax_chains) and each torsion's
    phase puts the starting dihedral at its minimum, so the start carries little
    strain.  The charge groups are residue-like runs of 10-15 chain atoms, which
    a random walk stretches over up to ~10 A; with switch-atom cut-offs two
    groups whose switch atoms lie beyond 10 A leave their closest atoms without
    any non-bonded interaction, and chains then pass through each other and the
    dynamics fails within ~100 steps.  The topology therefore asks for the
    any-atom cut-offs (switch_atoms 0: nbpplis2_lrf, nbpwlis2_lrf, nbqplis2),
    under which the system is stable.

    Waters: 3,000 atoms at >= 2.5 A non-bonded spacing fill most of the sphere
    (random close packing of 2.5 A spheres is ~0.078 A^-3, i.e. >= 39,000 of the
    sphere's 65,450 A^3), and the walk spreads them over all of it, so the
    waters that fit (O >= 2.6 A from every solute atom) number ~200, not the
    ~1,500 the configuration's prose expects; 1,500 waters alone need 44,900
    A^3 at 0.0334 A^-3."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    Xl, kinds, lbonds = random_tree_solute(rng)
    from scipy.spatial import cKDTree
    # self-avoiding chains, restarted where a chain gets stuck
    pts = [p for p in Xl]
    chains = []
    cell = max(2.5, min_dist)

    grid: dict = {}

    def gkey(p):
        return tuple((p // cell).astype(int))

    def add(p):
        grid.setdefault(gkey(p), []).append(len(pts) - 1)

    for k in range(len(pts)):
        grid.setdefault(gkey(pts[k]), []).append(k)

    def free(p, skip):
        if np.linalg.norm(p) > radius - 0.5:
            return False
        kx, ky, kz = gkey(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get((kx + dx, ky + dy, kz + dz), ()):
                        if q != skip and np.linalg.norm(pts[q] - p) < min_dist:
                            return False
        return True

    total = 0
    while total < n_polymer:
        for _ in range(5000):
            start = rng.uniform(-radius, radius, size=3)
            if np.linalg.norm(start) < radius - 1.0 and free(start, -1):
                break
        chain = [len(pts)]
        pts.append(start)
        add(start)
        total += 1
        while total < n_polymer:
            ok = False
            for _ in range(60):
                u = rng.normal(size=3)
                u /= np.linalg.norm(u)
                c = pts[chain[-1]] + 1.5 * u
                # chain angles within [100, max_angle] degrees (no near-linear angle terms)
                if len(chain) > 1 and not 100 <= _angle(pts[chain[-2]], pts[chain[-1]], c) <= max_angle:
                    continue
                if free(c, chain[-1]):
                    ok = True
                    break
            if not ok:
                break
            pts.append(c)
            add(c)
            chain.append(len(pts) - 1)
            total += 1
        chains.append(chain)
    n_lig = len(Xl)
    X = np.array(pts)
    if relax:
        X = _relax_chains(X, n_lig, chains, radius)
    n = len(X)
    types, _ = _tree_types(kinds)
    iac = [0 if k < 0 else k + 1 for k in kinds] + [1 + int(rng.integers(len(TYPE_TABLE))) for _ in range(n - n_lig)]
    top = Topology(title="polymer_sphere", rexcl_o=restrain_beyond, rwat=radius, types=types,
                   switch_atoms=switch_atoms)
    top.x = [tuple(float(c) for c in p) for p in X]
    top.iac = iac
    crg = _solute_charges(rng, kinds)
    pbonds = [(a, b) for ch in chains for a, b in zip(ch[:-1], ch[1:])]
    # residue-like charge groups of 10-15 consecutive chain atoms, net charge -1/0/+1
    groups = []
    for ch in chains:
        k = 0
        while k < len(ch):
            m = int(rng.integers(10, 16))
            groups.append(ch[k:k + m])
            k += m
    pcrg = np.zeros(n)
    for g in groups:
        net = float(rng.choice([-1.0, 0.0, 1.0]))
        pcrg[g] = _net_zero_charges(rng, len(g), sd=charge_sd, total=net)
    top.crg = crg + [float(v) for v in pcrg[n_lig:]]
    _solute_terms(top, Xl, lbonds, rng)
    # polymer terms (harmonic bonds/angles, torsions along the chains)
    nbp = [[] for _ in range(n)]
    for i, j in pbonds:
        nbp[i].append(j)
        nbp[j].append(i)
    for i, j in pbonds:
        top.bond_lib.append((500.0, round(float(np.linalg.norm(X[i] - X[j])), 4)))
        top.bonds.append((i, j, len(top.bond_lib)))
    for ch in chains:
        for a, b, c in zip(ch[:-2], ch[1:-1], ch[2:]):
            top.angle_lib.append((angle_fk, round(_angle(X[a], X[b], X[c]), 3)))
            top.angles.append((a, b, c, len(top.angle_lib)))
        for a, b, c, d in zip(ch[:-3], ch[1:-2], ch[2:-1], ch[3:]):
            fk, mult = round(float(rng.uniform(0.2, 1.5)), 3), float(rng.integers(1, 4))
            if relax:
                # the phase that puts the starting dihedral at the term's minimum
                phase = round(float((mult * dihedral_deg(X[a], X[b], X[c], X[d]) - 180.0) % 360.0), 2)
            else:
                phase = float(rng.choice([0.0, 180.0]))
            top.tor_lib.append((fk, mult, phase, 1))
            top.tors.append((a, b, c, d, len(top.tor_lib)))
    top.nat_solute = n
    top.nbonds_solute, top.nangles_solute = len(top.bonds), len(top.angles)
    top.ntors_solute, top.nimps_solute = len(top.tors), len(top.imps)
    nbl = [[] for _ in range(n_lig)]
    for i, j in lbonds:
        nbl[i].append(j)
        nbl[j].append(i)
    for i in range(n_lig):
        if kinds[i] >= 0:
            top.cgps.append((i, [i] + sorted(j for j in nbl[i] if kinds[j] < 0)))
    for g in groups:
        top.cgps.append((g[len(g) // 2], sorted(g)))
    top.ncgp_solute = len(top.cgps)
    top.mol_starts = [0] + [ch[0] for ch in chains]
    top.res_starts = [0] + [g[0] for g in groups]
    top.res_names = ["LIG"] + ["POL"] * len(groups)
    _finish_solute_lists(top, lbonds + pbonds, n)
    top.excl = [bool(np.linalg.norm(X[i]) > restrain_beyond) for i in range(n)]
    waters = lattice_waters(radius, rng, avoid=X, r_o=2.6)
    _add_waters(top, waters, excl_radius=restrain_beyond)
    tp = os.path.join(outdir, name + ".top")
    top.write(tp)
    fp = os.path.join(outdir, name + ".fep")
    heavy = [i for i in range(n_lig) if kinds[i] >= 0]
    _fep_file(fp, types, iac, top.crg, heavy[:8])
    inp = os.path.join(outdir, name + ".inp")
    write_inp(inp, tp, fp, steps=steps, stepsize=2.0, seed=1, lambdas=lambdas, shake_hydrogens=True,
              q_cutoff=99.0, shell_radius=shell_radius if shell_radius is not None else restrain_beyond - 0.01)
    return Generated(inp, tp, fp, len(top.x), len(waters))


def window_lambdas(n_windows: int) -> list[tuple[float, float]]:
    """Uniform lambda windows (lambda_1, 1 - lambda_1) from 1 to 0."""
    return [(1.0 - k / (n_windows - 1), k / (n_windows - 1)) for k in range(n_windows)]
