// setup.cpp -- prepare a parsed Q system the way qdyn does before md_run.
//
// Order follows src/q6/qdyn.f90:80-96: topology (md.f90:14705), prep_coord
// (13596), get_fep (1472), prep_sim (13787), init_shake (2326),
// make_nbqqlist (1022), shrink_topology (14569), and with a seed maxwell
// (3787), initial_shaking (2506), stop_cm_translation (14670).  This is
// one-off host set-up; the per-step work runs in the CUDA engine.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "qsystem.hpp"

namespace qb {

namespace {

// randm (md.f90:14408-14442): LCG with mult 31415821, modulus 1e8; the
// returned value is formed in single precision.
struct Randm {
  bool init = false;
  int irand = 0;
  double next(int &ig) {
    const int m = 100000000, m1 = 10000, mult = 31415821;
    if (!init) { init = true; irand = std::abs(ig) % m; }
    int irandh = irand / m1, irandl = irand % m1;
    int multh = mult / m1, multl = mult % m1;
    irand = ((irandh * multl + irandl * multh) % m1) * m1 + irandl * multl;
    irand = (irand + 1) % m;
    float r = (float)(irand / 10) * 10.0f / (float)m;
    if (r <= 0.0f || r > 1.0f) r = 0.0f;
    ig = irand;
    return (double)r;
  }
};

// shake (md.f90:14445-14566) on host, used only by initial_shaking.
int host_shake(System &s, std::vector<double> &xx, std::vector<double> &x) {
  int total = 0;
  for (size_t m = 0; m < s.sh_first.size(); m++) {
    int f = s.sh_first[m], n = s.sh_n[m];
    std::vector<char> ready(n, 0);
    int nits = 0;
    for (;;) {
      for (int c = 0; c < n; c++) {
        if (ready[c]) continue;
        int i = s.sh_i[f + c], j = s.sh_j[f + c];
        double xij[3], xxij[3];
        for (int k = 0; k < 3; k++) xij[k] = x[3 * i + k] - x[3 * j + k];
        double xij2 = xij[0] * xij[0] + xij[1] * xij[1] + xij[2] * xij[2];
        double diff = s.sh_d2[f + c] - xij2;
        if (std::fabs(diff) < 0.0001 * s.sh_d2[f + c]) ready[c] = 1;
        for (int k = 0; k < 3; k++) xxij[k] = xx[3 * i + k] - xx[3 * j + k];
        double scp = xij[0] * xxij[0] + xij[1] * xxij[1] + xij[2] * xxij[2];
        double wi = s.winv[i], wj = s.winv[j];
        float wsum = s.winv[i] + s.winv[j];
        double corr = diff / (2.0 * scp * (double)wsum);
        for (int k = 0; k < 3; k++) {
          x[3 * i + k] += xxij[k] * corr * wi;
          x[3 * j + k] -= xxij[k] * corr * wj;
        }
      }
      nits++;
      bool all = true;
      for (int c = 0; c < n; c++) all = all && ready[c];
      if (all) break;
      if (nits >= 1000) fail(QB_ERR_SHAKE, "shake failure during initial shaking");
    }
    total += nits;
  }
  return s.top.nmol ? total / s.top.nmol : 0;
}

}  // namespace

// put_back_in_box (md.f90:15477-15600): molecules whose centre of mass left
// the box (centred on the solute's mean position unless the centre is rigid)
// move by one edge length per axis.
void put_back_in_box(System &s) {
  const Topology &t = s.top;
  const RunInput &in = s.in;
  const int N = s.natom, NS = t.nat_solute, nmol = t.nmol;
  if (!in.rigid_box_center) {
    const int n = NS > 0 ? NS : N;
    double c[3] = {0, 0, 0};
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) c[k] += s.x[3 * i + k];
    for (int k = 0; k < 3; k++) s.boxc[k] = c[k] / n;
  }
  int first = 0, last = nmol;   // [first, last) molecules
  if (nmol > 1) {
    const int nsolv = (N - NS) / (t.istart_mol[nmol - 1] - t.istart_mol[nmol - 2]);
    if (!in.put_solute_back_in_box) first = nmol - nsolv;
    if (!in.put_solvent_back_in_box) last = nmol - nsolv;
  }
  for (int m = first; m < last; m++) {
    double cm[3] = {0, 0, 0};
    for (int j = t.istart_mol[m]; j < t.istart_mol[m + 1]; j++)
      for (int k = 0; k < 3; k++) cm[k] += s.x[3 * j + k] * s.mass_box[j];
    for (int k = 0; k < 3; k++) {
      cm[k] = cm[k] * s.mol_minv[m];
      const double hi = s.boxc[k] + s.boxl[k] / 2, lo = s.boxc[k] - s.boxl[k] / 2;
      double sh = 0.0;
      if (cm[k] > hi) sh = -s.boxl[k];
      else if (cm[k] < lo) sh = s.boxl[k];
      if (sh != 0.0)
        for (int j = t.istart_mol[m]; j < t.istart_mol[m + 1]; j++) s.x[3 * j + k] += sh;
    }
  }
}

void prepare(System &s) {
  RunInput &in = s.in;
  Topology &t = s.top;
  Fep &f = s.fep;
  char buf[512];

  // ---------------------------------------------------------- topology()
  read_topology(in.top_file, t);
  if (t.ivdw_rule != 1 && t.ivdw_rule != 2) fail(QB_ERR_PARSE, "unknown LJ combination rule in the topology");
  // arithmetic rule: epsilon -> sqrt(|epsilon|) now (md.f90:14747-14751),
  // before the FEP file's soft-core table is built from it
  if (t.ivdw_rule == 2)
    for (auto &ty : t.iaclib)
      for (int k = 0; k < 3; k++) ty.bvdw[k] = std::sqrt(std::fabs(ty.bvdw[k]));
  if (t.solvent_type == 2 && t.nat_pro > t.nat_solute)
    fail(QB_ERR_UNSUPPORTED, "mixed or non-3-atomic solvent (solvent_type 2) is not supported");
  if (t.solvent_type != 0 && t.solvent_type != 1 && t.nat_pro > t.nat_solute)
    fail(QB_ERR_PARSE, "unknown solvent type in the topology");
  if (t.ff_type < 1 || t.ff_type > 3) fail(QB_ERR_UNSUPPORTED, "unknown force-field type in the topology");
  s.natom = t.nat_pro;
  s.nwat = (s.natom - t.nat_solute) / 3;
  const int N = s.natom, NS = t.nat_solute;
  // boundary (md.f90:14752-14788): the same in topology and input; the box
  // must hold twice every cut-off
  if (in.box != t.use_pbc) fail(QB_ERR_PARSE, "Must have same boundary (sphere or box) in topology and input file");
  if (t.use_pbc) {
    const double box_min = std::min(t.boxlength[0], std::min(t.boxlength[1], t.boxlength[2]));
    if (!(box_min > in.Rcpp * 2)) fail(QB_ERR_PARSE, "Solute-solute cut-off radii too large");
    if (!(box_min > in.Rcww * 2)) fail(QB_ERR_PARSE, "Solvent-solvent cut-off radii too large");
    if (!(box_min > in.Rcpw * 2)) fail(QB_ERR_PARSE, "Solute-solvent cut-off radii too large");
    if (!(box_min > in.Rcq * 2)) fail(QB_ERR_PARSE, "Q-atom cut-off radii too large");
    if (!(box_min > in.RcLRF * 2)) fail(QB_ERR_PARSE, "LRF cut-off radii too large");
    for (int k = 0; k < 3; k++) { s.boxl[k] = t.boxlength[k]; s.boxc[k] = t.boxcenter[k]; }
  }
  const double deg2rad = fortran_deg2rad();
  for (auto &a : t.ang_th0) a = deg2rad * a;
  for (auto &p : t.tor_paths) p = 1.0f / p;
  for (auto &d : t.tor_deltor) d = (float)(deg2rad * (double)d);
  for (auto &d : t.imp_imp0) d = (float)(deg2rad * (double)d);
  s.ljcod.assign((size_t)t.natyps * t.natyps, 1);
  for (auto &p : t.lj2) {
    s.ljcod[(size_t)p.first * t.natyps + p.second] = 2;
    s.ljcod[(size_t)p.second * t.natyps + p.first] = 2;
  }

  // -------------------------------------------------------- prep_coord()
  // the restrained shell exists in the sphere only (md.f90:13627)
  if (!t.use_pbc && in.rexcl_i > t.rexcl_o) fail(QB_ERR_PARSE, "inner radius of restrained shell must be < exclusion radius");
  double rexcl_i = in.rexcl_i;
  s.shell.assign(N, 0);
  s.nshellats = 0;
  if (!t.use_pbc && rexcl_i >= 0) {
    if (rexcl_i <= 1.00) rexcl_i = rexcl_i * t.rexcl_o;
    double rin2 = rexcl_i * rexcl_i;
    for (int ig = 0; ig < t.ncgp_solute; ig++) {
      int sw = t.cgp_iswitch[ig];
      if (t.excl[sw] || !t.heavy[sw]) continue;
      double r2;
      if (t.iuse_switch_atom == 1) {  // make_shell (md.f90:13694)
        r2 = 0;
        for (int k = 0; k < 3; k++) { double d = t.xtop[3 * sw + k] - t.xpcent[k]; r2 += d * d; }
      } else {  // make_shell2 (md.f90:13727): charge group centre
        double c[3] = {0, 0, 0};
        for (int a = t.cgp_first[ig]; a <= t.cgp_last[ig]; a++)
          for (int k = 0; k < 3; k++) c[k] += t.xtop[3 * t.cgpatom[a] + k];
        double nn = (double)(float)(t.cgp_last[ig] - t.cgp_first[ig] + 1);
        r2 = 0;
        for (int k = 0; k < 3; k++) { c[k] /= nn; double d = c[k] - t.xpcent[k]; r2 += d * d; }
      }
      if (r2 > rin2)
        for (int a = t.cgp_first[ig]; a <= t.cgp_last[ig]; a++) { s.nshellats++; s.shell[t.cgpatom[a]] = 1; }
    }
  }
  in.rexcl_i = rexcl_i;
  s.iqatom.assign(N, -1);
  s.x.assign(t.xtop.begin(), t.xtop.end());
  s.v.assign(3 * (size_t)N, 0.0);

  // ------------------------------------------------------------ get_fep()
  const int S = (int)in.lambdas.size();
  f.nstates = 0;
  f.nqat = 0;
  if (S > 0) {
    read_fep_atoms(in.fep_file, t, f, S);
    if (f.nstates != S) {
      std::snprintf(buf, sizeof buf, "FEP file has %d states but the input gives %d lambda values", f.nstates, S);
      fail(QB_ERR_PARSE, buf);
    }
    for (int i = 0; i < f.nqat; i++) {
      if (f.iqseq[i] >= 0) s.iqatom[f.iqseq[i]] = i;
      else fail(QB_ERR_PARSE, "Q-atom not defined in [atoms]");
    }
    f.qcrg.assign((size_t)f.nqat * S, 0.0f);
    for (int i = 0; i < f.nqat; i++)
      for (int j = 0; j < S; j++) f.qcrg[i * S + j] = t.crg[f.iqseq[i]];
    read_fep(in.fep_file, t, f);
    // arithmetic rule: the Q-atom types' epsilons (LJ codes 1 and 3) are
    // square-rooted after the soft-core table (md.f90:1519-1523)
    if (t.ivdw_rule == 2 && f.qvdw_flag)
      for (int k = 0; k < f.nqlib; k++) {
        f.qbvdw[3 * k + 0] = std::sqrt(f.qbvdw[3 * k + 0]);
        f.qbvdw[3 * k + 2] = std::sqrt(f.qbvdw[3 * k + 2]);
      }
    // remove redefined interactions from the topology (md.f90:1512-1598)
    for (auto &b : t.bnd)
      for (auto &q : f.qbnd)
        if ((b.i == q.i && b.j == q.j) || (b.i == q.j && b.j == q.i)) b.cod = 0;
    for (auto &a : t.ang)
      for (auto &q : f.qang)
        if ((a.i == q.i && a.j == q.j && a.k == q.k) || (a.i == q.k && a.j == q.j && a.k == q.i)) a.cod = 0;
    for (auto &tt : t.tor)
      for (auto &q : f.qtor)
        if (((tt.i == q.i && tt.j == q.j && tt.k == q.k && tt.l == q.l) ||
             (tt.i == q.l && tt.j == q.k && tt.k == q.j && tt.l == q.i)) && tt.cod != 0)
          tt.cod = 0;
    if (t.ff_type == 3) {
      // CHARMM: an improper goes when one of its ends is an end of the Q
      // improper and its two centre atoms are both among the Q improper's
      // four atoms (md.f90:1574-1594)
      for (auto &im : t.imp)
        for (auto &q : f.qimp) {
          auto in4 = [&](int a) { return a == q.i || a == q.j || a == q.k || a == q.l; };
          bool end = im.i == q.i || im.i == q.l || im.l == q.i || im.l == q.l;
          if (end && in4(im.j) && in4(im.k) && im.cod != 0) im.cod = 0;
        }
    } else {
      for (auto &im : t.imp)
        for (auto &q : f.qimp)
          if (((im.j == q.j && im.k == q.k) || (im.j == q.k && im.k == q.j)) && im.cod != 0) im.cod = 0;
    }
    // special exclusions that hold in every state go to the exclusion lists
    for (auto &e : f.exspec) {
      if (e.i < 0 || e.i >= N || e.j < 0 || e.j >= N) fail(QB_ERR_PARSE, "invalid special exclusion data");
      if (s.iqatom[e.i] < 0 || s.iqatom[e.j] < 0) {
        bool any = false, all = true;
        for (int st = 0; st < S; st++) { any = any || e.flag[st]; all = all && e.flag[st]; }
        if (any) {
          if (!all) fail(QB_ERR_PARSE, "special exclusion of a non-Q pair must hold in all states");
          int i = e.i, j = e.j;
          if (std::abs(j - i) <= QB_NBR_RANGE) {
            if (i < j) t.listex[i] |= 1u << (j - i - 1);
            else t.listex[j] |= 1u << (i - j - 1);
          } else {
            t.listexlong.push_back({i, j});
          }
        }
      }
    }
  }
  const int nq = f.nqat;

  // ----------------------------------------------------------- prep_sim()
  s.crgtot = 0;
  s.crgQtot = 0;
  s.rwat = t.rwat;
  if (s.nwat > 0 && t.use_pbc) {
    // periodic box: no solvent sphere or polarisation shells (md.f90:13806)
    s.crg_ow = t.crg[NS];
    s.crg_hw = -s.crg_ow / 2.0f;
    in.wpol_restr = false;
    s.nwpolr_shell = 0;
  } else if (s.nwat > 0) {
    s.crg_ow = t.crg[NS];
    s.crg_hw = -s.crg_ow / 2.0f;
    // wat_sphere (md.f90:14961)
    if (in.rwat_in > 0.) s.rwat = in.rwat_in;
    double ctot = 0.0, cq = 0.0;
    for (int i = 0; i < NS; i++)
      if (!t.excl[i] && s.iqatom[i] < 0) ctot += t.crg[i];
    for (int i = 0; i < nq; i++)
      for (int st = 0; st < S; st++) {
        ctot += f.qcrg[i * S + st] * in.lambdas[st];
        cq += f.qcrg[i * S + st] * in.lambdas[st];
      }
    s.crgtot = ctot;
    s.crgQtot = in.wpol_born ? cq : 0.0;
    s.fk_wsphere = in.fk_wsphere == -1 ? 60.0 : in.fk_wsphere;
    s.fkwpol = in.fkwpol == -1 ? 20.0 : in.fkwpol;
    s.Dwmz = in.Dwmz == -1 ? 0.26 * std::exp(-0.19 * (s.rwat - 15.)) + 0.74 : in.Dwmz;
    s.awmz = in.awmz == -1 ? 0.2 / (1. + std::exp(0.4 * (s.rwat - 25.))) + 0.3 : in.awmz;
    if (in.wpol_restr) {
      // wat_shells (md.f90:15044)
      int bndcodw = t.bnd.back().cod, angcodw = t.ang.back().cod;
      if (bndcodw <= 0 || angcodw <= 0) fail(QB_ERR_PARSE, "last bond/angle of the topology must be a water term");
      s.mu_w = (float)(-(double)s.crg_ow * t.bond_b0[bndcodw - 1] * std::cos(t.ang_th0[angcodw - 1] / 2));
      const double pi = fortran_pi();
      double drs = (double)(3.0001f / 0.5f);
      s.nwpolr_shell = (int)(-0.5 + std::sqrt(2 * drs + 0.25));
      int ns = s.nwpolr_shell;
      s.ws_rout.assign(ns, 0); s.ws_dr.assign(ns, 0); s.ws_cstb.assign(ns, 0); s.ws_theta_corr.assign(ns, 0);
      double rout = s.rwat;
      for (int is = 0; is < ns; is++) {
        s.ws_rout[is] = (float)rout;
        double dr = (double)(0.5f * (float)(is + 1));
        double ri = rout - dr;
        s.ws_dr[is] = (float)dr;
        double rshell = std::pow(0.5 * (rout * rout * rout + ri * ri * ri), (double)(1.0f / 3.0f));
        float rm = kRhoWat * s.mu_w * 4.0f;
        s.ws_cstb[is] = (float)(s.crgQtot * (double)0.98750f / ((double)rm * pi * (rshell * rshell)));
        rout = rout - dr;
      }
    }
  }
  s.iwhich_cgp.assign(N, 0);
  for (int ig = 0; ig < t.ncgp; ig++)
    for (int a = t.cgp_first[ig]; a <= t.cgp_last[ig]; a++) s.iwhich_cgp[t.cgpatom[a]] = ig;
  s.winv.resize(N);
  s.mass.resize(N);
  for (int i = 0; i < N; i++) {
    s.mass[i] = t.iaclib[t.iac[i]].mass;
    s.winv[i] = (float)(1.0 / s.mass[i]);
  }
  const double sqc = std::sqrt(t.coulomb_constant);
  for (auto &c : t.crg) c = (float)((double)c * sqc);
  s.crg_ow = (float)((double)s.crg_ow * sqc);
  s.crg_hw = (float)((double)s.crg_hw * sqc);
  s.qcrg_scaled.resize(f.qcrg.size());
  for (size_t i = 0; i < f.qcrg.size(); i++) s.qcrg_scaled[i] = (float)((double)f.qcrg[i] * sqc);

  // --------------------------------------------------------- init_shake()
  const int nmol = t.nmol;
  std::vector<std::vector<int>> mi(nmol), mj(nmol);
  std::vector<std::vector<double>> md2(nmol);
  double exclshk = 0;
  auto shaken = [&](int ia, int ja) {
    return (in.shake_hydrogens && (!t.heavy[ia] || !t.heavy[ja])) || (in.shake_solute && ia < NS) ||
           (in.shake_solvent && ia >= NS);
  };
  {
    int mol = -1;
    for (auto &b : t.bnd) {
      while (b.i >= t.istart_mol[mol + 1]) mol++;
      if (b.cod == 0) continue;
      if (shaken(b.i, b.j)) {
        if (t.excl[b.i]) exclshk += 0.5;
        if (t.excl[b.j]) exclshk += 0.5;
        mi[mol].push_back(b.i);
        mj[mol].push_back(b.j);
        md2[mol].push_back(t.bond_b0[b.cod - 1] * t.bond_b0[b.cod - 1]);
        b.cod = -1;
      }
    }
  }
  for (auto &q : f.qshake) {
    int mol = 0;
    while (q.i >= t.istart_mol[mol + 1]) mol++;
    double dd = 0;
    for (int st = 0; st < S; st++) dd += in.lambdas[st] * q.dist[st];
    size_t c = 0;
    for (; c < mi[mol].size(); c++)
      if ((q.i == mi[mol][c] && q.j == mj[mol][c]) || (q.j == mi[mol][c] && q.i == mj[mol][c])) break;
    if (c == mi[mol].size()) { mi[mol].push_back(0); mj[mol].push_back(0); md2[mol].push_back(0); }
    mi[mol][c] = q.i; mj[mol][c] = q.j; md2[mol][c] = dd * dd;
  }
  int solute_shake = 0;
  for (int m = 0; m < nmol - s.nwat; m++) solute_shake += (int)mi[m].size();
  // molecules without constraints are squeezed out (md.f90:2437-2452)
  std::vector<int> order;
  {
    std::vector<int> slot(nmol);
    for (int m = 0; m < nmol; m++) slot[m] = m;
    std::vector<size_t> cnt(nmol);
    for (int m = 0; m < nmol; m++) cnt[m] = mi[m].size();
    int trg = 0, src = 1;
    while (src < nmol) {
      if (cnt[trg] == 0) {
        slot[trg] = slot[src]; cnt[trg] = cnt[src];
        cnt[src] = 0; slot[src] = -1;
        src++;
      } else {
        trg++;
        if (trg == src) src++;
      }
    }
    int shake_molecules = nmol > 0 ? trg + 1 : 0;
    for (int m = 0; m < shake_molecules; m++) order.push_back(cnt[m] ? slot[m] : -1);
  }
  s.sh_first.clear(); s.sh_n.clear(); s.sh_i.clear(); s.sh_j.clear(); s.sh_d2.clear();
  for (int m : order) {
    s.sh_first.push_back((int)s.sh_i.size());
    int n = m < 0 ? 0 : (int)mi[m].size();
    s.sh_n.push_back(n);
    for (int c = 0; c < n; c++) { s.sh_i.push_back(mi[m][c]); s.sh_j.push_back(mj[m][c]); s.sh_d2.push_back(md2[m][c]); }
  }
  s.shake_constraints = (int)s.sh_i.size();
  s.Ndegf = 3 * N - s.shake_constraints;
  s.Ndegfree = (int)((double)(s.Ndegf - 3 * t.nexats) + exclshk);
  s.Ndegf_solvent = s.Ndegf - 3 * NS + solute_shake;
  s.Ndegf_solute = s.Ndegf - s.Ndegf_solvent;
  s.Ndegfree_solvent = 3 * (N - NS) - (s.shake_constraints - solute_shake);
  s.Ndegfree_solute = s.Ndegfree - s.Ndegfree_solvent;
  bool sep = in.separate_scaling;
  if ((long long)s.Ndegfree_solvent * s.Ndegfree_solute == 0) { s.detail_temps = false; sep = false; }
  else s.detail_temps = true;
  in.separate_scaling = sep;
  // angles whose end atoms are constrained are dropped (md.f90:2490-2502)
  for (size_t c = 0; c < s.sh_i.size(); c++) {
    int ia = s.sh_i[c], ja = s.sh_j[c];
    for (auto &a : t.ang)
      if ((a.i == ia && a.k == ja) || (a.i == ja && a.k == ia)) { a.cod = 0; break; }
  }

  // ------------------------------------------------------ make_nbqqlist()
  s.qconn.assign((size_t)S * NS * nq, 9);
  auto QC = [&](int st, int i, int iq) -> signed char & { return s.qconn[((size_t)st * NS + i) * nq + iq]; };
  if (nq > 0) {
    for (int iq = 0; iq < nq; iq++)
      for (int st = 0; st < S; st++) QC(st, f.iqseq[iq], iq) = 1;
    // find_bonded (md.f90:7352): depth-limited walk over solute and Q bonds
    struct Walk {
      System &s; int S, NS, nq;
      signed char &qc(int st, int i, int iq) { return s.qconn[((size_t)st * NS + i) * nq + iq]; }
      void go(int iq, int cur, int level, int st) {
        auto &t = s.top;
        for (int b = 0; b < t.nbonds_solute; b++) {
          auto &bd = t.bnd[b];
          if (bd.cod == 0) continue;
          int nc = -1;
          if (bd.i == cur) nc = bd.j;
          else if (bd.j == cur) nc = bd.i;
          if (nc < 0) continue;
          int nl = level + 1;
          if (qc(st, nc, iq) > nl) { qc(st, nc, iq) = (signed char)nl; if (nl < 4) go(iq, nc, nl, st); }
        }
        for (auto &q : s.fep.qbnd) {
          if (q.cod[st] <= 0) continue;
          int nc = -1;
          if (q.i == cur) nc = q.j;
          else if (q.j == cur) nc = q.i;
          if (nc < 0) continue;
          int nl = level + 1;
          if (qc(st, nc, iq) > nl) { qc(st, nc, iq) = (signed char)nl; if (nl < 4) go(iq, nc, nl, st); }
        }
      }
    } walk{s, S, NS, nq};
    for (int iq = 0; iq < nq; iq++)
      for (int st = 0; st < S; st++) walk.go(iq, f.iqseq[iq], 1, st);
    for (auto &e : f.exspec) {
      int iq = s.iqatom[e.i];
      if (iq >= 0 && e.j < NS)
        for (int st = 0; st < S; st++) if (e.flag[st]) QC(st, e.j, iq) = 0;
      iq = s.iqatom[e.j];
      if (iq >= 0 && e.i < NS)
        for (int st = 0; st < S; st++) if (e.flag[st]) QC(st, e.i, iq) = 0;
    }
  }
  // nbqqlist (md.f90:7449)
  {
    std::vector<std::vector<int>> L_iq(S), L_j(S), L_jq(S), L_lj(S);
    std::vector<std::vector<double>> L_el(S);
    for (int iq = 0; iq < nq - 1; iq++)
      for (int jq = iq + 1; jq < nq; jq++) {
        int j = f.iqseq[jq];
        for (int st = 0; st < S; st++) {
          if (QC(st, j, iq) <= 3) continue;
          int lj;
          if (QC(st, j, iq) == 4) lj = 3;
          else if (!f.qvdw_flag) lj = s.ljcod[(size_t)t.iac[f.iqseq[iq]] * t.natyps + t.iac[j]];
          else {
            lj = 1;
            for (auto &p : f.soft_pairs)
              if ((iq == p.first && jq == p.second) || (jq == p.first && iq == p.second)) { lj = 2; break; }
          }
          double el = 1.0;
          for (auto &e : f.el_scale)
            if ((iq == e.iq && jq == e.jq) || (iq == e.jq && jq == e.iq)) { el = e.s[st]; break; }
          L_iq[st].push_back(iq); L_j[st].push_back(j); L_jq[st].push_back(jq); L_lj[st].push_back(lj); L_el[st].push_back(el);
        }
      }
    for (int j = 0; j < NS; j++) {
      if (s.iqatom[j] >= 0) continue;
      bool near = false;
      for (int st = 0; st < S && !near; st++)
        for (int iq = 0; iq < nq; iq++) if (QC(st, j, iq) <= 3) { near = true; break; }
      if (!near) continue;
      for (int iq = 0; iq < nq; iq++)
        for (int st = 0; st < S; st++) {
          if (QC(st, j, iq) < 4) continue;
          int lj;
          if (QC(st, j, iq) == 4) lj = 3;
          else if (f.qvdw_flag) lj = 1;
          else lj = s.ljcod[(size_t)t.iac[f.iqseq[iq]] * t.natyps + t.iac[j]];
          L_iq[st].push_back(iq); L_j[st].push_back(j); L_jq[st].push_back(-1); L_lj[st].push_back(lj); L_el[st].push_back(1.0);
        }
    }
    s.nbqq_count.assign(S, 0); s.nbqq_off.assign(S, 0);
    s.nbqq_iq.clear(); s.nbqq_j.clear(); s.nbqq_jq.clear(); s.nbqq_ljcod.clear(); s.nbqq_el_scale.clear();
    for (int st = 0; st < S; st++) {
      s.nbqq_off[st] = (int)s.nbqq_iq.size();
      s.nbqq_count[st] = (int)L_iq[st].size();
      s.nbqq_iq.insert(s.nbqq_iq.end(), L_iq[st].begin(), L_iq[st].end());
      s.nbqq_j.insert(s.nbqq_j.end(), L_j[st].begin(), L_j[st].end());
      s.nbqq_jq.insert(s.nbqq_jq.end(), L_jq[st].begin(), L_jq[st].end());
      s.nbqq_ljcod.insert(s.nbqq_ljcod.end(), L_lj[st].begin(), L_lj[st].end());
      s.nbqq_el_scale.insert(s.nbqq_el_scale.end(), L_el[st].begin(), L_el[st].end());
    }
  }

  // ----------------------------------------------------- shrink_topology()
  {
    auto shrink = [&](auto &vec, int &nsol, auto drop) {
      int n = (int)vec.size();
      int i = 0;
      while (i < n) {
        if (drop(vec[i])) {
          if (i < nsol) { vec[i] = vec[nsol - 1]; vec[nsol - 1] = vec[n - 1]; nsol--; }
          else vec[i] = vec[n - 1];
          n--;
          continue;
        }
        i++;
      }
      vec.resize(n);
    };
    shrink(t.bnd, t.nbonds_solute, [](const Topology::Bond &b) { return b.cod <= 0; });
    shrink(t.ang, t.nangles_solute, [](const Topology::Angle &a) { return a.cod == 0; });
    bool xb = in.exclude_bonded;
    shrink(t.tor, t.ntors_solute, [&](const Topology::Tors &q) {
      return (xb && t.excl[q.i] && t.excl[q.j] && t.excl[q.k] && t.excl[q.l]) || q.cod == 0;
    });
    shrink(t.imp, t.nimps_solute, [&](const Topology::Tors &q) {
      return (xb && t.excl[q.i] && t.excl[q.j] && t.excl[q.k] && t.excl[q.l]) || q.cod == 0;
    });
  }
  // resolve parameters per term
  s.bi.clear(); s.bj.clear(); s.bfk.clear(); s.bb0.clear();
  for (auto &b : t.bnd) { s.bi.push_back(b.i); s.bj.push_back(b.j); s.bfk.push_back(t.bond_fk[b.cod - 1]); s.bb0.push_back(t.bond_b0[b.cod - 1]); }
  s.nb_solute = t.nbonds_solute;
  s.ai.clear(); s.aj.clear(); s.ak.clear(); s.afk.clear(); s.ath0.clear(); s.aufk.clear(); s.aur0.clear();
  // Urey-Bradley terms act only under the CHARMM force field (md.f90:13498-13504)
  const bool ub = t.ff_type == 3;
  for (auto &a : t.ang) {
    s.ai.push_back(a.i); s.aj.push_back(a.j); s.ak.push_back(a.k);
    s.afk.push_back(t.ang_fk[a.cod - 1]); s.ath0.push_back(t.ang_th0[a.cod - 1]);
    s.aufk.push_back(ub ? t.ang_ureyfk[a.cod - 1] : 0.0); s.aur0.push_back(ub ? t.ang_ureyr0[a.cod - 1] : 0.0);
  }
  s.na_solute = t.nangles_solute;
  s.ti.clear(); s.tj.clear(); s.tk.clear(); s.tl.clear(); s.tfk.clear(); s.trm.clear(); s.tdel.clear(); s.tpaths.clear();
  for (auto &q : t.tor) {
    s.ti.push_back(q.i); s.tj.push_back(q.j); s.tk.push_back(q.k); s.tl.push_back(q.l);
    s.tfk.push_back(t.tor_fk[q.cod - 1]); s.trm.push_back(t.tor_rmult[q.cod - 1]);
    s.tdel.push_back(t.tor_deltor[q.cod - 1]); s.tpaths.push_back(t.tor_paths[q.cod - 1]);
  }
  s.nt_solute = t.ntors_solute;
  s.ii.clear(); s.ij.clear(); s.ik.clear(); s.il.clear(); s.ifk.clear(); s.iimp0.clear();
  for (auto &q : t.imp) {
    s.ii.push_back(q.i); s.ij.push_back(q.j); s.ik.push_back(q.k); s.il.push_back(q.l);
    s.ifk.push_back(t.imp_fk[q.cod - 1]); s.iimp0.push_back(t.imp_imp0[q.cod - 1]);
  }
  s.ni_solute = t.nimps_solute;
  // Q bonded terms, parameters per state
  auto qflat = [&](auto &list, auto on_of, auto set_params) {
    for (size_t k = 0; k < list.size(); k++)
      for (int st = 0; st < S; st++) on_of(k, st, list[k].cod[st]), set_params(k, st, list[k].cod[st]);
  };
  (void)qflat;
  s.qbnd_i.clear(); s.qbnd_j.clear();
  for (auto &q : f.qbnd) { s.qbnd_i.push_back(q.i); s.qbnd_j.push_back(q.j); }
  size_t nqb = f.qbnd.size();
  s.qbnd_on.assign(nqb * S, 0); s.qbnd_Dmz.assign(nqb * S, 0); s.qbnd_amz.assign(nqb * S, 0);
  s.qbnd_r0.assign(nqb * S, 0); s.qbnd_fk.assign(nqb * S, 0);
  for (size_t k = 0; k < nqb; k++)
    for (int st = 0; st < S; st++) {
      int c = f.qbnd[k].cod[st];
      if (c > 0) {
        auto &L = f.qbondlib[c - 1];
        s.qbnd_on[k * S + st] = 1; s.qbnd_Dmz[k * S + st] = L.Dmz; s.qbnd_amz[k * S + st] = L.amz;
        s.qbnd_r0[k * S + st] = L.r0; s.qbnd_fk[k * S + st] = L.fk;
      }
    }
  s.qang_i.clear(); s.qang_j.clear(); s.qang_k.clear();
  for (auto &q : f.qang) { s.qang_i.push_back(q.i); s.qang_j.push_back(q.j); s.qang_k.push_back(q.k); }
  size_t nqa = f.qang.size();
  s.qang_on.assign(nqa * S, 0); s.qang_fk.assign(nqa * S, 0); s.qang_th0.assign(nqa * S, 0);
  s.qang_ureyfk.assign(nqa * S, 0); s.qang_ureyr0.assign(nqa * S, 0);
  for (size_t k = 0; k < nqa; k++)
    for (int st = 0; st < S; st++) {
      int c = f.qang[k].cod[st];
      if (c > 0) {
        auto &L = f.qanglib[c - 1];
        s.qang_on[k * S + st] = 1; s.qang_fk[k * S + st] = L.fk; s.qang_th0[k * S + st] = L.ang0;
        if (ub) { s.qang_ureyfk[k * S + st] = L.ureyfk; s.qang_ureyr0[k * S + st] = L.ureyr0; }
      }
    }
  auto flat4 = [&](std::vector<Fep::QTor> &L, std::vector<int> &I, std::vector<int> &J, std::vector<int> &K,
                   std::vector<int> &Lx, std::vector<unsigned char> &on) {
    I.clear(); J.clear(); K.clear(); Lx.clear();
    for (auto &q : L) { I.push_back(q.i); J.push_back(q.j); K.push_back(q.k); Lx.push_back(q.l); }
    on.assign(L.size() * S, 0);
  };
  flat4(f.qtor, s.qtor_i, s.qtor_j, s.qtor_k, s.qtor_l, s.qtor_on);
  s.qtor_fk.assign(f.qtor.size() * S, 0); s.qtor_rmult.assign(f.qtor.size() * S, 0); s.qtor_deltor.assign(f.qtor.size() * S, 0);
  for (size_t k = 0; k < f.qtor.size(); k++)
    for (int st = 0; st < S; st++) {
      int c = f.qtor[k].cod[st];
      if (c > 0) {
        s.qtor_on[k * S + st] = 1; s.qtor_fk[k * S + st] = f.qfktor[c - 1];
        s.qtor_rmult[k * S + st] = f.qrmult[c - 1]; s.qtor_deltor[k * S + st] = f.qdeltor[c - 1];
      }
    }
  flat4(f.qimp, s.qimp_i, s.qimp_j, s.qimp_k, s.qimp_l, s.qimp_on);
  s.qimp_fk.assign(f.qimp.size() * S, 0); s.qimp_imp0.assign(f.qimp.size() * S, 0);
  for (size_t k = 0; k < f.qimp.size(); k++)
    for (int st = 0; st < S; st++) {
      int c = f.qimp[k].cod[st];
      if (c > 0) { s.qimp_on[k * S + st] = 1; s.qimp_fk[k * S + st] = f.qfkimp[c - 1]; s.qimp_imp0[k * S + st] = f.qimp0[c - 1]; }
    }
  s.offd_i.clear(); s.offd_j.clear(); s.offd_k.clear(); s.offd_l.clear(); s.offd_A.clear(); s.offd_mu.clear();
  for (auto &o : f.offd) {
    s.offd_i.push_back(o.i); s.offd_j.push_back(o.j); s.offd_k.push_back(o.k); s.offd_l.push_back(o.l);
    s.offd_A.push_back(o.A); s.offd_mu.push_back(o.mu);
  }
  // Morse couplings (md.f90:13910-13925, 14008-14018, 14135-14145, 14280-14290).
  // qangle takes an angle's first coupling, qurey_bradley, qtorsion and
  // qimproper its last.  In state st, EMorseD(ib) holds what qbond computed in
  // the latest state <= st that has the bond; a coupled term present in a
  // state before any such state would read a previous step's value.
  auto resolve = [&](const std::vector<Fep::Coupling> &cpl, size_t nterm, const std::vector<int> &cod_of_term,
                     bool first, std::vector<int> &bond, std::vector<int> *flag, std::vector<int> &src,
                     const char *what) {
    bond.assign(nterm, -1);
    if (flag) flag->assign(nterm, 0);
    src.assign(nterm * S, -1);
    for (auto &c : cpl) {
      if (first && bond[c.term] >= 0) continue;
      bond[c.term] = c.bond;
      if (flag) (*flag)[c.term] = c.flag;
    }
    for (size_t t = 0; t < nterm; t++) {
      if (bond[t] < 0) continue;
      int last = -1;
      for (int st = 0; st < S; st++) {
        if (f.qbnd[bond[t]].cod[st] > 0) last = st;
        if (cod_of_term[t * S + st] > 0) {
          if (last < 0)
            fail(QB_ERR_UNSUPPORTED, std::string("coupled Q ") + what + " " + std::to_string(t + 1) +
                                         " is present in a state before its Morse bond is (EMorseD from a previous step)");
          src[t * S + st] = last;
        }
      }
    }
  };
  {
    std::vector<int> ca(f.qang.size() * S), ct(f.qtor.size() * S), ci(f.qimp.size() * S);
    for (size_t k = 0; k < f.qang.size(); k++) for (int st = 0; st < S; st++) ca[k * S + st] = f.qang[k].cod[st];
    for (size_t k = 0; k < f.qtor.size(); k++) for (int st = 0; st < S; st++) ct[k * S + st] = f.qtor[k].cod[st];
    for (size_t k = 0; k < f.qimp.size(); k++) for (int st = 0; st < S; st++) ci[k * S + st] = f.qimp[k].cod[st];
    resolve(f.ang_coupl, f.qang.size(), ca, true, s.qang_cpl, nullptr, s.qang_cpl_src, "angle");
    resolve(f.ang_coupl, f.qang.size(), ca, false, s.qang_cpl_ub, nullptr, s.qang_cpl_ub_src, "angle");
    resolve(f.tor_coupl, f.qtor.size(), ct, false, s.qtor_cpl, nullptr, s.qtor_cpl_src, "torsion");
    resolve(f.imp_coupl, f.qimp.size(), ci, false, s.qimp_cpl, &s.qimp_cpl_flag, s.qimp_cpl_src, "improper");
  }

  // water parameters used by the SPC kernels (md.f90:11834-11841, 11320-11325)
  if (s.nwat > 0) {
    s.iac_ow = t.iac[NS];
    s.iac_hw = t.iac[NS + 1];
    int lj = s.ljcod[(size_t)s.iac_ow * t.natyps + s.iac_ow] - 1;
    const auto &O = t.iaclib[s.iac_ow];
    lj_pair(t.ivdw_rule == 2, O.avdw[lj], O.avdw[lj], O.bvdw[lj], O.bvdw[lj], s.A_OO, s.B_OO);
    // The arithmetic rule's water routines (nonbon2_ww, nonbon2_qw) and the
    // geometric 3-atom solvent's (nonbond_3atomsolvent, nonbond_qw_3atom)
    // take LJ on every site pair; the SPC routines take O-O only.  Site 2 and
    // 3 are one hydrogen type here, with charge -crg_ow/2 (the value the Q-water
    // terms use, md.f90:13799-13801).
    if (t.solvent_type == 1 && (t.iac[NS + 1] != t.iac[NS + 2] || t.crg[NS + 1] != t.crg[NS + 2] ||
                                t.crg[NS + 1] != -t.crg[NS] / 2.0f))
      fail(QB_ERR_UNSUPPORTED, "3-atom solvent whose two light sites differ or are not -1/2 the first site's charge");
    const auto &H = t.iaclib[s.iac_hw];
    bool h_lj = H.bvdw[0] != 0.0 || H.bvdw[1] != 0.0;
    s.ww_hlj = (t.ivdw_rule == 2 || t.solvent_type == 1) && h_lj;
    if (s.ww_hlj) {
      int loh = s.ljcod[(size_t)s.iac_ow * t.natyps + s.iac_hw] - 1;
      int lhh = s.ljcod[(size_t)s.iac_hw * t.natyps + s.iac_hw] - 1;
      lj_pair(t.ivdw_rule == 2, O.avdw[loh], H.avdw[loh], O.bvdw[loh], H.bvdw[loh], s.A_OH, s.B_OH);
      lj_pair(t.ivdw_rule == 2, H.avdw[lhh], H.avdw[lhh], H.bvdw[lhh], H.bvdw[lhh], s.A_HH, s.B_HH);
    }
  }
  s.type_mass.resize(t.natyps); s.type_avdw.resize(3 * (size_t)t.natyps); s.type_bvdw.resize(3 * (size_t)t.natyps);
  for (int i = 0; i < t.natyps; i++) {
    s.type_mass[i] = t.iaclib[i].mass;
    for (int k = 0; k < 3; k++) { s.type_avdw[3 * i + k] = t.iaclib[i].avdw[k]; s.type_bvdw[3 * i + k] = t.iaclib[i].bvdw[k]; }
  }
  s.heavy_u8 = t.heavy;
  // restraint arrays
  for (auto &r : in.rseq) { s.rseq_i.push_back(r.i); s.rseq_j.push_back(r.j); s.rseq_fk.push_back(r.fk); s.rseq_ih.push_back(r.ih); s.rseq_tc.push_back(r.to_center); }
  for (auto &r : in.rpos) { s.rpos_i.push_back(r.i); s.rpos_ipsi.push_back(r.ipsi); for (int k = 0; k < 3; k++) { s.rpos_x.push_back(r.x[k]); s.rpos_fk.push_back(r.fk[k]); } }
  for (auto &r : in.rdis) { s.rdis_i.push_back(r.i); s.rdis_j.push_back(r.j); s.rdis_ipsi.push_back(r.ipsi); s.rdis_d1.push_back(r.d1); s.rdis_d2.push_back(r.d2); s.rdis_fk.push_back(r.fk); }
  for (auto &r : in.rang) { s.rang_i.push_back(r.i); s.rang_j.push_back(r.j); s.rang_k.push_back(r.k); s.rang_ipsi.push_back(r.ipsi); s.rang_ang.push_back(r.ang); s.rang_fk.push_back(r.fk); }
  for (auto &r : in.rwal) { s.rwal_i.push_back(r.i); s.rwal_j.push_back(r.j); s.rwal_ih.push_back(r.ih); s.rwal_d.push_back(r.d); s.rwal_fk.push_back(r.fk); s.rwal_a.push_back(r.aMorse); s.rwal_dm.push_back(r.dMorse); }
  for (auto &r : in.rseq) if (r.i < 0 || r.j >= N || r.i > r.j) fail(QB_ERR_PARSE, "sequence restraint atoms out of range");
  for (auto &r : in.rpos) if (r.i < 0 || r.i >= N || r.ipsi < 0 || r.ipsi > S) fail(QB_ERR_PARSE, "atom restraint out of range");
  for (auto &r : in.rdis) if (r.i < 0 || r.i >= N || r.j < 0 || r.j >= N || r.ipsi < 0 || r.ipsi > S) fail(QB_ERR_PARSE, "distance restraint out of range");
  for (auto &r : in.rang) if (r.i < 0 || r.k >= N || r.ipsi < 0 || r.ipsi > S) fail(QB_ERR_PARSE, "angle restraint out of range");
  for (auto &r : in.rwal) if (r.i < 0 || r.j >= N) fail(QB_ERR_PARSE, "wall restraint out of range");

  // ------------------------------------------------------- coordinates/velocities
  if (in.restart) {
    std::vector<float> tc = s.ws_theta_corr;
    // a periodic box's restart holds its edge lengths and centre after the
    // velocities (md.f90:13670-13676)
    read_restart(in.restart_file, N, s.x, s.v, s.nwpolr_shell, &tc, t.use_pbc ? s.boxl : nullptr,
                 t.use_pbc ? s.boxc : nullptr);
    s.ws_theta_corr = tc;
  }
  if (t.use_pbc) {
    // molecule masses (md.f90:13861-13882): 1/sum of the type masses, and the
    // per-atom mass as 1/winv in single precision
    s.mol_minv.assign(t.nmol, 0.0);
    for (int m = 0; m < t.nmol; m++) {
      double tot = 0.0;
      for (int j = t.istart_mol[m]; j < t.istart_mol[m + 1]; j++) tot += t.iaclib[t.iac[j]].mass;
      s.mol_minv[m] = 1. / tot;
    }
    s.mass_box.resize(N);
    for (int i = 0; i < N; i++) s.mass_box[i] = (double)(1.0f / s.winv[i]);
    // control_box (md.f90:13852-13858): a new box size, molecules put back
    if (in.control_box) {
      for (int k = 0; k < 3; k++) s.boxl[k] = in.new_boxl[k];
      if (in.put_solute_back_in_box || in.put_solvent_back_in_box) put_back_in_box(s);
    }
  }
  s.randm_started = 0;
  s.randm_state = 0;
  if (in.iseed > 0) {
    // maxwell (md.f90:3787) with gauss (1453) on randm (14408)
    Randm rng;
    int ig = in.iseed;
    double kT = (double)kBoltz * in.Tmaxw;
    for (int i = 0; i < N; i++) {
      double sd = std::sqrt(kT / s.mass[i]);
      for (int k = 0; k < 3; k++) {
        double a = 0.0;
        for (int r = 0; r < 12; r++) a += rng.next(ig);
        s.v[3 * i + k] = (a - 6.0) * sd + 0.0;
      }
    }
    // randm keeps one sequence per run: the volume moves continue it
    s.randm_started = 1;
    s.randm_state = rng.irand;
    s.log += "maxwell velocities generated\n";
    // initial_shaking (md.f90:2506)
    std::vector<double> xx = s.x;
    host_shake(s, xx, s.x);
    xx.resize(s.x.size());
    for (size_t k = 0; k < xx.size(); k++) xx[k] = s.x[k] - in.dt * s.v[k];
    host_shake(s, s.x, xx);
    for (size_t k = 0; k < xx.size(); k++) s.v[k] = (s.x[k] - xx[k]) / in.dt;
    // stop_cm_translation (md.f90:14670)
    double tot = 0, vcm[3] = {0, 0, 0};
    for (int i = 0; i < N; i++) {
      tot += s.mass[i];
      for (int k = 0; k < 3; k++) vcm[k] += s.mass[i] * s.v[3 * i + k];
    }
    for (int k = 0; k < 3; k++) vcm[k] /= tot;
    for (int i = 0; i < N; i++)
      for (int k = 0; k < 3; k++) s.v[3 * i + k] -= vcm[k];
  }
}

void System::fill_view(qb_sysview *v) const {
  std::memset(v, 0, sizeof *v);
  const Topology &t = top;
  v->natom = natom; v->nat_solute = t.nat_solute; v->nwat = nwat;
  v->ncgp = t.ncgp; v->ncgp_solute = t.ncgp_solute; v->natyps = t.natyps;
  v->nqat = fep.nqat; v->nstates = (int)in.lambdas.size();
  v->nbonds = (int)bi.size(); v->nbonds_solute = nb_solute;
  v->nangles = (int)ai.size(); v->nangles_solute = na_solute;
  v->ntors = (int)ti.size(); v->ntors_solute = nt_solute;
  v->nimps = (int)ii.size(); v->nimps_solute = ni_solute;
  v->nmol = t.nmol;
  v->ff_type = t.ff_type; v->ivdw_rule = t.ivdw_rule; v->solvent_type = t.solvent_type;
  v->iuse_switch_atom = t.iuse_switch_atom;
  v->el14_scale = t.el14_scale; v->coulomb_constant = t.coulomb_constant;
  v->nsteps = in.nsteps; v->NBcycle = in.NBcycle; v->iout_cycle = in.iout_cycle; v->iene_cycle = in.iene_cycle;
  v->itemp_cycle = in.itemp_cycle; v->itrj_cycle = in.itrj_cycle;
  v->stepsize_fs = in.stepsize; v->dt = in.dt; v->Temp0 = in.Temp0; v->tau_T = in.tau_T; v->Tmaxw = in.Tmaxw;
  v->iseed = in.iseed; v->separate_scaling = in.separate_scaling;
  v->shake_solvent = in.shake_solvent; v->shake_solute = in.shake_solute; v->shake_hydrogens = in.shake_hydrogens;
  v->use_LRF = in.use_LRF; v->force_rms = in.force_rms;
  v->Rcpp = in.Rcpp; v->Rcww = in.Rcww; v->Rcpw = in.Rcpw; v->Rcq = in.Rcq; v->RcLRF = in.RcLRF;
  for (int k = 0; k < 3; k++) { v->xpcent[k] = t.xpcent[k]; v->xwcent[k] = t.xwcent[k]; }
  v->rexcl_o = t.rexcl_o; v->rexcl_i = in.rexcl_i; v->rwat = rwat;
  v->fk_pshell = in.fk_pshell; v->fk_fix = 200.0;
  v->fk_wsphere = fk_wsphere; v->Dwmz = Dwmz; v->awmz = awmz; v->fkwpol = fkwpol;
  v->wpol_restr = in.wpol_restr && nwat > 0; v->wpol_born = in.wpol_born;
  v->nexats = t.nexats; v->nexwat = t.nexwat; v->nshellats = nshellats;
  v->xtop = t.xtop.data(); v->x0 = x.data(); v->v0 = this->v.data();
  v->iac = t.iac.data(); v->crg = t.crg.data(); v->winv = winv.data(); v->mass = mass.data();
  v->heavy = heavy_u8.data(); v->excl = t.excl.data(); v->shell = shell.data();
  v->iqatom = iqatom.data(); v->iwhich_cgp = iwhich_cgp.data();
  v->type_mass = type_mass.data(); v->type_avdw = type_avdw.data(); v->type_bvdw = type_bvdw.data();
  v->ljcod = ljcod.data();
  v->listex_bits = t.listex.data(); v->list14_bits = t.list14.data();
  v->nexlong = (int)t.listexlong.size(); v->n14long = (int)t.list14long.size();
  v->listexlong = t.listexlong.empty() ? nullptr : &t.listexlong[0].first;
  v->list14long = t.list14long.empty() ? nullptr : &t.list14long[0].first;
  v->cgp_iswitch = t.cgp_iswitch.data(); v->cgp_first = t.cgp_first.data(); v->cgp_last = t.cgp_last.data();
  v->cgpatom = t.cgpatom.data();
  v->istart_mol = t.istart_mol.data();
  v->bnd_i = bi.data(); v->bnd_j = bj.data(); v->bnd_fk = bfk.data(); v->bnd_b0 = bb0.data();
  v->ang_i = ai.data(); v->ang_j = aj.data(); v->ang_k = ak.data(); v->ang_fk = afk.data(); v->ang_th0 = ath0.data();
  v->ang_ureyfk = aufk.data(); v->ang_ureyr0 = aur0.data();
  v->tor_i = ti.data(); v->tor_j = tj.data(); v->tor_k = tk.data(); v->tor_l = tl.data();
  v->tor_fk = tfk.data(); v->tor_rmult = trm.data(); v->tor_deltor = tdel.data(); v->tor_paths = tpaths.data();
  v->imp_i = ii.data(); v->imp_j = ij.data(); v->imp_k = ik.data(); v->imp_l = il.data();
  v->imp_fk = ifk.data(); v->imp_imp0 = iimp0.data();
  v->crg_ow = crg_ow; v->crg_hw = crg_hw; v->A_OO = A_OO; v->B_OO = B_OO;
  v->ww_hlj = ww_hlj; v->A_OH = A_OH; v->B_OH = B_OH; v->A_HH = A_HH; v->B_HH = B_HH;
  v->iac_ow = iac_ow; v->iac_hw = iac_hw;
  v->nwpolr_shell = (in.wpol_restr && nwat > 0) ? nwpolr_shell : 0;
  v->wshell_rout = ws_rout.data(); v->wshell_dr = ws_dr.data(); v->wshell_cstb = ws_cstb.data();
  v->wshell_theta_corr0 = ws_theta_corr.data();
  v->lambda = in.lambdas.data();
  v->iqseq = fep.iqseq.data(); v->qcrg = qcrg_scaled.data();
  v->qvdw_flag = fep.qvdw_flag; v->nqlib = fep.nqlib; v->qq_use_library_charges = fep.qq_use_library_charges;
  v->qiac = fep.qiac.data(); v->qavdw = fep.qavdw.data(); v->qbvdw = fep.qbvdw.data();
  v->sc_lookup = fep.sc_lookup.data(); v->qconn = qconn.data();
  v->nbqq_count = nbqq_count.data(); v->nbqq_off = nbqq_off.data();
  v->nbqq_iq = nbqq_iq.data(); v->nbqq_j = nbqq_j.data(); v->nbqq_jq = nbqq_jq.data();
  v->nbqq_ljcod = nbqq_ljcod.data(); v->nbqq_el_scale = nbqq_el_scale.data();
  v->nqbond = (int)qbnd_i.size(); v->nqangle = (int)qang_i.size(); v->nqtor = (int)qtor_i.size(); v->nqimp = (int)qimp_i.size();
  v->qbnd_i = qbnd_i.data(); v->qbnd_j = qbnd_j.data(); v->qbnd_on = qbnd_on.data();
  v->qbnd_Dmz = qbnd_Dmz.data(); v->qbnd_amz = qbnd_amz.data(); v->qbnd_r0 = qbnd_r0.data(); v->qbnd_fk = qbnd_fk.data();
  v->qang_i = qang_i.data(); v->qang_j = qang_j.data(); v->qang_k = qang_k.data(); v->qang_on = qang_on.data();
  v->qang_fk = qang_fk.data(); v->qang_th0 = qang_th0.data();
  v->qang_ureyfk = qang_ureyfk.data(); v->qang_ureyr0 = qang_ureyr0.data();
  v->qtor_i = qtor_i.data(); v->qtor_j = qtor_j.data(); v->qtor_k = qtor_k.data(); v->qtor_l = qtor_l.data();
  v->qtor_on = qtor_on.data(); v->qtor_fk = qtor_fk.data(); v->qtor_rmult = qtor_rmult.data(); v->qtor_deltor = qtor_deltor.data();
  v->qimp_i = qimp_i.data(); v->qimp_j = qimp_j.data(); v->qimp_k = qimp_k.data(); v->qimp_l = qimp_l.data();
  v->qimp_on = qimp_on.data(); v->qimp_fk = qimp_fk.data(); v->qimp_imp0 = qimp_imp0.data();
  v->noffd = (int)offd_i.size();
  v->offd_i = offd_i.data(); v->offd_j = offd_j.data(); v->offd_k = offd_k.data(); v->offd_l = offd_l.data();
  v->offd_A = offd_A.data(); v->offd_mu = offd_mu.data();
  v->qang_cpl = qang_cpl.data(); v->qang_cpl_ub = qang_cpl_ub.data(); v->qtor_cpl = qtor_cpl.data();
  v->qimp_cpl = qimp_cpl.data(); v->qimp_cpl_flag = qimp_cpl_flag.data();
  v->qang_cpl_src = qang_cpl_src.data(); v->qang_cpl_ub_src = qang_cpl_ub_src.data();
  v->qtor_cpl_src = qtor_cpl_src.data(); v->qimp_cpl_src = qimp_cpl_src.data();
  v->shake_molecules = (int)sh_first.size(); v->shake_constraints = shake_constraints;
  v->shake_mol_first = sh_first.data(); v->shake_mol_n = sh_n.data();
  v->shake_i = sh_i.data(); v->shake_j = sh_j.data(); v->shake_dist2 = sh_d2.data();
  v->nrstr_seq = (int)rseq_i.size(); v->nrstr_pos = (int)rpos_i.size(); v->nrstr_dist = (int)rdis_i.size();
  v->nrstr_angl = (int)rang_i.size(); v->nrstr_wall = (int)rwal_i.size();
  v->rseq_i = rseq_i.data(); v->rseq_j = rseq_j.data(); v->rseq_ih = rseq_ih.data(); v->rseq_to_center = rseq_tc.data(); v->rseq_fk = rseq_fk.data();
  v->rpos_i = rpos_i.data(); v->rpos_ipsi = rpos_ipsi.data(); v->rpos_x = rpos_x.data(); v->rpos_fk = rpos_fk.data();
  v->rdis_i = rdis_i.data(); v->rdis_j = rdis_j.data(); v->rdis_ipsi = rdis_ipsi.data();
  v->rdis_d1 = rdis_d1.data(); v->rdis_d2 = rdis_d2.data(); v->rdis_fk = rdis_fk.data();
  v->rang_i = rang_i.data(); v->rang_j = rang_j.data(); v->rang_k = rang_k.data(); v->rang_ipsi = rang_ipsi.data();
  v->rang_ang = rang_ang.data(); v->rang_fk = rang_fk.data();
  v->rwal_i = rwal_i.data(); v->rwal_j = rwal_j.data(); v->rwal_ih = rwal_ih.data(); v->rwal_d = rwal_d.data();
  v->rwal_fk = rwal_fk.data(); v->rwal_aMorse = rwal_a.data(); v->rwal_dMorse = rwal_dm.data();
  v->Ndegf = Ndegf; v->Ndegfree = Ndegfree; v->Ndegf_solute = Ndegf_solute; v->Ndegf_solvent = Ndegf_solvent;
  v->Ndegfree_solute = Ndegfree_solute; v->Ndegfree_solvent = Ndegfree_solvent; v->detail_temps = detail_temps;
  v->use_pbc = t.use_pbc;
  if (t.use_pbc) {
    v->rigid_box_center = in.rigid_box_center;
    v->put_solute_back_in_box = in.put_solute_back_in_box;
    v->put_solvent_back_in_box = in.put_solvent_back_in_box;
    v->constant_pressure = in.constant_pressure;
    v->ivolume_cycle = in.ivolume_cycle;
    v->pressure_seed = in.pressure_seed;
    v->max_vol_displ = in.max_vol_displ;
    v->pressure = in.pressure;
    for (int k = 0; k < 3; k++) { v->boxlength[k] = boxl[k]; v->boxcenter[k] = boxc[k]; }
    v->mol_mass_inv = mol_minv.data();
    v->mass_box = mass_box.data();
  }
  v->qswitch = fep.qswitch;
  v->randm_started = randm_started;
  v->randm_state = randm_state;
}

}  // namespace qb
