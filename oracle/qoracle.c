/*
 * qoracle.c -- CPU oracle for the Q MD step.  TEST INFRASTRUCTURE ONLY.
 *
 * Only the test suite, the smoke check and bench.py's CPU-baseline leg use this
 * file, and only to check or to time against; the product (libqb) never calls
 * it.  It is a plain-C restatement of the sphere/SPC/geometric-rule path of
 * Q's Fortran qdyn, in FP64, keeping the single-precision roundings of the
 * reference (charge products, inverse masses, torsion/improper parameters,
 * water-shell data, Boltzmann constant).
 *
 * Each routine names the reference routine it follows (src/q6/md.f90 unless
 * stated).  Parity is pinned against the reference's own known answers:
 * test/q6/test1 (Q-surr energies of eq1 at steps 0, 50 and the final step,
 * within the 10-seed bounds of qsurr_benchmark.en) and
 * test/3.shake/p-p/benzene (eq1.log energy summaries); see tests/.
 *
 * Input is a prepared system (include/qb_system.h), i.e. the state qdyn holds
 * when md_run starts.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "qb_system.h"
#include "qoracle.h"

typedef struct { int i, j, lj; } pair_t;
typedef struct { int iq, j, lj, qlj; } qpair_t;
typedef struct { double c[3], p0, p1[3], p2[9], p3[27]; } lrf_t;

struct qo_state {
  const qb_sysview *s;
  int N, NS, nwat, S, nq;
  double *x, *v, *d, *xx;
  double E[QB_NE];
  double EQ[QB_MAX_STATES * QB_NEQ];
  /* lists */
  pair_t *pp; int npp, cpp;
  pair_t *pw; int npw, cpw;
  int *ww; int nww, cww;          /* per water: neighbours' O atoms, 0-terminated as -1 */
  qpair_t *qp; int nqp, cqp; int qp_done;
  int *qw; int nqw;
  lrf_t *lrf;
  /* thermostat */
  double Temp, Tfree, Tfree_solute, Tfree_solvent, Temp_solute, Temp_solvent;
  double Tscale_solute, Tscale_solvent;
  /* water polarisation */
  float *theta_corr, *avtheta, *avn_insh;
  int *n_insh, *list_sh, *nsort;
  double *theta, *theta0, *tdum;
  int istep;
  int status;
  /* history */
  int hcap, hcount[2];
  int *hstep[2];
  double *hE[2], *hEQ[2], *hR[2];
  double offd_r[QB_MAX_STATES];     /* r_kl of this step's off-diagonal functions */
  double ekinmax;
  double kinetic;
  /* periodic box: edge lengths, inv_boxl, centre; randm's sequence; volume moves */
  double boxl[3], iboxl[3], boxc[3];
  int rand_started, irand;
  long long vol_tries, vol_acc;
};

static const float kBoltz = 0.001986f;
static double fpi(void) { return (double)(4.0f * atanf(1.0f)); }

#define X(a, k) st->x[3 * (a) + (k)]
#define D(a, k) st->d[3 * (a) + (k)]
#define EQV(s, k) st->EQ[(s) * QB_NEQ + (k)]

static void *grow(void *p, int *cap, int need, size_t elem) {
  if (need <= *cap) return p;
  int nc = *cap ? *cap : 1024;
  while (nc < need) nc *= 2;
  p = realloc(p, (size_t)nc * elem);
  *cap = nc;
  return p;
}

/* ------------------------------------------------------------ pair lists */

static int excluded_pair(const qb_sysview *s, int i, int j) {
  int d = j - i;
  if (abs(d) <= QB_NBR_RANGE) {
    if (i < j) return (s->listex_bits[i] >> (d - 1)) & 1u;
    return (s->listex_bits[j] >> (-d - 1)) & 1u;
  }
  for (int n = 0; n < s->nexlong; n++) {
    int a = s->listexlong[2 * n], b = s->listexlong[2 * n + 1];
    if ((a == i && b == j) || (a == j && b == i)) return 1;
  }
  return 0;
}

static int is14_pair(const qb_sysview *s, int i, int j) {
  int d = j - i, r = 0;
  if (abs(d) <= QB_NBR_RANGE) {
    if (i < j) return (s->list14_bits[i] >> (d - 1)) & 1u;
    return (s->list14_bits[j] >> (-d - 1)) & 1u;
  }
  for (int n = 0; n < s->n14long; n++) {
    int a = s->list14long[2 * n], b = s->list14long[2 * n + 1];
    if ((a == i && b == j) || (a == j && b == i)) r = 1;
  }
  return r;
}

static int ljcode(const qb_sysview *s, int ti, int tj) { return s->ljcod[ti * s->natyps + tj]; }

/* all-zero pair test of nbpplist (md.f90:5495-5501) */
static int zero_pair(const qb_sysview *s, int i, int j, int lj) {
  float qq = s->crg[i] * s->crg[j];
  int ti = s->iac[i], tj = s->iac[j];
  return qq == 0.0f && s->type_avdw[3 * ti + lj - 1] * s->type_avdw[3 * tj + lj - 1] == 0.0 &&
         s->type_bvdw[3 * ti + lj - 1] * s->type_bvdw[3 * tj + lj - 1] == 0.0;
}

/* periodic box (use_PBC): boxlength * nint(d * inv_boxl), the lattice vector
 * that brings displacement d to its nearest image (md.f90:5352-5354) */
static double img(const qo_state *st, int k, double d) { return st->boxl[k] * (double)lround(d * st->iboxl[k]); }

static double dist2(qo_state *st, int a, int b) {
  double dx = X(a, 0) - X(b, 0), dy = X(a, 1) - X(b, 1), dz = X(a, 2) - X(b, 2);
  if (st->s->use_pbc) { dx -= img(st, 0, dx); dy -= img(st, 1, dy); dz -= img(st, 2, dz); }
  return dx * dx + dy * dy + dz * dz;
}

/* the switching atom of an atom's charge group */
static int sw_of(const qo_state *st, int a) { return st->s->cgp_iswitch[st->s->iwhich_cgp[a]]; }

/* image shift t[3] = L nint((x_b - x_a) / L) of the pair of reference atoms
 * (a, b); zero in the sphere */
static void pair_shift(qo_state *st, int a, int b, double t[3]) {
  for (int k = 0; k < 3; k++) t[k] = st->s->use_pbc ? img(st, k, X(b, k) - X(a, k)) : 0.0;
}

/* multipole contribution of charge q at offset dr from a group centre
 * (md.f90:5581-5636) */
static void lrf_add(lrf_t *L, double q, const double dr[3]) {
  double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
  double f0 = q / (r2 * sqrt(r2));
  L->p0 += f0 * r2;
  for (int k = 0; k < 3; k++) L->p1[k] -= f0 * dr[k];
  double f1 = 3. * f0 / r2;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      L->p2[3 * a + b] += f1 * dr[a] * dr[b];
      if (a == b) L->p2[3 * a + b] -= f0;
    }
  double f2 = -f1 / r2;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      for (int c = 0; c < 3; c++) {
        double t = 5. * dr[a] * dr[b] * dr[c];
        /* subtract r2*dr for each matching index pair (3x when a=b=c) */
        if (a == b && b == c) t -= r2 * 3. * dr[a];
        else {
          if (a == b) t -= r2 * dr[c];
          if (a == c) t -= r2 * dr[b];
          if (b == c) t -= r2 * dr[a];
        }
        L->p3[9 * a + 3 * b + c] += f2 * t;
      }
}

/* the charges of group from_group into group into's multipoles; in a box at
 * the image of from_group's switching atom nearest into's centre
 * (nbpplist_box_lrf md.f90:5842-5856) */
static void lrf_group_from_atoms(qo_state *st, int into, int from_group, int skip_q) {
  const qb_sysview *s = st->s;
  double t[3] = {0, 0, 0};
  if (s->use_pbc) {
    int sw = s->cgp_iswitch[from_group];
    for (int k = 0; k < 3; k++) t[k] = img(st, k, X(sw, k) - st->lrf[into].c[k]);
  }
  for (int a = s->cgp_first[from_group]; a <= s->cgp_last[from_group]; a++) {
    int i = s->cgpatom[a];
    if (skip_q && s->iqatom[i] >= 0) continue;
    double dr[3] = {X(i, 0) - st->lrf[into].c[0] - t[0], X(i, 1) - st->lrf[into].c[1] - t[1],
                    X(i, 2) - st->lrf[into].c[2] - t[2]};
    lrf_add(&st->lrf[into], (double)s->crg[i], dr);
  }
}

/* cgp_centers (md.f90:1000) */
static void cgp_centers(qo_state *st) {
  const qb_sysview *s = st->s;
  for (int g = 0; g < s->ncgp; g++) {
    lrf_t *L = &st->lrf[g];
    memset(L, 0, sizeof *L);
    for (int a = s->cgp_first[g]; a <= s->cgp_last[g]; a++)
      for (int k = 0; k < 3; k++) L->c[k] += X(s->cgpatom[a], k);
    double n = (double)(float)(s->cgp_last[g] - s->cgp_first[g] + 1);
    for (int k = 0; k < 3; k++) L->c[k] /= n;
  }
}

/* nbpplist / nbpplist_lrf (md.f90:5175, 5448) */
static void list_pp(qo_state *st) {
  const qb_sysview *s = st->s;
  double rc2 = s->Rcpp * s->Rcpp, rl2 = s->RcLRF * s->RcLRF;
  st->npp = 0;
  for (int ig = 0; ig < s->ncgp_solute; ig++) {
    int is = s->cgp_iswitch[ig];
    if (s->excl[is]) continue;
    for (int jg = 0; jg < s->ncgp_solute; jg++) {
      int IG = ig + 1, JG = jg + 1;
      if ((IG > JG && (IG + JG) % 2 == 0) || (IG < JG && (IG + JG) % 2 == 1)) continue;
      int js = s->cgp_iswitch[jg];
      if (s->excl[js]) continue;
      double r2;
      int inside;
      if (s->iuse_switch_atom == 1) {
        r2 = dist2(st, is, js);
        inside = r2 <= rc2;
      } else {
        /* nbpplis2_lrf (md.f90:4926-4970): inside when any atom pair is; r2
           keeps the last pair computed (the groups' last atoms when none is) */
        inside = 0;
        r2 = 0;
        for (int ia = s->cgp_first[ig]; ia <= s->cgp_last[ig] && !inside; ia++)
          for (int ja = s->cgp_first[jg]; ja <= s->cgp_last[jg]; ja++) {
            r2 = dist2(st, s->cgpatom[ia], s->cgpatom[ja]);
            if (r2 <= rc2) { inside = 1; break; }
          }
      }
      if (inside) {
        for (int ia = s->cgp_first[ig]; ia <= s->cgp_last[ig]; ia++) {
          int i = s->cgpatom[ia];
          if (s->iqatom[i] >= 0) continue;
          for (int ja = s->cgp_first[jg]; ja <= s->cgp_last[jg]; ja++) {
            int j = s->cgpatom[ja];
            if (ig == jg && i >= j) continue;
            if (s->iqatom[j] >= 0) continue;
            int lj = ljcode(s, s->iac[i], s->iac[j]);
            if (zero_pair(s, i, j, lj)) continue;
            if (excluded_pair(s, i, j)) continue;
            st->pp = grow(st->pp, &st->cpp, st->npp + 1, sizeof(pair_t));
            st->pp[st->npp].i = i;
            st->pp[st->npp].j = j;
            st->pp[st->npp].lj = is14_pair(s, i, j) ? 3 : lj;
            st->npp++;
          }
        }
      } else if (s->use_LRF && r2 <= rl2) {
        lrf_group_from_atoms(st, jg, ig, 1);
        lrf_group_from_atoms(st, ig, jg, 1);
      }
    }
  }
}

/* nbpwlist / nbpwlist_lrf (md.f90:6684, 6864) */
static void list_pw(qo_state *st) {
  const qb_sysview *s = st->s;
  double rc2 = s->Rcpw * s->Rcpw, rl2 = s->RcLRF * s->RcLRF;
  st->npw = 0;
  for (int ig = 0; ig < s->ncgp_solute; ig++) {
    int is = s->cgp_iswitch[ig];
    if (s->excl[is]) continue;
    for (int iw = 0; iw < st->nwat; iw++) {
      int o = st->NS + 3 * iw;
      if (s->excl[o]) continue;
      double r2;
      int inside;
      if (s->iuse_switch_atom == 1) {
        r2 = dist2(st, is, o);
        inside = r2 <= rc2;
      } else {
        /* nbpwlis2_lrf (md.f90:6500-6516): any atom of the group within the
           cut-off of the water O; r2 keeps the last distance computed */
        inside = 0;
        r2 = 0;
        for (int ia = s->cgp_first[ig]; ia <= s->cgp_last[ig] && !inside; ia++) {
          r2 = dist2(st, s->cgpatom[ia], o);
          if (r2 <= rc2) inside = 1;
        }
      }
      if (inside) {
        for (int ia = s->cgp_first[ig]; ia <= s->cgp_last[ig]; ia++) {
          int i = s->cgpatom[ia];
          if (s->iqatom[i] >= 0) continue;
          for (int j = o; j < o + 3; j++) {
            int lj = ljcode(s, s->iac[i], s->iac[j]);
            if (zero_pair(s, i, j, lj)) continue;
            st->pw = grow(st->pw, &st->cpw, st->npw + 1, sizeof(pair_t));
            st->pw[st->npw].i = i;
            st->pw[st->npw].j = j;
            st->pw[st->npw].lj = lj;
            st->npw++;
          }
        }
      } else if (s->use_LRF && r2 <= rl2) {
        int jg = s->iwhich_cgp[o];
        lrf_group_from_atoms(st, jg, ig, 1);
        lrf_group_from_atoms(st, ig, jg, 0);
      }
    }
  }
}

/* nbwwlist / nbwwlist_lrf (md.f90:8233, 8370) */
static void list_ww(qo_state *st) {
  const qb_sysview *s = st->s;
  double rc2 = s->Rcww * s->Rcww, rl2 = s->RcLRF * s->RcLRF;
  st->nww = 0;
  for (int iw = 0; iw < st->nwat; iw++) {
    int io = st->NS + 3 * iw;
    if (!s->excl[io]) {
      for (int jw = 0; jw < st->nwat; jw++) {
        int jo = st->NS + 3 * jw;
        if (s->excl[jo]) continue;
        int IW = iw + 1, JW = jw + 1;
        if ((IW > JW && (IW + JW) % 2 == 0) || (IW < JW && (IW + JW) % 2 == 1) || IW == JW) continue;
        double r2 = dist2(st, io, jo);
        if (r2 <= rc2) {
          st->ww = grow(st->ww, &st->cww, st->nww + 1, sizeof(int));
          st->ww[st->nww++] = jo;
        } else if (s->use_LRF && r2 <= rl2) {
          int jg = s->iwhich_cgp[jo], ig = s->iwhich_cgp[io];
          lrf_group_from_atoms(st, jg, ig, 0);
          lrf_group_from_atoms(st, ig, jg, 0);
        }
      }
    }
    st->ww = grow(st->ww, &st->cww, st->nww + 1, sizeof(int));
    st->ww[st->nww++] = -1;
  }
}

/* nbqplist (md.f90:7875): built once when Rcq exceeds the sphere */
static void list_qp(qo_state *st) {
  const qb_sysview *s = st->s;
  if (!s->use_pbc && st->qp_done && s->Rcq > s->rexcl_o) return;
  st->nqp = 0;
  if (st->nq == 0) return;
  double rc2 = s->Rcq * s->Rcq;
  for (int ig = 0; ig < s->ncgp_solute; ig++) {
    int sw = s->cgp_iswitch[ig];
    if (s->excl[sw]) continue;
    int inside = 0;
    if (s->use_pbc) {
      /* nbqplist_box (md.f90:7969): the switching atom's nearest image of the Q switching atom */
      inside = dist2(st, sw, s->qswitch) <= rc2;
    } else if (s->iuse_switch_atom == 1) {
      double r2 = 0;
      for (int k = 0; k < 3; k++) { double d = X(sw, k) - s->xpcent[k]; r2 += d * d; }
      inside = r2 <= rc2;
    } else {
      /* nbqplis2 (md.f90:7700-7716): any atom of the group within Rcq */
      for (int ia = s->cgp_first[ig]; ia <= s->cgp_last[ig] && !inside; ia++) {
        int i = s->cgpatom[ia];
        double r2 = 0;
        for (int k = 0; k < 3; k++) { double d = X(i, k) - s->xpcent[k]; r2 += d * d; }
        inside = r2 <= rc2;
      }
    }
    if (!inside) continue;
    for (int ia = s->cgp_first[ig]; ia <= s->cgp_last[ig]; ia++) {
      int i = s->cgpatom[ia];
      int near = 0;
      for (int ss = 0; ss < st->S && !near; ss++)
        for (int iq = 0; iq < st->nq; iq++)
          if (s->qconn[((size_t)ss * st->NS + i) * st->nq + iq] <= 3) { near = 1; break; }
      if (near) continue;
      for (int iq = 0; iq < st->nq; iq++) {
        st->qp = grow(st->qp, &st->cqp, st->nqp + 1, sizeof(qpair_t));
        qpair_t *p = &st->qp[st->nqp++];
        p->iq = iq;
        p->j = i;
        p->lj = ljcode(s, s->iac[i], s->iac[s->iqseq[iq]]);
        if (s->qconn[((size_t)0 * st->NS + i) * st->nq + iq] == 4) p->lj = 3;
        p->qlj = p->lj == 2 ? 1 : p->lj;
      }
    }
  }
  st->qp_done = 1;
}

/* nbqwlist (md.f90:8066) */
static void list_qw(qo_state *st) {
  const qb_sysview *s = st->s;
  if (!s->use_pbc && s->Rcq > s->rexcl_o && st->nqw > 0) return;
  st->nqw = 0;
  if (st->nq == 0) return;
  double rc2 = s->Rcq * s->Rcq;
  for (int iw = 0; iw < st->nwat; iw++) {
    int o = st->NS + 3 * iw;
    if (s->excl[o]) continue;
    double r2 = 0;
    if (s->use_pbc) {
      r2 = dist2(st, o, s->qswitch);   /* nbqwlist_box (md.f90:8123) */
    } else {
      for (int k = 0; k < 3; k++) { double d = X(o, k) - s->xpcent[k]; r2 += d * d; }
    }
    if (r2 <= rc2) st->qw[st->nqw++] = o;
  }
}

/* make_pair_lists (md.f90:3716); the box branch calls the *_box lists, which
 * are the sphere lists with nearest-image distances (dist2) */
static void make_pair_lists(qo_state *st) {
  if (st->s->use_LRF) cgp_centers(st);
  list_pp(st);
  list_pw(st);
  list_qp(st);
  list_ww(st);
  list_qw(st);
}

/* ------------------------------------------------------------- nonbonded */

static double avdw(const qb_sysview *s, int t, int lj) { return s->type_avdw[3 * t + lj - 1]; }
static double bvdw(const qb_sysview *s, int t, int lj) { return s->type_bvdw[3 * t + lj - 1]; }

/* LJ coefficients of a pair, V = A/r^12 - B/r^6.  Geometric rule
   (nonbond_*): A = a_i a_j, B = b_i b_j.  Arithmetic rule (nonbon2_*,
   md.f90:8972-9089; a = R*, b = sqrt(eps) after set-up):
   A = b_i b_j (a_i + a_j)^12, B = 2 b_i b_j (a_i + a_j)^6. */
static void ljp(const qb_sysview *s, double ai, double aj, double bi, double bj, double *A, double *B) {
  if (s->ivdw_rule != 2) {
    *A = ai * aj;
    *B = bi * bj;
    return;
  }
  double a = ai + aj;
  a = a * a;
  a = a * a * a;
  double e = bi * bj;
  *A = e * a * a;
  *B = 2.0 * e * a;
}

static void apply_pair(qo_state *st, int i, int j, double dv, const double dx[3]) {
  for (int k = 0; k < 3; k++) { D(i, k) -= dv * dx[k]; D(j, k) += dv * dx[k]; }
}

/* nonbond_pp (md.f90:10387) */
static void nonbond_pp(qo_state *st) {
  const qb_sysview *s = st->s;
  for (int p = 0; p < st->npp; p++) {
    int i = st->pp[p].i, j = st->pp[p].j, lj = st->pp[p].lj;
    double t[3];
    pair_shift(st, sw_of(st, i), sw_of(st, j), t);   /* nonbond_pp_box (md.f90:10508-10519) */
    double dx[3] = {X(j, 0) - X(i, 0) - t[0], X(j, 1) - X(i, 1) - t[1], X(j, 2) - X(i, 2) - t[2]};
    double r2 = 1. / (dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    double r = sqrt(r2), r6 = r2 * r2 * r2;
    float qq = s->crg[i] * s->crg[j];
    double Vel = (double)qq * r;
    if (lj == 3) Vel = Vel * s->el14_scale;
    int ti = s->iac[i], tj = s->iac[j];
    double Va, Vb;
    if (s->ivdw_rule == 2) {   /* nonbon2_pp (md.f90:8972) */
      double A, B;
      ljp(s, avdw(s, ti, lj), avdw(s, tj, lj), bvdw(s, ti, lj), bvdw(s, tj, lj), &A, &B);
      Va = A * r6 * r6;
      Vb = B * r6;
    } else {
      Va = r6 * r6 * avdw(s, ti, lj) * avdw(s, tj, lj);
      Vb = r6 * bvdw(s, ti, lj) * bvdw(s, tj, lj);
    }
    double dv = r2 * (-Vel - 12. * Va + 6. * Vb);
    apply_pair(st, i, j, dv, dx);
    st->E[QB_E_PP_EL] += Vel;
    st->E[QB_E_PP_VDW] += Va - Vb;
  }
}

/* nonbond_pw (md.f90:10631) */
static void nonbond_pw(qo_state *st) {
  const qb_sysview *s = st->s;
  for (int p = 0; p < st->npw; p++) {
    int i = st->pw[p].i, j = st->pw[p].j, lj = st->pw[p].lj;
    int ti = s->iac[i], tj = s->iac[j];
    double aLJ, bLJ;
    ljp(s, avdw(s, ti, lj), avdw(s, tj, lj), bvdw(s, ti, lj), bvdw(s, tj, lj), &aLJ, &bLJ);
    double t[3];
    pair_shift(st, sw_of(st, i), sw_of(st, j), t);   /* nonbond_pw_box (md.f90:10693-10699) */
    double dx[3] = {X(j, 0) - X(i, 0) - t[0], X(j, 1) - X(i, 1) - t[1], X(j, 2) - X(i, 2) - t[2]};
    double r2 = 1. / (dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    double r = sqrt(r2), r6 = r2 * r2 * r2, r12 = r6 * r6;
    float qq = s->crg[i] * s->crg[j];
    double Vel = (double)qq * r, Va = aLJ * r12, Vb = bLJ * r6;
    double dv = r2 * (-Vel - 12. * Va + 6. * Vb);
    apply_pair(st, i, j, dv, dx);
    st->E[QB_E_PW_EL] += Vel;
    st->E[QB_E_PW_VDW] += Va - Vb;
  }
}

/* nonbond_qp (md.f90:10980) and nonbond_qp_qvdw (md.f90:11138) */
static void nonbond_qp(qo_state *st) {
  const qb_sysview *s = st->s;
  int S = st->S;
  int ncol = s->natyps + st->nq;
  for (int p = 0; p < st->nqp; p++) {
    int iq = st->qp[p].iq, j = st->qp[p].j, lj = st->qp[p].lj, qlj = st->qp[p].qlj;
    int i = s->iqseq[iq];
    int tj = s->iac[j];
    double t[3] = {0, 0, 0};
    if (s->use_pbc) pair_shift(st, s->qswitch, sw_of(st, j), t);   /* nonbond_qp_box (md.f90:11060-11068) */
    double dx[3] = {X(j, 0) - X(i, 0) - t[0], X(j, 1) - X(i, 1) - t[1], X(j, 2) - X(i, 2) - t[2]};
    double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
    if (!s->qvdw_flag) {
      r2 = 1. / r2;
      double r6 = r2 * r2 * r2, r = sqrt(r2);
      for (int ss = 0; ss < S; ss++) {
        int ti = s->iac[i];
        double aLJ, bLJ;
        ljp(s, avdw(s, ti, lj), avdw(s, tj, lj), bvdw(s, ti, lj), bvdw(s, tj, lj), &aLJ, &bLJ);
        float qq = s->qcrg[iq * S + ss] * s->crg[j];
        double Vel = (double)qq * r;
        if (lj == 3) Vel = Vel * s->el14_scale;
        double Va = aLJ * r6 * r6, Vb = bLJ * r6;
        double dv = r2 * (-Vel - 12. * Va + 6. * Vb) * s->lambda[ss];
        apply_pair(st, i, j, dv, dx);
        EQV(ss, QB_EQ_QP_EL) += Vel;
        EQV(ss, QB_EQ_QP_VDW) += Va - Vb;
      }
    } else {
      double r6 = r2 * r2 * r2;
      r2 = 1. / r2;
      double r = sqrt(r2);
      for (int ss = 0; ss < S; ss++) {
        int ti = s->qiac[iq * S + ss];
        double aLJ, bLJ;
        ljp(s, s->qavdw[3 * ti + qlj - 1], avdw(s, tj, lj), s->qbvdw[3 * ti + qlj - 1], bvdw(s, tj, lj), &aLJ, &bLJ);
        float qq = s->qcrg[iq * S + ss] * s->crg[j];
        double Vel = (double)qq * r;
        if (lj == 3) Vel = Vel * s->el14_scale;
        double r6sc = r6 + s->sc_lookup[((size_t)iq * ncol + tj) * S + ss];
        double Va = aLJ / (r6sc * r6sc), Vb = bLJ / r6sc;
        double dv = r2 * (-Vel - (12. * Va - 6. * Vb) * (r6 / r6sc)) * s->lambda[ss];
        apply_pair(st, i, j, dv, dx);
        EQV(ss, QB_EQ_QP_EL) += Vel;
        EQV(ss, QB_EQ_QP_VDW) += Va - Vb;
      }
    }
  }
}

/* nonbond_ww_spc (md.f90:11823) */
static void nonbond_ww(qo_state *st) {
  const qb_sysview *s = st->s;
  const float qo = s->crg_ow, qh = s->crg_hw;
  const float qoo = qo * qo, qoh = qo * qh, qhh = qh * qh;
  int ip = 0;
  for (int iw = 0; iw < st->nwat; iw++) {
    int io = st->NS + 3 * iw;
    for (; st->ww[ip] >= 0; ip++) {
      int jo = st->ww[ip];
      double t[3];
      pair_shift(st, io, jo, t);   /* nonbond_ww_spc_box (md.f90:12078-12100) */
      for (int a = 0; a < 3; a++) {
        int ia = io + a;
        for (int b = 0; b < 3; b++) {
          int jb = jo + b;
          double dx[3] = {X(jb, 0) - X(ia, 0) - t[0], X(jb, 1) - X(ia, 1) - t[1], X(jb, 2) - X(ia, 2) - t[2]};
          double rinv = sqrt(1.0 / (dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]));
          double r2 = rinv * rinv;
          float qq = (a == 0 && b == 0) ? qoo : ((a == 0 || b == 0) ? qoh : qhh);
          double Vel = (double)qq * rinv, dv;
          /* nonbon2_ww (md.f90:10099) and nonbond_3atomsolvent (12317) take LJ on
           * all nine site pairs; nonbond_ww_spc (11823) on O-O only */
          if ((a == 0 && b == 0) || s->ww_hlj) {
            double A = (a == 0 && b == 0) ? s->A_OO : ((a == 0 || b == 0) ? s->A_OH : s->A_HH);
            double B = (a == 0 && b == 0) ? s->B_OO : ((a == 0 || b == 0) ? s->B_OH : s->B_HH);
            double r6 = r2 * r2 * r2;
            double Va = A * r6 * r6, Vb = B * r6;
            st->E[QB_E_WW_VDW] += Va - Vb;
            dv = r2 * (-Vel - 12. * Va + 6. * Vb);
          } else {
            dv = r2 * (-Vel);
          }
          st->E[QB_E_WW_EL] += Vel;
          apply_pair(st, ia, jb, dv, dx);
        }
      }
    }
    ip++; /* skip terminator */
  }
}

/* nonbond_qw_spc (md.f90:11302); with hydrogen LJ, nonbon2_qw (9798) and
 * nonbond_qw_3atom (11545): both hydrogen sites add LJ with the hydrogen
 * type's parameters and soft-core shift sc_lookup(iq, iac_hw, state) */
static void nonbond_qw(qo_state *st) {
  const qb_sysview *s = st->s;
  int S = st->S, ncol = s->natyps + st->nq;
  int iac_ow = s->iac_ow, iac_hw = s->iac_hw;
  double aO[2] = {avdw(s, iac_ow, 1), avdw(s, iac_ow, 2)}, bO[2] = {bvdw(s, iac_ow, 1), bvdw(s, iac_ow, 2)};
  double aH[2] = {avdw(s, iac_hw, 1), avdw(s, iac_hw, 2)}, bH[2] = {bvdw(s, iac_hw, 1), bvdw(s, iac_hw, 2)};
  for (int jw = 0; jw < st->nqw; jw++) {
    int j = st->qw[jw];
    double t[3] = {0, 0, 0};
    if (s->use_pbc) pair_shift(st, s->qswitch, j, t);   /* nonbond_qw_spc_box (md.f90:11440-11446) */
    for (int iq = 0; iq < st->nq; iq++) {
      int i = s->iqseq[iq];
      double dO[3], dH1[3], dH2[3];
      for (int k = 0; k < 3; k++) {
        dO[k] = X(j, k) - X(i, k) - t[k];
        dH1[k] = X(j + 1, k) - X(i, k) - t[k];
        dH2[k] = X(j + 2, k) - X(i, k) - t[k];
      }
      double r2O = dO[0] * dO[0] + dO[1] * dO[1] + dO[2] * dO[2];
      double rH1 = sqrt(1.0 / (dH1[0] * dH1[0] + dH1[1] * dH1[1] + dH1[2] * dH1[2]));
      double rH2 = sqrt(1.0 / (dH2[0] * dH2[0] + dH2[1] * dH2[1] + dH2[2] * dH2[2]));
      double r6hc = r2O * r2O * r2O;
      r2O = 1.0 / r2O;
      double rO = sqrt(r2O);
      double r2H1 = rH1 * rH1, r2H2 = rH2 * rH2;
      double r6sc = r6hc, dvO = 0, dvH1 = 0, dvH2 = 0, Va = 0, Vb = 0;
      int lj = ljcode(s, iac_ow, s->iac[i]);
      if (!s->qvdw_flag) {
        double r6O = 1. / r6hc, A, B;
        ljp(s, avdw(s, s->iac[i], lj), aO[lj - 1], bvdw(s, s->iac[i], lj), bO[lj - 1], &A, &B);
        Va = A * r6O * r6O;
        Vb = B * r6O;
      }
      int ljh = s->ww_hlj ? ljcode(s, iac_hw, s->iac[i]) : 1;
      double r6H[2] = {r2H1 * r2H1 * r2H1, r2H2 * r2H2 * r2H2}, VaH[2] = {0, 0}, VbH[2] = {0, 0};
      if (s->ww_hlj && !s->qvdw_flag) {
        double A, B;
        ljp(s, avdw(s, s->iac[i], ljh), aH[ljh - 1], bvdw(s, s->iac[i], ljh), bH[ljh - 1], &A, &B);
        for (int h = 0; h < 2; h++) { VaH[h] = A * r6H[h] * r6H[h]; VbH[h] = B * r6H[h]; }
      }
      for (int ss = 0; ss < S; ss++) {
        if (s->qvdw_flag) {
          int ti = s->qiac[iq * S + ss];
          double A, B;
          ljp(s, s->qavdw[3 * ti], aO[lj - 1], s->qbvdw[3 * ti], bO[lj - 1], &A, &B);
          r6sc = r6hc + s->sc_lookup[((size_t)iq * ncol + iac_ow) * S + ss];
          Va = A / (r6sc * r6sc);
          Vb = B / r6sc;
        }
        float qq = s->qcrg[iq * S + ss];
        double VelO = (double)(s->crg_ow * qq) * rO;
        double VelH1 = (double)(s->crg_hw * qq) * rH1;
        double VelH2 = (double)(s->crg_hw * qq) * rH2;
        double lam = s->lambda[ss];
        dvO += r2O * (-VelO - ((12. * Va - 6. * Vb) * (r6hc / r6sc))) * lam;
        if (s->ww_hlj) {
          double fH[2] = {1.0, 1.0};
          if (s->qvdw_flag) {
            int ti = s->qiac[iq * S + ss];
            double A, B, sc = s->sc_lookup[((size_t)iq * ncol + iac_hw) * S + ss];
            ljp(s, s->qavdw[3 * ti], aH[ljh - 1], s->qbvdw[3 * ti], bH[ljh - 1], &A, &B);
            for (int h = 0; h < 2; h++) {
              double d6 = 1.0 / r6H[h], r6s = d6 + sc;
              VaH[h] = A / (r6s * r6s);
              VbH[h] = B / r6s;
              fH[h] = d6 / r6s;
            }
          }
          dvH1 += r2H1 * (-VelH1 - (12. * VaH[0] - 6. * VbH[0]) * fH[0]) * lam;
          dvH2 += r2H2 * (-VelH2 - (12. * VaH[1] - 6. * VbH[1]) * fH[1]) * lam;
          EQV(ss, QB_EQ_QW_VDW) += VaH[0] + VaH[1] - VbH[0] - VbH[1];
        } else {
          dvH1 -= r2H1 * VelH1 * lam;
          dvH2 -= r2H2 * VelH2 * lam;
        }
        EQV(ss, QB_EQ_QW_EL) += VelO + VelH1 + VelH2;
        EQV(ss, QB_EQ_QW_VDW) += Va - Vb;
      }
      for (int k = 0; k < 3; k++) {
        D(i, k) -= dvO * dO[k] + dvH1 * dH1[k] + dvH2 * dH2[k];
        D(j, k) += dvO * dO[k];
        D(j + 1, k) += dvH1 * dH1[k];
        D(j + 2, k) += dvH2 * dH2[k];
      }
    }
  }
}

/* nonbond_qq (md.f90:10763) / nonbon2_qq (9385); with qq_use_library_charges,
 * nonbond_qq_lib_charges (10872): Q-Q pairs take both atoms' topology charges,
 * and nonbon2_qq_lib_charges (9494): every pair takes crg(i).  A Q-Q soft pair
 * (LJ code 2) multiplies A and B under either rule (9426). */
static void nonbond_qq(qo_state *st) {
  const qb_sysview *s = st->s;
  int S = st->S, ncol = s->natyps + st->nq;
  for (int ss = 0; ss < S; ss++) {
    for (int p = s->nbqq_off[ss]; p < s->nbqq_off[ss] + s->nbqq_count[ss]; p++) {
      int iq = s->nbqq_iq[p], j = s->nbqq_j[p], jq = s->nbqq_jq[p], lj = s->nbqq_ljcod[p];
      int i = s->iqseq[iq];
      int lib = s->qq_use_library_charges && jq >= 0;
      int lib_i = s->qq_use_library_charges && (jq >= 0 || s->ivdw_rule == 2);
      double qi = lib_i ? (double)s->crg[i] : s->qcrg[iq * S + ss], qj, aLJ, bLJ;
      double el = s->nbqq_el_scale[p];
      if (!s->qvdw_flag) {
        int ti = s->iac[i], tj = s->iac[j];
        ljp(s, avdw(s, ti, lj), avdw(s, tj, lj), bvdw(s, ti, lj), bvdw(s, tj, lj), &aLJ, &bLJ);
        qj = jq >= 0 && !lib ? (double)s->qcrg[jq * S + ss] : (double)s->crg[j];
      } else {
        int ti = s->qiac[iq * S + ss];
        double ai = s->qavdw[3 * ti + lj - 1], bi = s->qbvdw[3 * ti + lj - 1];
        if (jq >= 0) {
          int tj = s->qiac[jq * S + ss];
          if (lj == 2) { aLJ = ai * s->qavdw[3 * tj + 1]; bLJ = bi * s->qbvdw[3 * tj + 1]; }
          else ljp(s, ai, s->qavdw[3 * tj + lj - 1], bi, s->qbvdw[3 * tj + lj - 1], &aLJ, &bLJ);
          qj = lib ? (double)s->crg[j] : s->qcrg[jq * S + ss];
        } else {
          if (lj == 2) { ai = s->qavdw[3 * ti]; bi = s->qbvdw[3 * ti]; }
          int tj = s->iac[j];
          ljp(s, ai, avdw(s, tj, lj), bi, bvdw(s, tj, lj), &aLJ, &bLJ);
          qj = s->crg[j];
        }
      }
      double dx[3] = {X(j, 0) - X(i, 0), X(j, 1) - X(i, 1), X(j, 2) - X(i, 2)};
      double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
      double r6hc = r2 * r2 * r2;
      /* jq = -1 reads column natyps-1+0 = the reference's sc_lookup(iq, natyps+0, s) */
      int col = s->natyps + jq;
      double r6 = r2 * r2 * r2 + s->sc_lookup[((size_t)iq * ncol + col) * S + ss];
      r6 = 1. / r6;
      double r12 = r6 * r6;
      r2 = 1. / r2;
      double r = sqrt(r2);
      double Vel = qi * qj * r * el, Va, Vb, dv;
      if (lj == 3) Vel = Vel * s->el14_scale;
      if (s->qvdw_flag && jq >= 0 && lj == 2) {
        Va = aLJ * exp(-bLJ / r);
        Vb = 0.0;
        dv = r2 * (-Vel - bLJ * Va / r) * s->lambda[ss];
      } else {
        Va = aLJ * r12;
        Vb = bLJ * r6;
        dv = r2 * (-Vel - (12. * Va - 6. * Vb) * r6hc * r6) * s->lambda[ss];
      }
      apply_pair(st, i, j, dv, dx);
      if (jq >= 0) { EQV(ss, QB_EQ_QQ_EL) += Vel; EQV(ss, QB_EQ_QQ_VDW) += Va - Vb; }
      else { EQV(ss, QB_EQ_QP_EL) += Vel; EQV(ss, QB_EQ_QP_VDW) += Va - Vb; }
    }
  }
}

/* lrf_taylor (md.f90:3646) */
static void lrf_taylor(qo_state *st) {
  const qb_sysview *s = st->s;
  for (int i = 0; i < st->N; i++) {
    if (s->excl[i] || s->iqatom[i] >= 0) continue;
    const lrf_t *L = &st->lrf[s->iwhich_cgp[i]];
    double dr[3] = {L->c[0] - X(i, 0), L->c[1] - X(i, 1), L->c[2] - X(i, 2)};
    double V = L->p0 + L->p1[0] * dr[0] + L->p1[1] * dr[1] + L->p1[2] * dr[2];
    for (int a = 0; a < 3; a++)
      V += 0.5 * (L->p2[3 * a] * dr[0] + L->p2[3 * a + 1] * dr[1] + L->p2[3 * a + 2] * dr[2]) * dr[a];
    double q = (double)s->crg[i];
    st->E[QB_E_LRF] += 0.5 * q * V;
    for (int c = 0; c < 3; c++) {
      double df = L->p1[c] + L->p2[3 * c] * dr[0] + L->p2[3 * c + 1] * dr[1] + L->p2[3 * c + 2] * dr[2];
      for (int a = 0; a < 3; a++) {
        const double *p = &L->p3[9 * c + 3 * a];
        df += 0.5 * (p[0] * dr[0] + p[1] * dr[1] + p[2] * dr[2]) * dr[a];
      }
      D(i, c) -= q * df;
    }
  }
}

/* --------------------------------------------------------------- bonded */

static double bonds(qo_state *st, int b0, int b1) {
  const qb_sysview *s = st->s;
  double e = 0;
  for (int b = b0; b < b1; b++) {
    int i = s->bnd_i[b], j = s->bnd_j[b];
    double r[3] = {X(j, 0) - X(i, 0), X(j, 1) - X(i, 1), X(j, 2) - X(i, 2)};
    double bl = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    double db = bl - s->bnd_b0[b];
    e += 0.5 * s->bnd_fk[b] * db * db;
    double dv = s->bnd_fk[b] * db / bl;
    for (int k = 0; k < 3; k++) { D(j, k) += r[k] * dv; D(i, k) -= r[k] * dv; }
  }
  return e;
}

/* angle (md.f90:814) */
static void angle_grad(const double rji[3], const double rjk[3], double *theta, double di[3], double dk[3],
                       double tiny_f1) {
  double bji2inv = 1. / (rji[0] * rji[0] + rji[1] * rji[1] + rji[2] * rji[2]);
  double bjk2inv = 1. / (rjk[0] * rjk[0] + rjk[1] * rjk[1] + rjk[2] * rjk[2]);
  double bjiinv = sqrt(bji2inv), bjkinv = sqrt(bjk2inv);
  double scp = (rji[0] * rjk[0] + rji[1] * rjk[1] + rji[2] * rjk[2]) * bjiinv * bjkinv;
  if (scp > 1.0) scp = 1.0;
  else if (scp < -1.0) scp = -1.0;
  double ang = acos(scp);
  double f1 = sin(ang);
  if (fabs(f1) < 1.e-12) f1 = tiny_f1;
  else f1 = -1.0 / f1;
  for (int k = 0; k < 3; k++) {
    di[k] = f1 * (rjk[k] * bjiinv * bjkinv - scp * rji[k] * bji2inv);
    dk[k] = f1 * (rji[k] * bjiinv * bjkinv - scp * rjk[k] * bjk2inv);
  }
  *theta = ang;
}

static double angles(qo_state *st, int a0, int a1) {
  const qb_sysview *s = st->s;
  double e = 0;
  for (int a = a0; a < a1; a++) {
    int i = s->ang_i[a], j = s->ang_j[a], k = s->ang_k[a];
    double rji[3], rjk[3], di[3], dk[3], th;
    for (int c = 0; c < 3; c++) { rji[c] = X(i, c) - X(j, c); rjk[c] = X(k, c) - X(j, c); }
    angle_grad(rji, rjk, &th, di, dk, -1.e12);
    double da = th - s->ang_th0[a];
    e += 0.5 * s->ang_fk[a] * da * da;
    double dv = s->ang_fk[a] * da;
    for (int c = 0; c < 3; c++) {
      D(i, c) += dv * di[c];
      D(k, c) += dv * dk[c];
      D(j, c) -= dv * (di[c] + dk[c]);
    }
  }
  return e;
}

/* urey_bradley (md.f90:904): k (r13 - r0)^2 over the angles' 1-3 pairs with k > 0 */
static double urey_bradley(qo_state *st, int a0, int a1) {
  const qb_sysview *s = st->s;
  double e = 0;
  for (int a = a0; a < a1; a++) {
    double fk = s->ang_ureyfk[a];
    if (!(fk > 0.)) continue;
    int i = s->ang_i[a], k = s->ang_k[a];
    double rik[3] = {X(k, 0) - X(i, 0), X(k, 1) - X(i, 1), X(k, 2) - X(i, 2)};
    double dik = sqrt(rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2]);
    double ru = dik - s->ang_ureyr0[a];
    e += fk * ru * ru;
    double du = 2 * fk * ru / dik;
    for (int c = 0; c < 3; c++) { D(k, c) += du * rik[c]; D(i, c) -= du * rik[c]; }
  }
  return e;
}

/* dihedral geometry shared by torsion (14793), improper (1677),
 * improper2 (1789): phi and the 12 gradient components */
static double dihedral(qo_state *st, int i, int j, int k, int l, double dp[12]) {
  double rji[3], rjk[3], rkl[3], rnj[3], rnk[3], di[3], dl[3], rki[3], rlj[3];
  for (int c = 0; c < 3; c++) { rji[c] = X(i, c) - X(j, c); rjk[c] = X(k, c) - X(j, c); rkl[c] = X(l, c) - X(k, c); }
  rnj[0] = rji[1] * rjk[2] - rji[2] * rjk[1];
  rnj[1] = rji[2] * rjk[0] - rji[0] * rjk[2];
  rnj[2] = rji[0] * rjk[1] - rji[1] * rjk[0];
  rnk[0] = -rjk[1] * rkl[2] + rjk[2] * rkl[1];
  rnk[1] = -rjk[2] * rkl[0] + rjk[0] * rkl[2];
  rnk[2] = -rjk[0] * rkl[1] + rjk[1] * rkl[0];
  double bj2inv = 1. / (rnj[0] * rnj[0] + rnj[1] * rnj[1] + rnj[2] * rnj[2]);
  double bk2inv = 1. / (rnk[0] * rnk[0] + rnk[1] * rnk[1] + rnk[2] * rnk[2]);
  double bjinv = sqrt(bj2inv), bkinv = sqrt(bk2inv);
  double scp = (rnj[0] * rnk[0] + rnj[1] * rnk[1] + rnj[2] * rnk[2]) * (bjinv * bkinv);
  double phi;
  if (scp > 1.0) { scp = 1.0; phi = acosf(1.0f); }
  else if (scp < -1.0) { scp = -1.0; phi = acosf(-1.0f); }
  else phi = acos(scp);
  double sgn = rjk[0] * (rnj[1] * rnk[2] - rnj[2] * rnk[1]) + rjk[1] * (rnj[2] * rnk[0] - rnj[0] * rnk[2]) +
               rjk[2] * (rnj[0] * rnk[1] - rnj[1] * rnk[0]);
  if (sgn < 0) phi = -phi;
  double f1 = sin(phi);
  if (fabs(f1) < 1.e-12) f1 = 1.e-12;
  f1 = -1.0 / f1;
  for (int c = 0; c < 3; c++) {
    di[c] = f1 * (rnk[c] * (bjinv * bkinv) - scp * rnj[c] * bj2inv);
    dl[c] = f1 * (rnj[c] * (bjinv * bkinv) - scp * rnk[c] * bk2inv);
    rki[c] = rji[c] - rjk[c];
    rlj[c] = -rjk[c] - rkl[c];
  }
  dp[0] = rjk[1] * di[2] - rjk[2] * di[1];
  dp[1] = rjk[2] * di[0] - rjk[0] * di[2];
  dp[2] = rjk[0] * di[1] - rjk[1] * di[0];
  dp[3] = rki[1] * di[2] - rki[2] * di[1] + rkl[1] * dl[2] - rkl[2] * dl[1];
  dp[4] = rki[2] * di[0] - rki[0] * di[2] + rkl[2] * dl[0] - rkl[0] * dl[2];
  dp[5] = rki[0] * di[1] - rki[1] * di[0] + rkl[0] * dl[1] - rkl[1] * dl[0];
  dp[6] = rlj[1] * dl[2] - rlj[2] * dl[1] - rji[1] * di[2] + rji[2] * di[1];
  dp[7] = rlj[2] * dl[0] - rlj[0] * dl[2] - rji[2] * di[0] + rji[0] * di[2];
  dp[8] = rlj[0] * dl[1] - rlj[1] * dl[0] - rji[0] * di[1] + rji[1] * di[0];
  dp[9] = rjk[1] * dl[2] - rjk[2] * dl[1];
  dp[10] = rjk[2] * dl[0] - rjk[0] * dl[2];
  dp[11] = rjk[0] * dl[1] - rjk[1] * dl[0];
  return phi;
}

static void apply4(qo_state *st, int i, int j, int k, int l, double dv, const double dp[12]) {
  int at[4] = {i, j, k, l};
  for (int a = 0; a < 4; a++)
    for (int c = 0; c < 3; c++) D(at[a], c) += dv * dp[3 * a + c];
}

static double torsions(qo_state *st, int t0, int t1) {
  const qb_sysview *s = st->s;
  double e = 0, dp[12];
  for (int t = t1 - 1; t >= t0; t--) {
    double phi = dihedral(st, s->tor_i[t], s->tor_j[t], s->tor_k[t], s->tor_l[t], dp);
    double arg = (double)s->tor_rmult[t] * phi - (double)s->tor_deltor[t];
    e += (double)s->tor_fk[t] * (1.0 + cos(arg)) * (double)s->tor_paths[t];
    float rf = s->tor_rmult[t] * s->tor_fk[t];
    double dv = -((double)rf * sin(arg) * (double)s->tor_paths[t]);
    apply4(st, s->tor_i[t], s->tor_j[t], s->tor_k[t], s->tor_l[t], dv, dp);
  }
  return e;
}

static double impropers(qo_state *st, int t0, int t1) {
  const qb_sysview *s = st->s;
  double e = 0, dp[12];
  double pi = fpi();
  for (int t = t1 - 1; t >= t0; t--) {
    double phi = dihedral(st, s->imp_i[t], s->imp_j[t], s->imp_k[t], s->imp_l[t], dp);
    double dv;
    if (s->ff_type == 2) { /* improper2: periodic */
      double arg = 2 * phi - (double)s->imp_imp0[t];
      e += (double)s->imp_fk[t] * (1 + cos(arg));
      dv = -2 * (double)s->imp_fk[t] * sin(arg);
    } else { /* improper: harmonic */
      double arg = phi - (double)s->imp_imp0[t];
      arg = arg - 2. * pi * (double)lround(arg / (2. * pi));
      dv = (double)s->imp_fk[t] * arg;
      e += 0.5 * dv * arg;
    }
    apply4(st, s->imp_i[t], s->imp_j[t], s->imp_k[t], s->imp_l[t], dv, dp);
  }
  return e;
}

/* EMorseD of Q bond b as qbond computed it in state ss, and dMorse_i
 * (md.f90:14086-14108); dMorse_j = -dMorse_i */
static double morse_gamma(qo_state *st, int b, int ss, double dmi[3]) {
  const qb_sysview *s = st->s;
  int S = st->S, i = s->qbnd_i[b], j = s->qbnd_j[b];
  double r[3] = {X(j, 0) - X(i, 0), X(j, 1) - X(i, 1), X(j, 2) - X(i, 2)};
  double bl = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  double amz = s->qbnd_amz[b * S + ss];
  double db = bl - s->qbnd_r0[b * S + ss];
  double fexp = exp(-amz * db);
  if (db > 0) {
    for (int k = 0; k < 3; k++) dmi[k] = +2. * amz * (fexp - fexp * fexp) * s->lambda[ss] / bl * r[k];
    return -(fexp * fexp - 2. * fexp);
  }
  dmi[0] = dmi[1] = dmi[2] = 0;
  return 1.0;
}

static void morse_apply(qo_state *st, int b, const double dmi[3], double e) {
  int i = st->s->qbnd_i[b], j = st->s->qbnd_j[b];
  for (int k = 0; k < 3; k++) { D(i, k) += dmi[k] * e; D(j, k) += -dmi[k] * e; }
}

/* qbond (14060), qangle (13896), qtorsion (14262), qimproper (14117); terms
 * coupled to a Morse bond are scaled by gamma = EMorseD, with the bond's
 * values from the state qbond last set them in */
static void qbonded(qo_state *st, int ss) {
  const qb_sysview *s = st->s;
  int S = st->S;
  double lam = s->lambda[ss];
  for (int b = 0; b < s->nqbond; b++) {
    if (!s->qbnd_on[b * S + ss]) continue;
    int i = s->qbnd_i[b], j = s->qbnd_j[b];
    double r[3] = {X(j, 0) - X(i, 0), X(j, 1) - X(i, 1), X(j, 2) - X(i, 2)};
    double bl = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    double Dmz = s->qbnd_Dmz[b * S + ss], amz = s->qbnd_amz[b * S + ss], fk = s->qbnd_fk[b * S + ss];
    double db = bl - s->qbnd_r0[b * S + ss];
    double fexp = exp(-amz * db);
    double be = Dmz * (fexp * fexp - 2. * fexp) + 0.5 * fk * db * db;
    EQV(ss, QB_EQ_BOND) += be;
    double dv = (2. * Dmz * amz * (fexp - fexp * fexp) + fk * db) * lam / bl;
    for (int k = 0; k < 3; k++) { D(i, k) -= dv * r[k]; D(j, k) += dv * r[k]; }
  }
  for (int a = 0; a < s->nqangle; a++) {
    if (!s->qang_on[a * S + ss]) continue;
    int i = s->qang_i[a], j = s->qang_j[a], k = s->qang_k[a];
    double rji[3], rjk[3];
    for (int c = 0; c < 3; c++) { rji[c] = X(i, c) - X(j, c); rjk[c] = X(k, c) - X(j, c); }
    double bji = sqrt(rji[0] * rji[0] + rji[1] * rji[1] + rji[2] * rji[2]);
    double bjk = sqrt(rjk[0] * rjk[0] + rjk[1] * rjk[1] + rjk[2] * rjk[2]);
    double scp = (rji[0] * rjk[0] + rji[1] * rjk[1] + rji[2] * rjk[2]) / (bji * bjk);
    if (scp > 1.0) scp = 1.0;
    if (scp < -1.0) scp = -1.0;
    double ang = acos(scp);
    double fk = s->qang_fk[a * S + ss];
    double da = ang - s->qang_th0[a * S + ss];
    int cb = s->qang_cpl[a];
    double gamma = 1.0, dmi[3];
    if (cb >= 0) gamma = morse_gamma(st, cb, s->qang_cpl_src[a * S + ss], dmi);
    double ae = 0.5 * fk * da * da;
    EQV(ss, QB_EQ_ANGLE) += ae * gamma;
    double dv = gamma * fk * da * lam;
    double f1 = sin(ang);
    if (fabs(f1) < 1.e-12) f1 = 1.e-12;
    f1 = -1.0 / f1;
    for (int c = 0; c < 3; c++) {
      double di = f1 * (rjk[c] / (bji * bjk) - scp * rji[c] / (bji * bji));
      double dk = f1 * (rji[c] / (bji * bjk) - scp * rjk[c] / (bjk * bjk));
      D(i, c) += dv * di;
      D(k, c) += dv * dk;
      D(j, c) -= dv * (di + dk);
    }
    if (cb >= 0) morse_apply(st, cb, dmi, ae);
    /* qurey_bradley (md.f90:13992): energy only, its gradient is never applied
     * (a Morse coupling's is) */
    double ufk = s->qang_ureyfk[a * S + ss];
    if (ufk != 0.) {
      double rik[3] = {X(k, 0) - X(i, 0), X(k, 1) - X(i, 1), X(k, 2) - X(i, 2)};
      double ru = sqrt(rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2]) - s->qang_ureyr0[a * S + ss];
      double eu = ufk * ru * ru, g = 1.0;
      int cu = s->qang_cpl_ub[a];
      if (cu >= 0) g = morse_gamma(st, cu, s->qang_cpl_ub_src[a * S + ss], dmi);
      EQV(ss, QB_EQ_ANGLE) += eu * g;
      if (cu >= 0) morse_apply(st, cu, dmi, eu);
    }
  }
  double dp[12], pi = fpi();
  for (int t = 0; t < s->nqtor; t++) {
    if (!s->qtor_on[t * S + ss]) continue;
    double phi = dihedral(st, s->qtor_i[t], s->qtor_j[t], s->qtor_k[t], s->qtor_l[t], dp);
    double rm = s->qtor_rmult[t * S + ss], fk = s->qtor_fk[t * S + ss];
    double arg = rm * phi - s->qtor_deltor[t * S + ss];
    int cb = s->qtor_cpl[t];
    double gamma = 1.0, dmi[3];
    if (cb >= 0) gamma = morse_gamma(st, cb, s->qtor_cpl_src[t * S + ss], dmi);
    double pe = fk * (1.0 + cos(arg));
    EQV(ss, QB_EQ_TORSION) += pe * gamma;
    double dv = -rm * fk * sin(arg) * gamma * lam;
    apply4(st, s->qtor_i[t], s->qtor_j[t], s->qtor_k[t], s->qtor_l[t], dv, dp);
    if (cb >= 0) morse_apply(st, cb, dmi, pe);
  }
  for (int t = 0; t < s->nqimp; t++) {
    if (!s->qimp_on[t * S + ss]) continue;
    double phi = dihedral(st, s->qimp_i[t], s->qimp_j[t], s->qimp_k[t], s->qimp_l[t], dp);
    double arg = phi - s->qimp_imp0[t * S + ss];
    arg = arg - 2. * pi * (double)lround(arg / (2. * pi));
    int cb = s->qimp_cpl[t];
    double gamma = 1.0, dmi[3];
    if (cb >= 0) {
      gamma = morse_gamma(st, cb, s->qimp_cpl_src[t * S + ss], dmi);
      if (s->qimp_cpl_flag[t] == 1) gamma = 1 - gamma;
    }
    double dv = s->qimp_fk[t * S + ss] * arg;
    double pe = 0.5 * dv * arg;
    EQV(ss, QB_EQ_IMPROPER) += pe * gamma;
    dv = dv * gamma * lam;
    apply4(st, s->qimp_i[t], s->qimp_j[t], s->qimp_k[t], s->qimp_l[t], dv, dp);
    if (cb >= 0) morse_apply(st, cb, dmi, pe);
  }
}

/* ------------------------------------------------------------ restraints */

/* fix_shell (md.f90:1414) */
static void fix_shell(qo_state *st) {
  const qb_sysview *s = st->s;
  for (int i = 0; i < st->N; i++) {
    if (!(s->excl[i] || s->shell[i])) continue;
    double fk = s->excl[i] ? s->fk_fix : s->fk_pshell;
    double dr[3] = {X(i, 0) - s->xtop[3 * i], X(i, 1) - s->xtop[3 * i + 1], X(i, 2) - s->xtop[3 * i + 2]};
    double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
    double e = 0.5 * fk * r2;
    if (s->excl[i]) st->E[QB_E_RST_FIX] += e;
    if (s->shell[i]) st->E[QB_E_RST_SHELL] += e;
    for (int k = 0; k < 3; k++) D(i, k) += fk * dr[k];
  }
}

static void rst_energy(qo_state *st, int ipsi, double e) {
  if (ipsi == 0) {
    for (int k = 0; k < st->S; k++) EQV(k, QB_EQ_RESTRAINT) += e;
    if (st->S == 0) st->E[QB_E_RST_PROTEIN] += e;
  } else {
    EQV(ipsi - 1, QB_EQ_RESTRAINT) += e;
  }
}

/* p_restrain (md.f90:12940) */
static void p_restrain(qo_state *st) {
  const qb_sysview *s = st->s;
  for (int r = 0; r < s->nrstr_seq; r++) {
    double fk = s->rseq_fk[r];
    int ih = s->rseq_ih[r], tc = s->rseq_to_center[r];
    if (tc == 1 || tc == 2) {
      double dr[3] = {0, 0, 0}, tot = 0;
      int n = 0;
      for (int i = s->rseq_i[r]; i <= s->rseq_j[r]; i++) {
        if (!(s->heavy[i] || ih == 1)) continue;
        double w = tc == 2 ? s->mass[i] : 1.0;
        n++;
        tot += w;
        for (int k = 0; k < 3; k++) dr[k] += (X(i, k) - s->xtop[3 * i + k]) * w;
      }
      if ((tc == 1 && n > 0) || (tc == 2 && tot > 0)) {
        for (int k = 0; k < 3; k++) dr[k] = tc == 1 ? dr[k] / n : dr[k] / tot;
        double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        st->E[QB_E_RST_PROTEIN] += 0.5 * fk * r2;
        for (int i = s->rseq_i[r]; i <= s->rseq_j[r]; i++) {
          if (!(s->heavy[i] || ih == 1)) continue;
          for (int k = 0; k < 3; k++)
            D(i, k) += tc == 1 ? fk * dr[k] * s->mass[i] / (double)12.010f : fk * dr[k];
        }
      }
    } else {
      for (int i = s->rseq_i[r]; i <= s->rseq_j[r]; i++) {
        if (!(s->heavy[i] || ih == 1)) continue;
        double dr[3] = {X(i, 0) - s->xtop[3 * i], X(i, 1) - s->xtop[3 * i + 1], X(i, 2) - s->xtop[3 * i + 2]};
        double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        st->E[QB_E_RST_PROTEIN] += 0.5 * fk * r2;
        for (int k = 0; k < 3; k++) D(i, k) += fk * dr[k];
      }
    }
  }
  for (int r = 0; r < s->nrstr_pos; r++) {
    int ipsi = s->rpos_ipsi[r], i = s->rpos_i[r];
    double dr[3], wgt = ipsi != 0 ? s->lambda[ipsi - 1] : 1.0, e = 0;
    for (int k = 0; k < 3; k++) dr[k] = X(i, k) - s->rpos_x[3 * r + k];
    for (int k = 0; k < 3; k++) e += 0.5 * s->rpos_fk[3 * r + k] * dr[k] * dr[k];
    for (int k = 0; k < 3; k++) D(i, k) += s->rpos_fk[3 * r + k] * dr[k] * wgt;
    rst_energy(st, ipsi, e);
  }
  for (int r = 0; r < s->nrstr_dist; r++) {
    int ipsi = s->rdis_ipsi[r], i = s->rdis_i[r], j = s->rdis_j[r];
    double dr[3] = {X(j, 0) - X(i, 0), X(j, 1) - X(i, 1), X(j, 2) - X(i, 2)};
    if (s->use_pbc)   /* md.f90:13096-13101 */
      for (int k = 0; k < 3; k++) dr[k] -= img(st, k, dr[k]);
    double wgt = ipsi != 0 ? s->lambda[ipsi - 1] : 1.0;
    double b = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]), db;
    if (b < s->rdis_d1[r]) db = b - s->rdis_d1[r];
    else if (b > s->rdis_d2[r]) db = b - s->rdis_d2[r];
    else continue;
    double e = 0.5 * s->rdis_fk[r] * db * db, dv = wgt * s->rdis_fk[r] * db / b;
    for (int k = 0; k < 3; k++) { D(j, k) += dr[k] * dv; D(i, k) -= dr[k] * dv; }
    rst_energy(st, ipsi, e);
  }
  for (int r = 0; r < s->nrstr_angl; r++) {
    int ipsi = s->rang_ipsi[r], i = s->rang_i[r], j = s->rang_j[r], k = s->rang_k[r];
    double d1[3], d2[3];
    for (int c = 0; c < 3; c++) { d1[c] = X(i, c) - X(j, c); d2[c] = X(k, c) - X(j, c); }
    if (s->use_pbc)   /* md.f90:13160-13168 */
      for (int c = 0; c < 3; c++) { d1[c] -= img(st, c, d1[c]); d2[c] -= img(st, c, d2[c]); }
    double wgt = ipsi != 0 ? s->lambda[ipsi - 1] : 1.0;
    double r2ij = d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2], r2jk = d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2];
    double rij = sqrt(r2ij), rjk = sqrt(r2jk);
    double scp = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) / (rij * rjk);
    if (scp > 1.0) scp = 1.0;
    if (scp < -1.0) scp = -1.0;
    double th = acos(scp);
    double db = th - s->rang_ang[r] * (fpi() / 180.0);
    double e = 0.5 * s->rang_fk[r] * db * db, dv = wgt * s->rang_fk[r] * db;
    double f1 = sin(th);
    if (fabs(f1) < 1.e-12) f1 = -1.e12;
    else f1 = -1.0 / f1;
    for (int c = 0; c < 3; c++) {
      double di = f1 * (d2[c] / (rij * rjk) - scp * d1[c] / r2ij);
      double dk = f1 * (d1[c] / (rij * rjk) - scp * d2[c] / r2jk);
      D(i, c) += dv * di;
      D(k, c) += dv * dk;
      D(j, c) -= dv * (di + dk);
    }
    rst_energy(st, ipsi, e);
  }
  for (int r = 0; r < s->nrstr_wall; r++) {
    double fk = s->rwal_fk[r];
    for (int i = s->rwal_i[r]; i <= s->rwal_j[r]; i++) {
      if (!(s->heavy[i] || s->rwal_ih[r] == 1)) continue;
      double dr[3] = {X(i, 0) - s->xwcent[0], X(i, 1) - s->xwcent[1], X(i, 2) - s->xwcent[2]};
      double b = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
      double db = b - s->rwal_d[r], e, dv;
      if (db > 0.) { e = 0.5 * fk * db * db - s->rwal_dMorse[r]; dv = fk * db / b; }
      else {
        double fexp = exp(s->rwal_aMorse[r] * db);
        e = s->rwal_dMorse[r] * (fexp * fexp - 2. * fexp);
        dv = -2. * s->rwal_dMorse[r] * s->rwal_aMorse[r] * (fexp - fexp * fexp) / b;
      }
      st->E[QB_E_RST_PROTEIN] += e;
      for (int k = 0; k < 3; k++) D(i, k) += dv * dr[k];
    }
  }
}

/* restrain_solvent (md.f90:14910) */
static void restrain_solvent(qo_state *st) {
  const qb_sysview *s = st->s;
  double shift = s->fk_wsphere != 0. ? sqrt((double)kBoltz * st->Tfree / s->fk_wsphere) : 0.;
  for (int g = s->ncgp_solute; g < s->ncgp; g++) {
    int i = s->cgp_iswitch[g];
    if (s->excl[i]) continue;
    double dr[3] = {X(i, 0) - s->xwcent[0], X(i, 1) - s->xwcent[1], X(i, 2) - s->xwcent[2]};
    double b = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    double db = b - (s->rwat - shift), e, dv;
    if (db > 0) { e = 0.5 * s->fk_wsphere * db * db - s->Dwmz; dv = s->fk_wsphere * db / b; }
    else if (b > 0.0) {
      double fexp = exp(s->awmz * db);
      e = s->Dwmz * (fexp * fexp - 2. * fexp);
      dv = -2. * s->Dwmz * s->awmz * (fexp - fexp * fexp) / b;
    } else { dv = 0; e = 0; }
    st->E[QB_E_RST_SOLVENT_RADIAL] += e;
    for (int k = 0; k < 3; k++) D(i, k) += dv * dr[k];
  }
}

/* watpol (md.f90:15122) */
static void watpol(qo_state *st) {
  const qb_sysview *s = st->s;
  const int ns = s->nwpolr_shell, nw = st->nwat;
  const double pi = fpi();
  if (ns == 0) return;
  for (int is = 0; is < ns; is++) st->n_insh[is] = 0;
  for (int iw = 0; iw < nw; iw++) {
    st->theta[iw] = 0.0;
    st->theta0[iw] = 0.0;
    int i = st->NS + 3 * iw;
    if (s->excl[i]) continue;
    double rmu[3], rcu[3];
    for (int k = 0; k < 3; k++) rmu[k] = X(i + 1, k) + X(i + 2, k) - 2. * X(i, k);
    double rm = sqrt(rmu[0] * rmu[0] + rmu[1] * rmu[1] + rmu[2] * rmu[2]);
    for (int k = 0; k < 3; k++) rmu[k] /= rm;
    for (int k = 0; k < 3; k++) rcu[k] = X(i, k) - s->xwcent[k];
    double rc = sqrt(rcu[0] * rcu[0] + rcu[1] * rcu[1] + rcu[2] * rcu[2]);
    for (int k = 0; k < 3; k++) rcu[k] /= rc;
    double scp = rmu[0] * rcu[0] + rmu[1] * rcu[1] + rmu[2] * rcu[2];
    if (scp > 1.0) scp = 1.0;
    if (scp < -1.0) scp = -1.0;
    st->theta[iw] = acos(scp);
    st->tdum[iw] = st->theta[iw];
    float inner = s->wshell_rout[ns - 1] - s->wshell_dr[ns - 1];
    if (rc > (double)inner) {
      int is;
      for (is = ns - 1; is >= 1; is--)
        if (rc <= (double)s->wshell_rout[is]) break;
      st->list_sh[is * nw + st->n_insh[is]++] = iw;
    }
  }
  for (int is = 0; is < ns; is++) {
    int n = st->n_insh[is];
    for (int il = 0; il < n; il++) {
      double tmin = 2. * pi;
      int jmin = -1;
      for (int jl = 0; jl < n; jl++) {
        int jw = st->list_sh[is * nw + jl];
        if (st->tdum[jw] < tmin) { jmin = jw; tmin = st->theta[jw]; }
      }
      st->nsort[is * nw + il] = jmin;
      st->tdum[jmin] = 99999.;
    }
  }
  if (st->istep != 0 && st->istep % 100 == 0) {
    for (int is = 0; is < ns; is++) {
      st->avtheta[is] = st->avtheta[is] / (float)100;
      st->avn_insh[is] = st->avn_insh[is] / (float)100;
      st->theta_corr[is] = st->theta_corr[is] + st->avtheta[is] - acosf(s->wshell_cstb[is]);
      st->avtheta[is] = 0.0f;
      st->avn_insh[is] = 0.0f;
    }
  }
  for (int is = 0; is < ns; is++) {
    int n = st->n_insh[is];
    if (n == 0) continue;
    double avtdum = 0.0;
    for (int il = 0; il < n; il++) {
      int iw = st->nsort[is * nw + il];
      float arg = 1.0f + (1.0f - 2.0f * (float)(il + 1)) / (float)n;
      double th0 = (double)acosf(arg);
      th0 = th0 - 3. * sin(th0) * (double)s->wshell_cstb[is] / 2.;
      if (th0 < 0.0) th0 = 0.0;
      if (th0 > pi) th0 = pi;
      st->theta0[il] = th0;
      avtdum += st->theta[iw];
      double dth = st->theta[iw] - th0 + (double)st->theta_corr[is];
      st->E[QB_E_RST_WATER_POL] += 0.5 * s->fkwpol * dth * dth;
      double dv = s->fkwpol * dth;
      int i = st->NS + 3 * iw;
      double rmu[3], rcu[3];
      for (int k = 0; k < 3; k++) rmu[k] = X(i + 1, k) + X(i + 2, k) - 2. * X(i, k);
      double rm = sqrt(rmu[0] * rmu[0] + rmu[1] * rmu[1] + rmu[2] * rmu[2]);
      for (int k = 0; k < 3; k++) rmu[k] /= rm;
      for (int k = 0; k < 3; k++) rcu[k] = X(i, k) - s->xwcent[k];
      double rc = sqrt(rcu[0] * rcu[0] + rcu[1] * rcu[1] + rcu[2] * rcu[2]);
      for (int k = 0; k < 3; k++) rcu[k] /= rc;
      double scp = rmu[0] * rcu[0] + rmu[1] * rcu[1] + rmu[2] * rcu[2];
      if (scp > 1.0) scp = 1.0;
      if (scp < -1.0) scp = -1.0;
      double f0 = sin(acos(scp));
      if (fabs(f0) < 1.e-12) f0 = 1.e-12;
      f0 = -1.0 / f0;
      f0 = dv * f0;
      for (int k = 0; k < 3; k++) {
        double f1 = (rcu[k] - rmu[k] * scp) / rm;
        double f2 = (rmu[k] - rcu[k] * scp) / rc;
        D(i, k) += f0 * (-2. * f1 + f2);
        D(i + 1, k) += f0 * f1;
        D(i + 2, k) += f0 * f1;
      }
    }
    st->avtheta[is] = (float)((double)st->avtheta[is] + avtdum / (double)(float)n);
    st->avn_insh[is] = st->avn_insh[is] + (float)n;
  }
}

/* ---------------------------------------------------------- pot_energy */

/* pot_energy (md.f90:13278) */
static void pot_energy(qo_state *st) {
  const qb_sysview *s = st->s;
  memset(st->E, 0, sizeof st->E);
  st->E[QB_E_KINETIC] = st->kinetic;
  for (int k = 0; k < st->S; k++) {
    double lam = s->lambda[k];
    memset(&st->EQ[k * QB_NEQ], 0, QB_NEQ * sizeof(double));
    EQV(k, QB_EQ_LAMBDA) = lam;
  }
  memset(st->d, 0, 3 * (size_t)st->N * sizeof(double));
  nonbond_pp(st);
  nonbond_pw(st);
  nonbond_qp(st);
  if (st->N > st->NS) {
    nonbond_ww(st);
    nonbond_qw(st);
  }
  if (s->use_LRF) lrf_taylor(st);
  st->E[QB_E_P_BOND] = bonds(st, 0, s->nbonds_solute);
  st->E[QB_E_W_BOND] = bonds(st, s->nbonds_solute, s->nbonds);
  st->E[QB_E_P_ANGLE] = angles(st, 0, s->nangles_solute);
  st->E[QB_E_W_ANGLE] = angles(st, s->nangles_solute, s->nangles);
  if (s->ff_type == 3) {
    st->E[QB_E_P_ANGLE] += urey_bradley(st, 0, s->nangles_solute);
    st->E[QB_E_W_ANGLE] += urey_bradley(st, s->nangles_solute, s->nangles);
  }
  st->E[QB_E_P_TORSION] = torsions(st, 0, s->ntors_solute);
  st->E[QB_E_W_TORSION] = torsions(st, s->ntors_solute, s->ntors);
  st->E[QB_E_P_IMPROPER] = impropers(st, 0, s->nimps_solute);
  st->E[QB_E_W_IMPROPER] = impropers(st, s->nimps_solute, s->nimps);
  /* the sphere's restraints (none in a periodic box, md.f90:13345-13356) */
  if (!s->use_pbc) fix_shell(st);
  p_restrain(st);
  if (st->nwat > 0 && !s->use_pbc) {
    restrain_solvent(st);
    if (s->wpol_restr) watpol(st);
  }
  nonbond_qq(st);
  for (int k = 0; k < st->S; k++) qbonded(st, k);
  for (int k = 0; k < st->S; k++) {
    double lam = s->lambda[k];
    EQV(k, QB_EQ_QX_EL) = EQV(k, QB_EQ_QQ_EL) + EQV(k, QB_EQ_QP_EL) + EQV(k, QB_EQ_QW_EL);
    EQV(k, QB_EQ_QX_VDW) = EQV(k, QB_EQ_QQ_VDW) + EQV(k, QB_EQ_QP_VDW) + EQV(k, QB_EQ_QW_VDW);
    EQV(k, QB_EQ_TOTAL) = EQV(k, QB_EQ_BOND) + EQV(k, QB_EQ_ANGLE) + EQV(k, QB_EQ_TORSION) + EQV(k, QB_EQ_IMPROPER) +
                          EQV(k, QB_EQ_QX_EL) + EQV(k, QB_EQ_QX_VDW) + EQV(k, QB_EQ_RESTRAINT);
    st->E[QB_E_Q_BOND] += EQV(k, QB_EQ_BOND) * lam;
    st->E[QB_E_Q_ANGLE] += EQV(k, QB_EQ_ANGLE) * lam;
    st->E[QB_E_Q_TORSION] += EQV(k, QB_EQ_TORSION) * lam;
    st->E[QB_E_Q_IMPROPER] += EQV(k, QB_EQ_IMPROPER) * lam;
    st->E[QB_E_QX_EL] += EQV(k, QB_EQ_QX_EL) * lam;
    st->E[QB_E_QX_VDW] += EQV(k, QB_EQ_QX_VDW) * lam;
    st->E[QB_E_RST_PROTEIN] += EQV(k, QB_EQ_RESTRAINT) * lam;
  }
  double *E = st->E;
  E[QB_E_RST_TOTAL] = E[QB_E_RST_FIX] + E[QB_E_RST_SHELL] + E[QB_E_RST_PROTEIN] + E[QB_E_RST_SOLVENT_RADIAL] +
                      E[QB_E_RST_WATER_POL];
  E[QB_E_POTENTIAL] = E[QB_E_P_BOND] + E[QB_E_W_BOND] + E[QB_E_P_ANGLE] + E[QB_E_W_ANGLE] + E[QB_E_P_TORSION] +
                      E[QB_E_P_IMPROPER] + E[QB_E_PP_EL] + E[QB_E_PP_VDW] + E[QB_E_PW_EL] + E[QB_E_PW_VDW] +
                      E[QB_E_WW_EL] + E[QB_E_WW_VDW] + E[QB_E_Q_BOND] + E[QB_E_Q_ANGLE] + E[QB_E_Q_TORSION] +
                      E[QB_E_Q_IMPROPER] + E[QB_E_QX_EL] + E[QB_E_QX_VDW] + E[QB_E_RST_TOTAL] + E[QB_E_LRF];
}

/* ------------------------------------------------------------ dynamics */

/* temperature (md.f90:3813) */
static void temperature(qo_state *st) {
  const qb_sysview *s = st->s;
  double Tsolute = 0, Tfree_solute = 0, Tsolvent = 0, Tfree_solvent = 0;
  for (int i = 0; i < st->N; i++) {
    double e = 0.5 * s->mass[i] *
               (st->v[3 * i] * st->v[3 * i] + st->v[3 * i + 1] * st->v[3 * i + 1] + st->v[3 * i + 2] * st->v[3 * i + 2]);
    if (i < st->NS) { Tsolute += e; if (!s->excl[i]) Tfree_solute += e; }
    else { Tsolvent += e; if (!s->excl[i]) Tfree_solvent += e; }
  }
  double Tfree = Tfree_solvent + Tfree_solute;
  double Temp = Tsolute + Tsolvent;
  st->kinetic = Temp;
  const double kb = (double)kBoltz;
  Temp = 2.0 * Temp / kb / (double)(float)s->Ndegf;
  Tfree = 2.0 * Tfree / kb / (double)(float)s->Ndegfree;
  st->Temp_solute = Tsolute;
  st->Temp_solvent = Tsolvent;
  st->Tfree_solute = Tfree_solute;
  st->Tfree_solvent = Tfree_solvent;
  if (s->detail_temps) {
    st->Tfree_solute = 2.0 * Tfree_solute / kb / (double)(float)s->Ndegfree_solute;
    st->Tfree_solvent = 2.0 * Tfree_solvent / kb / (double)(float)s->Ndegfree_solvent;
  }
  if (s->separate_scaling) {
    if (st->Tfree_solvent != 0) st->Tscale_solvent = s->Temp0 / st->Tfree_solvent - 1.0;
    st->Tscale_solvent = sqrt(1 + s->dt / s->tau_T * st->Tscale_solvent);
    if (st->Tfree_solute != 0) st->Tscale_solute = s->Temp0 / st->Tfree_solute - 1.0;
    st->Tscale_solute = sqrt(1 + s->dt / s->tau_T * st->Tscale_solute);
  } else {
    if (Tfree != 0) st->Tscale_solvent = s->Temp0 / Tfree - 1.0;
    st->Tscale_solvent = sqrt(1 + s->dt / s->tau_T * st->Tscale_solvent);
    st->Tscale_solute = st->Tscale_solvent;
  }
  st->Temp = Temp;
  st->Tfree = Tfree;
}

/* shake (md.f90:14445): Gauss-Seidel per molecule */
static int shake(qo_state *st, const double *xx, double *x) {
  const qb_sysview *s = st->s;
  for (int m = 0; m < s->shake_molecules; m++) {
    int f = s->shake_mol_first[m], n = s->shake_mol_n[m];
    char ready[4096];
    char *rd = n <= 4096 ? ready : (char *)malloc(n);
    memset(rd, 0, n);
    int nits = 0;
    for (;;) {
      for (int c = 0; c < n; c++) {
        if (rd[c]) continue;
        int i = s->shake_i[f + c], j = s->shake_j[f + c];
        double xij[3], xxij[3];
        for (int k = 0; k < 3; k++) xij[k] = x[3 * i + k] - x[3 * j + k];
        double xij2 = xij[0] * xij[0] + xij[1] * xij[1] + xij[2] * xij[2];
        double d2 = s->shake_dist2[f + c];
        double diff = d2 - xij2;
        if (fabs(diff) < 0.0001 * d2) rd[c] = 1;
        for (int k = 0; k < 3; k++) xxij[k] = xx[3 * i + k] - xx[3 * j + k];
        double scp = xij[0] * xxij[0] + xij[1] * xxij[1] + xij[2] * xxij[2];
        float wsum = s->winv[i] + s->winv[j];
        double corr = diff / (2. * scp * (double)wsum);
        for (int k = 0; k < 3; k++) {
          x[3 * i + k] += xxij[k] * corr * (double)s->winv[i];
          x[3 * j + k] -= xxij[k] * corr * (double)s->winv[j];
        }
      }
      nits++;
      int all = 1;
      for (int c = 0; c < n; c++) all &= rd[c];
      if (all) break;
      if (nits >= 1000) {
        if (rd != ready) free(rd);
        return -1;
      }
    }
    if (rd != ready) free(rd);
  }
  return 0;
}

/* offdiag (md.f90:12911): distance of each off-diagonal function's Q atoms */
static void offdiag(qo_state *st) {
  const qb_sysview *s = st->s;
  for (int io = 0; io < s->noffd; io++) {
    int k = s->iqseq[s->offd_k[io]], l = s->iqseq[s->offd_l[io]];
    st->offd_r[io] = sqrt((X(l, 0) - X(k, 0)) * (X(l, 0) - X(k, 0)) + (X(l, 1) - X(k, 1)) * (X(l, 1) - X(k, 1)) +
                          (X(l, 2) - X(k, 2)) * (X(l, 2) - X(k, 2)));
  }
}

static void record(qo_state *st, int kind) {
  int S = st->S;
  int c = st->hcount[kind];
  if (c >= st->hcap) return;
  memcpy(&st->hR[kind][(size_t)c * QB_MAX_STATES], st->offd_r, QB_MAX_STATES * sizeof(double));
  st->hstep[kind][c] = st->istep;
  memcpy(&st->hE[kind][(size_t)c * QB_NE], st->E, QB_NE * sizeof(double));
  memcpy(&st->hEQ[kind][(size_t)c * S * QB_NEQ], st->EQ, (size_t)S * QB_NEQ * sizeof(double));
  st->hcount[kind]++;
}

/* ---------------------------------------------------------- periodic box */

/* randm (md.f90:14408-14442): one sequence, seeded by the first call */
static double randm(qo_state *st, int seed) {
  const int m = 100000000, m1 = 10000, mult = 31415821;
  if (!st->rand_started) { st->rand_started = 1; st->irand = abs(seed) % m; }
  int ih = st->irand / m1, il = st->irand % m1;
  int r = ((ih * (mult % m1) + il * (mult / m1)) % m1) * m1 + il * (mult % m1);
  r = (r + 1) % m;
  st->irand = r;
  float v = (float)(r / 10) * 10.0f / (float)m;
  if (v <= 0.0f || v > 1.0f) v = 0.0f;
  return (double)v;
}

/* put_back_in_box (md.f90:15477-15600) */
static void put_back_in_box(qo_state *st) {
  const qb_sysview *s = st->s;
  int nmol = s->nmol;
  if (!s->rigid_box_center) {
    int n = st->NS > 0 ? st->NS : st->N;
    double c[3] = {0, 0, 0};
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) c[k] += X(i, k);
    for (int k = 0; k < 3; k++) st->boxc[k] = c[k] / n;
  }
  int first = 0, last = nmol;
  if (nmol > 1) {
    int nsolv = (st->N - st->NS) / (s->istart_mol[nmol - 1] - s->istart_mol[nmol - 2]);
    if (!s->put_solute_back_in_box) first = nmol - nsolv;
    if (!s->put_solvent_back_in_box) last = nmol - nsolv;
  }
  for (int m = first; m < last; m++) {
    double cm[3] = {0, 0, 0};
    for (int j = s->istart_mol[m]; j < s->istart_mol[m + 1]; j++)
      for (int k = 0; k < 3; k++) cm[k] += X(j, k) * s->mass_box[j];
    for (int k = 0; k < 3; k++) {
      cm[k] = cm[k] * s->mol_mass_inv[m];
      double hi = st->boxc[k] + st->boxl[k] / 2, lo = st->boxc[k] - st->boxl[k] / 2, sh = 0.0;
      if (cm[k] > hi) sh = -st->boxl[k];
      else if (cm[k] < lo) sh = st->boxl[k];
      if (sh != 0.0)
        for (int j = s->istart_mol[m]; j < s->istart_mol[m + 1]; j++) X(j, k) += sh;
    }
  }
}

/* new_potential (md.f90:15846-15972): the nonbonded, restraint, LRF and Q-Q
 * terms at the current coordinates; the bonded terms of the total come from
 * `old` */
static void new_potential(qo_state *st, const double *old) {
  const qb_sysview *s = st->s;
  double *E = st->E;
  int zero[] = {QB_E_POTENTIAL, QB_E_PP_EL, QB_E_PP_VDW, QB_E_PW_EL, QB_E_PW_VDW, QB_E_WW_EL, QB_E_WW_VDW,
                QB_E_QX_EL, QB_E_QX_VDW, QB_E_RST_PROTEIN, QB_E_LRF};
  for (size_t k = 0; k < sizeof zero / sizeof zero[0]; k++) E[zero[k]] = 0.0;
  int zq[] = {QB_EQ_QQ_EL, QB_EQ_QQ_VDW, QB_EQ_QP_EL, QB_EQ_QP_VDW, QB_EQ_QW_EL, QB_EQ_QW_VDW, QB_EQ_RESTRAINT};
  for (int k = 0; k < st->S; k++)
    for (size_t c = 0; c < sizeof zq / sizeof zq[0]; c++) EQV(k, zq[c]) = 0.0;
  memset(st->d, 0, 3 * (size_t)st->N * sizeof(double));
  nonbond_pp(st);
  nonbond_pw(st);
  nonbond_qp(st);
  if (st->N > st->NS) {
    nonbond_ww(st);
    nonbond_qw(st);
  }
  if (s->use_LRF) lrf_taylor(st);
  p_restrain(st);
  nonbond_qq(st);
  for (int k = 0; k < st->S; k++) {
    double lam = s->lambda[k];
    EQV(k, QB_EQ_QX_EL) = EQV(k, QB_EQ_QQ_EL) + EQV(k, QB_EQ_QP_EL) + EQV(k, QB_EQ_QW_EL);
    EQV(k, QB_EQ_QX_VDW) = EQV(k, QB_EQ_QQ_VDW) + EQV(k, QB_EQ_QP_VDW) + EQV(k, QB_EQ_QW_VDW);
    E[QB_E_QX_EL] += EQV(k, QB_EQ_QX_EL) * lam;
    E[QB_E_QX_VDW] += EQV(k, QB_EQ_QX_VDW) * lam;
    E[QB_E_RST_PROTEIN] += EQV(k, QB_EQ_RESTRAINT) * lam;
  }
  E[QB_E_POTENTIAL] = old[QB_E_P_BOND] + old[QB_E_W_BOND] + old[QB_E_P_ANGLE] + old[QB_E_W_ANGLE] +
                      old[QB_E_P_TORSION] + old[QB_E_P_IMPROPER] + E[QB_E_PP_EL] + E[QB_E_PP_VDW] + E[QB_E_PW_EL] +
                      E[QB_E_PW_VDW] + E[QB_E_WW_EL] + E[QB_E_WW_VDW] + old[QB_E_Q_BOND] + old[QB_E_Q_ANGLE] +
                      old[QB_E_Q_TORSION] + old[QB_E_Q_IMPROPER] + E[QB_E_QX_EL] + E[QB_E_QX_VDW] +
                      E[QB_E_RST_PROTEIN] + E[QB_E_LRF];
}

/* MC_volume (md.f90:15615-15840): returns 0, or 10 (QB_ERR_STATE) when the
 * new box is too small for a cut-off (the reference dies) */
static int mc_volume(qo_state *st) {
  const qb_sysview *s = st->s;
  size_t n3 = 3 * (size_t)st->N;
  double *old_x = (double *)malloc(n3 * sizeof(double));
  lrf_t *old_lrf = NULL;
  double old_E[QB_NE], old_EQ[QB_MAX_STATES * QB_NEQ], old_boxl[3], old_inv[3];
  memcpy(old_x, st->x, n3 * sizeof(double));
  memcpy(old_E, st->E, sizeof old_E);
  memcpy(old_boxl, st->boxl, sizeof old_boxl);
  memcpy(old_inv, st->iboxl, sizeof old_inv);
  if (s->use_LRF) {
    old_lrf = (lrf_t *)malloc(((size_t)s->ncgp + 1) * sizeof(lrf_t));
    memcpy(old_lrf, st->lrf, (size_t)s->ncgp * sizeof(lrf_t));
  }
  new_potential(st, old_E);
  memcpy(old_E, st->E, sizeof old_E);
  memcpy(old_EQ, st->EQ, sizeof old_EQ);
  double old_V = old_boxl[0] * old_boxl[1] * old_boxl[2];
  double r = randm(st, s->pressure_seed);
  r = r * 2 - 1;
  double deltaV = r * s->max_vol_displ, new_V = deltaV + old_V;
  double ratio = pow(new_V / old_V, (double)(1.0f / 3.0f));
  for (int k = 0; k < 3; k++) { st->boxl[k] = st->boxl[k] * ratio; st->iboxl[k] = 1.0 / st->boxl[k]; }
  double bmin = fmin(st->boxl[0], fmin(st->boxl[1], st->boxl[2]));
  if (!(bmin > s->Rcpp * 2) || !(bmin > s->Rcww * 2) || !(bmin > s->Rcpw * 2) || !(bmin > s->Rcq * 2) ||
      !(bmin > s->RcLRF * 2)) {
    free(old_x); free(old_lrf);
    return 10;
  }
  for (int m = 0; m < s->nmol; m++) {
    double cm[3] = {0, 0, 0}, mv[3];
    for (int j = s->istart_mol[m]; j < s->istart_mol[m + 1]; j++)
      for (int k = 0; k < 3; k++) cm[k] += X(j, k) * s->mass_box[j];
    for (int k = 0; k < 3; k++) {
      cm[k] = cm[k] * s->mol_mass_inv[m];
      mv[k] = ((cm[k] - st->boxc[k]) * st->boxl[k] / old_boxl[k] + st->boxc[k]) - cm[k];
    }
    for (int j = s->istart_mol[m]; j < s->istart_mol[m + 1]; j++)
      for (int k = 0; k < 3; k++) X(j, k) += mv[k];
  }
  if (s->use_LRF) {
    cgp_centers(st);
    list_pp(st);
    list_pw(st);
    list_ww(st);
  }
  new_potential(st, old_E);
  double deltaE = st->E[QB_E_POTENTIAL] - old_E[QB_E_POTENTIAL];
  double deltaW = deltaE + s->pressure * deltaV - (double)((float)s->nmol * kBoltz) * s->Temp0 * log(new_V / old_V);
  int acc = 1;
  if (deltaW > 0.0) {
    double u = randm(st, s->pressure_seed);
    acc = !(u > exp(-deltaW / (double)kBoltz / s->Temp0));
  }
  st->vol_tries++;
  if (acc) {
    st->vol_acc++;
  } else {
    memcpy(st->x, old_x, n3 * sizeof(double));
    memcpy(st->E, old_E, sizeof old_E);
    memcpy(st->EQ, old_EQ, (size_t)st->S * QB_NEQ * sizeof(double));
    memcpy(st->boxl, old_boxl, sizeof old_boxl);
    memcpy(st->iboxl, old_inv, sizeof old_inv);
    if (s->use_LRF) memcpy(st->lrf, old_lrf, (size_t)s->ncgp * sizeof(lrf_t));
  }
  free(old_x);
  free(old_lrf);
  return 0;
}

/* ------------------------------------------------------------- public */

qo_state *qo_create(const qb_sysview *s, int history_capacity) {
  qo_state *st = (qo_state *)calloc(1, sizeof *st);
  st->s = s;
  st->N = s->natom;
  st->NS = s->nat_solute;
  st->nwat = s->nwat;
  st->S = s->nstates;
  st->nq = s->nqat;
  size_t n3 = 3 * (size_t)st->N;
  st->x = (double *)malloc(n3 * sizeof(double));
  st->v = (double *)malloc(n3 * sizeof(double));
  st->d = (double *)calloc(n3, sizeof(double));
  st->xx = (double *)malloc(n3 * sizeof(double));
  memcpy(st->x, s->x0, n3 * sizeof(double));
  memcpy(st->v, s->v0, n3 * sizeof(double));
  st->qw = (int *)malloc(((size_t)st->nwat + 1) * sizeof(int));
  st->lrf = (lrf_t *)calloc((size_t)s->ncgp + 1, sizeof(lrf_t));
  int ns = s->nwpolr_shell;
  st->theta_corr = (float *)calloc(ns + 1, sizeof(float));
  st->avtheta = (float *)calloc(ns + 1, sizeof(float));
  st->avn_insh = (float *)calloc(ns + 1, sizeof(float));
  for (int k = 0; k < ns; k++) st->theta_corr[k] = s->wshell_theta_corr0[k];
  st->n_insh = (int *)calloc(ns + 1, sizeof(int));
  st->list_sh = (int *)malloc(((size_t)ns * st->nwat + 1) * sizeof(int));
  st->nsort = (int *)malloc(((size_t)ns * st->nwat + 1) * sizeof(int));
  st->theta = (double *)calloc((size_t)st->nwat + 1, sizeof(double));
  st->theta0 = (double *)calloc((size_t)st->nwat + 1, sizeof(double));
  st->tdum = (double *)calloc((size_t)st->nwat + 1, sizeof(double));
  st->hcap = history_capacity;
  for (int k = 0; k < 2; k++) {
    st->hstep[k] = (int *)malloc((size_t)(history_capacity + 1) * sizeof(int));
    st->hE[k] = (double *)malloc((size_t)(history_capacity + 1) * QB_NE * sizeof(double));
    st->hEQ[k] = (double *)malloc((size_t)(history_capacity + 1) * (st->S + 1) * QB_NEQ * sizeof(double));
    st->hR[k] = (double *)calloc((size_t)(history_capacity + 1) * QB_MAX_STATES, sizeof(double));
  }
  if (s->use_pbc)
    for (int k = 0; k < 3; k++) {
      st->boxl[k] = s->boxlength[k];
      st->iboxl[k] = 1.0 / s->boxlength[k];
      st->boxc[k] = s->boxcenter[k];
    }
  st->rand_started = s->randm_started;
  st->irand = s->randm_state;
  /* md_run start: initial temperature (md.f90:3960-3963) */
  st->Tscale_solute = st->Tscale_solvent = 1.0;
  temperature(st);
  st->E[QB_E_KINETIC] = st->kinetic;
  return st;
}

void qo_destroy(qo_state *st) {
  if (!st) return;
  free(st->x); free(st->v); free(st->d); free(st->xx);
  free(st->pp); free(st->pw); free(st->ww); free(st->qp); free(st->qw); free(st->lrf);
  free(st->theta_corr); free(st->avtheta); free(st->avn_insh); free(st->n_insh);
  free(st->list_sh); free(st->nsort); free(st->theta); free(st->theta0); free(st->tdum);
  for (int k = 0; k < 2; k++) { free(st->hstep[k]); free(st->hE[k]); free(st->hEQ[k]); free(st->hR[k]); }
  free(st);
}

/* one pass of the md_run loop body (md.f90:4003-4175) */
int qo_run(qo_state *st, int nsteps) {
  const qb_sysview *s = st->s;
  const double dt = s->dt;
  for (int n = 0; n < nsteps; n++) {
    if (st->istep % s->NBcycle == 0) {
      if (s->use_pbc && (s->put_solute_back_in_box || s->put_solvent_back_in_box)) put_back_in_box(st);
      make_pair_lists(st);
    }
    pot_energy(st);
    if (s->noffd > 0) offdiag(st);
    st->E[QB_E_KINETIC] = st->kinetic;
    for (int i = 0; i < st->N; i++) {
      double ts = i < st->NS ? st->Tscale_solute : st->Tscale_solvent;
      double w = (double)s->winv[i];
      for (int k = 0; k < 3; k++) {
        int a = 3 * i + k;
        st->v[a] = (st->v[a] - st->d[a] * w * dt) * ts;
        st->xx[a] = st->x[a];
        st->x[a] = st->x[a] + st->v[a] * dt;
      }
    }
    if (s->shake_constraints > 0) {
      if (shake(st, st->xx, st->x) != 0) { st->status = 5; return 5; }
      for (int a = 0; a < 3 * st->N; a++) st->v[a] = (st->x[a] - st->xx[a]) / dt;
    }
    temperature(st);
    st->E[QB_E_KINETIC] = st->kinetic;
    /* constant pressure: a volume move before the step's output (md.f90:4137-4141) */
    if (s->use_pbc && s->constant_pressure && st->istep % s->ivolume_cycle == 0 && st->istep > 0)
      if (mc_volume(st) != 0) { st->status = 10; return 10; }
    if (st->istep % s->iene_cycle == 0 && st->istep > 0) record(st, 1);
    if (st->istep % s->iout_cycle == 0) record(st, 0);
    st->istep++;
  }
  return 0;
}

/* make_pair_lists + pot_energy after the loop (md.f90:4186-4188) */
int qo_final_energy(qo_state *st) {
  make_pair_lists(st);
  pot_energy(st);
  st->E[QB_E_KINETIC] = st->kinetic;
  return 0;
}

void qo_energies(const qo_state *st, double *E, double *EQ) {
  memcpy(E, st->E, QB_NE * sizeof(double));
  if (EQ) memcpy(EQ, st->EQ, (size_t)st->S * QB_NEQ * sizeof(double));
}
void qo_gradient(const qo_state *st, double *d) { memcpy(d, st->d, 3 * (size_t)st->N * sizeof(double)); }
void qo_coords(const qo_state *st, double *x) { memcpy(x, st->x, 3 * (size_t)st->N * sizeof(double)); }
void qo_velocities(const qo_state *st, double *v) { memcpy(v, st->v, 3 * (size_t)st->N * sizeof(double)); }
void qo_set_coords(qo_state *st, const double *x) { memcpy(st->x, x, 3 * (size_t)st->N * sizeof(double)); }
void qo_set_velocities(qo_state *st, const double *v) { memcpy(st->v, v, 3 * (size_t)st->N * sizeof(double)); }
void qo_theta_corr(const qo_state *st, float *tc) {
  memcpy(tc, st->theta_corr, (size_t)st->s->nwpolr_shell * sizeof(float));
}
void qo_temperature(const qo_state *st, double *out) {
  out[0] = st->Temp; out[1] = st->Tfree; out[2] = st->Tfree_solute; out[3] = st->Tfree_solvent;
  out[4] = st->Tscale_solvent;
}
int qo_history(const qo_state *st, int kind, int *steps, double *E, double *EQ) {
  int c = st->hcount[kind];
  if (steps) memcpy(steps, st->hstep[kind], (size_t)c * sizeof(int));
  if (E) memcpy(E, st->hE[kind], (size_t)c * QB_NE * sizeof(double));
  if (EQ) memcpy(EQ, st->hEQ[kind], (size_t)c * st->S * QB_NEQ * sizeof(double));
  return c;
}
/* r_kl of every record's off-diagonal functions: count*noffd doubles */
int qo_offdiag(const qo_state *st, int kind, double *rkl) {
  int c = st->hcount[kind], n = st->s->noffd;
  for (int r = 0; r < c; r++)
    for (int io = 0; io < n; io++) rkl[(size_t)r * n + io] = st->hR[kind][(size_t)r * QB_MAX_STATES + io];
  return c;
}
/* pair counts of the current lists: pp, pw, ww molecule pairs, qp, qw waters */
void qo_list_counts(const qo_state *st, int *out) {
  out[0] = st->npp; out[1] = st->npw; out[2] = st->nww - st->nwat; out[3] = st->nqp; out[4] = st->nqw;
}
int qo_status(const qo_state *st) { return st->status; }

void qo_box(const qo_state *st, double *box6) {
  for (int k = 0; k < 3; k++) { box6[k] = st->boxl[k]; box6[3 + k] = st->boxc[k]; }
}
void qo_volume_moves(const qo_state *st, long long *tries, long long *accepted) {
  *tries = st->vol_tries;
  *accepted = st->vol_acc;
}
