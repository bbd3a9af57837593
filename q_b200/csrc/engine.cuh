// engine.cuh -- device-side data layout of a batch of Q systems.
//
// All systems of a batch live in one set of device arrays, concatenated; a
// per-system SysDev record holds each system's offsets and scalar parameters.
// Global indices: atoms g = aoff + i, waters gw = woff + iw (O atom
// aoff + nsol + 3*iw), charge groups gc = coff + ig, Q atoms gq = qoff + iq.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "qb.h"
#include "ljrule.hpp"

namespace qb {

constexpr int MAXS = QB_MAX_STATES;
// LRF record of a charge group: centre[3], phi0, phi1[3], the 6 distinct
// components of the symmetric phi2 (xx,xy,xz,yy,yz,zz) and the 10 of phi3
// (xxx,xxy,xxz,xyy,xyz,xzz,yyy,yyz,yzz,zzz), and the group's radius (largest
// distance of a member atom from the centre).
constexpr int LRF_STRIDE = 24;
constexpr int MAX_SHELLS = 4;
// one history record: step, E[QB_NE], EQ[MAXS*QB_NEQ], r_kl of the off-diagonal functions [MAXS]
constexpr int HIST_REC = 1 + QB_NE + MAXS * QB_NEQ + MAXS;
constexpr int NQ_SHARED = 64;    // Q atoms whose water forces are reduced in shared memory
// F_SHAKE: in a SHAKE constraint; F_SH3: in a 3-constraint molecule, moved by k_leapfrog_shake3
enum AtomFlags : uint8_t { F_EXCL = 1, F_SHELL = 2, F_HEAVY = 4, F_SHAKE = 8, F_SH3 = 16 };

// A non-Q atom of a solute charge group with its interaction parameters for
// the water O and H sites: LJ products A(O), B(O), A(H), B(H) and single
// precision charge products q(O), q(H).
struct PwAtom {
  double4 lj;
  float2 q;
  int atom, pad;
};

// Per-system record (read-only on the device during a run).
struct SysDev {
  int aoff, natom, nsol, nwat, woff, coff, ncgp, ncgp_sol;
  int qoff, nq, S, natyps, ljoff, qlib_off, sc_off, qconn_off;
  int lrft_off, nlrft;        // LRF gather tiles (group ranges)
  // static term ranges (global offsets into term arrays)
  int b_off, nb, nb_sol, a_off, na, na_sol, t_off, nt, nt_sol, i_off, ni, ni_sol;
  int qb_off, nqb, qa_off, nqa, qt_off, nqt, qi_off, nqi;
  int noffd, offd_k[MAXS], offd_l[MAXS];   // off-diagonal functions: their Q atoms (batch atom index)
  int qq_off, nqq;            // flattened nbqq entries of all states
  int sh_off, nsh;            // shake molecules
  int rs_off, nrs, rp_off, nrp, rd_off, nrd, ra_off, nra, rw_off, nrw;
  // dynamic list segments
  int pp_off, pp_cap, qp_off, qp_cap, qw_off, qw_cap;
  int csoff;                  // first solute group of this system among all systems' solute groups
  int ff_type, use_lrf, qvdw, wpol, nshell, iac_ow, separate_scaling, has_shake, detail_temps;
  int qp_once;                // lists with Q atoms are built once (Rcq > exclusion radius)
  int qq_lib;                 // Q-Q pairs take the topology charges
  int iout, iene, NB;
  int Ndegf, Ndegfree, Ndegfree_sol, Ndegfree_solv;
  double dt, Temp0, tau_T, el14, A_OO, B_OO;
  double Rcpp2, Rcpw2, Rcww2, Rcq2, RcLRF2;
  float crg_ow, crg_hw;
  double xp[3], xw[3], rwat, fk_ws, Dwmz, awmz, fkwpol, fk_pshell, fk_fix;
  float ws_rout[MAX_SHELLS], ws_dr[MAX_SHELLS], ws_cstb[MAX_SHELLS];
  double lambda[MAXS];
  double aO[2], bO[2];
  // water hydrogens with LJ (arithmetic rule, 3-atom solvent): O-H and H-H
  // products for water-water, the hydrogen type's columns for Q-water
  int hlj, iac_hw;
  double A_OH, B_OH, A_HH, B_HH, aH[2], bH[2];
  int arith;                       // 1: arithmetic LJ combination rule (lj_pair)
  // 1: solute charge-group cut-offs on switch atoms (nbpplist_lrf ...); 0: on
  // any atom pair (nbpplis2_lrf, nbpwlis2_lrf, nbqplis2: iuse_switch_atom 0)
  int switch_atoms;
  // periodic box (use_PBC): every pair takes the nearest image of its charge
  // groups' switching atoms; the Q-atom lists centre on atom qswitch
  int pbc, qswitch;
  int mol_off, nmol;              // molecules: P.mol_first[mol_off .. mol_off + nmol] (global atoms, + end)
  int put_first, put_last;        // molecules put back in the box, [first, last)
  int rigid_center;               // box centre fixed (rigid_box_center)
  double origin[3];               // FP32 coordinate origin of the mixed kernels (sphere: solute centre)
};

// Per-system state written by the device.
struct SysState {
  double Tscale_sol, Tscale_solv, Temp, Tfree, Tfree_sol, Tfree_solv, kinetic;
  float theta_corr[MAX_SHELLS], avtheta[MAX_SHELLS], avn_insh[MAX_SHELLS];
  int istep, status, pp_n, pw_n, qp_n, qw_n, lists_built, hist_n[2];
  // status as of the start of the current step (k_finish copies status into
  // it): the kernels that move atoms read this word, so an error raised in
  // the middle of a step takes effect for every kernel from the next step on
  int frozen;
  int shake_its_max;                 // most SHAKE iterations of one molecule since the counters were reset
  unsigned long long shake_its;      // SHAKE iterations summed over molecules and steps
  // periodic box: edge lengths, their inverses (1/L in FP64) and centre;
  // volume move in progress (mc: 1 while the trial box is evaluated) and the
  // edge lengths before it.  The last fields of the record: the host writes
  // them as one block.
  double boxl[3], iboxl[3], boxc[3];
  int mc;
  double mc_oldl[3];
};

// The energy-record buffer as the kernels see it, read through a device
// pointer so that captured graphs stay valid when the buffer grows.
struct HistRef {
  double *hist;
  int cap;
};

struct DevPtrs {
  int nsys, natoms_tot, nwat_tot, ncgp_tot, nshake_tot;
  SysDev *sys;
  SysState *st;
  // atoms
  double4 *x, *v, *xx, *d;
  float4 *wrec;              // per-water position records of the water-water kernel
  float4 *wrec32;            // their FP32 form (mixed engine): the packed and FP32 water-water kernels'
  double *wtheta;            // per water: dipole angle of the polarisation restraint
  int8_t *wshell;            // per water: polarisation shell (-1: none)
  int *wrank;                // per water: rank in its shell
  int *wshn;                 // [s*MAX_SHELLS + shell] members
  float *crg, *winv;
  double *mass;
  int *iac, *iq, *cgp, *asys;
  uint8_t *flags;
  double *lja, *ljb;        // [3*g + code-1]
  uint32_t *lx, *l14;       // exclusion / 1-4 bits per atom (solute atoms)
  // exclusion / 1-4 pairs beyond the bit range, per atom: partners (global
  // atoms, both directions) of atom g at [exo[g], exo[g+1]) and [l14o[g], l14o[g+1])
  int *exo, *exq, *l14o, *l14q;
  uint8_t *ljcod;           // per system natyps^2
  const double *xtop;       // [3*g]
  // charge groups
  int *cg_first, *cg_last, *cg_sw, *cg_atoms, *cg_sys;
  double *lrf;              // [gc*LRF_STRIDE]
  int2 *lrft;               // per system segments: [first, end) local groups of a tile
  // Q atoms
  int *iqseq;               // global atom of global Q atom
  float *qcrg;              // [gq*MAXS + st]
  int *qiac;                // [gq*MAXS + st] local Q type
  double *qavdw, *qbvdw;    // per system segments [qlib_off + 3*t + code-1]
  double *sc;               // per system segments [sc_off + (iq*(natyps+nq)+col)*S + st]
  int8_t *qconn;            // per system segments [qconn_off + (st*nsol + i)*nq + iq]
  int4 *qq;                 // (gq, gj, gjq or -1, lj | st<<8)
  double *qq_el;
  // bonded terms (global atom indices)
  int2 *bij; double2 *bpar;               // fk, b0
  int4 *aijk; double2 *apar, *aub;        // fk, th0; Urey-Bradley k, r0
  int4 *tijkl; float4 *tpar;              // fk, rmult, deltor, paths
  int4 *iijkl; float2 *ipar;              // fk, imp0
  int2 *qbij; uint8_t *qb_on; double4 *qbpar;           // [term*MAXS+st] Dmz, amz, r0, fk
  int4 *qaijk; uint8_t *qa_on; double2 *qapar, *qaub;   // fk, th0; Urey-Bradley k, r0
  // EVB Morse couplings: per Q angle (qangle's bond, qurey_bradley's bond), torsion (bond, 0),
  // improper (bond, flag) with the bond as a global Q-bond index or -1; per (term, state) the
  // state whose bond values apply
  int2 *qa_cpl, *qt_cpl, *qi_cpl;
  int8_t *qa_src, *qa_src_ub, *qt_src, *qi_src;
  int4 *qtijkl; uint8_t *qt_on; double4 *qtpar;         // fk, rmult, deltor
  int4 *qiijkl; uint8_t *qi_on; double2 *qipar;         // fk, imp0
  // shake
  int *sh_first, *sh_n, *sh_sys; int2 *sh_ij; double *sh_d2;
  int4 *sh3_at; double4 *sh3_d2; int nsh3;   // three-atom, three-constraint molecules (relabelled), system in .w
  // every other molecule (one block each): atoms, constraints in level order
  int4 *shg_info;    // atom offset, atom count, constraint offset, constraint count
  int4 *shg_info2;   // level offset, level count, system, global scratch offset (-1: shared memory)
  int *shg_at;       // global atoms of each molecule
  int2 *shg_c;       // constraints (local atom indices), level order
  double *shg_d2;
  int *shg_lev;      // level starts (level count + 1 per molecule)
  double4 *shg_scratch;
  int nshg;
  size_t shg_smem;   // dynamic shared memory of the general SHAKE kernel
  // restraints (global atoms)
  int4 *rs; double *rs_fk;                 // i, j, ih, to_center
  int2 *rp; double *rp_x, *rp_fk;          // i, ipsi; x[3], fk[3]
  int4 *rd; double4 *rd_p;                 // i, j, ipsi; d1, d2, fk
  int4 *ra; double2 *ra_p;                 // i, j, k, ipsi; ang, fk
  int4 *rw; double4 *rw_p;                 // i, j, ih; d, fk, aMorse, dMorse
  // dynamic lists
  int4 *pp;                                // i, j, lj
  uint16_t *pwg;                           // [solute group*pwg_cap + k] local water index
  int *pwg_n, pwg_cap;                     // waters listed per solute group
  struct PwAtom *pwa;                      // non-Q atoms of each solute group (static)
  int *pwg_off;                            // [solute group] first entry in pwa; one extra at the end
  int4 *qp;                                // gq, j, lj, qlj
  int *qw;                                 // water O atoms
  uint16_t *ww;                            // [gw*ww_cap + k] local water index
  int *ww_mid;                             // per water: list entries below its own index (ascending lists)
  int *lf_atoms, n_lf;
  // blocks of the per-water kernels, (system, first index) each, only where
  // a system has work: the water pass (256 waters or solute atoms), the
  // polarisation forces (WPOL_BLOCK waters) and Q-water (128 list entries)
  int2 *pk_tiles, *wp_tiles, *qw_tiles;
  int n_pk_tiles, n_wp_tiles, n_qw_tiles;
  int2 *pw_groups;                         // (system, solute group) of systems with waters
  int n_pw_groups;                     // atoms k_leapfrog moves (all but 3-constraint molecules')
  int *ww_n, *ww_sp;                       // count per water; [gw*ww_nch + c] count below chunk c's end
  int ww_cap, ww_chunk, ww_nch;
  int2 *ww_tiles;                          // water-water force blocks: (system, first water)
  int n_ww_tiles;
  int lrf_tpb;                             // source tiles swept by one block of the LRF gather
  // energies
  double *kin;                             // [s*4] kinetic energy of this step: solute all, free, solvent all, free
  int kin_nblk;
  double *E;                               // [s*QB_NE]
  double *EQ;                              // [(s*MAXS + st)*QB_NEQ]
  double *offd_r;                          // [s*MAXS + io] r_kl of this step's off-diagonal functions
  // history [kind][s][rec][QB_NE + MAXS*QB_NEQ + 1]
  double *hist;
  int hist_cap;
  HistRef *hr;               // device copy of (hist, hist_cap) for the kernels
  // periodic box: molecule starts, 1/molecule mass, per-atom mass (1/winv)
  int *mol_first;
  double *mol_minv, *mass_box;
};

}  // namespace qb
