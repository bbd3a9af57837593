/*
 * qb_system.h -- flat, read-only view of one prepared Q MD system.
 *
 * A "prepared system" is the state Q's qdyn holds when it enters md_run
 * (src/q6/qdyn.f90:80-96): the .inp file parsed (md.f90:2528 initialize), the
 * topology read (topo.f90:529 topo_read, md.f90:14705 topology), restart or
 * topology coordinates loaded (md.f90:13596 prep_coord), the FEP file applied
 * (md.f90:1472 get_fep, qatom.f90:253/874), charges scaled and water shells set
 * up (md.f90:13787 prep_sim, 14961 wat_sphere, 15044 wat_shells), SHAKE
 * constraints collected (md.f90:2326 init_shake), the Q-Q list built
 * (md.f90:1022 make_nbqqlist), removed terms dropped (md.f90:14569
 * shrink_topology) and, when a seed is given, Maxwell velocities drawn and
 * shaken (md.f90:3787 maxwell, 2506 initial_shaking, 14670 stop_cm_translation).
 *
 * Every index in this view is 0-based (the reference is 1-based).  Bonded terms
 * carry their parameters resolved per term.  Single-precision storage that the
 * reference uses (charges, inverse masses, torsion/improper parameters, water
 * shell data) is kept single precision here so that any consumer reproduces the
 * same rounding.
 *
 * The view points into memory owned by the qb_handle it came from; it stays
 * valid until qb_close().
 */
#ifndef QB_SYSTEM_H
#define QB_SYSTEM_H

#ifdef __cplusplus
extern "C" {
#endif

#define QB_MAX_STATES 10   /* qatom.f90:37 max_states */
#define QB_NBR_RANGE 25    /* topo.f90:30 max_nbr_range */

/* Energy vector layout: the reference's `energies` type (nrgy.f90:43-49). */
enum qb_energy_index {
  QB_E_POTENTIAL = 0, QB_E_KINETIC, QB_E_LRF,
  QB_E_P_BOND, QB_E_P_ANGLE, QB_E_P_TORSION, QB_E_P_IMPROPER,
  QB_E_W_BOND, QB_E_W_ANGLE, QB_E_W_TORSION, QB_E_W_IMPROPER,
  QB_E_Q_BOND, QB_E_Q_ANGLE, QB_E_Q_TORSION, QB_E_Q_IMPROPER,
  QB_E_PP_EL, QB_E_PP_VDW, QB_E_PW_EL, QB_E_PW_VDW, QB_E_WW_EL, QB_E_WW_VDW,
  QB_E_QX_EL, QB_E_QX_VDW,
  QB_E_RST_TOTAL, QB_E_RST_FIX, QB_E_RST_SHELL, QB_E_RST_PROTEIN,
  QB_E_RST_SOLVENT_RADIAL, QB_E_RST_WATER_POL,
  QB_NE /* = 29 */
};

/* Per-state energy layout: the reference's `q_energies` type (nrgy.f90:51-58);
 * this is also the payload order of one .en record after the state index. */
enum qb_qenergy_index {
  QB_EQ_LAMBDA = 0, QB_EQ_TOTAL,
  QB_EQ_BOND, QB_EQ_ANGLE, QB_EQ_TORSION, QB_EQ_IMPROPER,
  QB_EQ_QX_EL, QB_EQ_QX_VDW, QB_EQ_QQ_EL, QB_EQ_QQ_VDW,
  QB_EQ_QP_EL, QB_EQ_QP_VDW, QB_EQ_QW_EL, QB_EQ_QW_VDW,
  QB_EQ_RESTRAINT,
  QB_NEQ /* = 15 */
};

typedef struct qb_sysview {
  /* ---- sizes ---- */
  int natom, nat_solute, nwat;
  int ncgp, ncgp_solute, natyps;
  int nqat, nstates;
  int nbonds, nbonds_solute, nangles, nangles_solute;
  int ntors, ntors_solute, nimps, nimps_solute;
  int nmol;

  /* ---- force-field switches ---- */
  int ff_type;          /* 1 GROMOS (harmonic impropers), 2 AMBER (periodic), 3 CHARMM */
  int ivdw_rule;        /* 1 geometric (type_avdw/bvdw = sqrt A, sqrt B); 2 arithmetic (R*, sqrt(eps)) */
  int solvent_type;     /* 0 SPC-like 3-site water */
  int iuse_switch_atom; /* 1: charge-group cut-off on switching atoms */
  double el14_scale, coulomb_constant;

  /* ---- run control (md.f90:2528 initialize) ---- */
  int nsteps, NBcycle, iout_cycle, iene_cycle, itemp_cycle, itrj_cycle;
  double stepsize_fs, dt, Temp0, tau_T, Tmaxw;
  int iseed, separate_scaling;
  int shake_solvent, shake_solute, shake_hydrogens;
  int use_LRF, force_rms;
  double Rcpp, Rcww, Rcpw, Rcq, RcLRF;

  /* ---- sphere and solvent restraints ---- */
  double xpcent[3], xwcent[3];
  double rexcl_o, rexcl_i, rwat;
  double fk_pshell, fk_fix;
  double fk_wsphere, Dwmz, awmz, fkwpol;
  int wpol_restr, wpol_born;
  int nexats, nexwat, nshellats;

  /* ---- per atom ---- */
  const double *xtop;         /* [3*natom] topology coordinates */
  const double *x0, *v0;      /* [3*natom] coordinates/velocities entering md_run */
  const int *iac;             /* [natom] atom type, 0-based */
  const float *crg;           /* [natom] charge * sqrt(coulomb_constant), float storage */
  const float *winv;          /* [natom] 1/mass, float storage (md.f90:13858) */
  const double *mass;         /* [natom] mass from the type library */
  const unsigned char *heavy; /* [natom] */
  const unsigned char *excl;  /* [natom] outside the simulation sphere */
  const unsigned char *shell; /* [natom] in the restrained shell */
  const int *iqatom;          /* [natom] -1 or Q-atom index */
  const int *iwhich_cgp;      /* [natom] charge group of the atom */

  /* ---- atom types ---- */
  const double *type_mass;    /* [natyps] */
  const double *type_avdw;    /* [natyps*3] sqrt(A) for LJ codes 1,2,3 (3 = 1-4) */
  const double *type_bvdw;    /* [natyps*3] sqrt(B) */
  const unsigned char *ljcod; /* [natyps*natyps] 1 or 2 */

  /* ---- neighbour exclusion/1-4 data for solute atoms (topo.f90:991-1045) ---- */
  const unsigned int *listex_bits; /* [nat_solute] bit k-1: listex(k,i), pair (i, i+k) */
  const unsigned int *list14_bits; /* [nat_solute] bit k-1: list14(k,i) */
  int nexlong, n14long;
  const int *listexlong;      /* [2*nexlong] pairs */
  const int *list14long;      /* [2*n14long] pairs */

  /* ---- charge groups ---- */
  const int *cgp_iswitch, *cgp_first, *cgp_last; /* [ncgp]; first/last index cgpatom */
  const int *cgpatom;                            /* [natom] */

  /* ---- molecules ---- */
  const int *istart_mol; /* [nmol+1], last entry = natom */

  /* ---- bonded terms, parameters resolved per term (after shrink_topology) ---- */
  const int *bnd_i, *bnd_j;            const double *bnd_fk, *bnd_b0;
  const int *ang_i, *ang_j, *ang_k;    const double *ang_fk, *ang_th0;
  const double *ang_ureyfk, *ang_ureyr0; /* Urey-Bradley k and 1-3 r0; zero unless ff_type 3 */
  const int *tor_i, *tor_j, *tor_k, *tor_l;
  const float *tor_fk, *tor_rmult, *tor_deltor, *tor_paths; /* paths already inverted */
  const int *imp_i, *imp_j, *imp_k, *imp_l;
  const float *imp_fk, *imp_imp0;

  /* ---- water ---- */
  float crg_ow, crg_hw;           /* scaled charges of water O and H */
  double A_OO, B_OO;              /* O-O LJ products (md.f90:11836-11841) */
  int ww_hlj;                     /* water hydrogens carry LJ in the water-water and Q-water terms
                                     (nonbon2_ww/nonbon2_qw, nonbond_3atomsolvent/nonbond_qw_3atom) */
  double A_OH, B_OH, A_HH, B_HH;  /* O-H and H-H LJ products, when ww_hlj */
  int iac_ow, iac_hw;
  int nwpolr_shell;
  const float *wshell_rout, *wshell_dr, *wshell_cstb; /* [nwpolr_shell] */
  const float *wshell_theta_corr0;                    /* initial theta_corr */

  /* ---- Q atoms / FEP ---- */
  const double *lambda;        /* [nstates] */
  const int *iqseq;            /* [nqat] atom index */
  const float *qcrg;           /* [nqat*nstates] scaled, index iq*nstates+s */
  int qvdw_flag;
  int qq_use_library_charges; /* Q-Q pairs take the topology charges (nonbond_qq_lib_charges) */
  int nqlib;
  const int *qiac;             /* [nqat*nstates] Q atom type (0-based into qavdw) */
  const double *qavdw, *qbvdw; /* [nqlib*3] */
  const double *sc_lookup;     /* [(nqat*(natyps+nqat))*nstates], index (iq*(natyps+nqat)+col)*nstates+s */
  const signed char *qconn;    /* [nstates*nat_solute*nqat], index (s*nat_solute+i)*nqat+iq */
  /* Q-Q and Q-near-neighbour pairs per state (md.f90:7449 nbqqlist) */
  const int *nbqq_count;       /* [nstates] */
  const int *nbqq_off;         /* [nstates] offset into the arrays below */
  const int *nbqq_iq, *nbqq_j, *nbqq_jq, *nbqq_ljcod; /* jq = -1: j is not a Q atom */
  const double *nbqq_el_scale;
  /* Q bonded terms, parameters per state (cod > 0 in that state); present[] 0/1 */
  int nqbond, nqangle, nqtor, nqimp;
  const int *qbnd_i, *qbnd_j;  const unsigned char *qbnd_on;
  const double *qbnd_Dmz, *qbnd_amz, *qbnd_r0, *qbnd_fk;   /* [n*nstates] */
  const int *qang_i, *qang_j, *qang_k; const unsigned char *qang_on;
  const double *qang_fk, *qang_th0;
  const double *qang_ureyfk, *qang_ureyr0;  /* [n*nstates]; zero unless ff_type 3 */
  const int *qtor_i, *qtor_j, *qtor_k, *qtor_l; const unsigned char *qtor_on;
  const double *qtor_fk, *qtor_rmult, *qtor_deltor;
  const int *qimp_i, *qimp_j, *qimp_k, *qimp_l; const unsigned char *qimp_on;
  const double *qimp_fk, *qimp_imp0;
  /* EVB off-diagonal functions Hij = A exp(-mu r_kl) (qatom.f90:1515-1555; offdiag, md.f90:12911) */
  int noffd;
  const int *offd_i, *offd_j;  /* states, 1-based as the FEP and energy files give them */
  const int *offd_k, *offd_l;  /* Q atoms, 0-based */
  const double *offd_A, *offd_mu;
  /* EVB Morse couplings of Q terms to Q bonds (qatom.f90:1404-1497): per term the coupled Q bond
   * (-1: none; angles: qangle's first coupling, qurey_bradley's last), impropers' flag (1: gamma =
   * 1 - EMorseD), and per (term, state) the state whose qbond values EMorseD holds there */
  const int *qang_cpl, *qang_cpl_ub, *qtor_cpl, *qimp_cpl, *qimp_cpl_flag;   /* [n] */
  const int *qang_cpl_src, *qang_cpl_ub_src, *qtor_cpl_src, *qimp_cpl_src;   /* [n*nstates] */

  /* ---- SHAKE (md.f90:2326 init_shake) ---- */
  int shake_molecules, shake_constraints;
  const int *shake_mol_first, *shake_mol_n; /* [shake_molecules] into constraint arrays */
  const int *shake_i, *shake_j;
  const double *shake_dist2;

  /* ---- restraints (.inp sections) ---- */
  int nrstr_seq, nrstr_pos, nrstr_dist, nrstr_angl, nrstr_wall;
  const int *rseq_i, *rseq_j, *rseq_ih, *rseq_to_center; const double *rseq_fk;
  const int *rpos_i, *rpos_ipsi; const double *rpos_x, *rpos_fk; /* x, fk: [3*n] */
  const int *rdis_i, *rdis_j, *rdis_ipsi; const double *rdis_d1, *rdis_d2, *rdis_fk;
  const int *rang_i, *rang_j, *rang_k, *rang_ipsi; const double *rang_ang, *rang_fk;
  const int *rwal_i, *rwal_j, *rwal_ih; const double *rwal_d, *rwal_fk, *rwal_aMorse, *rwal_dMorse;

  /* ---- temperature bookkeeping (md.f90:2460-2480) ---- */
  int Ndegf, Ndegfree, Ndegf_solute, Ndegf_solvent, Ndegfree_solute, Ndegfree_solvent;
  int detail_temps;

  /* ---- periodic box (topology boundary "PBC", .inp [PBC], md.f90:2583-2656) ----
   * Pairs take the nearest image of their charge groups' reference atoms;
   * no excluded atoms, restrained shell, solvent sphere or polarisation. */
  int use_pbc;
  int rigid_box_center, put_solute_back_in_box, put_solvent_back_in_box;
  int constant_pressure;        /* NPT: Monte Carlo volume moves (MC_volume, md.f90:15615) */
  int ivolume_cycle, pressure_seed;
  double max_vol_displ;         /* A^3 */
  double pressure;              /* kcal/mol/A^3 (bar * 1.43836e-5) */
  double boxlength[3], boxcenter[3];
  const double *mol_mass_inv;   /* [nmol] 1 / molecule mass */
  const double *mass_box;       /* [natom] mass as 1.0/winv in single precision (md.f90:13882) */
  int qswitch;                  /* atom the Q-atom lists centre on in a box (-1: none) */
  /* randm's state after the Maxwell velocities (randm_started: seeded), which
   * the volume moves continue (md.f90:14408) */
  int randm_started, randm_state;
} qb_sysview;

#ifdef __cplusplus
}
#endif
#endif /* QB_SYSTEM_H */
