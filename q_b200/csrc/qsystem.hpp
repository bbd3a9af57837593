// qsystem.hpp -- host-side representation of one prepared Q system.
//
// Holds what qdyn has in memory when md_run starts (src/q6/qdyn.f90:80-96).
// Filled by the readers in qfiles.cpp and the set-up in setup.cpp; exported to
// the CUDA engine and to callers as a qb_sysview (include/qb_system.h).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "qb.h"
#include "ljrule.hpp"

namespace qb {

// Error carrying a qb_status code; converted to a return value at the C ABI.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string &msg) { throw Error(code, msg); }

struct SeqRestraint { int i, j; double fk; int ih, to_center; };
struct PosRestraint { int i; double x[3], fk[3]; int ipsi; };
struct DistRestraint { int i, j; double d1, d2, fk; int ipsi; };
struct AngRestraint { int i, j, k; double ang, fk; int ipsi; };
struct WallRestraint { int i, j; double d, fk, aMorse, dMorse; int ih; };

// Parsed .inp (md.f90:2528-3262 initialize), values after its defaults.
struct RunInput {
  std::string inp_path, dir;
  int nsteps = 0;
  double stepsize = 0, dt = 0, Temp0 = 0, tau_T = 0, Tmaxw = 0;
  int iseed = 0;
  bool have_tmaxw = false;
  bool separate_scaling = false;
  bool shake_solvent = true, shake_solute = false, shake_hydrogens = false;
  bool use_LRF = false, force_rms = false;
  double Rcpp = 10, Rcww = 10, Rcpw = 10, Rcq = 99, RcLRF = 99;
  double rexcl_i = 0.85, fk_pshell = 10;
  bool exclude_bonded = false;
  double rwat_in = 0, fk_wsphere = -1, Dwmz = -1, awmz = -1, fkwpol = -1;
  bool wpol_restr = true, wpol_born = true;
  int NBcycle = 10, iout_cycle = 10, itemp_cycle = 10, iene_cycle = 0, itrj_cycle = 0;
  std::string top_file, restart_file, xfin_file, trj_file, ene_file, fep_file;
  bool restart = false;
  std::vector<double> lambdas;
  std::vector<SeqRestraint> rseq;
  std::vector<PosRestraint> rpos;
  std::vector<DistRestraint> rdis;
  std::vector<AngRestraint> rang;
  std::vector<WallRestraint> rwal;
  // [PBC] (md.f90:2583-2656)
  bool box = false, rigid_box_center = false, constant_pressure = false, control_box = false;
  bool put_solvent_back_in_box = false, put_solute_back_in_box = false;
  double max_vol_displ = 0, pressure_bar = 1.0, pressure = 0, new_boxl[3] = {0, 0, 0};
  int pressure_seed = 3781, ivolume_cycle = 10;
};

struct TypeLib { double mass; double avdw[3]; double bvdw[3]; };

// Topology as read by topo_read (topo.f90:529-1079); indices 0-based.
struct Topology {
  std::string title;
  double version = 2;
  int ff_type = 1;
  int nat_pro = 0, nat_solute = 0;
  std::vector<double> xtop;
  std::vector<int> iac;
  std::vector<unsigned char> heavy;
  std::vector<float> crg;
  struct Bond { int i, j, cod; };
  struct Angle { int i, j, k, cod; };
  struct Tors { int i, j, k, l, cod; };
  std::vector<Bond> bnd; int nbonds_solute = 0;
  std::vector<double> bond_fk, bond_b0;
  std::vector<Angle> ang; int nangles_solute = 0;
  std::vector<double> ang_fk, ang_th0;
  std::vector<double> ang_ureyfk, ang_ureyr0;   // optional Urey-Bradley columns (0 when absent)
  std::vector<Tors> tor; int ntors_solute = 0;
  std::vector<float> tor_fk, tor_rmult, tor_deltor, tor_paths;
  std::vector<Tors> imp; int nimps_solute = 0; int imp_type = 1;
  std::vector<float> imp_fk, imp_imp0;
  int ncgp = 0, ncgp_solute = 0, iuse_switch_atom = 1;
  std::vector<int> cgp_iswitch, cgp_first, cgp_last, cgpatom;
  int natyps = 0, ivdw_rule = 1;
  double el14_scale = 0.5, coulomb_constant = 332.0;
  std::vector<TypeLib> iaclib;
  std::vector<std::pair<int, int>> lj2;
  std::vector<unsigned int> list14, listex;   // bit k-1 for pair (i, i+k), per solute atom
  std::vector<std::pair<int, int>> list14long, listexlong;
  int nres = 0, nres_solute = 0;
  std::vector<int> res_start;
  std::vector<std::string> res_name;
  int nmol = 0;
  std::vector<int> istart_mol;
  std::vector<std::string> tac;
  int solvent_type = 0;
  bool use_pbc = false;
  double boxlength[3] = {0, 0, 0}, boxcenter[3] = {0, 0, 0};   // periodic box (topo.f90:1031-1033)
  double rexcl_o = 0, rwat = 0, xpcent[3] = {0, 0, 0}, xwcent[3] = {0, 0, 0};
  int nexats = 0, nexwat = 0;
  std::vector<unsigned char> excl;
};

// FEP data as read by qatom_load_atoms/qatom_load_fep (qatom.f90:253, 874).
struct Fep {
  int nstates = 0, nqat = 0, offset = 0;
  int qswitch = -1;   // periodic box: atom the Q-atom lists are centred on ([PBC] switching_atom, 0-based)
  bool qq_use_library_charges = false, softcore_use_max_potential = false;
  std::vector<int> iqseq;                    // atom index per Q atom (0-based, -1 unused)
  std::vector<float> qcrg;                   // [nqat*nstates] unscaled until set-up
  bool qvdw_flag = false;
  int nqlib = 0;
  std::vector<std::string> qtac;
  std::vector<double> qavdw, qbvdw, qmass;   // [nqlib*3]
  std::vector<int> qiac;                     // [nqat*nstates]
  std::vector<std::pair<int, int>> soft_pairs;       // q-atom indices
  struct ElScale { int iq, jq; double s[QB_MAX_STATES]; };
  std::vector<ElScale> el_scale;
  struct ExSpec { int i, j; bool flag[QB_MAX_STATES]; };
  std::vector<ExSpec> exspec;
  struct QBondLib { double Dmz, amz, r0, fk; };
  std::vector<QBondLib> qbondlib;            // index = type-1
  struct QBnd { int i, j; int cod[QB_MAX_STATES]; };
  std::vector<QBnd> qbnd;
  struct QAngLib { double fk, ang0, ureyfk, ureyr0; };
  std::vector<QAngLib> qanglib;
  struct QAng { int i, j, k; int cod[QB_MAX_STATES]; };
  std::vector<QAng> qang;
  std::vector<double> qfktor, qrmult, qdeltor;
  struct QTor { int i, j, k, l; int cod[QB_MAX_STATES]; };
  std::vector<QTor> qtor;
  std::vector<double> qfkimp, qimp0;
  std::vector<QTor> qimp;
  // EVB Morse couplings: Q term, Q bond (0-based), flag (1: gamma = 1 - EMorseD; impropers only)
  struct Coupling { int term, bond, flag; };
  std::vector<Coupling> ang_coupl, tor_coupl, imp_coupl;
  int nang_coupl = 0, ntor_coupl = 0, nimp_coupl = 0, nqshake = 0, noffd = 0;
  struct OffD { int i, j, k, l; double A, mu; };   // states 1-based, Q atoms 0-based
  std::vector<OffD> offd;
  struct QShake { int i, j; double dist[QB_MAX_STATES]; };
  std::vector<QShake> qshake;
  std::vector<double> alpha_max;             // [nqat*nstates]
  std::vector<double> sc_lookup;             // [nqat*(natyps+nqat)*nstates] (view layout)
};

// The prepared system.
struct System {
  RunInput in;
  Topology top;
  Fep fep;
  int natom = 0, nwat = 0;
  std::vector<int> iqatom, iwhich_cgp;
  std::vector<float> winv;
  std::vector<double> mass;
  std::vector<unsigned char> shell;
  int nshellats = 0;
  float crg_ow = 0, crg_hw = 0, mu_w = 0;
  double A_OO = 0, B_OO = 0;
  int ww_hlj = 0;
  double A_OH = 0, B_OH = 0, A_HH = 0, B_HH = 0;
  int iac_ow = -1, iac_hw = -1;
  double crgtot = 0, crgQtot = 0;
  double fk_wsphere = 60, Dwmz = 0, awmz = 0, fkwpol = 20, rwat = 0;
  int nwpolr_shell = 0;
  std::vector<float> ws_rout, ws_dr, ws_cstb, ws_theta_corr;
  std::vector<double> x, v;
  std::vector<unsigned char> ljcod;          // [natyps*natyps]
  std::vector<double> type_mass, type_avdw, type_bvdw;
  // flattened Q data
  std::vector<signed char> qconn;            // [nstates*nat_solute*nqat]
  std::vector<int> nbqq_count, nbqq_off, nbqq_iq, nbqq_j, nbqq_jq, nbqq_ljcod;
  std::vector<double> nbqq_el_scale;
  std::vector<float> qcrg_scaled;
  std::vector<int> qbnd_i, qbnd_j, qang_i, qang_j, qang_k;
  std::vector<int> qtor_i, qtor_j, qtor_k, qtor_l, qimp_i, qimp_j, qimp_k, qimp_l;
  std::vector<unsigned char> qbnd_on, qang_on, qtor_on, qimp_on;
  std::vector<double> qbnd_Dmz, qbnd_amz, qbnd_r0, qbnd_fk, qang_fk, qang_th0, qang_ureyfk, qang_ureyr0;
  std::vector<double> qtor_fk, qtor_rmult, qtor_deltor, qimp_fk, qimp_imp0;
  std::vector<int> offd_i, offd_j, offd_k, offd_l; std::vector<double> offd_A, offd_mu;
  // Morse coupling of each Q angle (qangle's, then qurey_bradley's), torsion and improper: the
  // bond or -1, the flag, and per state the state whose qbond values EMorseD holds there
  std::vector<int> qang_cpl, qang_cpl_ub, qtor_cpl, qimp_cpl, qimp_cpl_flag;
  std::vector<int> qang_cpl_src, qang_cpl_ub_src, qtor_cpl_src, qimp_cpl_src;
  // resolved bonded terms (after shrink_topology)
  std::vector<int> bi, bj; std::vector<double> bfk, bb0; int nb_solute = 0;
  std::vector<int> ai, aj, ak; std::vector<double> afk, ath0, aufk, aur0; int na_solute = 0;
  std::vector<int> ti, tj, tk, tl; std::vector<float> tfk, trm, tdel, tpaths; int nt_solute = 0;
  std::vector<int> ii, ij, ik, il; std::vector<float> ifk, iimp0; int ni_solute = 0;
  // shake
  std::vector<int> sh_first, sh_n, sh_i, sh_j; std::vector<double> sh_d2;
  int shake_constraints = 0;
  int Ndegf = 0, Ndegfree = 0, Ndegf_solute = 0, Ndegf_solvent = 0;
  int Ndegfree_solute = 0, Ndegfree_solvent = 0;
  bool detail_temps = false;
  // restraint arrays for the view
  std::vector<int> rseq_i, rseq_j, rseq_ih, rseq_tc; std::vector<double> rseq_fk;
  std::vector<int> rpos_i, rpos_ipsi; std::vector<double> rpos_x, rpos_fk;
  std::vector<int> rdis_i, rdis_j, rdis_ipsi; std::vector<double> rdis_d1, rdis_d2, rdis_fk;
  std::vector<int> rang_i, rang_j, rang_k, rang_ipsi; std::vector<double> rang_ang, rang_fk;
  std::vector<int> rwal_i, rwal_j, rwal_ih; std::vector<double> rwal_d, rwal_fk, rwal_a, rwal_dm;
  std::vector<unsigned char> heavy_u8;
  // periodic box: edge lengths and centre (topology, restart, control_box),
  // 1/molecule mass and the per-atom mass put_back_in_box and MC_volume use
  double boxl[3] = {0, 0, 0}, boxc[3] = {0, 0, 0};
  std::vector<double> mol_minv, mass_box;
  // randm's sequence after the Maxwell velocities (started: it was seeded)
  int randm_started = 0, randm_state = 0;
  std::string log;   // qdyn-style set-up messages

  void fill_view(qb_sysview *v) const;
};

// qfiles.cpp
void read_inp(const std::string &path, RunInput &in);
void read_topology(const std::string &path, Topology &t);
void read_fep_atoms(const std::string &path, const Topology &t, Fep &f, int nstates_inp);
void read_fep(const std::string &path, const Topology &t, Fep &f);
void read_restart(const std::string &path, int natom, std::vector<double> &x,
                  std::vector<double> &v, int nshell, std::vector<float> *theta_corr,
                  double *boxl = nullptr, double *boxc = nullptr);
void write_restart(const std::string &path, int natom, const double *x, const double *v,
                   int nshell, const float *theta_corr, const double *box6 = nullptr);
void append_energy_frame(const std::string &path, int nstates, const double *EQ, int noffd, const int *ij,
                         const double *hr);

// setup.cpp
void prepare(System &s);
void put_back_in_box(System &s);

// Fortran single-precision constants that the reference mixes into FP64 math.
constexpr float kBoltz = 0.001986f;     // md.f90:41
constexpr float kRhoWat = 0.0335f;      // md.f90:40
// pi = 4.0*atan(1.0) evaluated in single precision (md.f90:382)
double fortran_pi();
double fortran_deg2rad();

}  // namespace qb

// Opaque handle of the C ABI: one prepared system.
struct qb_handle {
  qb::System sys;
};
