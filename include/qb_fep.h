/* qb_fep.h -- free-energy analysis of per-state energy series on the GPU.
 *
 * Replaces qfep (src/q6/qfep.f90:200-762), the program that reads qdyn's
 * energy files (nrgy.f90:94-119) and reports, per pair of adjacent windows,
 * Zwanzig forward/reverse, thermodynamic integration, overlap sampling (Lu)
 * and Bennett's acceptance ratio, plus the energy-gap binned reaction free
 * energies.  Arrays use qfep's indexing: a "file" is one lambda window, and
 * the per-window arrays run 0..nfiles+1 with entry i belonging to file i
 * (1-based), exactly as qfep prints them (dG(ifile-1) beside lambda(ifile)).
 *
 * EVB: with nnoffd > 0 the states are coupled through qfep's parametrised
 * off-diagonal elements Hij(r) of the first off-diagonal distance r_xy that
 * qdyn stored in each record (qfep.f90:160-172, 274-318); the ground-state
 * energy is the lowest eigenvalue of the EVB matrix.  qfep's other mode,
 * predefined elements read from the energy files (noffd > 0 on its first
 * input line), reads no off-diagonal values there (nnoffd is never set) and
 * is not part of this path.
 */
#ifndef QB_FEP_H
#define QB_FEP_H

#ifdef __cplusplus
extern "C" {
#endif

#define QB_FEP_MAX_STATES 4     /* qfep's mxstates */
#define QB_FEP_MAX_BINS 598     /* qfep's mxbin less the two spare bins */
#define QB_FEP_BAR_MAX_ITER 1000
#define QB_FEP_MAX_PAIRS 16     /* QB_FEP_MAX_STATES squared: the EVB parameter matrices */
#define QB_FEP_PART2_W 9        /* gap centre, dGv(1), dGv(2), dGg, points, c1^2, c2^2, printed (0/1), <r_xy> */
#define QB_FEP_PART3_W 8        /* gap centre, <dGg>, <dGg norm>, points, c1^2, c2^2, r_xy, printed (0/1) */

/* Analysis parameters: qfep's interactive input (qfep.f90:87-172). */
typedef struct qb_fep_params {
  double rt;               /* kT, kcal/mol */
  int nskip;               /* records to skip at the start of every file */
  int gas;                 /* >0: totals from the Q bonded, Q-Q and restraint terms only (qfep.f90:257) */
  int nbins;               /* energy-gap bins (Part 2) */
  int nmin;                /* minimum points per bin */
  double alfa[QB_FEP_MAX_STATES];   /* shift of each state's total; alfa[0] is taken as 0 */
  double coeff[QB_FEP_MAX_STATES];  /* linear combination of states defining the energy gap */
  /* EVB off-diagonal elements (qfep.f90:163-172, 286-299): for nnoffd > 0,
   * Hij = A exp(-mu (r - rxy0)) exp(-eta (r - rxy0)^2) with the parameters of
   * (i, j), or of (j, i) where A(i, j) is 0; matrices [i*4 + j], 0-based. */
  int nnoffd;
  double evb_A[QB_FEP_MAX_PAIRS];
  double evb_mu[QB_FEP_MAX_PAIRS];
  double evb_eta[QB_FEP_MAX_PAIRS];
  double evb_rxy0[QB_FEP_MAX_PAIRS];
  const double *rxy;       /* qb_fep_analyze with nnoffd > 0: r_xy of every record, file after file */
} qb_fep_params;

/* Results; every pointer is a caller-owned buffer of the stated size, or NULL
 * to skip that output. */
typedef struct qb_fep_result {
  double *lambda;          /* [nfiles*nstates] from each file's first record */
  int *npts;               /* [nfiles] records per file */
  double *avEQ;            /* [nfiles*nstates*15] Part 0 averages of the q_energies components */
  double *dgf;             /* [nfiles+2] Zwanzig forward, entry i for files i -> i+1 */
  double *dgfsum;          /* [nfiles+2] */
  double *dgr;             /* [nfiles+2] Zwanzig reverse, entry i for files i -> i-1 */
  double *dgrsum;          /* [nfiles+2] */
  double *dG;              /* [nfiles+2] mean of forward and reverse, accumulated */
  double *dgti;            /* [nfiles+2] <V2 - V1> of file i */
  double *dgtisum;         /* [nfiles+2] trapezoid over lambda(1) */
  double *dglu;            /* [nfiles+2] overlap sampling, files i, i+1 */
  double *dglusum;         /* [nfiles+2] */
  double *dgbar;           /* [nfiles+2] BAR, files i, i+1 */
  double *dgbarsum;        /* [nfiles+2] */
  int *bar_iterations;     /* [nfiles+2] iterations to |change| <= 0.001, -1 if not within QB_FEP_BAR_MAX_ITER */
  double *gap_range;       /* [2] minimum and maximum energy gap */
  double *part2;           /* [nfiles*(nbins+2)*QB_FEP_PART2_W], bin index 1..nbins */
  double *part3;           /* [(nbins+2)*QB_FEP_PART3_W] */
} qb_fep_result;

/* Analysis of energy series held in host memory: `energies` holds, file
 * after file, npts[f] records of nstates q_energies (15 doubles each, in the
 * .en record order of nrgy.f90:32-41).  nfiles >= 2, 1 <= nstates <= 4. */
int qb_fep_analyze(const double *energies, const int *npts, int nfiles, int nstates, const qb_fep_params *p,
                   int device, qb_fep_result *out);

/* The same analysis of a batch's own energy-file records, read in place on
 * the GPU: file f is system sys[f] of the batch (its records at the energy
 * interval since the last qb_batch_clear_history). */
struct qb_batch;
int qb_batch_fep(struct qb_batch *b, const int *sys, int nfiles, const qb_fep_params *p, qb_fep_result *out);

#ifdef __cplusplus
}
#endif
#endif
