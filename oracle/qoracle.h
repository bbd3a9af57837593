/*
 * qoracle.h -- CPU oracle of the Q MD step (TEST INFRASTRUCTURE ONLY: used by
 * tests/, the smoke check and bench.py's CPU-baseline leg as the checker; the
 * product never links it).  See qoracle.c.
 */
#ifndef QORACLE_H
#define QORACLE_H
#include "qb_system.h"

typedef struct qo_state qo_state;

/* Copy the prepared system's coordinates/velocities and compute the initial
 * temperature, as md_run does before its loop. */
qo_state *qo_create(const qb_sysview *s, int history_capacity);
void qo_destroy(qo_state *st);
/* nsteps passes of the md_run loop body; returns 0, 5 (SHAKE failure) or 10
 * (a volume move left the box too small for a cut-off). */
int qo_run(qo_state *st, int nsteps);
/* post-loop list rebuild and potential evaluation */
int qo_final_energy(qo_state *st);
void qo_energies(const qo_state *st, double *E, double *EQ);
void qo_gradient(const qo_state *st, double *d);
void qo_coords(const qo_state *st, double *x);
void qo_velocities(const qo_state *st, double *v);
void qo_set_coords(qo_state *st, const double *x);
void qo_set_velocities(qo_state *st, const double *v);
void qo_theta_corr(const qo_state *st, float *tc);
void qo_temperature(const qo_state *st, double *out);
int qo_history(const qo_state *st, int kind, int *steps, double *E, double *EQ);
int qo_offdiag(const qo_state *st, int kind, double *rkl);
void qo_list_counts(const qo_state *st, int *out);
int qo_status(const qo_state *st);
/* periodic box: edge lengths then centre; Monte Carlo volume moves tried and accepted */
void qo_box(const qo_state *st, double *box6);
void qo_volume_moves(const qo_state *st, long long *tries, long long *accepted);
#endif
