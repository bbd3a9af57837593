/*
 * qb.h -- C ABI of libqb, a B200 (sm_100a) replacement for the MD step of Q's
 * qdyn (src/q6/md.f90:3917 md_run and everything it calls).
 *
 * The reference exposes no in-process interface: its boundary is the
 * executable `qdyn[p] <file.inp>` (src/q6/qdyn.f90:18-134) plus its file
 * contracts (.inp/.top/.fep/.re in, .en/.re/log out).  These entry points are
 * what a host (ctypes from Python, or any FFI) binds to reproduce that
 * executable in-process and to run many systems (lambda windows, replicas,
 * spheres) together on one GPU.
 *
 * Conventions
 *  - Every function returns an int status (enum qb_status); no exception or
 *    longjmp crosses the ABI.  qb_last_error() returns the message of the last
 *    failure on the calling thread.
 *  - The library owns all host and device state.  Callers pass host buffers
 *    they own; data moves only inside the get/set calls.
 *  - Handles are not thread-safe; distinct handles may be used from distinct
 *    threads.  One batch runs on one CUDA stream.
 *  - Atom, system and state indices are 0-based.
 */
#ifndef QB_H
#define QB_H

#include <stddef.h>
#include "qb_system.h"
#include "qb_fep.h"
#include "qb_mlp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Each reference failure path named on the right. */
enum qb_status {
  QB_OK = 0,
  QB_ERR_ARG = 1,           /* invalid argument */
  QB_ERR_IO = 2,            /* cannot open/read/write a file (md.f90:1382 open_files) */
  QB_ERR_PARSE = 3,         /* invalid .inp/.top/.fep/.re content (md.f90:2528, topo.f90:1073, qatom.f90:874) */
  QB_ERR_UNSUPPORTED = 4,   /* valid Q input outside this engine's scope (e.g. any-atom cut-offs in a periodic box) */
  QB_ERR_SHAKE = 5,         /* SHAKE did not converge in 1000 iterations (md.f90:14533-14551 'shake failure') */
  QB_ERR_NAN = 6,           /* non-finite energy or coordinate */
  QB_ERR_LIST_OVERFLOW = 7, /* a pair list exceeded its device capacity */
  QB_ERR_TIMEOUT = 8,       /* a bounded device wait gave up */
  QB_ERR_CUDA = 9,          /* CUDA runtime error, or no usable GPU */
  QB_ERR_STATE = 10         /* call not valid in the handle's current state */
};

/* Arithmetic mode of the per-step kernels. */
enum qb_precision {
  QB_FP64 = 0,   /* all pair math in FP64: the plain engine, parity mode */
  QB_MIXED = 1   /* FP32 pair math, compensated FP64 energy/force sums; FP64 LRF, SHAKE, update */
};

typedef struct qb_options {
  int precision;   /* enum qb_precision */
  int device;      /* CUDA device ordinal */
  int verbose;     /* 0 quiet, 1 print the qdyn-style setup log on stdout */
  int reserved[5];
} qb_options;

typedef struct qb_handle qb_handle; /* one prepared system, host side */
typedef struct qb_batch qb_batch;   /* device-resident systems stepped together */

/* Library version string, e.g. "qb 0.1.0 (sm_100a)". */
int qb_version(char *buf, size_t n);

/* Message of the last failure on this thread ("" if none). */
int qb_last_error(char *buf, size_t n);

/* Number of usable CUDA devices (0 on a machine without a GPU). */
int qb_device_count(int *out);

/* ---------------------------------------------------------------- systems */

/* Parse an .inp file and everything it names, and prepare the system exactly
 * as qdyn does before its first step (qdyn.f90:80-96).  Host only: needs no GPU.
 * Replaces: `qdyn <file.inp>` startup, src/q6/qdyn.f90:80-96. */
int qb_open(const char *inp_path, const qb_options *opt, qb_handle **out);

/* Same, with the [lambdas] and random_seed of the .inp overridden (n_lambda = 0
 * or seed < 0 keeps the file's value).  Used to fan one .inp out into windows
 * and replicas.  Replaces: editing md_X.inp per window (QligFEP qligfep.py:723). */
int qb_open_override(const char *inp_path, const qb_options *opt,
                     const double *lambdas, int n_lambda, int seed, qb_handle **out);

/* Flat read-only view of the prepared system (valid until qb_close). */
int qb_get_view(const qb_handle *h, qb_sysview *out);

void qb_close(qb_handle *h);

/* ------------------------------------------------------------------ batch */

/* Upload n prepared systems to the GPU and compute their initial temperatures
 * (md.f90:3960-3963).  Systems step together; each keeps its own pair-list
 * interval, output intervals and parameters. */
int qb_batch_create(qb_handle *const *systems, int n, const qb_options *opt, qb_batch **out);

/* Advance every system by nsteps MD steps with md_run's per-step semantics
 * (md.f90:4003-4175): pair lists every NBcycle steps, potential and gradient,
 * leapfrog with Berendsen scaling, SHAKE, temperature.  Energy summaries are
 * recorded on the device at each system's output/energy intervals.
 * Energies are evaluated on the steps that record them and on the last step
 * of the call (qb_batch_energies then reads complete values).  In the mixed
 * precision engine those steps evaluate the water-water pairs in FP64; the
 * other steps evaluate the water-water forces alone, in packed FP32.
 * A system that raises an error on the device (e.g. QB_ERR_SHAKE) stops at
 * the failing step, as md_run stops there: its coordinates stay those the
 * step produced (positions at the step's start = x - v*dt), its step count
 * and records stop, and the call returns the first such error once the
 * other systems have finished their steps.
 * Replaces: the `do istep` loop of md_run, src/q6/md.f90:4003-4175. */
int qb_batch_run(qb_batch *b, int nsteps);

/* qb_batch_run with the step loop bracketed by CUDA events on the batch
 * stream: device_ms receives the elapsed device time of the nsteps steps and
 * kernel_launches the number of kernels launched for them (either may be NULL). */
int qb_batch_run_timed(qb_batch *b, int nsteps, double *device_ms, long long *kernel_launches);

/* The post-loop evaluation of md_run (md.f90:4186-4188): rebuild the lists and
 * evaluate the potential at the final coordinates, for the FINAL summary. */
int qb_batch_final_energy(qb_batch *b);

/* Lists and gradient at the current coordinates, as qb_batch_final_energy,
 * evaluated the way a step of the given kind evaluates them: energies = 1 as
 * the steps that record energies (every energy term, FP64 water-water pairs),
 * energies = 0 as the other steps (mixed precision engine: water-water forces
 * in packed FP32 and no water-water energy).  Lets a caller check the force
 * path of the non-recording steps. */
int qb_batch_evaluate(qb_batch *b, int energies);

/* Energies of system `sys` from the last potential evaluation.
 * E_out: QB_NE doubles; EQ_out: nstates*QB_NEQ doubles (may be NULL). */
int qb_batch_energies(qb_batch *b, int sys, double *E_out, double *EQ_out);

/* Temperatures after the last step: out[0..4] = Temp, Tfree, Tfree_solute,
 * Tfree_solvent, Tscale_solvent. */
int qb_batch_temperature(qb_batch *b, int sys, double *out);

/* Gradient dU/dx from the last potential evaluation, 3*natom doubles. */
int qb_batch_gradient(qb_batch *b, int sys, double *d_out);

/* Coordinates of one system, 3*natom doubles.  Setting them marks the pair
 * lists and LRF multipoles of every system stale: they are rebuilt before the
 * next step, as qdyn builds them at step 0 of a restart. */
int qb_batch_get_coords(qb_batch *b, int sys, double *x_out);
int qb_batch_set_coords(qb_batch *b, int sys, const double *x_in);
int qb_batch_get_velocities(qb_batch *b, int sys, double *v_out);
int qb_batch_set_velocities(qb_batch *b, int sys, const double *v_in);

/* The same for every system at once, in batch order: 3*natom doubles per
 * system, back to back (3 * the batch's total atom count).  Each call makes
 * one device copy through page-locked staging that the batch owns, instead of
 * one small copy per system.  Setting marks the lists stale as above. */
int qb_batch_get_coords_all(qb_batch *b, double *x_out);
int qb_batch_set_coords_all(qb_batch *b, const double *x_in);
int qb_batch_get_velocities_all(qb_batch *b, double *v_out);
int qb_batch_set_velocities_all(qb_batch *b, const double *v_in);

/* Water polarisation shell corrections (float theta_corr, md.f90:15205). */
int qb_batch_get_theta_corr(qb_batch *b, int sys, float *out, int n);

/* Energy records gathered during qb_batch_run for system `sys`:
 * count = number of records; steps[i], E[i*QB_NE...], EQ[i*nstates*QB_NEQ...],
 * kin (E%kinetic at the record) included in E.  Buffers may be NULL to query
 * the count.  kind: 0 = output summaries (iout_cycle), 1 = energy file (iene_cycle). */
int qb_batch_history(qb_batch *b, int sys, int kind, int *count, int *steps,
                     double *E, double *EQ);
int qb_batch_clear_history(qb_batch *b);

/* Records of every system at once (kind as above), in two device copies.
 * One record is QB_HIST_REC doubles: step, E[QB_NE], EQ[QB_MAX_STATES][QB_NEQ],
 * r_kl[QB_MAX_STATES] (the off-diagonal distances).  counts: nsys ints, the
 * records of each system (at most max_records are returned); records:
 * nsys*max_records*QB_HIST_REC doubles, system s's record r at
 * (s*max_records + r)*QB_HIST_REC.  With records NULL, counts receives every
 * system's full record count (max_records is not applied).  bytes (may be
 * NULL) receives the bytes copied from the device. */
#define QB_HIST_REC (1 + QB_NE + QB_MAX_STATES * QB_NEQ + QB_MAX_STATES)
int qb_batch_history_all(qb_batch *b, int kind, int max_records, int *counts, double *records, size_t *bytes);

/* Steps taken by the batch since it was created (the host's step counter;
 * a system that failed stops its own count, qb_batch_status). */
int qb_batch_step_count(qb_batch *b, long long *out);

/* Periodic box of system `sys`: box6 = edge lengths (3) then centre (3), as
 * the restart file's box records hold them; tries/accepted (may be NULL): the
 * Monte Carlo volume moves of a constant-pressure run so far.  Zeros for a
 * sphere.  Replaces: boxlength/boxcenter, volume_try/volume_acc,
 * src/q6/md.f90:15452-15475, 15812-15816. */
int qb_batch_box(qb_batch *b, int sys, double *box6, long long *tries, long long *accepted);

/* The off-diagonal elements of the same records: for every record and every
 * off-diagonal function io of the system's FEP file, Hij = A exp(-mu r_kl)
 * and r_kl, the distance of its two Q atoms at that step (offdiag,
 * src/q6/md.f90:12911-12937).  out: count*noffd*2 doubles (Hij, r_kl), or
 * NULL to query the count.  kind 2 gives one record: the values of the
 * latest force evaluation in the run loop (those qdyn's final summary prints). */
int qb_batch_offdiag(qb_batch *b, int sys, int kind, int *count, double *out);

/* Run-time choices of the step kernels.  No counterpart in the reference
 * (qdyn has no tile sizes).  None changes the model: only the order in which
 * atomic sums add up, so results differ at rounding level. */
typedef struct qb_tuning {
  int lrf_tiles_per_block;    /* source-group tiles one block of the LRF gather sweeps (>= 1) */
  int ww_chunk;               /* waters staged in shared memory per pass of the water-water kernel:
                                 a multiple of 32 between ww_chunk_min and ww_chunk_max */
  int side_streams;           /* 1: a step's force kernels fork over two side streams; 0: one stream */
  int ww_waters_per_block;    /* waters of one system per block of the water-water kernels: a multiple of
                                 32 up to 256 (smaller blocks: more of them, a shorter last wave, more
                                 staging of each system's records) */
  int water_pass_per_atom;    /* 1: the water pass takes one thread per water atom (the default when three
                                 threads per water fit on the GPU at once); 0: one thread per water */
  int ww_chunk_min, ww_chunk_max;  /* the batch's allowed range (read only) */
  int trials;                 /* autotune: settings timed */
  double ms_per_step;         /* autotune: device ms per step of the chosen setting */
  double ms_per_step_before;  /* autotune: of the setting it started from */
} qb_tuning;

int qb_batch_get_tuning(qb_batch *b, qb_tuning *out);
/* Applies lrf_tiles_per_block, ww_chunk, side_streams, ww_waters_per_block and
 * water_pass_per_atom (QB_ERR_ARG when out of range); the pair lists are rebuilt
 * before the next step. */
int qb_batch_set_tuning(qb_batch *b, const qb_tuning *t);
/* Times steps_per_trial MD steps (rounded up to whole pair-list cycles, each
 * after a cycle of warm-up) for candidate settings, one parameter at a time
 * (LRF tiles per block 1..16, the water chunk at its maximum, a half and a
 * quarter, 32/64/128/192/256 waters per water-water block, the water pass's
 * threads per water or per atom, side streams on/off),
 * keeps the fastest and reports it.  The trial
 * steps are real MD steps of every system (count them as equilibration); the
 * energy records they make are cleared. */
int qb_batch_autotune(qb_batch *b, int steps_per_trial, qb_tuning *out);

/* Per-system status (enum qb_status) raised on the device, e.g. QB_ERR_SHAKE. */
int qb_batch_status(qb_batch *b, int sys, int *status);

/* Kernel timing: when enabled, every kernel launch in qb_batch_run is bracketed
 * with CUDA events on the batch stream.  names/ms/launches receive up to n
 * entries (names as a '\n'-separated list). */
int qb_batch_set_profiling(qb_batch *b, int on);
int qb_batch_profile(qb_batch *b, char *names, size_t names_len, double *ms,
                     long long *launches, int n, int *n_kernels);

/* Device work totals of the last qb_batch_run (for roofline arithmetic):
 * out[0] ww molecule pairs/step (sum over systems), out[1] pw pairs,
 * out[2] pp pairs, out[3] qp pairs, out[4] qw (q, water) pairs, out[5] atoms,
 * out[6] shake constraints, out[7] charge groups, out[8] SHAKE iterations per
 * molecule and step on average (the niter shake() returns, md.f90:14560),
 * out[9] most SHAKE iterations of one molecule in one step.  Fills up to n
 * (at most QB_WORKLOAD_N) entries. */
#define QB_WORKLOAD_N 10
int qb_batch_workload(qb_batch *b, double *out, int n);

void qb_batch_destroy(qb_batch *b);

/* ------------------------------------------------------ allocation-free path */

#define QB_STATIC_WW_MAX_WATERS 4096
#define QB_STATIC_WW_MAX_NEIGHBOURS 192
#define QB_STATIC_WW_SCRATCH_BYTES \
  ((size_t)(QB_STATIC_WW_MAX_WATERS * QB_STATIC_WW_MAX_NEIGHBOURS + QB_STATIC_WW_MAX_WATERS) * 4)

/* SPC/TIP3P water-water electrostatic and Lennard-Jones energy and gradient of
 * one water sphere, computed on buffers the caller owns, with no device memory
 * allocated by the call.  This entry point has no counterpart in the
 * reference.  It exists for hosts that cannot let a library call cudaMalloc:
 * callers that hand out device memory only from their own pool (a framework's
 * caching allocator, a pre-sized arena in a long-running service) or that
 * forbid allocation on the calling thread.
 *
 * x:      device, 9*nwat doubles, waters as O,H,H with x,y,z each
 * crg_ow, crg_hw: the O and H charges already multiplied by the square root
 *         of the Coulomb constant, as qdyn stores them after prep_sim
 *         (src/q6/md.f90:13884-13891) and as qb_sysview's crg_ow/crg_hw hold
 *         them: for TIP3P with the default constant 332, crg_ow =
 *         -0.834f*sqrtf(332).  Plain topology charges give an electrostatic
 *         energy 332 times too small; the call cannot detect that.
 * A_OO, B_OO: the O-O Lennard-Jones products, E = A_OO/r^12 - B_OO/r^6 (for
 *         the geometric rule the products of the O type's avdw and bvdw
 *         columns, A = 4*eps*sigma^12, B = 4*eps*sigma^6), as qb_sysview's
 *         A_OO/B_OO hold them.
 * cutoff: the O-O cut-off (Angstrom) of the neighbour list.
 * excl:   device, nwat flags (1 = water outside the sphere), or NULL
 * grad:   device, 9*nwat doubles, overwritten with dU/dx
 * energy: device, 2 doubles, overwritten with (electrostatic, van der Waals)
 * status: device, 1 int, overwritten: 0, or QB_ERR_LIST_OVERFLOW when a water
 *         has more than QB_STATIC_WW_MAX_NEIGHBOURS neighbours
 * stream: cudaStream_t (NULL = default stream); the work is queued on it and
 *         the call returns without waiting.
 *
 * Its scratch (the neighbour list) is a fixed array in the library's device
 * memory: every GPU that loads the library holds QB_STATIC_WW_SCRATCH_BYTES
 * (about 3 MB) until the process exits.  Systems above
 * QB_STATIC_WW_MAX_WATERS waters are rejected with QB_ERR_ARG.  All calls on a
 * device share that array and it keeps the last call's contents (the call
 * rewrites everything it reads), so calls that overlap on the GPU -- on two
 * streams, or from two threads -- race and must be serialised by the caller.
 * The first call on each device (per CUDA context) looks up the array's device
 * address with that device current; make that first call before any stream
 * capture.  A cudaDeviceReset discards the array with the context; the next
 * call in the new context looks the address up again. */
int qb_ww_energy_static(const double *x, int nwat, float crg_ow, float crg_hw, double A_OO, double B_OO,
                        double cutoff, const unsigned char *excl, double *grad, double *energy, int *status,
                        void *stream);

/* Measured FMA throughput of the CUDA cores of `device` (TFLOP/s, FMA = 2
 * FLOP) in FP64 (precision QB_FP64) or FP32 (QB_MIXED): the denominator of the
 * pair kernels' roofline. */
int qb_peak_flops(int device, int precision, double *tflops);

/* ------------------------------------------------------------------ files */

/* Write a qdyn restart file: gfortran unformatted sequential records
 * (nat3, x), (nat3, v), and (nshell, theta_corr) when nshell > 0.
 * Replaces: write_xfin, src/q6/md.f90:15452-15470. */
int qb_write_re(const char *path, int natom, const double *x, const double *v,
                int nshell, const float *theta_corr);

/* The same with a periodic box's two records after them: box6 = edge
 * lengths, then centre (md.f90:15471-15474). */
int qb_write_re_box(const char *path, int natom, const double *x, const double *v,
                    int nshell, const float *theta_corr, const double *box6);

/* Append one energy-file frame: per state a record (int32 state, 15 doubles)
 * and one empty off-diagonal record.  Replaces: put_ene, src/q6/nrgy.f90:94-119. */
int qb_append_en(const char *path, int nstates, const double *EQ);

/* The same frame with its off-diagonal record: noffd entries of (int32 i,
 * int32 j, double Hij, double r_kl), nrgy.f90:60-65.  ij: 2*noffd state
 * numbers (1-based); hr: 2*noffd doubles (Hij, r_kl). */
int qb_append_en_offd(const char *path, int nstates, const double *EQ, int noffd, const int *ij, const double *hr);

/* Maxwell-Boltzmann velocities drawn exactly as qdyn draws them: gauss (12
 * uniforms from randm) per component, sd = sqrt(boltz*T/mass), before initial
 * shaking.  v_out: 3*natom doubles.
 * Replaces: maxwell/gauss/randm, src/q6/md.f90:3787-3810, 1453-1469, 14408-14442. */
int qb_maxwell(int seed, double temperature, int natom, const double *mass, double *v_out);

#ifdef __cplusplus
}
#endif
#endif /* QB_H */
