/*
 * oracle.h -- CPU oracle for the NEXD-3D time loop (TEST INFRASTRUCTURE).
 *
 * A C++ restatement of subroutine timeloop3D (src/timeloopMod.f90:42-674)
 * with waveMod (src/waveMod.f90:29-405) and rungekuttaMod
 * (src/rungekuttaMod.f90:27-120), run on the same nexd_desc the GPU library
 * consumes.  It is the checker for the GPU path: only the tests, the smoke
 * check and the CPU-baseline leg of bench.py call it.  Nothing in the
 * product (libnexd.so, libnexd_host.so, the nexd_b200 package) links or
 * calls it.
 *
 * Pinning: in FP32 with the reference's RK2 it reproduces the reference's
 * own golden seismograms simulations/brick/ref/seismo.* (see tests).
 */
#ifndef NEXD_ORACLE_H
#define NEXD_ORACLE_H

#include "../include/nexd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Runs steps 1..it_end.  precision: 32 or 64.  traces: (nrec,nt,9,nbatch),
 * zero-filled beyond it_end.  field (may be NULL): final q, (K*Np,9,nbatch)
 * in FP64.  nthreads <= 0 uses all OpenMP threads.  Returns 0 or an error
 * code (message via oracle_last_error). */
int oracle_run(const nexd_desc* d, int precision, int it_end, float* traces, double* field, int nthreads);

/* One right-hand side evaluation for batch member 0 at step `it` (1-based)
 * and stage `stage` (0-based).  Inputs (FP64): q (K*Np,9); theta
 * (K*Np,6*nMB) or NULL (start value); aux (K*Np,27) or NULL (zero).  Outputs:
 * rq (K*Np,9); arq (K*Np,6*nMB) or NULL; auxr (K*Np,27) or NULL (zero outside
 * PML elements). */
int oracle_rhs(const nexd_desc* d, int precision, int it, int stage, const double* q, const double* theta,
               const double* aux, double* rq, double* arq, double* auxr);

/* oracle_run with the reference's NPML energy and STA/LTA trigger
 * (src/timeloopMod.f90:482-542) armed: energy (nt, nbatch) FP64 history,
 * pml_switch (nbatch) step at which the NPML was switched off (0 = never).
 * formula 0: the reference's strain expression; 1: isotropic compliance. */
int oracle_run_trigger(const nexd_desc* d, int precision, int it_end, float* traces, double* field, int nthreads,
                       int avg_window1, int avg_window2, double sta_lta_trigger, double f0, int formula,
                       double* energy, int* pml_switch);

int oracle_last_error(char* buf, size_t len);

/* Seconds the last oracle_run / oracle_run_trigger on this thread spent in its
 * time-step loop (operator and state set-up excluded): the CPU baseline's
 * timed region. */
double oracle_loop_seconds(void);

/* Reproduces two of the reference's quirks in later oracle_run calls (all
 * threads; 0 restores the default, a correct NPML):
 *   bit 1  the NPML auxiliary equation of every PML element is driven by the
 *          flux arrays ftemp/gtemp/htemp as the element loop leaves them, i.e.
 *          the LAST element's flux (src/rungekuttaMod.f90:52-63 called with
 *          them at src/timeloopMod.f90:479-480); the default uses each
 *          element's own flux;
 *   bit 2  the flux columns elasticFluxes never writes (f(:,5), g(:,6),
 *          h(:,4), src/waveMod.f90:37-62) keep the values the previous element
 *          left in them; the default has them zero.
 * With either bit the element loop runs serially in mesh order, as in the
 * reference.  Returns 0, or NEXD_ERR_INVALID for flags outside 0..3. */
int oracle_set_ref_quirks(int flags);

#ifdef __cplusplus
}
#endif

#endif
