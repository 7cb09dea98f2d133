/*
 * nexd_solve -- command-line driver of the B200 time loop, in plain C.
 *
 * The C counterpart of program_solver (src/program_solver.f90:71 calling
 * timeloop3D, src/timeloopMod.f90:42-674) for a single partition: it reads a
 * reference simulation directory -- the mesher inputs cubit/{coord,mesh,mat,
 * matprop,free,absorb} with data/{parfile,source,stations}, or with
 * --database the files the reference's mesher writes (out/meshVar000001,
 * srcVar000001, recVar000001, as readMesh / readSrc / readRec read them) --
 * through libnexd_host.so, runs every time step on the GPU through the C-ABI
 * of libnexd.so (nexd_create / nexd_run / nexd_get_traces / nexd_destroy),
 * and writes the reference's seismogram files out/seismo.{x,y,z}.%07d.sd{u,v,a}
 * (src/timeloopMod.f90:591-620) and, with the NPML trigger armed, the energy
 * history out/energy (src/timeloopMod.f90:637-641).
 *
 *   nexd_solve <simulation dir> [--database] [--order N] [--cfl C] [--nt NT]
 *              [--contraction fp32|bf16x3|auto] [--trigger W1,W2,THRESHOLD,F0]
 *              [--out DIR]
 *
 * Exit status 0 on success; on failure the library's message is printed and
 * the status is the nexd_status code (the reference stops instead).
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "nexd.h"
#include "nexd_host.h"

static int fail_host(const char* what, int st) {
  char msg[512];
  nexd_mesh_last_error(msg, sizeof msg);
  fprintf(stderr, "nexd_solve: %s failed (%d): %s\n", what, st, msg);
  return st;
}

static int fail_gpu(const nexd_ctx* ctx, const char* what, int st) {
  char msg[512];
  nexd_last_error(ctx, msg, sizeof msg);
  fprintf(stderr, "nexd_solve: %s failed (%d): %s\n", what, st, msg);
  return st;
}

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* Two-column ASCII time series, one line per step, step it at (it - 1) dt:
 * the time axis of the reference's own output files (its seismograms start
 * at t = 0, simulations/brick/ref/seismo.*). */
static int write_energy(const char* outdir, const double* energy, int nt, double dt) {
  char path[8192];
  snprintf(path, sizeof path, "%s/energy", outdir);
  FILE* f = fopen(path, "w");
  if (!f) return NEXD_ERR_INVALID;
  for (int it = 1; it <= nt; ++it) fprintf(f, "%15.7e %15.7e\n", (it - 1) * dt, energy[it - 1]);
  fclose(f);
  return NEXD_OK;
}

static void usage(void) {
  fprintf(stderr,
          "usage: nexd_solve <simulation dir> [--database] [--order N] [--cfl C] [--nt NT]\n"
          "                  [--contraction fp32|bf16x3|auto] [--trigger W1,W2,THRESHOLD,F0] [--out DIR]\n");
}

int main(int argc, char** argv) {
  if (argc < 2 || argv[1][0] == '-') {
    usage();
    return NEXD_ERR_INVALID;
  }
  const char* dir = argv[1];
  const char* outdir = NULL;
  int database = 0, contraction = NEXD_CONTRACT_FP32, trigger = 0;
  int w1 = 10, w2 = 2;
  double thr = 0.1, f0 = 1.0;
  nexd_build_opts o;
  memset(&o, 0, sizeof o);
  o.N = 4;
  o.init_value = 1e-24; /* the reference's start value of every field */
  for (int i = 2; i < argc; ++i) {
    const char* a = argv[i];
    const char* v = i + 1 < argc ? argv[i + 1] : NULL;
    if (!strcmp(a, "--database")) {
      database = 1;
    } else if (!strcmp(a, "--order") && v) {
      o.N = atoi(v), ++i;
    } else if (!strcmp(a, "--cfl") && v) {
      o.cfl = atof(v), ++i;
    } else if (!strcmp(a, "--nt") && v) {
      o.nt = atoi(v), ++i;
    } else if (!strcmp(a, "--out") && v) {
      outdir = v, ++i;
    } else if (!strcmp(a, "--contraction") && v) {
      if (!strcmp(v, "fp32")) contraction = NEXD_CONTRACT_FP32;
      else if (!strcmp(v, "bf16x3")) contraction = NEXD_CONTRACT_BF16X3;
      else if (!strcmp(v, "auto")) contraction = NEXD_CONTRACT_AUTO;
      else { usage(); return NEXD_ERR_INVALID; }
      ++i;
    } else if (!strcmp(a, "--trigger") && v) {
      if (sscanf(v, "%d,%d,%lf,%lf", &w1, &w2, &thr, &f0) != 4) { usage(); return NEXD_ERR_INVALID; }
      trigger = 1, ++i;
    } else {
      usage();
      return NEXD_ERR_INVALID;
    }
  }
  char outbuf[4096];
  if (!outdir) {
    snprintf(outbuf, sizeof outbuf, "%s/out", dir);
    outdir = outbuf;
  }
  mkdir(outdir, 0755); /* the reference's out/ directory; an existing one is kept */

  /* readMesh / readSrc / readRec / prepareSources (src/timeloopMod.f90:137-300) */
  nexd_mesh* mesh = NULL;
  int st = database ? nexd_mesh_load_database(dir, &o, &mesh) : nexd_mesh_build(dir, &o, &mesh);
  if (st) return fail_host(database ? "reading the database files" : "building the mesh", st);
  const nexd_desc* d = nexd_mesh_desc(mesh);

  /* the time loop (src/timeloopMod.f90:357-589) on the GPU */
  nexd_ctx* ctx = NULL;
  st = nexd_create(d, &ctx);
  if (st) {
    fail_gpu(NULL, "nexd_create", st);
    nexd_mesh_free(mesh);
    return st;
  }
  if (contraction != NEXD_CONTRACT_FP32 && (st = nexd_set_contraction(ctx, contraction))) goto gpu_error;
  if (trigger && (st = nexd_pml_trigger(ctx, w1, w2, thr, f0, 0))) goto gpu_error;
  const double t_start = now_s();
  if ((st = nexd_run(ctx, 1, d->nt))) goto gpu_error;
  const double t_run = now_s() - t_start;

  /* seismograms (src/timeloopMod.f90:591-620) */
  const size_t ntr = (size_t)d->nrec * d->nt * NEXD_NCOMP * d->nbatch;
  float* traces = (float*)malloc((ntr ? ntr : 1) * sizeof(float));
  if (!traces) { st = NEXD_ERR_NOMEM; goto gpu_error; }
  if ((st = nexd_get_traces(ctx, traces))) { free(traces); goto gpu_error; }
  if (d->nrec > 0 && (st = nexd_mesh_write_seismograms(mesh, outdir, traces, d->nt, 0))) {
    free(traces);
    nexd_destroy(ctx);
    int rc = fail_host("writing the seismograms", st);
    nexd_mesh_free(mesh);
    return rc;
  }
  free(traces);
  if (trigger) {
    double* energy = (double*)calloc((size_t)d->nt * d->nbatch, sizeof(double));
    int32_t* sw = (int32_t*)calloc((size_t)d->nbatch, sizeof(int32_t));
    if (!energy || !sw) { free(energy); free(sw); st = NEXD_ERR_NOMEM; goto gpu_error; }
    if ((st = nexd_get_energy(ctx, energy, sw))) { free(energy); free(sw); goto gpu_error; }
    write_energy(outdir, energy, d->nt, d->dt);
    if (sw[0] > 0) printf("PML was switched off at time step %d\n", sw[0]);
    free(energy);
    free(sw);
  }
  printf("nexd_solve: %d elements, N=%d, dt=%.9e, %d steps in %.3f s; seismograms of %d receivers in %s\n",
         d->nelem, d->N, d->dt, d->nt, t_run, d->nrec, outdir);
  nexd_destroy(ctx);
  nexd_mesh_free(mesh);
  return 0;

gpu_error:
  fail_gpu(ctx, "the time loop", st);
  nexd_destroy(ctx);
  nexd_mesh_free(mesh);
  return st;
}
