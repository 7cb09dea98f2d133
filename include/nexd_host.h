/*
 * nexd_host.h -- C-ABI of the host-side database builder (libnexd_host.so).
 *
 * Stands in for the Fortran host of the reference where no Fortran compiler
 * exists: it reads a reference simulation directory (cubit/coord, mesh, mat,
 * matprop, free, absorb; data/parfile, source, stations), restates the
 * single-partition mesher createMesh (src/meshMod.f90:45-1393) and the
 * pre-loop set-up of timeloop3D (src/timeloopMod.f90:137-356), and hands out
 * the nexd_desc that libnexd.so's nexd_create consumes.  It also writes the
 * reference seismogram files (src/timeloopMod.f90:591-620, src/plotMod.f90:27-38).
 */
#ifndef NEXD_HOST_H
#define NEXD_HOST_H

#include "nexd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nexd_mesh nexd_mesh;

typedef struct nexd_build_opts {
  int32_t N;              /* polynomial order (the reference's compile-time ORDER) */
  int32_t timeint;        /* > 0 overrides par%timeint (4 = LSERK4) */
  double cfl;             /* > 0 overrides par%cfl */
  int32_t nt;             /* > 0 overrides par%nt */
  double t0;              /* > 0 overrides the reference's t0 = 1.2/f0 */
  int32_t stf_stage_time; /* 1: sample the STF at each RK stage time */
  double init_value;      /* start value of the fields (reference: 1e-24) */
  int32_t nbatch;         /* independent wavefields; source i drives wavefield i % nbatch */
} nexd_build_opts;

typedef struct nexd_mesh_info {
  double dtfactor;   /* mesh%dtfactor (src/meshMod.f90:1134-1155) */
  double dt;         /* dtfactor * cfl */
  double minGLL;
  double cfl;
  int32_t nglob;
  int32_t ncoord;
  const double* vx; /* (nglob) node coordinates */
  const double* vy;
  const double* vz;
  const double* mass;  /* (Np,Np) */
  const double* vdm;   /* (Np,Np) */
  const double* src_rst; /* (3,nsrc) located reference coordinates */
  const double* rec_rst; /* (3,nrec) */
  const int32_t* recnr;  /* (nrec) station numbers */
  const double* mu;      /* (K) relaxed (or unrelaxed when attenuation is on) */
  const double* lambda;  /* (K) */
  int32_t n_warnings;
} nexd_mesh_info;

/* Reads directory `dir` and builds the database.  opts may be NULL (defaults:
 * N=4, parfile values, reference t0 and STF sampling, init 1e-24). */
int nexd_mesh_build(const char* dir, const nexd_build_opts* opts, nexd_mesh** out);

/* Writes the reference's database files for one partition into `outdir`:
 * meshVar000001 (writeMeshVar, src/meshMod.f90:1401-1504) and, when the mesh
 * has sources / receivers, srcVar000001 / recVar000001 (writeSrcVar /
 * writeRecVar, src/sourceReceiverMod.f90:615-648), as Fortran sequential
 * unformatted records with 4-byte markers, REAL(4) and INTEGER(4) data. */
int nexd_mesh_write_database(const nexd_mesh* mesh, const char* outdir);

/* Builds the database from `dir`/data/parfile and `dir`/out/{meshVar,srcVar,
 * recVar}000001 -- the files the reference's mesher writes with nproc = 1 --
 * as timeloop3D's readMesh / readSrc / readRec do (src/timeloopMod.f90:137-160,
 * src/meshMod.f90:1506-1640, src/sourceReceiverMod.f90:653-741).  The order
 * comes from the files (opts->N is ignored); a partition with MPI interfaces
 * is rejected with NEXD_ERR_INVALID. */
int nexd_mesh_load_database(const char* dir, const nexd_build_opts* opts, nexd_mesh** out);

/* Descriptor view into the database; valid until nexd_mesh_free. */
const nexd_desc* nexd_mesh_desc(const nexd_mesh* mesh);

int nexd_mesh_get_info(const nexd_mesh* mesh, nexd_mesh_info* out);

/* Writes out/seismo.{x,y,z}.%07d.sd{u,v,a} for batch member `batch` from
 * traces laid out as nexd_get_traces returns them, nt_written rows each. */
int nexd_mesh_write_seismograms(const nexd_mesh* mesh, const char* outdir, const float* traces,
                                int32_t nt_written, int32_t batch);

/* ---- Partitions: the mesher's domain decomposition for nproc > 1 ------------
 * The reference's mesher partitions the elements with METIS and hands every
 * rank its elements and the interface arrays (src/meshMod.f90:382-504,
 * 669-1110).  nexd_partition_create splits a descriptor into `nparts`
 * partition descriptors, each with the halo descriptor nexd_create_partition
 * takes: `part` (K values, 0-based) gives each element's partition (a METIS
 * result, for instance) or, when NULL, the elements are split by recursive
 * coordinate bisection of the centroids `centroid` (3,K) into parts whose
 * sizes differ by at most one.  Partition descriptors keep the elements,
 * sources and receivers in their original order and share the operators with
 * `desc`, which must outlive the partition set. */
typedef struct nexd_partition nexd_partition;
typedef struct nexd_part_view {
  const nexd_desc* desc;
  const nexd_halo_desc* halo;
  int32_t nelem;
  const int32_t* elem_global; /* (nelem) 1-based element in the whole mesh */
  int32_t nsrc;
  const int32_t* src_global;  /* (nsrc) 1-based source in the whole mesh */
  int32_t nrec;
  const int32_t* rec_global;  /* (nrec) 1-based receiver in the whole mesh */
} nexd_part_view;
int nexd_partition_create(const nexd_desc* desc, int32_t nparts, const int32_t* part, const double* centroid,
                          nexd_partition** out);
/* View of partition `index` (0-based); valid until nexd_partition_free. */
int nexd_partition_get(const nexd_partition* parts, int32_t index, nexd_part_view* out);
int nexd_partition_count(const nexd_partition* parts, int32_t* nparts);
void nexd_partition_free(nexd_partition* parts);

/* Message of the last failed call on this thread. */
int nexd_mesh_last_error(char* buf, size_t len);

void nexd_mesh_free(nexd_mesh* mesh);

#ifdef __cplusplus
}
#endif

#endif /* NEXD_HOST_H */
