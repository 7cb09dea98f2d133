// Host-side mesh database: the single-partition restatement of the NEXD-3D
// mesher (program_mesher -> createMesh, src/meshMod.f90:45-1393) plus the
// solver-side preparation timeloop3D does before its hot loop
// (src/timeloopMod.f90:137-356).  Produces the nexd_desc consumed by the GPU
// library and by the CPU oracle.
#pragma once
#include <string>
#include <vector>

#include "../../include/nexd.h"
#include "dg_operators.hpp"

namespace nexd {

// Parameters read from data/parfile (src/parameterMod.f90:30-103).
struct Parfile {
  bool log = false, external = true, vtk = false, movie = false, attenuation = false, set_pml = false;
  int nproc = 1, frame = 10, timeint = 2, nt = 1000;
  double cfl = 0.4, f0_att = 1.0, fr_att = 1.0;
  double pml_delta = 0.0, pml_rc = 0.01, pml_kmax = 1.0, pml_afac = 1.0;
  int avg_window1 = 10, avg_window2 = 2;
  double sta_lta_trigger = 0.1;
};

struct Source {
  double xyz[3] = {0, 0, 0};
  int type = 0;  // 0 force, 1 moment tensor
  int stf = 2;   // 1 Gauss, 2 Ricker
  double f0 = 1.0, factor = 1.0;
  double angle_force[3] = {0, 0, 1};  // normalised at read time
  double M[6] = {0, 0, 0, 0, 0, 0};   // Mxx Myy Mzz Mxy Mxz Myz
  // located
  int elem = 0;  // 1-based
  double rst[3] = {0, 0, 0};
};

struct Receiver {
  int nr = 0;
  double xyz[3] = {0, 0, 0};
  int elem = 0;  // 1-based
  double rst[3] = {0, 0, 0};
};

struct BuildOptions {
  int N = 4;                 // polynomial order
  int timeint = -1;          // override par%timeint when > 0 (4 = LSERK4)
  double cfl = -1.0;         // override par%cfl when > 0
  int nt = -1;               // override par%nt when > 0
  double t0 = -1.0;          // source time shift; <0: reference 1.2/f0 (src/sourceReceiverMod.f90:765)
  int stf_stage_time = 0;    // 1: evaluate the STF at each RK stage time
  double init_value = 1e-24; // src/timeloopMod.f90:184-195
  int nbatch = 1;            // independent wavefields; sources are dealt round-robin
};

struct MeshDB {
  int N = 0, Np = 0, NpF = 0, nelem = 0, nglob = 0, ncoord = 0, nMB = 0;
  DGOperators op;
  Parfile par;
  BuildOptions opt;
  std::vector<double> coord;  // (3,ncoord)
  std::vector<int> elem;      // (4,K) 1-based vertex ids
  std::vector<int> neighbor;  // (4,K) 1-based, 0 boundary
  std::vector<int> face;      // (4,K)
  std::vector<int> mat, pml;  // (K)
  int nmat = 0;
  std::vector<double> matval;  // (nmat,11): rho vp vs mu lambda qp qs (cubit/matprop, src/meshMod.f90:261-272)
  std::vector<double> vp, vs, rho, qp, qs, mu, lambda, vpu, vsu, muu, lambdau;  // (K)
  std::vector<double> ylambda, ymu;  // (nMB,K)
  std::vector<double> wl, wk;
  std::vector<double> metric, jac, sJ, fscale;     // (9,K) (K) (4,K) (4,K)
  std::vector<double> nn, st, tt;                  // (3,4,K)
  std::vector<double> vx, vy, vz;                  // (K*Np)
  std::vector<int> ibt, ibn;                       // (NpF,4,K) 1-based
  std::vector<int> fmask1;                         // (NpF,4) 1-based
  double dtfactor = 0.0, minGLL_jac = 0.0, dt = 0.0;
  double pmlxmin = 0, pmlxmax = 0, pmlymin = 0, pmlymax = 0, pmlzmin = 0, pmlzmax = 0;
  // PML
  std::vector<int> pmlcheck;        // (K)
  std::vector<double> pml_profiles; // (K*Np,9)
  // sources / receivers
  std::vector<Source> src;
  std::vector<Receiver> rec;
  std::vector<int> srcelem, srctype, recelem, srcbatch;
  std::vector<double> srcInt, srcangle, srcM, stf, recInt;
  int stf_per_step = 1;
  double f0max = 0.0;
  // column-major flattened operators
  std::vector<double> Dr, Ds, Dt, lift, invmass, mass, V;
  nexd_desc desc{};
  std::vector<std::string> warnings;
};

// Reads a reference simulation directory (cubit/{coord,mesh,mat,matprop,free,
// absorb}, data/{parfile,source,stations}) and builds the database.
// Throws std::runtime_error with a message on any inconsistency the reference
// mesher would stop on.
void build_from_directory(const std::string& dir, const BuildOptions& opt, MeshDB& db);

// Reads data/parfile of `dir` into db.par and applies the option overrides.
void init_parameters(const std::string& dir, const BuildOptions& opt, MeshDB& db);

// Solver-side set-up once mesh, sources and receivers are known: NPML
// profiles, source/receiver interpolation and STF tables, operators in the
// descriptor (src/timeloopMod.f90:137-356).
void prepare_solver(MeshDB& db);

// Database files of the reference's mesher -> solver hand-off for one
// partition (nproc = 1): out/meshVar000001 (writeMeshVar / readMeshVar,
// src/meshMod.f90:1401-1640), srcVar000001 / recVar000001 (writeSrcVar,
// writeRecVar, readSrcVar, readRecVar, src/sourceReceiverMod.f90:615-702),
// as Fortran sequential unformatted records.
void write_database(const MeshDB& db, const std::string& outdir);
// Builds the database from `dir`/data/parfile and the files above in
// `dir`/out, as the reference's timeloop3D does with readMesh / readSrc /
// readRec (src/timeloopMod.f90:137-160).  The order comes from the files.
void build_from_database(const std::string& dir, const BuildOptions& opt, MeshDB& db);

// Parfile / source-file readers (src/parameterMod.f90, src/fileParameterMod.f90,
// src/sourceReceiverMod.f90:36-201).
Parfile read_parfile(const std::string& path);
std::vector<Source> read_sources(const std::string& path);
std::vector<Receiver> read_stations(const std::string& path);

// Source-time functions (src/stfMod.f90:25-45).
double stf_ricker(double t, double f0, double t0, double factor);
double stf_gauss(double t, double f0, double t0, double factor);

// Zener fit (src/anelasticMod.f90:27-179).
void anelastic_precalc(double f0, double fr, int nMB, std::vector<double>& wl, std::vector<double>& wk);
void anelastic_coefficients(double Qp, double Qs, double vp, double vs, double rho, double f0,
                            const std::vector<double>& wl, const std::vector<double>& wk, double* ylambda,
                            double* ymu, double& lambda_u, double& mu_u);

// Writes reference seismogram files seismo.{x,y,z}.%07d.sd{u,v,a} from traces
// (nrec, nt, 9) with time axis t(it) = it*dt (src/timeloopMod.f90:319-321,591-620).
void write_seismograms(const std::string& outdir, const MeshDB& db, const float* traces, int nt, int batch);

}  // namespace nexd
