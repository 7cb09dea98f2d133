// CPU oracle: restatement of NEXD-3D's timeloop3D (TEST INFRASTRUCTURE; see
// oracle.h).  Templated on the working precision so it can run as the
// reference does (FP32, CUSTOM_REAL = SIZE_REAL, src/constants.h:25) and in
// FP64.
//
// Formulation notes (each is an algebraic identity of the reference's code,
// not a change of method):
//  * volume term: the reference evaluates dFdr = Dr*F etc. (81 matvecs) and
//    combines rq = rx*dFdr + sx*dFds + tx*dFdt + ... (src/timeloopMod.f90:
//    407-420).  For affine elements rx..tz are element constants, so the
//    oracle forms Dx = rx*Dr + sx*Ds + tx*Dt once per element and applies it
//    to the same flux columns F, G, H;
//  * the NPML auxiliary equation uses each element's own flux F
//    (dF'/dt = -alpha F' - d/kappa (F' + F)).  The reference passes the flux
//    arrays of the last element of the loop to RungeKuttaSteps
//    (src/timeloopMod.f90:479-480 with src/rungekuttaMod.f90:52-63), which
//    applies one element's flux to all PML elements; the oracle follows the
//    NPML equations instead;
//  * elasticFluxes leaves F(:,5), G(:,6), H(:,4) unwritten
//    (src/waveMod.f90:37-62); outside PML elements they hold zero, and the
//    oracle uses zero everywhere.
#include "oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;
// seconds spent in the time-step loop of the last oracle_run (set-up excluded)
thread_local double g_loop_seconds = 0.0;
// Reference quirks reproduced on request (oracle_set_ref_quirks): bit 1 the
// NPML auxiliary equation driven by the last element's flux, bit 2 the flux
// columns elasticFluxes never writes carried over from element to element.
int g_ref_quirks = 0;

// Carpenter & Kennedy (1994) five-stage fourth-order 2N-storage coefficients.
const double kRK4A[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                         -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kRK4B[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                         1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                         2277821191437.0 / 14882151754819.0};

template <class R>
using M9 = R[9][9];

template <class R>
void getT(const double* n, const double* s, const double* t, R T[9][9]) {
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) T[i][j] = 0;
  // src/waveMod.f90:161-213
  R n1 = n[0], n2 = n[1], n3 = n[2], s1 = s[0], s2 = s[1], s3 = s[2], t1 = t[0], t2 = t[1], t3 = t[2];
  T[0][0] = n1 * n1; T[0][1] = s1 * s1; T[0][2] = t1 * t1; T[0][3] = 2 * n1 * s1; T[0][4] = 2 * s1 * t1; T[0][5] = 2 * n1 * t1;
  T[1][0] = n2 * n2; T[1][1] = s2 * s2; T[1][2] = t2 * t2; T[1][3] = 2 * n2 * s2; T[1][4] = 2 * s2 * t2; T[1][5] = 2 * n2 * t2;
  T[2][0] = n3 * n3; T[2][1] = s3 * s3; T[2][2] = t3 * t3; T[2][3] = 2 * n3 * s3; T[2][4] = 2 * s3 * t3; T[2][5] = 2 * n3 * t3;
  T[3][0] = n2 * n1; T[3][1] = s2 * s1; T[3][2] = t2 * t1; T[3][3] = n2 * s1 + n1 * s2; T[3][4] = s2 * t1 + s1 * t2; T[3][5] = n2 * t1 + n1 * t2;
  T[4][0] = n3 * n2; T[4][1] = s3 * s2; T[4][2] = t3 * t2; T[4][3] = n3 * s2 + n2 * s3; T[4][4] = s3 * t2 + s2 * t3; T[4][5] = n3 * t2 + n2 * t3;
  T[5][0] = n3 * n1; T[5][1] = s3 * s1; T[5][2] = t3 * t1; T[5][3] = n3 * s1 + n1 * s3; T[5][4] = s3 * t1 + s1 * t3; T[5][5] = n3 * t1 + n1 * t3;
  T[6][6] = n1; T[6][7] = s1; T[6][8] = t1;
  T[7][6] = n2; T[7][7] = s2; T[7][8] = t2;
  T[8][6] = n3; T[8][7] = s3; T[8][8] = t3;
}

template <class R>
void getInvT(const double* n, const double* s, const double* t, R T[9][9]) {
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) T[i][j] = 0;
  // src/waveMod.f90:215-267
  R n1 = n[0], n2 = n[1], n3 = n[2], s1 = s[0], s2 = s[1], s3 = s[2], t1 = t[0], t2 = t[1], t3 = t[2];
  T[0][0] = n1 * n1; T[0][1] = n2 * n2; T[0][2] = n3 * n3; T[0][3] = 2 * n2 * n1; T[0][4] = 2 * n3 * n2; T[0][5] = 2 * n3 * n1;
  T[1][0] = s1 * s1; T[1][1] = s2 * s2; T[1][2] = s3 * s3; T[1][3] = 2 * s2 * s1; T[1][4] = 2 * s3 * s2; T[1][5] = 2 * s3 * s1;
  T[2][0] = t1 * t1; T[2][1] = t2 * t2; T[2][2] = t3 * t3; T[2][3] = 2 * t2 * t1; T[2][4] = 2 * t3 * t2; T[2][5] = 2 * t3 * t1;
  T[3][0] = n1 * s1; T[3][1] = n2 * s2; T[3][2] = n3 * s3; T[3][3] = n2 * s1 + n1 * s2; T[3][4] = n3 * s2 + n2 * s3; T[3][5] = n3 * s1 + n1 * s3;
  T[4][0] = s1 * t1; T[4][1] = s2 * t2; T[4][2] = s3 * t3; T[4][3] = s2 * t1 + s1 * t2; T[4][4] = s3 * t2 + s2 * t3; T[4][5] = s3 * t1 + s1 * t3;
  T[5][0] = n1 * t1; T[5][1] = n2 * t2; T[5][2] = n3 * t3; T[5][3] = n2 * t1 + n1 * t2; T[5][4] = n3 * t2 + n2 * t3; T[5][5] = n3 * t1 + n1 * t3;
  T[6][6] = n1; T[6][7] = n2; T[6][8] = n3;
  T[7][6] = s1; T[7][7] = s2; T[7][8] = s3;
  T[8][6] = t1; T[8][7] = t2; T[8][8] = t3;
}

template <class R>
void mm9(const R A[9][9], const R B[9][9], R C[9][9]) {
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) {
      R s = 0;
      for (int k = 0; k < 9; ++k) s += A[i][k] * B[k][j];
      C[i][j] = s;
    }
}

template <class R>
struct Oracle {
  const nexd_desc& d;
  int K, Np, NpF, nMB, nt, nstage, nspt;
  size_t ng;
  bool att, pml;
  std::vector<R> Dr, Ds, Dt, lift;  // column-major copies of the desc operators
  std::vector<int> fmask;           // 0-based, [f*NpF+i]
  std::vector<R> metric, fscale, efv, anel, wl;
  std::vector<R> VT, VTfree, aVT, aVTfree;  // per element-face, row-major 9x9 / 6x9
  std::vector<R> prof;                       // (ng,9)
  std::vector<int> pmlc;
  std::vector<R> srcpat;  // (nsrc, 9, Np) source pattern in rq units per unit stf

  // state of one batch member
  std::vector<R> q, qm, qn, rq, th, thm, thn, arq, aux, auxm, auxn, auxr, resq, resth, resaux, ux, ax;
  // reference quirks: the flux arrays ftemp, gtemp, htemp of timeloop3D as
  // the element loop leaves them (the last element's values; columns that
  // elasticFluxes does not write keep the values of earlier elements), (9, Np)
  int quirks = 0;
  std::vector<R> lastF, lastG, lastH;
  // NPML trigger (src/timeloopMod.f90:508-542)
  bool trig = false;
  int tw1 = 10, tw2 = 2, tformula = 0, timecrit = 0;
  double tthr = 0.1;
  std::vector<double> mass;  // (Np,Np) column-major, M = (V V^T)^-1
  double* energy_out = nullptr;
  int* switch_out = nullptr;

  void arm(int w1, int w2, double thr, double f0, int formula) {
    trig = true;
    tw1 = w1;
    tw2 = w2;
    tthr = thr;
    tformula = formula;
    timecrit = int(float(2.4 / f0 / d.dt));
    // mass = inverse of invmass (Gauss-Jordan, partial pivoting)
    std::vector<double> A(d.invmass, d.invmass + size_t(Np) * Np);
    mass.assign(size_t(Np) * Np, 0.0);
    for (int i = 0; i < Np; ++i) mass[size_t(i) * Np + i] = 1.0;
    for (int c = 0; c < Np; ++c) {
      int p = c;
      for (int r = c + 1; r < Np; ++r)
        if (std::fabs(A[size_t(c) * Np + r]) > std::fabs(A[size_t(c) * Np + p])) p = r;
      for (int j = 0; j < Np; ++j) {
        std::swap(A[size_t(j) * Np + c], A[size_t(j) * Np + p]);
        std::swap(mass[size_t(j) * Np + c], mass[size_t(j) * Np + p]);
      }
      const double piv = A[size_t(c) * Np + c];
      for (int j = 0; j < Np; ++j) { A[size_t(j) * Np + c] /= piv; mass[size_t(j) * Np + c] /= piv; }
      for (int r = 0; r < Np; ++r) {
        if (r == c) continue;
        const double f = A[size_t(c) * Np + r];
        for (int j = 0; j < Np; ++j) {
          A[size_t(j) * Np + r] -= f * A[size_t(j) * Np + c];
          mass[size_t(j) * Np + r] -= f * mass[size_t(j) * Np + c];
        }
      }
    }
  }

  // energy_loc(it) of src/timeloopMod.f90:491-514 for the current q
  double energy() const {
    double total = 0.0;
#pragma omp parallel for reduction(+ : total) schedule(static)
    for (int e = 0; e < K; ++e) {
      const size_t g0 = size_t(e) * Np;
      const double lam = d.lambdau[e], mu = d.muu[e], rho = d.rho[e];
      std::vector<double> x(size_t(15) * Np);  // v (3), e (6), q1..q6
      for (int j = 0; j < Np; ++j) {
        double qq[9];
        for (int c = 0; c < 9; ++c) qq[c] = double(q[size_t(c) * ng + g0 + j]);
        double ev[6];
        if (tformula == 0) {
          const double t1 = 1.0 / (4 * mu * mu + 6 * mu * lam);
          ev[0] = (2 * (lam + mu) * qq[0] - lam * (qq[1] + qq[2])) / t1;
          ev[1] = (2 * (lam + mu) * qq[1] - lam * (qq[0] + qq[2])) / t1;
          ev[2] = (2 * (lam + mu) * qq[2] - lam * (qq[0] + qq[0])) / t1;
        } else {
          const double t1 = 4 * mu * mu + 6 * mu * lam;
          ev[0] = (2 * (lam + mu) * qq[0] - lam * (qq[1] + qq[2])) / t1;
          ev[1] = (2 * (lam + mu) * qq[1] - lam * (qq[0] + qq[2])) / t1;
          ev[2] = (2 * (lam + mu) * qq[2] - lam * (qq[0] + qq[1])) / t1;
        }
        for (int c = 3; c < 6; ++c) ev[c] = qq[c] / (2 * mu);
        for (int c = 0; c < 3; ++c) x[size_t(c) * Np + j] = qq[6 + c];
        for (int c = 0; c < 6; ++c) x[size_t(3 + c) * Np + j] = ev[c];
        for (int c = 0; c < 6; ++c) x[size_t(9 + c) * Np + j] = qq[c];
      }
      auto quad = [&](int a, int b) {  // x_a^T M x_b
        double s = 0.0;
        for (int n = 0; n < Np; ++n) {
          double mb = 0.0;
          for (int k = 0; k < Np; ++k) mb += mass[size_t(k) * Np + n] * x[size_t(b) * Np + k];
          s += x[size_t(a) * Np + n] * mb;
        }
        return s;
      };
      const double kin = rho * (quad(0, 0) + quad(1, 1) + quad(2, 2));
      const double pot = quad(9, 3) + quad(10, 4) + quad(11, 5) + 2 * (quad(12, 6) + quad(13, 7) + quad(14, 8));
      total += 0.5 * d.jacobian[e] * (kin + pot);
    }
    return total;
  }

  explicit Oracle(const nexd_desc& desc) : d(desc) {
    K = d.nelem;
    Np = d.Np;
    NpF = d.NpF;
    nMB = d.attenuation ? d.nMB : 0;
    nt = d.nt;
    att = d.attenuation != 0;
    pml = d.set_pml != 0;
    ng = size_t(K) * Np;
    nstage = d.timeint == 4 ? 5 : (d.timeint == 3 ? 3 : (d.timeint == 2 ? 2 : 1));
    nspt = d.stf_per_step;
    Dr.resize(size_t(Np) * Np);
    Ds.resize(Dr.size());
    Dt.resize(Dr.size());
    for (size_t i = 0; i < Dr.size(); ++i) {
      Dr[i] = R(d.Dr[i]);
      Ds[i] = R(d.Ds[i]);
      Dt[i] = R(d.Dt[i]);
    }
    lift.resize(size_t(Np) * 4 * NpF);
    for (size_t i = 0; i < lift.size(); ++i) lift[i] = R(d.lift[i]);
    fmask.resize(size_t(4) * NpF);
    for (size_t i = 0; i < fmask.size(); ++i) fmask[i] = d.fmask[i] - 1;
    metric.resize(size_t(K) * 9);
    for (size_t i = 0; i < metric.size(); ++i) metric[i] = R(d.metric[i]);
    fscale.resize(size_t(K) * 4);
    for (size_t i = 0; i < fscale.size(); ++i) fscale[i] = R(d.fscale[i]);
    efv.resize(size_t(K) * 4);
    VT.resize(size_t(K) * 4 * 81);
    VTfree.resize(VT.size());
    if (att) {
      aVT.resize(size_t(K) * 4 * 54);
      aVTfree.resize(aVT.size());
      anel.resize(size_t(K) * 3 * nMB);
      wl.resize(nMB);
      for (int l = 0; l < nMB; ++l) wl[l] = R(d.wl[l]);
    }
    // src/timeloopMod.f90:257-282
    for (int e = 0; e < K; ++e) {
      const R lam = R(d.lambdau[e]), mu = R(d.muu[e]), rho = R(d.rho[e]), vp = R(d.vpu[e]), vs = R(d.vsu[e]);
      efv[size_t(e) * 4 + 0] = -(lam + 2 * mu);
      efv[size_t(e) * 4 + 1] = -lam;
      efv[size_t(e) * 4 + 2] = -mu;
      efv[size_t(e) * 4 + 3] = R(-1.0) / rho;
      R APA[9][9] = {};
      APA[0][0] = vp; APA[0][6] = -(lam + 2 * mu);
      APA[1][0] = (lam * vp) / (lam + 2 * mu); APA[1][6] = -lam;
      APA[2][0] = (lam * vp) / (lam + 2 * mu); APA[2][6] = -lam;
      APA[3][3] = vs; APA[3][7] = -mu;
      APA[5][5] = vs; APA[5][8] = -mu;
      APA[6][0] = R(-1) / rho; APA[6][6] = vp;
      APA[7][3] = R(-1) / rho; APA[7][7] = vs;
      APA[8][5] = R(-1) / rho; APA[8][8] = vs;
      R APAf[9][9];
      // APA * free, free = diag(-2,0,0,-2,0,-2,0,0,0) (src/timeloopMod.f90:207-216)
      const R fr[9] = {-2, 0, 0, -2, 0, -2, 0, 0, 0};
      for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) APAf[i][j] = APA[i][j] * fr[j];
      R aAPA[9][9] = {};  // rows 0..5 used (src/waveMod.f90:146-159)
      if (att) {
        aAPA[0][0] = R(1) / (vp * rho); aAPA[0][6] = -1;
        aAPA[3][3] = R(1) / (2 * vs * rho); aAPA[3][7] = R(-0.5);
        aAPA[5][5] = R(1) / (2 * vs * rho); aAPA[5][8] = R(-0.5);
      }
      R aAPAf[9][9];
      for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) aAPAf[i][j] = aAPA[i][j] * fr[j];
      for (int f = 0; f < 4; ++f) {
        const double* n = &d.nnormal[(size_t(e) * 4 + f) * 3];
        const double* s = &d.stangential[(size_t(e) * 4 + f) * 3];
        const double* t = &d.ttangential[(size_t(e) * 4 + f) * 3];
        R T[9][9], iT[9][9], tmp[9][9], out[9][9];
        getT<R>(n, s, t, T);
        getInvT<R>(n, s, t, iT);
        mm9<R>(APA, iT, tmp);
        mm9<R>(T, tmp, out);
        for (int i = 0; i < 81; ++i) VT[(size_t(e) * 4 + f) * 81 + i] = out[i / 9][i % 9];
        mm9<R>(APAf, iT, tmp);
        mm9<R>(T, tmp, out);
        for (int i = 0; i < 81; ++i) VTfree[(size_t(e) * 4 + f) * 81 + i] = out[i / 9][i % 9];
        if (att) {
          R aT[9][9] = {};  // aT = T(1:6,1:6)
          for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) aT[i][j] = T[i][j];
          mm9<R>(aAPA, iT, tmp);
          mm9<R>(aT, tmp, out);
          for (int i = 0; i < 54; ++i) aVT[(size_t(e) * 4 + f) * 54 + i] = out[i / 9][i % 9];
          mm9<R>(aAPAf, iT, tmp);
          mm9<R>(aT, tmp, out);
          for (int i = 0; i < 54; ++i) aVTfree[(size_t(e) * 4 + f) * 54 + i] = out[i / 9][i % 9];
        }
      }
      if (att)
        for (int l = 0; l < nMB; ++l) {
          const R a1 = -lam * R(d.ylambda[size_t(e) * nMB + l]);
          const R a2 = -2 * mu * R(d.ymu[size_t(e) * nMB + l]);
          anel[(size_t(e) * nMB + l) * 3 + 0] = a1;
          anel[(size_t(e) * nMB + l) * 3 + 1] = a2;
          anel[(size_t(e) * nMB + l) * 3 + 2] = a1 + a2;
        }
    }
    if (pml) {
      prof.resize(ng * 9);
      for (size_t i = 0; i < prof.size(); ++i) prof[i] = R(d.pml_profiles[i]);
      pmlc.assign(d.pmlcheck, d.pmlcheck + K);
    }
    // Source patterns: invmass * (srcInt * a) / J [/ rho] (src/timeloopMod.f90:327-356)
    srcpat.assign(size_t(d.nsrc) * 9 * Np, R(0));
    for (int i = 0; i < d.nsrc; ++i) {
      const int e = d.srcelem[i] - 1;
      std::vector<R> si(Np);
      for (int j = 0; j < Np; ++j) si[j] = R(d.srcInt[size_t(i) * Np + j]);
      auto add = [&](int field, R amp) {
        std::vector<R> v(Np);
        for (int j = 0; j < Np; ++j) v[j] = si[j] * amp;
        for (int j = 0; j < Np; ++j) {
          R acc = 0;
          for (int k = 0; k < Np; ++k) acc += R(d.invmass[size_t(k) * Np + j]) * v[k];
          srcpat[(size_t(i) * 9 + field) * Np + j] = acc / R(d.jacobian[e]);
        }
      };
      if (d.srctype[i] == 0) {
        for (int c = 0; c < 3; ++c) add(6 + c, R(d.srcangle_force[size_t(i) * 3 + c]) / R(d.rho[e]));
      } else {
        const double* M = &d.srcM[size_t(i) * 6];  // Mxx Myy Mzz Mxy Mxz Myz
        // ms = sym(M); rq(:,1:6) += (Mxx,Myy,Mzz,Mxy,Myz,Mxz)
        add(0, R(M[0]));
        add(1, R(M[1]));
        add(2, R(M[2]));
        add(3, R(M[3]));
        add(4, R(M[5]));
        add(5, R(M[4]));
      }
    }
  }

  void alloc() {
    q.assign(ng * 9, R(d.init_value));
    qm = q;
    qn = q;
    rq.assign(ng * 9, R(d.init_value));
    resq.assign(ng * 9, R(0));
    ux.assign(ng * 3, R(d.init_value));
    ax.assign(ng * 3, R(d.init_value));
    if (att) {
      th.assign(ng * 6 * nMB, R(d.init_value));
      thm = th;
      thn = th;
      arq.assign(ng * 6 * nMB, R(d.init_value));
      resth.assign(ng * 6 * nMB, R(0));
    }
    if (pml) {
      aux.assign(ng * 27, R(0));  // fprime, gprime, hprime = 0 (src/timeloopMod.f90:252-254)
      auxm = aux;
      auxn = aux;
      auxr.assign(ng * 27, R(0));
      resaux.assign(ng * 27, R(0));
    }
    // ftemp = gtemp = htemp = 0 once before the time loop (src/timeloopMod.f90:224-226)
    lastF.assign(size_t(9) * Np, R(0));
    lastG.assign(size_t(9) * Np, R(0));
    lastH.assign(size_t(9) * Np, R(0));
  }

  // Per-thread scratch for one element.
  struct Scratch {
    std::vector<R> F, G, H, Dx, Dy, Dz, out, flux, aflux, sf, dv, alift;
  };

  // q arrays are (ng,9) column-major: field f of node g at [f*ng+g]
  void rhs_element(int e, const std::vector<R>& Q, const std::vector<R>* TH, const std::vector<R>* AUX, int it,
                   int stage, int batch) {
    thread_local Scratch S;
    const size_t g0 = size_t(e) * Np;
    const R* m = &metric[size_t(e) * 9];
    const R e1 = efv[size_t(e) * 4], e2 = efv[size_t(e) * 4 + 1], e3 = efv[size_t(e) * 4 + 2],
            e4 = efv[size_t(e) * 4 + 3];
    // flux columns stored (9, Np): column i of node j at [i*Np + j]
    S.F.assign(size_t(9) * Np, R(0));
    S.G.assign(size_t(9) * Np, R(0));
    S.H.assign(size_t(9) * Np, R(0));
    R* F = S.F.data();
    R* G = S.G.data();
    R* H = S.H.data();
    auto qv = [&](int f, int j) { return Q[size_t(f) * ng + g0 + j]; };
    // elasticFluxes (src/waveMod.f90:29-63)
    for (int j = 0; j < Np; ++j) {
      const R q1 = qv(0, j), q2 = qv(1, j), q3 = qv(2, j), q4 = qv(3, j), q5 = qv(4, j), q6 = qv(5, j),
              q7 = qv(6, j), q8 = qv(7, j), q9 = qv(8, j);
      F[0 * Np + j] = e1 * q7; F[1 * Np + j] = e2 * q7; F[2 * Np + j] = e2 * q7; F[3 * Np + j] = e3 * q8;
      F[5 * Np + j] = e3 * q9; F[6 * Np + j] = e4 * q1; F[7 * Np + j] = e4 * q4; F[8 * Np + j] = e4 * q6;
      G[0 * Np + j] = e2 * q8; G[1 * Np + j] = e1 * q8; G[2 * Np + j] = e2 * q8; G[3 * Np + j] = e3 * q7;
      G[4 * Np + j] = e3 * q9; G[6 * Np + j] = e4 * q4; G[7 * Np + j] = e4 * q2; G[8 * Np + j] = e4 * q5;
      H[0 * Np + j] = e2 * q9; H[1 * Np + j] = e2 * q9; H[2 * Np + j] = e1 * q9; H[4 * Np + j] = e3 * q8;
      H[5 * Np + j] = e3 * q7; H[6 * Np + j] = e4 * q6; H[7 * Np + j] = e4 * q5; H[8 * Np + j] = e4 * q3;
    }
    if (quirks & 2) {
      // f(:,5), g(:,6), h(:,4) are not written by elasticFluxes
      // (src/waveMod.f90:37-62): they keep what the previous element left
      for (int j = 0; j < Np; ++j) {
        F[4 * Np + j] = lastF[4 * Np + j];
        G[5 * Np + j] = lastG[5 * Np + j];
        H[3 * Np + j] = lastH[3 * Np + j];
      }
    }
    const bool pml_el = pml && pmlc[e];
    if (pml_el) {
      // F <- (F' + F)/kx (src/timeloopMod.f90:399-405) and the NPML
      // auxiliary right-hand side (src/rungekuttaMod.f90:52-63)
      for (int j = 0; j < Np; ++j) {
        const size_t g = g0 + j;
        const R ddx = prof[g], ddy = prof[ng + g], ddz = prof[2 * ng + g];
        const R alx = prof[3 * ng + g], aly = prof[4 * ng + g], alz = prof[5 * ng + g];
        const R kx = prof[6 * ng + g], ky = prof[7 * ng + g], kz = prof[8 * ng + g];
        for (int i = 0; i < 9; ++i) {
          const R fp = (*AUX)[size_t(i) * ng + g], gp = (*AUX)[size_t(9 + i) * ng + g],
                  hp = (*AUX)[size_t(18 + i) * ng + g];
          const R f = F[i * Np + j], gg = G[i * Np + j], h = H[i * Np + j];
          if (!(quirks & 1)) {
            auxr[size_t(i) * ng + g] = -alx * fp - ddx / kx * (fp + f);
            auxr[size_t(9 + i) * ng + g] = -aly * gp - ddy / ky * (gp + gg);
            auxr[size_t(18 + i) * ng + g] = -alz * hp - ddz / kz * (hp + h);
          }
          F[i * Np + j] = (fp + f) / kx;
          G[i * Np + j] = (gp + gg) / ky;
          H[i * Np + j] = (hp + h) / kz;
        }
      }
    }
    if (quirks) {
      // what ftemp, gtemp, htemp hold after this element (serial loop)
      std::copy(F, F + size_t(9) * Np, lastF.begin());
      std::copy(G, G + size_t(9) * Np, lastG.begin());
      std::copy(H, H + size_t(9) * Np, lastH.begin());
    }
    // Dx = rx Dr + sx Ds + tx Dt etc., column-major (Dx[k*Np+n] = Dx(n,k))
    const size_t NN = size_t(Np) * Np;
    S.Dx.resize(NN);
    S.Dy.resize(NN);
    S.Dz.resize(NN);
    R* Dx = S.Dx.data();
    R* Dy = S.Dy.data();
    R* Dz = S.Dz.data();
    for (size_t k = 0; k < NN; ++k) {
      Dx[k] = m[0] * Dr[k] + m[3] * Ds[k] + m[6] * Dt[k];
      Dy[k] = m[1] * Dr[k] + m[4] * Ds[k] + m[7] * Dt[k];
      Dz[k] = m[2] * Dr[k] + m[5] * Ds[k] + m[8] * Dt[k];
    }
    S.out.assign(size_t(9) * Np, R(0));
    R* out = S.out.data();
    // rq(:,i) = Dx F(:,i) + Dy G(:,i) + Dz H(:,i)  (src/timeloopMod.f90:407-420)
    for (int k = 0; k < Np; ++k) {
      const R* dxk = Dx + size_t(k) * Np;
      const R* dyk = Dy + size_t(k) * Np;
      const R* dzk = Dz + size_t(k) * Np;
      for (int i = 0; i < 9; ++i) {
        const R f = F[i * Np + k], g = G[i * Np + k], h = H[i * Np + k];
        R* o = out + size_t(i) * Np;
        for (int n = 0; n < Np; ++n) o[n] += dxk[n] * f + dyk[n] * g + dzk[n] * h;
      }
    }
    // computeExactRiemannSF (src/waveMod.f90:269-336), flux stored (4NpF, 9)
    const int nf = 4 * NpF;
    S.flux.assign(size_t(nf) * 9, R(0));
    R* flux = S.flux.data();
    R* aflux = nullptr;
    if (att) {
      S.aflux.assign(size_t(nf) * 6, R(0));
      aflux = S.aflux.data();
    }
    for (int is = 0; is < 4; ++is) {
      const int in = d.neighbor[size_t(e) * 4 + is];
      const int fc = d.face[size_t(e) * 4 + is];
      const R* vt = &VT[(size_t(e) * 4 + is) * 81];
      const R* vtf = &VTfree[(size_t(e) * 4 + is) * 81];
      const R* avt = att ? &aVT[(size_t(e) * 4 + is) * 54] : nullptr;
      const R* avtf = att ? &aVTfree[(size_t(e) * 4 + is) * 54] : nullptr;
      for (int i = 0; i < NpF; ++i) {
        const size_t gt = g0 + fmask[size_t(is) * NpF + i];
        R dq[9];
        const R* mat;
        const R* amat;
        R sign = 1;
        if (in > 0) {
          const size_t gn = size_t(d.ibn[(size_t(e) * 4 + is) * NpF + i] - 1);
          for (int c = 0; c < 9; ++c) dq[c] = Q[size_t(c) * ng + gn] - Q[size_t(c) * ng + gt];
          mat = vt;
          amat = avt;
        } else if (fc == -1) {
          for (int c = 0; c < 9; ++c) dq[c] = Q[size_t(c) * ng + gt];
          mat = vtf;
          amat = avtf;
        } else {
          for (int c = 0; c < 9; ++c) dq[c] = Q[size_t(c) * ng + gt];
          mat = vt;
          amat = avt;
          sign = -1;
        }
        const int row = is * NpF + i;
        for (int r = 0; r < 9; ++r) {
          R s = 0;
          for (int c = 0; c < 9; ++c) s += mat[r * 9 + c] * dq[c];
          flux[size_t(r) * nf + row] = sign * s;
        }
        if (att)
          for (int r = 0; r < 6; ++r) {
            R s = 0;
            for (int c = 0; c < 9; ++c) s += amat[r * 9 + c] * dq[c];
            aflux[size_t(r) * nf + row] = sign * s;
          }
      }
    }
    // rq(:,c) += LIFT (fscale * flux(:,c) / 2) (src/timeloopMod.f90:463-465)
    const R* fsc = &fscale[size_t(e) * 4];
    for (int j = 0; j < nf; ++j) {
      const R* lj = &lift[size_t(j) * Np];
      const R sc = fsc[j / NpF];
      for (int c = 0; c < 9; ++c) {
        const R s = sc * flux[size_t(c) * nf + j] / R(2);
        R* o = out + size_t(c) * Np;
        for (int n = 0; n < Np; ++n) o[n] += lj[n] * s;
      }
    }
    // anelastic part (src/timeloopMod.f90:426-461)
    if (att) {
      const R* th = (*TH).data();
      // velocity gradient dv(c,d) = D_d v_c, stored [(c*3+d)*Np + n]
      S.dv.assign(size_t(9) * Np, R(0));
      R* dv = S.dv.data();
      for (int k = 0; k < Np; ++k)
        for (int c = 0; c < 3; ++c) {
          const R v = Q[size_t(6 + c) * ng + g0 + k];
          for (int n = 0; n < Np; ++n) {
            dv[(size_t(c) * 3 + 0) * Np + n] += Dx[size_t(k) * Np + n] * v;
            dv[(size_t(c) * 3 + 1) * Np + n] += Dy[size_t(k) * Np + n] * v;
            dv[(size_t(c) * 3 + 2) * Np + n] += Dz[size_t(k) * Np + n] * v;
          }
        }
      // LIFT(fscale * aflux / 2) for the 6 columns (the mechanism factor wl is applied below)
      S.alift.assign(size_t(6) * Np, R(0));
      R* al = S.alift.data();
      for (int j = 0; j < nf; ++j) {
        const R* lj = &lift[size_t(j) * Np];
        const R sc = fsc[j / NpF];
        for (int c = 0; c < 6; ++c) {
          const R s = sc * aflux[size_t(c) * nf + j] / R(2);
          for (int n = 0; n < Np; ++n) al[size_t(c) * Np + n] += lj[n] * s;
        }
      }
      for (int l = 0; l < nMB; ++l) {
        const R w = wl[l];
        for (int n = 0; n < Np; ++n) {
          auto D = [&](int c, int dd) { return dv[(size_t(c) * 3 + dd) * Np + n]; };
          // anelasticFluxes (src/waveMod.f90:65-91): temp2 = -w v, temp1 = -w/2 v
          R vol[6];
          vol[0] = -w * D(0, 0);
          vol[1] = -w * D(1, 1);
          vol[2] = -w * D(2, 2);
          vol[3] = R(-0.5) * w * D(1, 0) + R(-0.5) * w * D(0, 1);
          vol[4] = R(-0.5) * w * D(2, 1) + R(-0.5) * w * D(1, 2);
          vol[5] = R(-0.5) * w * D(2, 0) + R(-0.5) * w * D(0, 2);
          for (int j = 0; j < 6; ++j) {
            const size_t idx = (size_t(l) * 6 + j) * ng + g0 + n;
            arq[idx] = vol[j] + w * al[size_t(j) * Np + n] - w * th[idx];
          }
        }
      }
      for (int n = 0; n < Np; ++n)
        for (int l = 0; l < nMB; ++l) {
          const R c1 = anel[(size_t(e) * nMB + l) * 3], c2 = anel[(size_t(e) * nMB + l) * 3 + 1],
                  c3 = anel[(size_t(e) * nMB + l) * 3 + 2];
          auto T_ = [&](int j) { return th[(size_t(l) * 6 + j) * ng + g0 + n]; };
          out[0 * Np + n] += c3 * T_(0) + c1 * (T_(1) + T_(2));
          out[1 * Np + n] += c3 * T_(1) + c1 * (T_(2) + T_(0));
          out[2 * Np + n] += c3 * T_(2) + c1 * (T_(0) + T_(1));
          out[3 * Np + n] += c2 * T_(3);
          out[4 * Np + n] += c2 * T_(4);
          out[5 * Np + n] += c2 * T_(5);
        }
    }
    // sources (src/timeloopMod.f90:467-475)
    for (int i = 0; i < d.nsrc; ++i) {
      if (d.srcelem[i] - 1 != e) continue;
      const int b = (d.nbatch > 1 && d.srcbatch) ? d.srcbatch[i] : 0;
      if (b != batch) continue;
      const int sidx = nspt == 1 ? 0 : std::min(stage, nspt - 1);
      const R s = R(d.stf[(size_t(i) * nt + (it - 1)) * nspt + sidx]);
      for (int c = 0; c < 9; ++c)
        for (int n = 0; n < Np; ++n) out[size_t(c) * Np + n] += srcpat[(size_t(i) * 9 + c) * Np + n] * s;
    }
    for (int c = 0; c < 9; ++c)
      for (int n = 0; n < Np; ++n) rq[size_t(c) * ng + g0 + n] = out[size_t(c) * Np + n];
  }

  void rhs_all(const std::vector<R>& Q, const std::vector<R>* TH, const std::vector<R>* AUX, int it, int stage,
               int batch) {
    if (!quirks) {
#pragma omp parallel for schedule(dynamic, 64)
      for (int e = 0; e < K; ++e) rhs_element(e, Q, TH, AUX, it, stage, batch);
      return;
    }
    // the reference's order: one element after the other, the flux arrays
    // carried from each element to the next (src/timeloopMod.f90:395-476)
    for (int e = 0; e < K; ++e) rhs_element(e, Q, TH, AUX, it, stage, batch);
    if ((quirks & 1) && pml) {
      // RungeKuttaSteps applies ftemp(j,i) -- the LAST element's flux, modified
      // when that element is in the PML -- to node j of every PML element
      // (src/rungekuttaMod.f90:52-63, called at src/timeloopMod.f90:479-480)
      for (int e = 0; e < K; ++e) {
        if (!pmlc[e]) continue;
        for (int j = 0; j < Np; ++j) {
          const size_t g = size_t(e) * Np + j;
          const R ddx = prof[g], ddy = prof[ng + g], ddz = prof[2 * ng + g];
          const R alx = prof[3 * ng + g], aly = prof[4 * ng + g], alz = prof[5 * ng + g];
          const R kx = prof[6 * ng + g], ky = prof[7 * ng + g], kz = prof[8 * ng + g];
          for (int i = 0; i < 9; ++i) {
            const R fp = (*AUX)[size_t(i) * ng + g], gp = (*AUX)[size_t(9 + i) * ng + g],
                    hp = (*AUX)[size_t(18 + i) * ng + g];
            auxr[size_t(i) * ng + g] = -alx * fp - ddx / kx * (fp + lastF[size_t(i) * Np + j]);
            auxr[size_t(9 + i) * ng + g] = -aly * gp - ddy / ky * (gp + lastG[size_t(i) * Np + j]);
            auxr[size_t(18 + i) * ng + g] = -alz * hp - ddz / kz * (hp + lastH[size_t(i) * Np + j]);
          }
        }
      }
    }
  }

  static R rk2(R a, R an, R dadt, R dt, int irk) {
    // src/rungekuttaMod.f90:90-103
    return irk == 1 ? a + dadt * dt : R(0.5) * (an + a + dadt * dt);
  }
  static R rk3(R a, R an, R dadt, R dt, int irk) {
    // src/rungekuttaMod.f90:105-120
    if (irk == 1) return a + dadt * dt;
    if (irk == 2) return R(0.75) * an + R(0.25) * (a + dadt * dt);
    return (R(1) / R(3)) * an + (R(2) / R(3)) * (a + dadt * dt);
  }

  void update(std::vector<R>& a, const std::vector<R>& an, const std::vector<R>& dadt, std::vector<R>& res, R dt,
              int irk, size_t n, const std::vector<char>* mask = nullptr) {
    const int ti = d.timeint;
    const double A = kRK4A[irk - 1], B = kRK4B[irk - 1];
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
      if (mask && !(*mask)[size_t(i) % ng]) continue;
      if (ti == 4) {
        res[i] = R(A) * res[i] + dt * dadt[i];
        a[i] = a[i] + R(B) * res[i];
      } else if (ti == 3) {
        a[i] = rk3(a[i], an[i], dadt[i], dt, irk);
      } else {
        a[i] = rk2(a[i], an[i], dadt[i], dt, irk);  // Euler is RK2's first stage
      }
    }
  }

  void run(int it_end, float* traces, double* field, int batch) {
    alloc();
    const R dt = R(d.dt);
    const int nrec = d.nrec;
    std::vector<char> pmlnode;
    if (pml) {
      pmlnode.assign(ng, 0);
      for (int e = 0; e < K; ++e)
        if (pmlc[e])
          for (int j = 0; j < Np; ++j) pmlnode[size_t(e) * Np + j] = 1;
    }
    const size_t toff = size_t(batch) * nrec * nt * 9;
    const auto loop_start = std::chrono::steady_clock::now();
    struct LoopTimer {  // adds the time-loop seconds of this run to g_loop_seconds
      std::chrono::steady_clock::time_point t0;
      ~LoopTimer() { g_loop_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
    } loop_timer{loop_start};
    for (int it = 1; it <= it_end; ++it) {
      // receivers (src/timeloopMod.f90:358-373)
      for (int r = 0; r < nrec; ++r) {
        const size_t g0 = size_t(d.recelem[r] - 1) * Np;
        R acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < Np; ++j) {
          const R w = R(d.recInt[size_t(r) * Np + j]);
          for (int c = 0; c < 3; ++c) {
            acc[c] += ux[size_t(c) * ng + g0 + j] * w;
            acc[3 + c] += q[size_t(6 + c) * ng + g0 + j] * w;
            acc[6 + c] += ax[size_t(c) * ng + g0 + j] * w;
          }
        }
        for (int c = 0; c < 9; ++c) traces[toff + (size_t(c) * nt + (it - 1)) * nrec + r] = float(acc[c]);
      }
      for (int irk = 1; irk <= nstage; ++irk) {
        qm = q;
        if (irk == 1) qn = q;
        if (att) {
          thm = th;
          if (irk == 1) thn = th;
        }
        if (pml) {
          auxm = aux;
          if (irk == 1) auxn = aux;
        }
        rhs_all(qm, att ? &thm : nullptr, pml ? &auxm : nullptr, it, irk - 1, batch);
        update(q, qn, rq, resq, dt, irk, ng * 9);
        if (att) update(th, thn, arq, resth, dt, irk, ng * 6 * nMB);
        if (pml) update(aux, auxn, auxr, resaux, dt, irk, ng * 27, &pmlnode);
        if (irk == nstage) {
          // src/timeloopMod.f90:482-488
          for (int c = 0; c < 3; ++c)
            for (size_t g = 0; g < ng; ++g) {
              ux[size_t(c) * ng + g] = ux[size_t(c) * ng + g] + dt * q[size_t(6 + c) * ng + g];
              ax[size_t(c) * ng + g] = rq[size_t(6 + c) * ng + g];
            }
        }
      }
      if (trig && pml) {
        double* E = energy_out + size_t(batch) * nt;
        E[it - 1] = energy();
        if (switch_out[batch] == 0 && it > timecrit) {
          float avg1 = 0.f, avg2 = 0.f;
          for (int i = 1; i <= tw1; ++i)
            if (it - i > 0) avg1 += float(E[it - i - 1] / tw1);
          for (int i = 1; i <= tw2; ++i)
            if (it - i > 0) avg2 += float(E[it - i - 1] / tw2);
          const float sta_lta = avg2 / avg1;
          if (std::fabs(sta_lta - 1.f) > float(tthr)) {
            switch_out[batch] = it;  // pmlcheck(:) = .false.
            std::fill(pmlc.begin(), pmlc.end(), 0);
          }
        }
      }
      bool finite = true;
      for (size_t g = 0; g < ng && finite; g += 97) finite = std::isfinite(double(q[size_t(6) * ng + g]));
      if (!finite) throw std::runtime_error("non-finite wavefield in the oracle");
    }
    if (field)
      for (size_t i = 0; i < ng * 9; ++i) field[size_t(batch) * ng * 9 + i] = double(q[i]);
  }
};

struct TriggerCfg {
  int w1, w2, formula;
  double thr, f0;
  double* energy;
  int* sw;
};

template <class R>
int run_t(const nexd_desc* d, int it_end, float* traces, double* field, const TriggerCfg* tc = nullptr) {
  g_loop_seconds = 0.0;
  Oracle<R> o(*d);
  o.quirks = g_ref_quirks;
  std::fill(traces, traces + size_t(d->nrec) * d->nt * 9 * std::max(1, d->nbatch), 0.0f);
  const int nb = std::max(1, d->nbatch);
  if (tc) {
    o.arm(tc->w1, tc->w2, tc->thr, tc->f0, tc->formula);
    o.energy_out = tc->energy;
    o.switch_out = tc->sw;
    std::fill(tc->energy, tc->energy + size_t(nb) * d->nt, 0.0);
    std::fill(tc->sw, tc->sw + nb, 0);
  }
  for (int b = 0; b < nb; ++b) {
    if (o.pml) o.pmlc.assign(d->pmlcheck, d->pmlcheck + d->nelem);
    o.run(it_end, traces, field, b);
  }
  return 0;
}

template <class R>
int rhs_t(const nexd_desc* d, int it, int stage, const double* q, const double* theta, const double* aux,
          double* rq, double* arq, double* auxr) {
  Oracle<R> o(*d);
  o.alloc();
  for (size_t i = 0; i < o.ng * 9; ++i) o.q[i] = R(q[i]);
  if (o.att && theta)
    for (size_t i = 0; i < o.th.size(); ++i) o.th[i] = R(theta[i]);
  if (o.pml && aux)
    for (size_t i = 0; i < o.aux.size(); ++i) o.aux[i] = R(aux[i]);
  o.rhs_all(o.q, o.att ? &o.th : nullptr, o.pml ? &o.aux : nullptr, it, stage, 0);
  for (size_t i = 0; i < o.ng * 9; ++i) rq[i] = double(o.rq[i]);
  if (arq && o.att)
    for (size_t i = 0; i < o.arq.size(); ++i) arq[i] = double(o.arq[i]);
  if (auxr && o.pml)
    for (size_t i = 0; i < o.auxr.size(); ++i) auxr[i] = double(o.auxr[i]);
  return 0;
}

bool check_desc(const nexd_desc* d) {
  if (!d) { g_err = "null descriptor"; return false; }
  if (d->abi_version != NEXD_ABI_VERSION) { g_err = "ABI version mismatch"; return false; }
  if (d->nelem <= 0 || d->Np <= 0 || d->nt <= 0) { g_err = "empty mesh or no steps"; return false; }
  if (d->timeint < 1 || d->timeint > 4) { g_err = "timeint must be 1..4"; return false; }
  return true;
}

}  // namespace

extern "C" {

int oracle_run(const nexd_desc* d, int precision, int it_end, float* traces, double* field, int nthreads) {
  if (!check_desc(d) || !traces) return NEXD_ERR_INVALID;
  if (it_end < 0 || it_end > d->nt) { g_err = "it_end out of range"; return NEXD_ERR_INVALID; }
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  try {
    return precision == 32 ? run_t<float>(d, it_end, traces, field) : run_t<double>(d, it_end, traces, field);
  } catch (const std::exception& e) {
    g_err = e.what();
    return NEXD_ERR_NONFINITE;
  }
}

int oracle_run_trigger(const nexd_desc* d, int precision, int it_end, float* traces, double* field, int nthreads,
                       int avg_window1, int avg_window2, double sta_lta_trigger, double f0, int formula,
                       double* energy, int* pml_switch) {
  if (!check_desc(d) || !traces || !energy || !pml_switch) return NEXD_ERR_INVALID;
  if (!d->set_pml) { g_err = "the trigger needs set_pml"; return NEXD_ERR_INVALID; }
  if (it_end < 0 || it_end > d->nt) { g_err = "it_end out of range"; return NEXD_ERR_INVALID; }
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  TriggerCfg tc{avg_window1, avg_window2, formula, sta_lta_trigger, f0, energy, pml_switch};
  try {
    return precision == 32 ? run_t<float>(d, it_end, traces, field, &tc) : run_t<double>(d, it_end, traces, field, &tc);
  } catch (const std::exception& e) {
    g_err = e.what();
    return NEXD_ERR_NONFINITE;
  }
}

int oracle_rhs(const nexd_desc* d, int precision, int it, int stage, const double* q, const double* theta,
               const double* aux, double* rq, double* arq, double* auxr) {
  if (!check_desc(d) || !q || !rq) return NEXD_ERR_INVALID;
  try {
    return precision == 32 ? rhs_t<float>(d, it, stage, q, theta, aux, rq, arq, auxr)
                           : rhs_t<double>(d, it, stage, q, theta, aux, rq, arq, auxr);
  } catch (const std::exception& e) {
    g_err = e.what();
    return NEXD_ERR_INVALID;
  }
}

double oracle_loop_seconds() { return g_loop_seconds; }

int oracle_set_ref_quirks(int flags) {
  if (flags < 0 || flags > 3) {
    g_err = "ref_quirks flags must be 0..3";
    return NEXD_ERR_INVALID;
  }
  g_ref_quirks = flags;
  return 0;
}

int oracle_last_error(char* buf, size_t len) {
  if (!buf || !len) return NEXD_ERR_INVALID;
  std::strncpy(buf, g_err.c_str(), len - 1);
  buf[len - 1] = 0;
  return 0;
}
}
