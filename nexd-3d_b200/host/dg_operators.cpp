// FP64 restatement of the NEXD-3D reference-element operators.
// Reference: src/gllMod.f90, src/warpfactorMod.f90, src/nodesMod.f90,
// src/jacobiMod.f90, src/simplexMod.f90, src/tetTrafoMod.f90,
// src/vandermondeMod.f90, src/dmatricesMod.f90, src/liftMod.f90,
// src/meshMod.f90:601-663.
#include "dg_operators.hpp"

#include <cmath>
#include <stdexcept>

namespace nexd {

Mat matmul(const Mat& A, const Mat& B) {
  if (A.cols != B.rows) throw std::runtime_error("matmul: shape mismatch");
  Mat C(A.rows, B.cols);
  for (int j = 0; j < B.cols; ++j)
    for (int k = 0; k < A.cols; ++k) {
      const double b = B(k, j);
      if (b == 0.0) continue;
      for (int i = 0; i < A.rows; ++i) C(i, j) += A(i, k) * b;
    }
  return C;
}

Mat transpose(const Mat& A) {
  Mat T(A.cols, A.rows);
  for (int j = 0; j < A.cols; ++j)
    for (int i = 0; i < A.rows; ++i) T(j, i) = A(i, j);
  return T;
}

// Gauss-Jordan elimination with partial pivoting (the reference calls
// LAPACK getrf/getri, src/matrixMod.f90:27-53).
bool invert(Mat& A) {
  const int n = A.rows;
  if (A.cols != n) return false;
  Mat inv(n, n);
  for (int i = 0; i < n; ++i) inv(i, i) = 1.0;
  Mat a = A;
  for (int c = 0; c < n; ++c) {
    int p = c;
    double best = std::fabs(a(c, c));
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(a(r, c)) > best) { best = std::fabs(a(r, c)); p = r; }
    if (best == 0.0) return false;
    if (p != c)
      for (int j = 0; j < n; ++j) { std::swap(a(c, j), a(p, j)); std::swap(inv(c, j), inv(p, j)); }
    const double d = 1.0 / a(c, c);
    for (int j = 0; j < n; ++j) { a(c, j) *= d; inv(c, j) *= d; }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = a(r, c);
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) { a(r, j) -= f * a(c, j); inv(r, j) -= f * inv(c, j); }
    }
  }
  A = inv;
  return true;
}

double warp_alpha(int N) {
  // balpha table, src/constants.h:32-33 (Warburton's optimised warp values).
  static const double tab[15] = {0.0000, 0.0000, 0.0000, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577,
                                 1.1603, 1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655};
  if (N < 1 || N > 15) return 0.0;
  return tab[N - 1];
}

// Gauss-Lobatto-Legendre nodes by Newton iteration from Chebyshev-Lobatto
// guesses, descending from +1 to -1 (src/gllMod.f90:27-56).
static std::vector<double> gll_nodes(int N) {
  const int ngll = N + 1, p = N;
  std::vector<double> x(ngll), V(ngll + 1);
  for (int i = 0; i < ngll; ++i) {
    x[i] = std::cos(M_PI * i / p);
    double xold = 2.0;
    for (int it = 0; it < 200 && std::fabs(x[i] - xold) > 1e-15; ++it) {
      xold = x[i];
      V[1] = 1.0;
      V[2] = x[i];
      for (int k = 2; k <= p; ++k) V[k + 1] = ((2.0 * k - 1.0) * x[i] * V[k] - (k - 1.0) * V[k - 1]) / k;
      x[i] = xold - (x[i] * V[ngll] - V[p]) / (ngll * V[ngll]);
    }
  }
  return x;
}

// Warp function interpolated at xout (src/warpfactorMod.f90:28-66).
static void warpfactor(int N, const std::vector<double>& xgll, const std::vector<double>& xout,
                       std::vector<double>& w) {
  const int ngll = N + 1;
  const double dx = 2.0 / (ngll - 1);
  std::vector<double> xeq(ngll);
  for (int i = 0; i < ngll; ++i) xeq[i] = (ngll - 1 - i) * dx - 1.0;
  w.assign(xout.size(), 0.0);
  for (size_t k = 0; k < xout.size(); ++k) {
    double d = 0.0;
    for (int i = 0; i < ngll; ++i) {
      const double e = xgll[i] - xeq[i];
      double p1 = 1.0, p2 = 1.0;
      for (int j = 0; j < ngll; ++j)
        if (i != j) { p1 *= (xout[k] - xeq[j]); p2 *= (xeq[i] - xeq[j]); }
      d += e * (p1 / p2);
    }
    const bool interior = std::fabs(xout[k]) < (1.0 - 1e-10);
    w[k] = interior ? d / (1.0 - xout[k] * xout[k]) : 0.0;
  }
}

// Blend & warp on one face triangle (src/warpfactorMod.f90:68-113).
static void shiftwarp(int N, double alpha, const std::vector<double>& L1, const std::vector<double>& L2,
                      const std::vector<double>& L3, std::vector<double>& x, std::vector<double>& y) {
  const size_t n = L1.size();
  const std::vector<double> xgll = gll_nodes(N);
  std::vector<double> a1(n), a2(n), a3(n), w1, w2, w3;
  for (size_t i = 0; i < n; ++i) { a1[i] = L3[i] - L2[i]; a2[i] = L1[i] - L3[i]; a3[i] = L2[i] - L1[i]; }
  warpfactor(N, xgll, a1, w1);
  warpfactor(N, xgll, a2, w2);
  warpfactor(N, xgll, a3, w3);
  x.resize(n);
  y.resize(n);
  for (size_t i = 0; i < n; ++i) {
    const double warp1 = 4.0 * L2[i] * L3[i] * w1[i] * (1.0 + (alpha * L1[i]) * (alpha * L1[i]));
    const double warp2 = 4.0 * L1[i] * L3[i] * w2[i] * (1.0 + (alpha * L2[i]) * (alpha * L2[i]));
    const double warp3 = 4.0 * L1[i] * L2[i] * w3[i] * (1.0 + (alpha * L3[i]) * (alpha * L3[i]));
    x[i] = warp1 + std::cos(2.0 * M_PI / 3.0) * warp2 + std::cos(4.0 * M_PI / 3.0) * warp3;
    y[i] = std::sin(2.0 * M_PI / 3.0) * warp2 + std::sin(4.0 * M_PI / 3.0) * warp3;
  }
}

void nodes_rst(int N, double alpha, std::vector<double>& r, std::vector<double>& s, std::vector<double>& t) {
  const int p = N;
  const int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  std::vector<double> re(Np), se(Np), te(Np);
  int sk = 0;
  for (int n = 1; n <= p + 1; ++n)
    for (int m = 1; m <= p + 2 - n; ++m)
      for (int q = 1; q <= p + 3 - n - m; ++q) {
        re[sk] = -1.0 + (q - 1.0) * 2.0 / p;
        se[sk] = -1.0 + (m - 1.0) * 2.0 / p;
        te[sk] = -1.0 + (n - 1.0) * 2.0 / p;
        ++sk;
      }
  std::vector<double> L1(Np), L2(Np), L3(Np), L4(Np);
  for (int i = 0; i < Np; ++i) {
    L1[i] = (1.0 + te[i]) / 2.0;
    L2[i] = (1.0 + se[i]) / 2.0;
    L3[i] = -(1.0 + re[i] + se[i] + te[i]) / 2.0;
    L4[i] = (1.0 + re[i]) / 2.0;
  }
  const double s3 = std::sqrt(3.0), s6 = std::sqrt(6.0);
  const double v1[3] = {-1.0, -1.0 / s3, -1.0 / s6}, v2[3] = {1.0, -1.0 / s3, -1.0 / s6},
               v3[3] = {0.0, 2.0 / s3, -1.0 / s6}, v4[3] = {0.0, 0.0, 3.0 / s6};
  double t1[4][3], t2[4][3];
  for (int j = 0; j < 3; ++j) {
    t1[0][j] = v2[j] - v1[j];
    t1[1][j] = v2[j] - v1[j];
    t1[2][j] = v3[j] - v2[j];
    t1[3][j] = v3[j] - v1[j];
    t2[0][j] = v3[j] - 0.5 * (v1[j] + v2[j]);
    t2[1][j] = v4[j] - 0.5 * (v1[j] + v2[j]);
    t2[2][j] = v4[j] - 0.5 * (v2[j] + v3[j]);
    t2[3][j] = v4[j] - 0.5 * (v1[j] + v3[j]);
  }
  for (int i = 0; i < 4; ++i) {
    const double n1 = std::sqrt(t1[i][0] * t1[i][0] + t1[i][1] * t1[i][1] + t1[i][2] * t1[i][2]);
    const double n2 = std::sqrt(t2[i][0] * t2[i][0] + t2[i][1] * t2[i][1] + t2[i][2] * t2[i][2]);
    for (int j = 0; j < 3; ++j) { t1[i][j] /= n1; t2[i][j] /= n2; }
  }
  std::vector<double> X(Np * 3), shift(Np * 3, 0.0);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < 3; ++j) X[i * 3 + j] = L3[i] * v1[j] + L4[i] * v2[j] + L2[i] * v3[j] + L1[i] * v4[j];
  const double tol = 1e-10;
  for (int f = 0; f < 4; ++f) {
    const std::vector<double>*La, *Lb, *Lc, *Ld;
    if (f == 0) { La = &L1; Lb = &L2; Lc = &L3; Ld = &L4; }
    else if (f == 1) { La = &L2; Lb = &L1; Lc = &L3; Ld = &L4; }
    else if (f == 2) { La = &L3; Lb = &L1; Lc = &L4; Ld = &L2; }
    else { La = &L4; Lb = &L1; Lc = &L3; Ld = &L2; }
    std::vector<double> w1, w2;
    shiftwarp(N, alpha, *Lb, *Lc, *Ld, w1, w2);
    for (int j = 0; j < Np; ++j) {
      const double la = (*La)[j], lb = (*Lb)[j], lc = (*Lc)[j], ld = (*Ld)[j];
      double blend = lb * lc * ld;
      const double denom = (lb + 0.5 * la) * (lc + 0.5 * la) * (ld + 0.5 * la);
      if (denom > tol) blend = (1.0 + (alpha * la) * (alpha * la)) * blend / denom;
      for (int d = 0; d < 3; ++d) shift[j * 3 + d] += blend * w1[j] * t1[f][d] + blend * w2[j] * t2[f][d];
    }
    // Face nodes take the face warp alone.  The reference's edge test is
    // always true (src/nodesMod.f90:139-143 sets bool(2) twice), so every node
    // with La < tol is replaced; for face-interior nodes the other faces'
    // blends vanish, so the result equals Warburton's construction.
    for (int j = 0; j < Np; ++j)
      if ((*La)[j] < tol)
        for (int d = 0; d < 3; ++d) shift[j * 3 + d] = w1[j] * t1[f][d] + w2[j] * t2[f][d];
  }
  for (int i = 0; i < Np * 3; ++i) X[i] += shift[i];
  // xyzToRst (src/tetTrafoMod.f90:57-92)
  Mat A(3, 3);
  for (int j = 0; j < 3; ++j) {
    A(j, 0) = 0.5 * (v2[j] - v1[j]);
    A(j, 1) = 0.5 * (v3[j] - v1[j]);
    A(j, 2) = 0.5 * (v4[j] - v1[j]);
  }
  invert(A);
  r.resize(Np);
  s.resize(Np);
  t.resize(Np);
  for (int i = 0; i < Np; ++i) {
    double b[3];
    for (int j = 0; j < 3; ++j) b[j] = X[i * 3 + j] - 0.5 * (v2[j] + v3[j] + v4[j] - v1[j]);
    r[i] = A(0, 0) * b[0] + A(0, 1) * b[1] + A(0, 2) * b[2];
    s[i] = A(1, 0) * b[0] + A(1, 1) * b[1] + A(1, 2) * b[2];
    t[i] = A(2, 0) * b[0] + A(2, 1) * b[1] + A(2, 2) * b[2];
  }
}

// Normalised Jacobi polynomial P_n^{(alpha,beta)} (src/jacobiMod.f90:28-68).
// The reference evaluates the gamma function with an FP32 Lanczos routine
// (src/rosettaGammaMod.f90:23); std::tgamma is used here.
static double jacobiP(double x, double alpha, double beta, int n) {
  const double gamma0 = std::pow(2.0, alpha + beta + 1.0) / (alpha + beta + 1.0) * std::tgamma(alpha + 1.0) *
                        std::tgamma(beta + 1.0) / std::tgamma(alpha + beta + 1.0);
  double p0 = 1.0 / std::sqrt(gamma0);
  if (n == 0) return p0;
  const double gamma1 = (alpha + 1.0) * (beta + 1.0) / (alpha + beta + 3.0) * gamma0;
  double p1 = ((alpha + beta + 2.0) * x / 2.0 + (alpha - beta) / 2.0) / std::sqrt(gamma1);
  if (n == 1) return p1;
  double aold = 2.0 / (2.0 + alpha + beta) * std::sqrt((alpha + 1.0) * (beta + 1.0) / (alpha + beta + 3.0));
  for (int i = 1; i <= n - 1; ++i) {
    const double h1 = 2.0 * i + alpha + beta;
    const double anew = 2.0 / (h1 + 2.0) *
                        std::sqrt((i + 1.0) * (i + 1.0 + alpha + beta) * (i + 1.0 + alpha) * (i + 1.0 + beta) /
                                  (h1 + 1.0) / (h1 + 3.0));
    const double bnew = -(alpha * alpha - beta * beta) / h1 / (h1 + 2.0);
    const double p2 = 1.0 / anew * (-aold * p0 + (x - bnew) * p1);
    aold = anew;
    p0 = p1;
    p1 = p2;
  }
  return p1;
}

static double grad_jacobiP(double x, double alpha, double beta, int n) {
  if (n == 0) return 0.0;
  return std::sqrt(n * (n + alpha + beta + 1.0)) * jacobiP(x, alpha + 1.0, beta + 1.0, n - 1);
}

static const double kEps = 1e-10;

// rstToAbc (src/tetTrafoMod.f90:94-115).
static void rst_to_abc(double r, double s, double t, double& a, double& b, double& c) {
  a = (std::fabs(s + t) > kEps) ? 2.0 * (1.0 + r) / (-s - t) - 1.0 : -1.0;
  b = (std::fabs(t - 1.0) > kEps) ? 2.0 * (1.0 + s) / (1.0 - t) - 1.0 : -1.0;
  c = t;
}

static double simplex3dp(double a, double b, double c, int i, int j, int k) {
  const double h1 = jacobiP(a, 0.0, 0.0, i);
  const double h2 = jacobiP(b, 2.0 * i + 1.0, 0.0, j);
  const double h3 = jacobiP(c, 2.0 * (i + j) + 2.0, 0.0, k);
  return 2.0 * std::sqrt(2.0) * h1 * h2 * std::pow(1.0 - b, i) * h3 * std::pow(1.0 - c, i + j);
}

// gradSimplex3DP (src/simplexMod.f90:111-165).
static void grad_simplex3dp(double a, double b, double c, int id, int jd, int kd, double& dr, double& ds,
                            double& dt) {
  const double fa = jacobiP(a, 0.0, 0.0, id), dfa = grad_jacobiP(a, 0.0, 0.0, id);
  const double gb = jacobiP(b, 2.0 * id + 1.0, 0.0, jd), dgb = grad_jacobiP(b, 2.0 * id + 1.0, 0.0, jd);
  const double hc = jacobiP(c, 2.0 * (id + jd) + 2.0, 0.0, kd),
               dhc = grad_jacobiP(c, 2.0 * (id + jd) + 2.0, 0.0, kd);
  double vr = dfa * (gb * hc);
  if (id > 0) vr *= std::pow(0.5 * (1.0 - b), id - 1.0);
  if (id + jd > 0) vr *= std::pow(0.5 * (1.0 - c), id + jd - 1.0);
  double vs = 0.5 * (1.0 + a) * vr;
  double tmp = dgb * std::pow(0.5 * (1.0 - b), id);
  if (id > 0) tmp += (-0.5 * id) * (gb * std::pow(0.5 * (1.0 - b), id - 1.0));
  if (id + jd > 0) tmp *= std::pow(0.5 * (1.0 - c), id + jd - 1.0);
  tmp = fa * tmp * hc;
  vs += tmp;
  double vt = 0.5 * (1.0 + a) * vr + 0.5 * (1.0 + b) * tmp;
  tmp = dhc * std::pow(0.5 * (1.0 - c), id + jd);
  if (id + jd > 0) tmp -= 0.5 * (id + jd) * (hc * std::pow(0.5 * (1.0 - c), id + jd - 1.0));
  tmp = fa * (gb * tmp);
  tmp *= std::pow(0.5 * (1.0 - b), id);
  vt += tmp;
  const double sc = std::pow(2.0, 2.0 * id + jd + 1.5);
  dr = sc * vr;
  ds = sc * vs;
  dt = sc * vt;
}

Mat vandermonde3d(int N, const std::vector<double>& r, const std::vector<double>& s,
                  const std::vector<double>& t) {
  const int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  const int n = int(r.size());
  Mat V(n, Np);
  for (int p = 0; p < n; ++p) {
    double a, b, c;
    rst_to_abc(r[p], s[p], t[p], a, b, c);
    int sk = 0;
    for (int i = 0; i <= N; ++i)
      for (int j = 0; j <= N - i; ++j)
        for (int k = 0; k <= N - i - j; ++k) V(p, sk++) = simplex3dp(a, b, c, i, j, k);
  }
  return V;
}

static void grad_vandermonde3d(int N, const std::vector<double>& r, const std::vector<double>& s,
                               const std::vector<double>& t, Mat& Vr, Mat& Vs, Mat& Vt) {
  const int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  const int n = int(r.size());
  Vr = Mat(n, Np);
  Vs = Mat(n, Np);
  Vt = Mat(n, Np);
  for (int p = 0; p < n; ++p) {
    double a, b, c;
    rst_to_abc(r[p], s[p], t[p], a, b, c);
    int sk = 0;
    for (int i = 0; i <= N; ++i)
      for (int j = 0; j <= N - i; ++j)
        for (int k = 0; k <= N - i - j; ++k) {
          grad_simplex3dp(a, b, c, i, j, k, Vr(p, sk), Vs(p, sk), Vt(p, sk));
          ++sk;
        }
  }
}

// 2D face Vandermonde (src/vandermondeMod.f90:30-44, src/simplexMod.f90:28-42).
static Mat vandermonde2d(int N, const std::vector<double>& r, const std::vector<double>& s) {
  const int NpF = (N + 1) * (N + 2) / 2;
  const int n = int(r.size());
  Mat V(n, NpF);
  for (int p = 0; p < n; ++p) {
    const double a = (std::fabs(s[p] - 1.0) > kEps) ? 2.0 * (1.0 + r[p]) / (1.0 - s[p]) - 1.0 : -1.0;
    const double b = s[p];
    int sk = 0;
    for (int i = 0; i <= N; ++i)
      for (int j = 0; j <= N - i; ++j) {
        const double h1 = jacobiP(a, 0.0, 0.0, i);
        const double h2 = jacobiP(b, 2.0 * i + 1.0, 0.0, j);
        V(p, sk++) = std::sqrt(2.0) * h1 * h2 * std::pow(1.0 - b, i);
      }
  }
  return V;
}

DGOperators build_operators(int N) {
  if (N < 1 || N > 10) throw std::runtime_error("polynomial order must be in 1..10");
  DGOperators op;
  op.N = N;
  op.Np = (N + 1) * (N + 2) * (N + 3) / 6;
  op.NpF = (N + 1) * (N + 2) / 2;
  const int Np = op.Np, NpF = op.NpF;
  nodes_rst(N, warp_alpha(N), op.r, op.s, op.t);
  op.minGLL = std::fabs(op.r[0] - op.r[1]);
  op.V = vandermonde3d(N, op.r, op.s, op.t);
  op.invV = op.V;
  if (!invert(op.invV)) throw std::runtime_error("singular Vandermonde matrix");
  op.mass = matmul(transpose(op.invV), op.invV);
  op.invmass = matmul(op.V, transpose(op.V));
  Mat Vr, Vs, Vt;
  grad_vandermonde3d(N, op.r, op.s, op.t, Vr, Vs, Vt);
  op.Dr = matmul(Vr, op.invV);
  op.Ds = matmul(Vs, op.invV);
  op.Dt = matmul(Vt, op.invV);
  // Face masks in increasing node order (src/meshMod.f90:627-661).
  op.fmask.assign(size_t(NpF) * 4, -1);
  const double tol = 1e-7;
  for (int f = 0; f < 4; ++f) {
    int d = 0;
    for (int i = 0; i < Np; ++i) {
      double v;
      if (f == 0) v = op.t[i] + 1.0;
      else if (f == 1) v = op.s[i] + 1.0;
      else if (f == 2) v = 1.0 + op.r[i] + op.s[i] + op.t[i];
      else v = 1.0 + op.r[i];
      if (std::fabs(v) < tol) {
        if (d >= NpF) throw std::runtime_error("face mask overflow");
        op.fmask[size_t(f) * NpF + d++] = i;
      }
    }
    if (d != NpF) throw std::runtime_error("face mask incomplete");
  }
  // LIFT = V (V^T E) with E the face mass matrices (src/liftMod.f90:28-76).
  Mat E(Np, 4 * NpF);
  for (int f = 0; f < 4; ++f) {
    std::vector<double> fr(NpF), fs(NpF);
    for (int i = 0; i < NpF; ++i) {
      const int id = op.fmask[size_t(f) * NpF + i];
      if (f == 0) { fr[i] = op.r[id]; fs[i] = op.s[id]; }
      else if (f == 1) { fr[i] = op.r[id]; fs[i] = op.t[id]; }
      else { fr[i] = op.s[id]; fs[i] = op.t[id]; }
    }
    Mat V2 = vandermonde2d(N, fr, fs);
    Mat inv2 = V2;
    if (!invert(inv2)) throw std::runtime_error("singular face Vandermonde matrix");
    Mat mF = matmul(transpose(inv2), inv2);
    for (int i = 0; i < NpF; ++i)
      for (int j = 0; j < NpF; ++j) E(op.fmask[size_t(f) * NpF + i], f * NpF + j) += mF(i, j);
  }
  op.lift = matmul(op.V, matmul(transpose(op.V), E));
  return op;
}

}  // namespace nexd
