// Single-partition mesh database builder (restates src/meshMod.f90:45-1393
// with nproc = 1) and the pre-loop set-up of timeloop3D
// (src/timeloopMod.f90:137-356).
#include "mesh_db.hpp"

#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace nexd {

namespace {

std::string lower(std::string s) {
  for (auto& c : s) c = char(std::tolower(unsigned(c)));
  return s;
}

// One "name = value" line of a parameter file (src/fileParameterMod.f90:26-92).
struct ParLine {
  std::string name, value;
};

std::vector<ParLine> read_par_lines(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::vector<ParLine> out;
  std::string line;
  while (std::getline(f, line)) {
    size_t b = line.find_first_not_of(" \t\r");
    if (b == std::string::npos) { out.push_back({}); continue; }
    line = line.substr(b);
    if (line[0] == '#') { out.push_back({}); continue; }
    const size_t eq = line.find('=');
    if (eq == std::string::npos) { out.push_back({}); continue; }
    std::string name;
    for (size_t i = 0; i < eq; ++i)
      if (line[i] != ' ' && line[i] != '\t') name += line[i];
    std::string rest = line.substr(eq + 1);
    std::istringstream is(rest);
    std::string v;
    is >> v;  // list-directed read takes the first token
    // a trailing comma ends a list-directed item
    const size_t comma = v.find(',');
    if (comma != std::string::npos) v = v.substr(0, comma);
    out.push_back({name, v});
  }
  return out;
}

const std::string& par_value(const std::vector<ParLine>& lines, const std::string& name, size_t from,
                             const std::string& path) {
  for (size_t i = from; i < lines.size(); ++i)
    if (lines[i].name == name) return lines[i].value;
  throw std::runtime_error("Parameter not found in parameter file " + path + ": " + name);
}

bool as_logical(const std::string& v) {
  std::string s = lower(v);
  if (!s.empty() && s[0] == '.') s = s.substr(1);
  if (!s.empty() && s[0] == 't') return true;
  if (!s.empty() && s[0] == 'f') return false;
  throw std::runtime_error("not a logical value: " + v);
}

double as_real(const std::string& v) {
  std::string s = v;
  for (auto& c : s)
    if (c == 'd' || c == 'D') c = 'e';
  char* end = nullptr;
  const double x = std::strtod(s.c_str(), &end);
  if (end == s.c_str()) throw std::runtime_error("not a number: " + v);
  return x;
}

int as_int(const std::string& v) {
  char* end = nullptr;
  const long x = std::strtol(v.c_str(), &end, 10);
  if (end == v.c_str()) throw std::runtime_error("not an integer: " + v);
  return int(x);
}

std::ifstream open_or_throw(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  return f;
}

// Face vertex triples in the order tet_mesh_neighbor_tets records them:
// face j (1..4) of the search is the face opposite vertex j
// (src/tetraNeighborMod.f90:563-764).
const int kOpp[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};

// Reference face numbering: face 1 (t=-1) is opposite vertex 4, face 2 (s=-1)
// opposite vertex 3, face 3 opposite vertex 1, face 4 opposite vertex 2
// (the neighbour reorder at src/meshMod.f90:255-258).
const int kFaceOppVertex[4] = {3, 2, 0, 1};  // 0-based vertex opposite reference face f
// side(j): reference face number of the face opposite vertex j (src/meshMod.f90:131-134)
const int kSide[4] = {3, 4, 2, 1};

}  // namespace

Parfile read_parfile(const std::string& path) {
  const auto L = read_par_lines(path);
  Parfile p;
  p.log = as_logical(par_value(L, "log", 0, path));
  p.external = as_logical(par_value(L, "external", 0, path));
  p.nproc = as_int(par_value(L, "nproc", 0, path));
  p.vtk = as_logical(par_value(L, "vtk", 0, path));
  p.movie = as_logical(par_value(L, "movie", 0, path));
  p.frame = as_int(par_value(L, "frame", 0, path));
  p.timeint = as_int(par_value(L, "timeint", 0, path));
  p.nt = as_int(par_value(L, "nt", 0, path));
  p.cfl = as_real(par_value(L, "cfl", 0, path));
  p.attenuation = as_logical(par_value(L, "attenuation", 0, path));
  p.f0_att = as_real(par_value(L, "f0_att", 0, path));
  p.fr_att = as_real(par_value(L, "fr_att", 0, path));
  p.set_pml = as_logical(par_value(L, "set_pml", 0, path));
  p.pml_delta = as_real(par_value(L, "pml_delta", 0, path));
  p.pml_rc = as_real(par_value(L, "pml_rc", 0, path));
  p.pml_kmax = as_real(par_value(L, "pml_kmax", 0, path));
  p.pml_afac = as_real(par_value(L, "pml_afac", 0, path));
  p.avg_window1 = as_int(par_value(L, "avg_window1", 0, path));
  p.avg_window2 = as_int(par_value(L, "avg_window2", 0, path));
  p.sta_lta_trigger = as_real(par_value(L, "sta_lta_trigger", 0, path));
  return p;
}

std::vector<Source> read_sources(const std::string& path) {
  const auto L = read_par_lines(path);
  const int nsrc = as_int(par_value(L, "nsrc", 0, path));
  if (nsrc < 0) throw std::runtime_error("Number of source is negative. ABORT!");
  std::vector<Source> out(nsrc);
  size_t from = 0;
  for (int i = 0; i < nsrc; ++i) {
    // setFilePosition("source", i+1): parameters are read after that line
    size_t pos = L.size();
    for (size_t k = from; k < L.size(); ++k)
      if (L[k].name == "source" && as_int(L[k].value) == i + 1) { pos = k + 1; break; }
    if (pos == L.size()) throw std::runtime_error("Parameter source not found in " + path);
    from = pos;
    Source& s = out[i];
    s.xyz[0] = as_real(par_value(L, "xsource", pos, path));
    s.xyz[1] = as_real(par_value(L, "ysource", pos, path));
    s.xyz[2] = as_real(par_value(L, "zsource", pos, path));
    s.type = as_int(par_value(L, "sourcetype", pos, path));
    s.stf = as_int(par_value(L, "stf", pos, path));
    s.f0 = as_real(par_value(L, "f0", pos, path));
    if (s.f0 <= 0.0) throw std::runtime_error("Source frequency is zero or negative. ABORT!");
    s.factor = as_real(par_value(L, "factor", pos, path));
    s.angle_force[0] = as_real(par_value(L, "xangle_force", pos, path));
    s.angle_force[1] = as_real(par_value(L, "yangle_force", pos, path));
    s.angle_force[2] = as_real(par_value(L, "zangle_force", pos, path));
    const double n = std::sqrt(s.angle_force[0] * s.angle_force[0] + s.angle_force[1] * s.angle_force[1] +
                               s.angle_force[2] * s.angle_force[2]);
    for (double& a : s.angle_force) a /= n;  // src/sourceReceiverMod.f90:77-78
    static const char* mk[6] = {"Mxx", "Myy", "Mzz", "Mxy", "Mxz", "Myz"};
    for (int c = 0; c < 6; ++c) s.M[c] = as_real(par_value(L, mk[c], pos, path));
  }
  return out;
}

std::vector<Receiver> read_stations(const std::string& path) {
  auto f = open_or_throw(path);
  int n = 0;
  f >> n;
  std::vector<Receiver> out(n);
  for (int i = 0; i < n; ++i) {
    f >> out[i].nr >> out[i].xyz[0] >> out[i].xyz[1] >> out[i].xyz[2];
    if (!f) throw std::runtime_error("truncated stations file " + path);
  }
  return out;
}

double stf_ricker(double t, double f0, double t0, double factor) {
  const double a = M_PI * M_PI * f0 * f0;
  return -factor * (1.0 - 2.0 * a * (t - t0) * (t - t0)) * std::exp(-a * (t - t0) * (t - t0));
}

double stf_gauss(double t, double f0, double t0, double factor) {
  const double a = M_PI * M_PI * f0 * f0;
  return -factor * std::exp(-a * (t - t0) * (t - t0));
}

// Time derivatives of the two STFs, used when the STF is evaluated at RK
// stage times for moment-tensor sources.
static double stf_ricker_dt(double t, double f0, double t0, double factor) {
  const double a = M_PI * M_PI * f0 * f0, u = t - t0;
  return -factor * std::exp(-a * u * u) * (-4.0 * a * u - 2.0 * a * u * (1.0 - 2.0 * a * u * u));
}
static double stf_gauss_dt(double t, double f0, double t0, double factor) {
  const double a = M_PI * M_PI * f0 * f0, u = t - t0;
  return -factor * std::exp(-a * u * u) * (-2.0 * a * u);
}

void anelastic_precalc(double f0, double fr, int nMB, std::vector<double>& wl, std::vector<double>& wk) {
  const int m = 2 * nMB - 1;
  wk.assign(m, 0.0);
  wl.assign(nMB, 0.0);
  const double wmax = 2.5 * M_PI * f0, wmin = f0 / std::sqrt(fr);
  if (nMB > 1) {
    for (int i = 0; i < m; ++i) wk[i] = std::exp(std::log(wmin) + double(i) / (2.0 * (nMB - 1)) * std::log(fr));
  } else {
    for (auto& w : wk) w = wmax;
  }
  int c = 0;
  for (int i = 0; i < m; ++i)
    if (i % 2 == 0) wl[c++] = wk[i];
}

// Least squares min ||A x - b|| for full-column-rank A (m >= n) by Householder
// QR, the method of LAPACK xGELS used at src/linearSystemMod.f90:26-66.
static std::vector<double> lstsq_qr(std::vector<double> A, int m, int n, std::vector<double> b) {
  for (int k = 0; k < n; ++k) {
    double nrm = 0.0;
    for (int i = k; i < m; ++i) nrm += A[size_t(k) * m + i] * A[size_t(k) * m + i];
    nrm = std::sqrt(nrm);
    if (nrm == 0.0) throw std::runtime_error("rank-deficient least-squares system");
    const double alpha = (A[size_t(k) * m + k] > 0) ? -nrm : nrm;
    std::vector<double> v(m, 0.0);
    for (int i = k; i < m; ++i) v[i] = A[size_t(k) * m + i];
    v[k] -= alpha;
    double vn = 0.0;
    for (int i = k; i < m; ++i) vn += v[i] * v[i];
    if (vn == 0.0) continue;
    for (int j = k; j < n; ++j) {
      double d = 0.0;
      for (int i = k; i < m; ++i) d += v[i] * A[size_t(j) * m + i];
      d = 2.0 * d / vn;
      for (int i = k; i < m; ++i) A[size_t(j) * m + i] -= d * v[i];
    }
    double d = 0.0;
    for (int i = k; i < m; ++i) d += v[i] * b[i];
    d = 2.0 * d / vn;
    for (int i = k; i < m; ++i) b[i] -= d * v[i];
  }
  std::vector<double> x(n, 0.0);
  for (int k = n - 1; k >= 0; --k) {
    double s = b[k];
    for (int j = k + 1; j < n; ++j) s -= A[size_t(j) * m + k] * x[j];
    x[k] = s / A[size_t(k) * m + k];
  }
  return x;
}

void anelastic_coefficients(double Qp, double Qs, double vp, double vs, double rho, double f0,
                            const std::vector<double>& wl, const std::vector<double>& wk, double* ylambda,
                            double* ymu, double& lambda_u, double& mu_u) {
  const int nMB = int(wl.size()), m = 2 * nMB - 1;
  std::vector<double> Mp(size_t(m) * nMB), Ms(size_t(m) * nMB);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < nMB; ++j) {
      Mp[size_t(j) * m + i] = (wl[j] * wk[i] + wl[j] * wl[j] / Qp) / (wl[j] * wl[j] + wk[i] * wk[i]);
      Ms[size_t(j) * m + i] = (wl[j] * wk[i] + wl[j] * wl[j] / Qs) / (wl[j] * wl[j] + wk[i] * wk[i]);
    }
  const std::vector<double> yp = lstsq_qr(Mp, m, nMB, std::vector<double>(m, 1.0 / Qp));
  const std::vector<double> ys = lstsq_qr(Ms, m, nMB, std::vector<double>(m, 1.0 / Qs));
  auto unrelaxed = [&](const std::vector<double>& y, double v) {
    double th1 = 1.0, th2 = 0.0;
    for (int j = 0; j < nMB; ++j) {
      const double q = f0 / wl[j];
      th1 -= y[j] / (1.0 + q * q);
      th2 += y[j] * q / (1.0 + q * q);
    }
    const double R = std::sqrt(th1 * th1 + th2 * th2);
    return rho * v * v * (R + th1) / (2.0 * R * R);
  };
  const double Mup = unrelaxed(yp, vp), Mus = unrelaxed(ys, vs);
  mu_u = Mus;
  lambda_u = Mup - 2.0 * mu_u;
  for (int j = 0; j < nMB; ++j) {
    ylambda[j] = (1.0 + (2.0 * mu_u) / lambda_u) * yp[j] - (2.0 * mu_u) / lambda_u * ys[j];
    ymu[j] = ys[j];
  }
}

// Snap reference coordinates that are +-1 up to rounding, so vertex and edge
// nodes reproduce the mesh vertices exactly (the FP32 reference gets exact
// vertex coordinates, which the source/receiver search relies on for ties).
static void snap_rst(std::vector<double>& v) {
  for (double& x : v) {
    if (std::fabs(x - 1.0) < 1e-12) x = 1.0;
    if (std::fabs(x + 1.0) < 1e-12) x = -1.0;
  }
}

namespace {

struct Locator {
  const MeshDB& db;
  std::vector<double> r, s, t;  // search node set (balpha(NGLL), src/sourceReceiverMod.f90:233)
  Mat vdmTinv;
  explicit Locator(const MeshDB& d) : db(d) {
    nodes_rst(d.N, warp_alpha(d.N + 1), r, s, t);
    snap_rst(r);
    snap_rst(s);
    snap_rst(t);
    Mat V = vandermonde3d(d.N, r, s, t);
    vdmTinv = transpose(V);
    if (!invert(vdmTinv)) throw std::runtime_error("singular search Vandermonde");
  }
  void xyz_of(int ie, double rr, double ss, double tt, double out[3]) const {
    const int* e = &db.elem[size_t(ie) * 4];
    for (int c = 0; c < 3; ++c)
      out[c] = 0.5 * (-(1.0 + rr + ss + tt) * db.coord[size_t(e[0] - 1) * 3 + c] +
                      (1.0 + rr) * db.coord[size_t(e[1] - 1) * 3 + c] +
                      (1.0 + ss) * db.coord[size_t(e[2] - 1) * 3 + c] + (1.0 + tt) * db.coord[size_t(e[3] - 1) * 3 + c]);
  }
  // findSource / findReceiver (src/sourceReceiverMod.f90:204-528).
  void locate(const double target[3], int& elem_out, double rst_out[3], const char* what, int idx) const {
    const int K = db.nelem, Np = db.Np;
    std::vector<char> check(K, 1);
    int besave = 1;
    for (;;) {
      double eps = 1e7, sr = 0, ss = 0, stt = 0;
      int found = -1;
      for (int ie = 0; ie < K; ++ie) {
        if (!check[ie]) continue;
        for (int i = 0; i < Np; ++i) {
          const size_t g = size_t(ie) * Np + i;
          const double d = std::sqrt((db.vx[g] - target[0]) * (db.vx[g] - target[0]) +
                                     (db.vy[g] - target[1]) * (db.vy[g] - target[1]) +
                                     (db.vz[g] - target[2]) * (db.vz[g] - target[2]));
          if (d < eps) {
            eps = d;
            sr = r[i];
            ss = s[i];
            stt = t[i];
            found = ie;
          }
        }
      }
      if (found < 0) throw std::runtime_error(std::string("could not find ") + what);
      const int ie = found;
      const double* m = &db.metric[size_t(ie) * 9];  // rx ry rz sx sy sz tx ty tz
      for (int it = 1; it <= 4; ++it) {
        double xyz[3];
        xyz_of(ie, sr, ss, stt, xyz);
        // Interpolating the element-constant metric reproduces it (the
        // weights sum to one), so the correction is the affine Newton step.
        const double dx = target[0] - xyz[0], dy = target[1] - xyz[1], dz = target[2] - xyz[2];
        sr += m[0] * dx + m[1] * dy + m[2] * dz;
        ss += m[3] * dx + m[4] * dy + m[5] * dz;
        stt += m[6] * dx + m[7] * dy + m[8] * dz;
      }
      bool reject = !(sr == sr) || !(ss == ss) || !(stt == stt) || sr < -1.001 || sr > 1.001 || ss < -1.001 ||
                    ss > 1.001 || stt < -1.001 || stt > -0.999 - sr - ss;
      if (reject) {
        check[ie] = 0;
        ++besave;
        if (besave > 20) {
          char buf[256];
          std::snprintf(buf, sizeof buf, "ERROR, could not find %s %d at global coordinates %g %g %g", what, idx,
                        target[0], target[1], target[2]);
          throw std::runtime_error(buf);
        }
        continue;
      }
      if (sr > 1.0) sr = 1.0;
      if (sr < -1.0) sr = -1.0;
      if (ss > 1.0) ss = 1.0;
      if (ss < -1.0) ss = -1.0;
      if (stt < -1.0) stt = -1.0;
      if (stt > -1.0 - sr - ss) stt = -1.0 - sr - ss;
      elem_out = ie + 1;
      rst_out[0] = sr;
      rst_out[1] = ss;
      rst_out[2] = stt;
      return;
    }
  }
};

}  // namespace

static void read_cubit(const std::string& dir, MeshDB& db, std::vector<std::array<int, 4>>& freef,
                       std::vector<std::array<int, 4>>& absf) {
  {
    auto f = open_or_throw(dir + "/cubit/coord");
    f >> db.ncoord;
    db.coord.assign(size_t(db.ncoord) * 3, 0.0);
    db.pmlxmin = db.pmlymin = db.pmlzmin = 1e10;
    db.pmlxmax = db.pmlymax = db.pmlzmax = 0.0;  // src/meshMod.f90:197-202
    for (int i = 0; i < db.ncoord; ++i) {
      int id;
      f >> id >> db.coord[size_t(i) * 3] >> db.coord[size_t(i) * 3 + 1] >> db.coord[size_t(i) * 3 + 2];
      if (!f) throw std::runtime_error("truncated cubit/coord");
      const double* c = &db.coord[size_t(i) * 3];
      db.pmlxmin = std::min(db.pmlxmin, c[0]);
      db.pmlxmax = std::max(db.pmlxmax, c[0]);
      db.pmlymin = std::min(db.pmlymin, c[1]);
      db.pmlymax = std::max(db.pmlymax, c[1]);
      db.pmlzmin = std::min(db.pmlzmin, c[2]);
      db.pmlzmax = std::max(db.pmlzmax, c[2]);
    }
  }
  {
    auto f = open_or_throw(dir + "/cubit/mesh");
    f >> db.nelem;
    const int K = db.nelem;
    db.elem.assign(size_t(K) * 4, 0);
    db.vp.assign(K, 0);
    db.vs.assign(K, 0);
    db.rho.assign(K, 0);
    db.qp.assign(K, 0);
    db.qs.assign(K, 0);
    for (int i = 0; i < K; ++i) {
      int id;
      f >> id >> db.elem[size_t(i) * 4] >> db.elem[size_t(i) * 4 + 1] >> db.elem[size_t(i) * 4 + 2] >>
          db.elem[size_t(i) * 4 + 3] >> db.vp[i] >> db.vs[i] >> db.rho[i] >> db.qp[i] >> db.qs[i];
      if (!f) throw std::runtime_error("truncated cubit/mesh");
      if (db.vp[i] <= 0.0 || db.vs[i] <= 0.0)
        throw std::runtime_error("ERROR! vp or vs is zero or negative for at least one element. Stop!");
      if (db.vp[i] <= db.vs[i]) throw std::runtime_error("ERROR! vp is not larger than vs for at least one element. Stop!");
      for (int j = 0; j < 4; ++j) {
        const int v = db.elem[size_t(i) * 4 + j];
        if (v < 1 || v > db.ncoord) throw std::runtime_error("cubit/mesh references a vertex outside cubit/coord");
      }
    }
    for (int i = 0; i < K; ++i)
      if (db.vp[i] <= std::sqrt(2.0) * db.vs[i]) {
        // The reference asks interactively (src/meshMod.f90:238-248); the
        // library continues and records a warning.
        db.warnings.push_back("Poisson number is zero or negative for at least one element");
        break;
      }
  }
  {
    auto f = open_or_throw(dir + "/cubit/mat");
    db.mat.assign(db.nelem, 0);
    db.pml.assign(db.nelem, 0);
    for (int i = 0; i < db.nelem; ++i) {
      int c, m, p;
      f >> c >> m >> p;
      if (!f) throw std::runtime_error("truncated cubit/mat");
      if (c < 1 || c > db.nelem) throw std::runtime_error("cubit/mat element id out of range");
      db.mat[c - 1] = m;
      db.pml[c - 1] = p;
    }
  }
  auto read_faces = [&](const std::string& name, std::vector<std::array<int, 4>>& out) {
    auto f = open_or_throw(dir + "/cubit/" + name);
    int n = 0;
    f >> n;
    out.resize(n);
    for (int i = 0; i < n; ++i) {
      f >> out[i][0] >> out[i][1] >> out[i][2] >> out[i][3];
      if (!f) throw std::runtime_error("truncated cubit/" + name);
      if (out[i][0] < 1 || out[i][0] > db.nelem) throw std::runtime_error("cubit/" + name + " element id out of range");
    }
  };
  read_faces("free", freef);
  read_faces("absorb", absf);
  // material table (optional here; the solver reads per-element values)
  std::ifstream mp(dir + "/cubit/matprop");
  if (mp) {
    mp >> db.nmat;
    if (!mp || db.nmat < 0) throw std::runtime_error("bad cubit/matprop");
    db.matval.assign(size_t(db.nmat) * 11, 0.0);
    for (int i = 0; i < db.nmat; ++i) {
      double id, dummy, vp, vs, rho, qp, qs;
      mp >> id >> dummy >> vp >> vs >> rho >> qp >> qs;
      if (!mp) throw std::runtime_error("truncated cubit/matprop");
      const size_t n = size_t(db.nmat);
      db.matval[i] = rho;
      db.matval[n + i] = vp;
      db.matval[2 * n + i] = vs;
      db.matval[3 * n + i] = vs * vs * rho;
      db.matval[4 * n + i] = vp * vp * rho - 2.0 * vs * vs * rho;
      db.matval[5 * n + i] = qp;
      db.matval[6 * n + i] = qs;
    }
  }
}

static void build_topology(MeshDB& db, const std::vector<std::array<int, 4>>& freef,
                           const std::vector<std::array<int, 4>>& absf) {
  const int K = db.nelem;
  // tet_mesh_neighbor_tets: neighbour across the face opposite vertex j.
  std::vector<int> ntemp(size_t(K) * 4, -1);
  struct Key {
    int a, b, c;
    bool operator==(const Key& o) const { return a == o.a && b == o.b && c == o.c; }
  };
  struct KeyHash {
    size_t operator()(const Key& k) const {
      return (size_t(k.a) * 73856093u) ^ (size_t(k.b) * 19349663u) ^ (size_t(k.c) * 83492791u);
    }
  };
  std::unordered_map<Key, std::vector<std::pair<int, int>>, KeyHash> faces;
  faces.reserve(size_t(K) * 3);
  for (int e = 0; e < K; ++e)
    for (int j = 0; j < 4; ++j) {
      int v[3] = {db.elem[size_t(e) * 4 + kOpp[j][0]], db.elem[size_t(e) * 4 + kOpp[j][1]],
                  db.elem[size_t(e) * 4 + kOpp[j][2]]};
      std::sort(v, v + 3);
      faces[Key{v[0], v[1], v[2]}].push_back({e, j});
    }
  for (auto& kv : faces) {
    auto& lst = kv.second;
    std::sort(lst.begin(), lst.end(), [](auto& x, auto& y) { return x.second != y.second ? x.second < y.second : x.first < y.first; });
    if (lst.size() == 2) {
      ntemp[size_t(lst[0].first) * 4 + lst[0].second] = lst[1].first + 1;
      ntemp[size_t(lst[1].first) * 4 + lst[1].second] = lst[0].first + 1;
    } else if (lst.size() > 2) {
      throw std::runtime_error("non-manifold face shared by more than two tetrahedra");
    }
  }
  db.neighbor.assign(size_t(K) * 4, 0);
  for (int e = 0; e < K; ++e) {
    // neighbor(1)=ntemp(4), (2)=ntemp(3), (3)=ntemp(1), (4)=ntemp(2)
    const int m[4] = {3, 2, 0, 1};
    for (int f = 0; f < 4; ++f) {
      const int n = ntemp[size_t(e) * 4 + m[f]];
      db.neighbor[size_t(e) * 4 + f] = n > 0 ? n : 0;
    }
  }
  db.face.assign(size_t(K) * 4, 0);
  for (int i = 0; i < K; ++i)
    for (int j = 0; j < 4; ++j) {
      const int c = db.neighbor[size_t(i) * 4 + j];
      if (c > 0)
        for (int k = 0; k < 4; ++k)
          if (db.neighbor[size_t(c - 1) * 4 + k] == i + 1) db.face[size_t(i) * 4 + j] = k + 1;
    }
  bool bad = false;
  std::string msg;
  auto assign = [&](const std::vector<std::array<int, 4>>& lst, int code) {
    for (const auto& fl : lst) {
      const int c = fl[0] - 1;
      bool check[4] = {false, false, false, false};
      for (int j = 0; j < 4; ++j)
        for (int k = 0; k < 3; ++k)
          if (db.elem[size_t(c) * 4 + j] == fl[k + 1]) check[j] = true;
      for (int j = 0; j < 4; ++j)
        if (!check[j]) {
          int& fv = db.face[size_t(c) * 4 + kSide[j] - 1];
          if (code == -2 && fv == -1) {
            bad = true;
            msg = "a face is assigned as free and absorbing boundary at the same time";
          }
          fv = code;
        }
      if (code == -2) {
        int sum = 0;
        for (int j = 0; j < 4; ++j) sum += db.face[size_t(c) * 4 + j];
        if (sum == -8) throw std::runtime_error("Found single element with only absorbing boundaries!");
      }
    }
  };
  assign(freef, -1);
  assign(absf, -2);
  for (int i = 0; i < K && !bad; ++i)
    for (int j = 0; j < 4; ++j)
      if (db.neighbor[size_t(i) * 4 + j] == 0 && db.face[size_t(i) * 4 + j] > -1) {
        bad = true;
        char buf[160];
        std::snprintf(buf, sizeof buf, "Face %d of element %d is a domain boundary but not assigned as free or absorbing boundary", j + 1, i + 1);
        msg = buf;
        break;
      }
  if (bad) throw std::runtime_error(msg + " -- ABORT!");
}

static void build_geometry(MeshDB& db) {
  const int K = db.nelem, Np = db.Np, NpF = db.NpF;
  const auto& op = db.op;
  db.nglob = K * Np;
  db.vx.assign(db.nglob, 0);
  db.vy.assign(db.nglob, 0);
  db.vz.assign(db.nglob, 0);
  db.metric.assign(size_t(K) * 9, 0);
  db.jac.assign(K, 0);
  db.sJ.assign(size_t(K) * 4, 0);
  db.fscale.assign(size_t(K) * 4, 0);
  db.nn.assign(size_t(K) * 12, 0);
  db.st.assign(size_t(K) * 12, 0);
  db.tt.assign(size_t(K) * 12, 0);
  std::vector<double> r = op.r, s = op.s, t = op.t;
  snap_rst(r);
  snap_rst(s);
  snap_rst(t);
  for (int e = 0; e < K; ++e) {
    const double* X[4];
    for (int j = 0; j < 4; ++j) X[j] = &db.coord[size_t(db.elem[size_t(e) * 4 + j] - 1) * 3];
    for (int j = 0; j < Np; ++j) {
      const size_t g = size_t(e) * Np + j;
      const double w1 = -(1.0 + r[j] + s[j] + t[j]), w2 = 1.0 + r[j], w3 = 1.0 + s[j], w4 = 1.0 + t[j];
      db.vx[g] = 0.5 * (w1 * X[0][0] + w2 * X[1][0] + w3 * X[2][0] + w4 * X[3][0]);
      db.vy[g] = 0.5 * (w1 * X[0][1] + w2 * X[1][1] + w3 * X[2][1] + w4 * X[3][1]);
      db.vz[g] = 0.5 * (w1 * X[0][2] + w2 * X[1][2] + w3 * X[2][2] + w4 * X[3][2]);
    }
    // geometricFactors3d for an affine map (src/geometricFactorsMod.f90:28-68)
    const double xr = 0.5 * (X[1][0] - X[0][0]), yr = 0.5 * (X[1][1] - X[0][1]), zr = 0.5 * (X[1][2] - X[0][2]);
    const double xs = 0.5 * (X[2][0] - X[0][0]), ys = 0.5 * (X[2][1] - X[0][1]), zs = 0.5 * (X[2][2] - X[0][2]);
    const double xt = 0.5 * (X[3][0] - X[0][0]), yt = 0.5 * (X[3][1] - X[0][1]), zt = 0.5 * (X[3][2] - X[0][2]);
    const double J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt);
    if (std::fabs(J) < 1e-300) throw std::runtime_error("Jacobian is zero in geometric factors");
    double* m = &db.metric[size_t(e) * 9];
    m[0] = (ys * zt - zs * yt) / J;   // rx
    m[1] = -(xs * zt - zs * xt) / J;  // ry
    m[2] = (xs * yt - ys * xt) / J;   // rz
    m[3] = -(yr * zt - zr * yt) / J;  // sx
    m[4] = (xr * zt - zr * xt) / J;   // sy
    m[5] = -(xr * yt - yr * xt) / J;  // sz
    m[6] = (yr * zs - zr * ys) / J;   // tx
    m[7] = -(xr * zs - zr * xs) / J;  // ty
    m[8] = (xr * ys - yr * xs) / J;   // tz
    db.jac[e] = J;
    // normals3d (src/normalsMod.f90:27-130)
    for (int f = 0; f < 4; ++f) {
      double n[3];
      for (int c = 0; c < 3; ++c) {
        const double rxc = m[c], sxc = m[3 + c], txc = m[6 + c];
        if (f == 0) n[c] = -txc;
        else if (f == 1) n[c] = -sxc;
        else if (f == 2) n[c] = rxc + sxc + txc;
        else n[c] = -rxc;
      }
      const double sj = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      for (int c = 0; c < 3; ++c) db.nn[size_t(e) * 12 + f * 3 + c] = n[c] / sj;
      db.sJ[size_t(e) * 4 + f] = sj * J;
      db.fscale[size_t(e) * 4 + f] = (sj * J) / J;
      // n, s, t frames (src/meshMod.f90:836-875)
      static const int cc[4] = {0, 0, 1, 0}, dd[4] = {1, 1, 2, 2};
      double sv[3];
      for (int c = 0; c < 3; ++c) sv[c] = X[dd[f]][c] - X[cc[f]][c];
      const double sn = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
      for (int c = 0; c < 3; ++c) sv[c] /= sn;
      const double* nv = &db.nn[size_t(e) * 12 + f * 3];
      double tv[3] = {nv[1] * sv[2] - nv[2] * sv[1], nv[2] * sv[0] - nv[0] * sv[2], nv[0] * sv[1] - nv[1] * sv[0]};
      const double tn = std::sqrt(tv[0] * tv[0] + tv[1] * tv[1] + tv[2] * tv[2]);
      for (int c = 0; c < 3; ++c) {
        db.st[size_t(e) * 12 + f * 3 + c] = sv[c];
        db.tt[size_t(e) * 12 + f * 3 + c] = tv[c] / tn;
      }
    }
  }
  // ibt / ibn with coordinate-matched permutation (src/meshMod.f90:939-987)
  db.ibt.assign(size_t(K) * 4 * NpF, 0);
  db.ibn.assign(size_t(K) * 4 * NpF, 0);
  for (int e = 0; e < K; ++e) {
    const int* v = &db.elem[size_t(e) * 4];
    double edges = 0.0;  // epsil: 1/30 of the mean edge length (src/meshMod.f90:366-378)
    for (int i = 0; i < 4; ++i)
      for (int j = i + 1; j < 4; ++j) {
        const double* a = &db.coord[size_t(v[i] - 1) * 3];
        const double* b = &db.coord[size_t(v[j] - 1) * 3];
        edges += std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
      }
    const double epsil = edges / 6.0 / 30.0;
    for (int is = 0; is < 4; ++is) {
      int* ibt = &db.ibt[(size_t(e) * 4 + is) * NpF];
      int* ibn = &db.ibn[(size_t(e) * 4 + is) * NpF];
      for (int i = 0; i < NpF; ++i) ibt[i] = e * Np + op.fmask[size_t(is) * NpF + i] + 1;
      const int in = db.neighbor[size_t(e) * 4 + is];
      if (in <= 0) continue;
      const int j = db.face[size_t(e) * 4 + is] - 1;
      for (int i = 0; i < NpF; ++i) {
        const size_t gt = size_t(ibt[i] - 1);
        int match = -1;
        for (int k = 0; k < NpF; ++k) {
          const size_t gn = size_t(in - 1) * Np + op.fmask[size_t(j) * NpF + k];
          if (std::fabs(db.vx[gt] - db.vx[gn]) < epsil && std::fabs(db.vy[gt] - db.vy[gn]) < epsil &&
              std::fabs(db.vz[gt] - db.vz[gn]) < epsil)
            match = int(gn) + 1;
        }
        if (match < 0) throw std::runtime_error("face nodes of neighbouring elements do not coincide");
        ibn[i] = match;
      }
    }
  }
  // dtfactor (src/meshMod.f90:1134-1160)
  double rtemp1 = 1e7;
  for (int e = 0; e < K; ++e) {
    double min2 = db.sJ[size_t(e) * 4];
    for (int f = 1; f < 4; ++f) min2 = std::min(min2, db.sJ[size_t(e) * 4 + f]);
    rtemp1 = std::min(rtemp1, db.jac[e] / min2);
  }
  double rtemp3 = 1e7;
  for (int e = 0; e < K; ++e) rtemp3 = std::min(rtemp3, 2.0 / 3.0 * op.minGLL * (rtemp1 / db.vpu[e]));
  db.dtfactor = rtemp3;
  db.minGLL_jac = op.minGLL * rtemp1;
}

// PMLPreCalculation + dampingProfile (src/pmlMod.f90:27-165).
static void build_pml(MeshDB& db) {
  const int K = db.nelem, Np = db.Np;
  const Parfile& par = db.par;
  const size_t ng = size_t(db.nglob);
  db.pmlcheck.assign(K, 0);
  db.pml_profiles.assign(ng * 9, 0.0);
  double* ddx = &db.pml_profiles[0];
  double* ddy = ddx + ng;
  double* ddz = ddy + ng;
  double* ax = ddz + ng;
  double* ay = ax + ng;
  double* az = ay + ng;
  double* kx = az + ng;
  double* ky = kx + ng;
  double* kz = ky + ng;
  for (size_t i = 0; i < ng; ++i) kx[i] = ky[i] = kz[i] = 1.0;
  if (!par.set_pml) return;
  const double amax = par.pml_afac * M_PI * db.f0max;
  const double delta = par.pml_delta;
  for (int e = 0; e < K; ++e) {
    if (db.pml[e] <= 0) continue;
    db.pmlcheck[e] = 1;
    double xm = 0, ym = 0, zm = 0;
    for (int j = 0; j < Np; ++j) {
      xm += db.vx[size_t(e) * Np + j] / Np;
      ym += db.vy[size_t(e) * Np + j] / Np;
      zm += db.vz[size_t(e) * Np + j] / Np;
    }
    int loc[3] = {0, 0, 0};
    if (xm < db.pmlxmin + delta) loc[0] = -1;
    if (xm > db.pmlxmax - delta) loc[0] = 1;
    if (ym < db.pmlymin + delta) loc[1] = -1;
    if (ym > db.pmlymax - delta) loc[1] = 1;
    if (zm < db.pmlzmin + delta) loc[2] = -1;
    // The reference tests zmean > pmlzmax + pml_delta (src/pmlMod.f90:136),
    // which never holds: a PML at the top face gets no z damping.  Kept.
    if (zm > db.pmlzmax + delta) loc[2] = 1;
    const double vpe = db.vp[e];
    auto profile = [&](int dir, double lo, double hi, const std::vector<double>& coordv, double* dd, double* al, double* kk) {
      if (loc[dir] == 0) return;
      const double ar = std::fabs(loc[dir] < 0 ? lo + delta : hi - delta);
      for (int j = 0; j < Np; ++j) {
        const size_t g = size_t(e) * Np + j;
        const double br = std::fabs(ar - std::fabs(coordv[g]));
        dd[g] = -3.0 / (2.0 * delta) * vpe * std::log(par.pml_rc) * (br / delta) * (br / delta);
        al[g] = amax * (1.0 - br / delta);
        kk[g] = 1.0 + par.pml_kmax * (br / delta) * (br / delta);
      }
    };
    profile(0, db.pmlxmin, db.pmlxmax, db.vx, ddx, ax, kx);
    profile(1, db.pmlymin, db.pmlymax, db.vy, ddy, ay, ky);
    profile(2, db.pmlzmin, db.pmlzmax, db.vz, ddz, az, kz);
  }
  const double p = 0.3;  // multiaxial mixing factors
  for (size_t i = 0; i < ng; ++i) {
    if (db.vx[i] > db.pmlxmin + delta && db.vx[i] < db.pmlxmax - delta && db.vy[i] > db.pmlymin + delta &&
        db.vy[i] < db.pmlymax - delta && db.vz[i] > db.pmlzmin + delta) {
      ddx[i] = ddy[i] = ddz[i] = 0.0;
      ax[i] = ay[i] = az[i] = 0.0;
      kx[i] = ky[i] = kz[i] = 1.0;
    }
    const double a = ddx[i], b = ddy[i], c = ddz[i];
    ddx[i] = a + p * b + p * c;
    ddy[i] = p * a + b + p * c;
    ddz[i] = p * a + p * b + c;
  }
}

static void prepare_sources(MeshDB& db) {
  const int Np = db.Np, nsrc = int(db.src.size()), nt = db.par.nt;
  const Mat vdmTinv = [&] {
    Mat v = transpose(db.op.V);
    invert(v);
    return v;
  }();
  db.srcelem.assign(nsrc, 0);
  db.srctype.assign(nsrc, 0);
  db.srcInt.assign(size_t(nsrc) * Np, 0.0);
  db.srcangle.assign(size_t(nsrc) * 3, 0.0);
  db.srcM.assign(size_t(nsrc) * 6, 0.0);
  db.srcbatch.assign(nsrc, 0);
  const int nstage = db.opt.stf_stage_time ? (db.par.timeint == 4 ? 5 : db.par.timeint) : 1;
  db.stf_per_step = nstage;
  db.stf.assign(size_t(nsrc) * nt * nstage, 0.0);
  // stage abscissae c_k of the integrators (the reference's TVD stages sit at
  // t, t+dt, t+dt/2 for RK3; RK2 at t, t+dt)
  std::vector<double> cst;
  if (db.par.timeint == 4)
    cst = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363183471.0,
           2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};
  else if (db.par.timeint == 3) cst = {0.0, 1.0, 0.5};
  else if (db.par.timeint == 2) cst = {0.0, 1.0};
  else cst = {0.0};
  for (int i = 0; i < nsrc; ++i) {
    const Source& s = db.src[i];
    db.srcelem[i] = s.elem;
    db.srctype[i] = s.type;
    db.srcbatch[i] = i % std::max(1, db.opt.nbatch);
    std::vector<double> pr = {s.rst[0]}, ps = {s.rst[1]}, pt = {s.rst[2]};
    Mat phi = vandermonde3d(db.N, pr, ps, pt);  // 1 x Np
    for (int a = 0; a < Np; ++a) {
      double acc = 0.0;
      for (int b = 0; b < Np; ++b) acc += vdmTinv(a, b) * phi(0, b);
      db.srcInt[size_t(i) * Np + a] = acc;
    }
    for (int c = 0; c < 3; ++c) db.srcangle[size_t(i) * 3 + c] = s.angle_force[c];
    for (int c = 0; c < 6; ++c) db.srcM[size_t(i) * 6 + c] = s.M[c];
    const double t0 = db.opt.t0 > 0.0 ? db.opt.t0 : 1.2 / s.f0;
    double* out = &db.stf[size_t(i) * nt * nstage];
    if (nstage == 1) {
      // plotstf(it,2) = -stf((it-1)*dt)  (src/sourceReceiverMod.f90:786-799)
      std::vector<double> tim(nt), val(nt);
      for (int it = 0; it < nt; ++it) {
        tim[it] = double(it) * db.dt;
        val[it] = s.stf == 1 ? -stf_gauss(tim[it], s.f0, t0, s.factor) : -stf_ricker(tim[it], s.f0, t0, s.factor);
      }
      if (s.type == 1 && nt >= 3) {
        // DerivateSTF (src/sourceReceiverMod.f90:816-839)
        std::vector<double> d(nt);
        double a = ((val[0] - val[1]) / (tim[0] - tim[1]) - (val[1] - val[2]) / (tim[1] - tim[2])) / (tim[0] - tim[2]);
        double b = (val[0] - val[1]) / (tim[0] - tim[1]) - a * (tim[0] + tim[1]);
        d[0] = 2 * a * tim[0] + b;
        const int n = nt;
        a = ((val[n - 3] - val[n - 2]) / (tim[n - 3] - tim[n - 2]) - (val[n - 2] - val[n - 1]) / (tim[n - 2] - tim[n - 1])) /
            (tim[n - 3] - tim[n - 1]);
        b = (val[n - 3] - val[n - 2]) / (tim[n - 3] - tim[n - 2]) - a * (tim[n - 3] + tim[n - 2]);
        d[n - 1] = 2 * a * tim[n - 1] + b;
        for (int k = 1; k < n - 1; ++k) d[k] = (val[k + 1] - val[k - 1]) / (tim[k + 1] - tim[k - 1]);
        val = d;
      }
      for (int it = 0; it < nt; ++it) out[it] = val[it];
    } else {
      for (int it = 0; it < nt; ++it)
        for (int k = 0; k < nstage; ++k) {
          const double tt = (double(it) + cst[k]) * db.dt;
          double v;
          if (s.type == 1)
            v = s.stf == 1 ? -stf_gauss_dt(tt, s.f0, t0, s.factor) : -stf_ricker_dt(tt, s.f0, t0, s.factor);
          else
            v = s.stf == 1 ? -stf_gauss(tt, s.f0, t0, s.factor) : -stf_ricker(tt, s.f0, t0, s.factor);
          out[size_t(it) * nstage + k] = v;
        }
    }
  }
  const int nrec = int(db.rec.size());
  db.recelem.assign(nrec, 0);
  db.recInt.assign(size_t(nrec) * Np, 0.0);
  for (int i = 0; i < nrec; ++i) {
    db.recelem[i] = db.rec[i].elem;
    std::vector<double> pr = {db.rec[i].rst[0]}, ps = {db.rec[i].rst[1]}, pt = {db.rec[i].rst[2]};
    Mat phi = vandermonde3d(db.N, pr, ps, pt);
    for (int a = 0; a < Np; ++a) {
      double acc = 0.0;
      for (int b = 0; b < Np; ++b) acc += vdmTinv(a, b) * phi(0, b);
      db.recInt[size_t(i) * Np + a] = acc;
    }
  }
}

static void fill_desc(MeshDB& db) {
  nexd_desc& d = db.desc;
  d = nexd_desc{};
  d.abi_version = NEXD_ABI_VERSION;
  d.N = db.N;
  d.Np = db.Np;
  d.NpF = db.NpF;
  d.nelem = db.nelem;
  d.nMB = db.nMB;
  d.attenuation = db.par.attenuation ? 1 : 0;
  d.set_pml = db.par.set_pml ? 1 : 0;
  d.timeint = db.par.timeint;
  d.nt = db.par.nt;
  d.dt = db.dt;
  d.init_value = db.opt.init_value;
  d.Dr = db.Dr.data();
  d.Ds = db.Ds.data();
  d.Dt = db.Dt.data();
  d.lift = db.lift.data();
  d.invmass = db.invmass.data();
  d.fmask = db.fmask1.data();
  d.metric = db.metric.data();
  d.jacobian = db.jac.data();
  d.fscale = db.fscale.data();
  d.nnormal = db.nn.data();
  d.stangential = db.st.data();
  d.ttangential = db.tt.data();
  d.rho = db.rho.data();
  d.vpu = db.vpu.data();
  d.vsu = db.vsu.data();
  d.lambdau = db.lambdau.data();
  d.muu = db.muu.data();
  d.ylambda = db.nMB ? db.ylambda.data() : nullptr;
  d.ymu = db.nMB ? db.ymu.data() : nullptr;
  d.wl = db.nMB ? db.wl.data() : nullptr;
  d.neighbor = db.neighbor.data();
  d.face = db.face.data();
  d.ibn = db.ibn.data();
  d.pmlcheck = db.pmlcheck.data();
  d.pml_profiles = db.pml_profiles.data();
  d.nsrc = int(db.src.size());
  d.srcelem = db.srcelem.data();
  d.srctype = db.srctype.data();
  d.srcInt = db.srcInt.data();
  d.srcangle_force = db.srcangle.data();
  d.srcM = db.srcM.data();
  d.stf_per_step = db.stf_per_step;
  d.stf = db.stf.data();
  d.nrec = int(db.rec.size());
  d.recelem = db.recelem.data();
  d.recInt = db.recInt.data();
  d.nbatch = std::max(1, db.opt.nbatch);
  d.srcbatch = db.srcbatch.data();
}

void init_parameters(const std::string& dir, const BuildOptions& opt, MeshDB& db) {
  db = MeshDB{};
  db.opt = opt;
  db.par = read_parfile(dir + "/data/parfile");
  if (opt.timeint > 0) db.par.timeint = opt.timeint;
  if (opt.cfl > 0) db.par.cfl = opt.cfl;
  if (opt.nt > 0) db.par.nt = opt.nt;
  if (db.par.timeint < 1 || db.par.timeint > 4) throw std::runtime_error("timeint must be 1..4");
  if (db.par.nt < 1) throw std::runtime_error("nt must be positive");
}

void build_from_directory(const std::string& dir, const BuildOptions& opt, MeshDB& db) {
  init_parameters(dir, opt, db);
  db.N = opt.N;
  db.op = build_operators(opt.N);
  db.Np = db.op.Np;
  db.NpF = db.op.NpF;
  std::vector<std::array<int, 4>> freef, absf;
  read_cubit(dir, db, freef, absf);
  build_topology(db, freef, absf);
  const int K = db.nelem;
  db.mu.resize(K);
  db.lambda.resize(K);
  for (int i = 0; i < K; ++i) {
    db.mu[i] = db.rho[i] * db.vs[i] * db.vs[i];
    db.lambda[i] = db.rho[i] * db.vp[i] * db.vp[i] - 2.0 * db.mu[i];
  }
  db.vpu = db.vp;
  db.vsu = db.vs;
  db.muu = db.mu;
  db.lambdau = db.lambda;
  if (db.par.attenuation) {
    db.nMB = 3;  // nMB (src/constants.h:36)
    anelastic_precalc(db.par.f0_att, db.par.fr_att, db.nMB, db.wl, db.wk);
    db.ylambda.assign(size_t(K) * db.nMB, 0.0);
    db.ymu.assign(size_t(K) * db.nMB, 0.0);
    for (int e = 0; e < K; ++e) {
      anelastic_coefficients(db.qp[e], db.qs[e], db.vp[e], db.vs[e], db.rho[e], db.par.f0_att, db.wl, db.wk,
                             &db.ylambda[size_t(e) * db.nMB], &db.ymu[size_t(e) * db.nMB], db.lambdau[e], db.muu[e]);
      db.vpu[e] = std::sqrt((db.lambdau[e] + 2.0 * db.muu[e]) / db.rho[e]);
      db.vsu[e] = std::sqrt(db.muu[e] / db.rho[e]);
    }
  }
  build_geometry(db);
  db.dt = db.dtfactor * db.par.cfl;
  db.src = read_sources(dir + "/data/source");
  db.rec = read_stations(dir + "/data/stations");
  {
    Locator loc(db);
    for (size_t i = 0; i < db.src.size(); ++i) loc.locate(db.src[i].xyz, db.src[i].elem, db.src[i].rst, "source", int(i) + 1);
    for (size_t i = 0; i < db.rec.size(); ++i) loc.locate(db.rec[i].xyz, db.rec[i].elem, db.rec[i].rst, "receiver", int(i) + 1);
  }
  prepare_solver(db);
}

void prepare_solver(MeshDB& db) {
  db.f0max = 0.0;
  for (const auto& s : db.src) db.f0max = std::max(db.f0max, s.f0);
  build_pml(db);
  prepare_sources(db);
  const int NpF = db.NpF;
  db.Dr = db.op.Dr.a;
  db.Ds = db.op.Ds.a;
  db.Dt = db.op.Dt.a;
  db.lift = db.op.lift.a;
  db.invmass = db.op.invmass.a;
  db.mass = db.op.mass.a;
  db.V = db.op.V.a;
  db.fmask1.resize(size_t(NpF) * 4);
  for (size_t i = 0; i < db.fmask1.size(); ++i) db.fmask1[i] = db.op.fmask[i] + 1;
  fill_desc(db);
}

// Two columns per line, time and value.  The time of step it is (it - 1) dt,
// as in the reference's own seismograms (simulations/brick/ref/seismo.*,
// first row at t = 0); the writer in src/timeloopMod.f90:337-339,591-620
// would label the same rows it*deltat.
void write_seismograms(const std::string& outdir, const MeshDB& db, const float* traces, int nt, int batch) {
  const int nrec = int(db.rec.size());
  static const char* comp[3] = {"x", "y", "z"};
  static const char* kind[3] = {"sdu", "sdv", "sda"};
  const size_t boff = size_t(batch) * nrec * db.par.nt * NEXD_NCOMP;
  for (int r = 0; r < nrec; ++r)
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c) {
        char name[512];
        std::snprintf(name, sizeof name, "%s/seismo.%s.%07d.%s", outdir.c_str(), comp[c], db.rec[r].nr, kind[k]);
        FILE* f = std::fopen(name, "w");
        if (!f) throw std::runtime_error(std::string("cannot write ") + name);
        const int ci = k * 3 + c;
        for (int it = 0; it < nt; ++it) {
          const float v = traces[boff + (size_t(ci) * db.par.nt + it) * nrec + r];
          std::fprintf(f, "   %.8E   %.8E\n", float(double(it) * db.dt), v);
        }
        std::fclose(f);
      }
}

}  // namespace nexd
