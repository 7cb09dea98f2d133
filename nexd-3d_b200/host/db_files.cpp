// The reference's mesher -> solver hand-off files for one partition, as
// Fortran sequential unformatted records (a 4-byte length before and after
// every record, native byte order, default INTEGER and LOGICAL of 4 bytes,
// REAL(CUSTOM_REAL) of 4 bytes, arrays in column-major order):
//   out/meshVar000001  writeMeshVar / readMeshVar (src/meshMod.f90:1401-1640)
//   out/srcVar000001   writeSrcVar / readSrcVar   (src/sourceReceiverMod.f90:615-680)
//   out/recVar000001   writeRecVar / readRecVar   (src/sourceReceiverMod.f90:636-702)
// The record order and shapes follow those routines; the values of the
// partition arrays are the ones the mesher produces with nproc = 1
// (src/meshMod.f90:669-1100: no MPI neighbours, mpi_nemax = nelem).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "mesh_db.hpp"

namespace nexd {

namespace {

constexpr int kNMB = 3;  // nMB (src/constants.h:36): the record shapes use it with or without attenuation

class RecordWriter {
 public:
  explicit RecordWriter(const std::string& path) : path_(path), f_(std::fopen(path.c_str(), "wb")) {
    if (!f_) throw std::runtime_error("cannot write " + path);
  }
  ~RecordWriter() {
    if (f_) std::fclose(f_);
  }
  void close() {
    if (f_ && std::fclose(f_) != 0) {
      f_ = nullptr;
      throw std::runtime_error("write error on " + path_);
    }
    f_ = nullptr;
  }
  void raw(const void* p, size_t bytes) {
    if (bytes > 0x7fffffffu) throw std::runtime_error("record of " + std::to_string(bytes) + " bytes in " + path_ +
                                                      " exceeds the 2 GiB single-record limit");
    const int32_t n = int32_t(bytes);
    bool ok = std::fwrite(&n, 4, 1, f_) == 1;
    if (bytes) ok = ok && std::fwrite(p, 1, bytes, f_) == bytes;
    ok = ok && std::fwrite(&n, 4, 1, f_) == 1;
    if (!ok) throw std::runtime_error("write error on " + path_);
  }
  void i4(int32_t v) { raw(&v, 4); }
  void r4(double v) {
    const float x = float(v);
    raw(&x, 4);
  }
  void i4s(const std::vector<int32_t>& v) { raw(v.data(), v.size() * 4); }
  void r4s(const std::vector<double>& v) {
    std::vector<float> x(v.begin(), v.end());
    raw(x.data(), x.size() * 4);
  }

 private:
  std::string path_;
  FILE* f_;
};

class RecordReader {
 public:
  explicit RecordReader(const std::string& path) : path_(path), f_(std::fopen(path.c_str(), "rb")) {
    if (!f_) throw std::runtime_error("error in databases, files not existing: " + path);
  }
  ~RecordReader() {
    if (f_) std::fclose(f_);
  }
  // Next record; its length must be `bytes` (any length when bytes < 0).
  std::vector<char> next(const char* name, long long bytes) {
    int32_t n0 = 0, n1 = 0;
    if (std::fread(&n0, 4, 1, f_) != 1) throw std::runtime_error(path_ + ": file ends before record " + name);
    if (n0 < 0) throw std::runtime_error(path_ + ": record " + name + " is split into sub-records (> 2 GiB)");
    if (bytes >= 0 && n0 != bytes)
      throw std::runtime_error(path_ + ": record " + name + " has " + std::to_string(n0) + " bytes, expected " +
                               std::to_string(bytes));
    std::vector<char> buf(static_cast<size_t>(n0));
    if (n0 && std::fread(buf.data(), 1, size_t(n0), f_) != size_t(n0))
      throw std::runtime_error(path_ + ": truncated record " + name);
    if (std::fread(&n1, 4, 1, f_) != 1 || n1 != n0)
      throw std::runtime_error(path_ + ": record markers of " + name + " do not match");
    ++count_;
    return buf;
  }
  int32_t i4(const char* name) {
    auto b = next(name, 4);
    int32_t v;
    std::memcpy(&v, b.data(), 4);
    return v;
  }
  double r4(const char* name) {
    auto b = next(name, 4);
    float v;
    std::memcpy(&v, b.data(), 4);
    return v;
  }
  std::vector<int32_t> i4s(const char* name, long long n) {
    auto b = next(name, n * 4);
    std::vector<int32_t> v(static_cast<size_t>(n));
    if (n) std::memcpy(v.data(), b.data(), size_t(n) * 4);
    return v;
  }
  std::vector<double> r4s(const char* name, long long n) {
    auto b = next(name, n * 4);
    std::vector<float> v(static_cast<size_t>(n));
    if (n) std::memcpy(v.data(), b.data(), size_t(n) * 4);
    return std::vector<double>(v.begin(), v.end());
  }
  void expect_end() {
    char c;
    if (std::fread(&c, 1, 1, f_) == 1)
      throw std::runtime_error(path_ + ": unexpected data after record " + std::to_string(count_));
  }

 private:
  std::string path_;
  FILE* f_;
  int count_ = 0;
};

std::string rank_file(const std::string& dir, const char* stem) {
  char name[64];
  std::snprintf(name, sizeof name, "/%s%06d", stem, 1);
  return dir + name;
}

// Vdmr = Dr V (gradVdm3d, since Dr = Vr V^-1) and the weak derivative
// Drw = V Vr^T (V V^T)^-1 (src/meshMod.f90:607-622).
void weak_operators(const DGOperators& op, Mat& Vr, Mat& Vs, Mat& Vt, Mat& Drw, Mat& Dsw, Mat& Dtw) {
  Vr = matmul(op.Dr, op.V);
  Vs = matmul(op.Ds, op.V);
  Vt = matmul(op.Dt, op.V);
  Mat VVt = matmul(op.V, transpose(op.V));
  if (!invert(VVt)) throw std::runtime_error("singular V V^T");
  Drw = matmul(matmul(op.V, transpose(Vr)), VVt);
  Dsw = matmul(matmul(op.V, transpose(Vs)), VVt);
  Dtw = matmul(matmul(op.V, transpose(Vt)), VVt);
}

// Node of element `e` (0-based) closest to xyz, 1-based global number: the
// initial guess findSource / findReceiver store in srci / reci.
int32_t nearest_node(const MeshDB& db, int e, const double* xyz) {
  int best = 0;
  double bd = 1e300;
  for (int j = 0; j < db.Np; ++j) {
    const size_t g = size_t(e) * db.Np + j;
    const double d = (db.vx[g] - xyz[0]) * (db.vx[g] - xyz[0]) + (db.vy[g] - xyz[1]) * (db.vy[g] - xyz[1]) +
                     (db.vz[g] - xyz[2]) * (db.vz[g] - xyz[2]);
    if (d < bd) {
      bd = d;
      best = int(g);
    }
  }
  return best + 1;
}

int order_of(int Np) {
  for (int N = 1; N <= 10; ++N)
    if ((N + 1) * (N + 2) * (N + 3) / 6 == Np) return N;
  throw std::runtime_error("meshVar: Dr is not Np x Np for any order 1..10");
}

}  // namespace

void write_database(const MeshDB& db, const std::string& outdir) {
  const int K = db.nelem, Np = db.Np, NpF = db.NpF, ncoord = db.ncoord;
  const size_t ng = size_t(K) * Np;
  const int nsrc = int(db.src.size()), nrec = int(db.rec.size());
  Mat Vr, Vs, Vt, Drw, Dsw, Dtw;
  weak_operators(db.op, Vr, Vs, Vt, Drw, Dsw, Dtw);
  {
    RecordWriter w(rank_file(outdir, "meshVar"));
    w.i4(int32_t(ng));   // nglob
    w.i4(K);             // nelem
    w.i4(db.nmat);       // nmat
    w.i4(ncoord);        // ncoord
    w.i4(0);             // pinterfaces
    w.i4(0);             // mpi_nn
    w.i4(0);             // mpi_nnmax
    w.i4(0);             // mpi_ne
    w.i4(K);             // mpi_nemax = largest partition
    w.i4(1);             // nproc
    w.i4(nsrc > 0);      // has_src (LOGICAL)
    w.i4(nrec > 0);      // has_rec
    w.r4(db.dtfactor);
    w.r4(db.minGLL_jac);
    w.r4s(db.op.invV.a);
    w.r4s(db.op.V.a);
    w.r4s(db.op.Dr.a);
    w.r4s(db.op.Ds.a);
    w.r4s(db.op.Dt.a);
    w.r4s(Drw.a);
    w.r4s(Dsw.a);
    w.r4s(Dtw.a);
    w.r4s(Vr.a);
    w.r4s(Vs.a);
    w.r4s(Vt.a);
    w.r4s(db.op.mass.a);
    w.r4s(db.op.lift.a);
    std::vector<int32_t> fmask(size_t(NpF) * 4);
    for (size_t i = 0; i < fmask.size(); ++i) fmask[i] = db.op.fmask[i] + 1;
    w.i4s(fmask);
    w.i4s(fmask);  // fmaskv(4*NpF) = fmask in face order (src/meshMod.f90:879-890)
    w.r4s(db.vx);
    w.r4s(db.vy);
    w.r4s(db.vz);
    {
      std::vector<double> mv = db.matval;
      mv.resize(size_t(db.nmat) * 11, 0.0);
      w.r4s(mv);
    }
    // geometric factors per node (element constants of the affine map)
    for (int m = 0; m < 9; ++m) {
      std::vector<double> v(ng);
      for (int e = 0; e < K; ++e) std::fill_n(&v[size_t(e) * Np], Np, db.metric[size_t(e) * 9 + m]);
      w.r4s(v);
    }
    {
      std::vector<double> v(ng);
      for (int e = 0; e < K; ++e) std::fill_n(&v[size_t(e) * Np], Np, db.jac[e]);
      w.r4s(v);
    }
    w.i4s(std::vector<int32_t>(db.mat.begin(), db.mat.end()));
    {
      std::vector<int32_t> ibool(ng);
      for (size_t i = 0; i < ng; ++i) ibool[i] = int32_t(i + 1);
      w.i4s(ibool);
    }
    // nx, ny, nz, sj, fscale per face node (4*NpF, nelem)
    auto per_face_node = [&](auto value) {
      std::vector<double> v(size_t(4) * NpF * K);
      for (int e = 0; e < K; ++e)
        for (int f = 0; f < 4; ++f) std::fill_n(&v[(size_t(e) * 4 + f) * NpF], NpF, value(e, f));
      w.r4s(v);
    };
    for (int c = 0; c < 3; ++c) per_face_node([&](int e, int f) { return db.nn[size_t(e) * 12 + f * 3 + c]; });
    per_face_node([&](int e, int f) { return db.sJ[size_t(e) * 4 + f]; });
    per_face_node([&](int e, int f) { return db.fscale[size_t(e) * 4 + f]; });
    w.r4s(db.nn);
    w.r4s(db.st);
    w.r4s(db.tt);
    w.r4s(db.coord);
    w.i4s(std::vector<int32_t>(db.elem.begin(), db.elem.end()));
    w.i4s(std::vector<int32_t>(db.neighbor.begin(), db.neighbor.end()));
    w.i4s(std::vector<int32_t>(db.face.begin(), db.face.end()));
    // vp vs rho mu lambda; mu, lambda are the unrelaxed moduli with attenuation
    // (src/meshMod.f90:892-922)
    w.r4s(db.vp);
    w.r4s(db.vs);
    w.r4s(db.rho);
    w.r4s(db.par.attenuation ? db.muu : db.mu);
    w.r4s(db.par.attenuation ? db.lambdau : db.lambda);
    w.r4s(db.qp);
    w.r4s(db.qs);
    w.r4s(db.vpu);
    w.r4s(db.vsu);
    w.r4s(db.muu);
    w.r4s(db.lambdau);
    {
      std::vector<double> yl(size_t(kNMB) * K, 0.0), ym(size_t(kNMB) * K, 0.0), wl(kNMB, 0.0);
      if (db.nMB == kNMB) {
        yl = db.ylambda;
        ym = db.ymu;
        wl = db.wl;
      }
      w.r4s(yl);
      w.r4s(ym);
      w.r4s(wl);
    }
    w.i4s(std::vector<int32_t>(db.pml.begin(), db.pml.end()));
    w.r4(db.pmlxmin);
    w.r4(db.pmlxmax);
    w.r4(db.pmlymin);
    w.r4(db.pmlymax);
    w.r4(db.pmlzmin);
    w.r4(db.pmlzmax);
    w.i4s(std::vector<int32_t>(db.ibt.begin(), db.ibt.end()));
    w.i4s(std::vector<int32_t>(db.ibn.begin(), db.ibn.end()));
    {
      std::vector<int32_t> l2g(ncoord);
      for (int i = 0; i < ncoord; ++i) l2g[i] = i + 1;
      w.i4s(l2g);
    }
    w.i4s(std::vector<int32_t>(size_t(16) * K, 0));       // mpi_interface(4,4,nelem)
    w.i4s({});                                            // mpi_neighbor(mpi_nn = 0)
    w.i4s({});                                            // mpi_connection(0, mpi_ne = 0, 2)
    w.i4s({});                                            // mpi_ninterface(0)
    w.i4s(std::vector<int32_t>(size_t(4) * K, 0));        // mpi_ibool(4, mpi_nemax)
    w.i4s(std::vector<int32_t>(size_t(NpF) * 4 * K, 0));  // mpi_ibt(NpF,4,nelem)
    w.i4s({});                                            // mpi_icon(mpi_nnmax = 0)
    w.r4(db.par.pml_delta);
    w.close();
  }
  if (nsrc > 0) {
    RecordWriter w(rank_file(outdir, "srcVar"));
    std::vector<double> xyz, rst, f0, fac, ang, M;
    std::vector<int32_t> el, si, ty, st;
    for (const auto& s : db.src) {
      xyz.insert(xyz.end(), s.xyz, s.xyz + 3);
      rst.insert(rst.end(), s.rst, s.rst + 3);
      el.push_back(s.elem);
      si.push_back(nearest_node(db, s.elem - 1, s.xyz));
      ty.push_back(s.type);
      st.push_back(s.stf);
      f0.push_back(s.f0);
      fac.push_back(s.factor);
      ang.insert(ang.end(), s.angle_force, s.angle_force + 3);
      M.insert(M.end(), s.M, s.M + 6);
    }
    w.i4(nsrc);
    w.r4s(xyz);
    w.r4s(rst);
    w.i4s(el);
    w.i4s(si);
    w.i4s(ty);
    w.i4s(st);
    w.r4s(f0);
    w.r4s(fac);
    w.r4s(ang);
    w.r4s(M);
    w.close();
  }
  if (nrec > 0) {
    RecordWriter w(rank_file(outdir, "recVar"));
    std::vector<double> xyz, rst;
    std::vector<int32_t> el, ri, nr;
    for (const auto& r : db.rec) {
      xyz.insert(xyz.end(), r.xyz, r.xyz + 3);
      rst.insert(rst.end(), r.rst, r.rst + 3);
      el.push_back(r.elem);
      ri.push_back(nearest_node(db, r.elem - 1, r.xyz));
      nr.push_back(r.nr);
    }
    w.i4(nrec);
    w.r4s(xyz);
    w.r4s(rst);
    w.i4s(el);
    w.i4s(ri);
    w.i4s(nr);
    w.close();
  }
}

void build_from_database(const std::string& dir, const BuildOptions& opt, MeshDB& db) {
  init_parameters(dir, opt, db);
  const std::string out = dir + "/out";
  RecordReader r(rank_file(out, "meshVar"));
  const int nglob = r.i4("nglob"), K = r.i4("nelem"), nmat = r.i4("nmat"), ncoord = r.i4("ncoord");
  const int pinterfaces = r.i4("pinterfaces"), mpi_nn = r.i4("mpi_nn"), mpi_nnmax = r.i4("mpi_nnmax");
  const int mpi_ne = r.i4("mpi_ne"), mpi_nemax = r.i4("mpi_nemax"), nproc = r.i4("nproc");
  if (K <= 0 || ncoord < 4 || nmat < 0 || nglob % K != 0)
    throw std::runtime_error("meshVar: inconsistent sizes (nglob, nelem, nmat, ncoord)");
  if (pinterfaces != 0 || mpi_nn != 0)
    throw std::runtime_error("meshVar: partition with MPI interfaces; this solver runs one partition per mesh");
  (void)nproc;
  const int has_src = r.i4("has_src"), has_rec = r.i4("has_rec");
  db.dtfactor = r.r4("dtfactor");
  db.minGLL_jac = r.r4("mingll_jac");
  // operators: Np from the Dr record, then the FP64 set of that order, checked against the file
  const long long npnp = -1;
  auto invV = r.next("invVdm", npnp);
  const int Np = int(std::lround(std::sqrt(double(invV.size() / 4))));
  if (size_t(Np) * Np * 4 != invV.size()) throw std::runtime_error("meshVar: invVdm is not square");
  db.N = order_of(Np);
  db.op = build_operators(db.N);
  db.Np = Np;
  db.NpF = db.op.NpF;
  const int NpF = db.NpF;
  if (nglob != K * Np) throw std::runtime_error("meshVar: nglob != nelem * Np");
  std::vector<double> fileV = r.r4s("Vdm", (long long)Np * Np);
  std::vector<double> fileDr = r.r4s("Dr", (long long)Np * Np);
  for (const char* nm : {"Ds", "Dt", "Drw", "Dsw", "Dtw", "Vdmr", "Vdms", "Vdmt", "mass"}) r.next(nm, 4LL * Np * Np);
  std::vector<double> fileLift = r.r4s("lift", 4LL * Np * NpF);
  {
    double dmax = 0, ref = 0, lmax = 0, lref = 0;
    for (size_t i = 0; i < fileDr.size(); ++i) {
      dmax = std::max(dmax, std::fabs(fileDr[i] - db.op.Dr.a[i]));
      ref = std::max(ref, std::fabs(db.op.Dr.a[i]));
    }
    for (size_t i = 0; i < fileLift.size(); ++i) {
      lmax = std::max(lmax, std::fabs(fileLift[i] - db.op.lift.a[i]));
      lref = std::max(lref, std::fabs(db.op.lift.a[i]));
    }
    if (dmax > 1e-4 * ref || lmax > 1e-4 * lref)
      throw std::runtime_error("meshVar: Dr / lift do not match the order-" + std::to_string(db.N) +
                               " operators of the reference node set");
  }
  {
    auto fm = r.i4s("fmask", 4LL * NpF);
    for (size_t i = 0; i < fm.size(); ++i)
      if (fm[i] != db.op.fmask[i] + 1) throw std::runtime_error("meshVar: fmask differs from the reference face masks");
    r.next("fmaskv", 16LL * NpF);
  }
  db.nelem = K;
  db.nglob = nglob;
  db.ncoord = ncoord;
  db.vx = r.r4s("vx", nglob);
  db.vy = r.r4s("vy", nglob);
  db.vz = r.r4s("vz", nglob);
  db.nmat = nmat;
  db.matval = r.r4s("matval", 11LL * nmat);
  std::vector<double> geo[9];
  static const char* gname[9] = {"rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz"};
  for (int m = 0; m < 9; ++m) geo[m] = r.r4s(gname[m], nglob);
  std::vector<double> jacn = r.r4s("jacobian", nglob);
  db.mat = r.i4s("mat", K);
  std::vector<int32_t> ibool = r.i4s("ibool", (long long)Np * K);
  for (long long i = 0; i < (long long)Np * K; ++i)
    if (ibool[size_t(i)] != i + 1) throw std::runtime_error("meshVar: ibool is not the element-major numbering");
  for (const char* nm : {"nx", "ny", "nz"}) r.next(nm, 16LL * NpF * K);
  std::vector<double> sjn = r.r4s("sj", 4LL * NpF * K);
  std::vector<double> fsn = r.r4s("fscale", 4LL * NpF * K);
  db.nn = r.r4s("nnormal", 12LL * K);
  db.st = r.r4s("stangential", 12LL * K);
  db.tt = r.r4s("ttangential", 12LL * K);
  db.coord = r.r4s("coord", 3LL * ncoord);
  db.elem = r.i4s("elem", 4LL * K);
  db.neighbor = r.i4s("neighbor", 4LL * K);
  db.face = r.i4s("face", 4LL * K);
  db.vp = r.r4s("vp", K);
  db.vs = r.r4s("vs", K);
  db.rho = r.r4s("rho", K);
  db.mu = r.r4s("mu", K);
  db.lambda = r.r4s("lambda", K);
  db.qp = r.r4s("qp", K);
  db.qs = r.r4s("qs", K);
  db.vpu = r.r4s("vpu", K);
  db.vsu = r.r4s("vsu", K);
  db.muu = r.r4s("muu", K);
  db.lambdau = r.r4s("lambdau", K);
  std::vector<double> yl = r.r4s("ylambda", (long long)kNMB * K);
  std::vector<double> ym = r.r4s("ymu", (long long)kNMB * K);
  std::vector<double> wl = r.r4s("wl", kNMB);
  if (db.par.attenuation) {
    db.nMB = kNMB;
    db.ylambda = yl;
    db.ymu = ym;
    db.wl = wl;
  }
  db.pml = r.i4s("pml", K);
  db.pmlxmin = r.r4("pmlxmin");
  db.pmlxmax = r.r4("pmlxmax");
  db.pmlymin = r.r4("pmlymin");
  db.pmlymax = r.r4("pmlymax");
  db.pmlzmin = r.r4("pmlzmin");
  db.pmlzmax = r.r4("pmlzmax");
  db.ibt = r.i4s("ibt", 4LL * NpF * K);
  db.ibn = r.i4s("ibn", 4LL * NpF * K);
  r.next("loc2glob_nodes", 4LL * ncoord);
  r.next("mpi_interface", 64LL * K);
  r.next("mpi_neighbor", 4LL * mpi_nn);
  r.next("mpi_connection", 8LL * mpi_nn * mpi_ne);
  r.next("mpi_ninterface", 4LL * mpi_nn);
  r.next("mpi_ibool", 16LL * mpi_nemax);
  r.next("mpi_ibt", 16LL * NpF * K);
  r.next("mpi_icon", 4LL * mpi_nnmax);
  const double pml_delta = r.r4("pml_delta");
  r.expect_end();
  (void)pml_delta;  // the solver takes pml_delta from the parfile, as timeloop3D does

  // per-element values of the affine elements (node 1 / face node 1)
  db.metric.assign(size_t(K) * 9, 0.0);
  db.jac.assign(K, 0.0);
  db.sJ.assign(size_t(K) * 4, 0.0);
  db.fscale.assign(size_t(K) * 4, 0.0);
  for (int e = 0; e < K; ++e) {
    for (int m = 0; m < 9; ++m) db.metric[size_t(e) * 9 + m] = geo[m][size_t(e) * Np];
    db.jac[e] = jacn[size_t(e) * Np];
    for (int f = 0; f < 4; ++f) {
      db.sJ[size_t(e) * 4 + f] = sjn[(size_t(e) * 4 + f) * NpF];
      db.fscale[size_t(e) * 4 + f] = fsn[(size_t(e) * 4 + f) * NpF];
    }
    for (int f = 0; f < 4; ++f) {
      const int nb = db.neighbor[size_t(e) * 4 + f], fc = db.face[size_t(e) * 4 + f];
      if (nb < 0 || nb > K) throw std::runtime_error("meshVar: neighbour out of range");
      if (nb == 0 && fc != -1 && fc != -2)
        throw std::runtime_error("meshVar: boundary face that is neither free (-1) nor absorbing (-2)");
    }
  }
  for (int i : db.ibn)
    if (i < 0 || i > nglob) throw std::runtime_error("meshVar: ibn out of range");
  db.dt = db.dtfactor * db.par.cfl;

  if (has_src) {
    RecordReader s(rank_file(out, "srcVar"));
    const int n = s.i4("nsrc");
    if (n < 0) throw std::runtime_error("srcVar: negative nsrc");
    auto xyz = s.r4s("srcxyz", 3LL * n), rst = s.r4s("srcrst", 3LL * n);
    auto el = s.i4s("srcelem", n);
    s.next("srci", 4LL * n);
    auto ty = s.i4s("srctype", n), st = s.i4s("srcstf", n);
    auto f0 = s.r4s("srcf0", n), fac = s.r4s("srcfactor", n);
    auto ang = s.r4s("srcangle_force", 3LL * n), M = s.r4s("srcM", 6LL * n);
    s.expect_end();
    db.src.resize(n);
    for (int i = 0; i < n; ++i) {
      Source& x = db.src[i];
      for (int c = 0; c < 3; ++c) {
        x.xyz[c] = xyz[size_t(i) * 3 + c];
        x.rst[c] = rst[size_t(i) * 3 + c];
        x.angle_force[c] = ang[size_t(i) * 3 + c];
      }
      for (int c = 0; c < 6; ++c) x.M[c] = M[size_t(i) * 6 + c];
      x.elem = el[i];
      if (x.elem < 1 || x.elem > K) throw std::runtime_error("srcVar: source element out of range");
      x.type = ty[i];
      x.stf = st[i];
      x.f0 = f0[i];
      x.factor = fac[i];
    }
  }
  if (has_rec) {
    RecordReader s(rank_file(out, "recVar"));
    const int n = s.i4("nrec");
    if (n < 0) throw std::runtime_error("recVar: negative nrec");
    auto xyz = s.r4s("recxyz", 3LL * n), rst = s.r4s("recrst", 3LL * n);
    auto el = s.i4s("recelem", n);
    s.next("reci", 4LL * n);
    auto nr = s.i4s("recnr", n);
    s.expect_end();
    db.rec.resize(n);
    for (int i = 0; i < n; ++i) {
      Receiver& x = db.rec[i];
      for (int c = 0; c < 3; ++c) {
        x.xyz[c] = xyz[size_t(i) * 3 + c];
        x.rst[c] = rst[size_t(i) * 3 + c];
      }
      x.elem = el[i];
      if (x.elem < 1 || x.elem > K) throw std::runtime_error("recVar: receiver element out of range");
      x.nr = nr[i];
    }
  }
  prepare_solver(db);
}

}  // namespace nexd
