// FP64 nodal-DG operators on the reference tetrahedron.
//
// Restates the operator setup the NEXD-3D mesher performs before writing its
// databases (src/meshMod.f90:601-663): warp & blend nodes (src/nodesMod.f90:29),
// orthonormal simplex basis (src/simplexMod.f90:44-165), Vandermonde matrices
// (src/vandermondeMod.f90:63-120), differentiation matrices Dr/Ds/Dt
// (src/dmatricesMod.f90:28-43), face masks (src/meshMod.f90:627-661) and the
// LIFT matrix (src/liftMod.f90:28-76).  The reference computes these in the
// solver's working precision (FP32 by default); this restatement computes them
// in FP64 for any order N = 1..10 and the GPU path rounds them once to FP32.
#pragma once
#include <vector>

namespace nexd {

// Column-major (Fortran order) dense matrix helpers.
struct Mat {
  int rows = 0, cols = 0;
  std::vector<double> a;
  Mat() = default;
  Mat(int r, int c) : rows(r), cols(c), a(size_t(r) * c, 0.0) {}
  double& operator()(int i, int j) { return a[size_t(j) * rows + i]; }
  double operator()(int i, int j) const { return a[size_t(j) * rows + i]; }
};

Mat matmul(const Mat& A, const Mat& B);
Mat transpose(const Mat& A);
// Inverse by LU with partial pivoting; returns false when singular.
bool invert(Mat& A);

struct DGOperators {
  int N = 0, Np = 0, NpF = 0;
  std::vector<double> r, s, t;  // reference-element nodes, size Np
  Mat V, invV, Dr, Ds, Dt, mass, invmass, lift;  // lift: Np x 4NpF
  std::vector<int> fmask;  // NpF x 4, column-major, 0-based node ids
  double minGLL = 0.0;     // |r(1) - r(2)|, used by the time-step estimate
};

// Builds all operators for polynomial order N (1 <= N <= 10).
// `alpha_order` selects the warp parameter balpha(alpha_order) of the
// reference table (the mesher uses balpha(ORDER), src/meshMod.f90:601).
DGOperators build_operators(int N);

// Node set on the equilateral tetrahedron mapped to (r,s,t) for warp
// parameter alpha (nodes3D + xyzToRst).
void nodes_rst(int N, double alpha, std::vector<double>& r, std::vector<double>& s,
               std::vector<double>& t);

// Warp parameter table balpha (src/constants.h:32-33), 1-based index N.
double warp_alpha(int N);

// Orthonormal-basis Vandermonde rows at arbitrary points: out is npts x Np.
Mat vandermonde3d(int N, const std::vector<double>& r, const std::vector<double>& s,
                  const std::vector<double>& t);

}  // namespace nexd
