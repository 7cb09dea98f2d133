// Learned absorbing boundary: a per-face MLP that predicts the exterior
// (ghost) state of an absorbing face from the interior face trace -- its
// features and arguments here, its tensor-core kernel in boundary_tc.cuh --
// and the elementwise training kernels (the training GEMMs are in
// mlp_tc.cuh).
//
// The reference's absorbing faces take the exterior state as zero, so the
// upwind flux only removes the incoming characteristics
// (computeExactRiemannSF with -VT, src/waveMod.f90:269-336).  The flux sees
// the exterior state only through three incoming characteristic values per
// face node, w = (n.S.n - Zp v.n, n.S.s - Zs v.s, n.S.t - Zs v.t), Zp = rho vp,
// Zs = rho vs.  Here the MLP predicts the exterior state q+ of every absorbing
// face from the interior trace q-; its incoming values are clamped to
// |w| <= rho_max |u-| with u- = (n.S.n + Zp v.n, ...) the interior's outgoing
// values (a pointwise reflection coefficient below rho_max < 1, so the
// boundary stays dissipative), and the ghost state carrying exactly those w
// (traction w_P n + w_S1 s + w_S2 t, zero velocity) goes into the ordinary
// interior-face flux.  rho_max = 0, or an MLP whose last layer is zero, gives
// the reference's boundary.
//
// Features of one face (n_in = 9 NpF), per face node in the face frame
// (outward normal n, tangents s, t of the element face), divided by Zp:
// three zeros in place of the trace's own incoming values (the network maps
// the outgoing wave to the incoming values it carries across an absorbing
// face, so it must not see, and send back, what arrives from inside), the
// outgoing values u (3) and the in-plane stresses (s.S.s, t.S.t, s.S.t); the
// face vector is divided by its RMS value r (scale equivariance: the physics
// is linear).  The first three outputs per node are the predicted exterior w
// in the same units (the other six are unused and trained towards zero).  Network: n_in -> H -> H -> n_in, GELU,
// parameters [W1 (H x n_in), b1, W2 (H x H), b2, W3 (n_in x H), b3] row-major.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "stage_kernel.cuh"

namespace nexd_dev {

constexpr int kMlpHidden = 128;

__host__ __device__ constexpr long long mlp_param_count(int nin, int h) {
  return (long long)h * nin + h + (long long)h * h + h + (long long)nin * h + nin;
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// Face-frame features of one node: q (9, Voigt xx yy zz xy yz xz, vx vy vz)
// -> x (9) = (0, 0, 0, u_P, u_S1, u_S2, s.S.s, t.S.t, s.S.t) / Zp with
// u = traction + Z velocity (normal: Zp, tangential: Zs); the incoming values
// w = traction - Z velocity are left out.
__device__ __forceinline__ void face_features(const float* q, const float* n, const float* s, const float* t,
                                              float izp, float ks, float* x) {
  const float* v = q + 6;
  const float vn = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
  const float vs = v[0] * s[0] + v[1] * s[1] + v[2] * s[2];
  const float vt = v[0] * t[0] + v[1] * t[1] + v[2] * t[2];
  // S.a for a = n, s, t
  auto sa = [&](const float* a, float* o) {
    o[0] = q[0] * a[0] + q[3] * a[1] + q[5] * a[2];
    o[1] = q[3] * a[0] + q[1] * a[1] + q[4] * a[2];
    o[2] = q[5] * a[0] + q[4] * a[1] + q[2] * a[2];
  };
  float sn[3], ss[3], st[3];
  sa(n, sn);
  sa(s, ss);
  sa(t, st);
  const float snn = izp * (sn[0] * n[0] + sn[1] * n[1] + sn[2] * n[2]);
  const float sns = izp * (sn[0] * s[0] + sn[1] * s[1] + sn[2] * s[2]);
  const float snt = izp * (sn[0] * t[0] + sn[1] * t[1] + sn[2] * t[2]);
  x[0] = 0.f;
  x[1] = 0.f;
  x[2] = 0.f;
  x[3] = snn + vn;
  x[4] = sns + ks * vs;
  x[5] = snt + ks * vt;
  x[6] = izp * (ss[0] * s[0] + ss[1] * s[1] + ss[2] * s[2]);
  x[7] = izp * (st[0] * t[0] + st[1] * t[1] + st[2] * t[2]);
  x[8] = izp * (ss[0] * t[0] + ss[1] * t[1] + ss[2] * t[2]);
}

struct GhostArgs {
  int nbf, nbatch, NpF;
  long long ldq;
  const float* q;            // current stage input, [b][9][ldq]
  const int* bf_elem;        // [nbf] internal element of the face
  const int* bf_face;        // [nbf] local face 0..3
  const float* geo;          // element records
  const unsigned char* pat;  // own face masks (patterns 0..3)
  int Np;
  const __nv_bfloat16* w;    // parameters, bf16
  float rho_max;             // bound of the incoming / outgoing characteristic ratio
  float* ghost;              // [b][nbf][9][NpF]
};

// ---------------------------------------------------------------------------
// Training (FP32): elementwise kernels and Adam (the GEMMs run on the tensor
// cores, mlp_tc.cuh).
// ---------------------------------------------------------------------------

// z[b][j] += bias[j]; a = gelu(z) (act) or a = z.
__global__ void bias_act_kernel(int rows, int cols, float* z, const float* bias, float* a, int act) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)rows * cols) return;
  const float v = z[i] + bias[i % cols];
  z[i] = v;
  a[i] = act ? gelu(v) : v;
}

// d[b][j] = d[b][j] * gelu'(z[b][j])
__global__ void gelu_back_kernel(long long n, float* d, const float* z) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] *= gelu_grad(z[i]);
}

// dy = 2 (y - t) / rows; per-block partial sums of (y - t)^2 (fixed order).
__global__ void mse_kernel(long long n, int rows, const float* y, const float* t, float* dy, float* partial) {
  __shared__ float red[256];
  float s = 0.f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    dy[i] = 2.f * d / rows;
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void sum_partials_kernel(int n, const float* partial, int rows, float* loss) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float s = 0.f;
  for (int i = 0; i < n; ++i) s += partial[i];
  *loss = s / rows;
}

// out[j] = sum_b d[b][j] (bias gradients), one thread per column.
__global__ void colsum_kernel(int rows, int cols, const float* d, float* out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  float s = 0.f;
  for (int b = 0; b < rows; ++b) s += d[(long long)b * cols + j];
  out[j] = s;
}

__global__ void adam_kernel(long long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void to_bf16_kernel(long long n, const float* src, __nv_bfloat16* dst) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

}  // namespace nexd_dev
