// Learned absorbing boundary: a per-face MLP that predicts the exterior
// (ghost) state of an absorbing face from the interior face trace, and the
// FP32 training kernels (forward, backward, Adam) for it.
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

constexpr int kGhostFaces = 16;  // faces per block pass
constexpr int kGhostThreads = 256;

// Shared memory: bf16 parameters + activation tiles [k][face] in FP32
// (features, two hidden layers, prediction) + the RMS scales.
__host__ __device__ constexpr size_t ghost_smem_bytes(int nin) {
  return size_t(mlp_param_count(nin, kMlpHidden)) * 2 + 16 +
         size_t(2 * nin + 2 * kMlpHidden + 1) * kGhostFaces * 4 + 16;
}

// Persistent: each block stages the bf16 parameters once, then loops over
// groups of kGhostFaces (batch member, face) pairs.  Layers: thread j of each
// half-block computes neuron j for 8 faces (FP32 accumulation).
__global__ void __launch_bounds__(kGhostThreads) ghost_kernel(const GhostArgs a) {
  extern __shared__ __align__(16) unsigned char gsm[];
  const int nin = 9 * a.NpF, H = kMlpHidden;
  const long long np_ = mlp_param_count(nin, H);
  __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(gsm);
  float* sx = reinterpret_cast<float*>(gsm + ((np_ * 2 + 15) / 16) * 16);  // [nin][F]
  float* sh1 = sx + nin * kGhostFaces;                                      // [H][F]
  float* sh2 = sh1 + H * kGhostFaces;                                       // [H][F]
  float* sy = sh2 + H * kGhostFaces;                                        // [nin][F] prediction
  float* sr = sy + nin * kGhostFaces;                                       // [F] RMS scale
  const int tid = threadIdx.x;
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.w);
    uint4* dst = reinterpret_cast<uint4*>(sw);
    const long long n16 = np_ * 2 / 16;
    for (long long i = tid; i < n16; i += blockDim.x) dst[i] = src[i];
    for (long long i = n16 * 8 + tid; i < np_; i += blockDim.x) sw[i] = a.w[i];
  }
  const __nv_bfloat16* W1 = sw;
  const __nv_bfloat16* b1 = W1 + (long long)H * nin;
  const __nv_bfloat16* W2 = b1 + H;
  const __nv_bfloat16* b2 = W2 + (long long)H * H;
  const __nv_bfloat16* W3 = b2 + H;
  const __nv_bfloat16* b3 = W3 + (long long)nin * H;
  const int total = a.nbf * a.nbatch;
  const int F = kGhostFaces;
  for (int g0 = blockIdx.x * F; g0 < total; g0 += gridDim.x * F) {
    __syncthreads();
    // features: one thread per (face, node)
    for (int i = tid; i < F * a.NpF; i += blockDim.x) {
      const int fl = i / a.NpF, fi = i - fl * a.NpF;
      const int gi = g0 + fl;
      float x[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (gi < total) {
        const int b = gi / a.nbf, g = gi - b * a.nbf;
        const int e = a.bf_elem[g], f = a.bf_face[g];
        const float* geo = a.geo + (long long)e * GEO_STRIDE;
        const long long node = (long long)e * a.Np + a.pat[f * a.NpF + fi];
        const float* qb = a.q + (long long)b * 9 * a.ldq + node;
        float q[9];
        for (int c = 0; c < 9; ++c) q[c] = qb[c * a.ldq];
        face_features(q, geo + G_N + 3 * f, geo + G_S + 3 * f, geo + G_T + 3 * f, geo[G_IZP],
                      geo[G_IZP] / geo[G_IZS], x);
      }
      for (int c = 0; c < 9; ++c) sx[(fi * 9 + c) * F + fl] = x[c];
    }
    __syncthreads();
    if (tid < F) {
      float ss = 0.f;
      for (int k = 0; k < nin; ++k) ss += sx[k * F + tid] * sx[k * F + tid];
      sr[tid] = sqrtf(ss / nin);
    }
    __syncthreads();
    for (int i = tid; i < nin * F; i += blockDim.x) {
      const float r = sr[i % F];
      sx[i] = r > 0.f ? sx[i] / r : 0.f;
    }
    __syncthreads();
    // dense layers: out[j][f] = act(sum_k W[j][k] in[k][f] + b[j]), 8 faces per thread
    auto layer = [&](const __nv_bfloat16* W, const __nv_bfloat16* bias, const float* in, int kin, float* out,
                     int nout, bool act) {
      for (int j2 = tid; j2 < 2 * nout; j2 += blockDim.x) {
        const int j = j2 >> 1, h = (j2 & 1) * 8;
        float acc[8];
        const float bj = __bfloat162float(bias[j]);
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u] = bj;
        const __nv_bfloat16* wr = W + (long long)j * kin;
        for (int k = 0; k < kin; ++k) {
          const float w = __bfloat162float(wr[k]);
          const float4 x0 = *reinterpret_cast<const float4*>(in + k * F + h);
          const float4 x1 = *reinterpret_cast<const float4*>(in + k * F + h + 4);
          acc[0] = fmaf(w, x0.x, acc[0]);
          acc[1] = fmaf(w, x0.y, acc[1]);
          acc[2] = fmaf(w, x0.z, acc[2]);
          acc[3] = fmaf(w, x0.w, acc[3]);
          acc[4] = fmaf(w, x1.x, acc[4]);
          acc[5] = fmaf(w, x1.y, acc[5]);
          acc[6] = fmaf(w, x1.z, acc[6]);
          acc[7] = fmaf(w, x1.w, acc[7]);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) out[j * F + h + u] = act ? gelu(acc[u]) : acc[u];
      }
    };
    layer(W1, b1, sx, nin, sh1, H, true);
    __syncthreads();
    layer(W2, b2, sh1, H, sh2, H, true);
    __syncthreads();
    layer(W3, b3, sh2, H, sy, nin, false);
    __syncthreads();
    for (int i = tid; i < F * a.NpF; i += blockDim.x) {
      const int fl = i / a.NpF, fi = i - fl * a.NpF;
      const int gi = g0 + fl;
      if (gi >= total) continue;
      const int b = gi / a.nbf, g = gi - b * a.nbf;
      const int e = a.bf_elem[g], f = a.bf_face[g];
      const float* geo = a.geo + (long long)e * GEO_STRIDE;
      // incoming values of the prediction, clamped by the outgoing values of the trace
      const float* x = sx + fi * 9 * F + fl;
      const float* y = sy + fi * 9 * F + fl;
      const float r = sr[fl] / geo[G_IZP];  // RMS scale times Zp
      float w[3];
      for (int k = 0; k < 3; ++k) {
        const float bnd = a.rho_max * fabsf(x[(3 + k) * F]);
        w[k] = r * fminf(fmaxf(y[k * F], -bnd), bnd);
      }
      // ghost: traction w0 n + w1 s + w2 t, zero velocity
      const float* n = geo + G_N + 3 * f;
      const float* s = geo + G_S + 3 * f;
      const float* t = geo + G_T + 3 * f;
      float q[9];
      // S = w0 n n + w1 (n s + s n) + w2 (n t + t n): S n = w0 n + w1 s + w2 t (n.n = 1, s.n = t.n = 0)
      auto comp = [&](int p, int q2) {
        return w[0] * n[p] * n[q2] + w[1] * (n[p] * s[q2] + s[p] * n[q2]) + w[2] * (n[p] * t[q2] + t[p] * n[q2]);
      };
      q[0] = comp(0, 0);
      q[1] = comp(1, 1);
      q[2] = comp(2, 2);
      q[3] = comp(0, 1);
      q[4] = comp(1, 2);
      q[5] = comp(0, 2);
      q[6] = q[7] = q[8] = 0.f;
      float* out = a.ghost + ((long long)b * a.nbf + g) * 9 * a.NpF + fi;
      for (int c = 0; c < 9; ++c) out[c * a.NpF] = q[c];
    }
  }
}

// ---------------------------------------------------------------------------
// Training (FP32): tiled GEMM C = op(A) op(B) (+ C), elementwise kernels, Adam.
// ---------------------------------------------------------------------------

// C[M][N] (row stride ldc) = sum_k A(m,k) B(k,n) (+ C when accumulate), where
// A(m,k) = TA ? A[k*lda + m] : A[m*lda + k] and B(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n].
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                   const float* __restrict__ B, int ldb, float* C, int ldc,
                                                   int accumulate) {
  constexpr int T = 64, KT = 16;
  __shared__ float sa[KT][T + 4];
  __shared__ float sb[KT][T + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * T, n0 = blockIdx.x * T;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += KT) {
    for (int i = threadIdx.x; i < KT * T; i += 256) {
      const int kk = i / T, mm = i - kk * T;
      const int m = m0 + mm, k = k0 + kk;
      sa[kk][mm] = (m < M && k < K) ? (TA ? A[(long long)k * lda + m] : A[(long long)m * lda + k]) : 0.f;
      const int n = n0 + mm;
      sb[kk][mm] = (n < N && k < K) ? (TB ? B[(long long)n * ldb + k] : B[(long long)k * ldb + n]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < KT; ++kk) {
      float av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        av[u] = sa[kk][ty + 16 * u];
        bv[u] = sb[kk][tx + 16 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(av[u], bv[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int m = m0 + ty + 16 * u, n = n0 + tx + 16 * v;
      if (m < M && n < N) {
        float* c = C + (long long)m * ldc + n;
        *c = accumulate ? *c + acc[u][v] : acc[u][v];
      }
    }
}

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
