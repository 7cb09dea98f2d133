// Wavefield energy and the NPML STA/LTA trigger (src/timeloopMod.f90:482-542).
//
// energy_kernel: per element 1/2 J [rho v^T M v + sum_{i<=3} q_i^T M e_i +
// 2 sum_{i>3} q_i^T M e_i] with the strain-like e from q (the reference's
// expression or the isotropic compliance), reduced per block in FP64 into
// `partials` (one slot per block and wavefield).  energy_finalize sums the
// partials in a fixed order (reproducible), stores E(it) and applies the
// reference's trigger rule on the device.
#pragma once
#include <cuda_runtime.h>

namespace nexd_dev {

struct EnergyArgs {
  int K, Np, nbatch;
  long long ldq;
  const float* q;       // [b][9][ldq], element-major nodes
  const float4* emat;   // [K] (rho, lambda, mu, J)
  const double* mass;   // [Np][Np] row-major M(n,k)
  double* partials;     // [nbatch][gridDim.x]
  int formula;          // 0 reference expression, 1 isotropic compliance
};

constexpr int kEnergyThreads = 256;

// The strain-like e is FP64 as in the reference (real(kind=8) :: e,
// src/timeloopMod.f90:120), whose expression reaches 1e30+ at ordinary
// stresses.
__device__ __forceinline__ void strain_of(const float* q, float lam_f, float mu_f, int formula, double* e) {
  const double lam = lam_f, mu = mu_f;
  const double q0 = q[0], q1 = q[1], q2 = q[2];
  const double a = 2.0 * (lam + mu);
  if (formula == 0) {
    // e(:,1..3) = (2(lambda+mu) q_i - lambda (q_j + q_k)) / temp1 with
    // temp1 = 1/(4 mu^2 + 6 mu lambda); e3 uses q1 + q1; e(:,4..6) = q/(2 mu)
    const double t1 = 1.0 / (4.0 * mu * mu + 6.0 * mu * lam);
    e[0] = (a * q0 - lam * (q1 + q2)) / t1;
    e[1] = (a * q1 - lam * (q0 + q2)) / t1;
    e[2] = (a * q2 - lam * (q0 + q0)) / t1;
  } else {
    const double t1 = 4.0 * mu * mu + 6.0 * mu * lam;
    e[0] = (a * q0 - lam * (q1 + q2)) / t1;
    e[1] = (a * q1 - lam * (q0 + q2)) / t1;
    e[2] = (a * q2 - lam * (q0 + q1)) / t1;
  }
  e[3] = q[3] / (2.0 * mu);
  e[4] = q[4] / (2.0 * mu);
  e[5] = q[5] / (2.0 * mu);
}

// Grid (nblocks, nbatch); dynamic shared memory: (Np*Np + E*9*Np) doubles, E = 256/Np.
__global__ void __launch_bounds__(kEnergyThreads) energy_kernel(const EnergyArgs a) {
  extern __shared__ __align__(16) double esm[];
  const int Np = a.Np, E = kEnergyThreads / Np;
  double* sM = esm;                // Np*Np
  double* sX = esm + Np * Np;      // [e][9][Np]: v_x, v_y, v_z, e_1..e_6
  __shared__ double red[kEnergyThreads / 32];
  const int tid = threadIdx.x, b = blockIdx.y;
  for (int i = tid; i < Np * Np; i += blockDim.x) sM[i] = a.mass[i];
  const int le = tid / Np, n = tid - le * Np;
  const float* q = a.q + (long long)b * 9 * a.ldq;
  double acc = 0.0;
  const int nchunk = (a.K + E - 1) / E;
  for (int ch = blockIdx.x; ch < nchunk; ch += gridDim.x) {
    const int e0 = ch * E;
    const int ne = min(E, a.K - e0);
    const bool active = le < ne;
    float qv[9];
    float4 em = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    if (active) {
      const long long node = (long long)(e0 + le) * Np + n;
#pragma unroll
      for (int c = 0; c < 9; ++c) qv[c] = q[c * a.ldq + node];
      em = a.emat[e0 + le];
      double e[6];
      strain_of(qv, em.y, em.z, a.formula, e);
      double* x = sX + le * 9 * Np + n;
      x[0] = qv[6];
      x[Np] = qv[7];
      x[2 * Np] = qv[8];
#pragma unroll
      for (int c = 0; c < 6; ++c) x[(3 + c) * Np] = e[c];
    }
    __syncthreads();
    if (active) {
      // (M x)(n) for the 9 rows, contracted with the node's own values
      double mx[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) mx[c] = 0.0;
      const double* xe = sX + le * 9 * Np;
      const double* Mrow = sM + n * Np;
      for (int k = 0; k < Np; ++k) {
        const double m = Mrow[k];
#pragma unroll
        for (int c = 0; c < 9; ++c) mx[c] = fma(m, xe[c * Np + k], mx[c]);
      }
      const double kin = double(qv[6]) * mx[0] + double(qv[7]) * mx[1] + double(qv[8]) * mx[2];
      const double pot = double(qv[0]) * mx[3] + double(qv[1]) * mx[4] + double(qv[2]) * mx[5] +
                         2.0 * (double(qv[3]) * mx[6] + double(qv[4]) * mx[7] + double(qv[5]) * mx[8]);
      acc += 0.5 * double(em.w) * (double(em.x) * kin + pot);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((tid & 31) == 0) red[tid >> 5] = acc;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int w = 0; w < kEnergyThreads / 32; ++w) s += red[w];
    a.partials[(long long)b * gridDim.x + blockIdx.x] = s;
  }
}

struct TriggerArgs {
  const double* partials;  // [nbatch][nparts]
  int nparts;
  double* energy;          // [nbatch][nt]
  int nt;
  const int* it_dev;       // current step (1-based)
  int armed;               // STA/LTA active
  int timecrit;            // int(2.4 / f0 / dt)
  int w1, w2;
  float threshold;
  int* pml_off;            // [nbatch]
  int* pml_switch;         // [nbatch]
};

// One block per wavefield: fixed-order sum of the partials, E(it), and the
// trigger rule of src/timeloopMod.f90:517-541 (averages in FP32 as there).
__global__ void energy_finalize(const TriggerArgs a) {
  __shared__ double red[256];
  const int b = blockIdx.x, tid = threadIdx.x;
  double s = 0.0;
  for (int i = tid; i < a.nparts; i += blockDim.x) s += a.partials[(long long)b * a.nparts + i];
  red[tid] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid != 0) return;
  const int it = *a.it_dev;
  double* E = a.energy + (long long)b * a.nt;
  E[it - 1] = red[0];
  if (!a.armed || a.pml_off[b] || it <= a.timecrit) return;
  float avg1 = 0.f, avg2 = 0.f;
  for (int i = 1; i <= a.w1; ++i)
    if (it - i > 0) avg1 += float(E[it - i - 1] / a.w1);
  for (int i = 1; i <= a.w2; ++i)
    if (it - i > 0) avg2 += float(E[it - i - 1] / a.w2);
  const float sta_lta = avg2 / avg1;
  if (fabsf(sta_lta - 1.f) > a.threshold) {
    a.pml_off[b] = 1;
    a.pml_switch[b] = it;
  }
}

}  // namespace nexd_dev
