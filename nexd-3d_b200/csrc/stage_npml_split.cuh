// NPML stage kernel with two threads per node (sm_100a, FP32).
//
// The same stage as stage_kernel<N, ATT, true, MODE> (the reference's element
// loop for PML elements, src/timeloopMod.f90:395-476 with 399-405, and the
// stage update of RungeKuttaSteps, src/rungekuttaMod.f90:27-88), with each
// node's work shared by two threads of a 512-thread block, so that the state
// a PML node carries (27 auxiliaries, their residuals and 9 profiles besides
// the 9 + 36 values of the ordinary update) is split between two register
// files and the kernel runs 16 warps per SM at <= 128 registers instead of 8
// warps at ~250:
//
//   thread A (tid < 256, node n of element le)     thread B (tid >= 256, same node)
//   loads the residual of q, theta, its residual    loads F', G', H', their residuals, profiles
//   face amplitudes of the chunk                     NPML update, modified contravariant fluxes
//   ------------------------------ barrier ----------------------------------------------
//   volume term of fields 0..5                      volume term of fields 6..8, velocity gradient
//   ------------------------------ barrier ----------------------------------------------
//   lift, memory variables, sources, receivers,
//   stage update of the node
//
// Every value is computed by the same operations in the same order as in
// stage_kernel, so the two kernels give identical results.
#pragma once
#include "stage_kernel.cuh"

namespace nexd_dev {

template <int N>
struct SplitOrder {
  using O = Order<N>;
  static constexpr int THREADS = 512;
  static constexpr int XS = 12;  // values B hands to A per node: volume of fields 6..8, velocity gradient
  static constexpr int SX = O::r4(O::E * O::Np * XS);
  static constexpr int smem_floats() { return O::smem_floats(true) + SX; }
};

// Barrier 1 for all 512 threads of the block, reached from the two roles'
// separate loops (a named barrier with an explicit count is defined for
// arrivals from different code locations).
__device__ __forceinline__ void block_sync_all() { asm volatile("bar.sync 1, 512;" ::: "memory"); }

// Starts the copies of the chunk after w (all threads of the block take part).
template <class O>
__device__ __forceinline__ void issue_next(const StageArgs& a, int w, int nwork, int nchunk, const int* sIds,
                                           float* buf, const unsigned char* sPat) {
  const int wn = w + gridDim.x;
  if (wn < nwork) {
    const Chunk cn = chunk_of<O::E>(a, wn, nchunk);
    const int wnn = wn + gridDim.x;
    Chunk cnn;
    if (wnn < nwork) cnn = chunk_of<O::E>(a, wnn, nchunk);
    issue_chunk<O>(a, cn, sIds, buf, wnn < nwork ? &cnn : nullptr, sPat);
  }
}

template <int N, bool ATT, int MODE>
__global__ void __launch_bounds__(512, 1) stage_npml_split_kernel(const StageArgs a) {
  using O = Order<N>;
  using S = SplitOrder<N>;
  constexpr int Np = O::Np, NpF = O::NpF, NF = O::NF, E = O::E, CS = O::CS, XS = S::XS;
  extern __shared__ __align__(16) float smem[];
  float* sD = smem;                    // 3*Np*Np: D[d][k][n]
  float* sL = sD + O::SD;              // LIFT in face-node pairs
  float* sBuf = sL + O::SL;            // 2 prefetch buffers
  float* sCF = sBuf + 2 * O::BUF;      // contravariant modified fluxes [e][k][CS]
  float* sAmp = sCF + O::SCF;          // face amplitudes, E*3*NFP
  unsigned char* sPat = reinterpret_cast<unsigned char*>(sAmp + O::SAMP);  // face patterns
  float* sX = sAmp + O::SAMP + O::SPAT;  // [e][n][XS]: B's volume results for A

  const int tid = threadIdx.x;
  for (int i = tid; i < 3 * Np * Np; i += blockDim.x) sD[i] = a.D[i];
  for (int i = tid; i < O::SL; i += blockDim.x) sL[i] = a.L[i];
  if (NpF & 1)  // padding slots of the amplitude pairs stay zero
    for (int i = tid; i < E * 3 * 4; i += blockDim.x)
      sAmp[(i >> 2) / 3 * O::AE + (i >> 2) % 3 * O::NFP + (i & 3) * 2 * O::NPAIR + NpF] = 0.f;
  for (int i = tid; i < a.npat * NpF; i += blockDim.x) sPat[i] = a.patterns[i];

  const int nel = a.e_end - a.e_begin;
  const int nchunk = (nel + E - 1) / E;
  const int nwork = nchunk * a.nbatch;
  const bool roleA = tid < 256;
  const int t = roleA ? tid : tid - 256;  // position within the role: the node mapping of stage_kernel
  int le, n;
  if constexpr (O::WARP_ALIGNED) {
    if (t < E * 32) {
      le = t >> 5;
      n = t & 31;
    } else {
      const int r = t - E * 32;
      le = r / (Np - 32);
      n = 32 + r - le * (Np - 32);
    }
  } else {
    le = t / Np;
    n = t - le * Np;
  }
  int w = blockIdx.x;
  if (w >= nwork) return;

  // prologue: connectivity of the first chunk straight from global memory
  {
    const Chunk c0 = chunk_of<E>(a, w, nchunk);
    const int wn = w + gridDim.x;
    Chunk c1;
    if (wn < nwork) c1 = chunk_of<E>(a, wn, nchunk);
    int* ids0 = reinterpret_cast<int*>(sBuf + O::BUF + O::SGEO + O::SQF + O::STR);  // scratch: buffer 1's ids slot
    for (int i = tid; i < c0.ne * 8; i += blockDim.x) {
      const int ee = i >> 3, k = i & 7;
      ids0[ee * 12 + k] = k < 4 ? reinterpret_cast<const int*>(a.nbr)[4 * (c0.e0 + ee) + k]
                                : reinterpret_cast<const int*>(a.fcode)[4 * (c0.e0 + ee) + k - 4];
    }
    __syncthreads();
    issue_chunk<O>(a, c0, ids0, sBuf, wn < nwork ? &c1 : nullptr, sPat);
  }

  // The roles run separate loops over the same chunks (so that the compiler
  // never holds both roles' state at once); they meet at a named barrier
  // for all 512 threads, three times per chunk.
  if (roleA) {
    for (int p = 0; w < nwork; w += gridDim.x, p ^= 1) {
      const Chunk ch = chunk_of<E>(a, w, nchunk);
      const int b = ch.b, e0 = ch.e0, ne = ch.ne;
      float* buf = sBuf + p * O::BUF;
      const float* sGeo = buf;
      const float* sTr = buf + O::SGEO + O::SQF;
      const float* sQF = buf + O::SGEO + int(((long long)e0 * Np) & 3);
      const int* sIds = reinterpret_cast<const int*>(sTr + O::STR);  // connectivity of the next chunk
      cp_async_wait_all();
      block_sync_all();  // (1) this chunk's data is in `buf`; the other buffer and work areas are free
      const bool active = le < ne;
      const int e = e0 + (active ? le : 0);
      const long long node = (long long)e * Np + n;
      const float* g = sGeo + le * O::GSTR;
      NodePrefetch<ATT, false, MODE> pf;
      if (active) pf.template load<Np>(a, b, e, node);
      issue_next<O>(a, w, nwork, nchunk, sIds, sBuf + (p ^ 1) * O::BUF, sPat);
      // ---- face amplitudes --------------------------------------------------------
      for (int i = t; i < ne * NF; i += 256) {
        const int ee = i / NF, j = i - ee * NF;
        const int f = j / NpF, fi = j - f * NpF;
        const float* ge = sGeo + ee * O::GSTR;
        const int code = sIds[ee * 12 + 8 + f];
        const int own = sPat[f * NpF + fi];  // patterns 0..3 are the element's own face masks
        const float* qo = sQF + ee * Np + own;
        float dq[9];
        const bool free_face = face_jump<NpF>(a, b, code, fi, sTr + i * 9, qo, O::QF, dq);
        float ap, as1, as2;
        face_amplitudes(ge, f, dq, free_face, ap, as1, as2);
        const float fs = ge[G_FS + f];
        float* am = sAmp + ee * O::AE + f * 2 * O::NPAIR + fi;
        am[0] = ap * fs;
        am[O::NFP] = as1 * fs;
        am[2 * O::NFP] = as2 * fs;
      }
      block_sync_all();  // (2) amplitudes and B's contravariant rows are in shared memory
      float rq[9];
      if (active) {
        const float* cfe = sCF + le * O::CFE;
        float2 acc[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) acc[j] = make_float2(0.f, 0.f);
#pragma unroll 5
        for (int k = 0; k < Np; ++k) {
          const float dx = sD[k * Np + n], dy = sD[Np * Np + k * Np + n], dz = sD[2 * Np * Np + k * Np + n];
          const float2 d0 = make_float2(dx, dx), d1 = make_float2(dy, dy), d2 = make_float2(dz, dz);
          const float2* cf = reinterpret_cast<const float2*>(cfe + k * CS);
#pragma unroll
          for (int j = 0; j < 3; ++j)
            acc[j] = __ffma2_rn(d0, cf[j], __ffma2_rn(d1, cf[5 + j], __ffma2_rn(d2, cf[10 + j], acc[j])));
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) { rq[2 * j] = acc[j].x; rq[2 * j + 1] = acc[j].y; }
      }
      block_sync_all();  // (3) B's volume results are in sX
      if (!active) continue;
      float vgrad[9];
      {
        const float4* xi = reinterpret_cast<const float4*>(sX + (le * Np + n) * XS);
        const float4 x0 = xi[0], x1 = xi[1], x2 = xi[2];
        rq[6] = x0.x; rq[7] = x0.y; rq[8] = x0.z;
        vgrad[0] = x0.w; vgrad[1] = x1.x; vgrad[2] = x1.y; vgrad[3] = x1.z;
        vgrad[4] = x1.w; vgrad[5] = x2.x; vgrad[6] = x2.y; vgrad[7] = x2.z; vgrad[8] = x2.w;
      }
      (void)vgrad;
      float sig_an[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) sig_an[c] = 0.f;
      (void)sig_an;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        float2 c0 = make_float2(0.f, 0.f), c1 = c0, c2 = c0;
        const float2* lp = reinterpret_cast<const float2*>(sL) + f * O::NPAIR * Np + n;
        const float* ax = sAmp + le * O::AE + f * 2 * O::NPAIR;
        constexpr int FULL = NpF / 2;
#pragma unroll
        for (int ip = 0; ip < FULL; ++ip) {
          const float2 l = lp[ip * Np];
          c0 = __ffma2_rn(l, *reinterpret_cast<const float2*>(ax + 2 * ip), c0);
          c1 = __ffma2_rn(l, *reinterpret_cast<const float2*>(ax + O::NFP + 2 * ip), c1);
          c2 = __ffma2_rn(l, *reinterpret_cast<const float2*>(ax + 2 * O::NFP + 2 * ip), c2);
        }
        if constexpr (NpF & 1) {
          const float l = reinterpret_cast<const float*>(lp + FULL * Np)[0];
          c0.x = fmaf(l, ax[2 * FULL], c0.x);
          c1.x = fmaf(l, ax[O::NFP + 2 * FULL], c1.x);
          c2.x = fmaf(l, ax[2 * O::NFP + 2 * FULL], c2.x);
        }
        face_expand<ATT>(g, f, c0.x + c0.y, c1.x + c1.y, c2.x + c2.y, rq, sig_an);
      }
      float Sv[6];
      if (ATT) {
        // S = -strain rate + lifted anelastic flux; d theta_l/dt = w_l (S - theta_l)
        Sv[0] = sig_an[0] - vgrad[0];
        Sv[1] = sig_an[1] - vgrad[4];
        Sv[2] = sig_an[2] - vgrad[8];
        Sv[3] = sig_an[3] - 0.5f * (vgrad[3] + vgrad[1]);
        Sv[4] = sig_an[4] - 0.5f * (vgrad[7] + vgrad[5]);
        Sv[5] = sig_an[5] - 0.5f * (vgrad[6] + vgrad[2]);
      }
      finish_node<Np, ATT, false, MODE>(a, b, e, node, rq, Sv, pf, sQF + le * Np + n, O::QF);
    }
  } else {
    for (int p = 0; w < nwork; w += gridDim.x, p ^= 1) {
      const Chunk ch = chunk_of<E>(a, w, nchunk);
      const int b = ch.b, e0 = ch.e0, ne = ch.ne;
      float* buf = sBuf + p * O::BUF;
      const float* sGeo = buf;
      const float* sTr = buf + O::SGEO + O::SQF;
      const float* sQF = buf + O::SGEO + int(((long long)e0 * Np) & 3);
      const int* sIds = reinterpret_cast<const int*>(sTr + O::STR);
      cp_async_wait_all();
      block_sync_all();  // (1)
      const bool active = le < ne;
      const int e = e0 + (active ? le : 0);
      const float* g = sGeo + le * O::GSTR;
      float pr[9], av[27], a2[27];
      if (active) {
        const bool need2 = (MODE == MODE_LSERK) || !a.stage_first;
        const float* x = a.aux + eblock<27, Np>(a.lda, b, e, n);
        const float* x2 = a.aux2 + eblock<27, Np>(a.lda, b, e, n);
        const float* pp = a.prof + (long long)e * 9 * Np + n;
#pragma unroll
        for (int i = 0; i < 27; ++i) av[i] = __ldcs(x + i * Np);
#pragma unroll
        for (int i = 0; i < 27; ++i) a2[i] = need2 ? __ldcs(x2 + i * Np) : 0.f;
#pragma unroll
        for (int i = 0; i < 9; ++i) pr[i] = __ldg(pp + i * Np);
      }
      issue_next<O>(a, w, nwork, nchunk, sIds, sBuf + (p ^ 1) * O::BUF, sPat);
      // ---- NPML auxiliary update and contravariant modified fluxes -----------------
      if (active) {
        float qv[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) qv[c] = sQF[c * O::QF + le * Np + n];
        float F[9], G[9], H[9];
        elastic_fluxes(g, qv, F, G, H);
        pml_update<Np, MODE>(a, b, e, n, a.pml_off[b] != 0, pr, av, a2, F, G, H);
        // the row as 8-byte stores (pairs of fields; field 8 with the zero pad)
        float2* cf = reinterpret_cast<float2*>(sCF + le * O::CFE + n * CS);
        float r[10], sv[10], tt[10];
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          r[i] = g[G_RX] * F[i] + g[G_RY] * G[i] + g[G_RZ] * H[i];
          sv[i] = g[G_SX] * F[i] + g[G_SY] * G[i] + g[G_SZ] * H[i];
          tt[i] = g[G_TX] * F[i] + g[G_TY] * G[i] + g[G_TZ] * H[i];
        }
        r[9] = sv[9] = tt[9] = 0.f;
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          cf[j] = make_float2(r[2 * j], r[2 * j + 1]);
          cf[5 + j] = make_float2(sv[2 * j], sv[2 * j + 1]);
          cf[10 + j] = make_float2(tt[2 * j], tt[2 * j + 1]);
        }
      }
      block_sync_all();  // (2)
      if (active) {
        const float* cfe = sCF + le * O::CFE;
        float2 acc3 = make_float2(0.f, 0.f);
        float acc8 = 0.f;
        float2 v01r = make_float2(0.f, 0.f), v01s = v01r, v01t = v01r;
        float v2r = 0.f, v2s = 0.f, v2t = 0.f;
        const float* qv = sQF + le * Np;
#pragma unroll 5
        for (int k = 0; k < Np; ++k) {
          const float dx = sD[k * Np + n], dy = sD[Np * Np + k * Np + n], dz = sD[2 * Np * Np + k * Np + n];
          const float2 d0 = make_float2(dx, dx), d1 = make_float2(dy, dy), d2 = make_float2(dz, dz);
          const float2* cf = reinterpret_cast<const float2*>(cfe + k * CS);
          acc3 = __ffma2_rn(d0, cf[3], __ffma2_rn(d1, cf[8], __ffma2_rn(d2, cf[13], acc3)));
          const float* c8 = cfe + k * CS + 8;
          acc8 = fmaf(dx, c8[0], fmaf(dy, c8[10], fmaf(dz, c8[20], acc8)));
          if (ATT) {
            const float2 v01 = make_float2(qv[6 * O::QF + k], qv[7 * O::QF + k]);
            const float v2 = qv[8 * O::QF + k];
            v01r = __ffma2_rn(d0, v01, v01r);
            v01s = __ffma2_rn(d1, v01, v01s);
            v01t = __ffma2_rn(d2, v01, v01t);
            v2r = fmaf(dx, v2, v2r);
            v2s = fmaf(dy, v2, v2s);
            v2t = fmaf(dz, v2, v2t);
          }
        }
        float x[XS];
        x[0] = acc3.x;
        x[1] = acc3.y;
        x[2] = acc8;
        const float vr[3] = {v01r.x, v01r.y, v2r}, vs3[3] = {v01s.x, v01s.y, v2s},
                    vt3[3] = {v01t.x, v01t.y, v2t};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          x[3 + c * 3 + 0] = ATT ? g[G_RX] * vr[c] + g[G_SX] * vs3[c] + g[G_TX] * vt3[c] : 0.f;
          x[3 + c * 3 + 1] = ATT ? g[G_RY] * vr[c] + g[G_SY] * vs3[c] + g[G_TY] * vt3[c] : 0.f;
          x[3 + c * 3 + 2] = ATT ? g[G_RZ] * vr[c] + g[G_SZ] * vs3[c] + g[G_TZ] * vt3[c] : 0.f;
        }
        // three 16-byte stores: 8 threads at a 12-word stride touch 32 different banks
        float4* xo = reinterpret_cast<float4*>(sX + (le * Np + n) * XS);
        xo[0] = make_float4(x[0], x[1], x[2], x[3]);
        xo[1] = make_float4(x[4], x[5], x[6], x[7]);
        xo[2] = make_float4(x[8], x[9], x[10], x[11]);
      }
      block_sync_all();  // (3)
    }
  }
  cp_async_wait_all();
}

}  // namespace nexd_dev
