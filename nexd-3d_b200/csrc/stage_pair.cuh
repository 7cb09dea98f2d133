// Stage kernel for elements outside the NPML with a thread per node pair
// (FP32, CUDA cores).
//
// Same stage and the same arithmetic, operation for operation, as
// stage_kernel<N, ATT, false, MODE> (results are bit-identical); a thread
// owns nodes p and p + NPP of one element (NPP = ceil(Np / 2)) and a chunk
// holds twice the elements.  The volume and lift loops then read each
// element value they broadcast (the wavefield of node k, the face
// amplitudes) once for two nodes: shared-memory vector loads of values every
// thread of an element reads cost the same wavefronts as loads of distinct
// values, and they dominate the single-node kernel's shared-memory pipe.
#pragma once
#include "stage_kernel.cuh"

namespace nexd_dev {

// d/dr, d/ds, d/dt of the 9 fields (packed pairs: fields 2j, 2j+1; pair 4 =
// field 8 + pad) -> the velocity-stress volume term and the velocity gradient.
template <bool ATT>
__device__ __forceinline__ void volume_combine(const float* g, const float2* ar, const float2* as_, const float2* at,
                                               float* rq, float* vgrad) {
  float dr[9], ds[9], dtt[9];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    dr[2 * j] = ar[j].x; dr[2 * j + 1] = ar[j].y;
    ds[2 * j] = as_[j].x; ds[2 * j + 1] = as_[j].y;
    dtt[2 * j] = at[j].x; dtt[2 * j + 1] = at[j].y;
  }
  dr[8] = ar[4].x; ds[8] = as_[4].x; dtt[8] = at[4].x;
  const float rx = g[G_RX], ry = g[G_RY], rz = g[G_RZ], sx = g[G_SX], sy = g[G_SY], sz = g[G_SZ],
              tx = g[G_TX], ty = g[G_TY], tz = g[G_TZ];
  auto DX = [&](int c) { return rx * dr[c] + sx * ds[c] + tx * dtt[c]; };
  auto DY = [&](int c) { return ry * dr[c] + sy * ds[c] + ty * dtt[c]; };
  auto DZ = [&](int c) { return rz * dr[c] + sz * ds[c] + tz * dtt[c]; };
  const float e1 = g[G_E1], e2 = g[G_E2], e3 = g[G_E3], e4 = g[G_E4];
  const float dxv = DX(6), dyv = DY(6), dzv = DZ(6);  // grad vx
  const float dxw = DX(7), dyw = DY(7), dzw = DZ(7);  // grad vy
  const float dxu = DX(8), dyu = DY(8), dzu = DZ(8);  // grad vz
  rq[0] = e1 * dxv + e2 * dyw + e2 * dzu;
  rq[1] = e2 * dxv + e1 * dyw + e2 * dzu;
  rq[2] = e2 * dxv + e2 * dyw + e1 * dzu;
  rq[3] = e3 * dxw + e3 * dyv;
  rq[4] = e3 * dyu + e3 * dzw;
  rq[5] = e3 * dxu + e3 * dzv;
  rq[6] = e4 * (DX(0) + DY(3) + DZ(5));
  rq[7] = e4 * (DX(3) + DY(1) + DZ(4));
  rq[8] = e4 * (DX(5) + DY(4) + DZ(2));
  if (ATT) {
    vgrad[0] = dxv; vgrad[1] = dyv; vgrad[2] = dzv;
    vgrad[3] = dxw; vgrad[4] = dyw; vgrad[5] = dzw;
    vgrad[6] = dxu; vgrad[7] = dyu; vgrad[8] = dzu;
  }
}

template <int N, bool ATT, int MODE>
__global__ void __launch_bounds__(256, 1) stage_pair_kernel(const StageArgs a) {
  using O = Order<N, 2>;
  constexpr int Np = O::Np, NpF = O::NpF, NF = O::NF, E = O::E, QS = O::QS, NPP = O::NPP;
  extern __shared__ __align__(16) float smem[];
  float* sD = smem;
  float* sL = sD + O::SD;
  float* sBuf = sL + O::SL;
  float* sQI = sBuf + 2 * O::BUF;
  float* sAmp = sQI + O::SQI;
  unsigned char* sPat = reinterpret_cast<unsigned char*>(sAmp + O::SAMP);

  const int tid = threadIdx.x;
  for (int i = tid; i < 3 * Np * Np; i += blockDim.x) sD[i] = a.D[i];
  for (int i = tid; i < O::SL; i += blockDim.x) sL[i] = a.L[i];
  if (NpF & 1)
    for (int i = tid; i < E * 3 * 4; i += blockDim.x)
      sAmp[(i >> 2) / 3 * O::AE + (i >> 2) % 3 * O::NFP + (i & 3) * 2 * O::NPAIR + NpF] = 0.f;
  for (int i = tid; i < a.npat * NpF; i += blockDim.x) sPat[i] = a.patterns[i];

  const int nel = a.e_end - a.e_begin;
  const int nchunk = (nel + E - 1) / E;
  const int nwork = nchunk * a.nbatch;
  const int le = tid / NPP;                 // element of this thread within the chunk
  const int n1 = tid - le * NPP;            // first node
  const int n2 = n1 + NPP;                  // second node (absent when n2 >= Np)
  const bool has2 = n2 < Np;
  const int n2c = has2 ? n2 : n1;           // loops run on a valid node; the result is dropped
  int w = blockIdx.x;
  if (w >= nwork) return;

  {
    const Chunk c0 = chunk_of<E>(a, w, nchunk);
    const int wn = w + gridDim.x;
    Chunk c1;
    if (wn < nwork) c1 = chunk_of<E>(a, wn, nchunk);
    int* ids0 = reinterpret_cast<int*>(sBuf + O::BUF + O::SGEO + O::SQF + O::STR);
    for (int i = tid; i < c0.ne * 8; i += blockDim.x) {
      const int ee = i >> 3, k = i & 7;
      ids0[ee * 12 + k] = k < 4 ? reinterpret_cast<const int*>(a.nbr)[4 * (c0.e0 + ee) + k]
                                : reinterpret_cast<const int*>(a.fcode)[4 * (c0.e0 + ee) + k - 4];
    }
    __syncthreads();
    issue_chunk<O>(a, c0, ids0, sBuf, wn < nwork ? &c1 : nullptr, sPat);
  }

  for (int p = 0; w < nwork; w += gridDim.x, p ^= 1) {
    const Chunk ch = chunk_of<E>(a, w, nchunk);
    const int b = ch.b, e0 = ch.e0, ne = ch.ne;
    float* buf = sBuf + p * O::BUF;
    const float* sGeo = buf;
    const float* sTr = buf + O::SGEO + O::SQF;
    // own wavefield of the chunk: field c of node n of element le at sQF[c * QF + le * Np + n]
    const float* sQF = buf + O::SGEO + int(((long long)e0 * Np) & 3);
    const int* sIds = reinterpret_cast<const int*>(sTr + O::STR);
    cp_async_wait_all();
    __syncthreads();

    const bool active = le < ne;
    const long long base = (long long)(e0 + (active ? le : 0)) * Np;
    NodePrefetch<ATT, false, MODE> pf1, pf2;
    if (active) {
      pf1.template load<Np>(a, b, e0 + le, base + n1);
      if (has2) pf2.template load<Np>(a, b, e0 + le, base + n2);
    }
    {
      const int wn = w + gridDim.x;
      if (wn < nwork) {
        const Chunk cn = chunk_of<E>(a, wn, nchunk);
        const int wnn = wn + gridDim.x;
        Chunk cnn;
        if (wnn < nwork) cnn = chunk_of<E>(a, wnn, nchunk);
        issue_chunk<O>(a, cn, sIds, sBuf + (p ^ 1) * O::BUF, wnn < nwork ? &cnn : nullptr, sPat);
      }
    }
    // interleaved own wavefield of both nodes
    if (active) {
      float* dst = sQI + le * O::QE;
#pragma unroll
      for (int c = 0; c < 9; ++c) dst[n1 * QS + c] = sQF[c * O::QF + le * Np + n1];
      if (has2) {
#pragma unroll
        for (int c = 0; c < 9; ++c) dst[n2 * QS + c] = sQF[c * O::QF + le * Np + n2];
      }
    }
    for (int i = tid; i < ne * NF; i += blockDim.x) {
      const int ee = i / NF, j = i - ee * NF;
      const int f = j / NpF, fi = j - f * NpF;
      const float* g = sGeo + ee * O::GSTR;
      const int code = sIds[ee * 12 + 8 + f];
      const int own = sPat[f * NpF + fi];
      const float* qo = sQF + ee * Np + own;
      float dq[9];
      const bool free_face = face_jump<NpF>(a, b, code, fi, sTr + i * 9, qo, O::QF, dq);
      float ap, as1, as2;
      face_amplitudes(g, f, dq, free_face, ap, as1, as2);
      const float fs = g[G_FS + f];
      float* am = sAmp + ee * O::AE + f * 2 * O::NPAIR + fi;
      am[0] = ap * fs;
      am[O::NFP] = as1 * fs;
      am[2 * O::NFP] = as2 * fs;
    }
    __syncthreads();
    if (!active) continue;

    const int e = e0 + le;
    const float* g = sGeo + le * O::GSTR;
    float rq1[9], rq2[9], vg1[9], vg2[9];
    (void)vg1;
    (void)vg2;
    // ---- volume term, both nodes ---------------------------------------------------
    {
      float2 ar1[5], as1[5], at1[5], ar2[5], as2[5], at2[5];
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        ar1[j] = make_float2(0.f, 0.f); as1[j] = ar1[j]; at1[j] = ar1[j];
        ar2[j] = ar1[j]; as2[j] = ar1[j]; at2[j] = ar1[j];
      }
      const float* qe = sQI + le * O::QE;
#pragma unroll 5
      for (int k = 0; k < Np; ++k) {
        const float* dk = sD + k * Np;
        const float x1 = dk[n1], y1 = dk[Np * Np + n1], z1 = dk[2 * Np * Np + n1];
        const float x2 = dk[n2c], y2 = dk[Np * Np + n2c], z2 = dk[2 * Np * Np + n2c];
        const float4 qa = ld4(qe + k * QS), qb = ld4(qe + k * QS + 4);
        const float2 qc = *reinterpret_cast<const float2*>(qe + k * QS + 8);
        const float2 qp[5] = {make_float2(qa.x, qa.y), make_float2(qa.z, qa.w), make_float2(qb.x, qb.y),
                              make_float2(qb.z, qb.w), qc};
        const float2 a1 = make_float2(x1, x1), b1 = make_float2(y1, y1), c1 = make_float2(z1, z1);
        const float2 a2 = make_float2(x2, x2), b2 = make_float2(y2, y2), c2 = make_float2(z2, z2);
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          ar1[j] = __ffma2_rn(a1, qp[j], ar1[j]);
          as1[j] = __ffma2_rn(b1, qp[j], as1[j]);
          at1[j] = __ffma2_rn(c1, qp[j], at1[j]);
          ar2[j] = __ffma2_rn(a2, qp[j], ar2[j]);
          as2[j] = __ffma2_rn(b2, qp[j], as2[j]);
          at2[j] = __ffma2_rn(c2, qp[j], at2[j]);
        }
      }
      volume_combine<ATT>(g, ar1, as1, at1, rq1, vg1);
      volume_combine<ATT>(g, ar2, as2, at2, rq2, vg2);
    }
    // ---- lift of the face amplitudes and expansion, both nodes -------------------------
    float sa1[6], sa2[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) { sa1[c] = 0.f; sa2[c] = 0.f; }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      float2 p0 = make_float2(0.f, 0.f), p1 = p0, p2 = p0, s0 = p0, s1 = p0, s2 = p0;
      const float2* lp = reinterpret_cast<const float2*>(sL) + f * O::NPAIR * Np;
      const float* ax = sAmp + le * O::AE + f * 2 * O::NPAIR;
#pragma unroll
      for (int ip = 0; ip < O::NPAIR; ++ip) {
        const float2 l1 = lp[ip * Np + n1], l2 = lp[ip * Np + n2c];
        const float2 u0 = *reinterpret_cast<const float2*>(ax + 2 * ip);
        const float2 u1 = *reinterpret_cast<const float2*>(ax + O::NFP + 2 * ip);
        const float2 u2 = *reinterpret_cast<const float2*>(ax + 2 * O::NFP + 2 * ip);
        p0 = __ffma2_rn(l1, u0, p0);
        p1 = __ffma2_rn(l1, u1, p1);
        p2 = __ffma2_rn(l1, u2, p2);
        s0 = __ffma2_rn(l2, u0, s0);
        s1 = __ffma2_rn(l2, u1, s1);
        s2 = __ffma2_rn(l2, u2, s2);
      }
      face_expand<ATT>(g, f, p0.x + p0.y, p1.x + p1.y, p2.x + p2.y, rq1, sa1);
      face_expand<ATT>(g, f, s0.x + s0.y, s1.x + s1.y, s2.x + s2.y, rq2, sa2);
    }
    // ---- memory variables, sources, receivers, stage update --------------------------
    auto strain = [&](const float* sig_an, const float* vgrad, float* S) {
      S[0] = sig_an[0] - vgrad[0];
      S[1] = sig_an[1] - vgrad[4];
      S[2] = sig_an[2] - vgrad[8];
      S[3] = sig_an[3] - 0.5f * (vgrad[3] + vgrad[1]);
      S[4] = sig_an[4] - 0.5f * (vgrad[7] + vgrad[5]);
      S[5] = sig_an[5] - 0.5f * (vgrad[6] + vgrad[2]);
    };
    float S[6];
    if (ATT) strain(sa1, vg1, S);
    finish_node<Np, ATT, false, MODE>(a, b, e, base + n1, rq1, S, pf1, sQF + le * Np + n1, O::QF);
    if (has2) {
      if (ATT) strain(sa2, vg2, S);
      finish_node<Np, ATT, false, MODE>(a, b, e, base + n2, rq2, S, pf2, sQF + le * Np + n2, O::QF);
    }
  }
  cp_async_wait_all();
}

}  // namespace nexd_dev
