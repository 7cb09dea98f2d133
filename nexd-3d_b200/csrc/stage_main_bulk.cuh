// Stage kernel for the elements outside the NPML with the memory variables
// moved by bulk copies (sm_100a, FP32, anelastic).
//
// The same stage as stage_kernel<N, true, false, MODE> (the reference's
// element loop, src/timeloopMod.f90:395-476, its Zener memory variables,
// 426-461, and the stage update of RungeKuttaSteps,
// src/rungekuttaMod.f90:27-88) with the same thread-per-node mapping and the
// same operations in the same order, so both kernels give identical results.
// stage_kernel prefetches 45 values per node into registers at the start of
// each chunk and stores 45 from registers in its update phase; here the 36
// memory variables and their residuals of a chunk (element-blocked, each
// element's block 16-byte aligned) move between global and shared memory as
// two 1-D bulk copies each way, issued by one thread while the block
// computes, and the threads update them in place (the layout of buffer B of
// stage_npml_bulk_kernel).  The load of a chunk's memory variables is issued
// after its face phase and completes on an mbarrier before its update phase;
// the store is issued at the start of the next chunk.
//
// To keep two blocks per SM (about 106 KB of shared memory each at N = 4),
// the own wavefield and the neighbour traces are single-buffered: the next
// chunk's copies start after this chunk's face phase, the last reader of
// both, and the update phase takes the own values from the interleaved copy
// the volume loop reads.  The LSERK residual of q (9 values per node) stays a
// register prefetch.
#pragma once
#include "stage_npml_bulk.cuh"

namespace nexd_dev {

template <int N, int NPT = 1>
struct MainBulkOrder {
  using O = Order<N, NPT>;
  static constexpr int Np = O::Np, E = O::E;
  static constexpr int FT = EBlock<6 * kNMB, Np>::FS;  // floats per element: memory variables
  static constexpr int STH = E * FT;
  // layout: D | LIFT | records x2 | connectivity x2 | own wavefield | traces |
  //         interleaved own wavefield | amplitudes | face patterns | theta | theta residual | mbarrier
  static constexpr int OFF_GEO = O::SD + O::SL;
  static constexpr int OFF_IDS = OFF_GEO + 2 * O::SGEO;
  static constexpr int OFF_Q = OFF_IDS + 2 * O::SIDS;
  static constexpr int OFF_TR = OFF_Q + O::SQF;
  static constexpr int OFF_QI = OFF_TR + O::STR;
  static constexpr int OFF_AMP = OFF_QI + O::SQI;
  static constexpr int OFF_PAT = OFF_AMP + O::SAMP;
  static constexpr int OFF_TH = OFF_PAT + O::SPAT;
  static constexpr int OFF_TH2 = OFF_TH + STH;
  static constexpr int MBAR_OFF = OFF_TH2 + STH;
  static constexpr int smem_floats() { return MBAR_OFF + 4; }
};

template <int N, int NPT = 1>
__device__ __forceinline__ void load_theta(const StageArgs& a, const Chunk& c, float* sTh, float* sTh2,
                                           uint32_t mbar) {
  using B = MainBulkOrder<N, NPT>;
  const long long bt = eblock_chunk<6 * kNMB, B::Np>(a.ldt, c);
  const uint32_t nt = uint32_t(c.ne) * B::FT * 4;
  mbar_expect_tx(mbar, 2 * nt);
  bulk_load(sTh, a.th + bt, nt, mbar);
  bulk_load(sTh2, a.th2 + bt, nt, mbar);
}
template <int N, int NPT = 1>
__device__ __forceinline__ void store_theta(const StageArgs& a, const Chunk& c, const float* sTh, const float* sTh2) {
  using B = MainBulkOrder<N, NPT>;
  const long long bt = eblock_chunk<6 * kNMB, B::Np>(a.ldt, c);
  const uint32_t nt = uint32_t(c.ne) * B::FT * 4;
  bulk_store(a.th + bt, sTh, nt);
  bulk_store(a.th2 + bt, sTh2, nt);
  bulk_commit();
}

// Update phase of one node of an anelastic element outside the NPML with its
// memory variables in shared memory (ths / th2s at a stride of Np floats,
// updated in place): Zener terms (src/timeloopMod.f90:426-461), point
// sources, the receiver acceleration and the stage update of q; res holds
// the node's residual of q (TVD: step-start q) and qown its interleaved own
// values.  The operations and their order are those of finish_node.
template <int Np, int MODE>
__device__ __forceinline__ void finish_theta_smem(const StageArgs& a, int b, int e, long long node, int n, float* rq,
                                                  const float* S, const float* res, float* ths, float* th2s,
                                                  const float* qown, const ElemScalars<true>& es) {
  const float* ae = es.ae;
#pragma unroll
  for (int l = 0; l < kNMB; ++l) {
    const float wl = a.wlv[l];
    float t[6], t2[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      t[j] = ths[(6 * l + j) * Np];
      t2[j] = th2s[(6 * l + j) * Np];
    }
    const float c1 = ae[3 * l], c2 = ae[3 * l + 1], c3 = ae[3 * l + 2];
    rq[0] += c3 * t[0] + c1 * (t[1] + t[2]);
    rq[1] += c3 * t[1] + c1 * (t[2] + t[0]);
    rq[2] += c3 * t[2] + c1 * (t[0] + t[1]);
    rq[3] += c2 * t[3];
    rq[4] += c2 * t[4];
    rq[5] += c2 * t[5];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const float r = wl * (S[j] - t[j]);
      const int o = (l * 6 + j) * Np;
      float nt_;
      if (MODE == MODE_LSERK) {
        const float rr = a.ca * t2[j] + a.dt * r;
        th2s[o] = rr;
        nt_ = t[j] + a.cb * rr;
      } else {
        float tn;
        if (a.stage_first) { th2s[o] = t[j]; tn = t[j]; } else { tn = t2[j]; }
        nt_ = a.ca * tn + a.cb * (t[j] + a.dt * r);
      }
      ths[o] = nt_;
    }
  }
  for (int s = es.src; s >= 0; s = a.src_next[s]) {
    if (a.src_batch[s] != b) continue;
    const int sidx = a.nspt == 1 ? 0 : min(a.stage, a.nspt - 1);
    const float amp = a.stf[((long long)s * a.nt + (*a.it_dev - 1)) * a.nspt + sidx];
    const float* sp = a.src_pat + (long long)s * 9 * Np + n;
#pragma unroll
    for (int c = 0; c < 9; ++c) rq[c] = fmaf(sp[c * Np], amp, rq[c]);
  }
  if (a.last_stage) {
    const int slot = es.slot;
    if (slot >= 0) {
      float* ab = a.abuf + ((long long)b * a.nslot + slot) * 3 * Np + n;
      ab[0] = rq[6];
      ab[Np] = rq[7];
      ab[2 * Np] = rq[8];
    }
  }
  float* qo = a.q_out + (long long)b * 9 * a.ldq + node;
  if (MODE == MODE_LSERK) {
    float* rsg = a.res + eblock<9, Np>(a.ldq, b, e, n);
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const float r = a.ca * res[c] + a.dt * rq[c];
      __stcs(rsg + c * Np, r);
      __stcs(qo + c * a.ldq, qown[c] + a.cb * r);
    }
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const float base = (a.ca != 0.f) ? a.ca * res[c] : 0.f;
      __stcs(qo + c * a.ldq, base + a.cb * (qown[c] + a.dt * rq[c]));
    }
  }
}

template <int N, int MODE>
__global__ void __launch_bounds__(256, 2) stage_main_bulk_kernel(const StageArgs a) {
  using O = Order<N>;
  using B = MainBulkOrder<N>;
  constexpr int Np = O::Np, NpF = O::NpF, NF = O::NF, E = O::E, QS = O::QS;
  extern __shared__ __align__(16) float smem[];
  float* sD = smem;
  float* sL = sD + O::SD;
  float* sQF0 = smem + B::OFF_Q;
  float* sTr = smem + B::OFF_TR;
  float* sQI = smem + B::OFF_QI;
  float* sAmp = smem + B::OFF_AMP;
  unsigned char* sPat = reinterpret_cast<unsigned char*>(smem + B::OFF_PAT);
  float* sTh = smem + B::OFF_TH;
  float* sTh2 = smem + B::OFF_TH2;
  const uint32_t mbarB = tc::smem_u32(smem + B::MBAR_OFF);

  const int tid = threadIdx.x;
  for (int i = tid; i < Np * Np; i += blockDim.x) {
    reinterpret_cast<float2*>(sD)[i] = make_float2(a.D[i], a.D[Np * Np + i]);
    sD[2 * Np * Np + i] = a.D[2 * Np * Np + i];
  }
  for (int i = tid; i < O::SL; i += blockDim.x) sL[i] = a.L[i];
  if (NpF & 1)
    for (int i = tid; i < E * 3 * 4; i += blockDim.x)
      sAmp[(i >> 2) / 3 * O::AE + (i >> 2) % 3 * O::NFP + (i & 3) * 2 * O::NPAIR + NpF] = 0.f;
  for (int i = tid; i < a.npat * NpF; i += blockDim.x) sPat[i] = a.patterns[i];

  const int nel = a.e_end - a.e_begin;
  const int nchunk = (nel + E - 1) / E;
  const int nwork = nchunk * a.nbatch;
  int le, n;
  if constexpr (O::WARP_ALIGNED) {
    if (tid < E * 32) {
      le = tid >> 5;
      n = tid & 31;
    } else {
      const int r = tid - E * 32;
      le = r / (Np - 32);
      n = 32 + r - le * (Np - 32);
    }
  } else {
    le = tid / Np;
    n = tid - le * Np;
  }
  int w = blockIdx.x;
  if (w >= nwork) return;
  auto geo_buf = [&](int p) { return smem + B::OFF_GEO + p * O::SGEO; };
  auto ids_buf = [&](int p) { return reinterpret_cast<int*>(smem + B::OFF_IDS + p * O::SIDS); };

  {
    const Chunk c0 = chunk_of<E>(a, w, nchunk);
    const int wn = w + gridDim.x;
    Chunk c1;
    if (wn < nwork) c1 = chunk_of<E>(a, wn, nchunk);
    int* ids0 = ids_buf(1);  // scratch: the connectivity of the first chunk
    for (int i = tid; i < c0.ne * 8; i += blockDim.x) {
      const int ee = i >> 3, k = i & 7;
      ids0[ee * 12 + k] = k < 4 ? reinterpret_cast<const int*>(a.nbr)[4 * (c0.e0 + ee) + k]
                                : reinterpret_cast<const int*>(a.fcode)[4 * (c0.e0 + ee) + k - 4];
    }
    if (tid == 0) {
      tc::mbar_init(mbarB, 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) load_theta<N>(a, c0, sTh, sTh2, mbarB);
    issue_main<O>(a, c0, geo_buf(0), sQF0, ids_buf(0), wn < nwork ? &c1 : nullptr);
    issue_traces<O>(a, c0, ids0, sTr, sPat);
    cp_async_commit();
  }

  bool ok = true;
  uint32_t phase = 0;
  Chunk prev;
  for (int p = 0; w < nwork; w += gridDim.x, p ^= 1, phase ^= 1) {
    const Chunk ch = chunk_of<E>(a, w, nchunk);
    const int b = ch.b, e0 = ch.e0, ne = ch.ne;
    const bool first = w == (int)blockIdx.x;
    const float* sGeo = geo_buf(p);
    const int* sIds = ids_buf(p);  // +0..7: connectivity of the next chunk; +8..11: this chunk's face codes
    const float* sQF = sQF0 + int(((long long)e0 * Np) & 3);
    cp_async_wait_all();
    __syncthreads();  // (1) this chunk's records, wavefield and traces are in place; the previous theta is final
    if (tid == 0 && !first) store_theta<N>(a, prev, sTh, sTh2);
    const bool active = le < ne;
    const long long node = (long long)(e0 + (active ? le : 0)) * Np + n;
    ElemScalars<true> es;
    es.load(a, b, e0 + (active ? le : 0));
    // residual of q (LSERK) or step-start q (TVD) of this node
    float res[9];
    if (active) {
      if (MODE == MODE_LSERK) {
        const float* rs = a.res + eblock<9, Np>(a.ldq, b, e0 + le, n);
#pragma unroll
        for (int c = 0; c < 9; ++c) res[c] = __ldcs(rs + c * Np);
      } else if (a.ca != 0.f) {
        const float* qn = a.q_n + (long long)b * 9 * a.ldq + node;
#pragma unroll
        for (int c = 0; c < 9; ++c) res[c] = __ldcs(qn + c * a.ldq);
      } else {
#pragma unroll
        for (int c = 0; c < 9; ++c) res[c] = 0.f;
      }
      // interleaved own wavefield for the volume loop and the update phase
      float* dst = sQI + le * O::QE + n * QS;
      const float* src = sQF + le * Np + n;
      constexpr int FS = O::QF;
      *reinterpret_cast<float4*>(dst) = make_float4(src[0], src[FS], src[2 * FS], src[3 * FS]);
      *reinterpret_cast<float4*>(dst + 4) = make_float4(src[4 * FS], src[5 * FS], src[6 * FS], src[7 * FS]);
      dst[8] = src[8 * FS];
    }
    // ---- face amplitudes ---------------------------------------------------------
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
    // the previous chunk's theta was read by its store: refill with this chunk's
    if (tid == 0 && !first) {
      bulk_wait_read();
      load_theta<N>(a, ch, sTh, sTh2, mbarB);
    }
    __syncthreads();  // (2) amplitudes and interleaved wavefield ready; own wavefield and traces free
    // ---- the next chunk's records, wavefield, connectivity and traces ---------------
    {
      const int wn = w + gridDim.x;
      if (wn < nwork) {
        const Chunk cn = chunk_of<E>(a, wn, nchunk);
        const int wnn = wn + gridDim.x;
        Chunk cnn;
        if (wnn < nwork) cnn = chunk_of<E>(a, wnn, nchunk);
        issue_main<O>(a, cn, geo_buf(p ^ 1), sQF0, ids_buf(p ^ 1), wnn < nwork ? &cnn : nullptr);
        issue_traces<O>(a, cn, sIds, sTr, sPat);
        cp_async_commit();
      }
    }
    if (!active) {
      prev = ch;
      continue;  // idle threads of a partial chunk (thread 0 is never idle)
    }

    const int e = e0 + le;
    const float* g = sGeo + le * O::GSTR;
    float rq[9];
    float vgrad[9];
    {
      float2 ar[4], as_[4], at[4];
      float r8 = 0.f, s8 = 0.f, t8 = 0.f;
#pragma unroll
      for (int j = 0; j < 4; ++j) { ar[j] = make_float2(0.f, 0.f); as_[j] = ar[j]; at[j] = ar[j]; }
      const float* qe = sQI + le * O::QE;
#pragma unroll
      for (int k = 0; k < Np; ++k) {
        const float2 drs = reinterpret_cast<const float2*>(sD)[k * Np + n];
        const float dx = drs.x, dy = drs.y, dz = sD[2 * Np * Np + k * Np + n];
        const float2 d0 = make_float2(dx, dx), d1 = make_float2(dy, dy), d2 = make_float2(dz, dz);
        const float4 qa = ld4(qe + k * QS), qb = ld4(qe + k * QS + 4);
        const float q8 = qe[k * QS + 8];
        const float2 qp[4] = {make_float2(qa.x, qa.y), make_float2(qa.z, qa.w), make_float2(qb.x, qb.y),
                              make_float2(qb.z, qb.w)};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          ar[j] = __ffma2_rn(d0, qp[j], ar[j]);
          as_[j] = __ffma2_rn(d1, qp[j], as_[j]);
          at[j] = __ffma2_rn(d2, qp[j], at[j]);
        }
        r8 = fmaf(dx, q8, r8);
        s8 = fmaf(dy, q8, s8);
        t8 = fmaf(dz, q8, t8);
      }
      float dr[9], ds[9], dtt[9];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        dr[2 * j] = ar[j].x; dr[2 * j + 1] = ar[j].y;
        ds[2 * j] = as_[j].x; ds[2 * j + 1] = as_[j].y;
        dtt[2 * j] = at[j].x; dtt[2 * j + 1] = at[j].y;
      }
      dr[8] = r8; ds[8] = s8; dtt[8] = t8;
      const float rx = g[G_RX], ry = g[G_RY], rz = g[G_RZ], sx = g[G_SX], sy = g[G_SY], sz = g[G_SZ],
                  tx = g[G_TX], ty = g[G_TY], tz = g[G_TZ];
#define DX(c) (rx * dr[c] + sx * ds[c] + tx * dtt[c])
#define DY(c) (ry * dr[c] + sy * ds[c] + ty * dtt[c])
#define DZ(c) (rz * dr[c] + sz * ds[c] + tz * dtt[c])
      const float e1 = g[G_E1], e2 = g[G_E2], e3 = g[G_E3], e4 = g[G_E4];
      const float dxv = DX(6), dyv = DY(6), dzv = DZ(6);
      const float dxw = DX(7), dyw = DY(7), dzw = DZ(7);
      const float dxu = DX(8), dyu = DY(8), dzu = DZ(8);
      rq[0] = e1 * dxv + e2 * dyw + e2 * dzu;
      rq[1] = e2 * dxv + e1 * dyw + e2 * dzu;
      rq[2] = e2 * dxv + e2 * dyw + e1 * dzu;
      rq[3] = e3 * dxw + e3 * dyv;
      rq[4] = e3 * dyu + e3 * dzw;
      rq[5] = e3 * dxu + e3 * dzv;
      rq[6] = e4 * (DX(0) + DY(3) + DZ(5));
      rq[7] = e4 * (DX(3) + DY(1) + DZ(4));
      rq[8] = e4 * (DX(5) + DY(4) + DZ(2));
      vgrad[0] = dxv; vgrad[1] = dyv; vgrad[2] = dzv;
      vgrad[3] = dxw; vgrad[4] = dyw; vgrad[5] = dzw;
      vgrad[6] = dxu; vgrad[7] = dyu; vgrad[8] = dzu;
#undef DX
#undef DY
#undef DZ
    }
    float sig_an[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) sig_an[c] = 0.f;
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
      face_expand<true>(g, f, c0.x + c0.y, c1.x + c1.y, c2.x + c2.y, rq, sig_an);
    }
    float S[6];
    S[0] = sig_an[0] - vgrad[0];
    S[1] = sig_an[1] - vgrad[4];
    S[2] = sig_an[2] - vgrad[8];
    S[3] = sig_an[3] - 0.5f * (vgrad[3] + vgrad[1]);
    S[4] = sig_an[4] - 0.5f * (vgrad[7] + vgrad[5]);
    S[5] = sig_an[5] - 0.5f * (vgrad[6] + vgrad[2]);
    // ---- memory variables (in shared memory), sources, receivers, stage update ------
    if (!tc::mbar_wait(mbarB, phase)) {
      atomicOr(a.flag, 8);
      ok = false;
    } else {
      finish_theta_smem<Np, MODE>(a, b, e, node, n, rq, S, res, sTh + le * B::FT + n, sTh2 + le * B::FT + n,
                                  sQI + le * O::QE + n * QS, es);
    }
    tc::fence_async_smem();  // this thread's writes to theta are seen by the bulk store
    prev = ch;
  }
  const bool all_ok = __syncthreads_and(ok);
  if (tid == 0) {
    if (all_ok) {
      store_theta<N>(a, prev, sTh, sTh2);
    } else {
      // a load did not complete in time: wait once more, bounded, for it
      tc::mbar_wait(mbarB, phase ^ 1, 1u << 24);
    }
    bulk_wait_all();
  }
  cp_async_wait_all();
}

}  // namespace nexd_dev
