// NPML stage kernel with the element-local state staged by bulk copies (sm_100a, FP32).
//
// The same stage as stage_kernel<N, ATT, true, MODE> (the reference's element
// loop for PML elements, src/timeloopMod.f90:395-476 with 399-405, and the
// stage update of RungeKuttaSteps, src/rungekuttaMod.f90:27-88), with the
// same thread-per-node mapping and the same operations in the same order, so
// both kernels give identical results.  What changes is how a chunk's
// element-local state reaches the threads.  stage_kernel loads it into
// registers at the start of each chunk (63 NPML values and 45 update values
// per node); those ~100 loads per thread are issued in one burst that the
// memory system accepts only as fast as earlier loads return, and the block
// (one per SM at this size) computes nothing meanwhile.  Here one thread
// moves each array's chunk range -- element-blocked, so one contiguous range
// per array -- with a 1-D bulk copy (cp.async.bulk, completion counted on an
// mbarrier, no multicast) into shared memory while the block computes:
//
//   buffer A   F', G', H', their residuals and the 9 damping profiles of the
//              chunk (read in the NPML phase); refilled with the next
//              chunk's as soon as the NPML phase has read it, so the copy
//              overlaps the volume, lift and update phases
//   buffer B   the LSERK residual of q, the memory variables and their
//              residuals (read in the update phase); refilled at the start
//              of each chunk, so the copy overlaps the face, NPML, volume
//              and lift phases
//
// Each range is widened to 16-byte boundaries (bulk copies move 16-byte
// multiples between 16-byte-aligned addresses); the arrays carry 4 floats of
// slack after their last element so the widened end stays inside them.  The
// waits on the mbarriers are bounded: after ~2^22 polls the kernel sets
// error bit 8 and leaves its chunk loop (every thread sees the same
// mbarrier), and the host reports NEXD_ERR_CUDA.
#pragma once
#include "stage_kernel.cuh"
#include "tc_gemm.cuh"

namespace nexd_dev {

template <int N>
struct BulkOrder {
  using O = Order<N>;
  static constexpr int Np = O::Np, E = O::E;
  static constexpr int w16(int x) { return O::r4(x + 6); }  // a range widened to 16-byte boundaries
  static constexpr int SAUX = w16(E * 27 * Np);             // F', G', H' (and their residuals)
  static constexpr int SPRF = w16(E * 9 * Np);              // damping profiles
  static constexpr int QR = w16(E * Np);                    // one field's row of the TVD step-start q
  static constexpr int SRES = (w16(E * 9 * Np) > 9 * QR) ? w16(E * 9 * Np) : 9 * QR;  // LSERK residual or TVD q
  static constexpr int STH = w16(E * 6 * kNMB * Np);        // memory variables (and their residuals)
  static constexpr int SA = 2 * SAUX + SPRF;
  static constexpr int SB = SRES + 2 * STH;
  // floats before the two mbarriers (8-byte aligned)
  static constexpr int MBAR_OFF = O::smem_floats(true) + SA + SB;
  static constexpr int smem_floats() { return MBAR_OFF + 4; }
};

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> shared of this CTA, completion counted on mbar (no multicast).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tc::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// One array's chunk range [base, base + cnt) floats widened to 16-byte
// boundaries: returns the bytes and starts the copy into dst; the value at
// base + x lands at dst[(base & 3) + x].
__device__ __forceinline__ uint32_t bulk_range(float* dst, const float* arr, long long base, long long cnt,
                                               uint32_t mbar) {
  const long long s0 = base & ~3LL;
  const long long s1 = (base + cnt + 3) & ~3LL;
  const uint32_t bytes = uint32_t((s1 - s0) * 4);
  bulk_load(dst, arr + s0, bytes, mbar);
  return bytes;
}
__device__ __forceinline__ uint32_t bulk_bytes(long long base, long long cnt) {
  return uint32_t((((base + cnt + 3) & ~3LL) - (base & ~3LL)) * 4);
}

// Buffer A of chunk c (one thread): F', G', H' [, residuals], profiles.
template <int N>
__device__ __forceinline__ void issue_state_a(const StageArgs& a, const Chunk& c, float* sAux, float* sAux2,
                                              float* sPrf, bool need2, uint32_t mbar) {
  constexpr int Np = Order<N>::Np;
  const long long ba = (long long)c.b * 27 * a.lda + (long long)c.e0 * 27 * Np, na = (long long)c.ne * 27 * Np;
  const long long bp = (long long)c.e0 * 9 * Np, np_ = (long long)c.ne * 9 * Np;
  uint32_t bytes = bulk_bytes(ba, na) * (need2 ? 2 : 1) + bulk_bytes(bp, np_);
  mbar_expect_tx(mbar, bytes);
  bulk_range(sAux, a.aux, ba, na, mbar);
  if (need2) bulk_range(sAux2, a.aux2, ba, na, mbar);
  bulk_range(sPrf, a.prof, bp, np_, mbar);
}

// Buffer B of chunk c (one thread): residual of q (LSERK) or step-start q
// rows (TVD, field-major: one range per field), memory variables [, residuals].
template <int N, bool ATT, int MODE>
__device__ __forceinline__ void issue_state_b(const StageArgs& a, const Chunk& c, float* sRes, float* sTh,
                                              float* sTh2, bool need2, uint32_t mbar) {
  constexpr int Np = Order<N>::Np, E = Order<N>::E;
  uint32_t bytes = 0;
  const bool resv = (MODE == MODE_LSERK) || a.ca != 0.f;
  const long long br = (long long)c.b * 9 * a.ldq + (long long)c.e0 * 9 * Np, nr = (long long)c.ne * 9 * Np;
  const long long bq = (long long)c.b * 9 * a.ldq + (long long)c.e0 * Np, nq = (long long)c.ne * Np;
  const long long bt = (long long)c.b * 6 * kNMB * a.ldt + (long long)c.e0 * 6 * kNMB * Np,
                  nth = (long long)c.ne * 6 * kNMB * Np;
  if (resv) {
    if (MODE == MODE_LSERK) bytes += bulk_bytes(br, nr);
    else
      for (int f = 0; f < 9; ++f) bytes += bulk_bytes(bq + f * a.ldq, nq);
  }
  if (ATT) bytes += bulk_bytes(bt, nth) * (need2 ? 2 : 1);
  mbar_expect_tx(mbar, bytes);
  if (resv) {
    if (MODE == MODE_LSERK) {
      bulk_range(sRes, a.res, br, nr, mbar);
    } else {
      // TVD: step-start q, field-major; field f of the chunk at sRes[f * QR]
      for (int f = 0; f < 9; ++f) bulk_range(sRes + f * BulkOrder<N>::QR, a.q_n, bq + f * a.ldq, nq, mbar);
    }
  }
  if (ATT) {
    bulk_range(sTh, a.th, bt, nth, mbar);
    if (need2) bulk_range(sTh2, a.th2, bt, nth, mbar);
  }
}

// pml_update with the node's damping profiles, auxiliaries and their
// residuals (TVD: step-start values) read from shared memory at a stride of
// Np floats; the same operations in the same order.
template <int Np, int MODE>
__device__ __forceinline__ void pml_update_strided(const StageArgs& a, int b, int e, int n, bool off, const float* pr,
                                                   const float* av, const float* a2, float* F, float* G, float* H) {
  if (off) return;  // pmlcheck(:) = .false.: ordinary element (src/timeloopMod.f90:537)
  const float ddx = pr[0], ddy = pr[Np], ddz = pr[2 * Np];
  const float alx = pr[3 * Np], aly = pr[4 * Np], alz = pr[5 * Np];
  const float ikx = 1.f / pr[6 * Np], iky = 1.f / pr[7 * Np], ikz = 1.f / pr[8 * Np];
  float* aux = a.aux + eblock<27, Np>(a.lda, b, e, n);
  float* aux2 = a.aux2 + eblock<27, Np>(a.lda, b, e, n);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const float fp = av[i * Np], gp = av[(9 + i) * Np], hp = av[(18 + i) * Np];
    const float rf = -alx * fp - ddx * ikx * (fp + F[i]);
    const float rg = -aly * gp - ddy * iky * (gp + G[i]);
    const float rh = -alz * hp - ddz * ikz * (hp + H[i]);
    const float phi = (fp + F[i]) * ikx, psi = (gp + G[i]) * iky, ome = (hp + H[i]) * ikz;
    float nf, ng_, nh;
    if (MODE == MODE_LSERK) {
      const float r1 = a.ca * a2[i * Np] + a.dt * rf;
      const float r2 = a.ca * a2[(9 + i) * Np] + a.dt * rg;
      const float r3 = a.ca * a2[(18 + i) * Np] + a.dt * rh;
      __stcs(aux2 + i * Np, r1);
      __stcs(aux2 + (9 + i) * Np, r2);
      __stcs(aux2 + (18 + i) * Np, r3);
      nf = fp + a.cb * r1;
      ng_ = gp + a.cb * r2;
      nh = hp + a.cb * r3;
    } else {
      float n1, n2, n3;
      if (a.stage_first) {
        __stcs(aux2 + i * Np, fp);
        __stcs(aux2 + (9 + i) * Np, gp);
        __stcs(aux2 + (18 + i) * Np, hp);
        n1 = fp; n2 = gp; n3 = hp;
      } else {
        n1 = a2[i * Np]; n2 = a2[(9 + i) * Np]; n3 = a2[(18 + i) * Np];
      }
      nf = a.ca * n1 + a.cb * (fp + a.dt * rf);
      ng_ = a.ca * n2 + a.cb * (gp + a.dt * rg);
      nh = a.ca * n3 + a.cb * (hp + a.dt * rh);
    }
    __stcs(aux + i * Np, nf);
    __stcs(aux + (9 + i) * Np, ng_);
    __stcs(aux + (18 + i) * Np, nh);
    F[i] = phi;
    G[i] = psi;
    H[i] = ome;
  }
}

// finish_node with the node's update-phase state read from shared memory:
// rs[c * rstride] the residual of q (TVD: step-start q), th / th2 the memory
// variables and their residuals (TVD: step-start values) at a stride of Np.
template <int Np, bool ATT, int MODE>
__device__ __forceinline__ void finish_node_strided(const StageArgs& a, int b, int e, long long node, float* rq,
                                                    const float* S, const float* rs, int rstride, const float* ths,
                                                    const float* th2s, const float* qown, int qstride, bool need2) {
  const int n = int(node - (long long)e * Np);
  if (ATT) {
    float* th = a.th + eblock<6 * kNMB, Np>(a.ldt, b, e, n);
    float* th2 = a.th2 + eblock<6 * kNMB, Np>(a.ldt, b, e, n);
    const float* ae = a.ael + (long long)e * 3 * kNMB;
#pragma unroll
    for (int l = 0; l < kNMB; ++l) {
      const float wl = a.wlv[l];
      float t[6], t2[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        t[j] = ths[(6 * l + j) * Np];
        t2[j] = need2 ? th2s[(6 * l + j) * Np] : 0.f;
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
          __stcs(th2 + o, rr);
          nt_ = t[j] + a.cb * rr;
        } else {
          float tn;
          if (a.stage_first) { __stcs(th2 + o, t[j]); tn = t[j]; } else { tn = t2[j]; }
          nt_ = a.ca * tn + a.cb * (t[j] + a.dt * r);
        }
        __stcs(th + o, nt_);
      }
    }
  }
  for (int s = a.src_head[e]; s >= 0; s = a.src_next[s]) {
    if (a.src_batch[s] != b) continue;
    const int sidx = a.nspt == 1 ? 0 : min(a.stage, a.nspt - 1);
    const float amp = a.stf[((long long)s * a.nt + (*a.it_dev - 1)) * a.nspt + sidx];
    const float* sp = a.src_pat + (long long)s * 9 * Np + n;
#pragma unroll
    for (int c = 0; c < 9; ++c) rq[c] = fmaf(sp[c * Np], amp, rq[c]);
  }
  if (a.last_stage) {
    const int slot = a.rec_slot[e];
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
      const float r = a.ca * rs[c * rstride] + a.dt * rq[c];
      __stcs(rsg + c * Np, r);
      __stcs(qo + c * a.ldq, qown[c * qstride] + a.cb * r);
    }
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const float base = (a.ca != 0.f) ? a.ca * rs[c * rstride] : 0.f;
      __stcs(qo + c * a.ldq, base + a.cb * (qown[c * qstride] + a.dt * rq[c]));
    }
  }
}

template <int N, bool ATT, int MODE>
__global__ void __launch_bounds__(256, 1) stage_npml_bulk_kernel(const StageArgs a) {
  using O = Order<N>;
  using B = BulkOrder<N>;
  constexpr int Np = O::Np, NpF = O::NpF, NF = O::NF, E = O::E, CS = O::CS;
  extern __shared__ __align__(16) float smem[];
  float* sD = smem;
  float* sL = sD + O::SD;
  float* sBuf = sL + O::SL;
  float* sCF = sBuf + 2 * O::BUF;
  float* sAmp = sCF + O::SCF;
  unsigned char* sPat = reinterpret_cast<unsigned char*>(sAmp + O::SAMP);
  float* sAux = sAmp + O::SAMP + O::SPAT;
  float* sAux2 = sAux + B::SAUX;
  float* sPrf = sAux2 + B::SAUX;
  float* sRes = sPrf + B::SPRF;
  float* sTh = sRes + B::SRES;
  float* sTh2 = sTh + B::STH;
  uint64_t* mbars = reinterpret_cast<uint64_t*>(smem + B::MBAR_OFF);
  const uint32_t mbarA = tc::smem_u32(mbars), mbarB = tc::smem_u32(mbars + 1);

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
  const bool need2 = (MODE == MODE_LSERK) || !a.stage_first;
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
    if (tid == 0) {
      tc::mbar_init(mbarA, 1);
      tc::mbar_init(mbarB, 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
      issue_state_a<N>(a, c0, sAux, sAux2, sPrf, need2, mbarA);
      issue_state_b<N, ATT, MODE>(a, c0, sRes, sTh, sTh2, need2, mbarB);
    }
    issue_chunk<O>(a, c0, ids0, sBuf, wn < nwork ? &c1 : nullptr, sPat);
  }

  uint32_t phase = 0;  // parity of both mbarriers' current phase (each completes once per chunk)
  for (int p = 0; w < nwork; w += gridDim.x, p ^= 1, phase ^= 1) {
    const Chunk ch = chunk_of<E>(a, w, nchunk);
    const int b = ch.b, e0 = ch.e0, ne = ch.ne;
    float* buf = sBuf + p * O::BUF;
    const float* sGeo = buf;
    const float* sTr = buf + O::SGEO + O::SQF;
    const float* sQF = buf + O::SGEO + int(((long long)e0 * Np) & 3);
    const int* sIds = reinterpret_cast<const int*>(sTr + O::STR);
    cp_async_wait_all();
    __syncthreads();  // (1) this chunk's records, wavefield and traces are in `buf`; buffer B is free
    const int wn = w + gridDim.x;
    Chunk cn;
    if (wn < nwork) cn = chunk_of<E>(a, wn, nchunk);
    if (tid == 0 && w != (int)blockIdx.x) {
      tc::fence_async_smem();
      issue_state_b<N, ATT, MODE>(a, ch, sRes, sTh, sTh2, need2, mbarB);
    }
    const bool active = le < ne;
    const long long node = (long long)(e0 + (active ? le : 0)) * Np + n;
    if (wn < nwork) {
      const int wnn = wn + gridDim.x;
      Chunk cnn;
      if (wnn < nwork) cnn = chunk_of<E>(a, wnn, nchunk);
      issue_chunk<O>(a, cn, sIds, sBuf + (p ^ 1) * O::BUF, wnn < nwork ? &cnn : nullptr, sPat);
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
    // ---- NPML: auxiliary update and contravariant modified fluxes ------------------
    const bool okA = tc::mbar_wait(mbarA, phase);
    if (active) {
      const float* g = sGeo + le * O::GSTR;
      float qv[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) qv[c] = sQF[c * O::QF + le * Np + n];
      float F[9], G[9], H[9];
      elastic_fluxes(g, qv, F, G, H);
      const int so = int(((long long)b * 27 * a.lda + (long long)e0 * 27 * Np) & 3) + le * 27 * Np + n;
      const float* ps = sPrf + int(((long long)e0 * 9 * Np) & 3) + le * 9 * Np + n;
      pml_update_strided<Np, MODE>(a, b, e0 + le, n, a.pml_off[b] != 0, ps, sAux + so, sAux2 + so, F, G, H);
      float2* cf = reinterpret_cast<float2*>(sCF + le * O::CFE + n * CS);
      float r[10], sv[10], t[10];
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        r[i] = g[G_RX] * F[i] + g[G_RY] * G[i] + g[G_RZ] * H[i];
        sv[i] = g[G_SX] * F[i] + g[G_SY] * G[i] + g[G_SZ] * H[i];
        t[i] = g[G_TX] * F[i] + g[G_TY] * G[i] + g[G_TZ] * H[i];
      }
      r[9] = ATT ? qv[6] : 0.f;
      sv[9] = ATT ? qv[7] : 0.f;
      t[9] = ATT ? qv[8] : 0.f;
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        cf[j] = make_float2(r[2 * j], r[2 * j + 1]);
        cf[5 + j] = make_float2(sv[2 * j], sv[2 * j + 1]);
        cf[10 + j] = make_float2(t[2 * j], t[2 * j + 1]);
      }
    }
    if (__syncthreads_or(!okA)) {  // (2) amplitudes and rows are in shared memory; buffer A is consumed
      if (tid == 0) atomicOr(a.flag, 8);
      break;
    }
    if (tid == 0 && wn < nwork) {
      tc::fence_async_smem();
      issue_state_a<N>(a, cn, sAux, sAux2, sPrf, need2, mbarA);
    }
    if (!active) {
      // idle threads of a partial chunk still take part in the update-phase wait below
      if (!tc::mbar_wait(mbarB, phase)) atomicOr(a.flag, 8);
      continue;
    }

    const int e = e0 + le;
    const float* g = sGeo + le * O::GSTR;
    float rq[9];
    float vgrad[9];
    (void)vgrad;
    {
#pragma unroll
      for (int c = 0; c < 9; ++c) rq[c] = 0.f;
      float2 acc[4];
      float acc8 = 0.f;
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[j] = make_float2(0.f, 0.f);
      float2 v01r = make_float2(0.f, 0.f), v01s = v01r, v01t = v01r;
      float v2r = 0.f, v2s = 0.f, v2t = 0.f;
      const float* cfe = sCF + le * O::CFE;
#pragma unroll 5
      for (int k = 0; k < Np; ++k) {
        const float2 drs = reinterpret_cast<const float2*>(sD)[k * Np + n];
        const float4 d = make_float4(drs.x, drs.y, sD[2 * Np * Np + k * Np + n], 0.f);
        const float2 d0 = make_float2(d.x, d.x), d1 = make_float2(d.y, d.y), d2 = make_float2(d.z, d.z);
        const float2* cf = reinterpret_cast<const float2*>(cfe + k * CS);
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[j] = __ffma2_rn(d0, cf[j], __ffma2_rn(d1, cf[5 + j], __ffma2_rn(d2, cf[10 + j], acc[j])));
        const float2 pr8 = cf[4], ps8 = cf[9], pt8 = cf[14];
        acc8 = fmaf(d.x, pr8.x, fmaf(d.y, ps8.x, fmaf(d.z, pt8.x, acc8)));
        if (ATT) {
          const float2 v01 = make_float2(pr8.y, ps8.y);
          const float v2 = pt8.y;
          v01r = __ffma2_rn(d0, v01, v01r);
          v01s = __ffma2_rn(d1, v01, v01s);
          v01t = __ffma2_rn(d2, v01, v01t);
          v2r = fmaf(d.x, v2, v2r);
          v2s = fmaf(d.y, v2, v2s);
          v2t = fmaf(d.z, v2, v2t);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) { rq[2 * j] = acc[j].x; rq[2 * j + 1] = acc[j].y; }
      rq[8] = acc8;
      const float vr[3] = {v01r.x, v01r.y, v2r}, vs3[3] = {v01s.x, v01s.y, v2s}, vt3[3] = {v01t.x, v01t.y, v2t};
      if (ATT) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          vgrad[c * 3 + 0] = g[G_RX] * vr[c] + g[G_SX] * vs3[c] + g[G_TX] * vt3[c];
          vgrad[c * 3 + 1] = g[G_RY] * vr[c] + g[G_SY] * vs3[c] + g[G_TY] * vt3[c];
          vgrad[c * 3 + 2] = g[G_RZ] * vr[c] + g[G_SZ] * vs3[c] + g[G_TZ] * vt3[c];
        }
      }
    }
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
    float S[6];
    if (ATT) {
      S[0] = sig_an[0] - vgrad[0];
      S[1] = sig_an[1] - vgrad[4];
      S[2] = sig_an[2] - vgrad[8];
      S[3] = sig_an[3] - 0.5f * (vgrad[3] + vgrad[1]);
      S[4] = sig_an[4] - 0.5f * (vgrad[7] + vgrad[5]);
      S[5] = sig_an[5] - 0.5f * (vgrad[6] + vgrad[2]);
    }
    // ---- memory variables, sources, receivers, stage update (state from buffer B)
    if (!tc::mbar_wait(mbarB, phase)) {
      atomicOr(a.flag, 8);
      continue;  // the next top-of-chunk barrier is reached by every thread
    }
    {
      const float* rs;
      int rstride;
      if (MODE == MODE_LSERK) {
        rs = sRes + int(((long long)b * 9 * a.ldq + (long long)e0 * 9 * Np) & 3) + le * 9 * Np + n;
        rstride = Np;
      } else {
        rs = sRes + int(((long long)b * 9 * a.ldq + (long long)e0 * Np) & 3) + le * Np + n;
        rstride = B::QR;
      }
      const int to = int(((long long)b * 6 * kNMB * a.ldt + (long long)e0 * 6 * kNMB * Np) & 3) + le * 6 * kNMB * Np + n;
      finish_node_strided<Np, ATT, MODE>(a, b, e, node, rq, S, rs, rstride, sTh + to, sTh2 + to,
                                         sQF + le * Np + n, O::QF, need2);
    }
  }
  cp_async_wait_all();
}

}  // namespace nexd_dev
