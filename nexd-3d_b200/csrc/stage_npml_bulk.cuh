// NPML stage kernel with the element-local state moved by bulk copies (sm_100a, FP32).
//
// The same stage as stage_kernel<N, ATT, true, MODE> (the reference's element
// loop for PML elements, src/timeloopMod.f90:395-476 with 399-405, and the
// stage update of RungeKuttaSteps, src/rungekuttaMod.f90:27-88), with the
// same thread-per-node mapping and the same operations in the same order, so
// both kernels give identical results.  What changes is how a chunk's
// element-local state reaches the threads and goes back.  stage_kernel loads
// it into registers at the start of each chunk (63 NPML values and 45 update
// values per node) and stores the new values from registers (108 per node);
// the memory system takes those ~200 instructions per thread in bursts only
// as fast as earlier ones complete, and the block (one per SM at this size)
// computes nothing meanwhile.  Here each array's chunk range -- element-
// blocked, each element's block 16-byte aligned (eblock), so one contiguous
// range per array -- moves between global and shared memory as one 1-D bulk
// copy (cp.async.bulk; loads complete on an mbarrier, stores in bulk groups;
// no multicast), and the threads update the state in place in shared memory:
//
//   buffer A   F', G', H', their residuals (TVD: step-start values) and the
//              9 damping profiles of the chunk, used in the NPML phase
//   buffer B   the LSERK residual of q (TVD: the step-start q, read only),
//              the memory variables and their residuals, used in the update
//              phase
//
// The block is warp-specialised: 8 compute warps and one producer warp (see
// kCompute below).  Per chunk the producer stores the previous chunk's B and
// loads this chunk's once the store has read it, and starts the next chunk's
// records, wavefield and connectivity (cp.async); after the compute warps'
// NPML phase (second barrier) it stores A, loads the next chunk's A and
// gathers the next chunk's neighbour traces.  The compute warps only compute.
//
// The profiles and the TVD step-start q keep their unpadded layouts: their
// ranges are widened to 16-byte boundaries for the loads (the arrays carry 4
// floats of slack after the last element) and never stored.  The new q is
// written with ordinary coalesced stores (field-major).  Waits on the
// mbarriers are bounded: after ~2^22 polls the kernel sets error bit 8 and
// the host reports NEXD_ERR_CUDA.
#pragma once
#include "stage_kernel.cuh"
#include "tc_gemm.cuh"

namespace nexd_dev {

template <int N>
struct BulkOrder {
  using O = Order<N>;
  static constexpr int Np = O::Np, E = O::E;
  static constexpr int w16(int x) { return O::r4(x + 6); }  // a range widened to 16-byte boundaries
  static constexpr int FA = EBlock<27, Np>::FS;             // floats per element: F', G', H'
  static constexpr int FR = EBlock<9, Np>::FS;              // residual of q
  static constexpr int FT = EBlock<6 * kNMB, Np>::FS;       // memory variables
  static constexpr int SAUX = E * FA;                       // F', G', H' (and their residuals)
  static constexpr int SPRF = w16(E * 9 * Np);              // damping profiles
  static constexpr int QR = w16(E * Np);                    // one field's row of the TVD step-start q
  static constexpr int SRES = (E * FR > 9 * QR) ? E * FR : 9 * QR;  // LSERK residual or TVD step-start q
  static constexpr int STH = E * FT;                        // memory variables (and their residuals)
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
// 1-D bulk copy shared -> global, tracked by bulk groups.
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(tc::smem_u32(src)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until the shared memory of every committed bulk store has been read.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Waits until every committed bulk store has completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// One unpadded array's chunk range [base, base + cnt) floats widened to
// 16-byte boundaries, copied into dst (the value at base + x lands at
// dst[(base & 3) + x]); returns the bytes.
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

// Per-element scalars of the update phase (first source, receiver slot on
// the last stage, Zener coefficients) and the NPML switch, loaded when the
// chunk starts: read where they are used, each is a dependent global load
// whose latency the block (one per SM) would wait out once per chunk.
template <bool ATT>
struct ElemScalars {
  int src, slot;
  bool off;
  float ae[ATT ? 3 * kNMB : 1];
  __device__ __forceinline__ void load(const StageArgs& a, int b, int e) {
    src = __ldg(a.src_head + e);
    slot = a.last_stage ? __ldg(a.rec_slot + e) : -1;
    off = a.pml_off[b] != 0;
    if (ATT) {
#pragma unroll
      for (int j = 0; j < 3 * kNMB; ++j) ae[j] = __ldg(a.ael + (long long)e * 3 * kNMB + j);
    }
  }
};

// First float of chunk c's range in an element-blocked array of F fields.
template <int F, int Np>
__device__ __forceinline__ long long eblock_chunk(long long ld, const Chunk& c) {
  return eblock<F, Np>(ld, c.b, c.e0, 0);
}

// Buffer A of chunk c (one thread): F', G', H', their residuals, profiles.
template <int N>
__device__ __forceinline__ void load_state_a(const StageArgs& a, const Chunk& c, float* sAux, float* sAux2,
                                             float* sPrf, uint32_t mbar) {
  using B = BulkOrder<N>;
  constexpr int Np = B::Np;
  const long long ba = eblock_chunk<27, Np>(a.lda, c);
  const uint32_t na = uint32_t(c.ne) * B::FA * 4;
  const long long bp = (long long)c.e0 * 9 * Np, np_ = (long long)c.ne * 9 * Np;
  mbar_expect_tx(mbar, 2 * na + bulk_bytes(bp, np_));
  bulk_load(sAux, a.aux + ba, na, mbar);
  bulk_load(sAux2, a.aux2 + ba, na, mbar);
  bulk_range(sPrf, a.prof, bp, np_, mbar);
}
template <int N>
__device__ __forceinline__ void store_state_a(const StageArgs& a, const Chunk& c, const float* sAux,
                                              const float* sAux2) {
  using B = BulkOrder<N>;
  const long long ba = eblock_chunk<27, B::Np>(a.lda, c);
  const uint32_t na = uint32_t(c.ne) * B::FA * 4;
  bulk_store(a.aux + ba, sAux, na);
  bulk_store(a.aux2 + ba, sAux2, na);
  bulk_commit();
}

// Buffer B of chunk c (one thread): residual of q (LSERK) or step-start q
// rows (TVD, field-major: one widened range per field), memory variables and
// their residuals.
template <int N, bool ATT, int MODE>
__device__ __forceinline__ void load_state_b(const StageArgs& a, const Chunk& c, float* sRes, float* sTh,
                                             float* sTh2, uint32_t mbar) {
  using B = BulkOrder<N>;
  constexpr int Np = B::Np;
  const bool resv = (MODE == MODE_LSERK) || a.ca != 0.f;
  const long long br = eblock_chunk<9, Np>(a.ldq, c);
  const uint32_t nr = uint32_t(c.ne) * B::FR * 4;
  const long long bq = (long long)c.b * 9 * a.ldq + (long long)c.e0 * Np, nq = (long long)c.ne * Np;
  const long long bt = eblock_chunk<6 * kNMB, Np>(a.ldt, c);
  const uint32_t nt = uint32_t(c.ne) * B::FT * 4;
  uint32_t bytes = 0;
  if (resv) {
    if (MODE == MODE_LSERK) bytes += nr;
    else
      for (int f = 0; f < 9; ++f) bytes += bulk_bytes(bq + f * a.ldq, nq);
  }
  if (ATT) bytes += 2 * nt;
  mbar_expect_tx(mbar, bytes);
  if (resv) {
    if (MODE == MODE_LSERK) {
      bulk_load(sRes, a.res + br, nr, mbar);
    } else {
      for (int f = 0; f < 9; ++f) bulk_range(sRes + f * B::QR, a.q_n, bq + f * a.ldq, nq, mbar);
    }
  }
  if (ATT) {
    bulk_load(sTh, a.th + bt, nt, mbar);
    bulk_load(sTh2, a.th2 + bt, nt, mbar);
  }
}
template <int N, bool ATT, int MODE>
__device__ __forceinline__ void store_state_b(const StageArgs& a, const Chunk& c, const float* sRes, const float* sTh,
                                              const float* sTh2) {
  using B = BulkOrder<N>;
  constexpr int Np = B::Np;
  if (MODE == MODE_LSERK) bulk_store(a.res + eblock_chunk<9, Np>(a.ldq, c), sRes, uint32_t(c.ne) * B::FR * 4);
  if (ATT) {
    const long long bt = eblock_chunk<6 * kNMB, Np>(a.ldt, c);
    bulk_store(a.th + bt, sTh, uint32_t(c.ne) * B::FT * 4);
    bulk_store(a.th2 + bt, sTh2, uint32_t(c.ne) * B::FT * 4);
  }
  bulk_commit();
}

// pml_update with the node's damping profiles pr, auxiliaries av and their
// residuals a2 (TVD: step-start values) in shared memory at a stride of Np
// floats, updated there in place; the same operations in the same order.
template <int Np, int MODE>
__device__ __forceinline__ void pml_update_smem(const StageArgs& a, bool off, const float* pr, float* av, float* a2,
                                                float* F, float* G, float* H) {
  if (off) return;  // pmlcheck(:) = .false.: ordinary element (src/timeloopMod.f90:537)
  const float ddx = pr[0], ddy = pr[Np], ddz = pr[2 * Np];
  const float alx = pr[3 * Np], aly = pr[4 * Np], alz = pr[5 * Np];
  const float ikx = 1.f / pr[6 * Np], iky = 1.f / pr[7 * Np], ikz = 1.f / pr[8 * Np];
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
      a2[i * Np] = r1;
      a2[(9 + i) * Np] = r2;
      a2[(18 + i) * Np] = r3;
      nf = fp + a.cb * r1;
      ng_ = gp + a.cb * r2;
      nh = hp + a.cb * r3;
    } else {
      float n1, n2, n3;
      if (a.stage_first) {
        a2[i * Np] = fp;
        a2[(9 + i) * Np] = gp;
        a2[(18 + i) * Np] = hp;
        n1 = fp; n2 = gp; n3 = hp;
      } else {
        n1 = a2[i * Np]; n2 = a2[(9 + i) * Np]; n3 = a2[(18 + i) * Np];
      }
      nf = a.ca * n1 + a.cb * (fp + a.dt * rf);
      ng_ = a.ca * n2 + a.cb * (gp + a.dt * rg);
      nh = a.ca * n3 + a.cb * (hp + a.dt * rh);
    }
    av[i * Np] = nf;
    av[(9 + i) * Np] = ng_;
    av[(18 + i) * Np] = nh;
    F[i] = phi;
    G[i] = psi;
    H[i] = ome;
  }
}

// finish_node with the node's update-phase state in shared memory, updated
// there in place: rs[c * rstride] the residual of q (TVD: step-start q, read
// only), th / th2 the memory variables and their residuals (TVD: step-start
// values) at a stride of Np.  The new q goes to global memory.
template <int Np, bool ATT, int MODE>
__device__ __forceinline__ void finish_node_smem(const StageArgs& a, int b, int e, long long node, float* rq,
                                                 const float* S, float* rs, int rstride, float* ths, float* th2s,
                                                 const float* qown, int qstride, const ElemScalars<ATT>& es) {
  const int n = int(node - (long long)e * Np);
  if (ATT) {
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
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const float r = a.ca * rs[c * rstride] + a.dt * rq[c];
      rs[c * rstride] = r;
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

// Threads of the bulk-copy NPML kernel: 8 compute warps (the node mapping of
// stage_kernel) and one producer warp that issues every copy of the chunk
// pipeline -- the next chunk's records, wavefield, connectivity and
// neighbour-trace gather (cp.async) and the bulk loads and stores of buffers
// A and B -- so the compute warps spend no issue slots on them and never wait
// at a barrier for a thread that is issuing copies.
constexpr int kCompute = 256;
constexpr int kBulkThreads = kCompute + 32;

template <int N, bool ATT, int MODE>
__global__ void __launch_bounds__(kBulkThreads, 1) stage_npml_bulk_kernel(const StageArgs a) {
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
  const bool producer = tid >= kCompute;
  const int lane = tid & 31;
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
  int le = E, n = 0;  // the producer warp holds no node
  if (!producer) {
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
  }
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
    if (tid == kCompute) {
      tc::mbar_init(mbarA, 1);
      tc::mbar_init(mbarB, 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (producer) {
      if (lane == 0) {
        load_state_a<N>(a, c0, sAux, sAux2, sPrf, mbarA);
        load_state_b<N, ATT, MODE>(a, c0, sRes, sTh, sTh2, mbarB);
      }
      issue_main<O>(a, c0, sBuf, sBuf + O::SGEO, reinterpret_cast<int*>(sBuf + O::SGEO + O::SQF + O::STR),
                    wn < nwork ? &c1 : nullptr, lane, 32);
      issue_traces<O>(a, c0, ids0, sBuf + O::SGEO + O::SQF, sPat, 0, -1, lane, 32);
      cp_async_commit();
    }
  }

  bool ok = true;
  uint32_t phase = 0;  // parity of both mbarriers' current phase (each completes once per chunk)
  Chunk prev;
  for (int p = 0; w < nwork; w += gridDim.x, p ^= 1, phase ^= 1) {
    const Chunk ch = chunk_of<E>(a, w, nchunk);
    const int b = ch.b, e0 = ch.e0, ne = ch.ne;
    const bool first = w == (int)blockIdx.x;
    float* buf = sBuf + p * O::BUF;
    const float* sGeo = buf;
    const float* sTr = buf + O::SGEO + O::SQF;
    const float* sQF = buf + O::SGEO + int(((long long)e0 * Np) & 3);
    const int* sIds = reinterpret_cast<const int*>(sTr + O::STR);
    cp_async_wait_all();  // the producer's copies of this chunk (the compute warps have none)
    __syncthreads();  // (1) records, wavefield and traces in `buf`; the previous chunk's buffer B is final
    const int wn = w + gridDim.x;
    Chunk cn;
    if (wn < nwork) cn = chunk_of<E>(a, wn, nchunk);
    float* nbuf = sBuf + (p ^ 1) * O::BUF;
    bool okA = true;
    const bool active = le < ne;
    const long long node = (long long)(e0 + (active ? le : 0)) * Np + n;
    ElemScalars<ATT> es;
    if (producer) {
      // the previous chunk's residual and memory variables go back, this
      // chunk's come in; the next chunk's records, wavefield and connectivity start
      if (lane == 0 && !first) {
        store_state_b<N, ATT, MODE>(a, prev, sRes, sTh, sTh2);
        bulk_wait_read();
        load_state_b<N, ATT, MODE>(a, ch, sRes, sTh, sTh2, mbarB);
      }
      if (wn < nwork) {
        const int wnn = wn + gridDim.x;
        Chunk cnn;
        if (wnn < nwork) cnn = chunk_of<E>(a, wnn, nchunk);
        issue_main<O>(a, cn, nbuf, nbuf + O::SGEO, reinterpret_cast<int*>(nbuf + O::SGEO + O::SQF + O::STR),
                      wnn < nwork ? &cnn : nullptr, lane, 32);
      }
    } else {
      es.load(a, b, e0 + (active ? le : 0));
      // ---- face amplitudes ---------------------------------------------------------
      for (int i = tid; i < ne * NF; i += kCompute) {
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
      // ---- NPML: auxiliary update (in place) and contravariant modified fluxes -------
      okA = tc::mbar_wait(mbarA, phase);
      if (active && okA) {
        const float* g = sGeo + le * O::GSTR;
        float qv[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) qv[c] = sQF[c * O::QF + le * Np + n];
        float F[9], G[9], H[9];
        elastic_fluxes(g, qv, F, G, H);
        const float* ps = sPrf + int(((long long)e0 * 9 * Np) & 3) + le * 9 * Np + n;
        pml_update_smem<Np, MODE>(a, es.off, ps, sAux + le * B::FA + n, sAux2 + le * B::FA + n, F, G, H);
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
      tc::fence_async_smem();  // this thread's writes to buffer A are seen by the bulk store
    }
    if (__syncthreads_or(!okA)) {  // (2) amplitudes and rows are in shared memory; buffer A is final
      ok = false;
      break;
    }
    if (producer) {
      // buffer A goes back and is refilled with the next chunk's; the next chunk's traces
      if (lane == 0) {
        store_state_a<N>(a, ch, sAux, sAux2);
        if (wn < nwork) {
          bulk_wait_read();
          load_state_a<N>(a, cn, sAux, sAux2, sPrf, mbarA);
        }
      }
      if (wn < nwork) issue_traces<O>(a, cn, sIds, nbuf + O::SGEO + O::SQF, sPat, 0, -1, lane, 32);
      cp_async_commit();
      prev = ch;
      continue;
    }
    if (!active) {
      prev = ch;
      continue;  // idle threads of a partial chunk
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
    // ---- memory variables, sources, receivers, stage update (state in buffer B) ---
    if (tc::mbar_wait(mbarB, phase)) {
      float* rs;
      int rstride;
      if (MODE == MODE_LSERK) {
        rs = sRes + le * B::FR + n;
        rstride = Np;
      } else {
        rs = sRes + int(((long long)b * 9 * a.ldq + (long long)e0 * Np) & 3) + le * Np + n;
        rstride = B::QR;
      }
      finish_node_smem<Np, ATT, MODE>(a, b, e, node, rq, S, rs, rstride, sTh + le * B::FT + n,
                                      sTh2 + le * B::FT + n, sQF + le * Np + n, O::QF, es);
    } else {
      atomicOr(a.flag, 8);
    }
    tc::fence_async_smem();  // this thread's writes to buffer B are seen by the bulk store
    prev = ch;
  }
  const bool all_ok = __syncthreads_and(ok);
  if (tid == kCompute) {
    if (all_ok) {
      store_state_b<N, ATT, MODE>(a, prev, sRes, sTh, sTh2);
    } else {
      // a load did not complete in time: wait once more, again bounded, for
      // the loads of this chunk still in flight before the block exits
      atomicOr(a.flag, 8);
      tc::mbar_wait(mbarA, phase, 1u << 24);
      tc::mbar_wait(mbarB, phase, 1u << 24);
    }
    bulk_wait_all();
  }
  cp_async_wait_all();
}

}  // namespace nexd_dev
