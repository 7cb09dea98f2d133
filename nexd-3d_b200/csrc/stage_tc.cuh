// Stage kernel with the element contraction on the tensor cores (sm_100a,
// tcgen05, three-way split BF16 with FP32 accumulation).
//
// Same stage as stage_kernel (src/timeloopMod.f90:395-476 and
// src/rungekuttaMod.f90:27-88), with the volume and surface terms written as
// one stacked contraction per chunk of E elements:
//
//   R[(e,c)][n] = sum_d sum_k D_d[n][k] X_d[(e,c)][k] + sum_j LIFT[n][j] Y[(e,c)][j]
//
// where, for column c < 9, X_d = rx_d F + ry_d G + rz_d H are the contravariant
// fluxes (NPML: the modified ones) and Y the upwind face flux fscale/2 *
// T(A+|A|)T^-1 dq expanded from its three characteristic amplitudes; columns
// 9..14 (anelastic) carry S = lifted anelastic flux - strain rate, whose
// volume part is the symmetric velocity gradient taken through the same
// D_d.  The operator [Dr Ds Dt LIFT] (K = 3 Np, padded to 16, + 4 NpF) sits in
// shared memory for the whole launch as bf16 h, m, l rows; the CUDA cores
// write the data operand as bf16 h, m, l; one thread issues the MMAs (the
// volume part as soon as its rows are written, so it runs on the tensor
// cores while the CUDA cores compute the face fluxes); the FP32 result in
// tensor memory is transposed through shared memory back to one thread per
// node, which adds the memory variables and sources and updates the state.
#pragma once
#include "stage_kernel.cuh"
#include "tc_gemm.cuh"

namespace nexd_dev {

template <int N>
struct TcOrder {
  using O = Order<N>;
  static constexpr int Np = O::Np, NpF = O::NpF, E = O::E;
  static constexpr int COLS = 16;                   // per element: 9 rq + 6 S + 1 pad
  static constexpr int ROWS = E * COLS;             // data rows in use
  static constexpr int MT = (ROWS + 127) / 128;     // 128-row MMA tiles
  static constexpr int KV = 3 * Np;                 // volume rows
  static constexpr int KV16 = (KV + 15) / 16 * 16;  // first face row
  static constexpr int KSV = KV16 / 16;             // volume MMA K steps
  static constexpr int KU = KV16 + 4 * NpF;         // K in use
  static constexpr int KS = (KU + 15) / 16;         // MMA K steps
  static constexpr int NP16 = (Np + 15) / 16 * 16;  // output nodes, padded
  static constexpr int BN = 3 * NP16;               // operator rows: h, m, l parts
  static constexpr int KSLAB = (KS + 3) / 4;        // 64-wide K slabs of the operator
  static constexpr uint32_t B_SLAB = BN / 8 * 1024;
  static constexpr uint32_t B_BYTES = KSLAB * B_SLAB;
  static constexpr uint32_t A_LBO = 1024;           // 64-row atoms
  static constexpr uint32_t A_SBO = MT * 2 * 1024;  // 8-deep K groups
  static constexpr uint32_t A_BYTES = KS * 2 * A_SBO;  // one of the h, m, l parts
  static constexpr int RS = Np | 1;                 // row stride of the transposed result (odd: no bank conflicts)
  static constexpr int TCOLS = MT * BN;             // accumulator columns
  static constexpr uint32_t TMEM_COLS = TCOLS <= 32 ? 32 : TCOLS <= 64 ? 64 : TCOLS <= 128 ? 128 : TCOLS <= 256 ? 256 : 512;
  // prefetch: records, own wavefield and connectivity double-buffered, face traces single
  static constexpr int PB = O::SGEO + O::SQF + O::SIDS;
  static constexpr size_t smem_bytes() {
    return 1024 + B_BYTES + 3 * size_t(A_BYTES) + size_t(2 * PB + O::STR + O::SPAT) * 4 + 16;
  }
  // the transposed result aliases the l data part below its first zero padding row
  static_assert(ROWS * RS * 4 <= (KV / 8) * A_SBO, "result buffer overlaps the zero K padding");
  static_assert(BN % 16 == 0 && TCOLS <= 256 && MT == 1, "tile shape");
};

// Orders with a tensor-core stage kernel (the others exceed an SM's shared memory).
__host__ __device__ constexpr bool tc_order_supported(int N) { return N == 4; }

template <int N, bool ATT, bool PML, int MODE>
__global__ void __launch_bounds__(256, 1) stage_tc_kernel(const StageArgs a, const uint4* __restrict__ ops) {
  using O = Order<N>;
  using T = TcOrder<N>;
  constexpr int Np = O::Np, NpF = O::NpF, NF = O::NF, E = O::E;
  extern __shared__ __align__(16) unsigned char tsm[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tsm) + 1023) & ~uintptr_t(1023));
  unsigned char* sB = base;                  // operator: h, m, l rows
  unsigned char* sA = sB + T::B_BYTES;       // data operand: h, m, l parts, A_BYTES apart
  float* sR = reinterpret_cast<float*>(sA + 2 * T::A_BYTES);  // transposed result (aliases the l part)
  float* sPB = reinterpret_cast<float*>(sA + 3 * T::A_BYTES); // 2 x [records | wavefield | connectivity]
  float* sTr = sPB + 2 * T::PB;              // neighbour face traces of the current chunk
  unsigned char* sPat = reinterpret_cast<unsigned char*>(sTr + O::STR);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sPat + O::SPAT * 4);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int nel = a.e_end - a.e_begin;
  const int nchunk = (nel + E - 1) / E;
  const int nwork = nchunk * a.nbatch;
  int w = blockIdx.x;
  if (w >= nwork) return;

  for (int i = tid; i < int(T::B_BYTES / 16); i += blockDim.x) reinterpret_cast<uint4*>(sB)[i] = ops[i];
  for (int i = tid; i < int(3 * T::A_BYTES / 16); i += blockDim.x) reinterpret_cast<uint4*>(sA)[i] = make_uint4(0, 0, 0, 0);
  for (int i = tid; i < a.npat * NpF; i += blockDim.x) sPat[i] = a.patterns[i];
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tslot), T::TMEM_COLS);
  if (tid == 0) tc::mbar_init(tc::smem_u32(mbar), 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  auto geo_of = [&](int p) { return sPB + p * T::PB; };
  auto q_of = [&](int p) { return sPB + p * T::PB + O::SGEO; };
  auto ids_of = [&](int p) { return reinterpret_cast<int*>(sPB + p * T::PB + O::SGEO + O::SQF); };

  const int le = tid / Np;
  const int n = tid - le * Np;
  {
    const Chunk c0 = chunk_of<E>(a, w, nchunk);
    const int wn = w + gridDim.x;
    Chunk c1;
    if (wn < nwork) c1 = chunk_of<E>(a, wn, nchunk);
    int* ids0 = ids_of(1);  // scratch until the second chunk's copies land there
    for (int i = tid; i < c0.ne * 8; i += blockDim.x) {
      const int ee = i >> 3, k = i & 7;
      ids0[ee * 12 + k] = k < 4 ? reinterpret_cast<const int*>(a.nbr)[4 * (c0.e0 + ee) + k]
                                : reinterpret_cast<const int*>(a.fcode)[4 * (c0.e0 + ee) + k - 4];
    }
    __syncthreads();
    issue_main<O>(a, c0, geo_of(0), q_of(0), ids_of(0), wn < nwork ? &c1 : nullptr);
    issue_traces<O>(a, c0, ids0, sTr, sPat);
    cp_async_commit();
  }

  const uint32_t ah = tc::smem_u32(sA), bb = tc::smem_u32(sB);
  constexpr uint32_t id3 = tc::idesc_bf16(128, T::BN), id2 = tc::idesc_bf16(128, 2 * T::NP16),
                     id1 = tc::idesc_bf16(128, T::NP16);
  // MMAs of K steps [s0, s1): data h x (H|M|L), m x (H|M), l x H into the three column blocks
  auto issue_mmas = [&](int s0, int s1) {
    for (int s = s0; s < s1; ++s) {
      const uint32_t aoff = uint32_t(s) * 2 * T::A_SBO;
      const uint64_t db = tc::smem_desc(bb + (s / 4) * T::B_SLAB + (s % 4) * 32, 16, 1024);
      tc::mma_bf16(tmem, tc::smem_desc(ah + aoff, T::A_LBO, T::A_SBO), db, id3, s > 0);
      tc::mma_bf16(tmem, tc::smem_desc(ah + T::A_BYTES + aoff, T::A_LBO, T::A_SBO), db, id2, 1);
      tc::mma_bf16(tmem, tc::smem_desc(ah + 2 * T::A_BYTES + aoff, T::A_LBO, T::A_SBO), db, id1, 1);
    }
  };

  uint32_t phase = 0;
  for (int p = 0; w < nwork; w += gridDim.x, p ^= 1, phase ^= 1) {
    const Chunk ch = chunk_of<E>(a, w, nchunk);
    const int b = ch.b, e0 = ch.e0, ne = ch.ne;
    const float* sGeo = geo_of(p);
    // own wavefield of the chunk: field c of node n of element le at sQF[c * QF + le * Np + n]
    const float* sQF = q_of(p) + int(((long long)e0 * Np) & 3);
    const int* sIds = ids_of(p);
    cp_async_wait_all();
    __syncthreads();  // chunk data landed; the previous chunk's result buffer is consumed

    const bool active = le < ne;
    const long long node = (long long)(e0 + (active ? le : 0)) * Np + n;
    NodePrefetch<ATT, PML, MODE, true> pf;
    if (active) pf.template load<Np>(a, b, e0 + le, node);
    const int wn = w + gridDim.x;
    Chunk cn;
    if (wn < nwork) {
      cn = chunk_of<E>(a, wn, nchunk);
      const int wnn = wn + gridDim.x;
      Chunk cnn;
      if (wnn < nwork) cnn = chunk_of<E>(a, wnn, nchunk);
      issue_main<O>(a, cn, geo_of(p ^ 1), q_of(p ^ 1), ids_of(p ^ 1), wnn < nwork ? &cnn : nullptr);
      cp_async_commit();
    }

    // ---- volume fluxes: data rows K = d Np + node ------------------------------
    if (active) {
      const float* g = sGeo + le * O::GSTR;
      float qv[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) qv[c] = sQF[c * O::QF + le * Np + n];
      float F[9], G[9], H[9];
      elastic_fluxes(g, qv, F, G, H);
      if constexpr (PML) pml_node<Np, ATT, MODE>(a, b, e0 + le, n, pf, F, G, H);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float m0 = g[G_RX + 3 * d], m1 = g[G_RY + 3 * d], m2 = g[G_RZ + 3 * d];
        float v[16];
#pragma unroll
        for (int i = 0; i < 9; ++i) v[i] = m0 * F[i] + m1 * G[i] + m2 * H[i];
        if (ATT) {
          // minus the symmetric velocity gradient (its d-th contravariant part)
          const float vx = qv[6], vy = qv[7], vz = qv[8];
          v[9] = -(m0 * vx);
          v[10] = -(m1 * vy);
          v[11] = -(m2 * vz);
          v[12] = -0.5f * (m0 * vy + m1 * vx);
          v[13] = -0.5f * (m1 * vz + m2 * vy);
          v[14] = -0.5f * (m0 * vz + m2 * vx);
        } else {
#pragma unroll
          for (int c = 9; c < 15; ++c) v[c] = 0.f;
        }
        v[15] = 0.f;
        tc::store_a16x3(sA, T::A_BYTES, le * T::COLS, d * Np + n, v, T::A_LBO, T::A_SBO);
      }
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      issue_mmas(0, T::KSV);
    }

    // ---- face fluxes: data rows K = KV16 + face node (tensor cores busy) --------
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
      const float a0 = ap * fs, a1 = as1 * fs, a2 = as2 * fs;
      // the face flux of this face node: 9 fields, then the anelastic flux (zero when elastic)
      float v[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) v[c] = 0.f;
      face_expand<ATT>(g, f, a0, a1, a2, v, v + 9);
      tc::store_a16x3(sA, T::A_BYTES, ee * T::COLS, T::KV16 + j, v, T::A_LBO, T::A_SBO);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      issue_mmas(T::KSV, T::KS);
      tc::mma_commit(tc::smem_u32(mbar));
    }
    // the face traces of the next chunk (its connectivity arrived with this chunk)
    if (wn < nwork) {
      issue_traces<O>(a, cn, sIds, sTr, sPat);
      cp_async_commit();
    }

    const bool done = tc::mbar_wait(tc::smem_u32(mbar), phase);
    if (__syncthreads_or(!done)) {
      if (tid == 0) atomicOr(a.flag, 2);
      // The committed MMAs may still be writing the accumulator: wait once
      // more, again bounded, for their arrival before the TMEM is released
      // at the end of the kernel.
      tc::mbar_wait(tc::smem_u32(mbar), phase, 1u << 24);
      break;
    }
    tc::fence_after_sync();
    {
      // lane m holds row m: node columns n of the h, m, l blocks at n, NP16 + n, 2 NP16 + n;
      // warp w reads TMEM lanes 32 (w % 4) .. +31, warps 0-3 the column groups
      // 0, 64, ..., warps 4-7 the groups 32, 96, ...
      const int quarter = warp & 3;
      const int m = 32 * quarter + (tid & 31);
      const uint32_t ta = tmem + (uint32_t(32 * quarter) << 16);
      float* r = sR + m * T::RS;
#pragma unroll
      for (int c0 = 32 * (warp >> 2); c0 < T::NP16; c0 += 64) {
        constexpr int W32 = 32;
        float v0[W32], v1[W32], v2[W32];
        const bool wide = T::NP16 - c0 >= 32;
        if (wide) {
          tc::tmem_ld32(ta + c0, v0);
          tc::tmem_ld32(ta + T::NP16 + c0, v1);
          tc::tmem_ld32(ta + 2 * T::NP16 + c0, v2);
        } else {
          tc::tmem_ld16(ta + c0, v0);
          tc::tmem_ld16(ta + T::NP16 + c0, v1);
          tc::tmem_ld16(ta + 2 * T::NP16 + c0, v2);
        }
        tc::tmem_wait_ld();
        if (m < T::ROWS) {
#pragma unroll
          for (int k = 0; k < W32; ++k)
            if (c0 + k < Np && (wide || k < 16)) r[c0 + k] = (v0[k] + v1[k]) + v2[k];
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();

    // ---- memory variables, sources, receivers, stage update ---------------------
    if (active) {
      const int e = e0 + le;
      const float* r = sR + (le * T::COLS) * T::RS + n;
      float rq[9], S[6];
#pragma unroll
      for (int c = 0; c < 9; ++c) rq[c] = r[c * T::RS];
      if (ATT) {
#pragma unroll
        for (int c = 0; c < 6; ++c) S[c] = r[(9 + c) * T::RS];
      }
      finish_node<Np, ATT, PML, MODE>(a, b, e, node, rq, S, pf, sQF + le * Np + n, O::QF);
    }
  }
  cp_async_wait_all();
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, T::TMEM_COLS);
}

}  // namespace nexd_dev
