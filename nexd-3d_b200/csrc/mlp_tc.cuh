// tcgen05 GEMM of the boundary network's training (sm_100a):
//   C[M][N] (+)= sum_k A(m,k) B(k,n)
// with A(m,k) = TA ? A[k lda + m] : A[m lda + k] and
//      B(k,n) = TB ? B[n ldb + k] : B[k ldb + n], FP32 in and out.
//
// FP32-grade products come from the three-way split of both operands into
// BF16 parts (x = h + m + l, 24 significant bits together) and the six
// products above 2^-24 (Ah Bh, Ah Bm, Ah Bl, Am Bh, Am Bm, Al Bh), all
// accumulated in one FP32 accumulator in tensor memory.  One CTA of 128
// threads owns 128 rows (one TMEM lane each) and all N <= 256 columns; K
// runs in chunks of 64 that the CUDA cores stage into shared memory (load,
// split, store in the K-major 128-byte-swizzled layout of both operands)
// while the previous chunk's MMAs run (two staging buffers up to N = 160,
// one above); long K is split over CTAs whose partial sums a second kernel
// adds in a fixed order.  Every split has at least one k (the host sizes
// the splits).
#pragma once
#include "tc_gemm.cuh"

namespace nexd_dev {

constexpr int kTcgThreads = 128;
constexpr int kTcgMaxN = 256;
constexpr int kTcgMaxSplits = 32;
constexpr long long kMlpSplitFloats = 1LL << 22;  // split-K partial sums in the MLP workspace

__host__ __device__ constexpr int tcg_np(int N) { return (N + 15) / 16 * 16; }
// one K-major part of `rows` rows (a multiple of 8) and 64 k
__host__ __device__ constexpr uint32_t tcg_part_bytes(int rows) { return uint32_t(rows / 8) * 1024u; }
__host__ __device__ constexpr uint32_t tcg_buf_bytes(int NP) { return 3u * (tcg_part_bytes(128) + tcg_part_bytes(NP)); }
__host__ __device__ constexpr size_t tcg_smem_bytes(int NP, int nbuf) { return 1024 + nbuf * size_t(tcg_buf_bytes(NP)) + 64; }
// two staging buffers (staging overlaps the MMAs) when they fit, else one
__host__ __device__ constexpr int tcg_nbuf(int NP) { return tcg_smem_bytes(NP, 2) <= 227 * 1024 ? 2 : 1; }

// Instruction descriptor, kind::f16: bf16 x bf16 -> f32, A and B K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_kk(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// Byte offset of the 16-byte chunk kc (k = 8 kc .. 8 kc + 7) of row r in a
// K-major SWIZZLE_128B part: 8-row groups of 1024 bytes, chunk kc of row r
// stored at position kc ^ (r % 8).
__device__ __forceinline__ uint32_t kmajor_offset(int r, int kc) {
  return uint32_t(r >> 3) * 1024u + uint32_t(r & 7) * 128u + uint32_t((kc ^ (r & 7)) << 4);
}

struct TcGemmArgs {
  int M, N, K;
  const float* A;
  int lda;
  const float* B;
  int ldb;
  float* C;
  int ldc;
  int acc;        // C += product (single split)
  int kper;       // K per split (a multiple of 64)
  float* partial; // [splits][M][N] when gridDim.y > 1
};

// Loads 8 consecutive k of one row (zero outside [0, rows) x [k0, kend)),
// splits them and stores the three parts.
template <bool T>
__device__ __forceinline__ void stage_row8(unsigned char* part0, uint32_t part_bytes, const float* X, int ld, int row,
                                           int rows, int k0, int kend, int r, int kc) {
  float v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int k = k0 + kc * 8 + j;
    v[j] = (row < rows && k < kend) ? (T ? X[(long long)k * ld + row] : X[(long long)row * ld + k]) : 0.f;
  }
  uint4 h, m, l;
  tc::split3(v[0], v[1], h.x, m.x, l.x);
  tc::split3(v[2], v[3], h.y, m.y, l.y);
  tc::split3(v[4], v[5], h.z, m.z, l.z);
  tc::split3(v[6], v[7], h.w, m.w, l.w);
  const uint32_t o = kmajor_offset(r, kc);
  *reinterpret_cast<uint4*>(part0 + o) = h;
  *reinterpret_cast<uint4*>(part0 + part_bytes + o) = m;
  *reinterpret_cast<uint4*>(part0 + 2 * part_bytes + o) = l;
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(kTcgThreads, 1) tc_gemm_kernel(const TcGemmArgs g) {
  extern __shared__ __align__(16) unsigned char tcg_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tcg_raw) + 1023) & ~uintptr_t(1023));
  const int NP = tcg_np(g.N);
  const uint32_t PA = tcg_part_bytes(128), PB = tcg_part_bytes(NP), BUF = tcg_buf_bytes(NP);
  const int nbuf = tcg_nbuf(NP);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(base + nbuf * BUF);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * 128;
  const int kbeg = blockIdx.y * g.kper, kend = min(g.K, kbeg + g.kper);
  const int nch = (kend - kbeg + 63) / 64;
  const uint32_t ncols = NP <= 32 ? 32u : NP <= 64 ? 64u : NP <= 128 ? 128u : 256u;
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tslot), ncols);
  if (tid == 0) {
    tc::mbar_init(tc::smem_u32(&mbar[0]), 1);
    tc::mbar_init(tc::smem_u32(&mbar[1]), 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t id = idesc_bf16_kk(128, NP);
  bool ok = true;
  uint32_t ph[2] = {0u, 0u};
  for (int c = 0; c < nch; ++c) {
    const int p = c % nbuf;
    unsigned char* buf = base + p * BUF;
    if (c >= nbuf) {  // the buffer's previous chunk (c - nbuf) has been multiplied
      ok = tc::mbar_wait(tc::smem_u32(&mbar[p]), ph[p]) && ok;
      ph[p] ^= 1u;
      tc::fence_after_sync();
    }
    const int k0 = kbeg + c * 64;
    for (int i = tid; i < 128 * 8; i += kTcgThreads)
      stage_row8<TA>(buf, PA, g.A, g.lda, m0 + (i & 127), g.M, k0, kend, i & 127, i >> 7);
    for (int i = tid; i < NP * 8; i += kTcgThreads)
      stage_row8<!TB>(buf + 3 * PA, PB, g.B, g.ldb, i % NP, g.N, k0, kend, i % NP, i / NP);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t a = tc::smem_u32(buf), b = a + 3 * PA;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const uint64_t ah = tc::smem_desc(a + s * 32, 16, 1024), am = tc::smem_desc(a + PA + s * 32, 16, 1024),
                       al = tc::smem_desc(a + 2 * PA + s * 32, 16, 1024);
        const uint64_t bh = tc::smem_desc(b + s * 32, 16, 1024), bm = tc::smem_desc(b + PB + s * 32, 16, 1024),
                       bl = tc::smem_desc(b + 2 * PB + s * 32, 16, 1024);
        tc::mma_bf16(tmem, ah, bh, id, (c > 0 || s > 0) ? 1u : 0u);
        tc::mma_bf16(tmem, ah, bm, id, 1u);
        tc::mma_bf16(tmem, ah, bl, id, 1u);
        tc::mma_bf16(tmem, am, bh, id, 1u);
        tc::mma_bf16(tmem, am, bm, id, 1u);
        tc::mma_bf16(tmem, al, bh, id, 1u);
      }
      tc::mma_commit(tc::smem_u32(&mbar[p]));
    }
  }
  // the last commit covers every MMA of this CTA
  {
    const int p = (nch - 1) % nbuf;
    if (!tc::mbar_wait(tc::smem_u32(&mbar[p]), ph[p])) {
      ok = false;
      tc::mbar_wait(tc::smem_u32(&mbar[p]), ph[p], 1u << 24);  // give them longer before TMEM is released
    }
  }
  tc::fence_after_sync();
  // the same answer in every thread (the loads below are warp-collective);
  // a wait that ran out leaves NaN in this tile's outputs instead of the sums
  ok = __syncthreads_and(ok ? 1 : 0) != 0;
  const int m = m0 + tid;
  const uint32_t lane = tmem + (uint32_t(warp * 32) << 16);
  const bool single = gridDim.y == 1;
  for (int c0 = 0; c0 < NP; c0 += 32) {
    float v[32];
    const int nc = NP - c0 >= 32 ? 32 : 16;
    if (ok) {
      if (nc == 32) tc::tmem_ld32(lane + c0, v);
      else tc::tmem_ld16(lane + c0, v);
      tc::tmem_wait_ld();
    } else {
      for (int j = 0; j < 32; ++j) v[j] = __int_as_float(0x7fc00000);
    }
    if (m < g.M) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int n = c0 + j;
        if (j >= nc || n >= g.N) continue;
        if (single) {
          float* cp = g.C + (long long)m * g.ldc + n;
          *cp = g.acc ? *cp + v[j] : v[j];
        } else {
          g.partial[((long long)blockIdx.y * g.M + m) * g.N + n] = v[j];
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// C[m][n] (+)= sum over the splits, in split order.
__global__ void splitk_reduce_kernel(int M, int N, int splits, const float* __restrict__ partial, float* C, int ldc,
                                     int acc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)M * N) return;
  const int m = int(i / N), n = int(i - (long long)m * N);
  float s = acc ? C[(long long)m * ldc + n] : 0.f;
  for (int k = 0; k < splits; ++k) s += partial[(long long)k * M * N + i];
  C[(long long)m * ldc + n] = s;
}

}  // namespace nexd_dev
