// tcgen05 building blocks for the split-BF16 element contraction (sm_100a).
//
// The stage contraction is D[m][n] = sum_k A[m][k] * B[n][k] with
//   A: per-chunk data (rows m = element x column, K = contravariant volume
//      fluxes of every node and lifted face fluxes of every face node),
//      bf16, MN-major, 128-byte swizzle, staged by the CUDA cores;
//   B: the stacked operator [Dr Ds Dt LIFT] (rows n = output node), bf16,
//      K-major, 128-byte swizzle, staged once per block;
//   D: FP32 accumulator in tensor memory (lane m, column n).
// FP32-grade accuracy comes from three-way splits x = h + m + l (each bf16,
// 24 significant bits together) of both operands and the six products
// whose weight is above 2^-24: Ah(BH+BM+BL) + Am(BH+BM) + Al BH.  The BH, BM
// and BL rows sit side by side, so each data part is one MMA of 3, 2 or 1
// operator widths accumulating into column blocks that the epilogue adds.
//
// Shared-memory layouts (byte offsets; every atom 1024-byte aligned):
//   A (MN-major, SWIZZLE_128B): 64 rows x 8 k per 1024-byte atom, the 16-byte
//     chunk of rows [8c, 8c+8) at k-row r stored at chunk c ^ (r % 8);
//     atoms: M direction at a_lbo bytes, 8-k groups at a_sbo bytes.
//   B (K-major, SWIZZLE_128B): 8 rows x 64 k per 1024-byte atom, chunk
//     (k % 64) / 8 of row r stored at chunk ((k % 64) / 8) ^ (r % 8);
//     8-row groups at 1024 bytes, 64-k slabs at b_slab bytes.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace nexd_dev {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (SWIZZLE_128B, version 1, base offset 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3FFF);
  d |= uint64_t((lbo >> 4) & 0x3FFF) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFF) << 32;
  d |= uint64_t(1) << 46;  // descriptor version
  d |= uint64_t(2) << 61;  // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::f16: bf16 x bf16 -> f32, A MN-major, B K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4)                   // D format f32
         | (1u << 7)                 // A bf16
         | (1u << 10)                // B bf16
         | (1u << 15)                // A MN-major
         | (0u << 16)                // B K-major
         | (uint32_t(N >> 3) << 17)  // N / 8
         | (uint32_t(M >> 4) << 24); // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrives on the mbarrier once every tcgen05 operation issued so far by this
// thread has completed.
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(done)
      : "r"(mbar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the given phase parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit = 1u << 22) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(mbar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Executed by one full warp.
__device__ __forceinline__ void tmem_alloc(uint32_t slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive accumulator columns of this thread's lane (32x32b shape).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
// 16 consecutive accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// x = hi + lo with hi = bf16(x), lo = bf16(x - hi); packed pairs.
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// x = h + m + l, each bf16 (the remainders are exact in FP32), packed pairs.
__device__ __forceinline__ void split3(float x0, float x1, uint32_t& h, uint32_t& m, uint32_t& l) {
  const __nv_bfloat162 bh = __floats2bfloat162_rn(x0, x1);
  const float2 fh = __bfloat1622float2(bh);
  const float r0 = x0 - fh.x, r1 = x1 - fh.y;
  const __nv_bfloat162 bm = __floats2bfloat162_rn(r0, r1);
  const float2 fm = __bfloat1622float2(bm);
  const __nv_bfloat162 bl = __floats2bfloat162_rn(r0 - fm.x, r1 - fm.y);
  h = *reinterpret_cast<const uint32_t*>(&bh);
  m = *reinterpret_cast<const uint32_t*>(&bm);
  l = *reinterpret_cast<const uint32_t*>(&bl);
}

// Byte offset of the 16-byte chunk holding rows [m8, m8+8) (m8 % 8 == 0) at
// k-row k of an MN-major SWIZZLE_128B operand.
__device__ __forceinline__ uint32_t a_chunk_offset(int m8, int k, uint32_t a_lbo, uint32_t a_sbo) {
  const int r = k & 7;
  const int c = (m8 >> 3) & 7;
  return uint32_t(k >> 3) * a_sbo + uint32_t(m8 >> 6) * a_lbo + uint32_t(r) * 128u + uint32_t((c ^ r) << 4);
}

// Stores 16 values of rows [m16, m16+16) at k-row k as hi and lo parts.
__device__ __forceinline__ void store_a16(unsigned char* a_hi, unsigned char* a_lo, int m16, int k, const float* v,
                                          uint32_t a_lbo, uint32_t a_sbo) {
  uint4 h0, h1, l0, l1;
  split2(v[0], v[1], h0.x, l0.x);
  split2(v[2], v[3], h0.y, l0.y);
  split2(v[4], v[5], h0.z, l0.z);
  split2(v[6], v[7], h0.w, l0.w);
  split2(v[8], v[9], h1.x, l1.x);
  split2(v[10], v[11], h1.y, l1.y);
  split2(v[12], v[13], h1.z, l1.z);
  split2(v[14], v[15], h1.w, l1.w);
  const uint32_t o0 = a_chunk_offset(m16, k, a_lbo, a_sbo), o1 = a_chunk_offset(m16 + 8, k, a_lbo, a_sbo);
  *reinterpret_cast<uint4*>(a_hi + o0) = h0;
  *reinterpret_cast<uint4*>(a_hi + o1) = h1;
  *reinterpret_cast<uint4*>(a_lo + o0) = l0;
  *reinterpret_cast<uint4*>(a_lo + o1) = l1;
}

// Stores 16 values of rows [m16, m16+16) at k-row k as h, m and l parts
// (three operands of the same layout, `stride` bytes apart).
__device__ __forceinline__ void store_a16x3(unsigned char* a, uint32_t stride, int m16, int k, const float* v,
                                            uint32_t a_lbo, uint32_t a_sbo) {
  uint4 h0, h1, m0, m1, l0, l1;
  split3(v[0], v[1], h0.x, m0.x, l0.x);
  split3(v[2], v[3], h0.y, m0.y, l0.y);
  split3(v[4], v[5], h0.z, m0.z, l0.z);
  split3(v[6], v[7], h0.w, m0.w, l0.w);
  split3(v[8], v[9], h1.x, m1.x, l1.x);
  split3(v[10], v[11], h1.y, m1.y, l1.y);
  split3(v[12], v[13], h1.z, m1.z, l1.z);
  split3(v[14], v[15], h1.w, m1.w, l1.w);
  const uint32_t o0 = a_chunk_offset(m16, k, a_lbo, a_sbo), o1 = a_chunk_offset(m16 + 8, k, a_lbo, a_sbo);
  *reinterpret_cast<uint4*>(a + o0) = h0;
  *reinterpret_cast<uint4*>(a + o1) = h1;
  *reinterpret_cast<uint4*>(a + stride + o0) = m0;
  *reinterpret_cast<uint4*>(a + stride + o1) = m1;
  *reinterpret_cast<uint4*>(a + 2 * stride + o0) = l0;
  *reinterpret_cast<uint4*>(a + 2 * stride + o1) = l1;
}

}  // namespace tc
}  // namespace nexd_dev
