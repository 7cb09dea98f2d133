// The learned boundary's network on the tensor cores (sm_100a): the ghost
// states of 128 absorbing faces per tile, with the three dense layers as
// tcgen05 MMAs (BF16 weights, FP32 accumulation in tensor memory).
//
// Per face: features (face_features, boundary_mlp.cuh) -> RMS scale ->
// n_in -> 128 -> 128 -> n_in with GELU -> clamped incoming characteristics
// -> ghost traction.  Faces are the MMA rows (TMEM lanes); the activations
// are split into two BF16 parts (h + l, 16 significant bits), the weights
// are the network's BF16 values, and the products accumulate in FP32.
//
// Shared memory (every part 1024-byte aligned, K-major, 128-byte swizzle,
// 64 k per slab): the weight images W1 [128 x kin], W2 [128 x 128], W3
// [kin x 128] (staged once per CTA from an image packed once per network),
// and the activation operand A in h and l parts [128 x max(kin, 128)].
#pragma once
#include "boundary_mlp.cuh"
#include "mlp_tc.cuh"

namespace nexd_dev {

struct GhostTcLayout {
  int nin, kin;                  // input width, padded to a multiple of 16
  uint32_t w1, w2, w3, a_part;   // bytes of each image and of one activation part
  uint32_t slab1, slab3;         // bytes per 64-k slab of W1 (128 rows) and W3 (kin rows)
  __host__ __device__ static GhostTcLayout of(int nin) {
    GhostTcLayout L;
    L.nin = nin;
    L.kin = (nin + 15) / 16 * 16;
    const int s1 = (L.kin + 63) / 64;
    L.slab1 = tcg_part_bytes(128);
    L.slab3 = tcg_part_bytes(L.kin);
    L.w1 = uint32_t(s1) * L.slab1;
    L.w2 = 2u * tcg_part_bytes(128);
    L.w3 = 2u * L.slab3;
    L.a_part = uint32_t(s1 > 2 ? s1 : 2) * tcg_part_bytes(128);
    return L;
  }
  __host__ __device__ uint32_t weights() const { return w1 + w2 + w3; }
  __host__ __device__ size_t smem() const { return 1024 + size_t(weights()) + 2 * size_t(a_part) + 512 + 64; }
};

// Byte offset of element k of row r in a K-major image whose 64-k slabs are
// `slab` bytes apart.
__device__ __forceinline__ uint32_t kmajor_elem(int r, int k, uint32_t slab) {
  return uint32_t(k >> 6) * slab + kmajor_offset(r, (k & 63) >> 3) + uint32_t(k & 7) * 2;
}

// The weight images from the BF16 parameters [W1 (H x nin), b1, W2 (H x H),
// b2, W3 (nin x H), b3], zero in the padding.
__global__ void pack_ghost_weights_kernel(int nin, const __nv_bfloat16* __restrict__ w, unsigned char* img) {
  const GhostTcLayout L = GhostTcLayout::of(nin);
  const int H = kMlpHidden;
  const __nv_bfloat16* W1 = w;
  const __nv_bfloat16* W2 = W1 + (long long)H * nin + H;
  const __nv_bfloat16* W3 = W2 + (long long)H * H + H;
  const int n1 = H * L.kin, n2 = H * H, n3 = L.kin * H;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1 + n2 + n3; i += gridDim.x * blockDim.x) {
    if (i < n1) {
      const int r = i / L.kin, k = i - r * L.kin;
      *reinterpret_cast<__nv_bfloat16*>(img + kmajor_elem(r, k, L.slab1)) = k < nin ? W1[(long long)r * nin + k] : zero;
    } else if (i < n1 + n2) {
      const int j = i - n1, r = j / H, k = j - r * H;
      *reinterpret_cast<__nv_bfloat16*>(img + L.w1 + kmajor_elem(r, k, tcg_part_bytes(128))) = W2[(long long)r * H + k];
    } else {
      const int j = i - n1 - n2, r = j / H, k = j - r * H;
      *reinterpret_cast<__nv_bfloat16*>(img + L.w1 + L.w2 + kmajor_elem(r, k, L.slab3)) =
          r < nin ? W3[(long long)r * H + k] : zero;
    }
  }
}

struct GhostTcArgs {
  GhostArgs g;                 // faces, wavefield, parameters and ghost output
  const uint4* wimg;           // weight images (pack_ghost_weights_kernel)
  int* flag;                   // error bit 2: an MMA completion wait ran out
};

// One 8-value chunk kc of row m of the activation operand as h and l parts.
__device__ __forceinline__ void store_act8(unsigned char* ah, unsigned char* al, int m, int kc, const float* v) {
  uint4 h, l;
  tc::split2(v[0], v[1], h.x, l.x);
  tc::split2(v[2], v[3], h.y, l.y);
  tc::split2(v[4], v[5], h.z, l.z);
  tc::split2(v[6], v[7], h.w, l.w);
  const uint32_t o = uint32_t(kc >> 3) * tcg_part_bytes(128) + kmajor_offset(m, kc & 7);
  *reinterpret_cast<uint4*>(ah + o) = h;
  *reinterpret_cast<uint4*>(al + o) = l;
}

// One value at (row m, k) of the activation operand as h and l parts.
__device__ __forceinline__ void store_act1(unsigned char* ah, unsigned char* al, int m, int k, float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
  const uint32_t o = kmajor_elem(m, k, tcg_part_bytes(128));
  *reinterpret_cast<__nv_bfloat16*>(ah + o) = h;
  *reinterpret_cast<__nv_bfloat16*>(al + o) = l;
}

constexpr int kGhostTcThreads = 256;

// One accumulator column of this thread's lane.
__device__ __forceinline__ float tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
  return __uint_as_float(r);
}

// 256 threads: warps w and w + 4 share TMEM lanes 32 (w % 4) .. + 31, so
// thread (row, half) owns face `row` of the tile and half of its nodes (the
// features, and the outputs at the end) or half of the hidden columns.  The
// face's element record stays in registers, and so do the outgoing values of
// its nodes, which the output clamp needs.  Layer 1 runs on the unscaled
// features and its epilogue applies the RMS scale 1/r (the layer is linear).
template <int NPF>
__global__ void __launch_bounds__(kGhostTcThreads, 1) ghost_tc_kernel(const GhostTcArgs t) {
  constexpr int NIN = 9 * NPF, H = kMlpHidden, NPH = (NPF + 1) / 2;
  const GhostArgs& a = t.g;
  const GhostTcLayout L = GhostTcLayout::of(NIN);
  extern __shared__ __align__(16) unsigned char gt_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(gt_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sW = base;
  unsigned char* sAh = base + L.weights();
  unsigned char* sAl = sAh + L.a_part;
  float* sR = reinterpret_cast<float*>(sAl + L.a_part);  // [128] sum of squares, then the RMS scale
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sR + 128);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int row = (warp & 3) * 32 + (tid & 31), half = warp >> 2;
  const int fi0 = half ? NPH : 0, cnt = half ? NPF - NPH : NPH;  // this thread's face nodes
  const int total = a.nbf * a.nbatch, ntile = (total + 127) / 128;
  if (int(blockIdx.x) >= ntile) return;
  for (int i = tid; i < int(L.weights() / 16); i += kGhostTcThreads) reinterpret_cast<uint4*>(sW)[i] = t.wimg[i];
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tslot), 256);
  if (tid == 0) tc::mbar_init(tc::smem_u32(mbar), 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t lane = tmem + (uint32_t((warp & 3) * 32) << 16);
  const uint32_t w1 = tc::smem_u32(sW), w2 = w1 + L.w1, w3 = w2 + L.w2;
  const uint32_t ah = tc::smem_u32(sAh), al = tc::smem_u32(sAl);
  const __nv_bfloat16* bias1 = a.w + (long long)H * NIN;
  const __nv_bfloat16* bias2 = bias1 + H + (long long)H * H;
  const __nv_bfloat16* bias3 = bias2 + H + (long long)NIN * H;
  uint32_t phase = 0;
  bool ok = true;

  // D = A W^T over K = 16 ksteps; A in two parts, W one image
  auto layer = [&](uint32_t wimg, uint32_t wslab, int ksteps, int nout) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t id = idesc_bf16_kk(128, nout);
      for (int k = 0; k < ksteps; ++k) {
        const uint32_t so = uint32_t(k >> 2) * tcg_part_bytes(128) + uint32_t(k & 3) * 32;
        const uint64_t bd = tc::smem_desc(wimg + uint32_t(k >> 2) * wslab + uint32_t(k & 3) * 32, 16, 1024);
        tc::mma_bf16(tmem, tc::smem_desc(ah + so, 16, 1024), bd, id, k > 0 ? 1u : 0u);
        tc::mma_bf16(tmem, tc::smem_desc(al + so, 16, 1024), bd, id, 1u);
      }
      tc::mma_commit(tc::smem_u32(mbar));
    }
    if (!tc::mbar_wait(tc::smem_u32(mbar), phase)) {
      ok = false;
      tc::mbar_wait(tc::smem_u32(mbar), phase, 1u << 24);
    }
    phase ^= 1u;
    tc::fence_after_sync();
  };
  // hidden layer epilogue of this thread's 64 columns: GELU(scale D + b) as
  // the next layer's operand
  auto hidden = [&](const __nv_bfloat16* bias, float scale) {
#pragma unroll
    for (int h2 = 0; h2 < 2; ++h2) {
      const int c0 = half * 64 + h2 * 32;
      float v[32];
      tc::tmem_ld32(lane + c0, v);
      tc::tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = gelu(fmaf(v[j], scale, __bfloat162float(bias[c0 + j])));
#pragma unroll
      for (int q = 0; q < 4; ++q) store_act8(sAh, sAl, row, (c0 >> 3) + q, v + 8 * q);
    }
  };

  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    if (tid < 128) sR[tid] = 0.f;
    // this thread's face and its element record
    const int gi = tile * 128 + row;
    const bool valid = gi < total;
    int b = 0, g = 0, e = 0, f = 0;
    if (valid) {
      b = gi / a.nbf;
      g = gi - b * a.nbf;
      e = a.bf_elem[g];
      f = a.bf_face[g];
    }
    const float* geo = a.geo + (long long)e * GEO_STRIDE;
    float fn[3], fs[3], ft[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      fn[k] = geo[G_N + 3 * f + k];
      fs[k] = geo[G_S + 3 * f + k];
      ft[k] = geo[G_T + 3 * f + k];
    }
    const float izp = geo[G_IZP], kz = izp / geo[G_IZS];
    const float* qb = a.q + (long long)b * 9 * a.ldq + (long long)e * a.Np;
    const unsigned char* pat = a.pat + f * NPF + fi0;
    __syncthreads();  // sR cleared
    // features of this thread's nodes: unscaled into the operand, squares
    // summed per face, outgoing values kept
    float u[NPH][3];
    float ss = 0.f;
#pragma unroll
    for (int i = 0; i < NPH; ++i) {
      float x[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (i < cnt && valid) {
        const float* qn = qb + pat[i];
        float q[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) q[c] = qn[c * a.ldq];
        face_features(q, fn, fs, ft, izp, kz, x);
#pragma unroll
        for (int c = 0; c < 9; ++c) ss += x[c] * x[c];
      }
      u[i][0] = x[3];
      u[i][1] = x[4];
      u[i][2] = x[5];
      if (i < cnt) {
#pragma unroll
        for (int c = 0; c < 9; ++c) store_act1(sAh, sAl, row, 9 * (fi0 + i) + c, x[c]);
      }
    }
    atomicAdd(&sR[row], ss);
    for (int i = tid; i < 128 * (L.kin - NIN); i += kGhostTcThreads)
      store_act1(sAh, sAl, i & 127, NIN + (i >> 7), 0.f);
    __syncthreads();
    if (tid < 128) sR[tid] = sqrtf(sR[tid] / NIN);
    layer(w1, L.slab1, L.kin / 16, H);  // its barrier also publishes sR
    const float r = sR[row];
    hidden(bias1, r > 0.f ? 1.f / r : 0.f);
    layer(w2, tcg_part_bytes(128), H / 16, H);
    hidden(bias2, 1.f);
    layer(w3, L.slab3, H / 16, L.kin);
    // outputs of this thread's nodes: incoming values of the prediction,
    // clamped by the trace's outgoing values, as ghost traction (zero velocity)
    const float zr = r / izp, ir = r > 0.f ? 1.f / r : 0.f;
#pragma unroll
    for (int i = 0; i < NPH; ++i) {
      if (i >= cnt) continue;  // the same in the whole warp
      const int fi = fi0 + i;
      float y[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) y[k] = tmem_ld1(lane + uint32_t(9 * fi + k));
      tc::tmem_wait_ld();
      if (!valid) continue;
      float w[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float bnd = a.rho_max * fabsf(u[i][k] * ir);
        w[k] = zr * fminf(fmaxf(y[k] + __bfloat162float(bias3[9 * fi + k]), -bnd), bnd);
      }
      auto comp = [&](int p, int q2) {
        return w[0] * fn[p] * fn[q2] + w[1] * (fn[p] * fs[q2] + fs[p] * fn[q2]) + w[2] * (fn[p] * ft[q2] + ft[p] * fn[q2]);
      };
      float* out = a.ghost + ((long long)b * a.nbf + g) * 9 * NPF + fi;
      out[0 * NPF] = comp(0, 0);
      out[1 * NPF] = comp(1, 1);
      out[2 * NPF] = comp(2, 2);
      out[3 * NPF] = comp(0, 1);
      out[4 * NPF] = comp(1, 2);
      out[5 * NPF] = comp(0, 2);
      out[6 * NPF] = 0.f;
      out[7 * NPF] = 0.f;
      out[8 * NPF] = 0.f;
    }
    tc::fence_before_sync();
    __syncthreads();  // TMEM, the operand and sR are free for the next tile
    tc::fence_after_sync();
  }
  if (!__syncthreads_and(ok ? 1 : 0) && tid == 0) atomicOr(t.flag, 2);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

}  // namespace nexd_dev
