// Fused per-stage kernel of the nodal-DG velocity-stress solver (sm_100a).
//
// One launch evaluates, for a contiguous range of elements, everything the
// reference's element loop does in one RK stage (src/timeloopMod.f90:395-476)
// and the stage update of RungeKuttaSteps (src/rungekuttaMod.f90:27-88):
//   volume term     rq = Dx F + Dy G + Dz H   (F,G,H = elasticFluxes, src/waveMod.f90:29-63)
//   face term       rq += LIFT (fscale/2 * T (A+|A|) T^-1 dq)   (computeExactRiemannSF,
//                   src/waveMod.f90:269-336; LIFT src/liftMod.f90:28-76)
//   Zener terms     a_rq and the stress coupling (src/timeloopMod.f90:426-461)
//   NPML            F <- (F'+F)/kappa and the F' equation (src/timeloopMod.f90:399-405,
//                   src/rungekuttaMod.f90:52-63)
//   point sources   (src/timeloopMod.f90:467-475)
//   stage update    LSERK4 2N-storage, or the reference's TVD Euler/RK2/RK3.
//
// Design:
//  * persistent blocks: Dr/Ds/Dt and LIFT are staged in shared memory once per
//    block, then the block walks chunks of E elements (E*Np <= 256 threads);
//  * the wavefield is field-major [9][nodes] (the layout of q(nglob,9)); the
//    kernel reads q_in (own nodes + neighbour face traces) and writes q_out, so
//    neighbours never see a half-updated stage (ping-pong buffers);
//  * affine elements: the volume term differentiates the 9 fields once (27
//    Np x Np matvecs) and applies the element-constant metric and material;
//  * the upwind flux T (A+|A|) T^-1 has rank 3 (one P and two S
//    characteristics), so each face node contributes three amplitudes; LIFT is
//    applied to the amplitudes, which are expanded to the 9 fields from the
//    face frame (n, s, t), and the same lifted amplitudes give the anelastic
//    flux;
//  * NPML elements (grouped first in the internal element order) are handled
//    by the PML instantiation, which differentiates the 27 modified flux
//    columns through their contravariant components (Dr Fr + Ds Fs + Dt Ft).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nexd_dev {

// Sizes of one order.  NPT nodes per thread: 1 (a thread per node, E =
// 256 / Np elements per chunk) or 2 (a thread per node pair, twice the
// elements per chunk).
template <int N, int NPT = 1>
struct Order {
  static constexpr int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  static constexpr int NpF = (N + 1) * (N + 2) / 2;
  static constexpr int NF = 4 * NpF;
  static constexpr int THREADS = 256;
  static constexpr int NPP = (Np + NPT - 1) / NPT;    // threads per element
  static constexpr int E = NPT * (THREADS / Np);     // elements per chunk
  static constexpr int QS = 12;           // padded field stride of staged q (3 x float4)
  static constexpr int CS = 34;           // contravariant-flux row stride (PML): r 0..9, s 10..19, t 20..29
  // shared-memory section sizes in floats, each a multiple of 4 (float4 alignment)
  static constexpr int r4(int x) { return (x + 3) / 4 * 4; }
  static constexpr int SD = r4(3 * Np * Np);  // Dr, Ds, Dt (each kernel stages its own layout)
  static constexpr int NPAIR = (NpF + 1) / 2;  // face-node pairs per face (last one zero-padded when NpF is odd)
  static constexpr int NFP = 4 * 2 * NPAIR;     // padded face nodes per element
  static constexpr int SL = 4 * NPAIR * Np * 2; // LIFT as [face][pair][n][2]
  // one prefetch buffer: element records, own wavefield (field-major), the
  // neighbour face traces and the connectivity of the following chunk
  // element records at a 68-word stride: the same field of different
  // elements in one warp falls on different banks (a 64-word stride puts it
  // on one bank)
  static constexpr int GSTR = 68;
  static constexpr int SGEO = E * GSTR;
  // Own wavefield: one slot of QF floats per field holding the chunk's node
  // range [e0 Np, (e0 + ne) Np) widened to 16-byte boundaries (at most E Np
  // + 6 floats; none when Np is a multiple of 4), copied as QCH 16-byte
  // pieces per field; the chunk's first node sits at offset (e0 Np) mod 4.
  static constexpr int pow2ceil(int x) { return x <= 1 ? 1 : 2 * pow2ceil((x + 1) / 2); }
  static constexpr int QCH = pow2ceil((E * Np + (Np % 4 ? 6 : 0) + 3) / 4);
  static constexpr int QF = 4 * QCH;
  static constexpr int SQF = 9 * QF;
  static constexpr int STR = r4(E * NF * 9);
  static constexpr int SIDS = r4(E * 12);
  static constexpr int BUF = SGEO + SQF + STR + SIDS;
  // Warp-aligned node mapping (one node per thread, Np > 32): each of the
  // first E warps holds nodes 0..31 of one element and the remaining nodes of
  // all elements share the last warps, so no warp holds node n of one element
  // and node n+32 of another (the same bank of a Dr/Ds/Dt or LIFT row).
  static constexpr bool WARP_ALIGNED = NPT == 1 && Np > 32;
  // smallest x' >= x with x' = m (mod 32)
  static constexpr int at_bank(int x, int m) { return x + ((m - x % 32) + 32) % 32; }
  // Per-element strides of the work areas put the elements that share a warp
  // on different banks: = 16 (mod 32) words for two elements per warp; with
  // the warp-aligned mapping up to E elements share the last warp, and
  // strides of 4 (16-byte loads) or 2 (8-byte loads) words keep them apart.
  static constexpr int b16(int x) { return at_bank(x, 16); }
  static constexpr int QE = WARP_ALIGNED ? at_bank(Np * QS, 4) : b16(Np * QS);  // interleaved own wavefield
  static constexpr int CFE = WARP_ALIGNED ? at_bank(Np * CS, 2) : b16(Np * CS);  // contravariant fluxes (PML)
  static constexpr int AE = WARP_ALIGNED ? at_bank(3 * NFP, 2) : b16(3 * NFP);  // amplitudes per element
  static constexpr int SQI = E * QE;        // interleaved copy for the volume loop (non-PML)
  static constexpr int SAMP = r4(E * AE);   // amplitudes [e][comp][padded face node]
  static constexpr int SCF = r4(E * CFE);
  static constexpr int SPAT = r4(64 * NpF / 4 + 1);  // face patterns (bytes/4), up to 64 rows
  static constexpr int smem_floats(bool pml) {
    return SD + SL + 2 * BUF + (pml ? SCF : SQI) + SAMP + SPAT;
  }
};

// Per-element record, 64 floats.
enum GeoOffset {
  G_RX = 0, G_RY, G_RZ, G_SX, G_SY, G_SZ, G_TX, G_TY, G_TZ,
  G_FS = 9,    // fscale/2 of faces 0..3
  G_N = 13,    // outward normals (face*3 + c)
  G_S = 25,    // first tangent
  G_T = 37,    // second tangent
  G_E1 = 49,   // -(lambda+2mu)
  G_E2 = 50,   // -lambda
  G_E3 = 51,   // -mu
  G_E4 = 52,   // -1/rho
  G_VP = 53, G_VS = 54, G_L2M = 55, G_MU = 56, G_LAM = 57, G_IRHO = 58,
  G_C = 59,    // lambda/(lambda+2mu)
  G_IZP = 60,  // 1/(rho vp)
  G_IZS = 61,  // 1/(rho vs)
  G_AP = 62,   // 1/(lambda+2mu)
  G_AS = 63,   // 1/(2mu)
  GEO_STRIDE = 64
};

enum StageMode { MODE_LSERK = 0, MODE_TVD = 1 };

struct StageArgs {
  int e_begin, e_end;  // internal element range of this launch
  int nbatch;
  int nMB;
  long long ldq;       // field stride of q / res (nodes, padded)
  long long ldt;       // field stride of theta arrays
  long long lda;       // field stride of PML auxiliary arrays (PML nodes)
  const float* D;      // [3][Np][Np] as D[d][k][n]
  const float* L;      // [4][NPAIR][Np][2]: LIFT(n, face node) in face-node pairs
  const float* geo;    // [K][64]
  const int4* nbr;     // [K] internal neighbour per face, -1 on boundaries
  const int4* fcode;   // [K] per face: pattern id >= 0, -1 free, -2 absorbing
  const unsigned char* patterns;  // [npat][NpF] neighbour-local node of face node i
  int npat;
  const float* ael;    // [K][3*nMB]: -lam*Ylam, -2mu*Ymu, sum (src/timeloopMod.f90:274-282)
  const float* wl;     // [nMB]
  float wlv[3];        // the relaxation frequencies w_l as kernel parameters (nMB = 3)
  const float* prof;   // [Kpml][9][Np]: ddx ddy ddz ax ay az kx ky kz
  // state, batch member b at offset b*9*ldq (q/res), b*6*nMB*ldt (theta), b*27*lda (aux)
  const float* q_in;
  float* q_out;
  const float* q_n;    // TVD: step-start state (own nodes only)
  float* res;          // LSERK residual of q
  float* th;           // theta (in place)
  float* th2;          // LSERK: theta residual; TVD: step-start theta
  float* aux;          // PML F',G',H' (in place)
  float* aux2;         // LSERK: residual; TVD: step-start values
  float dt, ca, cb;    // LSERK: res = ca*res + dt*L, x += cb*res;  TVD: x = ca*xn + cb*(x + dt*L)
  int stage_first;     // TVD: first stage (stores the step-start theta/aux)
  // sources
  const int* src_head;   // [K] first source of the element or -1
  const int* src_next;   // [nsrc]
  const int* src_batch;  // [nsrc]
  const float* src_pat;  // [nsrc][9][Np]
  const float* stf;      // [nsrc][nt][nspt]
  int nt, nspt, stage;
  const int* it_dev;     // current step (1-based), kept on the device so a captured step replays
  // receivers
  const int* rec_slot;   // [K] slot of receiver elements or -1
  float* abuf;           // [nbatch][nslot][3][Np]: last-stage rq(7:9)
  int nslot;
  int last_stage;
  const int* pml_off;    // [nbatch] 1 once the STA/LTA trigger switched the NPML off
  int* flag;             // error bits: 1 non-finite trace (record kernel), 2 tensor-core wait timed out,
                         // 4 halo arrival wait ran out, 8 bulk-copy wait timed out
  const float* ghost;    // learned boundary: [nbatch][nbf][9][NpF] exterior states (face code -3 - index)
  int nbf;
};

// Jump q+ - q- at one face node for a face code: neighbour trace (>= 0),
// free surface (-1: own trace, flagged), absorbing (-2: exterior state zero)
// or learned absorbing (<= -3: exterior state from the ghost buffer).
template <int NpF>
__device__ __forceinline__ bool face_jump(const StageArgs& a, int b, int code, int fi, const float* tr, const float* qo,
                                          int qs, float* dq) {
  if (code >= 0) {
#pragma unroll
    for (int c = 0; c < 9; ++c) dq[c] = tr[c] - qo[c * qs];
    return false;
  }
  if (code == -1) {
#pragma unroll
    for (int c = 0; c < 9; ++c) dq[c] = qo[c * qs];
    return true;
  }
  if (code == -2) {
#pragma unroll
    for (int c = 0; c < 9; ++c) dq[c] = -qo[c * qs];
    return false;
  }
  const float* gh = a.ghost + ((long long)b * a.nbf + (-3 - code)) * 9 * NpF + fi;
#pragma unroll
  for (int c = 0; c < 9; ++c) dq[c] = gh[c * NpF] - qo[c * qs];
  return false;
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }

// Lifted upwind flux of face f expanded to the 9 fields and the anelastic
// stress flux, from the lifted amplitudes A0 (P), A1, A2 (S along s, t): the
// rank-3 form of T (A+|A|) T^-1 gives the stresses (Voigt xx yy zz xy yz xz)
// A0 [n n^T + c (s s^T + t t^T)] + A1 (n s^T + s n^T) + A2 (n t^T + t n^T),
// c = lambda/(lambda+2mu), evaluated with s s^T + t t^T = I - n n^T ((n, s, t)
// orthonormal) as n v^T + v n^T + c A0 I, v = (1-c)/2 A0 n + m,
// m = A1 s + A2 t; the velocities -(A0 n / Zp + m / Zs); the anelastic flux
// A0 n n^T / (lambda+2mu) + (n m^T + m n^T) / (2 mu) = n u^T + u n^T.
// Reads 9 words of the element record per face and accumulates into rq and
// sig_an.
template <bool ATT>
__device__ __forceinline__ void face_expand(const float* g, int f, float A0, float A1, float A2, float* rq,
                                            float* sig_an) {
  const float n0 = g[G_N + 3 * f], n1 = g[G_N + 3 * f + 1], n2 = g[G_N + 3 * f + 2];
  const float m0 = A1 * g[G_S + 3 * f] + A2 * g[G_T + 3 * f];
  const float m1 = A1 * g[G_S + 3 * f + 1] + A2 * g[G_T + 3 * f + 1];
  const float m2 = A1 * g[G_S + 3 * f + 2] + A2 * g[G_T + 3 * f + 2];
  const float c = g[G_C];
  const float h = 0.5f * (1.f - c) * A0, b = c * A0;
  const float v0 = fmaf(h, n0, m0), v1 = fmaf(h, n1, m1), v2 = fmaf(h, n2, m2);
  rq[0] += fmaf(2.f * n0, v0, b);
  rq[1] += fmaf(2.f * n1, v1, b);
  rq[2] += fmaf(2.f * n2, v2, b);
  rq[3] += n0 * v1 + v0 * n1;
  rq[4] += n1 * v2 + v1 * n2;
  rq[5] += n0 * v2 + v0 * n2;
  const float p = g[G_IZP] * A0, q = g[G_IZS];
  rq[6] -= fmaf(p, n0, q * m0);
  rq[7] -= fmaf(p, n1, q * m1);
  rq[8] -= fmaf(p, n2, q * m2);
  if (ATT) {
    const float ha = 0.5f * g[G_AP] * A0, as = g[G_AS];
    const float u0 = fmaf(ha, n0, as * m0), u1 = fmaf(ha, n1, as * m1), u2 = fmaf(ha, n2, as * m2);
    sig_an[0] += 2.f * n0 * u0;
    sig_an[1] += 2.f * n1 * u1;
    sig_an[2] += 2.f * n2 * u2;
    sig_an[3] += n0 * u1 + u0 * n1;
    sig_an[4] += n1 * u2 + u1 * n2;
    sig_an[5] += n0 * u2 + u0 * n2;
  }
}

// Characteristic amplitudes (a_p, a_s1, a_s2) of the upwind flux at one face
// node, given the jump dq (interior: q+ - q-, absorbing: -q-) or, for a free
// surface, the own trace.
__device__ __forceinline__ void face_amplitudes(const float* g, int f, const float* dq, bool free_face,
                                                float& ap, float& as1, float& as2) {
  const float nx = g[G_N + 3 * f], ny = g[G_N + 3 * f + 1], nz = g[G_N + 3 * f + 2];
  const float sx = g[G_S + 3 * f], sy = g[G_S + 3 * f + 1], sz = g[G_S + 3 * f + 2];
  const float tx = g[G_T + 3 * f], ty = g[G_T + 3 * f + 1], tz = g[G_T + 3 * f + 2];
  // traction of the stress jump
  const float tau_x = dq[0] * nx + dq[3] * ny + dq[5] * nz;
  const float tau_y = dq[3] * nx + dq[1] * ny + dq[4] * nz;
  const float tau_z = dq[5] * nx + dq[4] * ny + dq[2] * nz;
  const float snn = tau_x * nx + tau_y * ny + tau_z * nz;
  const float sns = tau_x * sx + tau_y * sy + tau_z * sz;
  const float snt = tau_x * tx + tau_y * ty + tau_z * tz;
  if (free_face) {
    // APA * diag(-2,0,0,-2,0,-2,0,0,0) (src/timeloopMod.f90:207-216, 269)
    ap = -2.f * g[G_VP] * snn;
    as1 = -2.f * g[G_VS] * sns;
    as2 = -2.f * g[G_VS] * snt;
  } else {
    const float vn = dq[6] * nx + dq[7] * ny + dq[8] * nz;
    const float vs_ = dq[6] * sx + dq[7] * sy + dq[8] * sz;
    const float vt = dq[6] * tx + dq[7] * ty + dq[8] * tz;
    ap = g[G_VP] * snn - g[G_L2M] * vn;
    as1 = g[G_VS] * sns - g[G_MU] * vs_;
    as2 = g[G_VS] * snt - g[G_MU] * vt;
  }
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// 16 bytes through L1 (.ca): tetrahedra of one hexahedron sit next to each
// other in the element order, so many neighbour face traces of a chunk are
// nodes of the same chunk and hit the lines its own-wavefield copies brought in
__device__ __forceinline__ void cp_async16_ca(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Work item w of a launch: batch member and first element of the chunk.
struct Chunk {
  int b, e0, ne;
};
template <int E>
__device__ __forceinline__ Chunk chunk_of(const StageArgs& a, int w, int nchunk) {
  Chunk c;
  c.b = w / nchunk;
  c.e0 = a.e_begin + (w - c.b * nchunk) * E;
  c.ne = min(E, a.e_end - c.e0);
  return c;
}

// Asynchronous copies of one chunk's element records (16-byte copies), own
// wavefield (field-major), the connectivity of the chunk after it (`next`,
// -1 for none) and the chunk's own face codes, shared by threads
// t0 .. t0 + nt - 1 (default: the whole block).  No commit.
template <class O>
__device__ __forceinline__ void issue_main(const StageArgs& a, const Chunk& c, float* bGeo, float* bQ, int* bIds,
                                           const Chunk* next, int t0 = -1, int nt = 0) {
  constexpr int Np = O::Np, E = O::E;
  const int tid = t0 < 0 ? int(threadIdx.x) : t0, nth = t0 < 0 ? int(blockDim.x) : nt;
  const float* qin = a.q_in + (long long)c.b * 9 * a.ldq;
  for (int i = tid; i < c.ne * (GEO_STRIDE / 4); i += nth)
    cp_async16(bGeo + (i / (GEO_STRIDE / 4)) * O::GSTR + 4 * (i % (GEO_STRIDE / 4)),
               a.geo + (long long)c.e0 * GEO_STRIDE + 4 * i);
  // per field the 16-byte pieces of [base, base + cnt) widened to 16-byte
  // boundaries; in bounds: the field stride ldq is a multiple of 64 nodes
  const long long base = (long long)c.e0 * Np;
  const long long s0 = base & ~3LL;
  const int npiece = int((base + c.ne * Np + 3 - s0) >> 2);
  for (int i = tid; i < 9 * O::QCH; i += nth) {
    const int f = i / O::QCH, j = i - f * O::QCH;
    if (j < npiece) cp_async16_ca(bQ + f * O::QF + 4 * j, qin + f * a.ldq + s0 + 4 * j);
  }
  if (next)
    for (int i = tid; i < next->ne * 2; i += nth) {
      const int ee = i >> 1;
      const int4* src = (i & 1) ? a.fcode + next->e0 + ee : a.nbr + next->e0 + ee;
      cp_async16(bIds + ee * 12 + (i & 1) * 4, src);
    }
  for (int i = tid; i < c.ne; i += nth) cp_async16(bIds + i * 12 + 8, a.fcode + c.e0 + i);
}

// Asynchronous gather of the neighbour face traces of one chunk's interior
// faces through the face patterns, using its connectivity `ids` (staged one
// chunk earlier): face nodes [lo, hi) of the chunk (hi < 0: all), shared by
// threads t0 .. t0 + nt - 1 (default: the whole block).  No commit.
template <class O>
__device__ __forceinline__ void issue_traces(const StageArgs& a, const Chunk& c, const int* ids, float* bTr,
                                             const unsigned char* pat, int lo = 0, int hi = -1, int t0 = -1,
                                             int nt = 0) {
  constexpr int Np = O::Np, NpF = O::NpF, NF = O::NF;
  const int tid = t0 < 0 ? int(threadIdx.x) : t0, nth = t0 < 0 ? int(blockDim.x) : nt;
  const float* qin = a.q_in + (long long)c.b * 9 * a.ldq;
  const int end = hi < 0 ? c.ne * NF : hi;
  for (int i = lo + tid; i < end; i += nth) {
    const int ee = i / NF, j = i - ee * NF;
    const int f = j / NpF, fi = j - f * NpF;
    const int code = ids[ee * 12 + 4 + f];
    if (code >= 0) {
      const int nb = ids[ee * 12 + f];
      const long long gn = (long long)nb * Np + pat[code * NpF + fi];
      float* dst = bTr + i * 9;
#pragma unroll
      for (int k = 0; k < 9; ++k) cp_async4(dst + k, qin + k * a.ldq + gn);
    }
  }
}

// All copies of one chunk into a prefetch buffer [records | wavefield |
// traces | connectivity], committed as one group.
template <class O>
__device__ __forceinline__ void issue_chunk(const StageArgs& a, const Chunk& c, const int* ids, float* buf,
                                            const Chunk* next, const unsigned char* pat) {
  float* bGeo = buf;
  float* bQ = bGeo + O::SGEO;
  float* bTr = bQ + O::SQF;
  int* bIds = reinterpret_cast<int*>(bTr + O::STR);
  issue_main<O>(a, c, bGeo, bQ, bIds, next);
  issue_traces<O>(a, c, ids, bTr, pat);
  cp_async_commit();
}

// Memory variables per mechanism set: the reference's nMB = 3 (src/constants.h:36).
constexpr int kNMB = 3;

// Element-local state (LSERK residual of q, memory variables and their
// residuals, NPML auxiliaries and their residuals) is element-blocked: field f
// of node n of element e of batch member b sits at
//   b F ld + e FS + f Np + n,   FS = F Np rounded up to a multiple of 4,
// so every field of a node is a compile-time offset from one address, and
// every element's block starts on a 16-byte boundary (so a chunk's block
// range can be moved by 1-D bulk copies).  ld is the per-field length (F ld
// >= elements x FS), F ld the batch stride.
template <int F, int Np>
struct EBlock {
  static constexpr int FS = (F * Np + 3) / 4 * 4;
};
template <int F, int Np>
__device__ __forceinline__ long long eblock(long long ld, int b, int e, int n) {
  return (long long)b * F * ld + (long long)e * EBlock<F, Np>::FS + n;
}

// Update-phase state of one node, loaded into registers when the chunk starts
// so the loads are in flight while the face, volume and lift terms run.  With
// EARLY the per-element scalars of the tail (Zener coefficients, first
// source, receiver slot, NPML switch) are prefetched too (kernels with one
// block per SM, where their latency is not hidden); otherwise they are read
// where they are used (kernels whose register budget is tight).
template <bool ATT, bool PML, int MODE, bool EARLY = false>
struct NodePrefetch {
  static constexpr int NTH = ATT ? 6 * kNMB : 1;
  static constexpr int NAX = PML ? 27 : 1;
  float res[9], th[NTH], th2[NTH], ax[NAX], ax2[NAX], pr[PML ? 9 : 1];
  float ae[(ATT && EARLY) ? 3 * kNMB : 1];  // per-element Zener coefficients
  int src, slot, pml_off;                   // first source of the element, receiver slot, NPML switched off

  __device__ __forceinline__ const float* zener(const StageArgs& a, int e) const {
    return EARLY ? ae : a.ael + (long long)e * 3 * kNMB;
  }
  __device__ __forceinline__ int first_source(const StageArgs& a, int e) const { return EARLY ? src : a.src_head[e]; }
  __device__ __forceinline__ int receiver_slot(const StageArgs& a, int e) const { return EARLY ? slot : a.rec_slot[e]; }
  __device__ __forceinline__ bool npml_off(const StageArgs& a, int b) const { return EARLY ? pml_off != 0 : a.pml_off[b] != 0; }

  template <int Np>
  __device__ __forceinline__ void load(const StageArgs& a, int b, int e, long long node) {
    const bool need2 = (MODE == MODE_LSERK) || !a.stage_first;
    if (EARLY) {
      src = __ldg(a.src_head + e);
      slot = a.last_stage ? __ldg(a.rec_slot + e) : -1;
      pml_off = PML ? a.pml_off[b] : 0;
      if (ATT) {
#pragma unroll
        for (int j = 0; j < 3 * kNMB; ++j) ae[j] = __ldg(a.ael + (long long)e * 3 * kNMB + j);
      }
    }
    const int n = int(node - (long long)e * Np);
    if (MODE == MODE_LSERK) {
      const float* rs = a.res + eblock<9, Np>(a.ldq, b, e, n);
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
    if (ATT) {
      const float* t = a.th + eblock<6 * kNMB, Np>(a.ldt, b, e, n);
      const float* t2 = a.th2 + eblock<6 * kNMB, Np>(a.ldt, b, e, n);
#pragma unroll
      for (int j = 0; j < NTH; ++j) th[j] = __ldcs(t + j * Np);
#pragma unroll
      for (int j = 0; j < NTH; ++j) th2[j] = need2 ? __ldcs(t2 + j * Np) : 0.f;
    }
    if (PML) {
      // PML elements come first internally, so element e is PML element e
      const float* x = a.aux + eblock<27, Np>(a.lda, b, e, n);
      const float* x2 = a.aux2 + eblock<27, Np>(a.lda, b, e, n);
      const float* p = a.prof + (long long)e * 9 * Np + n;
#pragma unroll
      for (int i = 0; i < 27; ++i) ax[i] = __ldcs(x + i * Np);
#pragma unroll
      for (int i = 0; i < 27; ++i) ax2[i] = need2 ? __ldcs(x2 + i * Np) : 0.f;
#pragma unroll
      for (int i = 0; i < 9; ++i) pr[i] = __ldg(p + i * Np);
    }
  }
};

// NPML auxiliary update of one node (src/timeloopMod.f90:399-405,
// src/rungekuttaMod.f90:52-63) and the fluxes the volume term differentiates:
// X, Y, Z = (F'+F)/kx, (G'+G)/ky, (H'+H)/kz, or F, G, H once the trigger
// switched the layer off.  F, G, H are overwritten.
// pr: the node's damping profiles, av / a2: its auxiliaries F', G', H' and
// their LSERK residuals (TVD: step-start values), as loaded for this stage.
template <int Np, int MODE>
__device__ __forceinline__ void pml_update(const StageArgs& a, int b, int e, int n, bool off, const float* pr,
                                           const float* av, const float* a2, float* F, float* G, float* H) {
  if (off) return;  // pmlcheck(:) = .false.: ordinary element (src/timeloopMod.f90:537)
  const float ddx = pr[0], ddy = pr[1], ddz = pr[2];
  const float alx = pr[3], aly = pr[4], alz = pr[5];
  const float ikx = 1.f / pr[6], iky = 1.f / pr[7], ikz = 1.f / pr[8];
  float* aux = a.aux + eblock<27, Np>(a.lda, b, e, n);
  float* aux2 = a.aux2 + eblock<27, Np>(a.lda, b, e, n);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const float fp = av[i], gp = av[9 + i], hp = av[18 + i];
    const float rf = -alx * fp - ddx * ikx * (fp + F[i]);
    const float rg = -aly * gp - ddy * iky * (gp + G[i]);
    const float rh = -alz * hp - ddz * ikz * (hp + H[i]);
    const float phi = (fp + F[i]) * ikx, psi = (gp + G[i]) * iky, ome = (hp + H[i]) * ikz;
    float nf, ng_, nh;
    if (MODE == MODE_LSERK) {
      const float r1 = a.ca * a2[i] + a.dt * rf;
      const float r2 = a.ca * a2[9 + i] + a.dt * rg;
      const float r3 = a.ca * a2[18 + i] + a.dt * rh;
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
        n1 = a2[i]; n2 = a2[9 + i]; n3 = a2[18 + i];
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

template <int Np, bool ATT, int MODE, bool EARLY>
__device__ __forceinline__ void pml_node(const StageArgs& a, int b, int e, int n,
                                         const NodePrefetch<ATT, true, MODE, EARLY>& p, float* F, float* G, float* H) {
  pml_update<Np, MODE>(a, b, e, n, p.npml_off(a, b), p.pr, p.ax, p.ax2, F, G, H);
}

// elasticFluxes (src/waveMod.f90:29-63) with e1..e4 = -(lambda+2mu), -lambda, -mu, -1/rho.
__device__ __forceinline__ void elastic_fluxes(const float* g, const float* qv, float* F, float* G, float* H) {
  const float e1 = g[G_E1], e2 = g[G_E2], e3 = g[G_E3], e4 = g[G_E4];
  F[0] = e1 * qv[6]; F[1] = e2 * qv[6]; F[2] = e2 * qv[6]; F[3] = e3 * qv[7]; F[4] = 0.f;
  F[5] = e3 * qv[8]; F[6] = e4 * qv[0]; F[7] = e4 * qv[3]; F[8] = e4 * qv[5];
  G[0] = e2 * qv[7]; G[1] = e1 * qv[7]; G[2] = e2 * qv[7]; G[3] = e3 * qv[6]; G[4] = e3 * qv[8];
  G[5] = 0.f; G[6] = e4 * qv[3]; G[7] = e4 * qv[1]; G[8] = e4 * qv[4];
  H[0] = e2 * qv[8]; H[1] = e2 * qv[8]; H[2] = e1 * qv[8]; H[3] = 0.f; H[4] = e3 * qv[7];
  H[5] = e3 * qv[6]; H[6] = e4 * qv[5]; H[7] = e4 * qv[4]; H[8] = e4 * qv[2];
}

// Everything after the spatial operator for one node: Zener memory variables
// (src/timeloopMod.f90:426-461) driven by S = lifted anelastic flux - strain
// rate, point sources (467-475), the receiver acceleration of the last stage,
// and the stage update of q.  rq holds the volume + surface term on entry.
template <int Np, bool ATT, bool PML, int MODE, bool EARLY>
__device__ __forceinline__ void finish_node(const StageArgs& a, int b, int e, long long node, float* rq, const float* S,
                                            const NodePrefetch<ATT, PML, MODE, EARLY>& p, const float* qown,
                                            int qstride) {
  const int n = int(node - (long long)e * Np);
  if (ATT) {
    float* th = a.th + eblock<6 * kNMB, Np>(a.ldt, b, e, n);
    float* th2 = a.th2 + eblock<6 * kNMB, Np>(a.ldt, b, e, n);
    const float* ae = p.zener(a, e);
#pragma unroll
    for (int l = 0; l < kNMB; ++l) {
      const float wl = a.wlv[l];
      const float* t = p.th + 6 * l;
      const float* t2 = p.th2 + 6 * l;
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
  for (int s = p.first_source(a, e); s >= 0; s = a.src_next[s]) {
    if (a.src_batch[s] != b) continue;
    const int sidx = a.nspt == 1 ? 0 : min(a.stage, a.nspt - 1);
    const float amp = a.stf[((long long)s * a.nt + (*a.it_dev - 1)) * a.nspt + sidx];
    const float* sp = a.src_pat + (long long)s * 9 * Np + n;
#pragma unroll
    for (int c = 0; c < 9; ++c) rq[c] = fmaf(sp[c * Np], amp, rq[c]);
  }
  if (a.last_stage) {
    const int slot = p.receiver_slot(a, e);
    if (slot >= 0) {
      float* ab = a.abuf + ((long long)b * a.nslot + slot) * 3 * Np + n;
      ab[0] = rq[6];
      ab[Np] = rq[7];
      ab[2 * Np] = rq[8];
    }
  }
  float* qo = a.q_out + (long long)b * 9 * a.ldq + node;
  if (MODE == MODE_LSERK) {
    float* rs = a.res + eblock<9, Np>(a.ldq, b, e, n);
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const float r = a.ca * p.res[c] + a.dt * rq[c];
      __stcs(rs + c * Np, r);
      __stcs(qo + c * a.ldq, qown[c * qstride] + a.cb * r);
    }
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const float base = (a.ca != 0.f) ? a.ca * p.res[c] : 0.f;
      __stcs(qo + c * a.ldq, base + a.cb * (qown[c * qstride] + a.dt * rq[c]));
    }
  }
}

// One block's share of a stage launch: the work items (wavefield, chunk)
// w0, w0 + wstep, ... of the launch's element range, with `smem` the block's
// dynamic shared memory (Order<N>::smem_floats(PML) floats).  stage_kernel
// runs it with w0 = blockIdx.x, wstep = gridDim.x; the multi-model kernel
// gives each block a share of one model's items.
template <int N, bool ATT, bool PML, int MODE>
__device__ __forceinline__ void stage_body(const StageArgs& a, int w0, int wstep, float* smem) {
  using O = Order<N>;
  constexpr int Np = O::Np, NpF = O::NpF, NF = O::NF, E = O::E, QS = O::QS, CS = O::CS;
  float* sD = smem;              // (Dr, Ds) pairs [k][n], then Dt [k][n]
  float* sL = sD + O::SD;        // LIFT in face-node pairs
  float* sBuf = sL + O::SL;      // 2 prefetch buffers
  float* sQI = sBuf + 2 * O::BUF;  // non-PML: interleaved own wavefield [e][k][QS]
  float* sCF = sQI;              // PML: contravariant modified fluxes [e][k][CS]
  float* sAmp = sQI + (PML ? O::SCF : O::SQI);  // E*3*NFP
  unsigned char* sPat = reinterpret_cast<unsigned char*>(sAmp + O::SAMP);  // face patterns

  const int tid = threadIdx.x;
  // Dr and Ds of a (k, node) as one 8-byte pair, then Dt
  for (int i = tid; i < Np * Np; i += blockDim.x) {
    reinterpret_cast<float2*>(sD)[i] = make_float2(a.D[i], a.D[Np * Np + i]);
    sD[2 * Np * Np + i] = a.D[2 * Np * Np + i];
  }
  for (int i = tid; i < O::SL; i += blockDim.x) sL[i] = a.L[i];
  if (NpF & 1)  // padding slots of the amplitude pairs stay zero
    for (int i = tid; i < E * 3 * 4; i += blockDim.x)
      sAmp[(i >> 2) / 3 * O::AE + (i >> 2) % 3 * O::NFP + (i & 3) * 2 * O::NPAIR + NpF] = 0.f;
  for (int i = tid; i < a.npat * NpF; i += blockDim.x) sPat[i] = a.patterns[i];

  const int nel = a.e_end - a.e_begin;
  const int nchunk = (nel + E - 1) / E;
  const int nwork = nchunk * a.nbatch;
  int le, n;  // element of this thread within the chunk, node of this thread
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
  int w = w0;
  if (w >= nwork) return;

  // prologue: connectivity of the first chunk straight from global memory
  {
    const Chunk c0 = chunk_of<E>(a, w, nchunk);
    const int wn = w + wstep;
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

  for (int p = 0; w < nwork; w += wstep, p ^= 1) {
    const Chunk ch = chunk_of<E>(a, w, nchunk);
    const int b = ch.b, e0 = ch.e0, ne = ch.ne;
    float* buf = sBuf + p * O::BUF;
    const float* sGeo = buf;
    const float* sTr = buf + O::SGEO + O::SQF;
    // own wavefield of the chunk: field c of node n of element le at sQF[c * QF + le * Np + n]
    const float* sQF = buf + O::SGEO + int(((long long)e0 * Np) & 3);
    const int* sIds = reinterpret_cast<const int*>(sTr + O::STR);  // connectivity of the next chunk
    cp_async_wait_all();
    __syncthreads();  // this chunk's data is in `buf`; the other buffer and work areas are free

    // ---- register prefetch of this node's update-phase state --------------------
    // (all loads of the chunk are in flight while the face, volume and lift
    // terms are computed; one block per SM keeps them in registers)
    const bool active = le < ne;
    const long long node = (long long)(e0 + (active ? le : 0)) * Np + n;
    NodePrefetch<ATT, PML, MODE> pf;
    if (active) pf.template load<Np>(a, b, e0 + le, node);
    // ---- start the next chunk's copies ------------------------------------------
    {
      const int wn = w + wstep;
      if (wn < nwork) {
        const Chunk cn = chunk_of<E>(a, wn, nchunk);
        const int wnn = wn + wstep;
        Chunk cnn;
        if (wnn < nwork) cnn = chunk_of<E>(a, wnn, nchunk);
        issue_chunk<O>(a, cn, sIds, sBuf + (p ^ 1) * O::BUF, wnn < nwork ? &cnn : nullptr, sPat);
      }
    }
    // ---- interleaved own wavefield for the volume loop ------------------------------
    if (!PML && active) {
      // two 16-byte stores and one 4-byte store: a 16-byte store of 8 threads
      // at a 12-word stride touches 32 different banks
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
      const int own = sPat[f * NpF + fi];  // patterns 0..3 are the element's own face masks
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

    // ---- PML: auxiliary update and contravariant modified fluxes ------------------
    float vgrad[9];  // d(v_c)/d(x_d) [c*3+d] (anelastic)
    (void)vgrad;
    if constexpr (PML) if (active) {
      const float* g = sGeo + le * O::GSTR;
      float qv[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) qv[c] = sQF[c * O::QF + le * Np + n];
      float F[9], G[9], H[9];
      elastic_fluxes(g, qv, F, G, H);
      pml_node<Np, ATT, MODE>(a, b, e0 + le, n, pf, F, G, H);
      // the row as 8-byte stores (pairs of fields; field 8 with the zero pad):
      // 16 threads at a 34-word stride touch 32 different banks
      float2* cf = reinterpret_cast<float2*>(sCF + le * O::CFE + n * CS);
      float r[10], sv[10], t[10];
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        r[i] = g[G_RX] * F[i] + g[G_RY] * G[i] + g[G_RZ] * H[i];
        sv[i] = g[G_SX] * F[i] + g[G_SY] * G[i] + g[G_SZ] * H[i];
        t[i] = g[G_TX] * F[i] + g[G_TY] * G[i] + g[G_TZ] * H[i];
      }
      // the pad slot of each row carries one velocity component (read with
      // field 8 of the row as one 8-byte load in the volume loop)
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
    __syncthreads();
    if (!active) continue;  // idle threads of a partial chunk (the next barrier is at the loop top)

    const int e = e0 + le;
    const float* g = sGeo + le * O::GSTR;
    float rq[9];
    // ---- volume term ------------------------------------------------------------
    if (!PML) {
      // d/dr, d/ds, d/dt of the 9 fields as packed pairs (fields 2j, 2j+1; pair 4 = field 8 + pad)
      // fields 0..7 as packed pairs, field 8 as scalars (its 4-byte load is one
      // shared-memory wavefront, a padded pair two)
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
#undef DX
#undef DY
#undef DZ
    } else {
#pragma unroll
      for (int c = 0; c < 9; ++c) rq[c] = 0.f;
      float2 acc[4];  // fields 0..7 in pairs; field 8 (its pair's second word is a velocity component)
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
        const float2 pr8 = cf[4], ps8 = cf[9], pt8 = cf[14];  // (field 8, velocity component)
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
    // ---- lift of the face amplitudes and expansion -------------------------------
    float sig_an[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) sig_an[c] = 0.f;
    (void)sig_an;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      float2 c0 = make_float2(0.f, 0.f), c1 = c0, c2 = c0;
      const float2* lp = reinterpret_cast<const float2*>(sL) + f * O::NPAIR * Np + n;
      const float* ax = sAmp + le * O::AE + f * 2 * O::NPAIR;
      // face-node pairs; with NpF odd the last face node alone (its pair's
      // second slot is zero padding), as 4-byte loads
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
    // ---- memory variables, sources, receivers, stage update ------------------------
    float S[6];
    if (ATT) {
      // S = -strain rate + lifted anelastic flux; d theta_l/dt = w_l (S - theta_l)
      S[0] = sig_an[0] - vgrad[0];
      S[1] = sig_an[1] - vgrad[4];
      S[2] = sig_an[2] - vgrad[8];
      S[3] = sig_an[3] - 0.5f * (vgrad[3] + vgrad[1]);
      S[4] = sig_an[4] - 0.5f * (vgrad[7] + vgrad[5]);
      S[5] = sig_an[5] - 0.5f * (vgrad[6] + vgrad[2]);
    }
    finish_node<Np, ATT, PML, MODE>(a, b, e, node, rq, S, pf, sQF + le * Np + n, O::QF);
  }
  cp_async_wait_all();
}

template <int N, bool ATT, bool PML, int MODE>
__global__ void __launch_bounds__(256, PML ? 1 : 2) stage_kernel(const StageArgs a) {
  extern __shared__ __align__(16) float smem[];
  stage_body<N, ATT, PML, MODE>(a, blockIdx.x, gridDim.x, smem);
}

// Receiver gather: one warp per (batch, receiver) (src/timeloopMod.f90:358-373).
struct RecordArgs {
  int nrec, nbatch, Np, nt;
  const int* it_dev;    // current step (1-based)
  long long ldq;
  const float* q;       // current wavefield
  const int* recelem;   // internal element of each receiver
  const int* recslot;   // abuf slot of each receiver
  const float* recInt;  // [nrec][Np]
  const float* abuf;    // [nbatch][nslot][3][Np]
  int nslot;
  float* u;             // [nbatch][nrec][3] displacement accumulators
  float* traces;        // (nrec, nt, 9, nbatch)
  float dt;
  int* flag;            // set to 1 on a non-finite value
};

__global__ void record_kernel(const RecordArgs a) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= a.nrec * a.nbatch) return;
  const int b = warp / a.nrec, r = warp - b * a.nrec;
  const int e = a.recelem[r];
  const float* q = a.q + (long long)b * 9 * a.ldq + (long long)e * a.Np;
  const float* ab = a.abuf + ((long long)b * a.nslot + a.recslot[r]) * 3 * a.Np;
  float v[3] = {0.f, 0.f, 0.f}, acc[3] = {0.f, 0.f, 0.f};
  for (int j = lane; j < a.Np; j += 32) {
    const float w = a.recInt[(long long)r * a.Np + j];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v[c] = fmaf(q[(6 + c) * a.ldq + j], w, v[c]);
      acc[c] = fmaf(ab[c * a.Np + j], w, acc[c]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
      acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    }
  if (lane == 0) {
    const int it = *a.it_dev;
    float* u = a.u + ((long long)b * a.nrec + r) * 3;
    const long long tb = (long long)b * 9 * a.nt * a.nrec;
    bool bad = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float uc = u[c];
      if (it > 1) uc += a.dt * v[c];
      u[c] = uc;
      a.traces[tb + ((long long)c * a.nt + (it - 1)) * a.nrec + r] = uc;
      a.traces[tb + ((long long)(3 + c) * a.nt + (it - 1)) * a.nrec + r] = v[c];
      a.traces[tb + ((long long)(6 + c) * a.nt + (it - 1)) * a.nrec + r] = acc[c];
      bad |= !isfinite(v[c]);
    }
    if (bad) atomicExch(a.flag, 1);
  }
}

// Advances the device step counter at the end of a step.
__global__ void tick_kernel(int* it_dev) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *it_dev += 1;
}

}  // namespace nexd_dev
