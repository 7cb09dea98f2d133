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
//    applied to the amplitudes and expanded with per-face 9x3 coefficients,
//    and the same lifted amplitudes give the anelastic flux;
//  * NPML elements (grouped first in the internal element order) are handled
//    by the PML instantiation, which differentiates the 27 modified flux
//    columns through their contravariant components (Dr Fr + Ds Fs + Dt Ft).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nexd_dev {

template <int N>
struct Order {
  static constexpr int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  static constexpr int NpF = (N + 1) * (N + 2) / 2;
  static constexpr int NF = 4 * NpF;
  static constexpr int THREADS = 256;
  static constexpr int E = THREADS / Np;  // elements per chunk
  static constexpr int QS = 12;           // padded field stride of staged q (3 x float4)
  static constexpr int GS = 36;           // per-face expansion coefficients
  static constexpr int CS = 28;           // padded contravariant-flux stride (PML)
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
  const float* L;      // [NF][Np] as L[j][n]
  const float* geo;    // [K][64]
  const int4* nbr;     // [K] internal neighbour per face, -1 on boundaries
  const int4* fcode;   // [K] per face: pattern id >= 0, -1 free, -2 absorbing
  const unsigned char* patterns;  // [npat][NpF] neighbour-local node of face node i
  const float* ael;    // [K][3*nMB]: -lam*Ylam, -2mu*Ymu, sum (src/timeloopMod.f90:274-282)
  const float* wl;     // [nMB]
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
  int nt, nspt, it, stage;
  // receivers
  const int* rec_slot;   // [K] slot of receiver elements or -1
  float* abuf;           // [nbatch][nslot][3][Np]: last-stage rq(7:9)
  int nslot;
  int last_stage;
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }

// Expansion coefficients of one face (the rank-3 form of T (A+|A|) T^-1).
__device__ __forceinline__ void face_coeffs(const float* g, int f, float* out) {
  const float nx = g[G_N + 3 * f], ny = g[G_N + 3 * f + 1], nz = g[G_N + 3 * f + 2];
  const float sx = g[G_S + 3 * f], sy = g[G_S + 3 * f + 1], sz = g[G_S + 3 * f + 2];
  const float tx = g[G_T + 3 * f], ty = g[G_T + 3 * f + 1], tz = g[G_T + 3 * f + 2];
  const float c = g[G_C];
  // P = n n^T + c (s s^T + t t^T)   (Voigt xx yy zz xy yz xz)
  out[0] = nx * nx + c * (sx * sx + tx * tx);
  out[1] = ny * ny + c * (sy * sy + ty * ty);
  out[2] = nz * nz + c * (sz * sz + tz * tz);
  out[3] = nx * ny + c * (sx * sy + tx * ty);
  out[4] = ny * nz + c * (sy * sz + ty * tz);
  out[5] = nx * nz + c * (sx * sz + tx * tz);
  // S1 = n s^T + s n^T
  out[6] = 2.f * nx * sx;
  out[7] = 2.f * ny * sy;
  out[8] = 2.f * nz * sz;
  out[9] = nx * sy + ny * sx;
  out[10] = ny * sz + nz * sy;
  out[11] = nx * sz + nz * sx;
  // S2 = n t^T + t n^T
  out[12] = 2.f * nx * tx;
  out[13] = 2.f * ny * ty;
  out[14] = 2.f * nz * tz;
  out[15] = nx * ty + ny * tx;
  out[16] = ny * tz + nz * ty;
  out[17] = nx * tz + nz * tx;
  const float izp = g[G_IZP], izs = g[G_IZS];
  out[18] = -nx * izp; out[19] = -ny * izp; out[20] = -nz * izp;
  out[21] = -sx * izs; out[22] = -sy * izs; out[23] = -sz * izs;
  out[24] = -tx * izs; out[25] = -ty * izs; out[26] = -tz * izs;
  // anelastic: n n^T / (lambda + 2 mu)
  const float ap = g[G_AP];
  out[27] = nx * nx * ap; out[28] = ny * ny * ap; out[29] = nz * nz * ap;
  out[30] = nx * ny * ap; out[31] = ny * nz * ap; out[32] = nx * nz * ap;
  out[33] = 0.f; out[34] = 0.f; out[35] = 0.f;
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

template <int N, bool ATT, bool PML, int MODE>
__global__ void __launch_bounds__(256) stage_kernel(const StageArgs a) {
  using O = Order<N>;
  constexpr int Np = O::Np, NpF = O::NpF, NF = O::NF, E = O::E, QS = O::QS, GS = O::GS, CS = O::CS;
  extern __shared__ __align__(16) float smem[];
  float* sD = smem;                          // 3*Np*Np
  float* sL = sD + 3 * Np * Np;              // NF*Np
  float* sGeo = sL + NF * Np;                // E*64
  float* sQ = sGeo + E * GEO_STRIDE;         // E*Np*QS
  float* sAmp = sQ + E * Np * QS;            // E*NF*4
  float* sG = sAmp + E * NF * 4;             // E*4*GS
  float* sCF = sG + E * 4 * GS;              // PML: E*Np*CS
  (void)sCF;

  const int tid = threadIdx.x;
  for (int i = tid; i < 3 * Np * Np; i += blockDim.x) sD[i] = a.D[i];
  for (int i = tid; i < NF * Np; i += blockDim.x) sL[i] = a.L[i];

  const int nel = a.e_end - a.e_begin;
  const int nchunk = (nel + E - 1) / E;
  const int nwork = nchunk * a.nbatch;
  const int le = tid / Np;       // element of this thread within the chunk
  const int n = tid - le * Np;   // node of this thread

  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int b = w / nchunk;
    const int e0 = a.e_begin + (w - b * nchunk) * E;
    const int ne = min(E, a.e_end - e0);
    const float* qin = a.q_in + (long long)b * 9 * a.ldq;
    __syncthreads();  // previous chunk done with shared memory (and operators staged)
    // ---- stage element records and own wavefield --------------------------------
    for (int i = tid; i < ne * GEO_STRIDE; i += blockDim.x) sGeo[i] = a.geo[(long long)e0 * GEO_STRIDE + i];
    {
      const long long base = (long long)e0 * Np;
      const int cnt = ne * Np;
      for (int i = tid; i < 9 * cnt; i += blockDim.x) {
        const int f = i / cnt, r = i - f * cnt;
        sQ[r * QS + f] = qin[f * a.ldq + base + r];
      }
    }
    __syncthreads();
    // ---- face amplitudes and expansion coefficients -----------------------------
    for (int i = tid; i < ne * NF; i += blockDim.x) {
      const int ee = i / NF, j = i - ee * NF;
      const int f = j / NpF, fi = j - f * NpF;
      const int e = e0 + ee;
      const float* g = sGeo + ee * GEO_STRIDE;
      const int code = reinterpret_cast<const int*>(a.fcode)[4 * e + f];
      // own face node: fmask(fi, f) is pattern row 4*f+? -> stored as pattern id of the identity map
      const int own = a.patterns[(size_t)f * NpF + fi];  // patterns 0..3 are the element's own face masks
      const float* qo = sQ + (ee * Np + own) * QS;
      float dq[9];
      bool free_face = false;
      if (code >= 0) {
        const int nb = reinterpret_cast<const int*>(a.nbr)[4 * e + f];
        const int nn = a.patterns[(size_t)code * NpF + fi];
        const long long gn = (long long)nb * Np + nn;
#pragma unroll
        for (int c = 0; c < 9; ++c) dq[c] = __ldg(qin + c * a.ldq + gn) - qo[c];
      } else if (code == -1) {
#pragma unroll
        for (int c = 0; c < 9; ++c) dq[c] = qo[c];
        free_face = true;
      } else {
#pragma unroll
        for (int c = 0; c < 9; ++c) dq[c] = -qo[c];
      }
      float ap, as1, as2;
      face_amplitudes(g, f, dq, free_face, ap, as1, as2);
      const float fs = g[G_FS + f];
      *reinterpret_cast<float4*>(sAmp + (ee * NF + j) * 4) = make_float4(ap * fs, as1 * fs, as2 * fs, 0.f);
    }
    for (int i = tid; i < ne * 4; i += blockDim.x) face_coeffs(sGeo + (i >> 2) * GEO_STRIDE, i & 3, sG + i * GS);

    // ---- PML: auxiliary update and contravariant modified fluxes ------------------
    float vgrad[9];  // d(v_c)/d(x_d) [c*3+d] (anelastic)
    (void)vgrad;
    if (PML) {
      if (le < ne) {
        const int e = e0 + le;
        const float* g = sGeo + le * GEO_STRIDE;
        const float* qn_ = sQ + (le * Np + n) * QS;
        float F[9], G[9], H[9];
        const float e1 = g[G_E1], e2 = g[G_E2], e3 = g[G_E3], e4 = g[G_E4];
        F[0] = e1 * qn_[6]; F[1] = e2 * qn_[6]; F[2] = e2 * qn_[6]; F[3] = e3 * qn_[7]; F[4] = 0.f;
        F[5] = e3 * qn_[8]; F[6] = e4 * qn_[0]; F[7] = e4 * qn_[3]; F[8] = e4 * qn_[5];
        G[0] = e2 * qn_[7]; G[1] = e1 * qn_[7]; G[2] = e2 * qn_[7]; G[3] = e3 * qn_[6]; G[4] = e3 * qn_[8];
        G[5] = 0.f; G[6] = e4 * qn_[3]; G[7] = e4 * qn_[1]; G[8] = e4 * qn_[4];
        H[0] = e2 * qn_[8]; H[1] = e2 * qn_[8]; H[2] = e1 * qn_[8]; H[3] = 0.f; H[4] = e3 * qn_[7];
        H[5] = e3 * qn_[6]; H[6] = e4 * qn_[5]; H[7] = e4 * qn_[4]; H[8] = e4 * qn_[2];
        const int slot = e;  // PML elements come first in the internal order
        const long long pn = (long long)slot * Np + n;
        const float* pr = a.prof + (long long)slot * 9 * Np + n;
        const float ddx = pr[0], ddy = pr[Np], ddz = pr[2 * Np];
        const float alx = pr[3 * Np], aly = pr[4 * Np], alz = pr[5 * Np];
        const float kx = pr[6 * Np], ky = pr[7 * Np], kz = pr[8 * Np];
        const float ikx = 1.f / kx, iky = 1.f / ky, ikz = 1.f / kz;
        float* aux = a.aux + (long long)b * 27 * a.lda + pn;
        float* aux2 = a.aux2 + (long long)b * 27 * a.lda + pn;
        float* cf = sCF + (le * Np + n) * CS;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          const float fp = aux[i * a.lda], gp = aux[(9 + i) * a.lda], hp = aux[(18 + i) * a.lda];
          const float rf = -alx * fp - ddx * ikx * (fp + F[i]);
          const float rg = -aly * gp - ddy * iky * (gp + G[i]);
          const float rh = -alz * hp - ddz * ikz * (hp + H[i]);
          const float phi = (fp + F[i]) * ikx, psi = (gp + G[i]) * iky, ome = (hp + H[i]) * ikz;
          cf[i] = g[G_RX] * phi + g[G_RY] * psi + g[G_RZ] * ome;
          cf[9 + i] = g[G_SX] * phi + g[G_SY] * psi + g[G_SZ] * ome;
          cf[18 + i] = g[G_TX] * phi + g[G_TY] * psi + g[G_TZ] * ome;
          float nf, ng_, nh;
          if (MODE == MODE_LSERK) {
            const float r1 = a.ca * aux2[i * a.lda] + a.dt * rf;
            const float r2 = a.ca * aux2[(9 + i) * a.lda] + a.dt * rg;
            const float r3 = a.ca * aux2[(18 + i) * a.lda] + a.dt * rh;
            aux2[i * a.lda] = r1;
            aux2[(9 + i) * a.lda] = r2;
            aux2[(18 + i) * a.lda] = r3;
            nf = fp + a.cb * r1;
            ng_ = gp + a.cb * r2;
            nh = hp + a.cb * r3;
          } else {
            float n1, n2, n3;
            if (a.stage_first) {
              aux2[i * a.lda] = fp;
              aux2[(9 + i) * a.lda] = gp;
              aux2[(18 + i) * a.lda] = hp;
              n1 = fp; n2 = gp; n3 = hp;
            } else {
              n1 = aux2[i * a.lda]; n2 = aux2[(9 + i) * a.lda]; n3 = aux2[(18 + i) * a.lda];
            }
            nf = a.ca * n1 + a.cb * (fp + a.dt * rf);
            ng_ = a.ca * n2 + a.cb * (gp + a.dt * rg);
            nh = a.ca * n3 + a.cb * (hp + a.dt * rh);
          }
          aux[i * a.lda] = nf;
          aux[(9 + i) * a.lda] = ng_;
          aux[(18 + i) * a.lda] = nh;
        }
      }
    }
    __syncthreads();
    if (le >= ne) continue;  // idle threads of a partial chunk (no barrier follows in this iteration)

    const int e = e0 + le;
    const float* g = sGeo + le * GEO_STRIDE;
    float rq[9];
    // ---- volume term ------------------------------------------------------------
    if (!PML) {
      float dr[9], ds[9], dtt[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) { dr[c] = 0.f; ds[c] = 0.f; dtt[c] = 0.f; }
      const float* qe = sQ + le * Np * QS;
#pragma unroll 5
      for (int k = 0; k < Np; ++k) {
        const float d0 = sD[k * Np + n], d1 = sD[Np * Np + k * Np + n], d2 = sD[2 * Np * Np + k * Np + n];
        const float4 qa = ld4(qe + k * QS), qb = ld4(qe + k * QS + 4);
        const float q8 = qe[k * QS + 8];
        const float qq[9] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w, q8};
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          dr[c] = fmaf(d0, qq[c], dr[c]);
          ds[c] = fmaf(d1, qq[c], ds[c]);
          dtt[c] = fmaf(d2, qq[c], dtt[c]);
        }
      }
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
      float vr[3] = {0.f, 0.f, 0.f}, vs3[3] = {0.f, 0.f, 0.f}, vt3[3] = {0.f, 0.f, 0.f};
      const float* cfe = sCF + le * Np * CS;
      const float* qe = sQ + le * Np * QS;
#pragma unroll 2
      for (int k = 0; k < Np; ++k) {
        const float d0 = sD[k * Np + n], d1 = sD[Np * Np + k * Np + n], d2 = sD[2 * Np * Np + k * Np + n];
        const float* cf = cfe + k * CS;
#pragma unroll
        for (int c = 0; c < 9; ++c) rq[c] = fmaf(d0, cf[c], fmaf(d1, cf[9 + c], fmaf(d2, cf[18 + c], rq[c])));
        if (ATT) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float v = qe[k * QS + 6 + c];
            vr[c] = fmaf(d0, v, vr[c]);
            vs3[c] = fmaf(d1, v, vs3[c]);
            vt3[c] = fmaf(d2, v, vt3[c]);
          }
        }
      }
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
      float A0 = 0.f, A1 = 0.f, A2 = 0.f;
      const float* am = sAmp + (le * NF + f * NpF) * 4;
      const float* lf = sL + f * NpF * Np + n;
#pragma unroll 5
      for (int i = 0; i < NpF; ++i) {
        const float l = lf[i * Np];
        const float4 v = ld4(am + i * 4);
        A0 = fmaf(l, v.x, A0);
        A1 = fmaf(l, v.y, A1);
        A2 = fmaf(l, v.z, A2);
      }
      const float* G = sG + (le * 4 + f) * GS;
      float X[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) X[c] = G[6 + c] * A1 + G[12 + c] * A2;
#pragma unroll
      for (int c = 0; c < 6; ++c) rq[c] += G[c] * A0 + X[c];
      rq[6] += G[18] * A0 + G[21] * A1 + G[24] * A2;
      rq[7] += G[19] * A0 + G[22] * A1 + G[25] * A2;
      rq[8] += G[20] * A0 + G[23] * A1 + G[26] * A2;
      if (ATT) {
        const float as = g[G_AS];
#pragma unroll
        for (int c = 0; c < 6; ++c) sig_an[c] += G[27 + c] * A0 + X[c] * as;
      }
    }
    const long long node = (long long)e * Np + n;
    // ---- Zener memory variables (src/timeloopMod.f90:426-461) ------------------
    if (ATT) {
      // S = -strain rate + lifted anelastic flux; d theta_l/dt = w_l (S - theta_l)
      float S[6];
      S[0] = sig_an[0] - vgrad[0];
      S[1] = sig_an[1] - vgrad[4];
      S[2] = sig_an[2] - vgrad[8];
      S[3] = sig_an[3] - 0.5f * (vgrad[3] + vgrad[1]);
      S[4] = sig_an[4] - 0.5f * (vgrad[7] + vgrad[5]);
      S[5] = sig_an[5] - 0.5f * (vgrad[6] + vgrad[2]);
      float* th = a.th + (long long)b * 6 * a.nMB * a.ldt + node;
      float* th2 = a.th2 + (long long)b * 6 * a.nMB * a.ldt + node;
      const float* ae = a.ael + (long long)e * 3 * a.nMB;
      for (int l = 0; l < a.nMB; ++l) {
        const float wl = a.wl[l];
        float t[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) t[j] = th[(l * 6 + j) * a.ldt];
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
          const long long o = (l * 6 + j) * a.ldt;
          float nt_;
          if (MODE == MODE_LSERK) {
            const float rr = a.ca * th2[o] + a.dt * r;
            th2[o] = rr;
            nt_ = t[j] + a.cb * rr;
          } else {
            float tn;
            if (a.stage_first) { th2[o] = t[j]; tn = t[j]; } else { tn = th2[o]; }
            nt_ = a.ca * tn + a.cb * (t[j] + a.dt * r);
          }
          th[o] = nt_;
        }
      }
    }
    // ---- point sources -----------------------------------------------------------
    for (int s = a.src_head[e]; s >= 0; s = a.src_next[s]) {
      if (a.src_batch[s] != b) continue;
      const int sidx = a.nspt == 1 ? 0 : min(a.stage, a.nspt - 1);
      const float amp = a.stf[((long long)s * a.nt + (a.it - 1)) * a.nspt + sidx];
      const float* p = a.src_pat + (long long)s * 9 * Np + n;
#pragma unroll
      for (int c = 0; c < 9; ++c) rq[c] = fmaf(p[c * Np], amp, rq[c]);
    }
    // ---- receiver acceleration (last stage) ----------------------------------------
    if (a.last_stage) {
      const int slot = a.rec_slot[e];
      if (slot >= 0) {
        float* ab = a.abuf + ((long long)b * a.nslot + slot) * 3 * Np + n;
        ab[0] = rq[6];
        ab[Np] = rq[7];
        ab[2 * Np] = rq[8];
      }
    }
    // ---- stage update ------------------------------------------------------------
    const float* qown = sQ + (le * Np + n) * QS;
    float* qo = a.q_out + (long long)b * 9 * a.ldq + node;
    if (MODE == MODE_LSERK) {
      float* rs = a.res + (long long)b * 9 * a.ldq + node;
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const float r = a.ca * rs[c * a.ldq] + a.dt * rq[c];
        rs[c * a.ldq] = r;
        qo[c * a.ldq] = qown[c] + a.cb * r;
      }
    } else {
      const float* qn = a.q_n + (long long)b * 9 * a.ldq + node;
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const float base = (a.ca != 0.f) ? a.ca * qn[c * a.ldq] : 0.f;
        qo[c * a.ldq] = base + a.cb * (qown[c] + a.dt * rq[c]);
      }
    }
  }
}

// Receiver gather: one warp per (batch, receiver) (src/timeloopMod.f90:358-373).
struct RecordArgs {
  int nrec, nbatch, Np, nt, it;
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
    float* u = a.u + ((long long)b * a.nrec + r) * 3;
    const long long tb = (long long)b * 9 * a.nt * a.nrec;
    bool bad = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float uc = u[c];
      if (a.it > 1) uc += a.dt * v[c];
      u[c] = uc;
      a.traces[tb + ((long long)c * a.nt + (a.it - 1)) * a.nrec + r] = uc;
      a.traces[tb + ((long long)(3 + c) * a.nt + (a.it - 1)) * a.nrec + r] = v[c];
      a.traces[tb + ((long long)(6 + c) * a.nt + (a.it - 1)) * a.nrec + r] = acc[c];
      bad |= !isfinite(v[c]);
    }
    if (bad) atomicExch(a.flag, 1);
  }
}

}  // namespace nexd_dev
