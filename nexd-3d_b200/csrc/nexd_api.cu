// C-ABI of libnexd.so (include/nexd.h): device set-up and the time loop.
//
// Replaces timeloop3D (src/timeloopMod.f90:42-674) for one partition (the
// whole mesh, or one part of it with a halo exchange, halo.cuh).
// Host work here is set-up only (FP64 -> FP32 element records, connectivity
// patterns, source patterns); every time step runs on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/nexd.h"
#include "energy_kernel.cuh"
#include "stage_kernel.cuh"
#include "stage_tc.cuh"
#include "stage_pair.cuh"
#include "stage_main_bulk.cuh"
#include "group_kernel.cuh"
#include "boundary_mlp.cuh"
#include "halo.cuh"
#include "mlp_tc.cuh"
#include "boundary_tc.cuh"

#include <unistd.h>

using namespace nexd_dev;

namespace {

thread_local std::string g_create_error;

// Carpenter & Kennedy (1994) 5-stage, 4th-order, 2N-storage coefficients.
const double kRK4A[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                         -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kRK4B[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                         1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                         2277821191437.0 / 14882151754819.0};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct nexd_ctx {
  std::string err;
  int N = 0, Np = 0, NpF = 0, K = 0, nMB = 0, nt = 0, nstage = 1, timeint = 4, nbatch = 1;
  int Kpml = 0;  // PML elements occupy internal indices [0, Kpml)
  int npat = 4;  // face pattern rows (4 own masks + neighbour maps)
  bool att = false, pml = false;
  double dt = 0.0;
  long long ldq = 0, ldt = 0, lda = 0;
  int nrec = 0, nslot = 0, nsrc = 0, nspt = 1;
  std::vector<int> new2old, old2new;
  cudaStream_t stream = nullptr;
  int device = 0;
  int nsm = 148;
  int grid_pml = 0, grid_main = 0;
  size_t smem_pml = 0, smem_main = 0;
  // device arrays
  float *D = nullptr, *L = nullptr, *geo = nullptr, *ael = nullptr, *wl = nullptr, *prof_dev = nullptr;
  float wl_host[3] = {0.f, 0.f, 0.f};  // relaxation frequencies (kernel parameters)
  int4 *nbr = nullptr, *fcode = nullptr;
  unsigned char* patterns = nullptr;
  float* qbuf[3] = {nullptr, nullptr, nullptr};
  float* res = nullptr;
  float *th = nullptr, *th2 = nullptr, *aux = nullptr, *aux2 = nullptr;
  int *src_head = nullptr, *src_next = nullptr, *src_batch = nullptr;
  float *src_pat = nullptr, *stf = nullptr;
  int *rec_slot = nullptr, *recelem = nullptr, *recslot_of_rec = nullptr;
  float *recInt = nullptr, *abuf = nullptr, *u = nullptr, *traces = nullptr;
  int* flag = nullptr;
  int cur = 0;  // index of the buffer holding the current wavefield
  int64_t launches = 0;
  std::vector<void*> allocations;
  // profiling: CUDA events around each launch on `stream`
  bool profiling = false;  // per-launch events (mode 1)
  bool span_timing = false; // run span events (modes 1 and 2)
  std::vector<cudaEvent_t> events;
  std::vector<int> ev_kind;  // kind of event pair i (events 2i, 2i+1)
  int ev_used = 0;
  cudaEvent_t span[2] = {nullptr, nullptr};
  nexd_profile prof{};
  // pinned staging for nexd_step_io
  float* pinned = nullptr;
  size_t pinned_floats = 0;
  // NPML energy / STA-LTA trigger
  int* pml_off = nullptr;     // [nbatch]
  int* pml_switch = nullptr;  // [nbatch]
  bool energy_on = false;
  int trig_w1 = 10, trig_w2 = 2, trig_timecrit = 0, trig_formula = 0;
  float trig_threshold = 0.1f;
  double* energy = nullptr;    // [nbatch][nt]
  double* partials = nullptr;  // [nbatch][energy_blocks]
  float4* emat = nullptr;      // [K] (rho, lambda, mu, J)
  double* mass = nullptr;      // [Np][Np]
  int energy_blocks = 0;
  // step counter on the device and two-step CUDA graphs (one per starting buffer parity)
  int* it_dev = nullptr;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  // one-step graphs per starting buffer (0..2) and the buffer each leaves current
  cudaGraphExec_t gexec1[3] = {nullptr, nullptr, nullptr};
  int gend1[3] = {0, 0, 0};
  int graph1_launches[3] = {0, 0, 0};
  int graph_launches = 0;      // kernels per captured two-step graph
  bool graph_energy = false;   // energy_on when the graphs were captured
  bool use_graphs = true;
  // element contraction: NEXD_CONTRACT_FP32 (CUDA cores) or NEXD_CONTRACT_BF16X3 (tensor cores)
  int contraction = NEXD_CONTRACT_FP32;
  int grid_div = 1;            // persistent grid divided by this (models sharing the GPU in a group)
  int kind[2] = {NEXD_CONTRACT_FP32, NEXD_CONTRACT_FP32};  // kernel per element class: [0] NPML, [1] the rest
  float tune_ms[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};  // autotune: [class][kind] ms per launch
  uint4* ops_tc = nullptr;     // packed operator of the tensor-core kernels (order 4)
  // learned absorbing boundary: absorbing faces, their ghost states and the MLP
  int nbf = 0;                       // absorbing faces
  int *bf_elem = nullptr, *bf_face = nullptr;  // [nbf] internal element, local face
  int4* fcode_learned = nullptr;     // face codes with absorbing faces as -3 - ghost index
  float* ghost = nullptr;            // [nbatch][nbf][9][NpF]
  __nv_bfloat16* mlp_w = nullptr;    // parameters in bf16
  float* mlp_stage = nullptr;        // FP32 upload buffer of the parameters
  bool mlp_on = false;
  float mlp_rho = 0.f;               // bound of the incoming / outgoing characteristic ratio
  int ghost_grid = 0;
  size_t ghost_smem = 0;
  uint4* mlp_wimg = nullptr;         // the network's weight images for the tensor cores
  // movie: nodal displacement and per-element frames (src/timeloopMod.f90:482-489, 576-581)
  int movie_frame = 0, movie_max = 0, movie_last_it = 0;
  float init_value = 0.f;            // start value of every field (the reference's 1e-24)
  float* movie_u = nullptr;          // [nbatch][3][ldq]
  float* movie_buf = nullptr;        // [max_frames][nbatch][K] (internal element order)
  int* gather_idx = nullptr;         // face-trace gather scratch
  float* gather_out = nullptr;
  int gather_cap = 0;
  // partition halo (nexd_create_partition): halo slots are elements K .. K + nhalo - 1
  int partition = 0;                 // 1-based partition number, 0 for a whole mesh
  int nhalo = 0;
  int npeer = 0;
  std::vector<int> peer_part, peer_nface, peer_goff;  // per neighbour: number, shared faces, first halo slot
  std::vector<HaloPeer> peers_h;     // writer's view of each neighbour (filled by nexd_halo_connect)
  std::vector<char> peer_linked;
  HaloPeer* peers_dev = nullptr;
  int* halo_src = nullptr;           // [entries] own node of each shared face node
  int* halo_dst = nullptr;           // [entries] node offset in the neighbour's halo
  int* halo_blocks = nullptr;        // [npeer] write blocks each neighbour sends per stage
  unsigned long long* halo_counters = nullptr;  // [npeer] arrivals from each neighbour
  unsigned long long* halo_expected = nullptr;  // [npeer] arrivals consumed
  int put_blocks = 0;
  unsigned long long halo_limit_ns = 5000000000ull;  // longest arrival wait
  std::vector<void*> ipc_opened;     // neighbours' buffers opened through CUDA IPC
};

namespace {

// Raises energy_kernel's dynamic shared-memory limit to the most the current
// device allows for it (opt-in maximum minus its static shared memory).
cudaError_t raise_energy_smem_limit() {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes fa{};
  e = cudaFuncGetAttributes(&fa, nexd_dev::energy_kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(nexd_dev::energy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              optin - int(fa.sharedSizeBytes));
}

int set_err(nexd_ctx* c, int code, const std::string& m) {
  if (c) c->err = m; else g_create_error = m;
  return code;
}

#define CUDA_TRY(ctx, call)                                                                  \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return set_err(ctx, e_ == cudaErrorMemoryAllocation ? NEXD_ERR_NOMEM : NEXD_ERR_CUDA,  \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                    \
  } while (0)

template <class T>
int dalloc(nexd_ctx* c, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  void* v = nullptr;
  cudaError_t e = cudaMalloc(&v, count * sizeof(T));
  if (e != cudaSuccess)
    return set_err(c, e == cudaErrorMemoryAllocation ? NEXD_ERR_NOMEM : NEXD_ERR_CUDA,
                   std::string("cudaMalloc: ") + cudaGetErrorString(e));
  c->allocations.push_back(v);
  *p = static_cast<T*>(v);
  return NEXD_OK;
}

template <class T>
int upload(nexd_ctx* c, T** p, const std::vector<T>& h) {
  int st = dalloc(c, p, h.size());
  if (st) return st;
  if (!h.empty()) CUDA_TRY(c, cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return NEXD_OK;
}

int fill(nexd_ctx* c, float* p, size_t n, float v) {
  std::vector<float> h(std::min<size_t>(n, size_t(1) << 24), v);
  for (size_t off = 0; off < n; off += h.size()) {
    const size_t m = std::min(h.size(), n - off);
    CUDA_TRY(c, cudaMemcpy(p + off, h.data(), m * sizeof(float), cudaMemcpyHostToDevice));
  }
  return NEXD_OK;
}

template <int N>
size_t smem_bytes(bool pml) {
  return size_t(Order<N>::smem_floats(pml)) * sizeof(float);
}

using KernelFn = void (*)(const StageArgs);

template <int N>
KernelFn pick(bool att, bool pml, int mode) {
  if (mode == MODE_LSERK) {
    if (att) return pml ? stage_kernel<N, true, true, MODE_LSERK> : stage_kernel<N, true, false, MODE_LSERK>;
    return pml ? stage_kernel<N, false, true, MODE_LSERK> : stage_kernel<N, false, false, MODE_LSERK>;
  }
  if (att) return pml ? stage_kernel<N, true, true, MODE_TVD> : stage_kernel<N, true, false, MODE_TVD>;
  return pml ? stage_kernel<N, false, true, MODE_TVD> : stage_kernel<N, false, false, MODE_TVD>;
}

KernelFn pick_kernel(int N, bool att, bool pml, int mode, size_t& smem) {
  switch (N) {
    case 1: smem = smem_bytes<1>(pml); return pick<1>(att, pml, mode);
    case 2: smem = smem_bytes<2>(pml); return pick<2>(att, pml, mode);
    case 3: smem = smem_bytes<3>(pml); return pick<3>(att, pml, mode);
    case 4: smem = smem_bytes<4>(pml); return pick<4>(att, pml, mode);
    case 5: smem = smem_bytes<5>(pml); return pick<5>(att, pml, mode);
    default: smem = 0; return nullptr;
  }
}

using TcKernelFn = void (*)(const StageArgs, const uint4*);

template <int N>
TcKernelFn pick_tc(bool att, bool pml, int mode) {
  if (mode == MODE_LSERK) {
    if (att) return pml ? stage_tc_kernel<N, true, true, MODE_LSERK> : stage_tc_kernel<N, true, false, MODE_LSERK>;
    return pml ? stage_tc_kernel<N, false, true, MODE_LSERK> : stage_tc_kernel<N, false, false, MODE_LSERK>;
  }
  if (att) return pml ? stage_tc_kernel<N, true, true, MODE_TVD> : stage_tc_kernel<N, true, false, MODE_TVD>;
  return pml ? stage_tc_kernel<N, false, true, MODE_TVD> : stage_tc_kernel<N, false, false, MODE_TVD>;
}

TcKernelFn pick_tc_kernel(int N, bool att, bool pml, int mode, size_t& smem) {
  switch (N) {
    case 4: smem = TcOrder<4>::smem_bytes(); return pick_tc<4>(att, pml, mode);
    default: smem = 0; return nullptr;
  }
}

// The stacked operator [Dr Ds Dt LIFT] of the tensor-core stage kernel as bf16
// H, M, L rows (row n' = output node, K-major, 128-byte swizzle): entry
// (n', d Np + k) = D_d(n', k), entry (n', KV16 + f NpF + i) = LIFT(n', f NpF + i),
// zero elsewhere; x = H + M + L with M = bf16(x - H), L = bf16(x - H - M) of
// the FP64 value.  (A two-part operator, a fixed 2^-17 relative change, moves
// the acceleration traces by ~1e-3: the derivative of a smooth field cancels
// about two digits of its terms.)
template <int N>
std::vector<uint16_t> pack_tc_operator(const nexd_desc* d) {
  using T = TcOrder<N>;
  constexpr int Np = T::Np;
  auto bf16_bits = [](double x) {
    const float f = float(x);
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return uint16_t((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);  // round to nearest even
  };
  auto bf16_value = [](uint16_t h) {
    const uint32_t u = uint32_t(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return double(f);
  };
  std::vector<uint16_t> out(T::B_BYTES / 2, 0);
  for (int np_ = 0; np_ < Np; ++np_)
    for (int k = 0; k < T::KU; ++k) {
      double x = 0.0;
      if (k < T::KV) {
        const int dd = k / Np, kk = k - dd * Np;
        const double* D = dd == 0 ? d->Dr : dd == 1 ? d->Ds : d->Dt;
        x = D[size_t(kk) * Np + np_];
      } else if (k >= T::KV16) {
        x = d->lift[size_t(k - T::KV16) * Np + np_];
      }
      uint16_t part[3];
      double r = x;
      for (int q = 0; q < 3; ++q) {
        part[q] = bf16_bits(r);
        r -= bf16_value(part[q]);
      }
      for (int q = 0; q < 3; ++q) {
        const int row = q * T::NP16 + np_, rr = row & 7, g = row >> 3, slab = k >> 6, kk = k & 63;
        const size_t off = size_t(slab) * T::B_SLAB + size_t(g) * 1024 + size_t(rr) * 128 +
                           size_t(((kk >> 3) ^ rr) << 4) + size_t(kk & 7) * 2;
        out[off / 2] = part[q];
      }
    }
  return out;
}

template <int N>
KernelFn pick_pair(bool att, int mode) {
  if (mode == MODE_LSERK) return att ? stage_pair_kernel<N, true, MODE_LSERK> : stage_pair_kernel<N, false, MODE_LSERK>;
  return att ? stage_pair_kernel<N, true, MODE_TVD> : stage_pair_kernel<N, false, MODE_TVD>;
}

// The node-pair FP32 kernel (elements outside the NPML; orders 2-5).
KernelFn pick_pair_kernel(int N, bool att, int mode, size_t& smem) {
  switch (N) {
    case 2: smem = size_t(Order<2, 2>::smem_floats(false)) * 4; return pick_pair<2>(att, mode);
    case 3: smem = size_t(Order<3, 2>::smem_floats(false)) * 4; return pick_pair<3>(att, mode);
    case 4: smem = size_t(Order<4, 2>::smem_floats(false)) * 4; return pick_pair<4>(att, mode);
    case 5: smem = size_t(Order<5, 2>::smem_floats(false)) * 4; return pick_pair<5>(att, mode);
    default: smem = 0; return nullptr;
  }
}

// Kernel kinds per element class: NEXD_CONTRACT_FP32, NEXD_CONTRACT_BF16X3,
// the node-pair FP32 kernel (elements outside the NPML) and the FP32 kernels
// whose element-local state moves by bulk copies (NPML elements: NPML and
// update-phase state; the rest, anelastic: memory variables); the last two
// give the same results as NEXD_CONTRACT_FP32 and are chosen by the autotune
// or pinned.
constexpr int KIND_FP32_PAIRS = 2;
constexpr int KIND_BULK = 3;
constexpr int NKINDS = 4;

template <int N>
KernelFn pick_bulk(bool att, int mode) {
  if (mode == MODE_LSERK) return att ? stage_npml_bulk_kernel<N, true, MODE_LSERK> : stage_npml_bulk_kernel<N, false, MODE_LSERK>;
  return att ? stage_npml_bulk_kernel<N, true, MODE_TVD> : stage_npml_bulk_kernel<N, false, MODE_TVD>;
}

// Orders whose bulk-staged NPML kernel fits the 227 KB of shared memory a
// block can have: 3 and 4 (orders 2 and 5 need 231 and 236 KB).
bool bulk_order_supported(int N) { return N == 3 || N == 4; }

// The FP32 NPML kernel with bulk-copied element-local state.
KernelFn pick_bulk_kernel(int N, bool att, int mode, size_t& smem) {
  switch (N) {
    case 3: smem = size_t(BulkOrder<3>::smem_floats()) * 4; return pick_bulk<3>(att, mode);
    case 4: smem = size_t(BulkOrder<4>::smem_floats()) * 4; return pick_bulk<4>(att, mode);
    default: smem = 0; return nullptr;
  }
}

template <int N>
KernelFn pick_main_bulk(int mode) {
  return mode == MODE_LSERK ? stage_main_bulk_kernel<N, MODE_LSERK> : stage_main_bulk_kernel<N, MODE_TVD>;
}

// The bulk-copy kernel for the elements outside the NPML (anelastic models,
// orders 2-5).
KernelFn pick_main_bulk_kernel(int N, int mode, size_t& smem) {
  switch (N) {
    case 2: smem = size_t(MainBulkOrder<2>::smem_floats()) * 4; return pick_main_bulk<2>(mode);
    case 3: smem = size_t(MainBulkOrder<3>::smem_floats()) * 4; return pick_main_bulk<3>(mode);
    case 4: smem = size_t(MainBulkOrder<4>::smem_floats()) * 4; return pick_main_bulk<4>(mode);
    case 5: smem = size_t(MainBulkOrder<5>::smem_floats()) * 4; return pick_main_bulk<5>(mode);
    default: smem = 0; return nullptr;
  }
}

// Whether the bulk-copy kernel exists for an element class of this context.
bool bulk_supported(int N, bool att, int cls) {
  return cls == 0 ? bulk_order_supported(N) : (att && N >= 2 && N <= 5);
}

// Threads per block of a kernel kind.
int kind_threads(int kind, bool pml) { return (kind == KIND_BULK && pml) ? kBulkThreads : 256; }

// Floats per element of an element-blocked array of F fields: F x Np
// padded to a multiple of 4 (EBlock in stage_kernel.cuh).
long long block_stride(int F, int Np) { return ((long long)F * Np + 3) / 4 * 4; }

int elements_per_chunk(int N) {
  const int Np = (N + 1) * (N + 2) * (N + 3) / 6;
  return 256 / Np;
}

int validate(const nexd_desc* d, bool partition_ok = false) {
  if (!d) return set_err(nullptr, NEXD_ERR_INVALID, "null descriptor");
  if (d->abi_version != NEXD_ABI_VERSION) return set_err(nullptr, NEXD_ERR_INVALID, "ABI version mismatch");
  if (d->N < 1 || d->N > 5)
    return set_err(nullptr, NEXD_ERR_UNSUPPORTED, "polynomial order must be 1..5 in this build");
  const int Np = (d->N + 1) * (d->N + 2) * (d->N + 3) / 6, NpF = (d->N + 1) * (d->N + 2) / 2;
  if (d->Np != Np || d->NpF != NpF) return set_err(nullptr, NEXD_ERR_INVALID, "Np/NpF inconsistent with N");
  if (d->nelem <= 0) return set_err(nullptr, NEXD_ERR_INVALID, "nelem must be positive");
  if (d->nt <= 0) return set_err(nullptr, NEXD_ERR_INVALID, "nt must be positive");
  if (!(d->dt > 0.0) || !std::isfinite(d->dt)) return set_err(nullptr, NEXD_ERR_INVALID, "dt must be positive");
  if (d->timeint < 1 || d->timeint > 4) return set_err(nullptr, NEXD_ERR_INVALID, "timeint must be 1..4");
  if (d->nbatch < 1) return set_err(nullptr, NEXD_ERR_INVALID, "nbatch must be >= 1");
  if (d->attenuation && (!d->wl || !d->ylambda || !d->ymu))
    return set_err(nullptr, NEXD_ERR_INVALID, "attenuation needs wl/ylambda/ymu");
  if (d->attenuation && d->nMB != nexd_dev::kNMB)
    return set_err(nullptr, NEXD_ERR_UNSUPPORTED, "attenuation supports nMB = 3 Zener mechanisms (the reference's nMB)");
  if (d->set_pml && (!d->pmlcheck || !d->pml_profiles))
    return set_err(nullptr, NEXD_ERR_INVALID, "set_pml needs pmlcheck and pml_profiles");
  const void* req[] = {d->Dr, d->Ds, d->Dt, d->lift, d->fmask, d->metric, d->jacobian, d->fscale, d->nnormal,
                       d->stangential, d->ttangential, d->rho, d->vpu, d->vsu, d->lambdau, d->muu, d->neighbor,
                       d->face, d->ibn};
  for (const void* p : req)
    if (!p) return set_err(nullptr, NEXD_ERR_INVALID, "descriptor has a null array");
  if (d->nsrc < 0 || d->nrec < 0) return set_err(nullptr, NEXD_ERR_INVALID, "negative source/receiver count");
  if (d->nsrc > 0 && (!d->srcelem || !d->srctype || !d->srcInt || !d->stf || !d->invmass || d->stf_per_step < 1))
    return set_err(nullptr, NEXD_ERR_INVALID, "sources need srcelem/srctype/srcInt/stf/invmass");
  if (d->nrec > 0 && (!d->recelem || !d->recInt)) return set_err(nullptr, NEXD_ERR_INVALID, "receivers need recelem/recInt");
  for (int i = 0; i < d->nsrc; ++i) {
    if (d->srcelem[i] < 1 || d->srcelem[i] > d->nelem) return set_err(nullptr, NEXD_ERR_INVALID, "srcelem out of range");
    if (d->srctype[i] != 0 && d->srctype[i] != 1) return set_err(nullptr, NEXD_ERR_INVALID, "srctype must be 0 or 1");
    if (d->srctype[i] == 0 && !d->srcangle_force) return set_err(nullptr, NEXD_ERR_INVALID, "force source without direction");
    if (d->srctype[i] == 1 && !d->srcM) return set_err(nullptr, NEXD_ERR_INVALID, "moment source without tensor");
    if (d->nbatch > 1 && d->srcbatch && (d->srcbatch[i] < 0 || d->srcbatch[i] >= d->nbatch))
      return set_err(nullptr, NEXD_ERR_INVALID, "srcbatch out of range");
  }
  for (int i = 0; i < d->nrec; ++i)
    if (d->recelem[i] < 1 || d->recelem[i] > d->nelem) return set_err(nullptr, NEXD_ERR_INVALID, "recelem out of range");
  // face masks index the element's own nodes (they become the byte-sized
  // face patterns of the stage kernels)
  for (int i = 0; i < 4 * NpF; ++i)
    if (d->fmask[i] < 1 || d->fmask[i] > Np) return set_err(nullptr, NEXD_ERR_INVALID, "fmask entry out of 1..Np");
  for (int e = 0; e < d->nelem; ++e) {
    for (int f = 0; f < 4; ++f) {
      const int nb = d->neighbor[4 * e + f], fc = d->face[4 * e + f];
      if (nb < 0 || nb > d->nelem) return set_err(nullptr, NEXD_ERR_INVALID, "neighbor index out of range");
      if (nb == 0 && fc == NEXD_FACE_PARTITION && !partition_ok)
        return set_err(nullptr, NEXD_ERR_INVALID, "face shared with another partition (-3) needs nexd_create_partition");
      if (nb == 0 && fc != -1 && fc != -2 && fc != NEXD_FACE_PARTITION)
        return set_err(nullptr, NEXD_ERR_INVALID, "boundary face that is neither free (-1) nor absorbing (-2)");
      if (nb > 0 && (fc < 1 || fc > 4)) return set_err(nullptr, NEXD_ERR_INVALID, "interior face without neighbour face id");
      if (nb > 0)
        for (int i = 0; i < NpF; ++i) {
          // ibn is a global 1-based node id that must lie inside the neighbour
          const long long gn = (long long)d->ibn[(size_t(e) * 4 + f) * NpF + i] - 1 - (long long)(nb - 1) * Np;
          if (gn < 0 || gn >= Np) return set_err(nullptr, NEXD_ERR_INVALID, "ibn does not point into the neighbour element");
        }
    }
    if (!(std::fabs(d->jacobian[e]) > 0.0)) return set_err(nullptr, NEXD_ERR_INVALID, "zero Jacobian");
    if (!(d->rho[e] > 0.0) || !(d->vpu[e] > 0.0) || !(d->vsu[e] > 0.0))
      return set_err(nullptr, NEXD_ERR_INVALID, "non-positive material value");
  }
  return NEXD_OK;
}

// The halo descriptor against its partition's descriptor (which passed
// validate): every shared face listed once, coded as shared in desc, with an
// index into the neighbour's list and a node matching that are permutations.
int validate_halo(const nexd_desc* d, const nexd_halo_desc* h) {
  if (!h) return set_err(nullptr, NEXD_ERR_INVALID, "null halo descriptor");
  if (h->partition < 1) return set_err(nullptr, NEXD_ERR_INVALID, "partition number must be >= 1");
  if (h->npeer < 0 || h->npeer > kHaloMaxPeers)
    return set_err(nullptr, NEXD_ERR_INVALID, "halo: neighbour count out of 0..64");
  if (h->npeer > 0 && (!h->peer || !h->nface || !h->elem || !h->side || !h->peer_index || !h->peer_node))
    return set_err(nullptr, NEXD_ERR_INVALID, "halo descriptor has a null array");
  const int K = d->nelem, NpF = d->NpF;
  long long total = 0;
  for (int p = 0; p < h->npeer; ++p) {
    if (h->peer[p] < 1 || h->peer[p] == h->partition)
      return set_err(nullptr, NEXD_ERR_INVALID, "halo: neighbour partition number invalid");
    for (int q = 0; q < p; ++q)
      if (h->peer[q] == h->peer[p]) return set_err(nullptr, NEXD_ERR_INVALID, "halo: neighbour listed twice");
    if (h->nface[p] < 1) return set_err(nullptr, NEXD_ERR_INVALID, "halo: neighbour without shared faces");
    total += h->nface[p];
  }
  if (total > 4LL * K) return set_err(nullptr, NEXD_ERR_INVALID, "halo: more shared faces than element faces");
  std::vector<char> seen(size_t(4) * K, 0);
  std::vector<char> used;
  long long i = 0;
  for (int p = 0; p < h->npeer; ++p) {
    used.assign(size_t(h->nface[p]), 0);
    for (int c = 0; c < h->nface[p]; ++c, ++i) {
      const int e = h->elem[i], f = h->side[i];
      if (e < 1 || e > K || f < 1 || f > 4) return set_err(nullptr, NEXD_ERR_INVALID, "halo: face element or side out of range");
      const size_t k = size_t(4) * (e - 1) + (f - 1);
      if (d->neighbor[k] != 0 || d->face[k] != NEXD_FACE_PARTITION)
        return set_err(nullptr, NEXD_ERR_INVALID, "halo: face is not coded as shared (-3) in the descriptor");
      if (seen[k]) return set_err(nullptr, NEXD_ERR_INVALID, "halo: face listed twice");
      seen[k] = 1;
      const int pi = h->peer_index[i];
      if (pi < 1 || pi > h->nface[p] || used[pi - 1])
        return set_err(nullptr, NEXD_ERR_INVALID, "halo: peer_index is not a permutation of the neighbour's faces");
      used[pi - 1] = 1;
      unsigned long long nodes = 0;
      for (int j = 0; j < NpF; ++j) {
        const int m = h->peer_node[i * NpF + j];
        if (m < 1 || m > NpF || (nodes >> (m - 1) & 1ull))
          return set_err(nullptr, NEXD_ERR_INVALID, "halo: peer_node is not a permutation of the face nodes");
        nodes |= 1ull << (m - 1);
      }
    }
  }
  for (size_t k = 0; k < seen.size(); ++k)
    if (d->face[k] == NEXD_FACE_PARTITION && d->neighbor[k] == 0 && !seen[k])
      return set_err(nullptr, NEXD_ERR_INVALID, "halo: a shared face (-3) is missing from the halo");
  return NEXD_OK;
}

}  // namespace

extern "C" {

// Shared memory and persistent grid of the two stage kernels (NPML elements,
// the rest) for the context's order, rheology, integrator and contraction.
int configure_launch(nexd_ctx* c) {
  const int mode = c->timeint == 4 ? MODE_LSERK : MODE_TVD;
  for (int which = 0; which < 2; ++which) {
    const bool pmlk = which == 0;
    size_t smem = 0;
    const void* fn;
    int E = elements_per_chunk(c->N);
    if (c->kind[which] == NEXD_CONTRACT_BF16X3) {
      fn = reinterpret_cast<const void*>(pick_tc_kernel(c->N, c->att, pmlk, mode, smem));
    } else if (c->kind[which] == KIND_FP32_PAIRS && !pmlk) {
      fn = reinterpret_cast<const void*>(pick_pair_kernel(c->N, c->att, mode, smem));
      E *= 2;
    } else if (c->kind[which] == KIND_BULK && pmlk) {
      fn = reinterpret_cast<const void*>(pick_bulk_kernel(c->N, c->att, mode, smem));
    } else if (c->kind[which] == KIND_BULK && c->att) {
      fn = reinterpret_cast<const void*>(pick_main_bulk_kernel(c->N, mode, smem));
    } else {
      fn = reinterpret_cast<const void*>(pick_kernel(c->N, c->att, pmlk, mode, smem));
    }
    if (!fn) return set_err(c, NEXD_ERR_UNSUPPORTED, "no stage kernel for this order and contraction");
    CUDA_TRY(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kind_threads(c->kind[which], pmlk), smem));
    if (per_sm < 1) return set_err(c, NEXD_ERR_UNSUPPORTED, "stage kernel does not fit on an SM");
    const int nel = pmlk ? c->Kpml : c->K - c->Kpml;
    const long long work = (long long)((nel + E - 1) / E) * c->nbatch;
    const int grid = int(std::max<long long>(1, std::min<long long>(work, (long long)per_sm * c->nsm / c->grid_div)));
    if (pmlk) { c->grid_pml = grid; c->smem_pml = smem; }
    else { c->grid_main = grid; c->smem_main = smem; }
  }
  return NEXD_OK;
}

}  // extern "C"

namespace {

int create_impl(const nexd_desc* d, const nexd_halo_desc* h, nexd_ctx** out) {
  if (!out) return set_err(nullptr, NEXD_ERR_INVALID, "null output pointer");
  *out = nullptr;
  int st = validate(d, h != nullptr);
  if (st) return st;
  if (h && (st = validate_halo(d, h))) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_err(nullptr, NEXD_ERR_NODEVICE, "no CUDA device visible");
  }
  nexd_ctx* c = new nexd_ctx;
  auto fail = [&](int code) {
    g_create_error = c->err;
    nexd_destroy(c);
    return code;
  };
  const int N = d->N, Np = d->Np, NpF = d->NpF, K = d->nelem, NF = 4 * NpF;
  c->N = N; c->Np = Np; c->NpF = NpF; c->K = K;
  // halo slot of each shared face: its position in the halo lists
  std::vector<int> halo_slot;
  if (h) {
    c->partition = h->partition;
    c->npeer = h->npeer;
    halo_slot.assign(size_t(4) * K, -1);
    for (int p = 0; p < h->npeer; ++p) {
      c->peer_part.push_back(h->peer[p]);
      c->peer_nface.push_back(h->nface[p]);
      c->peer_goff.push_back(c->nhalo);
      for (int i = 0; i < h->nface[p]; ++i, ++c->nhalo)
        halo_slot[size_t(4) * (h->elem[c->nhalo] - 1) + (h->side[c->nhalo] - 1)] = c->nhalo;
    }
  }
  c->att = d->attenuation != 0;
  c->pml = d->set_pml != 0;
  c->nMB = c->att ? d->nMB : 0;
  c->nt = d->nt;
  c->timeint = d->timeint;
  c->nstage = d->timeint == 4 ? 5 : (d->timeint == 3 ? 3 : (d->timeint == 2 ? 2 : 1));
  c->nbatch = d->nbatch;
  c->dt = d->dt;
  c->nsrc = d->nsrc;
  c->nrec = d->nrec;
  c->nspt = d->stf_per_step;
  if (cudaGetDevice(&c->device) != cudaSuccess) return fail(set_err(c, NEXD_ERR_CUDA, "cudaGetDevice failed"));
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_err(c, NEXD_ERR_CUDA, "cudaStreamCreate failed"));

  // ---- internal element order: PML elements first, each group in mesh order ----
  c->new2old.reserve(K);
  if (c->pml)
    for (int e = 0; e < K; ++e)
      if (d->pmlcheck[e]) c->new2old.push_back(e);
  c->Kpml = int(c->new2old.size());
  for (int e = 0; e < K; ++e)
    if (!(c->pml && d->pmlcheck[e])) c->new2old.push_back(e);
  c->old2new.assign(K, 0);
  for (int i = 0; i < K; ++i) c->old2new[c->new2old[i]] = i;

  // ---- face patterns: rows 0..3 own face masks, then neighbour maps ----
  std::vector<unsigned char> pat(size_t(4) * NpF);
  for (int f = 0; f < 4; ++f)
    for (int i = 0; i < NpF; ++i) pat[size_t(f) * NpF + i] = (unsigned char)(d->fmask[f * NpF + i] - 1);
  std::map<std::vector<unsigned char>, int> patid;
  std::vector<int> h_nbr(size_t(K) * 4, -1), h_fcode(size_t(K) * 4, -2);
  for (int ni = 0; ni < K; ++ni) {
    const int e = c->new2old[ni];
    for (int f = 0; f < 4; ++f) {
      const int nb = d->neighbor[4 * e + f];
      const bool shared = nb == 0 && d->face[4 * e + f] == NEXD_FACE_PARTITION;
      if (nb == 0 && !shared) {
        h_fcode[4 * ni + f] = d->face[4 * e + f];  // -1 free, -2 absorbing
        continue;
      }
      // a shared face reads its halo slot in its own face-node order
      std::vector<unsigned char> row(NpF);
      for (int i = 0; i < NpF; ++i) {
        if (shared) {
          row[i] = (unsigned char)i;
          continue;
        }
        const long long gn = (long long)d->ibn[(size_t(e) * 4 + f) * NpF + i] - 1 - (long long)(nb - 1) * Np;
        if (gn < 0 || gn >= Np) return fail(set_err(c, NEXD_ERR_INVALID, "ibn does not point into the neighbour element"));
        row[i] = (unsigned char)gn;
      }
      auto it = patid.find(row);
      int id;
      if (it == patid.end()) {
        id = 4 + int(patid.size());
        patid[row] = id;
        pat.insert(pat.end(), row.begin(), row.end());
      } else {
        id = it->second;
      }
      h_nbr[4 * ni + f] = shared ? K + halo_slot[4 * e + f] : c->old2new[nb - 1];
      h_fcode[4 * ni + f] = id;
    }
  }
  if (patid.size() + 4 > 64) return fail(set_err(c, NEXD_ERR_UNSUPPORTED, "too many distinct face permutations"));
  c->npat = 4 + int(patid.size());

  // ---- element records ----
  std::vector<float> h_geo(size_t(K) * GEO_STRIDE, 0.f);
  for (int ni = 0; ni < K; ++ni) {
    const int e = c->new2old[ni];
    float* g = &h_geo[size_t(ni) * GEO_STRIDE];
    for (int i = 0; i < 9; ++i) g[G_RX + i] = float(d->metric[9 * e + i]);
    for (int f = 0; f < 4; ++f) {
      g[G_FS + f] = float(0.5 * d->fscale[4 * e + f]);
      for (int k = 0; k < 3; ++k) {
        g[G_N + 3 * f + k] = float(d->nnormal[(size_t(e) * 4 + f) * 3 + k]);
        g[G_S + 3 * f + k] = float(d->stangential[(size_t(e) * 4 + f) * 3 + k]);
        g[G_T + 3 * f + k] = float(d->ttangential[(size_t(e) * 4 + f) * 3 + k]);
      }
    }
    const double lam = d->lambdau[e], mu = d->muu[e], rho = d->rho[e], vp = d->vpu[e], vs = d->vsu[e];
    g[G_E1] = float(-(lam + 2 * mu));
    g[G_E2] = float(-lam);
    g[G_E3] = float(-mu);
    g[G_E4] = float(-1.0 / rho);
    g[G_VP] = float(vp);
    g[G_VS] = float(vs);
    g[G_L2M] = float(lam + 2 * mu);
    g[G_MU] = float(mu);
    g[G_LAM] = float(lam);
    g[G_IRHO] = float(1.0 / rho);
    g[G_C] = float(lam / (lam + 2 * mu));
    g[G_IZP] = float(1.0 / (rho * vp));
    g[G_IZS] = float(1.0 / (rho * vs));
    g[G_AP] = float(1.0 / (lam + 2 * mu));
    g[G_AS] = float(1.0 / (2 * mu));
  }
  std::vector<float> h_D(size_t(3) * Np * Np), h_L;
  for (int k = 0; k < Np; ++k)
    for (int n = 0; n < Np; ++n) {
      h_D[size_t(k) * Np + n] = float(d->Dr[size_t(k) * Np + n]);
      h_D[size_t(Np) * Np + size_t(k) * Np + n] = float(d->Ds[size_t(k) * Np + n]);
      h_D[size_t(2) * Np * Np + size_t(k) * Np + n] = float(d->Dt[size_t(k) * Np + n]);
    }
  {
    // LIFT in face-node pairs: [face][pair][n][2], zero where NpF is odd
    const int npair = (NpF + 1) / 2;
    h_L.assign(size_t(4) * npair * Np * 2, 0.f);
    for (int f = 0; f < 4; ++f)
      for (int ip = 0; ip < npair; ++ip)
        for (int n = 0; n < Np; ++n)
          for (int h = 0; h < 2; ++h) {
            const int i = 2 * ip + h;
            if (i < NpF) h_L[((size_t(f) * npair + ip) * Np + n) * 2 + h] = float(d->lift[size_t(f * NpF + i) * Np + n]);
          }
  }
  std::vector<float> h_ael, h_wl;
  if (c->att) {
    h_ael.assign(size_t(K) * 3 * c->nMB, 0.f);
    for (int ni = 0; ni < K; ++ni) {
      const int e = c->new2old[ni];
      for (int l = 0; l < c->nMB; ++l) {
        const double a1 = -d->lambdau[e] * d->ylambda[size_t(e) * c->nMB + l];
        const double a2 = -2.0 * d->muu[e] * d->ymu[size_t(e) * c->nMB + l];
        h_ael[(size_t(ni) * c->nMB + l) * 3 + 0] = float(a1);
        h_ael[(size_t(ni) * c->nMB + l) * 3 + 1] = float(a2);
        h_ael[(size_t(ni) * c->nMB + l) * 3 + 2] = float(a1 + a2);
      }
    }
    for (int l = 0; l < c->nMB; ++l) h_wl.push_back(float(d->wl[l]));
    for (int l = 0; l < c->nMB && l < kNMB; ++l) c->wl_host[l] = h_wl[l];
  }
  std::vector<float> h_prof;
  if (c->pml && c->Kpml > 0) {
    // 4 floats of slack after the last element: the bulk-copy NPML kernel
    // copies a chunk's profiles widened to 16-byte boundaries
    h_prof.assign(size_t(c->Kpml) * 9 * Np + 4, 0.f);
    const size_t ng = size_t(K) * Np;
    for (int ni = 0; ni < c->Kpml; ++ni) {
      const int e = c->new2old[ni];
      for (int p = 0; p < 9; ++p)
        for (int n = 0; n < Np; ++n)
          h_prof[(size_t(ni) * 9 + p) * Np + n] = float(d->pml_profiles[p * ng + size_t(e) * Np + n]);
    }
  }

  // ---- sources: per-element lists and FP64-built patterns ----
  std::vector<int> h_head(K, -1), h_next(std::max(1, c->nsrc), -1), h_sb(std::max(1, c->nsrc), 0);
  std::vector<float> h_spat(size_t(std::max(1, c->nsrc)) * 9 * Np, 0.f);
  for (int i = c->nsrc - 1; i >= 0; --i) {
    const int e = d->srcelem[i] - 1, ni = c->old2new[e];
    h_next[i] = h_head[ni];
    h_head[ni] = i;
    h_sb[i] = (d->nbatch > 1 && d->srcbatch) ? d->srcbatch[i] : 0;
    // invmass * (srcInt * a) / J [/ rho]  (src/timeloopMod.f90:327-356)
    double amp[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (d->srctype[i] == 0) {
      for (int k = 0; k < 3; ++k) amp[6 + k] = d->srcangle_force[3 * i + k] / d->rho[e];
    } else {
      const double* M = &d->srcM[6 * i];  // Mxx Myy Mzz Mxy Mxz Myz -> fields xx yy zz xy yz xz
      amp[0] = M[0]; amp[1] = M[1]; amp[2] = M[2]; amp[3] = M[3]; amp[4] = M[5]; amp[5] = M[4];
    }
    for (int f = 0; f < 9; ++f) {
      if (amp[f] == 0.0) continue;
      for (int n = 0; n < Np; ++n) {
        double acc = 0.0;
        for (int k = 0; k < Np; ++k) acc += d->invmass[size_t(k) * Np + n] * d->srcInt[size_t(i) * Np + k] * amp[f];
        h_spat[(size_t(i) * 9 + f) * Np + n] = float(acc / d->jacobian[e]);
      }
    }
  }
  std::vector<float> h_stf(size_t(std::max(1, c->nsrc)) * c->nt * c->nspt, 0.f);
  for (size_t i = 0; i < size_t(c->nsrc) * c->nt * c->nspt; ++i) h_stf[i] = float(d->stf[i]);

  // ---- receivers ----
  std::vector<int> h_recslot_el(K, -1), h_recelem(std::max(1, c->nrec), 0), h_recslot(std::max(1, c->nrec), 0);
  std::vector<float> h_recInt(size_t(std::max(1, c->nrec)) * Np, 0.f);
  for (int r = 0; r < c->nrec; ++r) {
    const int ni = c->old2new[d->recelem[r] - 1];
    if (h_recslot_el[ni] < 0) h_recslot_el[ni] = c->nslot++;
    h_recelem[r] = ni;
    h_recslot[r] = h_recslot_el[ni];
    for (int n = 0; n < Np; ++n) h_recInt[size_t(r) * Np + n] = float(d->recInt[size_t(r) * Np + n]);
  }

  // ---- device memory ----
  const long long nodes = (long long)(K + c->nhalo) * Np;
  // per-field lengths: q field-major over own and halo nodes; the
  // element-blocked arrays (residual of q, memory variables, NPML
  // auxiliaries) hold each element's F x Np floats padded to a multiple of 4
  // (eblock in stage_kernel.cuh), so F ld >= elements x that
  auto ld_blocked = [&](long long nel, int F) { return F > 0 ? (nel * block_stride(F, Np) + F - 1) / F : 0LL; };
  c->ldq = (std::max(nodes, ld_blocked(K, 9)) + 63) / 64 * 64;
  c->ldt = (ld_blocked(K, 6 * c->nMB) + 63) / 64 * 64;
  c->lda = (ld_blocked(c->Kpml, 27) + 63) / 64 * 64;
  const int nb = c->nbatch;
  if ((st = upload(c, &c->D, h_D)) || (st = upload(c, &c->L, h_L)) || (st = upload(c, &c->geo, h_geo)) ||
      (st = upload(c, &c->patterns, pat)))
    return fail(st);
  {
    std::vector<int4> nb4(K), fc4(K);
    for (int i = 0; i < K; ++i) {
      nb4[i] = make_int4(h_nbr[4 * i], h_nbr[4 * i + 1], h_nbr[4 * i + 2], h_nbr[4 * i + 3]);
      fc4[i] = make_int4(h_fcode[4 * i], h_fcode[4 * i + 1], h_fcode[4 * i + 2], h_fcode[4 * i + 3]);
    }
    if ((st = upload(c, &c->nbr, nb4)) || (st = upload(c, &c->fcode, fc4))) return fail(st);
    // absorbing faces in internal element order: the learned boundary's ghost slots
    std::vector<int> bfe, bff;
    std::vector<int4> fl4 = fc4;
    for (int i = 0; i < K; ++i) {
      int* cs = reinterpret_cast<int*>(&fl4[i]);
      for (int f = 0; f < 4; ++f)
        if (cs[f] == -2) {
          cs[f] = -3 - int(bfe.size());
          bfe.push_back(i);
          bff.push_back(f);
        }
    }
    c->nbf = int(bfe.size());
    if (c->nbf > 0 &&
        ((st = upload(c, &c->bf_elem, bfe)) || (st = upload(c, &c->bf_face, bff)) || (st = upload(c, &c->fcode_learned, fl4))))
      return fail(st);
  }
  const int nq = (c->timeint == 3) ? 3 : 2;
  for (int i = 0; i < nq; ++i) {
    // + 4 floats of slack: the bulk-copy NPML kernel reads a chunk's rows
    // widened to 16-byte boundaries (TVD step-start wavefield)
    if ((st = dalloc(c, &c->qbuf[i], size_t(nb) * 9 * c->ldq + 4))) return fail(st);
    if ((st = fill(c, c->qbuf[i], size_t(nb) * 9 * c->ldq + 4, float(d->init_value)))) return fail(st);
    c->init_value = float(d->init_value);
  }
  if (h) {
    // this partition's shared face nodes in neighbour order: own node, and
    // the node offset in the neighbour's halo (slot of the same face there,
    // matching node)
    std::vector<int> hs, hd, blocks;
    for (int p = 0, i = 0; p < c->npeer; ++p) {
      HaloPeer hp{};
      hp.entry0 = int(hs.size());
      hp.block0 = c->put_blocks;
      for (int k = 0; k < c->peer_nface[p]; ++k, ++i) {
        const int ni = c->old2new[h->elem[i] - 1], f = h->side[i] - 1;
        for (int j = 0; j < NpF; ++j) {
          hs.push_back(ni * Np + d->fmask[f * NpF + j] - 1);
          hd.push_back((h->peer_index[i] - 1) * Np + h->peer_node[i * NpF + j] - 1);
        }
      }
      hp.nentry = int(hs.size()) - hp.entry0;
      const int nbk = (hp.nentry + kHaloThreads - 1) / kHaloThreads;
      blocks.push_back(nbk);  // the neighbour sends the same number (same shared faces)
      c->put_blocks += nbk;
      c->peers_h.push_back(hp);
    }
    c->peer_linked.assign(size_t(c->npeer), 0);
    if (c->npeer > 0) {
      if ((st = upload(c, &c->halo_src, hs)) || (st = upload(c, &c->halo_dst, hd)) ||
          (st = upload(c, &c->halo_blocks, blocks)) || (st = dalloc(c, &c->peers_dev, size_t(c->npeer))) ||
          (st = dalloc(c, &c->halo_counters, size_t(c->npeer))) || (st = dalloc(c, &c->halo_expected, size_t(c->npeer))))
        return fail(st);
      CUDA_TRY(c, cudaMemset(c->halo_counters, 0, c->npeer * sizeof(unsigned long long)));
      CUDA_TRY(c, cudaMemset(c->halo_expected, 0, c->npeer * sizeof(unsigned long long)));
    }
  }
  if (c->timeint == 4) {
    if ((st = dalloc(c, &c->res, size_t(nb) * 9 * c->ldq + 4))) return fail(st);  // + slack, as above
    CUDA_TRY(c, cudaMemset(c->res, 0, (size_t(nb) * 9 * c->ldq + 4) * sizeof(float)));
  }
  if (c->att) {
    const size_t n = size_t(nb) * 6 * c->nMB * c->ldt + 4;  // + slack, as above
    if ((st = dalloc(c, &c->th, n)) || (st = dalloc(c, &c->th2, n))) return fail(st);
    if ((st = fill(c, c->th, n, float(d->init_value)))) return fail(st);
    CUDA_TRY(c, cudaMemset(c->th2, 0, n * sizeof(float)));
    if ((st = upload(c, &c->ael, h_ael)) || (st = upload(c, &c->wl, h_wl))) return fail(st);
  }
  if (c->pml && c->Kpml > 0) {
    // + 4 floats of slack: the bulk-copy NPML kernel copies a chunk's
    // auxiliaries widened to 16-byte boundaries
    const size_t n = size_t(nb) * 27 * c->lda + 4;
    if ((st = dalloc(c, &c->aux, n)) || (st = dalloc(c, &c->aux2, n))) return fail(st);
    CUDA_TRY(c, cudaMemset(c->aux, 0, n * sizeof(float)));
    CUDA_TRY(c, cudaMemset(c->aux2, 0, n * sizeof(float)));
    if ((st = upload(c, &c->prof_dev, h_prof))) return fail(st);
  }
  if ((st = upload(c, &c->src_head, h_head)) || (st = upload(c, &c->src_next, h_next)) ||
      (st = upload(c, &c->src_batch, h_sb)) || (st = upload(c, &c->src_pat, h_spat)) || (st = upload(c, &c->stf, h_stf)))
    return fail(st);
  if ((st = upload(c, &c->rec_slot, h_recslot_el)) || (st = upload(c, &c->recelem, h_recelem)) ||
      (st = upload(c, &c->recslot_of_rec, h_recslot)) || (st = upload(c, &c->recInt, h_recInt)))
    return fail(st);
  {
    const size_t na = size_t(nb) * std::max(1, c->nslot) * 3 * Np;
    if ((st = dalloc(c, &c->abuf, na)) || (st = fill(c, c->abuf, na, float(d->init_value)))) return fail(st);
    // u accumulators start at the interpolated start value sum_j recInt(j) * init
    std::vector<float> h_u(size_t(nb) * std::max(1, c->nrec) * 3, 0.f);
    for (int b = 0; b < nb; ++b)
      for (int r = 0; r < c->nrec; ++r) {
        double s = 0.0;
        for (int n = 0; n < Np; ++n) s += float(d->recInt[size_t(r) * Np + n]) * float(d->init_value);
        for (int k = 0; k < 3; ++k) h_u[(size_t(b) * c->nrec + r) * 3 + k] = float(s);
      }
    if ((st = upload(c, &c->u, h_u))) return fail(st);
    const size_t nt_ = size_t(nb) * std::max(1, c->nrec) * c->nt * 9;
    if ((st = dalloc(c, &c->traces, nt_))) return fail(st);
    CUDA_TRY(c, cudaMemset(c->traces, 0, nt_ * sizeof(float)));
    if ((st = dalloc(c, &c->flag, 1))) return fail(st);
    CUDA_TRY(c, cudaMemset(c->flag, 0, sizeof(int)));
    if ((st = dalloc(c, &c->pml_off, size_t(nb))) || (st = dalloc(c, &c->pml_switch, size_t(nb)))) return fail(st);
    if ((st = dalloc(c, &c->it_dev, 1))) return fail(st);
    CUDA_TRY(c, cudaMemset(c->it_dev, 0, sizeof(int)));
    CUDA_TRY(c, cudaMemset(c->pml_off, 0, nb * sizeof(int)));
    CUDA_TRY(c, cudaMemset(c->pml_switch, 0, nb * sizeof(int)));
    // mass matrix M = (V V^T)^-1 and per-element energy constants, for the NPML trigger
    if (c->pml) {
      std::vector<double> Mi(d->invmass, d->invmass + size_t(Np) * Np), Mo(size_t(Np) * Np, 0.0);
      for (int i = 0; i < Np; ++i) Mo[size_t(i) * Np + i] = 1.0;
      for (int col = 0; col < Np; ++col) {  // Gauss-Jordan with partial pivoting
        int p = col;
        for (int r = col + 1; r < Np; ++r)
          if (std::fabs(Mi[size_t(col) * Np + r]) > std::fabs(Mi[size_t(col) * Np + p])) p = r;
        for (int j = 0; j < Np; ++j) {
          std::swap(Mi[size_t(j) * Np + col], Mi[size_t(j) * Np + p]);
          std::swap(Mo[size_t(j) * Np + col], Mo[size_t(j) * Np + p]);
        }
        const double piv = Mi[size_t(col) * Np + col];
        if (piv == 0.0) return fail(set_err(c, NEXD_ERR_INVALID, "singular invmass"));
        for (int j = 0; j < Np; ++j) { Mi[size_t(j) * Np + col] /= piv; Mo[size_t(j) * Np + col] /= piv; }
        for (int r = 0; r < Np; ++r) {
          if (r == col) continue;
          const double f = Mi[size_t(col) * Np + r];
          if (f == 0.0) continue;
          for (int j = 0; j < Np; ++j) {
            Mi[size_t(j) * Np + r] -= f * Mi[size_t(j) * Np + col];
            Mo[size_t(j) * Np + r] -= f * Mo[size_t(j) * Np + col];
          }
        }
      }
      std::vector<double> h_mass(size_t(Np) * Np);  // row-major M(n,k)
      for (int n = 0; n < Np; ++n)
        for (int k = 0; k < Np; ++k) h_mass[size_t(n) * Np + k] = Mo[size_t(k) * Np + n];
      std::vector<float4> h_emat(K);
      for (int ni = 0; ni < K; ++ni) {
        const int e = c->new2old[ni];
        h_emat[ni] = make_float4(float(d->rho[e]), float(d->lambdau[e]), float(d->muu[e]), float(d->jacobian[e]));
      }
      if ((st = upload(c, &c->mass, h_mass)) || (st = upload(c, &c->emat, h_emat))) return fail(st);
    }
  }
  // ---- launch configuration ----
  if (tc_order_supported(N)) {
    std::vector<uint16_t> ops = pack_tc_operator<4>(d);
    std::vector<uint4> ops4(ops.size() * 2 / sizeof(uint4));
    std::memcpy(ops4.data(), ops.data(), ops4.size() * sizeof(uint4));
    if ((st = upload(c, &c->ops_tc, ops4))) return fail(st);
  }
  if ((st = configure_launch(c))) return fail(st);
  // pinned staging of nexd_step_io: (stf_per_step, nsrc) samples in, (nrec,
  // 9, nbatch) samples out; allocated here so that no streaming step pays for it
  c->pinned_floats = std::max<size_t>(1, size_t(c->nspt) * c->nsrc + size_t(c->nrec) * 9 * c->nbatch);
  if (cudaMallocHost(&c->pinned, c->pinned_floats * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    c->pinned = nullptr;
    return fail(set_err(c, NEXD_ERR_NOMEM, "pinned staging buffer for nexd_step_io"));
  }
  CUDA_TRY(c, cudaDeviceSynchronize());
  *out = c;
  return NEXD_OK;
}

}  // namespace

extern "C" {

int nexd_create(const nexd_desc* d, nexd_ctx** out) { return create_impl(d, nullptr, out); }

int nexd_create_partition(const nexd_desc* d, const nexd_halo_desc* h, nexd_ctx** out) {
  if (!h) {
    if (out) *out = nullptr;
    return set_err(nullptr, NEXD_ERR_INVALID, "null halo descriptor");
  }
  return create_impl(d, h, out);
}

namespace {

int ev_begin(nexd_ctx* c, int kind) {
  if (!c->profiling) return -1;
  const int pair = c->ev_used++;
  while (int(c->events.size()) < 2 * c->ev_used) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    c->events.push_back(e);
  }
  if (int(c->ev_kind.size()) < c->ev_used) c->ev_kind.resize(c->ev_used);
  c->ev_kind[pair] = kind;
  cudaEventRecord(c->events[2 * pair], c->stream);
  return pair;
}

void ev_end(nexd_ctx* c, int pair) {
  if (pair >= 0) cudaEventRecord(c->events[2 * pair + 1], c->stream);
}

// Collects the timed pairs after the stream is synchronised.
void ev_collect(nexd_ctx* c) {
  for (int p = 0; p < c->ev_used; ++p) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->events[2 * p], c->events[2 * p + 1]) == cudaSuccess) {
      c->prof.ms[c->ev_kind[p]] += ms;
      c->prof.launches[c->ev_kind[p]] += 1;
    }
  }
  c->ev_used = 0;
}

// u += dt v at every node (after the step, as src/timeloopMod.f90:482-485) and,
// every `frame`-th step, the element mean of |u| (collectMovieMod.f90's cell
// value) into frame slot it/frame - 1.  Block: 256 threads = E elements x Np nodes.
__global__ void movie_kernel(const float* q, float* u, long long ldq, int K, int Np, int nbatch, float dt,
                             const int* it_dev, int frame, int max_frames, float* frames) {
  __shared__ float red[256];
  const int E = 256 / Np;
  const int le = threadIdx.x / Np, n = threadIdx.x - le * Np;
  const int b = blockIdx.y;
  const int e = blockIdx.x * E + le;
  float mag = 0.f;
  if (le < E && e < K) {
    const long long node = (long long)e * Np + n;
    const float* qb = q + (long long)b * 9 * ldq;
    float* ub = u + (long long)b * 3 * ldq;
    float s2 = 0.f;
    for (int c = 0; c < 3; ++c) {
      const float v = ub[c * ldq + node] + dt * qb[(6 + c) * ldq + node];
      ub[c * ldq + node] = v;
      s2 += v * v;
    }
    mag = sqrtf(s2);
  }
  red[threadIdx.x] = mag;
  __syncthreads();
  const int it = *it_dev;
  if (it % frame != 0 || it / frame > max_frames) return;
  if (le < E && n == 0 && e < K) {
    float sum = 0.f;
    for (int k = 0; k < Np; ++k) sum += red[le * Np + k];
    frames[((long long)(it / frame - 1) * nbatch + b) * K + e] = sum / Np;
  }
}

__global__ void set_step_kernel(int* it_dev, int it) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *it_dev = it;
}

// Enqueues `nsteps` steps on the context's stream; the step number comes from
// the device counter (set before, advanced by tick_kernel after each step).
using GhostTcFn = void (*)(const GhostTcArgs);
GhostTcFn ghost_tc_fn(int NpF) {
  switch (NpF) {
    case 3: return ghost_tc_kernel<3>;
    case 6: return ghost_tc_kernel<6>;
    case 10: return ghost_tc_kernel<10>;
    case 15: return ghost_tc_kernel<15>;
    case 21: return ghost_tc_kernel<21>;
    default: return nullptr;
  }
}

// Launches the stage kernel of one element class (NPML elements first in the
// internal order, then the rest) with the kernel kind chosen for it.
void launch_class(nexd_ctx* c, StageArgs& a, bool pml) {
  const int mode = c->timeint == 4 ? MODE_LSERK : MODE_TVD;
  const int cls = pml ? 0 : 1;
  size_t smem = 0;
  a.e_begin = pml ? 0 : c->Kpml;
  a.e_end = pml ? c->Kpml : c->K;
  const int grid = pml ? c->grid_pml : c->grid_main;
  const size_t sm = pml ? c->smem_pml : c->smem_main;
  if (c->kind[cls] == NEXD_CONTRACT_BF16X3) {
    TcKernelFn f = pick_tc_kernel(c->N, c->att, pml, mode, smem);
    f<<<grid, 256, sm, c->stream>>>(a, c->ops_tc);
  } else if (c->kind[cls] == KIND_FP32_PAIRS && !pml) {
    KernelFn f = pick_pair_kernel(c->N, c->att, mode, smem);
    f<<<grid, 256, sm, c->stream>>>(a);
  } else if (c->kind[cls] == KIND_BULK && pml) {
    KernelFn f = pick_bulk_kernel(c->N, c->att, mode, smem);
    f<<<grid, kBulkThreads, sm, c->stream>>>(a);
  } else if (c->kind[cls] == KIND_BULK && c->att) {
    KernelFn f = pick_main_bulk_kernel(c->N, mode, smem);
    f<<<grid, 256, sm, c->stream>>>(a);
  } else {
    KernelFn f = pick_kernel(c->N, c->att, pml, mode, smem);
    f<<<grid, 256, sm, c->stream>>>(a);
  }
}

// Stage arguments that do not change from stage to stage.
StageArgs base_args(nexd_ctx* c) {
  StageArgs a{};
  a.flag = c->flag;
  a.nbatch = c->nbatch;
  a.nMB = c->nMB;
  a.ldq = c->ldq;
  a.ldt = c->ldt;
  a.lda = c->lda;
  a.D = c->D;
  a.L = c->L;
  a.geo = c->geo;
  a.nbr = c->nbr;
  a.fcode = c->mlp_on ? c->fcode_learned : c->fcode;
  a.ghost = c->mlp_on ? c->ghost : nullptr;
  a.nbf = c->nbf;
  a.patterns = c->patterns;
  a.npat = c->npat;
  a.ael = c->ael;
  a.wl = c->wl;
  for (int l = 0; l < kNMB; ++l) a.wlv[l] = c->att && l < c->nMB ? c->wl_host[l] : 0.f;
  a.prof = c->prof_dev;
  a.res = c->res;
  a.th = c->th;
  a.th2 = c->th2;
  a.aux = c->aux;
  a.aux2 = c->aux2;
  a.dt = float(c->dt);
  a.src_head = c->src_head;
  a.src_next = c->src_next;
  a.src_batch = c->src_batch;
  a.src_pat = c->src_pat;
  a.stf = c->stf;
  a.nt = c->nt;
  a.nspt = c->nspt;
  a.it_dev = c->it_dev;
  a.rec_slot = c->rec_slot;
  a.abuf = c->abuf;
  a.nslot = std::max(1, c->nslot);
  a.pml_off = c->pml_off;
  return a;
}

// The receiver gather of the current step on `stream` (src/timeloopMod.f90:358-373).
void enqueue_record(nexd_ctx* c, cudaStream_t stream) {
  if (c->nrec * c->nbatch == 0) return;
  RecordArgs r{};
  r.nrec = c->nrec;
  r.nbatch = c->nbatch;
  r.Np = c->Np;
  r.nt = c->nt;
  r.ldq = c->ldq;
  r.recelem = c->recelem;
  r.recslot = c->recslot_of_rec;
  r.recInt = c->recInt;
  r.abuf = c->abuf;
  r.nslot = std::max(1, c->nslot);
  r.u = c->u;
  r.traces = c->traces;
  r.dt = float(c->dt);
  r.flag = c->flag;
  r.it_dev = c->it_dev;
  r.q = c->qbuf[c->cur];
  const int threads = 128;
  const int blocks = (c->nrec * c->nbatch * 32 + threads - 1) / threads;
  record_kernel<<<blocks, threads, 0, stream>>>(r);
  ++c->launches;
}

// Stage arguments of LSERK stage s from the current buffer (the stage writes
// the other one).
void lserk_stage_args(nexd_ctx* c, int s, StageArgs& a) {
  a.stage = s;
  a.last_stage = (s == c->nstage - 1);
  a.stage_first = (s == 0);
  a.ca = float(kRK4A[s]);
  a.cb = float(kRK4B[s]);
  a.q_in = c->qbuf[c->cur];
  a.q_out = c->qbuf[1 - c->cur];
  a.q_n = nullptr;
  a.e_begin = c->Kpml;
  a.e_end = c->K;
}

// The receiver gather at the start of a step.
void enqueue_step_head(nexd_ctx* c) {
  if (c->nrec * c->nbatch == 0) return;
  const int ev = ev_begin(c, NEXD_K_RECORD);
  enqueue_record(c, c->stream);
  ev_end(c, ev);
}

// Arguments of stage s of the current step; *in and *outb receive the
// buffers the stage reads and writes.
void plan_stage(nexd_ctx* c, int s, StageArgs& a, int* in_buf, int* out_buf) {
  a.stage = s;
  a.last_stage = (s == c->nstage - 1);
  a.stage_first = (s == 0);
  int in = c->cur, outb;
  const float* qn = nullptr;
  if (c->timeint == 4) {
    a.ca = float(kRK4A[s]);
    a.cb = float(kRK4B[s]);
    outb = 1 - c->cur;
  } else if (c->timeint == 1) {
    a.ca = 0.f; a.cb = 1.f;
    outb = 1 - c->cur;
  } else if (c->timeint == 2) {
    // stage 1: A -> B; stage 2: (A, B) -> A  (src/rungekuttaMod.f90:90-103)
    if (s == 0) { a.ca = 0.f; a.cb = 1.f; in = c->cur; outb = 1 - c->cur; }
    else { a.ca = 0.5f; a.cb = 0.5f; in = 1 - c->cur; outb = c->cur; qn = c->qbuf[c->cur]; }
  } else {
    // RK3: A -> B; (A,B) -> C; (A,C) -> A  (src/rungekuttaMod.f90:105-120)
    const int A = c->cur, B = (c->cur + 1) % 3, C = (c->cur + 2) % 3;
    if (s == 0) { a.ca = 0.f; a.cb = 1.f; in = A; outb = B; }
    else if (s == 1) { a.ca = 0.75f; a.cb = 0.25f; in = B; outb = C; qn = c->qbuf[A]; }
    else { a.ca = float(1.0 / 3.0); a.cb = float(2.0 / 3.0); in = C; outb = A; qn = c->qbuf[A]; }
  }
  a.q_in = c->qbuf[in];
  a.q_out = c->qbuf[outb];
  a.q_n = qn;
  *in_buf = in;
  *out_buf = outb;
}

// This partition's shared face traces of buffer `in` into its neighbours'
// halo slots (the stage's input), one arrival per write block.
void enqueue_halo_put(nexd_ctx* c, int in) {
  if (c->npeer == 0) return;
  HaloPutArgs h{};
  h.q = c->qbuf[in];
  h.ldq = c->ldq;
  h.nbatch = c->nbatch;
  h.which = in;
  h.npeer = c->npeer;
  h.peers = c->peers_dev;
  h.src = c->halo_src;
  h.dst = c->halo_dst;
  const int ev = ev_begin(c, NEXD_K_HALO);
  halo_put_kernel<<<c->put_blocks, kHaloThreads, 0, c->stream>>>(h);
  ev_end(c, ev);
  ++c->launches;
}

// The stage waits for every neighbour's writes of this stage.
void enqueue_halo_wait(nexd_ctx* c) {
  if (c->npeer == 0) return;
  HaloWaitArgs w{};
  w.counters = c->halo_counters;
  w.expected = c->halo_expected;
  w.blocks = c->halo_blocks;
  w.npeer = c->npeer;
  w.limit_ns = c->halo_limit_ns;
  w.flag = c->flag;
  const int ev = ev_begin(c, NEXD_K_HALO);
  halo_wait_kernel<<<1, 64, 0, c->stream>>>(w);
  ev_end(c, ev);
  ++c->launches;
}

// One stage's element loop: the learned-boundary exterior states (when on),
// then the NPML and the other elements.
void enqueue_stage_kernels(nexd_ctx* c, StageArgs& a) {
  if (c->mlp_on) {
    // exterior states of the absorbing faces from this stage's input
    GhostArgs ga{};
    ga.nbf = c->nbf;
    ga.nbatch = c->nbatch;
    ga.NpF = c->NpF;
    ga.Np = c->Np;
    ga.ldq = c->ldq;
    ga.q = a.q_in;
    ga.bf_elem = c->bf_elem;
    ga.bf_face = c->bf_face;
    ga.geo = c->geo;
    ga.pat = c->patterns;
    ga.w = c->mlp_w;
    ga.rho_max = c->mlp_rho;
    ga.ghost = c->ghost;
    GhostTcArgs ta{ga, c->mlp_wimg, c->flag};
    const int ev = ev_begin(c, NEXD_K_BOUNDARY);
    ghost_tc_fn(c->NpF)<<<c->ghost_grid, kGhostTcThreads, c->ghost_smem, c->stream>>>(ta);
    ev_end(c, ev);
    ++c->launches;
  }
  if (c->Kpml > 0) {
    const int ev = ev_begin(c, NEXD_K_STAGE_PML);
    launch_class(c, a, true);
    ev_end(c, ev);
    ++c->launches;
  }
  if (c->K > c->Kpml) {
    const int ev = ev_begin(c, NEXD_K_STAGE_MAIN);
    launch_class(c, a, false);
    ev_end(c, ev);
    ++c->launches;
  }
}

void end_stage(nexd_ctx* c, int outb) {
  if (c->timeint == 4 || c->timeint == 1) c->cur = outb;
}

// End of a step: NPML energy and trigger, movie frame, step counter.
void enqueue_step_tail(nexd_ctx* c) {
  if (c->energy_on) {
    // wavefield energy of step it and the STA/LTA rule (src/timeloopMod.f90:508-542)
    EnergyArgs ea{};
    ea.K = c->K;
    ea.Np = c->Np;
    ea.nbatch = c->nbatch;
    ea.ldq = c->ldq;
    ea.q = c->qbuf[c->cur];
    ea.emat = c->emat;
    ea.mass = c->mass;
    ea.partials = c->partials;
    ea.formula = c->trig_formula;
    const int E = kEnergyThreads / c->Np;
    const size_t smem = (size_t(c->Np) * c->Np + size_t(E) * 9 * c->Np) * sizeof(double);
    const int ev = ev_begin(c, NEXD_K_ENERGY);
    energy_kernel<<<dim3(c->energy_blocks, c->nbatch), kEnergyThreads, smem, c->stream>>>(ea);
    TriggerArgs ta{};
    ta.partials = c->partials;
    ta.nparts = c->energy_blocks;
    ta.energy = c->energy;
    ta.nt = c->nt;
    ta.it_dev = c->it_dev;
    ta.armed = 1;
    ta.timecrit = c->trig_timecrit;
    ta.w1 = c->trig_w1;
    ta.w2 = c->trig_w2;
    ta.threshold = c->trig_threshold;
    ta.pml_off = c->pml_off;
    ta.pml_switch = c->pml_switch;
    energy_finalize<<<c->nbatch, 256, 0, c->stream>>>(ta);
    ev_end(c, ev);
    c->launches += 2;
  }
  if (c->movie_frame > 0) {
    const int E = 256 / c->Np;
    movie_kernel<<<dim3((c->K + E - 1) / E, c->nbatch), 256, 0, c->stream>>>(
        c->qbuf[c->cur], c->movie_u, c->ldq, c->K, c->Np, c->nbatch, float(c->dt), c->it_dev, c->movie_frame,
        c->movie_max, c->movie_buf);
    ++c->launches;
  }
  tick_kernel<<<1, 32, 0, c->stream>>>(c->it_dev);
  ++c->launches;
}

void enqueue_body(nexd_ctx* c, int nsteps) {
  StageArgs a = base_args(c);
  for (int step = 0; step < nsteps; ++step) {
    enqueue_step_head(c);
    for (int s = 0; s < c->nstage; ++s) {
      int in, outb;
      plan_stage(c, s, a, &in, &outb);
      enqueue_halo_put(c, in);
      enqueue_halo_wait(c);
      enqueue_stage_kernels(c, a);
      end_stage(c, outb);
    }
    enqueue_step_tail(c);
  }
}

void drop_graphs(nexd_ctx* c) {
  for (auto& g : c->gexec)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for (auto& g : c->gexec1)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

// Captures `nsteps` steps starting from the current buffer into *exec and
// counts its kernels; the host-side buffer index advances as the steps do.
int capture_steps(nexd_ctx* c, int nsteps, cudaGraphExec_t* exec, int* nlaunch) {
  const int64_t before = c->launches;
  cudaGraph_t g = nullptr;
  CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  enqueue_body(c, nsteps);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  *nlaunch = int(c->launches - before);  // kernels in the captured graph
  c->launches = before;                  // counted when the graph runs
  if (e != cudaSuccess) return set_err(c, NEXD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_err(c, NEXD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  return NEXD_OK;
}

// Enqueues steps it_begin..it_end: pairs of steps replay a captured two-step
// graph (the ping-pong parity returns to its start after two steps for every
// integrator), a leftover single step replays a one-step graph of its
// starting buffer (the streaming call nexd_step_io runs one step at a time);
// profiled runs launch kernel by kernel.
int enqueue_steps(nexd_ctx* c, int it_begin, int it_end) {
  c->movie_last_it = std::max(c->movie_last_it, it_end);
  set_step_kernel<<<1, 32, 0, c->stream>>>(c->it_dev, it_begin);
  int n = it_end - it_begin + 1;
  if (c->profiling || !c->use_graphs) {
    enqueue_body(c, n);
    return NEXD_OK;
  }
  if (c->graph_energy != c->energy_on) {
    drop_graphs(c);
    c->graph_energy = c->energy_on;
  }
  // LSERK4 and Euler flip the buffer parity every step (an odd number of
  // stages), so runs start at either parity: the graphs of both are captured
  // the first time one is needed, so that no later run pays for a capture
  const bool flips = (c->timeint == 4 || c->timeint == 1) && (c->nstage & 1);
  const int p = c->cur;
  if (n >= 2) {
    for (int k = 0; k < (flips ? 2 : 1); ++k) {
      const int q = k == 0 ? p : 1 - p;
      if (c->gexec[q]) continue;
      c->cur = q;
      const int st = capture_steps(c, 2, &c->gexec[q], &c->graph_launches);
      const int end = c->cur;
      c->cur = p;
      if (st) return st;
      if (end != q) return set_err(c, NEXD_ERR_CUDA, "two-step graph changed the buffer parity");
    }
    for (; n >= 2; n -= 2) {
      CUDA_TRY(c, cudaGraphLaunch(c->gexec[p], c->stream));
      c->launches += c->graph_launches;
    }
  }
  if (n == 1) {
    const int q = c->cur;
    for (int k = 0; k < (flips ? 2 : 1); ++k) {
      const int r = k == 0 ? q : 1 - q;
      if (c->gexec1[r]) continue;
      c->cur = r;
      const int st = capture_steps(c, 1, &c->gexec1[r], &c->graph1_launches[r]);
      c->gend1[r] = c->cur;  // capture advanced the host-side buffer index
      c->cur = q;
      if (st) return st;
    }
    CUDA_TRY(c, cudaGraphLaunch(c->gexec1[q], c->stream));
    c->launches += c->graph1_launches[q];
    c->cur = c->gend1[q];
  }
  return NEXD_OK;
}

// Synchronises, collects profiling events and checks the non-finite flag.
// A partition steps only when every neighbour is linked.
int check_linked(nexd_ctx* c) {
  for (int p = 0; p < c->npeer; ++p)
    if (!c->peer_linked[p])
      return set_err(c, NEXD_ERR_INVALID, "partition not linked to all neighbours (nexd_halo_connect)");
  return NEXD_OK;
}

int finish(nexd_ctx* c) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(c, NEXD_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  int flag = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (c->profiling) ev_collect(c);
  if (flag & 4) return set_err(c, NEXD_ERR_TIMEOUT, "halo arrival wait ran out: a neighbour partition did not write its traces");
  if (flag & 2) return set_err(c, NEXD_ERR_CUDA, "tensor-core completion wait timed out (stage or boundary network kernel)");
  if (flag & 8) return set_err(c, NEXD_ERR_CUDA, "bulk-copy completion wait timed out (NPML stage kernel)");
  if (flag) return set_err(c, NEXD_ERR_NONFINITE, "non-finite value in the wavefield at a receiver");
  return NEXD_OK;
}

}  // namespace

int nexd_run(nexd_ctx* c, int32_t it_begin, int32_t it_end) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (it_begin < 1 || it_end > c->nt || it_begin > it_end) return set_err(c, NEXD_ERR_INVALID, "step range out of 1..nt");
  if (int st = check_linked(c)) return st;
  if (c->span_timing) {
    if (!c->span[0]) {
      CUDA_TRY(c, cudaEventCreate(&c->span[0]));
      CUDA_TRY(c, cudaEventCreate(&c->span[1]));
    }
    CUDA_TRY(c, cudaEventRecord(c->span[0], c->stream));
  }
  if (int st = enqueue_steps(c, it_begin, it_end)) return st;
  if (c->span_timing) CUDA_TRY(c, cudaEventRecord(c->span[1], c->stream));
  int st = finish(c);
  if (c->span_timing && st == NEXD_OK) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->span[0], c->span[1]) == cudaSuccess) c->prof.span_ms += ms;
  }
  return st;
}

int nexd_step_io(nexd_ctx* c, int32_t it, const float* stf_in, float* traces_out) {
  if (!c || !traces_out) return set_err(c, NEXD_ERR_INVALID, "null argument");
  if (it < 1 || it > c->nt) return set_err(c, NEXD_ERR_INVALID, "step out of 1..nt");
  if (int st = check_linked(c)) return st;
  const size_t nin = size_t(c->nspt) * c->nsrc, nout = size_t(c->nrec) * 9 * c->nbatch;
  if (!c->pinned || c->pinned_floats < nin + nout) return set_err(c, NEXD_ERR_INVALID, "no pinned staging buffer");
  if (stf_in && nin > 0) {
    std::memcpy(c->pinned, stf_in, nin * sizeof(float));
    // row s of (nspt, nsrc) goes to stf[s][it-1][:]
    CUDA_TRY(c, cudaMemcpy2DAsync(c->stf + size_t(it - 1) * c->nspt, size_t(c->nt) * c->nspt * sizeof(float), c->pinned,
                                  size_t(c->nspt) * sizeof(float), size_t(c->nspt) * sizeof(float), c->nsrc,
                                  cudaMemcpyHostToDevice, c->stream));
  }
  if (int st = enqueue_steps(c, it, it)) return st;
  if (nout > 0) {
    // (nrec, nt, 9*nbatch) column it-1 -> (nrec, 9*nbatch)
    CUDA_TRY(c, cudaMemcpy2DAsync(c->pinned + nin, size_t(c->nrec) * sizeof(float),
                                  c->traces + size_t(it - 1) * c->nrec, size_t(c->nt) * c->nrec * sizeof(float),
                                  size_t(c->nrec) * sizeof(float), size_t(9) * c->nbatch, cudaMemcpyDeviceToHost,
                                  c->stream));
  }
  int st = finish(c);
  if (st) return st;
  if (nout > 0) std::memcpy(traces_out, c->pinned + nin, nout * sizeof(float));
  return NEXD_OK;
}

namespace {

// Times `reps` launches of one class's stage kernel with the current kind.
// The launches are first stages with cb = 0 (LSERK: ca = 0; TVD: ca = 1) and
// no receiver capture: they rewrite only the residuals, the step-start copies
// and the other wavefield buffer, which the next first stage rewrites anyway,
// and leave theta, the NPML auxiliaries and the current wavefield as they
// were.  The step counter is set to a valid step for the source lookup (every
// run sets it again).
int time_class(nexd_ctx* c, bool pml, int reps, float& ms) {
  StageArgs a = base_args(c);
  a.stage = 0;
  a.stage_first = 1;
  a.last_stage = 0;
  a.ca = c->timeint == 4 ? 0.f : 1.f;
  a.cb = 0.f;
  set_step_kernel<<<1, 32, 0, c->stream>>>(c->it_dev, 1);
  a.q_in = c->qbuf[c->cur];
  a.q_out = c->qbuf[(c->cur + 1) % (c->timeint == 3 ? 3 : 2)];
  a.q_n = c->qbuf[c->cur];
  cudaEvent_t e0, e1;
  CUDA_TRY(c, cudaEventCreate(&e0));
  CUDA_TRY(c, cudaEventCreate(&e1));
  launch_class(c, a, pml);  // warm-up
  CUDA_TRY(c, cudaEventRecord(e0, c->stream));
  for (int i = 0; i < reps; ++i) launch_class(c, a, pml);
  CUDA_TRY(c, cudaEventRecord(e1, c->stream));
  CUDA_TRY(c, cudaEventSynchronize(e1));
  CUDA_TRY(c, cudaGetLastError());
  float t = 0.f;
  CUDA_TRY(c, cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ms = t / float(reps);
  return NEXD_OK;
}

// Picks, per element class, the fastest on this mesh of the FP32 CUDA-core
// kernel, the tensor-core kernel (order 4; FP32-accurate, agrees with the
// FP32 kernel to FP32 rounding, not bit for bit) and the FP32 variants with
// the same results: the node-pair kernel outside the NPML (orders 2-5), the
// kernels with bulk-copied element-local state (NPML elements: orders 3, 4;
// the rest: anelastic models, orders 2-5).
int autotune(nexd_ctx* c) {
  if (int st = finish(c)) return st;  // at a step boundary
  for (int cls = 0; cls < 2; ++cls) {
    const int nel = cls == 0 ? c->Kpml : c->K - c->Kpml;
    if (nel == 0) continue;
    int best = NEXD_CONTRACT_FP32;
    for (int k = 0; k < NKINDS; ++k) {
      if (k == NEXD_CONTRACT_BF16X3 && !tc_order_supported(c->N)) continue;
      if (k == KIND_FP32_PAIRS && (cls == 0 || c->N < 2 || c->N > 5)) continue;
      if (k == KIND_BULK && !bulk_supported(c->N, c->att, cls)) continue;
      c->kind[cls] = k;
      if (int st = configure_launch(c)) return st;
      if (int st = time_class(c, cls == 0, 3, c->tune_ms[cls][k])) return st;
      if (c->tune_ms[cls][k] < c->tune_ms[cls][best]) best = k;
    }
    c->kind[cls] = best;
  }
  return configure_launch(c);
}

}  // namespace

int nexd_set_contraction(nexd_ctx* c, int32_t mode) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (mode != NEXD_CONTRACT_FP32 && mode != NEXD_CONTRACT_BF16X3 && mode != NEXD_CONTRACT_AUTO &&
      mode != NEXD_CONTRACT_FP32_PAIRS)
    return set_err(c, NEXD_ERR_INVALID, "unknown contraction mode");
  if (mode == NEXD_CONTRACT_FP32_PAIRS && (c->N < 2 || c->N > 5))
    return set_err(c, NEXD_ERR_UNSUPPORTED, "the node-pair kernel covers orders 2 to 5");
  if (mode == NEXD_CONTRACT_BF16X3 && !tc_order_supported(c->N))
    return set_err(c, NEXD_ERR_UNSUPPORTED, "the tensor-core contraction covers order 4");
  const int old[2] = {c->kind[0], c->kind[1]};
  int st;
  if (mode == NEXD_CONTRACT_AUTO) {
    st = autotune(c);
  } else if (mode == NEXD_CONTRACT_FP32_PAIRS) {
    c->kind[0] = NEXD_CONTRACT_FP32;
    c->kind[1] = KIND_FP32_PAIRS;
    st = configure_launch(c);
  } else {
    c->kind[0] = c->kind[1] = mode;
    st = configure_launch(c);
  }
  if (st) {
    c->kind[0] = old[0];
    c->kind[1] = old[1];
    configure_launch(c);
    return st;
  }
  c->contraction = mode;
  drop_graphs(c);
  return NEXD_OK;
}

int nexd_set_contraction_kinds(nexd_ctx* c, const int32_t* kinds) {
  if (!c || !kinds) return set_err(c, NEXD_ERR_INVALID, "null argument");
  for (int cls = 0; cls < 2; ++cls) {
    const int k = kinds[cls];
    if (k != NEXD_CONTRACT_FP32 && k != NEXD_CONTRACT_BF16X3 && !(cls == 1 && k == KIND_FP32_PAIRS) &&
        k != KIND_BULK)
      return set_err(c, NEXD_ERR_INVALID, "unknown kernel kind for this element class");
    if (k == KIND_BULK && !bulk_supported(c->N, c->att, cls))
      return set_err(c, NEXD_ERR_UNSUPPORTED,
                     "the bulk-copy kernels cover NPML elements at orders 3 and 4 and anelastic elements at orders 2-5");
    if (k == NEXD_CONTRACT_BF16X3 && !tc_order_supported(c->N))
      return set_err(c, NEXD_ERR_UNSUPPORTED, "the tensor-core contraction covers order 4");
    if (k == KIND_FP32_PAIRS && (c->N < 2 || c->N > 5))
      return set_err(c, NEXD_ERR_UNSUPPORTED, "the node-pair kernel covers orders 2 to 5");
  }
  const int old[2] = {c->kind[0], c->kind[1]};
  c->kind[0] = kinds[0];
  c->kind[1] = kinds[1];
  if (const int st = configure_launch(c)) {
    c->kind[0] = old[0];
    c->kind[1] = old[1];
    configure_launch(c);
    return st;
  }
  drop_graphs(c);
  return NEXD_OK;
}

int nexd_get_contraction(const nexd_ctx* c, int32_t* kinds, float* tune_ms) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (kinds) {
    kinds[0] = c->kind[0];
    kinds[1] = c->kind[1];
  }
  if (tune_ms)
    for (int i = 0; i < 2 * NKINDS; ++i) tune_ms[i] = c->tune_ms[i / NKINDS][i % NKINDS];
  return NEXD_OK;
}

int nexd_pml_trigger(nexd_ctx* c, int32_t avg_window1, int32_t avg_window2, double sta_lta_trigger, double f0,
                     int32_t formula) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (!c->pml) return set_err(c, NEXD_ERR_INVALID, "the STA/LTA trigger needs set_pml");
  if (c->partition > 0)
    return set_err(c, NEXD_ERR_UNSUPPORTED, "the STA/LTA trigger sums the energy of the whole mesh: not on a partition");
  if (avg_window1 < 1 || avg_window2 < 1 || !(f0 > 0.0) || !(sta_lta_trigger >= 0.0) || (formula != 0 && formula != 1))
    return set_err(c, NEXD_ERR_INVALID, "bad trigger parameters");
  c->trig_w1 = avg_window1;
  c->trig_w2 = avg_window2;
  c->trig_threshold = float(sta_lta_trigger);
  c->trig_formula = formula;
  c->trig_timecrit = int(float(2.4 / f0 / c->dt));  // timecrit = 2.4/f0/deltat (integer)
  if (!c->energy) {
    c->energy_blocks = std::max(1, std::min(4 * c->nsm, (c->K + kEnergyThreads / c->Np - 1) / (kEnergyThreads / c->Np)));
    int st;
    if ((st = dalloc(c, &c->energy, size_t(c->nbatch) * c->nt)) ||
        (st = dalloc(c, &c->partials, size_t(c->nbatch) * c->energy_blocks)))
      return st;
    // the attribute is an upper bound shared by all callers of energy_kernel
    CUDA_TRY(c, raise_energy_smem_limit());
  }
  CUDA_TRY(c, cudaMemsetAsync(c->energy, 0, size_t(c->nbatch) * c->nt * sizeof(double), c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->energy_on = true;
  drop_graphs(c);  // the captured trigger launches hold the old parameters
  return NEXD_OK;
}

int nexd_get_energy(nexd_ctx* c, double* energy, int32_t* pml_switch) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (energy) {
    if (!c->energy) {
      std::fill(energy, energy + size_t(c->nbatch) * c->nt, 0.0);
    } else {
      CUDA_TRY(c, cudaMemcpyAsync(energy, c->energy, size_t(c->nbatch) * c->nt * sizeof(double),
                                  cudaMemcpyDeviceToHost, c->stream));
    }
  }
  if (pml_switch)
    CUDA_TRY(c, cudaMemcpyAsync(pml_switch, c->pml_switch, c->nbatch * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return NEXD_OK;
}

// ---- movie snapshots ---------------------------------------------------------

int nexd_movie(nexd_ctx* c, int32_t frame, int32_t max_frames) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (frame < 0 || (frame > 0 && max_frames < 1)) return set_err(c, NEXD_ERR_INVALID, "bad movie arguments");
  drop_graphs(c);
  if (frame == 0) {
    c->movie_frame = 0;
    return NEXD_OK;
  }
  int st;
  if (!c->movie_u) {
    const size_t n = size_t(c->nbatch) * 3 * c->ldq;
    if ((st = dalloc(c, &c->movie_u, n)) || (st = fill(c, c->movie_u, n, c->init_value))) return st;
  }
  if (max_frames > c->movie_max) {
    if ((st = dalloc(c, &c->movie_buf, size_t(max_frames) * c->nbatch * c->K))) return st;
    CUDA_TRY(c, cudaMemset(c->movie_buf, 0, size_t(max_frames) * c->nbatch * c->K * sizeof(float)));
    c->movie_max = max_frames;
  }
  c->movie_frame = frame;
  return NEXD_OK;
}

int nexd_get_movie(nexd_ctx* c, float* out, int32_t* nframes) {
  if (!c || !nframes) return set_err(c, NEXD_ERR_INVALID, "null argument");
  if (c->movie_frame <= 0 || !c->movie_buf) {
    *nframes = 0;
    return NEXD_OK;
  }
  const int nf = std::min(c->movie_max, c->movie_last_it / c->movie_frame);
  *nframes = nf;
  if (!out || nf == 0) return NEXD_OK;
  std::vector<float> h(size_t(nf) * c->nbatch * c->K);
  CUDA_TRY(c, cudaMemcpy(h.data(), c->movie_buf, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
  for (size_t fb = 0; fb < size_t(nf) * c->nbatch; ++fb)
    for (int ni = 0; ni < c->K; ++ni) out[fb * c->K + c->new2old[ni]] = h[fb * c->K + ni];
  return NEXD_OK;
}

// ---- learned absorbing boundary ---------------------------------------------

int nexd_boundary_faces(const nexd_ctx* c, int32_t* nbf, int32_t* elem, int32_t* face) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (nbf) *nbf = c->nbf;
  if ((elem || face) && c->nbf > 0) {
    std::vector<int> e(c->nbf), f(c->nbf);
    CUDA_TRY(const_cast<nexd_ctx*>(c), cudaMemcpy(e.data(), c->bf_elem, c->nbf * sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(const_cast<nexd_ctx*>(c), cudaMemcpy(f.data(), c->bf_face, c->nbf * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < c->nbf; ++i) {
      if (elem) elem[i] = c->new2old[e[i]] + 1;
      if (face) face[i] = f[i] + 1;
    }
  }
  return NEXD_OK;
}

int nexd_set_boundary_mlp(nexd_ctx* c, const float* params, int64_t count, float max_reflection) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (!params) {
    c->mlp_on = false;
    drop_graphs(c);
    return NEXD_OK;
  }
  if (c->nbf == 0) return set_err(c, NEXD_ERR_UNSUPPORTED, "the mesh has no absorbing faces");
  const int nin = 9 * c->NpF;
  if (count != mlp_param_count(nin, kMlpHidden))
    return set_err(c, NEXD_ERR_INVALID, "parameter count does not match a 9 NpF -> 128 -> 128 -> 9 NpF network");
  if (!(max_reflection >= 0.f && max_reflection < 1.f))
    return set_err(c, NEXD_ERR_INVALID, "max_reflection must be in [0, 1)");
  c->mlp_rho = max_reflection;
  int st;
  if (!c->mlp_w) {
    if ((st = dalloc(c, &c->mlp_stage, size_t(count))) || (st = dalloc(c, &c->mlp_w, size_t(count))) ||
        (st = dalloc(c, &c->ghost, size_t(c->nbatch) * c->nbf * 9 * c->NpF)))
      return st;
    const GhostTcLayout L = GhostTcLayout::of(nin);
    GhostTcFn fn = ghost_tc_fn(c->NpF);
    if (!fn) return set_err(c, NEXD_ERR_UNSUPPORTED, "no boundary network kernel for this order");
    if ((st = dalloc(c, &c->mlp_wimg, size_t(L.weights() / 16)))) return st;
    c->ghost_smem = L.smem();
    CUDA_TRY(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(c->ghost_smem)));
    int per_sm = 0;
    CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kGhostTcThreads, c->ghost_smem));
    if (per_sm < 1) return set_err(c, NEXD_ERR_UNSUPPORTED, "boundary network kernel does not fit on an SM");
    const long long tiles = ((long long)c->nbf * c->nbatch + 127) / 128;
    c->ghost_grid = int(std::max<long long>(1, std::min<long long>(tiles, (long long)per_sm * c->nsm)));
  }
  CUDA_TRY(c, cudaMemcpyAsync(c->mlp_stage, params, size_t(count) * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  to_bf16_kernel<<<unsigned((count + 255) / 256), 256, 0, c->stream>>>(count, c->mlp_stage, c->mlp_w);
  pack_ghost_weights_kernel<<<c->nsm, 256, 0, c->stream>>>(nin, c->mlp_w, reinterpret_cast<unsigned char*>(c->mlp_wimg));
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->mlp_on = true;
  drop_graphs(c);
  return NEXD_OK;
}

int nexd_get_ghost(nexd_ctx* c, float* out) {
  if (!c || !out) return set_err(c, NEXD_ERR_INVALID, "null argument");
  if (!c->ghost) return set_err(c, NEXD_ERR_INVALID, "no boundary MLP has been set");
  CUDA_TRY(c, cudaMemcpyAsync(out, c->ghost, size_t(c->nbatch) * c->nbf * 9 * c->NpF * sizeof(float),
                              cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return NEXD_OK;
}

}  // extern "C"

namespace {

// Face traces of the current wavefield: out[b][i][side][9][NpF], side 0 the
// element's own trace, side 1 the neighbour's (zero on boundary faces), both
// in the element's own face-node order.
__global__ void face_trace_kernel(int nf, int nbatch, int Np, int NpF, long long ldq, const float* q, const int* fe,
                                  const int* ff, const int4* nbr, const int4* fcode, const unsigned char* pat,
                                  float* out) {
  const long long n = (long long)nbatch * nf * NpF;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int fi = int(t % NpF);
    const long long bi = t / NpF;
    const int i = int(bi % nf), b = int(bi / nf);
    const int e = fe[i], f = ff[i];
    const float* qb = q + (long long)b * 9 * ldq;
    const long long own = (long long)e * Np + pat[f * NpF + fi];
    const int code = reinterpret_cast<const int*>(fcode)[4 * e + f];
    float* o = out + bi * 2 * 9 * NpF + fi;
    for (int c = 0; c < 9; ++c) o[c * NpF] = qb[c * ldq + own];
    if (code >= 0) {
      const int nb = reinterpret_cast<const int*>(nbr)[4 * e + f];
      const long long other = (long long)nb * Np + pat[code * NpF + fi];
      for (int c = 0; c < 9; ++c) o[(9 + c) * NpF] = qb[c * ldq + other];
    } else {
      for (int c = 0; c < 9; ++c) o[(9 + c) * NpF] = 0.f;
    }
  }
}

}  // namespace

extern "C" {

int nexd_get_face_traces(nexd_ctx* c, int32_t nfaces, const int32_t* elem, const int32_t* face, float* out) {
  if (!c || nfaces < 0 || (nfaces > 0 && (!elem || !face || !out))) return set_err(c, NEXD_ERR_INVALID, "bad arguments");
  if (nfaces == 0) return NEXD_OK;
  std::vector<int> idx(size_t(2) * nfaces);
  for (int i = 0; i < nfaces; ++i) {
    if (elem[i] < 1 || elem[i] > c->K || face[i] < 1 || face[i] > 4)
      return set_err(c, NEXD_ERR_INVALID, "face index out of range");
    idx[i] = c->old2new[elem[i] - 1];
    idx[nfaces + i] = face[i] - 1;
  }
  const size_t nout = size_t(c->nbatch) * nfaces * 2 * 9 * c->NpF;
  if (nfaces > c->gather_cap) {
    int st;
    if ((st = dalloc(c, &c->gather_idx, idx.size())) || (st = dalloc(c, &c->gather_out, nout))) return st;
    c->gather_cap = nfaces;
  }
  CUDA_TRY(c, cudaMemcpyAsync(c->gather_idx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  const long long items = (long long)c->nbatch * nfaces * c->NpF;
  face_trace_kernel<<<unsigned(std::min<long long>((items + 255) / 256, 4096)), 256, 0, c->stream>>>(
      nfaces, c->nbatch, c->Np, c->NpF, c->ldq, c->qbuf[c->cur], c->gather_idx, c->gather_idx + nfaces, c->nbr,
      c->fcode, c->patterns, c->gather_out);
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaMemcpyAsync(out, c->gather_out, nout * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return NEXD_OK;
}

// ---- MLP training kernels (device pointers owned by the caller) ----------------

int64_t nexd_mlp_param_count(int32_t n_in, int32_t n_hidden) { return mlp_param_count(n_in, n_hidden); }

int64_t nexd_mlp_workspace_floats(int32_t n_in, int32_t n_hidden, int32_t batch) {
  // activations and their gradients, loss partials, split-K partial sums
  return 6LL * batch * n_hidden + 2LL * batch * n_in + 256 + kMlpSplitFloats;
}

}  // extern "C"

namespace {

struct MlpView {
  const float *W1, *b1, *W2, *b2, *W3, *b3;
  float *Z1, *A1, *Z2, *A2, *Y, *dY, *dH1, *dH2, *partial, *splitk;
};

MlpView mlp_view(int nin, int H, int B, const float* p, float* work) {
  MlpView v;
  v.W1 = p;
  v.b1 = v.W1 + (long long)H * nin;
  v.W2 = v.b1 + H;
  v.b2 = v.W2 + (long long)H * H;
  v.W3 = v.b2 + H;
  v.b3 = v.W3 + (long long)nin * H;
  const long long BH = (long long)B * H, BI = (long long)B * nin;
  v.Z1 = work;
  v.A1 = v.Z1 + BH;
  v.Z2 = v.A1 + BH;
  v.A2 = v.Z2 + BH;
  v.Y = v.A2 + BH;
  v.dY = v.Y + BI;
  v.dH1 = v.dY + BI;
  v.dH2 = v.dH1 + BH;
  v.partial = v.dH2 + BH;
  v.splitk = v.partial + 256;
  return v;
}

// C = op(A) op(B) (+ C) on the tensor cores (mlp_tc.cuh): one CTA per 128
// rows, K split over CTAs when the rows alone leave SMs idle.
template <bool TA, bool TB>
void gemm(cudaStream_t s, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
          int acc, float* splitk) {
  static bool attr = false;  // one instantiation per (TA, TB)
  if (!attr) {
    cudaFuncSetAttribute(tc_gemm_kernel<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr = true;
  }
  const int NP = tcg_np(N);
  const int mt = (M + 127) / 128, nchunk = (K + 63) / 64;
  int splits = std::min(std::min(kTcgMaxSplits, std::max(1, 148 / mt)), nchunk);
  while (splits > 1 && (long long)splits * M * N > kMlpSplitFloats) --splits;
  const int cper = (nchunk + splits - 1) / splits;
  splits = (nchunk + cper - 1) / cper;  // every split gets at least one chunk
  TcGemmArgs g{M, N, K, A, lda, B, ldb, C, ldc, acc, cper * 64, splitk};
  tc_gemm_kernel<TA, TB><<<dim3(mt, splits), kTcgThreads, tcg_smem_bytes(NP, tcg_nbuf(NP)), s>>>(g);
  if (splits > 1) {
    const long long n = (long long)M * N;
    splitk_reduce_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(M, N, splits, splitk, C, ldc, acc);
  }
}

unsigned blocks_for(long long n) { return unsigned((n + 255) / 256); }

void mlp_forward(cudaStream_t s, int nin, int H, int B, const float* x, const MlpView& v) {
  gemm<false, true>(s, B, H, nin, x, nin, v.W1, nin, v.Z1, H, 0, v.splitk);
  bias_act_kernel<<<blocks_for((long long)B * H), 256, 0, s>>>(B, H, v.Z1, v.b1, v.A1, 1);
  gemm<false, true>(s, B, H, H, v.A1, H, v.W2, H, v.Z2, H, 0, v.splitk);
  bias_act_kernel<<<blocks_for((long long)B * H), 256, 0, s>>>(B, H, v.Z2, v.b2, v.A2, 1);
  gemm<false, true>(s, B, nin, H, v.A2, H, v.W3, H, v.Y, nin, 0, v.splitk);
  bias_act_kernel<<<blocks_for((long long)B * nin), 256, 0, s>>>(B, nin, v.Y, v.b3, v.Y, 0);
}

int mlp_check(int32_t n_in, int32_t n_hidden, int32_t batch) {
  if (n_in < 1 || n_hidden < 1 || batch < 1) return set_err(nullptr, NEXD_ERR_INVALID, "bad MLP dimensions");
  if (n_in > kTcgMaxN || n_hidden > kTcgMaxN)
    return set_err(nullptr, NEXD_ERR_UNSUPPORTED, "MLP layers wider than 256 are not supported");
  return NEXD_OK;
}

int mlp_status() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(nullptr, NEXD_ERR_CUDA, std::string("MLP kernel: ") + cudaGetErrorString(e));
  return NEXD_OK;
}

}  // namespace

extern "C" {

int nexd_mlp_forward(int32_t n_in, int32_t n_hidden, const float* params, const float* x, int32_t batch, float* y,
                     float* work, void* stream) {
  if (int st = mlp_check(n_in, n_hidden, batch)) return st;
  if (!params || !x || !y || !work) return set_err(nullptr, NEXD_ERR_INVALID, "null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  MlpView v = mlp_view(n_in, n_hidden, batch, params, work);
  mlp_forward(s, n_in, n_hidden, batch, x, v);
  cudaMemcpyAsync(y, v.Y, size_t(batch) * n_in * sizeof(float), cudaMemcpyDeviceToDevice, s);
  return mlp_status();
}

int nexd_mlp_loss_grad(int32_t n_in, int32_t n_hidden, const float* params, const float* x, const float* target,
                       int32_t batch, float* grads, float* loss, float* work, void* stream) {
  if (int st = mlp_check(n_in, n_hidden, batch)) return st;
  if (!params || !x || !target || !grads || !loss || !work) return set_err(nullptr, NEXD_ERR_INVALID, "null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nin = n_in, H = n_hidden, B = batch;
  MlpView v = mlp_view(nin, H, B, params, work);
  mlp_forward(s, nin, H, B, x, v);
  float* gW1 = grads;
  float* gb1 = gW1 + (long long)H * nin;
  float* gW2 = gb1 + H;
  float* gb2 = gW2 + (long long)H * H;
  float* gW3 = gb2 + H;
  float* gb3 = gW3 + (long long)nin * H;
  const long long n = (long long)B * nin;
  mse_kernel<<<256, 256, 0, s>>>(n, B, v.Y, target, v.dY, v.partial);
  sum_partials_kernel<<<1, 32, 0, s>>>(256, v.partial, B, loss);
  gemm<true, false>(s, nin, H, B, v.dY, nin, v.A2, H, gW3, H, 0, v.splitk);
  colsum_kernel<<<blocks_for(nin), 256, 0, s>>>(B, nin, v.dY, gb3);
  gemm<false, false>(s, B, H, nin, v.dY, nin, v.W3, H, v.dH2, H, 0, v.splitk);
  gelu_back_kernel<<<blocks_for((long long)B * H), 256, 0, s>>>((long long)B * H, v.dH2, v.Z2);
  gemm<true, false>(s, H, H, B, v.dH2, H, v.A1, H, gW2, H, 0, v.splitk);
  colsum_kernel<<<blocks_for(H), 256, 0, s>>>(B, H, v.dH2, gb2);
  gemm<false, false>(s, B, H, H, v.dH2, H, v.W2, H, v.dH1, H, 0, v.splitk);
  gelu_back_kernel<<<blocks_for((long long)B * H), 256, 0, s>>>((long long)B * H, v.dH1, v.Z1);
  gemm<true, false>(s, H, nin, B, v.dH1, H, x, nin, gW1, nin, 0, v.splitk);
  colsum_kernel<<<blocks_for(H), 256, 0, s>>>(B, H, v.dH1, gb1);
  return mlp_status();
}

int nexd_mlp_adam(int64_t count, float* params, const float* grads, float* m, float* v, int32_t step, float lr,
                  float beta1, float beta2, float eps, void* stream) {
  if (count < 1 || !params || !grads || !m || !v || step < 1) return set_err(nullptr, NEXD_ERR_INVALID, "bad Adam arguments");
  const float c1 = 1.f - std::pow(beta1, float(step)), c2 = 1.f - std::pow(beta2, float(step));
  adam_kernel<<<blocks_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(count, params, grads, m, v, lr, beta1,
                                                                                   beta2, eps, c1, c2);
  return mlp_status();
}

// ---- several models in one CUDA graph --------------------------------------------

}  // extern "C"

struct nexd_group {
  std::vector<nexd_ctx*> m;
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, span[2] = {nullptr, nullptr};
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t gexec = nullptr;
  cudaGraphExec_t gexec_flip = nullptr;  // the same two steps from the other buffer parity
  std::vector<int> parity;       // members' buffer parity when the graph was captured
  std::vector<int> graph_launches;
  float span_ms = 0.f;
  std::string err;
  // execution mode: 0 one CUDA-graph branch per member (each member's own
  // kernels), 1 one persistent launch per stage over all members
  int mode = 0;
  std::vector<int> bfirst;  // mode 1: first block of each member, then the grid size
  size_t gsmem = 0;         // mode 1: dynamic shared memory per block
  float branch_ms = 0.f, persist_ms = 0.f;  // autotune: three probe stages in each mode
};

namespace {

int gerr(nexd_group* g, int code, const std::string& msg) {
  if (g) g->err = msg;
  return set_err(nullptr, code, msg);
}

#define GCUDA(g, call)                                                                         \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return gerr(g, NEXD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

void drop_group_graph(nexd_group* g) {
  for (cudaGraphExec_t* x : {&g->gexec, &g->gexec_flip})
    if (*x) {
      cudaGraphExecDestroy(*x);
      *x = nullptr;
    }
}

// Every member flips its buffer parity each step (LSERK4 and Euler: an odd
// number of stages), so runs start at either parity.
bool members_flip(const nexd_group* g) {
  for (const nexd_ctx* c : g->m)
    if (!((c->timeint == 4 || c->timeint == 1) && (c->nstage & 1))) return false;
  return true;
}

// Members' work forked from the group stream and joined back: `body` enqueues
// one member's work on the member's stream.
template <class F>
int fork_join(nexd_group* g, F body) {
  GCUDA(g, cudaEventRecord(g->fork, g->s));
  for (size_t i = 0; i < g->m.size(); ++i) {
    nexd_ctx* c = g->m[i];
    GCUDA(g, cudaStreamWaitEvent(c->stream, g->fork, 0));
    body(i, c);
    GCUDA(g, cudaEventRecord(g->join[i], c->stream));
    GCUDA(g, cudaStreamWaitEvent(g->s, g->join[i], 0));
  }
  return NEXD_OK;
}

void enqueue_group_persistent(nexd_group* g, int nsteps);

// Captures two steps of every member from their current buffers into *exec.
int capture_group_once(nexd_group* g, cudaGraphExec_t* exec) {
  cudaGraph_t graph = nullptr;
  GCUDA(g, cudaStreamBeginCapture(g->s, cudaStreamCaptureModeThreadLocal));
  std::vector<int64_t> before(g->m.size());
  int st = NEXD_OK;
  if (g->mode == 1) {
    for (size_t i = 0; i < g->m.size(); ++i) before[i] = g->m[i]->launches;
    enqueue_group_persistent(g, 2);
  } else {
    st = fork_join(g, [&](size_t i, nexd_ctx* c) {
      before[i] = c->launches;
      enqueue_body(c, 2);
    });
  }
  cudaError_t e = cudaStreamEndCapture(g->s, &graph);
  for (size_t i = 0; i < g->m.size(); ++i) {
    g->graph_launches[i] = int(g->m[i]->launches - before[i]);
    g->m[i]->launches = before[i];
    g->parity[i] = g->m[i]->cur;
  }
  if (st) return st;
  if (e != cudaSuccess) return gerr(g, NEXD_ERR_CUDA, std::string("group capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return gerr(g, NEXD_ERR_CUDA, std::string("group instantiate: ") + cudaGetErrorString(e));
  return NEXD_OK;
}

// The group's two-step graph from the members' current buffers and, when
// every member flips parity each step, the one from the other parity too, so
// that no later run pays for a capture.
int capture_group(nexd_group* g) {
  drop_group_graph(g);
  if (int st = capture_group_once(g, &g->gexec)) return st;
  if (!members_flip(g)) return NEXD_OK;
  std::vector<int> base = g->parity;
  for (size_t i = 0; i < g->m.size(); ++i) g->m[i]->cur = 1 - base[i];
  const int st = capture_group_once(g, &g->gexec_flip);
  for (size_t i = 0; i < g->m.size(); ++i) g->m[i]->cur = base[i];
  g->parity = base;
  return st;
}

// Mode 1 covers groups of at most kGroupMax members that all step with LSERK4
// and have orders 2-5, no NPML elements, no energy trigger, movie or learned
// boundary, and an FP32 contraction outside the NPML (the FP32 or the
// bit-identical node-pair kernel: the persistent launch runs the FP32 body).
bool persistent_eligible(const nexd_group* g) {
  if (g->m.size() > size_t(kGroupMax)) return false;
  for (const nexd_ctx* c : g->m)
    if (c->timeint != 4 || c->Kpml > 0 || c->N < 2 || c->N > 5 || c->energy_on || c->movie_frame > 0 ||
        c->mlp_on || c->kind[1] == NEXD_CONTRACT_BF16X3)
      return false;
  return true;
}

// Shared memory of the persistent kernel (the largest order's need) and its
// blocks per SM.
int group_kernel_config(nexd_group* g, int* per_sm) {
  int smax = 0;
  for (const nexd_ctx* c : g->m) smax = std::max(smax, group_smem_floats(c->N));
  g->gsmem = size_t(smax) * sizeof(float);
  const void* fn = reinterpret_cast<const void*>(&group_stage_kernel<MODE_LSERK>);
  GCUDA(g, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(g->gsmem)));
  GCUDA(g, cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, 256, g->gsmem));
  if (*per_sm < 1) return gerr(g, NEXD_ERR_UNSUPPORTED, "the multi-model stage kernel does not fit on an SM");
  return NEXD_OK;
}

// Work items (wavefield, chunk) of a member's stage.
long long member_work(const nexd_ctx* c) {
  const int E = elements_per_chunk(c->N);
  return (long long)((c->K + E - 1) / E) * c->nbatch;
}

// Blocks of each member in proportion to cost[i] (its stage time when it runs
// alone on the whole GPU), at least one and at most its work items.
void share_blocks(nexd_group* g, const std::vector<double>& cost, int total) {
  const int n = int(g->m.size());
  double sum = 0.0;
  for (double x : cost) sum += x;
  g->bfirst.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    const long long want = std::llround(double(total) * cost[i] / std::max(sum, 1e-30));
    g->bfirst[i + 1] = g->bfirst[i] + int(std::max<long long>(1, std::min(member_work(g->m[i]), want)));
  }
}

// A cost model for mode 1 without measurements: work items x Np^2, anelastic
// elements half again as expensive.
std::vector<double> model_cost(const nexd_group* g) {
  std::vector<double> cost;
  for (const nexd_ctx* c : g->m) cost.push_back(double(member_work(c)) * c->Np * c->Np * (c->att ? 1.5 : 1.0));
  return cost;
}

// One persistent launch of stage `args` for every member, on the group stream.
void launch_group_stage(nexd_group* g, const std::vector<StageArgs>& args) {
  GroupStageArgs ga{};
  const int n = int(g->m.size());
  ga.nmodel = n;
  for (int i = 0; i < n; ++i) {
    ga.m[i] = args[i];
    ga.order[i] = g->m[i]->N;
    ga.att[i] = g->m[i]->att ? 1 : 0;
    ga.bfirst[i] = g->bfirst[i];
  }
  ga.bfirst[n] = g->bfirst[n];
  group_stage_kernel<MODE_LSERK><<<g->bfirst[n], 256, g->gsmem, g->s>>>(ga);
  ++g->m[0]->launches;  // one launch for the whole group, counted once
}

// nsteps LSERK4 steps of every member in mode 1: the members' receiver
// gathers, five persistent stage launches, the members' step counters.
void enqueue_group_persistent(nexd_group* g, int nsteps) {
  const int n = int(g->m.size());
  std::vector<StageArgs> args(n);
  for (int i = 0; i < n; ++i) args[i] = base_args(g->m[i]);
  for (int step = 0; step < nsteps; ++step) {
    for (nexd_ctx* c : g->m) enqueue_record(c, g->s);
    for (int st = 0; st < 5; ++st) {
      for (int i = 0; i < n; ++i) lserk_stage_args(g->m[i], st, args[i]);
      launch_group_stage(g, args);
      for (nexd_ctx* c : g->m) c->cur = 1 - c->cur;
    }
    for (nexd_ctx* c : g->m) {
      tick_kernel<<<1, 32, 0, g->s>>>(c->it_dev);
      ++c->launches;
    }
  }
}

// Harmless first-stage launches of every member (as in the contraction autotune).
void enqueue_probe(nexd_ctx* c, int reps) {
  StageArgs a = base_args(c);
  a.stage = 0;
  a.stage_first = 1;
  a.last_stage = 0;
  a.ca = c->timeint == 4 ? 0.f : 1.f;
  a.cb = 0.f;
  a.q_in = c->qbuf[c->cur];
  a.q_out = c->qbuf[(c->cur + 1) % (c->timeint == 3 ? 3 : 2)];
  a.q_n = c->qbuf[c->cur];
  set_step_kernel<<<1, 32, 0, c->stream>>>(c->it_dev, 1);
  for (int r = 0; r < reps; ++r) {
    if (c->Kpml > 0) launch_class(c, a, true);
    if (c->K > c->Kpml) launch_class(c, a, false);
  }
}

}  // namespace

extern "C" {

int nexd_group_create(nexd_ctx* const* members, int32_t n, nexd_group** out) {
  if (!out || !members || n < 1) return set_err(nullptr, NEXD_ERR_INVALID, "bad group arguments");
  *out = nullptr;
  auto* g = new nexd_group();
  for (int i = 0; i < n; ++i) {
    if (!members[i]) {
      delete g;
      return set_err(nullptr, NEXD_ERR_INVALID, "null member");
    }
    for (nexd_ctx* o : g->m)
      if (o == members[i]) {
        delete g;
        return set_err(nullptr, NEXD_ERR_INVALID, "a context appears twice in the group");
      }
    g->m.push_back(members[i]);
  }
  g->join.assign(n, nullptr);
  g->parity.assign(n, -1);
  g->graph_launches.assign(n, 0);
  cudaError_t e = cudaStreamCreateWithFlags(&g->s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming);
  for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&g->join[i], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreate(&g->span[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&g->span[1]);
  if (e != cudaSuccess) {
    nexd_group_destroy(g);
    return set_err(nullptr, NEXD_ERR_CUDA, std::string("group set-up: ") + cudaGetErrorString(e));
  }
  *out = g;
  return NEXD_OK;
}

int nexd_group_run(nexd_group* g, int32_t it_begin, int32_t it_end) {
  if (!g) return set_err(nullptr, NEXD_ERR_INVALID, "null group");
  for (nexd_ctx* c : g->m) {
    if (it_begin < 1 || it_end > c->nt || it_begin > it_end)
      return gerr(g, NEXD_ERR_INVALID, "step range out of 1..nt of a member");
    if (c->profiling) return gerr(g, NEXD_ERR_INVALID, "per-launch timing is on in a member");
  }
  GCUDA(g, cudaEventRecord(g->span[0], g->s));
  for (nexd_ctx* c : g->m) {
    set_step_kernel<<<1, 32, 0, g->s>>>(c->it_dev, it_begin);
    c->movie_last_it = std::max(c->movie_last_it, it_end);
  }
  int n = it_end - it_begin + 1;
  if (n >= 2) {
    bool same = g->gexec != nullptr, flipped = g->gexec_flip != nullptr;
    for (size_t i = 0; i < g->m.size(); ++i) {
      same = same && g->parity[i] == g->m[i]->cur;
      flipped = flipped && g->parity[i] == 1 - g->m[i]->cur;
    }
    if (!same && !flipped) {
      if (int st = capture_group(g)) return st;
      same = true;
    }
    cudaGraphExec_t x = same ? g->gexec : g->gexec_flip;
    for (; n >= 2; n -= 2) {
      GCUDA(g, cudaGraphLaunch(x, g->s));
      for (size_t i = 0; i < g->m.size(); ++i) g->m[i]->launches += g->graph_launches[i];
    }
  }
  if (n == 1) {
    if (g->mode == 1) {
      enqueue_group_persistent(g, 1);
    } else if (int st = fork_join(g, [&](size_t, nexd_ctx* c) { enqueue_body(c, 1); })) {
      return st;
    }
  }
  GCUDA(g, cudaEventRecord(g->span[1], g->s));
  GCUDA(g, cudaEventSynchronize(g->span[1]));
  GCUDA(g, cudaEventElapsedTime(&g->span_ms, g->span[0], g->span[1]));
  for (nexd_ctx* c : g->m)
    if (int st = finish(c)) return gerr(g, st, c->err);
  return NEXD_OK;
}

int nexd_group_autotune(nexd_group* g, int32_t* divisor) {
  if (!g) return set_err(nullptr, NEXD_ERR_INVALID, "null group");
  const int cand[3] = {1, 2, 4};
  float best_ms = 0.f;
  int best = 1;
  for (int k = 0; k < 3; ++k) {
    for (nexd_ctx* c : g->m) {
      c->grid_div = cand[k];
      if (int st = configure_launch(c)) return gerr(g, st, c->err);
    }
    if (int st = fork_join(g, [&](size_t, nexd_ctx* c) { enqueue_probe(c, 1); })) return st;  // warm-up
    GCUDA(g, cudaEventRecord(g->span[0], g->s));
    if (int st = fork_join(g, [&](size_t, nexd_ctx* c) { enqueue_probe(c, 3); })) return st;
    GCUDA(g, cudaEventRecord(g->span[1], g->s));
    GCUDA(g, cudaEventSynchronize(g->span[1]));
    GCUDA(g, cudaGetLastError());
    float ms = 0.f;
    GCUDA(g, cudaEventElapsedTime(&ms, g->span[0], g->span[1]));
    if (k == 0 || ms < best_ms) {
      best_ms = ms;
      best = cand[k];
    }
  }
  // mode 1: each member's stage alone on the whole GPU sets its block share;
  // three probe stages of the persistent launch against the best branch time
  g->mode = 0;
  if (persistent_eligible(g)) {
    std::vector<double> cost;
    for (nexd_ctx* c : g->m) {
      c->grid_div = 1;
      if (int st = configure_launch(c)) return gerr(g, st, c->err);
      float ms = 0.f;
      if (int st = time_class(c, false, 3, ms)) return gerr(g, st, c->err);
      cost.push_back(ms);
    }
    int per_sm = 0;
    if (int st = group_kernel_config(g, &per_sm)) return st;
    share_blocks(g, cost, per_sm * g->m[0]->nsm);
    std::vector<StageArgs> args;
    for (nexd_ctx* c : g->m) {
      StageArgs a = base_args(c);
      lserk_stage_args(c, 0, a);
      a.last_stage = 0;
      a.ca = 0.f;
      a.cb = 0.f;  // rewrites only the residuals and the other buffer, as the contraction autotune's probes
      args.push_back(a);
      set_step_kernel<<<1, 32, 0, g->s>>>(c->it_dev, 1);
    }
    const int64_t l0 = g->m[0]->launches;
    launch_group_stage(g, args);  // warm-up
    GCUDA(g, cudaEventRecord(g->span[0], g->s));
    for (int r = 0; r < 3; ++r) launch_group_stage(g, args);
    GCUDA(g, cudaEventRecord(g->span[1], g->s));
    GCUDA(g, cudaEventSynchronize(g->span[1]));
    GCUDA(g, cudaGetLastError());
    g->m[0]->launches = l0;
    float pms = 0.f;
    GCUDA(g, cudaEventElapsedTime(&pms, g->span[0], g->span[1]));
    g->persist_ms = pms;
    g->branch_ms = best_ms;
    if (pms < best_ms) g->mode = 1;
  }
  for (nexd_ctx* c : g->m) {
    c->grid_div = best;
    if (int st = configure_launch(c)) return gerr(g, st, c->err);
    drop_graphs(c);
  }
  drop_group_graph(g);
  if (divisor) *divisor = best;
  return NEXD_OK;
}

int nexd_group_set_mode(nexd_group* g, int32_t mode) {
  if (!g) return set_err(nullptr, NEXD_ERR_INVALID, "null group");
  if (mode != 0 && mode != 1) return gerr(g, NEXD_ERR_INVALID, "group mode must be 0 or 1");
  if (mode == 1) {
    if (!persistent_eligible(g))
      return gerr(g, NEXD_ERR_UNSUPPORTED,
                  "one persistent launch covers at most 16 LSERK4 members of orders 2-5 without NPML, energy "
                  "trigger, movie, learned boundary or tensor-core contraction");
    int per_sm = 0;
    if (int st = group_kernel_config(g, &per_sm)) return st;
    if (g->bfirst.size() != g->m.size() + 1) share_blocks(g, model_cost(g), per_sm * g->m[0]->nsm);
  }
  g->mode = mode;
  drop_group_graph(g);
  return NEXD_OK;
}

int nexd_group_get_mode(const nexd_group* g, int32_t* mode, int32_t* blocks, double* tune_ms) {
  if (!g) return set_err(nullptr, NEXD_ERR_INVALID, "null group");
  if (mode) *mode = g->mode;
  if (blocks)
    for (size_t i = 0; i < g->m.size(); ++i)
      blocks[i] = g->bfirst.size() == g->m.size() + 1 ? g->bfirst[i + 1] - g->bfirst[i] : 0;
  if (tune_ms) {
    tune_ms[0] = g->branch_ms;
    tune_ms[1] = g->persist_ms;
  }
  return NEXD_OK;
}

int nexd_group_span(const nexd_group* g, double* span_ms) {
  if (!g || !span_ms) return set_err(nullptr, NEXD_ERR_INVALID, "null argument");
  *span_ms = g->span_ms;
  return NEXD_OK;
}

int nexd_group_destroy(nexd_group* g) {
  if (!g) return NEXD_OK;
  if (g->s) cudaStreamSynchronize(g->s);
  drop_group_graph(g);
  if (g->fork) cudaEventDestroy(g->fork);
  for (cudaEvent_t e : g->join)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : g->span)
    if (e) cudaEventDestroy(e);
  if (g->s) cudaStreamDestroy(g->s);
  delete g;
  return NEXD_OK;
}

}  // extern "C"

namespace {

// Scratch of nexd_wavefield_energy_noalloc: FP64 block partials of up to
// NEXD_NOALLOC_MAX_BATCH wavefields, then one total per wavefield.  Every GPU
// that loads the library holds it until the process exits.
constexpr int kNoAllocBlocks = 256;
constexpr int kNoAllocSlots = NEXD_NOALLOC_MAX_BATCH * kNoAllocBlocks + NEXD_NOALLOC_MAX_BATCH;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots];

// Device address of g_noalloc_scratch per device, looked up once per device
// with that device current.  Host code must never pass the symbol itself to
// a kernel: on the host it is only a stand-in, not a device address.
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[64] = {};

// Fixed-order sum of each wavefield's partials into its total slot.
__global__ void noalloc_sum(const double* partials, int nparts, double* totals) {
  __shared__ double red[256];
  const int b = blockIdx.x, tid = threadIdx.x;
  double s = 0.0;
  for (int i = tid; i < nparts; i += blockDim.x) s += partials[(long long)b * nparts + i];
  red[tid] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid == 0) totals[b] = red[0];
}

}  // namespace

extern "C" {

int nexd_wavefield_energy_noalloc(const float* q, int64_t ldq, int32_t nelem, int32_t Np, int32_t nbatch,
                                  const float* emat, const double* mass, int32_t formula, double* energy) {
  if (!q || !emat || !mass || !energy) return set_err(nullptr, NEXD_ERR_INVALID, "null argument");
  // The kernel reads emat as 16-byte vectors, mass as FP64 and q as FP32: a
  // misaligned caller pointer (a pool sub-allocation or a tensor view at an
  // odd offset) would fault the GPU, so it is refused before any launch.
  if (reinterpret_cast<uintptr_t>(emat) % 16 != 0)
    return set_err(nullptr, NEXD_ERR_INVALID, "emat must be 16-byte aligned (read as float4)");
  if (reinterpret_cast<uintptr_t>(mass) % 8 != 0)
    return set_err(nullptr, NEXD_ERR_INVALID, "mass must be 8-byte aligned (FP64)");
  if (reinterpret_cast<uintptr_t>(q) % 4 != 0 || reinterpret_cast<uintptr_t>(energy) % 8 != 0)
    return set_err(nullptr, NEXD_ERR_INVALID, "q must be 4-byte aligned and energy 8-byte aligned");
  if (nelem < 1 || Np < 1 || Np > kEnergyThreads || ldq < int64_t(nelem) * Np)
    return set_err(nullptr, NEXD_ERR_INVALID, "bad sizes (need nelem >= 1, 1 <= Np <= 256, ldq >= nelem*Np)");
  if (nbatch < 1 || nbatch > NEXD_NOALLOC_MAX_BATCH)
    return set_err(nullptr, NEXD_ERR_INVALID, "nbatch must be 1..64 (size of the static scratch array)");
  if (formula != 0 && formula != 1) return set_err(nullptr, NEXD_ERR_INVALID, "formula must be 0 or 1");
  const int E = kEnergyThreads / Np;
  const size_t smem = (size_t(Np) * Np + size_t(E) * 9 * Np) * sizeof(double);
  if (smem > 200 * 1024) return set_err(nullptr, NEXD_ERR_UNSUPPORTED, "Np too large for the energy kernel");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return set_err(nullptr, NEXD_ERR_NODEVICE, "no usable CUDA device");
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      // one-time set-up on this device (this device is current)
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return set_err(nullptr, NEXD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      e = raise_energy_smem_limit();
      if (e != cudaSuccess)
        return set_err(nullptr, NEXD_ERR_CUDA, std::string("energy kernel set-up: ") + cudaGetErrorString(e));
      g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_noalloc_ptr[dev];
  }
  const int nchunk = (nelem + E - 1) / E;
  const int nblk = std::max(1, std::min(kNoAllocBlocks, nchunk));
  double* partials = scratch;                                   // [nbatch][nblk], every slot written
  double* totals = scratch + NEXD_NOALLOC_MAX_BATCH * kNoAllocBlocks;  // [nbatch], every slot written
  EnergyArgs ea{};
  ea.K = nelem;
  ea.Np = Np;
  ea.nbatch = nbatch;
  ea.ldq = ldq;
  ea.q = q;
  ea.emat = reinterpret_cast<const float4*>(emat);
  ea.mass = mass;
  ea.partials = partials;
  ea.formula = formula;
  // Launched through cudaLaunchKernel so that each launch's own status is
  // checked: an earlier error left in the runtime by the host's other CUDA
  // code is neither reported as this call's failure nor cleared.
  int nparts = nblk;
  void* energy_params[] = {&ea};
  void* sum_params[] = {&partials, &nparts, &totals};
  cudaError_t e = cudaLaunchKernel(reinterpret_cast<const void*>(&energy_kernel), dim3(nblk, nbatch),
                                   dim3(kEnergyThreads), energy_params, smem, nullptr);
  if (e == cudaSuccess)
    e = cudaLaunchKernel(reinterpret_cast<const void*>(&noalloc_sum), dim3(nbatch), dim3(256), sum_params, 0,
                         nullptr);
  if (e != cudaSuccess) {
    cudaGetLastError();  // the launch error is this call's own
    return set_err(nullptr, NEXD_ERR_CUDA, std::string("energy launch: ") + cudaGetErrorString(e));
  }
  e = cudaMemcpy(energy, totals, size_t(nbatch) * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_err(nullptr, NEXD_ERR_CUDA, std::string("energy copy: ") + cudaGetErrorString(e));
  return NEXD_OK;
}

// ---------------------------------------------------------------------------
// Partition halo: export / connect / in-process run
// ---------------------------------------------------------------------------

int nexd_halo_export_peer(nexd_ctx* c, int32_t peer, nexd_halo_export* out) {
  if (!c || !out) return set_err(c, NEXD_ERR_INVALID, "null argument");
  if (peer < 0 || peer >= c->npeer) return set_err(c, NEXD_ERR_INVALID, "neighbour index out of range");
  std::memset(out, 0, sizeof(*out));
  out->abi_version = NEXD_ABI_VERSION;
  out->device = c->device;
  out->pid = int64_t(getpid());
  out->partition = c->partition;
  out->nface = c->peer_nface[peer];
  out->nbatch = c->nbatch;
  out->nbuf = c->timeint == 3 ? 3 : 2;
  out->ldq = c->ldq;
  out->halo_base = (long long)(c->K + c->peer_goff[peer]) * c->Np;
  out->counter_slot = peer;
  for (int i = 0; i < out->nbuf; ++i) {
    out->q[i] = uint64_t(reinterpret_cast<uintptr_t>(c->qbuf[i]));
    cudaIpcMemHandle_t hnd;
    if (cudaIpcGetMemHandle(&hnd, c->qbuf[i]) == cudaSuccess) std::memcpy(out->q_ipc[i], &hnd, 64);
    else cudaGetLastError();  // no IPC here: the export still links partitions of this process
  }
  out->counters = uint64_t(reinterpret_cast<uintptr_t>(c->halo_counters));
  cudaIpcMemHandle_t hnd;
  if (cudaIpcGetMemHandle(&hnd, c->halo_counters) == cudaSuccess) std::memcpy(out->counters_ipc, &hnd, 64);
  else cudaGetLastError();
  return NEXD_OK;
}

int nexd_halo_connect(nexd_ctx* c, int32_t peer, const nexd_halo_export* in) {
  if (!c || !in) return set_err(c, NEXD_ERR_INVALID, "null argument");
  if (peer < 0 || peer >= c->npeer) return set_err(c, NEXD_ERR_INVALID, "neighbour index out of range");
  if (in->abi_version != NEXD_ABI_VERSION) return set_err(c, NEXD_ERR_INVALID, "halo export: ABI version mismatch");
  if (in->partition != c->peer_part[peer])
    return set_err(c, NEXD_ERR_INVALID, "halo export comes from another partition than this neighbour");
  if (in->nface != c->peer_nface[peer])
    return set_err(c, NEXD_ERR_INVALID, "halo export: the neighbour shares a different number of faces");
  if (in->nbatch != c->nbatch || in->nbuf != (c->timeint == 3 ? 3 : 2))
    return set_err(c, NEXD_ERR_INVALID, "halo export: wavefield count or integrator differs from this partition");
  if (in->counter_slot < 0 || in->counter_slot >= kHaloMaxPeers || in->ldq <= 0 || in->halo_base < 0 ||
      in->halo_base + (long long)in->nface * c->Np > in->ldq)
    return set_err(c, NEXD_ERR_INVALID, "halo export: inconsistent layout");
  HaloPeer& hp = c->peers_h[peer];
  hp.ldq = in->ldq;
  hp.base = in->halo_base;
  if (in->pid == int64_t(getpid())) {
    // a partition of this process: its device addresses as they are
    for (int i = 0; i < 3; ++i) hp.q[i] = i < in->nbuf ? reinterpret_cast<float*>(uintptr_t(in->q[i])) : nullptr;
    hp.counter = reinterpret_cast<unsigned long long*>(uintptr_t(in->counters)) + in->counter_slot;
    if (in->device != c->device) {
      const cudaError_t e = cudaDeviceEnablePeerAccess(in->device, 0);
      if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled)
        return set_err(c, NEXD_ERR_CUDA, std::string("peer access to the neighbour's GPU: ") + cudaGetErrorString(e));
      cudaGetLastError();
    }
  } else {
    // another process: open its buffers through CUDA IPC (peer access enabled on first use)
    auto open = [&](const unsigned char* bytes, void** p) -> int {
      cudaIpcMemHandle_t hnd;
      std::memcpy(&hnd, bytes, 64);
      const cudaError_t e = cudaIpcOpenMemHandle(p, hnd, cudaIpcMemLazyEnablePeerAccess);
      if (e != cudaSuccess) return set_err(c, NEXD_ERR_CUDA, std::string("cudaIpcOpenMemHandle: ") + cudaGetErrorString(e));
      c->ipc_opened.push_back(*p);
      return NEXD_OK;
    };
    for (int i = 0; i < 3; ++i) {
      hp.q[i] = nullptr;
      if (i >= in->nbuf) continue;
      void* p = nullptr;
      if (int st = open(in->q_ipc[i], &p)) return st;
      hp.q[i] = static_cast<float*>(p);
    }
    void* p = nullptr;
    if (int st = open(in->counters_ipc, &p)) return st;
    hp.counter = static_cast<unsigned long long*>(p) + in->counter_slot;
  }
  CUDA_TRY(c, cudaMemcpy(c->peers_dev + peer, &hp, sizeof(HaloPeer), cudaMemcpyHostToDevice));
  const unsigned long long zero = 0;
  CUDA_TRY(c, cudaMemcpy(c->halo_counters + peer, &zero, sizeof(zero), cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemcpy(c->halo_expected + peer, &zero, sizeof(zero), cudaMemcpyHostToDevice));
  c->peer_linked[peer] = 1;
  drop_graphs(c);  // captured graphs hold the neighbour table as it was
  return NEXD_OK;
}

int nexd_halo_set_timeout(nexd_ctx* c, double seconds) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (!(seconds > 0.0) || seconds > 60.0) return set_err(c, NEXD_ERR_INVALID, "halo wait limit out of (0, 60] s");
  c->halo_limit_ns = (unsigned long long)(seconds * 1e9);
  drop_graphs(c);  // captured graphs hold the old limit
  return NEXD_OK;
}

int nexd_halo_bytes(const nexd_ctx* c, int64_t* bytes) {
  if (!c || !bytes) return set_err(nullptr, NEXD_ERR_INVALID, "null argument");
  long long n = 0;
  for (int p = 0; p < c->npeer; ++p) n += (long long)c->peer_nface[p] * c->NpF;
  *bytes = n * 9 * c->nbatch * int64_t(sizeof(float));
  return NEXD_OK;
}

int nexd_halo_run(nexd_ctx* const* parts, int32_t n, int32_t it_begin, int32_t it_end) {
  if (!parts || n < 1) return set_err(nullptr, NEXD_ERR_INVALID, "no partitions");
  for (int i = 0; i < n; ++i) {
    nexd_ctx* c = parts[i];
    if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null partition");
    for (int j = 0; j < i; ++j)
      if (parts[j] == c) return set_err(c, NEXD_ERR_INVALID, "partition listed twice");
    if (it_begin < 1 || it_end > c->nt || it_begin > it_end) return set_err(c, NEXD_ERR_INVALID, "step range out of 1..nt");
    if (int st = check_linked(c)) return st;
    if (c->device != parts[0]->device || c->timeint != parts[0]->timeint || c->cur != parts[0]->cur)
      return set_err(c, NEXD_ERR_INVALID, "partitions must share the GPU, the integrator and the step");
  }
  // every neighbour written to must be one of the partitions run here
  for (int i = 0; i < n; ++i)
    for (int p = 0; p < parts[i]->npeer; ++p) {
      bool found = false;
      for (int j = 0; j < n; ++j) found = found || parts[j]->partition == parts[i]->peer_part[p];
      if (!found) return set_err(parts[i], NEXD_ERR_INVALID, "a neighbour partition is not in this run");
    }
  // one stream for all: each stage's writes come before every wait on them
  cudaStream_t s = parts[0]->stream;
  std::vector<cudaStream_t> own(n);
  for (int i = 0; i < n; ++i) {
    own[i] = parts[i]->stream;
    CUDA_TRY(parts[i], cudaStreamSynchronize(own[i]));
    parts[i]->stream = s;
    parts[i]->movie_last_it = std::max(parts[i]->movie_last_it, it_end);
    set_step_kernel<<<1, 32, 0, s>>>(parts[i]->it_dev, it_begin);
  }
  // run span on the shared stream, booked to the first partition
  nexd_ctx* p0 = parts[0];
  if (p0->span_timing) {
    if (!p0->span[0]) {
      CUDA_TRY(p0, cudaEventCreate(&p0->span[0]));
      CUDA_TRY(p0, cudaEventCreate(&p0->span[1]));
    }
    CUDA_TRY(p0, cudaEventRecord(p0->span[0], s));
  }
  std::vector<StageArgs> a(n);
  for (int i = 0; i < n; ++i) a[i] = base_args(parts[i]);
  std::vector<int> in(n), outb(n);
  for (int it = it_begin; it <= it_end; ++it) {
    for (int i = 0; i < n; ++i) enqueue_step_head(parts[i]);
    for (int st = 0; st < parts[0]->nstage; ++st) {
      for (int i = 0; i < n; ++i) {
        plan_stage(parts[i], st, a[i], &in[i], &outb[i]);
        enqueue_halo_put(parts[i], in[i]);
      }
      for (int i = 0; i < n; ++i) {
        enqueue_halo_wait(parts[i]);
        enqueue_stage_kernels(parts[i], a[i]);
        end_stage(parts[i], outb[i]);
      }
    }
    for (int i = 0; i < n; ++i) enqueue_step_tail(parts[i]);
  }
  if (p0->span_timing) CUDA_TRY(p0, cudaEventRecord(p0->span[1], s));
  int status = NEXD_OK;
  for (int i = 0; i < n; ++i) {
    const int st = finish(parts[i]);
    if (st && status == NEXD_OK) status = st;
  }
  if (p0->span_timing && status == NEXD_OK) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p0->span[0], p0->span[1]) == cudaSuccess) p0->prof.span_ms += ms;
  }
  for (int i = 0; i < n; ++i) parts[i]->stream = own[i];
  return status;
}

int nexd_profile_enable(nexd_ctx* c, int32_t on) {
  if (!c) return set_err(nullptr, NEXD_ERR_INVALID, "null context");
  if (on < 0 || on > 2) return set_err(c, NEXD_ERR_INVALID, "timing mode must be 0, 1 or 2");
  c->profiling = on == 1;
  c->span_timing = on != 0;
  c->prof = nexd_profile{};
  c->prof.elements[NEXD_K_STAGE_PML] = c->Kpml;
  c->prof.elements[NEXD_K_STAGE_MAIN] = c->K - c->Kpml;
  c->ev_used = 0;
  return NEXD_OK;
}

int nexd_profile_get(const nexd_ctx* c, nexd_profile* out) {
  if (!c || !out) return NEXD_ERR_INVALID;
  *out = c->prof;
  return NEXD_OK;
}

int nexd_get_traces(nexd_ctx* c, float* out) {
  if (!c || !out) return set_err(c, NEXD_ERR_INVALID, "null argument");
  const size_t n = size_t(c->nbatch) * c->nrec * c->nt * 9;
  if (n == 0) return NEXD_OK;
  CUDA_TRY(c, cudaMemcpyAsync(out, c->traces, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return NEXD_OK;
}

namespace {
// Device layout of a state array: (pointer to batch member b, fields, field
// stride, elements covered).  q is field-major ([field][ld]); the memory
// variables and NPML auxiliaries are element-blocked ([element][field][Np],
// each element's nf x Np floats padded to a multiple of 4, within the batch
// member's nf * ld floats).
int state_view(nexd_ctx* c, int32_t which, int32_t b, float** base, int* nf, long long* ld, int* nel) {
  if (b < 0 || b >= c->nbatch) return set_err(c, NEXD_ERR_INVALID, "batch index out of range");
  if (which == NEXD_STATE_Q) {
    *base = c->qbuf[c->cur] + size_t(b) * 9 * c->ldq;
    *nf = 9; *ld = c->ldq; *nel = c->K;
  } else if (which == NEXD_STATE_THETA) {
    if (!c->att) return set_err(c, NEXD_ERR_INVALID, "no memory variables: attenuation is off");
    *base = c->th + size_t(b) * 6 * c->nMB * c->ldt;
    *nf = 6 * c->nMB; *ld = c->ldt; *nel = c->K;
  } else if (which == NEXD_STATE_PML) {
    if (!c->pml) return set_err(c, NEXD_ERR_INVALID, "no PML auxiliaries: set_pml is off");
    *base = c->aux ? c->aux + size_t(b) * 27 * c->lda : nullptr;
    *nf = 27; *ld = c->lda; *nel = c->Kpml;
  } else {
    return set_err(c, NEXD_ERR_INVALID, "unknown state array");
  }
  return NEXD_OK;
}
}  // namespace

int nexd_get_state(nexd_ctx* c, int32_t which, int32_t b, float* out) {
  if (!c || !out) return set_err(c, NEXD_ERR_INVALID, "null argument");
  float* base;
  int nf, nel;
  long long ld;
  if (int st = state_view(c, which, b, &base, &nf, &ld, &nel)) return st;
  const size_t nodes = size_t(c->K) * c->Np;
  std::fill(out, out + nodes * nf, 0.f);
  if (!base || nel == 0) return NEXD_OK;
  std::vector<float> h(size_t(nf) * ld);
  CUDA_TRY(c, cudaMemcpyAsync(h.data(), base, h.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const bool blocked = which != NEXD_STATE_Q;
  for (int f = 0; f < nf; ++f)
    for (int ni = 0; ni < nel; ++ni) {
      const int e = c->new2old[ni];
      const size_t dev = blocked ? size_t(ni) * block_stride(nf, c->Np) + size_t(f) * c->Np : f * ld + size_t(ni) * c->Np;
      std::memcpy(out + f * nodes + size_t(e) * c->Np, h.data() + dev, c->Np * sizeof(float));
    }
  return NEXD_OK;
}

int nexd_set_state(nexd_ctx* c, int32_t which, int32_t b, const float* in) {
  if (!c || !in) return set_err(c, NEXD_ERR_INVALID, "null argument");
  float* base;
  int nf, nel;
  long long ld;
  if (int st = state_view(c, which, b, &base, &nf, &ld, &nel)) return st;
  if (!base || nel == 0) return NEXD_OK;
  const size_t nodes = size_t(c->K) * c->Np;
  std::vector<float> h(size_t(nf) * ld, 0.f);
  if (which != NEXD_STATE_Q) {  // keep padding / untouched rows as they are
    CUDA_TRY(c, cudaMemcpyAsync(h.data(), base, h.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  const bool blocked = which != NEXD_STATE_Q;
  for (int f = 0; f < nf; ++f)
    for (int ni = 0; ni < nel; ++ni) {
      const int e = c->new2old[ni];
      const size_t dev = blocked ? size_t(ni) * block_stride(nf, c->Np) + size_t(f) * c->Np : f * ld + size_t(ni) * c->Np;
      std::memcpy(h.data() + dev, in + f * nodes + size_t(e) * c->Np, c->Np * sizeof(float));
    }
  CUDA_TRY(c, cudaMemcpyAsync(base, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return NEXD_OK;
}

int nexd_get_field(nexd_ctx* c, int32_t b, float* out) { return nexd_get_state(c, NEXD_STATE_Q, b, out); }

int nexd_set_field(nexd_ctx* c, int32_t b, const float* in) { return nexd_set_state(c, NEXD_STATE_Q, b, in); }

int nexd_last_error(const nexd_ctx* c, char* buf, size_t len) {
  if (!buf || len == 0) return NEXD_ERR_INVALID;
  const std::string& m = c ? c->err : g_create_error;
  std::strncpy(buf, m.c_str(), len - 1);
  buf[len - 1] = '\0';
  return NEXD_OK;
}

int nexd_launch_count(const nexd_ctx* c, int64_t* out) {
  if (!c || !out) return NEXD_ERR_INVALID;
  *out = c->launches;
  return NEXD_OK;
}

int nexd_destroy(nexd_ctx* c) {
  if (!c) return NEXD_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  for (void* p : c->ipc_opened) cudaIpcCloseMemHandle(p);
  for (void* p : c->allocations) cudaFree(p);
  for (cudaEvent_t e : c->events) cudaEventDestroy(e);
  for (cudaEvent_t e : c->span)
    if (e) cudaEventDestroy(e);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return NEXD_OK;
}

}  // extern "C"
