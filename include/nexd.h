/*
 * nexd.h -- C-ABI of the B200 time-stepping library (libnexd.so).
 *
 * Drop-in boundary for NEXD-3D's solver time loop:
 *   subroutine timeloop3D(par, myrank)   src/timeloopMod.f90:42-674
 * called from program_solver.f90:71.  A Fortran host keeps readMesh /
 * readSrc / readRec / prepareSources (src/meshMod.f90:1642-1658,
 * src/sourceReceiverMod.f90:705-839) and the seismogram writers
 * (src/timeloopMod.f90:591-656), fills one nexd_desc with plain pointers to
 * the arrays it already holds, and calls the entry points below through
 * ISO_C_BINDING instead of running the element loop itself.
 *
 * Conventions (all entry points):
 *  - every function returns an int status, NEXD_OK (0) on success; no entry
 *    point calls exit() or stop (the reference stops or MPI_Aborts,
 *    src/mpiMod.f90:287-307);
 *  - arrays are in Fortran (column-major) order with the shapes given in the
 *    comments, integer indices are 1-based as in the reference databases;
 *  - the caller owns every host array; nexd_create copies what it needs, so
 *    the descriptor may be freed after it returns;
 *  - the library owns device memory, one CUDA stream and its CUDA graphs;
 *  - a context is not thread-safe: use one context per host thread.
 */
#ifndef NEXD_H
#define NEXD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NEXD_ABI_VERSION 1

enum nexd_status {
  NEXD_OK = 0,
  NEXD_ERR_INVALID = 1,     /* bad argument or inconsistent descriptor */
  NEXD_ERR_CUDA = 2,        /* CUDA runtime error (message has the details) */
  NEXD_ERR_NOMEM = 3,       /* device allocation failed */
  NEXD_ERR_UNSUPPORTED = 4, /* valid but not supported by this build (e.g. order) */
  NEXD_ERR_NONFINITE = 5,   /* NaN/Inf detected in the wavefield */
  NEXD_ERR_NODEVICE = 6,    /* no CUDA device visible */
  NEXD_ERR_TIMEOUT = 7      /* a halo arrival wait ran out (a peer partition stopped) */
};

/* Face code of a face shared with another partition (nexd_desc.face). */
#define NEXD_FACE_PARTITION (-3)

/* Time integrators: 1..3 are the reference's `timeint` values
 * (src/timeloopMod.f90:230-248, src/rungekuttaMod.f90:27-120); 4 is the
 * Carpenter-Kennedy (1994) 2N-storage 5-stage 4th-order scheme. */
enum nexd_timeint { NEXD_EULER = 1, NEXD_RK2 = 2, NEXD_RK3 = 3, NEXD_LSERK4 = 4 };

/* Receiver trace components, in this order: plotu{x,y,z}, plotv{x,y,z},
 * plota{x,y,z} of src/timeloopMod.f90:358-373. */
#define NEXD_NCOMP 9

typedef struct nexd_desc {
  int32_t abi_version; /* NEXD_ABI_VERSION */
  int32_t N;           /* polynomial order (ORDER, src/constants.h:26) */
  int32_t Np;          /* (N+1)(N+2)(N+3)/6 */
  int32_t NpF;         /* (N+1)(N+2)/2 */
  int32_t nelem;       /* K, elements of the (single) partition */
  int32_t nMB;         /* Zener mechanisms; 0 when attenuation is off */
  int32_t attenuation; /* par%attenuation */
  int32_t set_pml;     /* par%set_pml */
  int32_t timeint;     /* enum nexd_timeint */
  int32_t nt;          /* par%nt */
  double dt;           /* deltat = dtfactor * cfl (src/timeloopMod.f90:199) */
  double init_value;   /* start value of every field; the reference uses 1e-24 */

  /* Reference-element operators, FP64 (mesh%Dr/Ds/Dt/lift/fmask). */
  const double* Dr;      /* (Np,Np) */
  const double* Ds;      /* (Np,Np) */
  const double* Dt;      /* (Np,Np) */
  const double* lift;    /* (Np,4*NpF) */
  const double* invmass; /* (Np,Np) = V V^T (src/timeloopMod.f90:302) */
  const int32_t* fmask;  /* (NpF,4), 1-based node ids */

  /* Affine-element geometry, one value per element (the reference stores the
   * same constant on every node: mesh%rx(ibool(1,ie)) etc.). */
  const double* metric;      /* (9,K): rx ry rz sx sy sz tx ty tz */
  const double* jacobian;    /* (K) */
  const double* fscale;      /* (4,K): sJ/J of each face */
  const double* nnormal;     /* (3,4,K) outward unit normal of each face */
  const double* stangential; /* (3,4,K) */
  const double* ttangential; /* (3,4,K) */

  /* Material (unrelaxed values when attenuation is on). */
  const double* rho;     /* (K) */
  const double* vpu;     /* (K) */
  const double* vsu;     /* (K) */
  const double* lambdau; /* (K) */
  const double* muu;     /* (K) */
  const double* ylambda; /* (nMB,K) */
  const double* ymu;     /* (nMB,K) */
  const double* wl;      /* (nMB) relaxation frequencies */

  /* Connectivity.  A face shared with another partition (the reference's
   * neighbor == -1 with mpi_interface set, src/meshMod.f90:768-790) has
   * neighbor 0 and face NEXD_FACE_PARTITION; its exterior trace comes from
   * the halo (nexd_create_partition). */
  const int32_t* neighbor; /* (4,K), 0 on a domain or partition boundary */
  const int32_t* face;     /* (4,K): neighbour's face 1..4, -1 free, -2 absorbing, -3 partition */
  const int32_t* ibn;      /* (NpF,4,K): neighbour's node id (global 1-based) matching
                              face node i of this element (src/meshMod.f90:939-987) */

  /* NPML (src/pmlMod.f90:90-165); ignored when set_pml == 0. */
  const int32_t* pmlcheck;     /* (K) 0/1 */
  const double* pml_profiles;  /* (K*Np,9): ddx ddy ddz alphax alphay alphaz kx ky kz */

  /* Sources (srcVar after prepareSources). */
  int32_t nsrc;
  const int32_t* srcelem;       /* (nsrc) 1-based */
  const int32_t* srctype;       /* (nsrc) 0 force, 1 moment tensor */
  const double* srcInt;         /* (Np,nsrc) interpolation weights */
  const double* srcangle_force; /* (3,nsrc) unit force direction */
  const double* srcM;           /* (6,nsrc) Mxx Myy Mzz Mxy Mxz Myz */
  int32_t stf_per_step;         /* 1: one value per step (reference); else one value per RK stage */
  const double* stf;            /* (stf_per_step,nt,nsrc): plotstf(:,2,:) as used in the source term */

  /* Receivers (recVar). */
  int32_t nrec;
  const int32_t* recelem; /* (nrec) 1-based */
  const double* recInt;   /* (Np,nrec) */

  /* Batched independent wavefields sharing this mesh (1 = one simulation).
   * Source i acts on wavefield srcbatch[i]; every wavefield records every
   * receiver. */
  int32_t nbatch;
  const int32_t* srcbatch; /* (nsrc) 0-based wavefield index, may be NULL when nbatch == 1 */
} nexd_desc;

typedef struct nexd_ctx nexd_ctx;

/* Builds device state from the descriptor (replaces the set-up part of
 * timeloop3D, src/timeloopMod.f90:162-356). */
int nexd_create(const nexd_desc* desc, nexd_ctx** out);

/* Advances time steps it_begin..it_end (1-based, inclusive), recording the
 * receiver traces of each step before its update, as the hot loop
 * src/timeloopMod.f90:357-589 does. */
int nexd_run(nexd_ctx* ctx, int32_t it_begin, int32_t it_end);

/* Copies receiver traces to `out`, shape (nrec, nt, 9, nbatch), for the steps
 * run so far (other steps hold 0). */
int nexd_get_traces(nexd_ctx* ctx, float* out);

/* Copies the velocity-stress wavefield of batch member `b` to `out`, shape
 * (K*Np, 9), the layout of q in src/timeloopMod.f90:107. */
int nexd_get_field(nexd_ctx* ctx, int32_t b, float* out);

/* Overwrites the wavefield of batch member `b` from `in`, shape (K*Np, 9). */
int nexd_set_field(nexd_ctx* ctx, int32_t b, const float* in);

/* State arrays for nexd_get_state / nexd_set_state. */
enum nexd_state {
  NEXD_STATE_Q = 0,     /* q (K*Np, 9), src/timeloopMod.f90:107 */
  NEXD_STATE_THETA = 1, /* theta (K*Np, 6, nMB), src/timeloopMod.f90:116 */
  NEXD_STATE_PML = 2    /* fprime, gprime, hprime as (K*Np, 27); zero outside PML elements */
};

/* Copies state array `which` (enum nexd_state) of batch member `b` to `out`. */
int nexd_get_state(nexd_ctx* ctx, int32_t which, int32_t b, float* out);

/* Overwrites state array `which` of batch member `b` from `in` (for PML
 * auxiliaries only the PML elements' rows are read). */
int nexd_set_state(nexd_ctx* ctx, int32_t which, int32_t b, const float* in);

/* Advances one time step `it` with host-supplied source samples and returns
 * that step's receiver samples: the streaming form of one iteration of the
 * hot loop (src/timeloopMod.f90:357-589) for hosts that produce the source
 * time function on the fly.  stf_in: (stf_per_step, nsrc) samples of step it
 * (replacing the descriptor's values for that step), may be NULL to keep
 * them; traces_out: (nrec, 9, nbatch) samples recorded at the start of step
 * it.  Host buffers are staged through pinned memory owned by the context. */
int nexd_step_io(nexd_ctx* ctx, int32_t it, const float* stf_in, float* traces_out);

/* Arms the reference's NPML stability trigger (src/timeloopMod.f90:508-542):
 * after every step the wavefield energy
 *   E = sum_e 1/2 J_e [rho v^T M v + sum_{i<=3} q_i^T M e_i + 2 sum_{i>3} q_i^T M e_i]
 * is reduced on the device (FP64); once it > 2.4/(f0 dt), the ratio of the
 * mean over the last avg_window2 steps to the mean over the last avg_window1
 * steps is tested against sta_lta_trigger and, when |ratio - 1| exceeds it,
 * the NPML of that wavefield is switched off for the rest of the run
 * (pmlcheck(:) = .false.).  formula 0 evaluates the strain e exactly as the
 * reference does (src/timeloopMod.f90:493-500, including e3 from q1+q1 and the
 * division by 1/(4mu^2+6mu*lambda)); formula 1 uses the isotropic compliance.
 * f0: the largest source centre frequency.  Requires set_pml. */
int nexd_pml_trigger(nexd_ctx* ctx, int32_t avg_window1, int32_t avg_window2, double sta_lta_trigger, double f0,
                     int32_t formula);

/* Energy history (nt, nbatch) of the steps run since nexd_pml_trigger (0
 * elsewhere) and, per wavefield, the step at which the NPML was switched off
 * (0 = never), the `pmlswitch` of the reference. */
int nexd_get_energy(nexd_ctx* ctx, double* energy, int32_t* pml_switch);

/* Wavefield energy of nbatch wavefields, computed from caller-provided device
 * arrays without allocating any device memory.  This entry point has no
 * counterpart in the reference: it exists for hosts that cannot call
 * cudaMalloc while they monitor a run -- a host whose device memory is owned
 * by another allocator (a framework's caching allocator or a pool reserved up
 * front, as an MPI Fortran host may do), or monitoring code that must not
 * incur cudaMalloc's implicit device synchronisation.
 *
 * Same computation as the trigger's energy (nexd_pml_trigger, formula 0 or 1);
 * the block partial sums go to a fixed scratch array inside libnexd.so
 * (NEXD_NOALLOC_MAX_BATCH wavefields x 256 blocks of FP64 plus one total per
 * wavefield: 16,448 doubles = 128.5 KiB), held by every GPU that loads the
 * library until the process exits.
 *   q:      device, field-major (nelem*Np nodes per field), field stride ldq,
 *           wavefield stride 9*ldq; 4-byte aligned
 *   emat:   device, (4, nelem) FP32: rho, lambda, mu, J per element; read as
 *           16-byte vectors, so it must be 16-byte aligned
 *   mass:   device, (Np, Np) FP64 mass matrix; 8-byte aligned
 *   energy: host, nbatch FP64 results; 8-byte aligned
 * A misaligned pointer is rejected with NEXD_ERR_INVALID before anything is
 * launched.  nbatch above NEXD_NOALLOC_MAX_BATCH is rejected with
 * NEXD_ERR_INVALID.  The
 * first call on a device looks up the scratch array's device address for that
 * device (cudaGetSymbolAddress); make that first call before any stream
 * capture.  Calls share the scratch array and leave their partial sums in it;
 * calls that overlap on the GPU (other threads, other streams) race on it.
 * Kernels run on the legacy default stream; the call returns after the
 * results are copied to `energy`. */
#define NEXD_NOALLOC_MAX_BATCH 64
int nexd_wavefield_energy_noalloc(const float* q, int64_t ldq, int32_t nelem, int32_t Np, int32_t nbatch,
                                  const float* emat, const double* mass, int32_t formula, double* energy);

/* Kernel kinds reported by nexd_profile_get. */
enum nexd_kernel_kind {
  NEXD_K_RECORD = 0,
  NEXD_K_STAGE_PML = 1,
  NEXD_K_STAGE_MAIN = 2,
  NEXD_K_ENERGY = 3,
  NEXD_K_BOUNDARY = 4,  /* learned-boundary ghost states */
  NEXD_K_HALO = 5,      /* partition halo writes and arrival waits */
  NEXD_K_COUNT = 6
};

typedef struct nexd_profile {
  int64_t launches[NEXD_K_COUNT]; /* launches per kernel kind since profiling was enabled */
  double ms[NEXD_K_COUNT];        /* summed device time (CUDA events on the library's stream) */
  int64_t elements[NEXD_K_COUNT]; /* elements processed per launch (stage kernels) */
  double span_ms;                 /* summed device time of whole nexd_run calls (first to last launch) */
} nexd_profile;

/* Arithmetic of the per-element contraction (volume derivatives and LIFT):
 * NEXD_CONTRACT_FP32 (default) FP32 on the CUDA cores, the reference's
 * arithmetic (src/timeloopMod.f90:407-465 in FP32); NEXD_CONTRACT_BF16X3 the
 * stacked [Dr Ds Dt LIFT] contraction on the tensor cores (tcgen05) with both
 * operands split three ways into BF16 parts (h + m + l, 24 significant bits)
 * and the six products above 2^-24 accumulated in FP32; order 4
 * (NEXD_ERR_UNSUPPORTED otherwise).  The state, the stage update and
 * everything else stay FP32.  No counterpart in the reference (its loop is
 * FP32 matvecs).
 * NEXD_CONTRACT_AUTO times the candidate kernels on this mesh (a few stage
 * launches at the current step boundary that leave the live state unchanged)
 * and keeps the fastest per element class (NPML elements, the rest): the FP32
 * kernel, the tensor-core kernel (order 4), outside the NPML an FP32 kernel
 * with a thread per node pair and on NPML elements an FP32 kernel with two
 * threads per node (orders 2-5; both bit-identical to the FP32 kernel).
 * Results of the FP32 and tensor-core kernels agree to FP32 rounding, not bit
 * for bit.  NEXD_CONTRACT_AUTO is accepted for every order. */
enum nexd_contraction {
  NEXD_CONTRACT_FP32 = 0,
  NEXD_CONTRACT_BF16X3 = 1,
  NEXD_CONTRACT_AUTO = 2,
  NEXD_CONTRACT_FP32_PAIRS = 3  /* FP32; the node-pair kernel outside the NPML (orders 2-5) */
};
int nexd_set_contraction(nexd_ctx* ctx, int32_t mode);

/* The kernel kind in use per element class (kinds[0] NPML elements, kinds[1]
 * the rest: NEXD_CONTRACT_FP32, NEXD_CONTRACT_BF16X3, 2 = the node-pair FP32
 * kernel (the rest) or 3 = the FP32 kernel whose element-local state moves
 * between global and shared memory by bulk copies) and, after an AUTO selection, the measured ms per stage launch
 * tune_ms[class * 4 + kind] (8 floats; 0 where not measured).  Either pointer
 * may be NULL. */
int nexd_get_contraction(const nexd_ctx* ctx, int32_t* kinds, float* tune_ms);

/* Pins the kernel per element class without timing: kinds[0] for NPML
 * elements (NEXD_CONTRACT_FP32, NEXD_CONTRACT_BF16X3 or 3 = the bulk-copy
 * kernel, orders 3 and 4), kinds[1] for the rest (the first two, 2 = the
 * node-pair FP32 kernel or 3 = the bulk-copy kernel, anelastic models,
 * orders 2-5), as nexd_get_contraction reports them -- e.g. to replay an earlier AUTO choice, so that repeated or
 * profiled runs use the same kernels.  NEXD_ERR_UNSUPPORTED for a kind the
 * order lacks, NEXD_ERR_INVALID for an unknown kind. */
int nexd_set_contraction_kinds(nexd_ctx* ctx, const int32_t* kinds);

/* ---- Movie snapshots (src/timeloopMod.f90:482-489, 576-581; collectMovieMod.f90) ----
 * With frame > 0 every step integrates the displacement u += dt v at every
 * node on the device (from the start value, 1e-24 in the reference) and every
 * frame-th step stores the per-element mean of |u| over the element's nodes
 * (the cell value collectMovie writes to movie_elem_it*.vtk) for up to
 * max_frames frames; frame = 0 switches it off. */
int nexd_movie(nexd_ctx* ctx, int32_t frame, int32_t max_frames);
/* Stored frames: *nframes; out (NULL to query) (nelem, nframes, nbatch) in the
 * mesh's element order. */
int nexd_get_movie(nexd_ctx* ctx, float* out, int32_t* nframes);

/* ---- Learned absorbing boundary (no counterpart in the reference) ----------
 * Absorbing faces (face code -2) normally take the exterior state as zero
 * (computeExactRiemannSF with -VT, src/waveMod.f90:269-336).  The upwind flux
 * sees the exterior state only through the incoming characteristic values
 * w = (n.S.n - Zp v.n, n.S.s - Zs v.s, n.S.t - Zs v.t) per face node (n the
 * outward normal, s, t the face tangents, Zp = rho vp, Zs = rho vs).  With a
 * boundary MLP set, every stage first predicts the exterior state of each
 * absorbing face from its interior trace: features per face node in the face
 * frame (v.n, v.s, v.t, n.S.n, n.S.s, n.S.t, s.S.s, t.S.t, s.S.t) with the
 * stresses divided by Zp, ordered node-major (feature index = 9 * face node +
 * component) in the element's own face-node order, the vector divided by its
 * RMS value r; network 9 NpF -> 128 -> 128 -> 9 NpF with GELU, applied with
 * BF16 weights and FP32 accumulation; the prediction (same units, times r)
 * gives w, clamped to |w| <= max_reflection |u| with u = (n.S.n + Zp v.n,
 * ...) the interior's outgoing values, so the boundary stays dissipative.
 * max_reflection = 0, or a network whose last layer is zero, reproduces the
 * plain absorbing boundary exactly. */

/* Absorbing faces in ghost-slot order: count, and (either may be NULL) the
 * 1-based element and face (1..4) of each. */
int nexd_boundary_faces(const nexd_ctx* ctx, int32_t* nbf, int32_t* elem, int32_t* face);
/* Sets the boundary MLP from FP32 parameters (host memory, count =
 * nexd_mlp_param_count(9 NpF, 128), layout [W1 (128 x 9NpF), b1, W2 (128 x 128),
 * b2, W3 (9NpF x 128), b3] row-major) and the reflection bound in [0, 1);
 * params NULL switches back to the plain absorbing boundary. */
int nexd_set_boundary_mlp(nexd_ctx* ctx, const float* params, int64_t count, float max_reflection);
/* The exterior states of the last stage (traction w_P n + w_S1 s + w_S2 t as a
 * stress, zero velocity): (NpF, 9, nbf, nbatch) floats. */
int nexd_get_ghost(nexd_ctx* ctx, float* out);
/* Face traces of the current wavefield for faces (elem 1-based, face 1..4):
 * out (NpF, 9, 2, nfaces, nbatch) floats, side 1 = the element's own trace,
 * side 2 = the neighbour's (zero on boundary faces), both in the element's
 * own face-node order.  Used to record training pairs from wide-NPML runs. */
int nexd_get_face_traces(nexd_ctx* ctx, int32_t nfaces, const int32_t* elem, const int32_t* face, float* out);

/* MLP training kernels (FP32; every pointer is device memory owned by the
 * caller; stream may be NULL).  Network n_in -> n_hidden -> n_hidden -> n_in,
 * GELU, parameters as above; work holds nexd_mlp_workspace_floats floats.
 * nexd_mlp_loss_grad: loss = mean over the batch of |y - target|^2 (summed
 * over outputs), written to *loss (device), and its gradient. */
int64_t nexd_mlp_param_count(int32_t n_in, int32_t n_hidden);
int64_t nexd_mlp_workspace_floats(int32_t n_in, int32_t n_hidden, int32_t batch);
int nexd_mlp_forward(int32_t n_in, int32_t n_hidden, const float* params, const float* x, int32_t batch, float* y,
                     float* work, void* stream);
int nexd_mlp_loss_grad(int32_t n_in, int32_t n_hidden, const float* params, const float* x, const float* target,
                       int32_t batch, float* grads, float* loss, float* work, void* stream);
int nexd_mlp_adam(int64_t count, float* params, const float* grads, float* m, float* v, int32_t step, float lr,
                  float beta1, float beta2, float eps, void* stream);

/* ---- Several models in one CUDA graph (no counterpart in the reference) ------
 * A group replays the steps of its member contexts (any orders, sizes,
 * rheologies and contractions) as one CUDA graph with one concurrent branch
 * per member on the member's stream, captured for two steps and replayed;
 * members keep their own state, step counter and traces, and a group run is
 * bit-identical to running the members one by one.  nexd_group_run runs steps
 * it_begin..it_end of every member (within every member's nt).
 * nexd_group_autotune times harmless first-stage launches of all members
 * running together (they leave the live state unchanged) with the members'
 * persistent grids divided by 1, 2 or 4 and keeps the fastest divisor, then
 * compares that with the single persistent launch (mode 1 below).
 * nexd_group_span: device time of the last nexd_group_run (CUDA events). */
typedef struct nexd_group nexd_group;
int nexd_group_create(nexd_ctx* const* members, int32_t n, nexd_group** out);
int nexd_group_run(nexd_group* group, int32_t it_begin, int32_t it_end);
int nexd_group_autotune(nexd_group* group, int32_t* divisor);
int nexd_group_span(const nexd_group* group, double* span_ms);
/* Execution mode of a group.  0: the graph holds one branch per member with
 * the member's own kernels (as above).  1: every LSERK stage of all members
 * is ONE persistent launch, whose blocks each work through a share of one
 * member's (wavefield, element chunk) work items with that member's order
 * and rheology -- the same per-element arithmetic as the member's FP32
 * kernel, so results are identical; the blocks are shared out in proportion
 * to each member's measured stage time.  Mode 1 covers up to 16 members that
 * step with LSERK4, have orders 2-5 and no NPML elements, energy trigger,
 * movie or learned boundary, and do not use the tensor-core contraction
 * (NEXD_ERR_UNSUPPORTED otherwise).  nexd_group_autotune measures both modes
 * (three probe stages each) and keeps the faster.  nexd_group_get_mode:
 * the mode, the blocks of each member in mode 1 (blocks may be NULL, else
 * sized to the member count) and the autotune's times (tune_ms[0] mode 0,
 * tune_ms[1] mode 1, ms for three probe stages; may be NULL). */
int nexd_group_set_mode(nexd_group* group, int32_t mode);
int nexd_group_get_mode(const nexd_group* group, int32_t* mode, int32_t* blocks, double* tune_ms);
int nexd_group_destroy(nexd_group* group);

/* ---- Partitions and the halo exchange (replaces SendRecVar, src/mpiMod.f90:310-351) ----
 * A mesh split into partitions runs one context per partition (one process
 * and GPU per partition, or several partitions of one process on one GPU).
 * The halo descriptor restates the reference's interface arrays of the
 * partition (src/meshMod.f90:1006-1110): the neighbour partitions
 * (mpi_neighbor), per neighbour the shared faces in connection order
 * (mpi_connection), and per face the index of the same face in the
 * neighbour's list (mpi_ibool) and the node matching (mpi_ibt).
 *
 * Each stage, before its element loop, every partition writes the face
 * traces of its interface faces straight into the halo slots of its
 * neighbours' wavefield (peer stores over NVLink, or plain stores when the
 * neighbour lives on the same GPU), then raises an arrival counter in the
 * neighbour's memory; the neighbour's stage starts once every neighbour's
 * counter has arrived (a bounded wait: NEXD_ERR_TIMEOUT after 5 s by default).  The
 * stage kernels read a halo slot like any neighbour element, so a
 * partitioned run gives results identical to the whole mesh in one context.
 * The NPML energy trigger needs a sum over partitions and is not supported
 * on partitions (NEXD_ERR_UNSUPPORTED). */
typedef struct nexd_halo_desc {
  int32_t partition;           /* this partition's number, 1-based (myrank + 1) */
  int32_t npeer;               /* neighbour partitions (mpi_nn) */
  const int32_t* peer;         /* (npeer) their partition numbers, 1-based (mpi_neighbor) */
  const int32_t* nface;        /* (npeer) faces shared with each neighbour (mpi_ninterface) */
  const int32_t* elem;         /* (sum nface) 1-based element of each shared face, grouped by
                                  neighbour in connection order (mpi_connection(:,:,1)) */
  const int32_t* side;         /* (sum nface) its face 1..4 (mpi_connection(:,:,2)) */
  const int32_t* peer_index;   /* (sum nface) 1-based index of the same face in the
                                  neighbour's list for this partition (mpi_ibool) */
  const int32_t* peer_node;    /* (NpF, sum nface) 1-based position, in the neighbour's
                                  face-node order, of the node matching face node j of
                                  this partition's face (mpi_ibt) */
} nexd_halo_desc;

/* nexd_create for one partition: desc describes the partition's own
 * elements (faces shared with neighbours coded NEXD_FACE_PARTITION) and halo
 * its interface.  Every NEXD_FACE_PARTITION face must appear exactly once in
 * halo.  The context runs only after nexd_halo_connect has linked it to
 * every neighbour. */
int nexd_create_partition(const nexd_desc* desc, const nexd_halo_desc* halo, nexd_ctx** out);

/* What a neighbour needs to write into this partition: exported by the
 * receiving partition for its neighbour `peer` (0-based index into
 * halo.peer), handed to that neighbour's process as bytes (MPI_Alltoall,
 * torch.distributed), and passed there to nexd_halo_connect. */
typedef struct nexd_halo_export {
  int32_t abi_version;       /* NEXD_ABI_VERSION */
  int32_t device;            /* CUDA device of the exporting context */
  int64_t pid;               /* exporting process id */
  int32_t partition;         /* exporting partition, 1-based (as in the neighbour's halo.peer) */
  int32_t nface;             /* faces shared with the importer */
  int32_t nbatch;
  int32_t nbuf;              /* wavefield buffers (2, or 3 for RK3) */
  int64_t ldq;               /* field stride of the wavefield buffers (floats) */
  int64_t halo_base;         /* node index of the first halo slot for the importer */
  int32_t counter_slot;      /* the importer's arrival counter in the exporter */
  int32_t reserved;
  uint64_t q[3];             /* device addresses, valid in the exporting process */
  uint64_t counters;         /* device address of the arrival counters (uint64 each) */
  unsigned char q_ipc[3][64];    /* cudaIpcMemHandle_t of each buffer (zero when unavailable) */
  unsigned char counters_ipc[64];
} nexd_halo_export;

int nexd_halo_export_peer(nexd_ctx* ctx, int32_t peer, nexd_halo_export* out);
/* Links this partition to its neighbour `peer` (0-based) from that
 * neighbour's export.  An export from the same process uses its device
 * addresses directly; one from another process is opened through CUDA IPC.
 * Resets the arrival counters of the pair. */
int nexd_halo_connect(nexd_ctx* ctx, int32_t peer, const nexd_halo_export* in);

/* Runs steps it_begin..it_end of n partitions that live in this process on
 * the current GPU, stage by stage in one stream: every partition's halo
 * writes of a stage, then every partition's stage (each arrival wait is met
 * when it starts).  Traces stay in each partition's context.  With
 * profiling on (nexd_profile_enable) the run span is booked to parts[0] and
 * each partition's launches to its own counters. */
int nexd_halo_run(nexd_ctx* const* parts, int32_t n, int32_t it_begin, int32_t it_end);

/* Limit of each arrival wait, in seconds (default 5, at most 60). */
int nexd_halo_set_timeout(nexd_ctx* ctx, double seconds);

/* Halo bytes written per stage (all neighbours, all wavefields). */
int nexd_halo_bytes(const nexd_ctx* ctx, int64_t* bytes_per_stage);

/* Timing of nexd_run with CUDA events on the library's stream, counters reset:
 * on = 0 off; 1 per-launch events per kernel kind plus the run span (steps are
 * launched one kernel at a time); 2 run span only (steps replay captured
 * two-step CUDA graphs, as without timing). */
int nexd_profile_enable(nexd_ctx* ctx, int32_t on);
int nexd_profile_get(const nexd_ctx* ctx, nexd_profile* out);

/* Last error message of ctx (or of the last failed nexd_create when ctx is
 * NULL), NUL-terminated and truncated to len bytes. */
int nexd_last_error(const nexd_ctx* ctx, char* buf, size_t len);

/* Number of kernel launches issued by nexd_run so far (for launch-count
 * reporting). */
int nexd_launch_count(const nexd_ctx* ctx, int64_t* out);

/* Frees device memory, the stream and graphs of ctx. */
int nexd_destroy(nexd_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* NEXD_H */
