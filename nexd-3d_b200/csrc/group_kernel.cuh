// Several models' stage in one persistent launch (sm_100a, FP32).
//
// A group of models of different sizes, orders and rheologies (each its own
// mesh, state and step counter) advances one LSERK stage with ONE launch:
// the blocks [bfirst[i], bfirst[i+1]) of the grid work on model i, block b
// taking that model's work items (wavefield, chunk of elements) b - bfirst[i],
// + (bfirst[i+1] - bfirst[i]), ... through the per-order stage body of
// stage_kernel (the reference's element loop and stage update,
// src/timeloopMod.f90:395-476, src/rungekuttaMod.f90:27-88), so each model
// gets exactly the result of its own stage_kernel launch.  The block shares
// are chosen on the host from each model's measured cost (the group
// autotune), so that all models finish the stage together.
//
// The models' stage arguments travel in the kernel's parameter space (up to
// kGroupMax models); the dynamic shared memory is the largest any member's
// order needs.
#pragma once
#include "stage_kernel.cuh"

namespace nexd_dev {

constexpr int kGroupMax = 16;

struct GroupStageArgs {
  StageArgs m[kGroupMax];     // each model's stage arguments for this stage
  int order[kGroupMax];       // polynomial order N (2..5)
  int att[kGroupMax];         // 1: anelastic (3 Zener mechanisms)
  int bfirst[kGroupMax + 1];  // blocks [bfirst[i], bfirst[i+1]) work on model i
  int nmodel;
};

// Shared memory one block needs for model orders up to 5 (elements outside the NPML).
__host__ __device__ constexpr int group_smem_floats(int N) {
  return N == 2 ? Order<2>::smem_floats(false)
       : N == 3 ? Order<3>::smem_floats(false)
       : N == 4 ? Order<4>::smem_floats(false)
       : N == 5 ? Order<5>::smem_floats(false) : 0;
}

template <int MODE>
__global__ void __launch_bounds__(256, 2) group_stage_kernel(const __grid_constant__ GroupStageArgs g) {
  extern __shared__ __align__(16) float smem[];
  int i = 0;
  while (i + 1 < g.nmodel && int(blockIdx.x) >= g.bfirst[i + 1]) ++i;
  const int w0 = int(blockIdx.x) - g.bfirst[i], wstep = g.bfirst[i + 1] - g.bfirst[i];
  if (w0 < 0 || wstep <= 0) return;
  const StageArgs& a = g.m[i];
  switch (g.order[i] * 2 + (g.att[i] ? 1 : 0)) {
    case 4: stage_body<2, false, false, MODE>(a, w0, wstep, smem); break;
    case 5: stage_body<2, true, false, MODE>(a, w0, wstep, smem); break;
    case 6: stage_body<3, false, false, MODE>(a, w0, wstep, smem); break;
    case 7: stage_body<3, true, false, MODE>(a, w0, wstep, smem); break;
    case 8: stage_body<4, false, false, MODE>(a, w0, wstep, smem); break;
    case 9: stage_body<4, true, false, MODE>(a, w0, wstep, smem); break;
    case 10: stage_body<5, false, false, MODE>(a, w0, wstep, smem); break;
    case 11: stage_body<5, true, false, MODE>(a, w0, wstep, smem); break;
    default: break;
  }
}

}  // namespace nexd_dev
