// Partition halo exchange (sm_100a): replaces SendRecVar
// (src/mpiMod.f90:310-351), which the reference calls once per RK stage
// before the element loop (src/timeloopMod.f90:393).
//
// Each partition keeps, after its own elements, one halo slot per face it
// shares with another partition: slot g holds in node j the neighbour's
// value at the node matching this partition's face node j (fmask order), so
// the stage kernels read it through the identity face pattern like any
// neighbour element.  Instead of packing a send buffer, exchanging it and
// unpacking it (the reference's q_send / MPI_ISSEND / qi), the sending
// partition stores its face traces straight into the receiver's halo slots
// (peer stores over NVLink when the receiver is another GPU) and then raises
// the receiver's arrival counter with a release add; the receiver's stage
// starts after a bounded acquire wait on its counters.
//
// Ordering: the wavefield buffers ping-pong between stages, so the slots a
// stage's writes land in were last read two stages earlier, and the writer
// only gets there after the receiver's data for the stage in between has
// arrived, i.e. after the receiver finished that earlier stage.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nexd_dev {

constexpr int kHaloThreads = 256;  // face nodes per write block
constexpr int kHaloMaxPeers = 64;

// One neighbour as the writer sees it.
struct HaloPeer {
  float* q[3];                  // the neighbour's wavefield buffers
  unsigned long long* counter;  // the neighbour's arrival counter for this partition
  long long ldq;                // the neighbour's field stride
  long long base;               // node index of the neighbour's first halo slot for this partition
  int entry0, nentry;           // this partition's face nodes for the neighbour: [entry0, entry0 + nentry)
  int block0;                   // first write block of the neighbour
};

struct HaloPutArgs {
  const float* q;               // own wavefield buffer `which` (input of the coming stage)
  long long ldq;
  int nbatch;
  int which;                    // buffer index 0..2, the same on every partition
  int npeer;
  const HaloPeer* peers;        // [npeer], blocks in neighbour order
  const int* src;               // [entries] own node index (internal element order)
  const int* dst;               // [entries] node offset from the neighbour's halo base
};

// One thread per (neighbour, shared face node): all 9 fields of every
// wavefield; then one release add per block on the neighbour's counter.
__global__ void __launch_bounds__(kHaloThreads) halo_put_kernel(const HaloPutArgs a) {
  int p = 0;
  while (p + 1 < a.npeer && int(blockIdx.x) >= a.peers[p + 1].block0) ++p;
  const HaloPeer& P = a.peers[p];
  const int i = (int(blockIdx.x) - P.block0) * kHaloThreads + int(threadIdx.x);
  if (i < P.nentry) {
    const long long s = a.src[P.entry0 + i];
    const long long d = P.base + a.dst[P.entry0 + i];
    float* rq = P.q[a.which];
    for (int b = 0; b < a.nbatch; ++b)
#pragma unroll
      for (int f = 0; f < 9; ++f) rq[(long long)(b * 9 + f) * P.ldq + d] = a.q[(long long)(b * 9 + f) * a.ldq + s];
  }
  // every thread's stores are visible system-wide before the block's arrival
  __threadfence_system();
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("red.release.sys.global.add.u64 [%0], 1;" ::"l"(P.counter) : "memory");
}

struct HaloWaitArgs {
  unsigned long long* counters;  // [npeer] arrivals, raised by the neighbours
  unsigned long long* expected;  // [npeer] arrivals consumed so far
  const int* blocks;             // [npeer] write blocks each neighbour sends per stage
  int npeer;
  unsigned long long limit_ns;   // longest wait
  int* flag;                     // error bits; 4: an arrival wait ran out
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits (at most limit_ns and 2^26 polls per neighbour) until every neighbour's
// writes of this stage have arrived; a wait that runs out sets flag bit 4
// and the stage goes ahead, so nothing hangs.
__global__ void halo_wait_kernel(const HaloWaitArgs a) {
  for (int p = threadIdx.x; p < a.npeer; p += blockDim.x) {
    const unsigned long long target = a.expected[p] + (unsigned long long)a.blocks[p];
    const unsigned long long t0 = global_ns();
    bool ok = false;
    for (int poll = 0; poll < (1 << 26); ++poll) {
      unsigned long long v;
      asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(a.counters + p) : "memory");
      if (v >= target) {
        ok = true;
        break;
      }
      if (global_ns() - t0 > a.limit_ns) break;
      __nanosleep(128);
    }
    if (!ok) atomicOr(a.flag, 4);
    a.expected[p] = target;
  }
}

}  // namespace nexd_dev
