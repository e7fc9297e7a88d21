// step_dev.cuh -- device pieces of a whole time step shared by the
// per-kernel step (captured in a CUDA graph) and the persistent fused step
// kernel: boundary-flux reduction of one member, the device-resident model
// clock, and a bounded grid barrier.
#pragma once
#include "f3d_common.cuh"

namespace f3d {

// Block-level deterministic reduction of one member's per-block flux partials
// into flux_step {W,E,S,N,U,D} and the Kahan-compensated running totals.
// Requires blockDim.x a power of two <= 256 and a __shared__ scratch of
// 2 * blockDim.x doubles.
__device__ __forceinline__ void member_flux_reduce(const MemberDev& m, int dirmask, double* sa,
                                                   double* sb) {
  double res[6] = {0, 0, 0, 0, 0, 0};
  for (int d = 0; d < 3; ++d) {
    if (!(dirmask & (1 << d))) continue;
    double a = 0.0, b = 0.0;
    const double* p = m.flux_part + 2LL * m.part_base[d];
    for (int s = threadIdx.x; s < m.part_count[d]; s += blockDim.x) {
      a = a + p[2 * s];
      b = b + p[2 * s + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) {
        sa[threadIdx.x] = sa[threadIdx.x] + sa[threadIdx.x + s];
        sb[threadIdx.x] = sb[threadIdx.x] + sb[threadIdx.x + s];
      }
      __syncthreads();
    }
    // x -> (W,E) = 0,1 ; y -> (S,N) = 2,3 ; z -> (D,U) = 5,4
    if (d == 0) { res[0] = sa[0]; res[1] = sb[0]; }
    if (d == 1) { res[2] = sa[0]; res[3] = sb[0]; }
    if (d == 2) { res[5] = sa[0]; res[4] = sb[0]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int q = 0; q < 6; ++q) {
      bool on = (q < 2) ? (dirmask & 1) : (q < 4) ? (dirmask & 2) : (dirmask & 4);
      if (!on) continue;
      m.flux_step[q] = res[q];
      double y = res[q] - m.flux_tot[6 + q];
      double t = m.flux_tot[q] + y;
      m.flux_tot[6 + q] = (t - m.flux_tot[q]) - y;
      m.flux_tot[q] = t;
    }
  }
}

// Device-resident clock: time += gl_dt, iiter += 1 (task_Fall3d.F90:299-300)
// and the interpolation factor of the next step (mod_F3D.F90:1437).
__device__ __forceinline__ void member_advance(MemberDev& m) {
  m.time = m.time + m.dt;
  m.iiter = m.iiter + 1;
  m.stime = (m.time - m.t_its) / (m.t_ite - m.t_its);
}

// Grid-wide barrier for a co-resident (cooperative) launch.  bar[0] counts
// arrivals, bar[1] is the generation.  Every wait is bounded: after `limit`
// polls (kSpinLimit unless f3d_set_wait_limit lowered it) the block records
// an error in *err and continues, so a barrier can never hang the GPU.
constexpr long long kSpinLimit = 1LL << 25;

// Poll limit of the bounded device waits for the next launches (host side;
// f3d_set_wait_limit, f3d_capi.cu).
long long wait_limit();

__device__ __forceinline__ void grid_barrier(unsigned int* bar, int* err, long long limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* gen = bar + 1;
    const unsigned int g0 = *gen;
    __threadfence();
    const unsigned int arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      bar[0] = 0u;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (*gen == g0) {
        if (++spins > limit) {
          atomicExch(err, 1);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Work-stealing index for the persistent kernel: one atomic per block.
__device__ __forceinline__ int grab_item(unsigned int* counter, int* slot) {
  __syncthreads();
  if (threadIdx.x == 0) *slot = (int)atomicAdd(counter, 1u);
  __syncthreads();
  return *slot;
}

// Arguments of the persistent fused step kernel.
struct FusedArgs {
  MemberDev* members;
  int nmembers;
  const WorkItem* work[3];
  int nwork[3];
  const int* prep_member;  // FP64 prep blocks: member and first block per member
  const int* prep_first;
  int nprep;
  unsigned int* counters;  // [0..5] phase work counters, [6..7] barrier
  int* err;
  int bpb;
  long long wait_limit;    // polls before a grid barrier gives up (kSpinLimit by default)
  int epi;                 // the z phase runs the wet deposition and decay epilogue
};

}  // namespace f3d
