// Shared device helpers for the B200 HPL solve path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "hplb.h"

#define HPLB_DEV __device__ __forceinline__

namespace hplb {

// Device status word layout (int32 each), written by kernels, read by the host
// after a synchronisation point.
enum : int {
  ST_TIMEOUT = 0,  // nonzero: a bounded device wait gave up (value = site id)
  ST_INFO    = 1,  // first zero-pivot column, 1-based (atomicMin-style, 0 = none)
  ST_COUNT   = 4
};

// Wait budget for every spin in this library (ns of %globaltimer).  Long enough
// for a co-scheduled trailing-update grid to drain, short enough that a lost
// block surfaces as HPLB_ERR_TIMEOUT instead of a hung GPU.
constexpr unsigned long long kWaitBudgetNs = 4000000000ull;

HPLB_DEV unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

HPLB_DEV int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

HPLB_DEV void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Pivot search order: the larger |v| wins, ties go to the lower row; r < 0
// marks "no candidate".  warp_argmax reduces the warp's (v, r) pairs in that
// order without branches: |v| as an unsigned 64-bit key reduced by two 32-bit
// max reductions (high word, then low word among the lanes holding the high
// maximum), the lowest matching row by a min reduction, the signed value
// taken from the lane that holds it.  Every lane gets the result; returns the
// winning lane, or -1 (v = 0, r = -1) if no lane has a candidate.  For finite
// values the order is that of a sequential scan with "strictly larger |v|
// replaces" over increasing rows (LAPACK's idamax); a NaN magnitude ranks
// above every finite one.
HPLB_DEV int warp_argmax(double& v, int& r) {
  const unsigned long long key =
      r >= 0 ? (unsigned long long)__double_as_longlong(fabs(v)) : 0ull;
  const unsigned hi   = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi  = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo  = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool     hit  = r >= 0 && hi == mhi && lo == mlo;
  const unsigned best = __reduce_min_sync(0xffffffffu, hit ? (unsigned)r : 0xffffffffu);
  const unsigned who  = __ballot_sync(0xffffffffu, hit && (unsigned)r == best);
  const int      wl   = who ? __ffs(who) - 1 : 0;
  v = __shfl_sync(0xffffffffu, v, wl);
  if(!who) {
    v = 0.0;
    r = -1;
    return -1;
  }
  r = (int)best;
  return wl;
}

// Grid-wide barrier for co-resident (cooperatively launched) grids, on a
// monotonic arrival counter: the gen-th barrier of a launch (1-based) returns
// once bar[0] >= gen * nblocks.  One atomic per block and no reset between
// barriers (the host zeroes bar[0] before every launch); 1.2 us per barrier on
// B200 against 2.9 us for a count-and-generation barrier.  Every wait is
// bounded: on expiry the block records `site` in status[ST_TIMEOUT] and the
// barrier returns false, as it does once any other block has timed out;
// callers then leave the kernel.
HPLB_DEV bool grid_sync(int* bar, int nblocks, int gen, int* status, int site) {
  __shared__ int s_ok;
  __syncthreads();
  if(threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    atomicAdd(bar, 1);
    const int                target = gen * nblocks;
    const unsigned long long t0     = globaltimer();
    unsigned                 polls  = 0;
    while(ld_acquire_gpu(bar) < target) {
      if((++polls & 31u) == 0) {
        if(ld_acquire_gpu(status + ST_TIMEOUT) != 0) {
          ok = 0;
          break;
        }
        if(globaltimer() - t0 > kWaitBudgetNs) {
          atomicCAS(status + ST_TIMEOUT, 0, site);
          ok = 0;
          break;
        }
      }
      __nanosleep(20);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Record the first (lowest) zero-pivot column, 1-based.
HPLB_DEV void record_info(int* status, int col1) {
  int old = status[ST_INFO];
  while(old == 0 || col1 < old) {
    const int prev = atomicCAS(status + ST_INFO, old, col1);
    if(prev == old) break;
    old = prev;
  }
}

}  // namespace hplb
