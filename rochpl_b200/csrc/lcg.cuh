// 64-bit LCG of HPL's matrix generator, shared by matgen and the fused
// residual.  X(n+1) = a X(n) + c mod 2^64 with a = 6364136223846793005,
// c = 1 (include/hpl_pmatgen.hpp:35-36).
#pragma once
#include <cstdint>

namespace hplb {

constexpr uint64_t kLcgMult = 6364136223846793005ull;
constexpr uint64_t kLcgAdd  = 1ull;

// Affine jump X -> a X + c.
struct Jump {
  uint64_t a, c;
};

// Apply x, then y.
__host__ __device__ inline Jump compose(Jump x, Jump y) {
  return Jump{y.a * x.a, y.a * x.c + y.c};
}

// Jump by k steps, by repeated squaring (the reference's HPL_xjumpm,
// src/matgen/HPL_xjumpm.cpp:81-91, loops k times; the constants are equal).
__host__ __device__ inline Jump jump_by(uint64_t k) {
  Jump acc{1, 0}, p{kLcgMult, kLcgAdd};
  while(k) {
    if(k & 1) acc = compose(acc, p);
    p = compose(p, p);
    k >>= 1;
  }
  return acc;
}

__host__ __device__ inline uint64_t apply(Jump j, uint64_t x) { return j.a * x + j.c; }

// Matrix entry from a state, with the reference's operation order
// (src/matgen/HPL_pdrandmat_device.cpp:65-73).  Every multiply or divide is by
// a power of two and therefore exact; the explicit _rn intrinsics keep the two
// rounded additions and the final subtraction from being contracted.
__device__ __forceinline__ double lcg_value(uint64_t r) {
  const double p1 = (double)(uint32_t)(r & 65535ull);
  const double p2 = (double)(uint32_t)((r >> 16) & 65535ull);
  const double p3 = (double)(uint32_t)((r >> 32) & 65535ull);
  const double p4 = (double)(uint32_t)((r >> 48) & 65535ull);
  double t = __dadd_rn(p1, __dmul_rn(p2, 65536.0));
  t        = __dmul_rn(__dmul_rn(t, 0x1p-31), 0.5);
  t        = __dadd_rn(t, p3);
  t        = __dadd_rn(t, __dmul_rn(p4, 65536.0));
  return __dsub_rn(0.5, __dmul_rn(__dmul_rn(t, 0x1p-31), 0.5));
}

}  // namespace hplb
