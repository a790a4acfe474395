// packed.cuh -- packed FP32x2 distance arithmetic of the search kernels (sm_100a).
//
// Two IEEE round-to-nearest operations per instruction, each element rounded on its own
// exactly like __fsub_rn / __fmul_rn / __fadd_rn, so two candidates' distances cost one
// instruction chain. tests/test_gpu_packed.py compiles tests/cuda/packed_probe.cu against
// this header and checks dist2_pair against the scalar dist2_ref (common.cuh) bit for bit.
#pragma once
#include <cstdint>

namespace rtnn {

__device__ __forceinline__ uint64_t pk2(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void upk2(uint64_t v, uint32_t& lo, uint32_t& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
// x * x + (+0) with one rounding: the bits of x * x for every x (a square is never -0)
__device__ __forceinline__ uint64_t sq2(uint64_t a) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(r) : "l"(a), "l"(0ull));
  return r;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
// dist2_ref of two points at once: ((dx*dx + dy*dy) + dz*dz), every step rounded, all
// packed. The squares are written as fused multiply-adds of +0 (one rounding, the exact
// bits of the product): a packed add of two packed products (mul.rn.f32x2) was measured
// to be fused into a single-rounding multiply-add by the compiler even with .rn (about
// 12 % of results off by an ulp).
__device__ __forceinline__ void dist2_pair(uint64_t qx, uint64_t qy, uint64_t qz, uint64_t px,
                                           uint64_t py, uint64_t pz, uint32_t& d0, uint32_t& d1) {
  const uint64_t dx = sub2(qx, px), dy = sub2(qy, py), dz = sub2(qz, pz);
  upk2(add2(add2(sq2(dx), sq2(dy)), sq2(dz)), d0, d1);
}

}  // namespace rtnn
