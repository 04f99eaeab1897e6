// rs_f32x2.cuh — packed FP32 pairs for the sm_100 f32x2 instructions
// (add/sub/mul/fma.rn.f32x2): two lanes per 64-bit register, each rounded as
// the scalar FP32 operation.
#pragma once

#include <cstdint>

namespace rs {

// lane 0 in the low word
using f2 = uint64_t;
__device__ __forceinline__ f2 pk(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ f2 bc(float v) { return pk(v, v); }
__device__ __forceinline__ float lo_of(f2 v) {
  float a;
  asm("{\n .reg .b32 t;\n mov.b64 {%0, t}, %1;\n}" : "=f"(a) : "l"(v));
  return a;
}
__device__ __forceinline__ float hi_of(f2 v) {
  float b;
  asm("{\n .reg .b32 t;\n mov.b64 {t, %0}, %1;\n}" : "=f"(b) : "l"(v));
  return b;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f2 ld2(const float *p) { return *reinterpret_cast<const f2 *>(p); }
__device__ __forceinline__ void st2(float *p, f2 v) { *reinterpret_cast<f2 *>(p) = v; }

}  // namespace rs
