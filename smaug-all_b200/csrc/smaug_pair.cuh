// smaug_pair.cuh -- two FP32 lanes in one 64-bit register pair, for the packed
// FP32 instructions of sm_100a (add/sub/mul/fma .rn.ftz.f32x2).
//
// Each lane is rounded exactly as the scalar instruction of the same name
// rounds it (round to nearest even, subnormals flushed as the -ftz=true build
// flushes them), so a computation written with these operations gives the
// same bits as its scalar form.  Negation is a multiply by -1 (exact, and it
// keeps the sign of zero), since the packed fma has no negated operand form.
#pragma once

namespace SMAUG_NS {

struct f2 {
  unsigned long long r;
};

__device__ __forceinline__ f2 f2_make(float lo, float hi) {
  f2 o;
  asm("mov.b64 %0, {%1, %2};" : "=l"(o.r) : "f"(lo), "f"(hi));
  return o;
}
__device__ __forceinline__ f2 f2_splat(float a) { return f2_make(a, a); }
__device__ __forceinline__ float f2_lo(f2 x) {
  float lo;
  asm("{\n\t.reg .f32 h;\n\tmov.b64 {%0, h}, %1;\n\t}" : "=f"(lo) : "l"(x.r));
  return lo;
}
__device__ __forceinline__ float f2_hi(f2 x) {
  float hi;
  asm("{\n\t.reg .f32 l;\n\tmov.b64 {l, %0}, %1;\n\t}" : "=f"(hi) : "l"(x.r));
  return hi;
}
__device__ __forceinline__ f2 operator+(f2 a, f2 b) {
  f2 o;
  asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(o.r) : "l"(a.r), "l"(b.r));
  return o;
}
__device__ __forceinline__ f2 operator-(f2 a, f2 b) {
  f2 o;
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(o.r) : "l"(a.r), "l"(b.r));
  return o;
}
__device__ __forceinline__ f2 operator*(f2 a, f2 b) {
  f2 o;
  asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(o.r) : "l"(a.r), "l"(b.r));
  return o;
}
// a * b + c with one rounding per lane
__device__ __forceinline__ f2 pfma(f2 a, f2 b, f2 c) {
  f2 o;
  asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(o.r) : "l"(a.r), "l"(b.r), "l"(c.r));
  return o;
}
__device__ __forceinline__ f2 pneg(f2 a) { return a * f2_splat(-1.0f); }

}  // namespace SMAUG_NS
