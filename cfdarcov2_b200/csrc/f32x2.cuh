// Packed FP32 pairs for sm_100a: add/sub/mul/fma.rn.f32x2 (PTX ISA 8.6+)
// apply one IEEE round-to-nearest operation to both halves of a 64-bit
// register pair, so a thread that owns two cells can advance both with one
// instruction per operation.  Each lane rounds exactly like the scalar
// instruction of the same name.  The mov.b64 pairings cost nothing when the
// two floats already sit in a register pair (a float2 from a vector load).
#pragma once

#define CFDB_F2_BINARY(name, op)                                                                       \
  __device__ __forceinline__ float2 name(float2 a, float2 b) {                                           \
    float2 r;                                                                                            \
    asm("{.reg .b64 ra, rb, rr;\n\tmov.b64 ra, {%2,%3};\n\tmov.b64 rb, {%4,%5};\n\t" op                   \
        " rr, ra, rb;\n\tmov.b64 {%0,%1}, rr;}"                                                          \
        : "=f"(r.x), "=f"(r.y)                                                                           \
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                                       \
    return r;                                                                                            \
  }

namespace f2 {
CFDB_F2_BINARY(add, "add.rn.f32x2")
CFDB_F2_BINARY(sub, "sub.rn.f32x2")
CFDB_F2_BINARY(mul, "mul.rn.f32x2")
// a * b + c, one rounding per lane
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) {
  float2 r;
  asm("{.reg .b64 ra, rb, rc, rr;\n\tmov.b64 ra, {%2,%3};\n\tmov.b64 rb, {%4,%5};\n\tmov.b64 rc, {%6,%7};\n\t"
      "fma.rn.f32x2 rr, ra, rb, rc;\n\tmov.b64 {%0,%1}, rr;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return r;
}
__device__ __forceinline__ float2 splat(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 neg(float2 a) { return make_float2(-a.x, -a.y); }
}  // namespace f2

#undef CFDB_F2_BINARY
