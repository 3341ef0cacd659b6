// CUDA qualifiers and intrinsics mapped to plain C++ for the host builds of the engine's
// per-thread arithmetic (tile_host.cpp, pipe_host.cpp).  Every fused or packed device operation
// becomes the scalar operation with the same single rounding, so the host build computes the
// device's bits; the harnesses are compiled with -ffp-contract=off.
#pragma once
#include <cmath>

#define __device__
#define __host__
#define __forceinline__ inline
#define __constant__
static inline double __fma_rn(double a, double b, double c) { return std::fma(a, b, c); }
static inline float __fmaf_rn(float a, float b, float c) { return std::fmaf(a, b, c); }
// packed FP32 pairs (sm_100 f32x2 instructions): lane by lane the scalar operations
struct float2 {
  float x, y;
};
static inline float2 make_float2(float a, float b) { return float2{a, b}; }
static inline float2 __ffma2_rn(float2 a, float2 b, float2 c) {
  return {std::fmaf(a.x, b.x, c.x), std::fmaf(a.y, b.y, c.y)};
}
static inline float2 __fadd2_rn(float2 a, float2 b) { return {a.x + b.x, a.y + b.y}; }
static inline float2 __fmul2_rn(float2 a, float2 b) { return {a.x * b.x, a.y * b.y}; }
