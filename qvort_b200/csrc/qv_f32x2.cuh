// qv_f32x2.cuh -- packed FP32 pairs on sm_100 (FADD2 / FMUL2 / FFMA2).
//
// A kernel that computes the same FP32 expression for two targets keeps the
// two values of each operand in one float2 and issues one packed instruction
// for both.  Each packed operation is, per component, the scalar
// round-to-nearest operation (__fadd_rn, __fmul_rn, __fmaf_rn), so a pair
// computes bit for bit what two scalar evaluations of the same expression
// compute; only the instruction count changes.
#pragma once
#include <cuda_runtime.h>

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as a + (-b): the same IEEE result, signed zeros included
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// component h (0: x, 1: y) of a pair
__device__ __forceinline__ float pick(float2 v, int h) { return h ? v.y : v.x; }
