// sellq.cuh -- the FP32 SELL-32 products of the mixed-precision solvers: a
// thread owns four consecutive rows of a slice, reads their entries as one
// 16-byte (FP32) or 8-byte (BF16) access per slice position and gathers the
// input vector for the four rows.  The gathered vectors are FP32, padded to
// the SELL row count with zeros and carry 8 elements of slack past it.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace ofg {
namespace {

__device__ __forceinline__ float4 load_vals(const float* p) { return *reinterpret_cast<const float4*>(p); }

__device__ __forceinline__ float4 load_vals(const __nv_bfloat16* p)
{
   const uint2 u = *reinterpret_cast<const uint2*>(p);
   const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&u.x);
   const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&u.y);
   const float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
   return make_float4(fa.x, fa.y, fb.x, fb.y);
}

// the columns of four adjacent SELL entries: absolute int32 columns, or
// 16-bit offsets from the rows r0 .. r0+3 (6 instead of 8 bytes per entry
// with FP32 values, 4 with BF16 values)
__device__ __forceinline__ int4 load_cols(const int32_t* p, int64_t)
{
   return *reinterpret_cast<const int4*>(p);
}

__device__ __forceinline__ int4 load_cols(const int16_t* p, int64_t r0)
{
   const short4 d = *reinterpret_cast<const short4*>(p);
   const int r = (int)r0;
   return make_int4(r + d.x, r + 1 + d.y, r + 2 + d.z, r + 3 + d.w);
}

// x[c .. c+3] with 16-byte loads: the aligned quad holding x[c] and, unless
// c is a multiple of 4, the next one, shifted by c mod 4.  The rows of a
// slice-uniform slice gather consecutive elements, so a thread's four
// gathers become one or two vector loads (8 lanes of a slice cover 32
// consecutive elements).  The second load may read up to 4 elements past
// the last row: the gathered vectors carry 8 elements of slack.
__device__ __forceinline__ float4 quad_at(const float* __restrict__ x, int c)
{
   const float4* x4 = reinterpret_cast<const float4*>(x);
   const float4 a = __ldg(x4 + (c >> 2));
   const int m = c & 3;
   if (m == 0) return a;
   const float4 b = __ldg(x4 + (c >> 2) + 1);
   if (m == 1) return make_float4(a.y, a.z, a.w, b.x);
   if (m == 2) return make_float4(a.z, a.w, b.x, b.y);
   return make_float4(a.w, b.x, b.y, b.z);
}

// the raw values of four adjacent SELL entries (FP32: 16 bytes, BF16: 8)
__device__ __forceinline__ float4 load_raw(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ uint2 load_raw(const __nv_bfloat16* p)
{
   return *reinterpret_cast<const uint2*>(p);
}
__device__ __forceinline__ float4 raw_f4(const float4 v) { return v; }
__device__ __forceinline__ float4 raw_f4(const uint2 u)
{
   const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&u.x);
   const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&u.y);
   const float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
   return make_float4(fa.x, fa.y, fb.x, fb.y);
}

// Positions whose values a thread loads before its first product in a
// uniform slice (BF16 values; half as many FP32 values).
constexpr int kHoist = 1;
// Resident 256-thread blocks per SM of the SELL product kernels (their
// register budget: 65536 / (256 * kQuadBlocks)), and the grid of the
// kernel chains they are part of.
constexpr int kQuadBlocks = 8;

// The four rows r0 .. r0+3 of a uniform slice: w positions, the offset of
// position k from tp[k].  The values of kHoist positions are loaded before
// the first of their products, so their DRAM latencies overlap (a rolled
// loop keeps one value line in flight per thread and waits a full DRAM
// latency per position); the products and sums keep the order k = 0 ..
// w-1, so the result is bit for bit the rolled loop's.
template <class V>
__device__ __forceinline__ float4 uniform_quad(const V* __restrict__ vp,
                                               const int16_t* __restrict__ tp, int32_t w,
                                               const float* __restrict__ x, int r0)
{
   constexpr int H = sizeof(V) == 2 ? kHoist : (kHoist + 1) / 2;
   using Raw = decltype(load_raw(vp));
   float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 1
   for (int32_t k0 = 0; k0 < w; k0 += H) {
      Raw raw[H];
#pragma unroll
      for (int q = 0; q < H; ++q)
         if (k0 + q < w) raw[q] = load_raw(vp + (k0 + q) * 32);
#pragma unroll
      for (int q = 0; q < H; ++q) {
         if (k0 + q >= w) break;
         const float4 a = raw_f4(raw[q]);
         const float4 xv = quad_at(x, r0 + tp[k0 + q]);
         acc.x += a.x * xv.x;
         acc.y += a.y * xv.y;
         acc.z += a.z * xv.z;
         acc.w += a.w * xv.w;
      }
   }
   return acc;
}

// y[r0 .. r0+3] = (M x)[r0 .. r0+3] for a SELL-32 matrix M: A itself, or
// G (lower rows) and G^T (upper rows) of the learned preconditioner, which
// live on A's slices with BF16 values (the preconditioner's own precision:
// M = G^T G is still one fixed symmetric positive definite operator).  V is
// the value type (float or BF16), I the column format (absolute int32 or
// 16-bit offsets); UNI reads a uniform slice's offsets from its table.
template <class V, class I, bool UNI>
__device__ __forceinline__ float4 sell_quad(const int32_t* __restrict__ sp,
                                            const I* __restrict__ scol,
                                            const V* __restrict__ sval,
                                            const float* __restrict__ x, int64_t r0,
                                            const int32_t* __restrict__ suni,
                                            const int16_t* __restrict__ stab)
{
   const int64_t s = r0 >> 5;
   const int lane0 = (int)(r0 & 31);
   const int32_t beg = sp[s], w = (sp[s + 1] - beg) >> 5;
   float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
   const V* vp = sval + beg + lane0;
   const int32_t u = UNI ? suni[s] : -1;
   if (u >= 0) return uniform_quad(vp, stab + u, w, x, (int)r0);
   const I* cp = scol + beg + lane0;
   auto step = [&](int32_t k) {
      const int4 c = load_cols(cp + k * 32, r0);
      const float4 a = load_vals(vp + k * 32);
      acc.x += a.x * __ldg(x + c.x);
      acc.y += a.y * __ldg(x + c.y);
      acc.z += a.z * __ldg(x + c.z);
      acc.w += a.w * __ldg(x + c.w);
   };
   if (UNI) {
#pragma unroll 1
      for (int32_t k = 0; k < w; ++k) step(k);
   }
   else {
#pragma unroll 4
      for (int32_t k = 0; k < w; ++k) step(k);
   }
   return acc;
}

}  // namespace
}  // namespace ofg
