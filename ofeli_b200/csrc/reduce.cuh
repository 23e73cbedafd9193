// reduce.cuh -- deterministic grid-wide reductions for the Krylov kernels.
//
// Every block adds its share, stores one partial per value and bumps an
// arrival counter; the last block to arrive sums the partials in block order
// with a fixed tree and runs the finisher on thread 0.  The grid size of a
// kernel depends only on the problem size, so results are bitwise
// reproducible from run to run.
#pragma once

#include "common.cuh"

namespace ofg {

constexpr int kRedBlock = 256;

// Returns true on thread 0 of the last block, with tot[] holding the sums.
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double* partials, unsigned* counter,
                                            double (&tot)[NV])
{
   __shared__ double sh[NV][kRedBlock / 32];
   __shared__ bool last;
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
   for (int i = 0; i < NV; ++i) {
      double s = warp_sum(v[i]);
      if (lane == 0) sh[i][wid] = s;
   }
   __syncthreads();
   if (threadIdx.x == 0) {
#pragma unroll
      for (int i = 0; i < NV; ++i) {
         double s = 0.0;
         for (int w = 0; w < nw; ++w) s += sh[i][w];
         partials[(size_t)blockIdx.x * NV + i] = s;
      }
      __threadfence();
      last = atomicAdd(counter, 1u) == gridDim.x - 1;
   }
   __syncthreads();
   if (!last) return false;
   __threadfence();
   double t[NV];
#pragma unroll
   for (int i = 0; i < NV; ++i) t[i] = 0.0;
   // L2 loads (the partials were published before the counter), unrolled so
   // that they are in flight together
#pragma unroll 4
   for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
      for (int i = 0; i < NV; ++i) t[i] += __ldcg(partials + (size_t)b * NV + i);
   __syncthreads();
#pragma unroll
   for (int i = 0; i < NV; ++i) {
      double s = warp_sum(t[i]);
      if (lane == 0) sh[i][wid] = s;
   }
   __syncthreads();
   if (threadIdx.x != 0) return false;
#pragma unroll
   for (int i = 0; i < NV; ++i) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += sh[i][w];
      tot[i] = s;
   }
   *counter = 0;
   return true;
}

// The same reduction split across a kernel boundary, for kernels chained on
// one stream with the same grid: every block of the producing kernel stores
// its partial sums and exits (no fence, no arrival counter, no last block);
// every block of the consuming kernel, which starts after the producer
// completed, sums all partials in grid_reduce's order, so each block holds
// bitwise the totals grid_reduce would have produced.
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double* partials)
{
   __shared__ double sh[NV][kRedBlock / 32];
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
   for (int i = 0; i < NV; ++i) {
      double s = warp_sum(v[i]);
      if (lane == 0) sh[i][wid] = s;
   }
   __syncthreads();
   if (threadIdx.x == 0) {
#pragma unroll
      for (int i = 0; i < NV; ++i) {
         double s = 0.0;
         for (int w = 0; w < nw; ++w) s += sh[i][w];
         partials[(size_t)blockIdx.x * NV + i] = s;
      }
   }
}

// Totals of the partials of `nblocks` producer blocks, in every thread.
template <int NV>
__device__ __forceinline__ void partials_total(const double* partials, unsigned nblocks,
                                               double (&tot)[NV])
{
   __shared__ double sh[NV][kRedBlock / 32];
   __shared__ double res[NV];
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
   double t[NV];
#pragma unroll
   for (int i = 0; i < NV; ++i) t[i] = 0.0;
#pragma unroll 4
   for (unsigned b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
      for (int i = 0; i < NV; ++i) t[i] += __ldcg(partials + (size_t)b * NV + i);
   __syncthreads();
#pragma unroll
   for (int i = 0; i < NV; ++i) {
      double s = warp_sum(t[i]);
      if (lane == 0) sh[i][wid] = s;
   }
   __syncthreads();
   if (threadIdx.x == 0) {
#pragma unroll
      for (int i = 0; i < NV; ++i) {
         double s = 0.0;
         for (int w = 0; w < nw; ++w) s += sh[i][w];
         res[i] = s;
      }
   }
   __syncthreads();
#pragma unroll
   for (int i = 0; i < NV; ++i) tot[i] = res[i];
}

}  // namespace ofg
