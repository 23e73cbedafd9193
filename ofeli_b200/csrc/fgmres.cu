// fgmres.cu -- the mixed-precision solver for nonsymmetric systems (the
// transient convection-diffusion steps): flexible GMRES(m), right
// preconditioned, with an FP32 matrix-vector product and an FP32
// preconditioner application, inside FP64 iterative refinement.
//
// Outer loop (FP64): r = b - A x with the FP64 SELL product; converged only
// when ||r|| / ||b|| <= toler.  Otherwise one FGMRES cycle solves A d = r
// from d = 0 and x += d.  A cycle (Saad's flexible GMRES):
//     v_0 = r / ||r||
//     for j = 0 .. m-1:
//        z_j = M^{-1} v_j         FP32 (DIAG, IDENT, or the learned G^T G
//                                   with BF16 factor values)
//        w   = A z_j              FP32 SELL product (FP32 or lossless BF16
//                                   values, 16-bit column offsets)
//        h   = V^T w; w -= V h    FP64 classical Gram-Schmidt, twice (CGS2)
//        h  += V^T w; w -= V h'
//        H(j+1, j) = ||w||, v_{j+1} = w / H(j+1, j)
//        Givens rotations of column j; |s_{j+1}| estimates ||r - A Z y||
//     d = Z y,  y = argmin ||beta e_1 - H y|| (back substitution)
// The cycle stops when the estimate fell by inner_tol, when it predicts the
// FP64 target (half of toler * ||b||), after m steps or at the iteration
// cap.  The preconditioned vectors Z are kept (FP32), which is what makes
// the method flexible: the preconditioner may change between steps, and
// the FP32 application of M is not an exact linear operator.
//
// OFELI's GMRes (include/solvers/GMRes.h:148-241) is FP64, left
// preconditioned, with modified Gram-Schmidt: its dot products are
// sequential (step k needs the vector left by step k-1), which here would
// be k+3 kernels per Arnoldi step.  Classical Gram-Schmidt computes all of a
// column's dot products in one pass, and the second pass restores the
// orthogonality MGS has (CGS2); an Arnoldi step is five kernels with DIAG
// (seven with the learned factor), chained by programmatic dependent launch:
//     [z_j (learned: t = G v_j, z_j = G^T t)] -> w = A z_j -> h = V^T w
//     -> w -= V h, h' = V^T w -> w -= V h', ||w||, rotations, stop test
//     -> v_{j+1}, z_{j+1}
// Every reduction is finished by the last block to arrive, in block order:
// results are bitwise reproducible.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "internal.cuh"
#include "reduce.cuh"
#include "sellq.cuh"

namespace ofg {
namespace {

constexpr int kMaxRestart = 64;
constexpr int kWarps = kRedBlock / 32;

struct FGState {
   double bnorm, rel;  // FP64 true residual ||b - A x|| / ||b||
   double beta;        // ||r|| at the start of the cycle
   double res;         // the cycle's residual estimate |s_{j+1}|
   double hnext;       // H(j+1, j) before its rotation: the scale of v_{j+1}
   int steps;          // Arnoldi steps completed in the cycle
   int stop;           // the cycle is over
   int done;           // FP64 true residual <= toler
   int skip_end;       // the cycle-end kernels of this batch do nothing
   int zero_diag;      // a diagonal entry is zero (FP32 values: checked with the first state read)
   int pad;
};

// r = b - q (FP64); ||r||, ||b|| (first call); the FP64 convergence test
__global__ void __launch_bounds__(kRedBlock, 8) fg_residual(int64_t n, const double* __restrict__ b,
                                                         const double* __restrict__ q, double* r,
                                                         FGState* S, double* partials,
                                                         unsigned* counter, double tol, int first,
                                                         int end)
{
   if (end && S->skip_end) return;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double bi = b[i], ri = bi - q[i];
      r[i] = ri;
      v[0] += ri * ri;
      if (first) v[1] += bi * bi;
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      if (first) {
         S->bnorm = sqrt(t[1]);
         if (S->bnorm == 0.0) S->bnorm = 1.0;
      }
      S->rel = sqrt(t[0]) / S->bnorm;
      S->done = S->rel <= tol ? 1 : 0;
   }
}

// The preconditioner input of step j from v_j (FP64, the four rows of
// quad i): z_j = D^{-1} v_j in FP32 (dinv = ones for IDENT), or, for the
// learned factor (dinv == nullptr), v_j in FP32 for the product with G.
__device__ __forceinline__ void precond_quad(int64_t i, const double2 a, const double2 b,
                                             const float* __restrict__ dinv, float* z)
{
   float4 v = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
   if (dinv) {
      const float4 d = *reinterpret_cast<const float4*>(dinv + i * 4);
      v.x *= d.x;
      v.y *= d.y;
      v.z *= d.z;
      v.w *= d.w;
   }
   *reinterpret_cast<float4*>(z + i * 4) = v;
}

// Start of a cycle: beta = ||r||, v_0 = r / beta (zero in the padding),
// s = (beta, 0, ...), and the preconditioner input of step 0.
__global__ void __launch_bounds__(kRedBlock) fg_begin(int64_t n, int64_t nquads,
                                                   const double* __restrict__ r, double* v0,
                                                   const float* __restrict__ dinv, float* z,
                                                   double* s, int m, FGState* S)
{
   pdl_wait();
   pdl_release();
   const double beta = S->rel * S->bnorm;
   const double sc = 1.0 / beta;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const int64_t r0 = i * 4;
      const double2 a = make_double2(r0 < n ? sc * r[r0] : 0.0, r0 + 1 < n ? sc * r[r0 + 1] : 0.0);
      const double2 b = make_double2(r0 + 2 < n ? sc * r[r0 + 2] : 0.0,
                                     r0 + 3 < n ? sc * r[r0 + 3] : 0.0);
      reinterpret_cast<double2*>(v0)[2 * i] = a;
      reinterpret_cast<double2*>(v0)[2 * i + 1] = b;
      precond_quad(i, a, b, dinv, z);
   }
   if (blockIdx.x == 0) {
      for (int j = threadIdx.x; j <= m; j += blockDim.x) s[j] = j == 0 ? beta : 0.0;
      if (threadIdx.x == 0) {
         S->beta = beta;
         S->res = beta;
         S->steps = 0;
         S->stop = 0;
      }
   }
}

// y = M x over four rows per thread (A, G or G^T)
template <class V, class I, bool UNI>
__global__ void __launch_bounds__(kRedBlock, kQuadBlocks) fg_product(int64_t nquads, const int32_t* __restrict__ sp,
                                                        const I* __restrict__ scol,
                                                        const V* __restrict__ sval,
                                                        const float* __restrict__ x, float* y,
                                                        const FGState* S, int* worked,
                                                        const int32_t* __restrict__ suni,
                                                        const int16_t* __restrict__ stab)
{
   pdl_wait();
   pdl_release();
   if (S->stop) return;
   prof_mark(worked);
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride)
      *reinterpret_cast<float4*>(y + i * 4) = sell_quad<V, I, UNI>(sp, scol, sval, x, i * 4, suni, stab);
}

// v_k[4i .. 4i+3] as two double2
__device__ __forceinline__ void load_v(const double* __restrict__ V, int64_t ld, int k, int64_t i,
                                       double2& a, double2& b)
{
   const double2* p = reinterpret_cast<const double2*>(V + (size_t)k * ld) + 2 * i;
   a = __ldg(p);
   b = __ldg(p + 1);
}

// Per-block sums of nk values (one accumulator per warp and value in
// shared memory), stored as partials[k * gridDim.x + block]; the last block
// to arrive sums every value's partials in block order into out[k].
// Returns true in the last block (after out[] is written and visible to its
// threads).
__device__ __forceinline__ bool multi_reduce(double (*acc)[kWarps], int nk, double* partials,
                                             unsigned* counter, double* out)
{
   __shared__ bool last;
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   __syncthreads();
   for (int k = threadIdx.x; k < nk; k += blockDim.x) {
      double s = 0.0;
      for (int w = 0; w < kWarps; ++w) s += acc[k][w];
      partials[(size_t)k * gridDim.x + blockIdx.x] = s;
      __threadfence();
   }
   __syncthreads();
   if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
   __syncthreads();
   if (!last) return false;
   __threadfence();
   for (int k = wid; k < nk; k += kWarps) {
      double s = 0.0;
      for (unsigned bb = lane; bb < gridDim.x; bb += 32) s += __ldcg(partials + (size_t)k * gridDim.x + bb);
      s = warp_sum(s);
      if (lane == 0) out[k] = s;
   }
   __syncthreads();
   if (threadIdx.x == 0) *counter = 0;
   return true;
}

// First Gram-Schmidt pass, dot products: h_k = (w, v_k) for k <= j, with w
// the FP32 product A z_j; stored in H's column j.
__global__ void __launch_bounds__(kRedBlock) fg_dots(int64_t nquads, const float* __restrict__ w32,
                                                     const double* __restrict__ V, int64_t ld, int j,
                                                     double* hcol, double* partials,
                                                     unsigned* counter, const FGState* S,
                                                     int* worked)
{
   __shared__ double acc[kMaxRestart + 1][kWarps];
   pdl_wait();
   pdl_release();
   if (S->stop) return;
   prof_mark(worked);
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   for (int k = threadIdx.x; k <= j; k += blockDim.x)
      for (int w = 0; w < kWarps; ++w) acc[k][w] = 0.0;
   __syncthreads();
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nquads; base += stride) {
      const int64_t i = base + threadIdx.x;
      float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
      if (i < nquads) q = *reinterpret_cast<const float4*>(w32 + i * 4);
      for (int k = 0; k <= j; ++k) {
         double t = 0.0;
         if (i < nquads) {
            double2 a, b;
            load_v(V, ld, k, i, a, b);
            t = (double)q.x * a.x + (double)q.y * a.y + (double)q.z * b.x + (double)q.w * b.y;
         }
         t = warp_sum(t);
         if (lane == 0) acc[k][wid] += t;
      }
   }
   multi_reduce(acc, j + 1, partials, counter, hcol);
}

// First Gram-Schmidt pass, update, and the second pass's dot products:
// w = A z_j - sum_k h_k v_k (FP64), h'_k = (w, v_k) into h2.
__global__ void __launch_bounds__(kRedBlock) fg_orth1(int64_t nquads, const float* __restrict__ w32,
                                                      const double* __restrict__ V, int64_t ld,
                                                      int j, const double* __restrict__ hcol,
                                                      double* w, double* h2, double* partials,
                                                      unsigned* counter, const FGState* S,
                                                      int* worked)
{
   __shared__ double acc[kMaxRestart + 1][kWarps];
   __shared__ double h[kMaxRestart + 1];
   pdl_wait();
   pdl_release();
   if (S->stop) return;
   prof_mark(worked);
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   for (int k = threadIdx.x; k <= j; k += blockDim.x) {
      h[k] = hcol[k];
      for (int q = 0; q < kWarps; ++q) acc[k][q] = 0.0;
   }
   __syncthreads();
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nquads; base += stride) {
      const int64_t i = base + threadIdx.x;
      double2 wa = make_double2(0.0, 0.0), wb = make_double2(0.0, 0.0);
      if (i < nquads) {
         const float4 q = *reinterpret_cast<const float4*>(w32 + i * 4);
         wa = make_double2(q.x, q.y);
         wb = make_double2(q.z, q.w);
         for (int k = 0; k <= j; ++k) {
            double2 a, b;
            load_v(V, ld, k, i, a, b);
            const double hk = h[k];
            wa.x -= hk * a.x;
            wa.y -= hk * a.y;
            wb.x -= hk * b.x;
            wb.y -= hk * b.y;
         }
         reinterpret_cast<double2*>(w)[2 * i] = wa;
         reinterpret_cast<double2*>(w)[2 * i + 1] = wb;
      }
      for (int k = 0; k <= j; ++k) {
         double t = 0.0;
         if (i < nquads) {
            double2 a, b;
            load_v(V, ld, k, i, a, b);
            t = wa.x * a.x + wa.y * a.y + wb.x * b.x + wb.y * b.y;
         }
         t = warp_sum(t);
         if (lane == 0) acc[k][wid] += t;
      }
   }
   multi_reduce(acc, j + 1, partials, counter, h2);
}

__device__ __forceinline__ void rotate(double& dx, double& dy, double cs, double sn)
{
   const double t = cs * dx + sn * dy;
   dy = cs * dy - sn * dx;
   dx = t;
}

// the Givens rotation that zeroes dy against dx (the form of GMRes.h:98-115)
__device__ __forceinline__ void set_rotation(double dx, double dy, double& cs, double& sn)
{
   if (dy == 0.0) {
      cs = 1.0;
      sn = 0.0;
   }
   else if (fabs(dy) > fabs(dx)) {
      const double t = dx / dy;
      sn = 1.0 / sqrt(1.0 + t * t);
      cs = t * sn;
   }
   else {
      const double t = dy / dx;
      cs = 1.0 / sqrt(1.0 + t * t);
      sn = t * cs;
   }
}

struct CycleRule {
   double inner_tol;  // stop when the estimate fell by this factor
   double target;     // ... or when it is below this (absolute) value
   int m;             // restart length
   int cap;           // steps allowed in this cycle (iteration cap)
};

// Second Gram-Schmidt pass: w -= sum_k h'_k v_k, ||w||; then (last block)
// H(k, j) = h_k + h'_k, H(j+1, j) = ||w||, the rotations of column j, the
// residual estimate and the stop decision.
__global__ void __launch_bounds__(kRedBlock) fg_orth2(int64_t nquads, double* w,
                                                      const double* __restrict__ V, int64_t ld,
                                                      int j, const double* __restrict__ h2,
                                                      double* H, double* s, double* cs, double* sn,
                                                      double* partials, unsigned* counter,
                                                      FGState* S, CycleRule rule, int* worked)
{
   __shared__ double h[kMaxRestart + 1];
   pdl_wait();
   pdl_release();
   if (S->stop) return;
   prof_mark(worked);
   for (int k = threadIdx.x; k <= j; k += blockDim.x) h[k] = h2[k];
   __syncthreads();
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      double2* wp = reinterpret_cast<double2*>(w) + 2 * i;
      double2 wa = wp[0], wb = wp[1];
      for (int k = 0; k <= j; ++k) {
         double2 a, b;
         load_v(V, ld, k, i, a, b);
         const double hk = h[k];
         wa.x -= hk * a.x;
         wa.y -= hk * a.y;
         wb.x -= hk * b.x;
         wb.y -= hk * b.y;
      }
      wp[0] = wa;
      wp[1] = wb;
      v[0] += wa.x * wa.x + wa.y * wa.y + wb.x * wb.x + wb.y * wb.y;
   }
   double t[1];
   if (!grid_reduce<1>(v, partials, counter, t)) return;
   const int ld_h = rule.m + 1;
   double* Hc = H + (size_t)j * ld_h;
   for (int k = 0; k <= j; ++k) Hc[k] += h[k];
   const double hn = sqrt(t[0]);
   Hc[j + 1] = hn;
   S->hnext = hn;
   for (int k = 0; k < j; ++k) rotate(Hc[k], Hc[k + 1], cs[k], sn[k]);
   set_rotation(Hc[j], Hc[j + 1], cs[j], sn[j]);
   rotate(Hc[j], Hc[j + 1], cs[j], sn[j]);
   rotate(s[j], s[j + 1], cs[j], sn[j]);
   const double res = fabs(s[j + 1]);
   S->res = res;
   S->steps = j + 1;
   // not finite, happy breakdown (w = 0), converged, or out of steps
   const bool stop = !(res > rule.inner_tol * S->beta) || !(res > rule.target) || !(hn > 0.0) ||
                     j + 1 >= rule.m || j + 1 >= rule.cap;
   if (stop) S->stop = 1;
}

// v_{j+1} = w / H(j+1, j) and the preconditioner input of step j+1
__global__ void __launch_bounds__(kRedBlock, 8) fg_next(int64_t nquads, const double* __restrict__ w,
                                                     double* vn, const float* __restrict__ dinv,
                                                     float* z, const FGState* S)
{
   pdl_wait();
   pdl_release();
   if (S->stop) return;
   const double sc = 1.0 / S->hnext;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const double2* wp = reinterpret_cast<const double2*>(w) + 2 * i;
      double2 a = wp[0], b = wp[1];
      a.x *= sc;
      a.y *= sc;
      b.x *= sc;
      b.y *= sc;
      reinterpret_cast<double2*>(vn)[2 * i] = a;
      reinterpret_cast<double2*>(vn)[2 * i + 1] = b;
      precond_quad(i, a, b, dinv, z);
   }
}

// The end of a batch of Arnoldi steps: when the cycle is over (stopped,
// or `last`: all m steps done), y = R^{-1} s over its S->steps columns (R
// = the rotated H); otherwise it marks the batch's cycle-end kernels (the
// solution update, the FP64 residual) to do nothing.
__global__ void fg_backsolve(const double* H, const double* s, double* y, int m, FGState* S,
                             int last)
{
   pdl_wait();
   pdl_release();
   if (threadIdx.x != 0 || blockIdx.x != 0) return;
   const int end = last || S->stop;
   S->skip_end = end ? 0 : 1;
   if (!end) return;
   const int ld = m + 1, k = S->steps;
   for (int i = 0; i < k; ++i) y[i] = s[i];
   for (int i = k - 1; i >= 0; --i) {
      y[i] /= H[(size_t)i * ld + i];
      for (int l = i - 1; l >= 0; --l) y[l] -= H[(size_t)i * ld + l] * y[i];
   }
}

// x += Z y (Z in FP32, y and x in FP64)
__global__ void __launch_bounds__(kRedBlock, 8) fg_update_x(int64_t n, double* x,
                                                         const float* __restrict__ Z, int64_t ldz,
                                                         const double* __restrict__ y,
                                                         const FGState* S)
{
   __shared__ double ys[kMaxRestart];
   pdl_wait();
   pdl_release();
   if (S->skip_end) return;
   const int k = S->steps;
   for (int l = threadIdx.x; l < k; l += blockDim.x) ys[l] = y[l];
   __syncthreads();
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      double xi = x[i];
      for (int l = 0; l < k; ++l) xi += ys[l] * (double)__ldg(Z + (size_t)l * ldz + i);
      x[i] = xi;
   }
}

// D^{-1} in FP32, zero in the padding; IDENT: ones
__global__ void fg_inv_diag(int64_t n, int64_t npad, const int32_t* dpos, const double* val,
                            float* dinv, int ident, int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += stride) {
      if (i >= n) {
         dinv[i] = 0.0f;
         continue;
      }
      if (ident) {
         dinv[i] = 1.0f;
         continue;
      }
      const int32_t k = dpos[i];
      const double a = k >= 0 ? val[k] : 0.0;
      if (!(fabs(a) > 0.0)) atomicOr(bad, 1);
      dinv[i] = (float)(1.0 / a);
   }
}

// BF16 copy of the values; *inexact = 1 when a value does not come back
// unchanged (a NaN never does)
__global__ void fg_cast_bf16(int64_t total, const double* __restrict__ src, __nv_bfloat16* dst,
                             int* inexact)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   int lost = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
      const double v = src[i];
      const __nv_bfloat16 h = (__nv_bfloat16)v;
      dst[i] = h;
      lost |= (double)__bfloat162float(h) != v;
   }
   if (__syncthreads_or(lost) && threadIdx.x == 0) atomicOr(inexact, 1);
}

bool mostly_uniform(const ofg_matrix* M)
{
   return M->utab_len > 0 && M->uni_nnz >= 0.9 * (double)M->nnz;
}

// One SELL-32 matrix in the FP32 solver's formats: its value array (FP32 or
// BF16) and column format (16-bit offsets, with or without uniform slices,
// or absolute columns).
struct Sell32 {
   const ofg_matrix* M = nullptr;
   const void* val = nullptr;
   bool bf16 = false, d16 = false, uni = false;
   double bytes = 0.0;  // algorithmic bytes of one product (values + indices)
};

void launch_product(const Sell32& P, int64_t nquads, unsigned grid, const float* x, float* y,
                    const FGState* S, int* worked)
{
   using bf = __nv_bfloat16;
   const ofg_matrix* M = P.M;
   const int32_t* su = P.uni ? M->sell_uni.p : nullptr;
   const int16_t* st = P.uni ? M->sell_utab.p : nullptr;
   if (P.bf16) {
      const bf* v = static_cast<const bf*>(P.val);
      if (P.uni)
         launch_pdl(fg_product<bf, int16_t, true>, grid, kRedBlock, nquads, M->sell_ptr.p,
                    M->sell_d16.p, v, x, y, S, worked, su, st);
      else if (P.d16)
         launch_pdl(fg_product<bf, int16_t, false>, grid, kRedBlock, nquads, M->sell_ptr.p,
                    M->sell_d16.p, v, x, y, S, worked, su, st);
      else
         launch_pdl(fg_product<bf, int32_t, false>, grid, kRedBlock, nquads, M->sell_ptr.p,
                    M->sell_col.p, v, x, y, S, worked, su, st);
   }
   else {
      const float* v = static_cast<const float*>(P.val);
      if (P.uni)
         launch_pdl(fg_product<float, int16_t, true>, grid, kRedBlock, nquads, M->sell_ptr.p,
                    M->sell_d16.p, v, x, y, S, worked, su, st);
      else if (P.d16)
         launch_pdl(fg_product<float, int16_t, false>, grid, kRedBlock, nquads, M->sell_ptr.p,
                    M->sell_d16.p, v, x, y, S, worked, su, st);
      else
         launch_pdl(fg_product<float, int32_t, false>, grid, kRedBlock, nquads, M->sell_ptr.p,
                    M->sell_col.p, v, x, y, S, worked, su, st);
   }
}

double index_bytes(const ofg_matrix* M, bool d16, bool uni)
{
   if (!d16) return 4.0 * M->nnz;
   if (!uni) return 2.0 * M->nnz;
   return 2.0 * (M->nnz - M->uni_nnz) + 2.0 * M->utab_len;
}

// the learned factor (G or G^T) in BF16 with the FP32 solver's index format
Sell32 factor_format(ofg_matrix* G)
{
   Sell32 f;
   ensure_sell(G);
   ensure_sell_bf16(G);
   f.M = G;
   f.val = G->sell_valbf.p;
   f.bf16 = true;
   f.d16 = ensure_sell_d16(G);
   if (f.d16) ensure_sell_uniform(G);
   f.uni = f.d16 && mostly_uniform(G);
   f.bytes = 2.0 * G->nnz + index_bytes(G, f.d16, f.uni);
   return f;
}

}  // namespace

void fgmres_mixed(ofg_prec* P, int inner_bits, const double* b, double* x, int m, int max_outer,
                  int max_inner, double inner_tol, double tol, int* outer, int* inner,
                  double* true_res, int* fell_back)
{
   ofg_matrix* A = P->A;
   OFG_REQUIRE(P->type == OFG_DIAG || P->type == OFG_IDENT || P->type == OFG_LEARNED, OFG_ERR_ARG,
               "the mixed-precision FGMRES takes DIAG, IDENT or LEARNED");
   OFG_REQUIRE(m >= 1 && m <= kMaxRestart, OFG_ERR_ARG, "restart length must be in 1 .. 64");
   OFG_REQUIRE(inner_bits == 32 || inner_bits == 16 || inner_bits == 0, OFG_ERR_ARG,
               "inner_bits must be 32, 16 or 0 (automatic)");
   OFG_REQUIRE(inner_tol > 0 && inner_tol < 1, OFG_ERR_ARG, "inner_tol must be in (0, 1)");
   const int64_t n = A->n;
   // FP32 values asked for: both SELL copies of new values in one pass
   if (inner_bits == 32) ensure_sell32(A);
   else ensure_sell(A);
   ensure_dpos(A);
   OFG_REQUIRE(A->dpos_complete, OFG_ERR_PIVOT, "a row has no diagonal entry");
   bool learned = P->type == OFG_LEARNED;
   Sell32 gl, gu;
   if (learned) {
      if (prec_stale(P)) prec_setup(P);
      OFG_REQUIRE(P->gl->nslices == A->nslices && P->gu->nslices == A->nslices, OFG_ERR_ARG,
                  "learned factor does not match the matrix");
      gl = factor_format(P->gl);
      gu = factor_format(P->gu);
   }
   const int64_t npad = A->nslices * 32, nquads = npad / 4, nv = npad > 0 ? npad : 4;
   Sell32 a;
   a.M = A;
   a.d16 = ensure_sell_d16(A);
   if (a.d16) ensure_sell_uniform(A);
   a.uni = a.d16 && mostly_uniform(A);
   // bad[0]: zero diagonal entry; bad[1]: a value of A is not exact in BF16
   DBuf<int> bad(2);
   bad.zero();
   DBuf<__nv_bfloat16> v16;
   if (inner_bits != 32) {
      v16.alloc(A->sell_val.n);
      fg_cast_bf16<<<grid_for(A->sell_val.n, 256), 256, 0, stream()>>>(A->sell_val.n,
                                                                       A->sell_val.p, v16.p,
                                                                       bad.p + 1);
      count_launch();
   }
   DBuf<FGState> S(1);
   S.zero();
   DBuf<float> dinv(nv);
   // with FP32 values nothing waits for the zero-diagonal flag: it travels
   // in the solver state and is checked at its first read
   fg_inv_diag<<<grid_for(nv, 256), 256, 0, stream()>>>(n, npad, A->dpos.p, A->val.p, dinv.p,
                                                         P->type == OFG_IDENT ? 1 : 0,
                                                         inner_bits == 32 ? &S.p->zero_diag : bad.p);
   count_launch();
   OFG_LAUNCH_CHECK();
   int hb[2] = {0, 0};
   if (inner_bits != 32) {
      bad.download(hb, 2);
      OFG_REQUIRE(!hb[0], OFG_ERR_PIVOT, "zero diagonal entry");
   }
   // automatic format: BF16 values only when every value is exact in BF16
   const bool use16 = inner_bits == 16 || (inner_bits == 0 && !hb[1]);
   if (use16) {
      a.bf16 = true;
      a.val = v16.p;
   }
   else {
      v16.release();
      ensure_sell32(A);
      a.val = A->sell_val32.p;
   }
   a.bytes = (use16 ? 2.0 : 4.0) * A->nnz + index_bytes(A, a.d16, a.uni);

   const int64_t ldz = nv + 8;  // Z vectors are gathered: 8 elements of slack
   DBuf<double> V((size_t)(m + 1) * nv), w(nv), r(n > 0 ? n : 1), q64(n > 0 ? n : 1);
   DBuf<float> Z((size_t)m * ldz), w32(nv), v32(learned ? ldz : 1), t32(learned ? ldz : 1);
   Z.zero();
   v32.zero();
   t32.zero();
   DBuf<double> H((size_t)(m + 1) * (m + 1)), s(m + 1), cs(m + 1), sn(m + 1), y(m + 1), h2(m + 1);
   const unsigned gq = grid_for(nquads, kRedBlock, kQuadBlocks);
   const unsigned gr = grid_for(nquads, kRedBlock, 4);
   const unsigned gn = grid_for(n, kRedBlock, 8);
   DBuf<double> partials((size_t)(kMaxRestart + 1) * std::max(gr, gn) + 8);
   DBuf<unsigned> counter(1);
   counter.zero();

   // end = 1: the cycle-end form, a no-op while S->skip_end is set
   auto true_residual = [&](int first, int end = 0) {
      spmv_sell(A, x, q64.p, end ? &S.p->skip_end : nullptr);
      fg_residual<<<gn, kRedBlock, 0, stream()>>>(n, b, q64.p, r.p, S.p, partials.p, counter.p, tol,
                                                  first, end);
      count_launch();
      OFG_LAUNCH_CHECK();
   };
   // z_j from the preconditioner input left by fg_begin / fg_next: with the
   // learned factor, t = G v_j and z_j = G^T t
   auto learned_z = [&](int j) {
      float* zj = Z.p + (size_t)j * ldz;
      int* worked = prof_begin();
      launch_product(gl, nquads, gq, v32.p, t32.p, S.p, worked);
      prof_end(PROF_LEARNED_APPLY, gl.bytes + 8.0 * n);
      worked = prof_begin();
      launch_product(gu, nquads, gq, t32.p, zj, S.p, worked);
      prof_end(PROF_LEARNED_APPLY, gu.bytes + 8.0 * n);
   };
   FGState h{};
   true_residual(1);
   S.download(&h, 1);
   OFG_REQUIRE(!h.zero_diag, OFG_ERR_PIVOT, "zero diagonal entry");
   int n_outer = 0, n_inner = 0, no_gain = 0;
   double last_rel = h.rel;
   while (!h.done && n_outer < max_outer && n_inner < max_inner && n > 0) {
      const float* pin = learned ? nullptr : dinv.p;
      float* pout = learned ? v32.p : Z.p;
      launch_pdl(fg_begin, gq, kRedBlock, n, nquads, r.p, V.p, pin, pout, s.p, m, S.p);
      if (learned) learned_z(0);
      const CycleRule rule{inner_tol, 0.5 * tol * h.bnorm, m, max_inner - n_inner};
      int j = 0;
      bool cycle_over = false;
      for (int batch = 4; !cycle_over; batch *= 2) {
         const int end = std::min(m, j + batch);
         for (; j < end; ++j) {
            float* zj = Z.p + (size_t)j * ldz;
            double* hcol = H.p + (size_t)j * (m + 1);
            int* worked = prof_begin();
            launch_product(a, nquads, gq, zj, w32.p, S.p, worked);
            prof_end(use16 ? PROF_SPMV16 : PROF_SPMV32, a.bytes + 12.0 * n);
            // algorithmic bytes: the basis vectors v_0 .. v_j (FP64) once per
            // pass over them, A z_j (FP32) and w (FP64) as each kernel moves them
            const double vb = 8.0 * (double)(j + 1) * n;
            worked = prof_begin();
            launch_pdl(fg_dots, gr, kRedBlock, nquads, w32.p, V.p, nv, j, hcol, partials.p,
                       counter.p, S.p, worked);
            prof_end(PROF_ORTH, vb + 4.0 * n);
            worked = prof_begin();
            launch_pdl(fg_orth1, gr, kRedBlock, nquads, w32.p, V.p, nv, j, hcol, w.p, h2.p,
                       partials.p, counter.p, S.p, worked);
            prof_end(PROF_ORTH, 2.0 * vb + 12.0 * n);
            worked = prof_begin();
            launch_pdl(fg_orth2, gr, kRedBlock, nquads, w.p, V.p, nv, j, h2.p, H.p, s.p, cs.p,
                       sn.p, partials.p, counter.p, S.p, rule, worked);
            prof_end(PROF_ORTH, vb + 16.0 * n);
            if (j + 1 < m) {
               float* pnext = learned ? v32.p : Z.p + (size_t)(j + 1) * ldz;
               launch_pdl(fg_next, gq, kRedBlock, nquads, w.p, V.p + (size_t)(j + 1) * nv, pin,
                          pnext, S.p);
               if (learned) learned_z(j + 1);
            }
         }
         // the cycle's end (back-substitution, x += Z y, the FP64 residual)
         // is enqueued after every batch and runs only when the cycle is
         // over, so one read of the state per batch decides
         launch_pdl(fg_backsolve, 1, 32, H.p, s.p, y.p, m, S.p, end == m ? 1 : 0);
         launch_pdl(fg_update_x, gn, kRedBlock, n, x, Z.p, ldz, y.p, S.p);
         OFG_LAUNCH_CHECK();
         true_residual(0, 1);
         S.download(&h, 1);
         cycle_over = !h.skip_end;
      }
      n_inner += h.steps;
      n_outer++;
      // the learned preconditioner must keep the FP64 residual falling;
      // otherwise the remaining cycles use the diagonal one
      if (learned) {
         no_gain = (h.rel > 0.5 * last_rel || !std::isfinite(h.rel)) ? no_gain + 1 : 0;
         if (!std::isfinite(h.rel) || no_gain >= 2) {
            learned = false;
            if (fell_back) *fell_back = 1;
            if (!std::isfinite(h.rel)) {
               OFG_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), stream()));
               true_residual(0);
               S.download(&h, 1);
            }
         }
      }
      last_rel = h.rel;
   }
   *outer = n_outer;
   *inner = n_inner;
   *true_res = h.rel;
}

}  // namespace ofg

using namespace ofg;

// Flexible GMRES(m) in mixed precision inside FP64 iterative refinement
// (see the top of this file).  P: DIAG, IDENT or LEARNED on its matrix.
extern "C" int ofg_fgmres_mixed(ofg_prec* P, int inner_bits, const double* b, double* x, int m,
                                int max_outer, int max_inner, double inner_tol, double toler,
                                int* outer, int* inner, double* true_res, int* fell_back)
{
   return guarded("ofg_fgmres_mixed", [&] {
      OFG_REQUIRE(P && b && x && outer && inner && true_res, OFG_ERR_ARG, "null argument");
      if (fell_back) *fell_back = 0;
      ofg_matrix* A = P->A;
      In<double> db(b, A->n);
      InOut<double> dx(x, A->n, true);
      fgmres_mixed(P, inner_bits, db.d, dx.d, m, max_outer, max_inner, inner_tol, toler, outer,
                   inner, true_res, fell_back);
      dx.finish();
   });
}
