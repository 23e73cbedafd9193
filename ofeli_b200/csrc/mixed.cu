// mixed.cu -- mixed-precision solve: FP64 iterative refinement whose
// correction is computed by preconditioned CG in FP32 (or with BF16 matrix
// values and FP32 vectors).
//
// Mode 0 (refinement with a kept Krylov direction): one PCG sequence runs in
// FP32; whenever its recursive residual has fallen by `inner_tol` since the
// last refinement, or predicts convergence, the host performs a refinement
// step in FP64:
//     x += x_lo;  x_lo = 0;  r = b - A x (FP64 SpMV);  r_lo = (float) r
// and the FP32 recurrence continues from the true residual with its search
// direction kept (the "reliable update" form of refinement: the Krylov space
// is not thrown away at every refinement, so the iteration count stays close
// to that of FP64 CG).
// Mode 1 (classic restarted refinement): every refinement solves
// A d = r / ||r|| from d = 0 to `inner_tol` and adds ||r|| d.
//
// FP64 is used only for b - A x, the refinement update x += ..., and the
// accumulation of every Krylov dot product.  One FP32 CG iteration streams
// 8*nnz + 56*n bytes (6*nnz + 56*n with BF16 values) against 12*nnz + 112*n
// in FP64.
//
// The FP32 vectors are padded to the SELL row count (a multiple of 32) with
// zeros, so every inner kernel moves 16-byte vectors: a thread owns four
// consecutive rows, reads their SELL slots as float4/int4 (four adjacent
// lanes of one slice column) and gathers x for the four rows.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "internal.cuh"
#include "reduce.cuh"

namespace ofg {
namespace {

struct MixState {
   double bnorm, rel;          // FP64 true residual
   double rho[2];              // rho of the last two iterations, indexed by it & 1
   double alpha, rn, rmark, res0;
   double beta;                // learned preconditioner: next direction's beta
   int it, pause, done, pad;
};

template <class T>
__global__ void cast_values(int64_t total, const double* __restrict__ src, T* dst)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
      dst[i] = (T)src[i];
}

// r = b - q (FP64); ||r||, ||b|| (first call); convergence test
__global__ void __launch_bounds__(kRedBlock, 8) mx_residual(int64_t n, const double* __restrict__ b,
                                                         const double* __restrict__ q, double* r,
                                                         MixState* S, double* partials,
                                                         unsigned* counter, double tol, int first)
{
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
         S->it = 0;
      }
      S->rel = sqrt(t[0]) / S->bnorm;
      S->done = S->rel <= tol ? 1 : 0;
   }
}

// r_lo = (float)(r * scale) (zero in the padding); rho = (r_lo, D r_lo),
// ||r_lo||; x_lo = 0; on a fresh start also p = D r_lo.  Without dinv (the
// learned preconditioner) only r_lo, ||r_lo|| and x_lo.
__global__ void __launch_bounds__(kRedBlock, 8) mx_load_residual(int64_t n, int64_t npad,
                                                              const double* __restrict__ r,
                                                              double scale,
                                                              const float* __restrict__ dinv,
                                                              float* rr0, float* rr1, float* p,
                                                              float* d, int fresh, MixState* S,
                                                              double* partials, unsigned* counter)
{
   // the learned iteration keeps r in two buffers, the current one by the
   // parity of the iteration count
   float* rr = (rr1 && (S->it & 1)) ? rr1 : rr0;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += stride) {
      const float ri = i < n ? (float)(r[i] * scale) : 0.0f;
      const float zi = dinv ? ri * dinv[i] : 0.0f;
      rr[i] = ri;
      d[i] = 0.0f;
      if (fresh && dinv) p[i] = zi;
      v[0] += (double)ri * (double)zi;
      v[1] += (double)ri * (double)ri;
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      if (dinv) S->rho[S->it & 1] = t[0];  // else set by the learned products
      S->rn = sqrt(t[1]);
      S->rmark = S->rn;
      if (fresh) S->res0 = S->rn;
      S->pause = 0;
   }
}

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

// q = A p over four rows per thread, (p, q) -> alpha
template <class T, class I>
__global__ void __launch_bounds__(kRedBlock, 8) mx_spmv(int64_t nquads, const int32_t* __restrict__ sp,
                                                     const I* __restrict__ scol,
                                                     const T* __restrict__ sval,
                                                     const float* __restrict__ p,
                                                     float* __restrict__ q, MixState* S,
                                                     double* partials, unsigned* counter,
                                                     int* worked)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   prof_mark(worked);
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nquads; t += stride) {
      const int64_t r0 = t * 4;
      const int64_t s = r0 >> 5;
      const int lane0 = (int)(r0 & 31);
      const int32_t beg = sp[s], w = (sp[s + 1] - beg) >> 5;
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      const I* cp = scol + beg + lane0;
      const T* vp = sval + beg + lane0;
#pragma unroll 8
      for (int32_t k = 0; k < w; ++k) {
         const int4 c = load_cols(cp + k * 32, r0);
         const float4 a = load_vals(vp + k * 32);
         acc.x += a.x * __ldg(p + c.x);
         acc.y += a.y * __ldg(p + c.y);
         acc.z += a.z * __ldg(p + c.z);
         acc.w += a.w * __ldg(p + c.w);
      }
      *reinterpret_cast<float4*>(q + r0) = acc;
      const float4 pr = *reinterpret_cast<const float4*>(p + r0);
      v[0] += (double)pr.x * acc.x + (double)pr.y * acc.y + (double)pr.z * acc.z +
              (double)pr.w * acc.w;
   }
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t)) S->alpha = S->rho[S->it & 1] / t[0];
}

// d += alpha p, r -= alpha q; ||r||, (r, D r) when JAC; decides when the
// host must refine (mode 0) or stop the inner solve (mode 1)
template <bool JAC>
__global__ void __launch_bounds__(kRedBlock, 8) mx_update(int64_t nquads, float* d,
                                                       const float* __restrict__ p, float* rr,
                                                       const float* __restrict__ q,
                                                       const float* __restrict__ dinv, MixState* S,
                                                       double* partials, unsigned* counter,
                                                       double delta, double tol, double scale,
                                                       int max_inner, int mode)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   const float a = (float)S->alpha;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   float4* d4 = reinterpret_cast<float4*>(d);
   float4* r4 = reinterpret_cast<float4*>(rr);
   const float4* p4 = reinterpret_cast<const float4*>(p);
   const float4* q4 = reinterpret_cast<const float4*>(q);
   const float4* m4 = reinterpret_cast<const float4*>(dinv);
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const float4 pi = p4[i], qi = q4[i];
      float4 di = d4[i], ri = r4[i];
      di.x += a * pi.x; di.y += a * pi.y; di.z += a * pi.z; di.w += a * pi.w;
      ri.x -= a * qi.x; ri.y -= a * qi.y; ri.z -= a * qi.z; ri.w -= a * qi.w;
      d4[i] = di;
      r4[i] = ri;
      v[0] += (double)ri.x * ri.x + (double)ri.y * ri.y + (double)ri.z * ri.z + (double)ri.w * ri.w;
      if (JAC) {
         const float4 mi = m4[i];
         v[1] += (double)ri.x * (ri.x * mi.x) + (double)ri.y * (ri.y * mi.y) +
                 (double)ri.z * (ri.z * mi.z) + (double)ri.w * (ri.w * mi.w);
      }
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      S->rn = sqrt(t[0]);
      const int it = S->it + 1;
      if (JAC) S->rho[it & 1] = t[1];
      S->it = it;
      if (mode == 0) {
         // refine when the residual fell by delta, or when the recurrence
         // says the FP64 target is reached
         if (S->rn <= delta * S->rmark || S->rn * scale <= tol * S->bnorm || it >= max_inner)
            S->pause = 1;
      }
      else if (S->rn <= delta * S->res0 || it >= max_inner) {
         S->pause = 1;
      }
   }
}

// p = D r + beta p, beta = rho_it / rho_{it-1}
__global__ void __launch_bounds__(kRedBlock, 8) mx_direction(int64_t nquads,
                                                          const float* __restrict__ rr,
                                                          const float* __restrict__ dinv, float* p,
                                                          const MixState* S)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   const int it = S->it;
   const float beta = (float)(S->rho[it & 1] / S->rho[(it + 1) & 1]);
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   float4* p4 = reinterpret_cast<float4*>(p);
   const float4* r4 = reinterpret_cast<const float4*>(rr);
   const float4* m4 = reinterpret_cast<const float4*>(dinv);
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const float4 ri = r4[i], mi = m4[i];
      float4 pi = p4[i];
      pi.x = ri.x * mi.x + beta * pi.x;
      pi.y = ri.y * mi.y + beta * pi.y;
      pi.z = ri.z * mi.z + beta * pi.z;
      pi.w = ri.w * mi.w + beta * pi.w;
      p4[i] = pi;
   }
}

// ---- learned preconditioner M = G^T G inside the FP32 iteration --------
// G (lower rows) and G^T (upper rows) are SELL-32 matrices on the same
// slices as A, with BF16 values (the preconditioner's own precision; the
// flexible CG absorbs it) and 16-bit column offsets where they fit; a
// thread owns four consecutive rows.
template <class V, class I>
__device__ __forceinline__ float4 sell_quad(const int32_t* __restrict__ sp,
                                            const I* __restrict__ scol,
                                            const V* __restrict__ sval,
                                            const float* __restrict__ x, int64_t r0)
{
   const int64_t s = r0 >> 5;
   const int lane0 = (int)(r0 & 31);
   const int32_t beg = sp[s], w = (sp[s + 1] - beg) >> 5;
   float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
   const I* cp = scol + beg + lane0;
   const V* vp = sval + beg + lane0;
#pragma unroll 4
   for (int32_t k = 0; k < w; ++k) {
      const int4 c = load_cols(cp + k * 32, r0);
      const float4 a = load_vals(vp + k * 32);
      acc.x += a.x * __ldg(x + c.x);
      acc.y += a.y * __ldg(x + c.y);
      acc.z += a.z * __ldg(x + c.z);
      acc.w += a.w * __ldg(x + c.w);
   }
   return acc;
}

// t = G r (r the current residual buffer)
template <class V, class I>
__global__ void __launch_bounds__(kRedBlock, 8) lg_lower(int64_t nquads, const int32_t* __restrict__ sp,
                                                      const I* __restrict__ scol,
                                                      const V* __restrict__ sval,
                                                      const float* r0, const float* r1, float* t,
                                                      const MixState* S, int* worked)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   prof_mark(worked);
   const float* __restrict__ r = (S->it & 1) ? r1 : r0;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride)
      *reinterpret_cast<float4*>(t + i * 4) = sell_quad(sp, scol, sval, r, i * 4);
}

// z = G^T t; rho = (r, z); beta of the next direction: flexible
// (Polak-Ribiere) -alpha (z, q) / rho_old, or rho / rho_old right after a
// refinement replaced r (fr = 1)
template <class V, class I>
__global__ void __launch_bounds__(kRedBlock, 8) lg_upper(int64_t nquads, const int32_t* __restrict__ sp,
                                                      const I* __restrict__ scol,
                                                      const V* __restrict__ sval,
                                                      const float* __restrict__ t, float* z,
                                                      const float* r0, const float* r1,
                                                      const float* __restrict__ q, MixState* S,
                                                      double* partials, unsigned* counter, int fr,
                                                      int* worked)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   prof_mark(worked);
   const float* __restrict__ r = (S->it & 1) ? r1 : r0;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const float4 zi = sell_quad(sp, scol, sval, t, i * 4);
      *reinterpret_cast<float4*>(z + i * 4) = zi;
      const float4 ri = *reinterpret_cast<const float4*>(r + i * 4);
      const float4 qi = *reinterpret_cast<const float4*>(q + i * 4);
      v[0] += (double)ri.x * zi.x + (double)ri.y * zi.y + (double)ri.z * zi.z + (double)ri.w * zi.w;
      v[1] += (double)qi.x * zi.x + (double)qi.y * zi.y + (double)qi.z * zi.z + (double)qi.w * zi.w;
   }
   double tt[2];
   if (grid_reduce<2>(v, partials, counter, tt)) {
      const int it = S->it;
      const double old = S->rho[(it + 1) & 1];
      S->rho[it & 1] = tt[0];
      S->beta = fr ? tt[0] / old : -S->alpha * tt[1] / old;
   }
}

// The learned iteration with two fused kernels.  Iteration k (S->it = k):
//   mx_spmv_dir: p_k = z + beta p_{k-1} (p_k = z on a fresh start), formed
//     for every gathered column and stored for the own rows, q = A p_k,
//     alpha = rho / (p_k, q);
//   lg_lower_upd: d += alpha p_k, r_{k+1} = r_k - alpha q for the own rows,
//     t = G r_{k+1} with r_{k+1} formed for every gathered column,
//     ||r_{k+1}|| and the stopping decisions of mx_update, then S->it = k+1;
//   lg_upper: z = G^T t, rho and beta (as above).
// Directions and residuals alternate between two buffers by the parity of
// k, so a gather never meets a value written by the same kernel; the fused
// forms use the same single-rounding expressions wherever a value is formed.
__device__ __forceinline__ float dir_at(const float* __restrict__ z, const float* __restrict__ pp,
                                        int c, float beta, int fresh)
{
   const float zc = __ldg(z + c);
   return fresh ? zc : __fmaf_rn(beta, __ldg(pp + c), zc);
}

template <class T, class I>
__global__ void __launch_bounds__(kRedBlock, 8) mx_spmv_dir(int64_t nquads, const int32_t* __restrict__ sp,
                                                         const I* __restrict__ scol,
                                                         const T* __restrict__ sval,
                                                         const float* __restrict__ z, float* p0,
                                                         float* p1, float* __restrict__ q,
                                                         MixState* S, double* partials,
                                                         unsigned* counter, int fresh, int* worked)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   prof_mark(worked);
   const int it = S->it;
   const float* __restrict__ pp = (it & 1) ? p0 : p1;
   float* __restrict__ pn = (it & 1) ? p1 : p0;
   const float beta = fresh ? 0.f : (float)S->beta;
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nquads; t += stride) {
      const int64_t r0 = t * 4;
      const int64_t s = r0 >> 5;
      const int lane0 = (int)(r0 & 31);
      const int32_t beg = sp[s], w = (sp[s + 1] - beg) >> 5;
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      const I* cp = scol + beg + lane0;
      const T* vp = sval + beg + lane0;
#pragma unroll 8
      for (int32_t k = 0; k < w; ++k) {
         const int4 c = load_cols(cp + k * 32, r0);
         const float4 a = load_vals(vp + k * 32);
         acc.x += a.x * dir_at(z, pp, c.x, beta, fresh);
         acc.y += a.y * dir_at(z, pp, c.y, beta, fresh);
         acc.z += a.z * dir_at(z, pp, c.z, beta, fresh);
         acc.w += a.w * dir_at(z, pp, c.w, beta, fresh);
      }
      *reinterpret_cast<float4*>(q + r0) = acc;
      const float4 zi = *reinterpret_cast<const float4*>(z + r0);
      float4 pi = zi;
      if (!fresh) {
         const float4 po = *reinterpret_cast<const float4*>(pp + r0);
         pi = make_float4(__fmaf_rn(beta, po.x, zi.x), __fmaf_rn(beta, po.y, zi.y),
                          __fmaf_rn(beta, po.z, zi.z), __fmaf_rn(beta, po.w, zi.w));
      }
      *reinterpret_cast<float4*>(pn + r0) = pi;
      v[0] += (double)pi.x * acc.x + (double)pi.y * acc.y + (double)pi.z * acc.z +
              (double)pi.w * acc.w;
   }
   double tt[1];
   if (grid_reduce<1>(v, partials, counter, tt)) S->alpha = S->rho[it & 1] / tt[0];
}

__device__ __forceinline__ float res_at(const float* __restrict__ r, const float* __restrict__ q,
                                        int c, float a)
{
   return __fmaf_rn(-a, __ldg(q + c), __ldg(r + c));
}

template <class V, class I>
__global__ void __launch_bounds__(kRedBlock, 8) lg_lower_upd(int64_t nquads,
                                                          const int32_t* __restrict__ sp,
                                                          const I* __restrict__ scol,
                                                          const V* __restrict__ sval, float* r0,
                                                          float* r1, const float* __restrict__ q,
                                                          const float* p0, const float* p1,
                                                          float* __restrict__ d,
                                                          float* __restrict__ t, MixState* S,
                                                          double* partials, unsigned* counter,
                                                          double delta, double tol, double scale,
                                                          int max_inner, int mode, int* worked)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   prof_mark(worked);
   const int it = S->it;
   const float* __restrict__ rc = (it & 1) ? r1 : r0;
   float* __restrict__ rn = (it & 1) ? r0 : r1;
   const float* __restrict__ p = (it & 1) ? p1 : p0;
   const float a = (float)S->alpha;
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const int64_t r0i = i * 4;
      const float4 ri = *reinterpret_cast<const float4*>(rc + r0i);
      const float4 qi = *reinterpret_cast<const float4*>(q + r0i);
      const float4 pi = *reinterpret_cast<const float4*>(p + r0i);
      float4 di = *reinterpret_cast<const float4*>(d + r0i);
      di = make_float4(__fmaf_rn(a, pi.x, di.x), __fmaf_rn(a, pi.y, di.y), __fmaf_rn(a, pi.z, di.z),
                       __fmaf_rn(a, pi.w, di.w));
      const float4 rv = make_float4(__fmaf_rn(-a, qi.x, ri.x), __fmaf_rn(-a, qi.y, ri.y),
                                    __fmaf_rn(-a, qi.z, ri.z), __fmaf_rn(-a, qi.w, ri.w));
      *reinterpret_cast<float4*>(d + r0i) = di;
      *reinterpret_cast<float4*>(rn + r0i) = rv;
      v[0] += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
      const int64_t s = r0i >> 5;
      const int lane0 = (int)(r0i & 31);
      const int32_t beg = sp[s], w = (sp[s + 1] - beg) >> 5;
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      const I* cp = scol + beg + lane0;
      const V* vp = sval + beg + lane0;
#pragma unroll 4
      for (int32_t k = 0; k < w; ++k) {
         const int4 c = load_cols(cp + k * 32, r0i);
         const float4 g = load_vals(vp + k * 32);
         acc.x += g.x * res_at(rc, q, c.x, a);
         acc.y += g.y * res_at(rc, q, c.y, a);
         acc.z += g.z * res_at(rc, q, c.z, a);
         acc.w += g.w * res_at(rc, q, c.w, a);
      }
      *reinterpret_cast<float4*>(t + r0i) = acc;
   }
   double tt[1];
   if (grid_reduce<1>(v, partials, counter, tt)) {
      S->rn = sqrt(tt[0]);
      const int itn = it + 1;
      S->it = itn;
      if (mode == 0) {
         if (S->rn <= delta * S->rmark || S->rn * scale <= tol * S->bnorm || itn >= max_inner)
            S->pause = 1;
      }
      else if (S->rn <= delta * S->res0 || itn >= max_inner) {
         S->pause = 1;
      }
   }
}

// x += scale * d (FP64)
__global__ void mx_correct(int64_t n, double* x, const float* __restrict__ d, double scale)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      x[i] += scale * (double)d[i];
}

// D^{-1} in FP32, zero in the padding; IDENT: ones
__global__ void inv_diag32(int64_t n, int64_t npad, const int32_t* dpos, const double* val,
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
      if (a == 0.0) atomicOr(bad, 1);
      dinv[i] = (float)(1.0 / a);
   }
}

}  // namespace

void solve_mixed(ofg_matrix* A, int prec_type, int inner_bits, int mode, const double* b, double* x,
                 int max_outer, int max_inner, double inner_tol, double tol, int* outer, int* inner,
                 double* true_res, ofg_prec* LP, int* fell_back)
{
   const bool learned = LP != nullptr;
   OFG_REQUIRE(learned || prec_type == OFG_DIAG || prec_type == OFG_IDENT, OFG_ERR_ARG,
               "mixed-precision inner solver supports DIAG and IDENT");
   OFG_REQUIRE(inner_bits == 32 || inner_bits == 16, OFG_ERR_ARG, "inner_bits must be 32 or 16");
   OFG_REQUIRE(mode == 0 || mode == 1, OFG_ERR_ARG, "mode must be 0 or 1");
   OFG_REQUIRE(inner_tol > 0 && inner_tol < 1, OFG_ERR_ARG, "inner_tol must be in (0, 1)");
   const int64_t n = A->n;
   ensure_sell(A);
   ensure_dpos(A);
   OFG_REQUIRE(A->dpos_complete, OFG_ERR_PIVOT, "a row has no diagonal entry");
   bool g16 = false;
   if (learned) {
      if (LP->version != A->version) prec_setup(LP);
      ensure_sell_bf16(LP->gl);
      ensure_sell_bf16(LP->gu);
      g16 = ensure_sell_d16(LP->gl) && ensure_sell_d16(LP->gu);
      OFG_REQUIRE(LP->gl->nslices == A->nslices && LP->gu->nslices == A->nslices, OFG_ERR_ARG,
                  "learned factor does not match the matrix");
   }
   const int64_t npad = A->nslices * 32, nquads = npad / 4;
   // 16-bit column offsets when every |column - row| fits (banded orderings,
   // structured meshes): 2 bytes less per entry streamed by every SpMV
   const bool a16 = ensure_sell_d16(A);
   const double aidx = a16 ? 2.0 : 4.0;
   DBuf<__nv_bfloat16> v16;
   if (inner_bits == 32) ensure_sell32(A);
   else {
      v16.alloc(A->sell_val.n);
      cast_values<__nv_bfloat16><<<grid_for(A->sell_val.n, 256), 256, 0, stream()>>>(
         A->sell_val.n, A->sell_val.p, v16.p);
      count_launch();
   }
   const int64_t nv = npad > 0 ? npad : 4;
   DBuf<float> dinv(nv), rr(nv), p(nv), q(nv), d(nv);
   DBuf<float> tz(learned ? nv : 1), zz(learned ? nv : 1);
   // the learned iteration's second residual and direction buffers
   DBuf<float> rr1(learned ? nv : 1), p1(learned ? nv : 1);
   DBuf<double> r(n > 0 ? n : 1), q64(n > 0 ? n : 1);
   DBuf<MixState> S(1);
   DBuf<int> bad(1);
   bad.zero();
   p.zero();
   q.zero();
   if (learned) {
      p1.zero();
      rr1.zero();
   }
   const unsigned g = grid_for(std::max<int64_t>(n, nquads), kRedBlock, 8);
   DBuf<double> partials(((size_t)g + 1) * 4 + 4);
   DBuf<unsigned> counter(1);
   counter.zero();
   inv_diag32<<<grid_for(nv, 256), 256, 0, stream()>>>(n, npad, A->dpos.p, A->val.p, dinv.p,
                                                        prec_type == OFG_IDENT ? 1 : 0, bad.p);
   count_launch();
   int hb = 0;
   bad.download(&hb, 1);
   OFG_REQUIRE(!hb, OFG_ERR_PIVOT, "zero diagonal entry");
   const float* jac = learned ? nullptr : dinv.p;
   const unsigned gq = grid_for(nquads, kRedBlock, 8);
   const unsigned gn = grid_for(n, kRedBlock, 8);
   auto true_residual = [&](int first) {
      spmv_sell(A, x, q64.p);
      mx_residual<<<gn, kRedBlock, 0, stream()>>>(n, b, q64.p, r.p, S.p, partials.p, counter.p,
                                                  tol, first);
      count_launch();
      OFG_LAUNCH_CHECK();
   };
   // the learned preconditioner's products: t = G r (plain, at the start of
   // an outer iteration; fused with the update inside it), z = G^T t with
   // rho and beta.  Algorithmic bytes: BF16 value + column index (2 or 4
   // bytes) per entry, the gathered input(s), the outputs, and the own-row
   // vectors of the fused update (r, q, p, d read; r, d written)
   const double gidx = g16 ? 2.0 : 4.0;
   double scale = 1.0;
   using bf = __nv_bfloat16;
   const bf* vl = reinterpret_cast<const bf*>(learned ? LP->gl->sell_valbf.p : nullptr);
   const bf* vu = reinterpret_cast<const bf*>(learned ? LP->gu->sell_valbf.p : nullptr);
   auto learned_lower = [&]() {
      int* worked = prof_begin();
      if (g16)
         launch_pdl(lg_lower<bf, int16_t>, gq, kRedBlock, nquads, LP->gl->sell_ptr.p,
                    LP->gl->sell_d16.p, vl, rr.p, rr1.p, tz.p, S.p, worked);
      else
         launch_pdl(lg_lower<bf, int32_t>, gq, kRedBlock, nquads, LP->gl->sell_ptr.p,
                    LP->gl->sell_col.p, vl, rr.p, rr1.p, tz.p, S.p, worked);
      prof_end(PROF_LEARNED_APPLY, (2.0 + gidx) * LP->gl->nnz + 8.0 * n);
   };
   auto learned_upper = [&](int fr) {
      int* worked = prof_begin();
      if (g16)
         launch_pdl(lg_upper<bf, int16_t>, gq, kRedBlock, nquads, LP->gu->sell_ptr.p,
                    LP->gu->sell_d16.p, vu, tz.p, zz.p, rr.p, rr1.p, q.p, S.p, partials.p,
                    counter.p, fr, worked);
      else
         launch_pdl(lg_upper<bf, int32_t>, gq, kRedBlock, nquads, LP->gu->sell_ptr.p,
                    LP->gu->sell_col.p, vu, tz.p, zz.p, rr.p, rr1.p, q.p, S.p, partials.p,
                    counter.p, fr, worked);
      prof_end(PROF_LEARNED_APPLY, (2.0 + gidx) * LP->gu->nnz + 16.0 * n);
   };
   auto learned_lower_update = [&]() {
      int* worked = prof_begin();
      if (g16)
         launch_pdl(lg_lower_upd<bf, int16_t>, gq, kRedBlock, nquads, LP->gl->sell_ptr.p,
                    LP->gl->sell_d16.p, vl, rr.p, rr1.p, q.p, p.p, p1.p, d.p, tz.p, S.p,
                    partials.p, counter.p, inner_tol, tol, scale, max_inner, mode, worked);
      else
         launch_pdl(lg_lower_upd<bf, int32_t>, gq, kRedBlock, nquads, LP->gl->sell_ptr.p,
                    LP->gl->sell_col.p, vl, rr.p, rr1.p, q.p, p.p, p1.p, d.p, tz.p, S.p,
                    partials.p, counter.p, inner_tol, tol, scale, max_inner, mode, worked);
      prof_end(PROF_LEARNED_APPLY, (2.0 + gidx) * LP->gl->nnz + 32.0 * n);
   };
   MixState h{};
   true_residual(1);
   S.download(&h, 1);
   int n_outer = 0;
   // mode 1 solves for d in units of ||r||; mode 0 keeps absolute units
   // (scale is declared with the launch helpers above)
   bool fresh = true;
   // stagnation watch of the learned iteration: the recursive residual must
   // halve within kStallIters iterations and stay finite, and the true
   // residual must fall at every refinement
   constexpr int kStallIters = 500;
   bool stalled = false;
   int no_gain = 0;
   double last_rel = h.rel;
   while (!h.done && n_outer < max_outer && h.it < max_inner && n > 0) {
      if (mode == 1) {
         scale = h.rel * h.bnorm;
         fresh = true;
      }
      mx_load_residual<<<gq, kRedBlock, 0, stream()>>>(n, npad, r.p, 1.0 / scale, jac, rr.p,
                                                       learned ? rr1.p : nullptr, p.p, d.p,
                                                       fresh ? 1 : 0, S.p, partials.p, counter.p);
      count_launch();
      // the learned iteration's first direction is formed by its first
      // mx_spmv_dir (p = z on a fresh start, z + beta p with fr = 1 after a
      // refinement in absolute units)
      bool dir_fresh = fresh;
      if (learned) {
         learned_lower();
         learned_upper(fresh ? 0 : 1);
      }
      else if (!fresh) {
         mx_direction<<<gq, kRedBlock, 0, stream()>>>(nquads, rr.p, dinv.p, p.p, S.p);
         count_launch();
      }
      fresh = false;
      int mark_it = h.it;
      double mark_rn = h.rel * h.bnorm / scale;
      int batch = 8;
      for (;;) {
         for (int k = 0; k < batch; ++k) {
            // the kernels of an iteration chain with programmatic dependent
            // launch: each one's blocks start while the previous one drains
            // its reduction tail
            int* worked = prof_begin();
            if (learned) {
               const int fr = dir_fresh ? 1 : 0;
               dir_fresh = false;
               if (inner_bits == 32 && a16)
                  launch_pdl(mx_spmv_dir<float, int16_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                             A->sell_d16.p, A->sell_val32.p, zz.p, p.p, p1.p, q.p, S.p,
                             partials.p, counter.p, fr, worked);
               else if (inner_bits == 32)
                  launch_pdl(mx_spmv_dir<float, int32_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                             A->sell_col.p, A->sell_val32.p, zz.p, p.p, p1.p, q.p, S.p,
                             partials.p, counter.p, fr, worked);
               else if (a16)
                  launch_pdl(mx_spmv_dir<__nv_bfloat16, int16_t>, gq, kRedBlock, nquads,
                             A->sell_ptr.p, A->sell_d16.p, v16.p, zz.p, p.p, p1.p, q.p, S.p,
                             partials.p, counter.p, fr, worked);
               else
                  launch_pdl(mx_spmv_dir<__nv_bfloat16, int32_t>, gq, kRedBlock, nquads,
                             A->sell_ptr.p, A->sell_col.p, v16.p, zz.p, p.p, p1.p, q.p, S.p,
                             partials.p, counter.p, fr, worked);
               // values + column indices, z and p_prev gathered, p and q written
               prof_end(inner_bits == 32 ? PROF_SPMV32 : PROF_SPMV16,
                        ((inner_bits == 32 ? 4.0 : 2.0) + aidx) * A->nnz + 16.0 * n + 4.0);
               learned_lower_update();
               learned_upper(0);
               continue;
            }
            if (inner_bits == 32 && a16)
               launch_pdl(mx_spmv<float, int16_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_d16.p, A->sell_val32.p, p.p, q.p, S.p, partials.p, counter.p,
                          worked);
            else if (inner_bits == 32)
               launch_pdl(mx_spmv<float, int32_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_col.p, A->sell_val32.p, p.p, q.p, S.p, partials.p, counter.p,
                          worked);
            else if (a16)
               launch_pdl(mx_spmv<__nv_bfloat16, int16_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_d16.p, v16.p, p.p, q.p, S.p, partials.p, counter.p, worked);
            else
               launch_pdl(mx_spmv<__nv_bfloat16, int32_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_col.p, v16.p, p.p, q.p, S.p, partials.p, counter.p, worked);
            // algorithmic bytes: value (4 or 2) + column index (4, or 2 as a
            // 16-bit offset) per entry, p gathered, q written, p read for the dot
            prof_end(inner_bits == 32 ? PROF_SPMV32 : PROF_SPMV16,
                     ((inner_bits == 32 ? 4.0 : 2.0) + aidx) * A->nnz + 12.0 * n + 4.0);
            launch_pdl(mx_update<true>, gq, kRedBlock, nquads, d.p, p.p, rr.p, q.p, dinv.p, S.p,
                       partials.p, counter.p, inner_tol, tol, scale, max_inner, mode);
            launch_pdl(mx_direction, gq, kRedBlock, nquads, rr.p, dinv.p, p.p, S.p);
         }
         OFG_LAUNCH_CHECK();
         S.download(&h, 1);
         if (learned) {
            if (!std::isfinite(h.rn)) stalled = true;
            else if (h.it - mark_it >= kStallIters) {
               if (h.rn > 0.5 * mark_rn) stalled = true;
               mark_it = h.it;
               mark_rn = h.rn;
            }
            if (stalled) break;
         }
         if (h.pause) break;
         batch = std::min(batch * 2, 64);
      }
      if (stalled) break;
      // refinement step in FP64
      mx_correct<<<gn, kRedBlock, 0, stream()>>>(n, x, d.p, scale);
      count_launch();
      true_residual(0);
      S.download(&h, 1);
      n_outer++;
      if (learned) {
         no_gain = (h.rel > 0.9 * last_rel) ? no_gain + 1 : 0;
         last_rel = h.rel;
         if (!std::isfinite(h.rel) || no_gain >= 3) {
            stalled = true;
            break;
         }
      }
   }
   if (learned && stalled && !h.done) {
      // fallback: the plain Jacobi iteration from the last x whose FP64
      // residual was measured (a non-finite x is reset to zero)
      if (!std::isfinite(h.rel)) OFG_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), stream()));
      if (fell_back) *fell_back = 1;
      int o2 = 0, i2 = 0;
      solve_mixed(A, OFG_DIAG, inner_bits, mode, b, x, std::max(1, max_outer - n_outer),
                  std::max(1, max_inner - h.it), inner_tol, tol, &o2, &i2, true_res, nullptr,
                  nullptr);
      *outer = n_outer + o2;
      *inner = h.it + i2;
      return;
   }
   *outer = n_outer;
   *inner = h.it;
   *true_res = h.rel;
}

}  // namespace ofg

using namespace ofg;

extern "C" int ofg_solve_mixed(ofg_matrix* A, int prec_type, int inner_bits, int mode,
                               const double* b, double* x, int max_outer, int max_inner,
                               double inner_tol, double toler, int* outer, int* inner,
                               double* true_res)
{
   return guarded("ofg_solve_mixed", [&] {
      OFG_REQUIRE(A && b && x && outer && inner && true_res, OFG_ERR_ARG, "null argument");
      In<double> db(b, A->n);
      InOut<double> dx(x, A->n, true);
      solve_mixed(A, prec_type, inner_bits, mode, db.d, dx.d, max_outer, max_inner, inner_tol,
                  toler, outer, inner, true_res, nullptr, nullptr);
      dx.finish();
   });
}

// Flexible CG with the learned preconditioner in FP32 inside FP64 iterative
// refinement (mode 0); falls back to the plain Jacobi iteration when the
// learned iteration stagnates (*fell_back = 1).  Convergence is declared on
// the FP64 true residual only.
extern "C" int ofg_fcg_learned(ofg_prec* P, int inner_bits, const double* b, double* x,
                               int max_outer, int max_inner, double inner_tol, double toler,
                               int* outer, int* inner, double* true_res, int* fell_back)
{
   return guarded("ofg_fcg_learned", [&] {
      OFG_REQUIRE(P && b && x && outer && inner && true_res, OFG_ERR_ARG, "null argument");
      OFG_REQUIRE(P->type == OFG_LEARNED, OFG_ERR_ARG, "not a learned preconditioner");
      if (fell_back) *fell_back = 0;
      ofg_matrix* A = P->A;
      In<double> db(b, A->n);
      InOut<double> dx(x, A->n, true);
      solve_mixed(A, OFG_DIAG, inner_bits, 0, db.d, dx.d, max_outer, max_inner, inner_tol, toler,
                  outer, inner, true_res, P, fell_back);
      dx.finish();
   });
}
