// mixed.cu -- mixed-precision solve: FP64 iterative refinement around a
// preconditioned CG that runs in FP32 (or with BF16 matrix values).
//
//   r = b - A x                     FP64 SpMV + FP64 residual norm
//   solve A d = r / ||r||           inner PCG, FP32 vectors, FP32/BF16 A,
//                                   Jacobi preconditioner in FP32, FP64 dots
//   x += ||r|| d                    FP64 update
// until ||b - A x|| / ||b|| <= toler.  Only the true residual, the refinement
// update and the Krylov dot products are FP64; the inner SpMV streams 8 (FP32)
// or 6 (BF16) bytes per nonzero instead of 12.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "internal.cuh"
#include "reduce.cuh"

namespace ofg {
namespace {

struct IRState {
   double bnorm, rnorm, rel;                  // outer
   double rho, rho_old, alpha, res0, res;     // inner (FP64 scalars)
   int it, done, pad0, pad1;
};

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

template <class T>
__global__ void cast_values(int64_t total, const double* __restrict__ src, T* dst)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
      dst[i] = (T)src[i];
}

__global__ void __launch_bounds__(kRedBlock) ir_residual(int64_t n, const double* __restrict__ b,
                                                         const double* __restrict__ q, double* r,
                                                         IRState* S, double* partials,
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
      }
      S->rnorm = sqrt(t[0]);
      S->rel = S->rnorm / S->bnorm;
      S->done = S->rel <= tol ? 1 : 0;
   }
}

// inner start: rr = r/||r|| (FP32), x32 = 0, z = D rr, p = z, rho = (rr, z)
__global__ void __launch_bounds__(kRedBlock) in_start(int64_t n, const double* __restrict__ r,
                                                      const float* __restrict__ dinv, float* rr,
                                                      float* p, float* d, IRState* S,
                                                      double* partials, unsigned* counter)
{
   const double sc = 1.0 / S->rnorm;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const float ri = (float)(r[i] * sc);
      const float zi = ri * dinv[i];
      rr[i] = ri;
      p[i] = zi;
      d[i] = 0.0f;
      v[0] += (double)ri * (double)zi;
      v[1] += (double)ri * (double)ri;
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      S->rho = t[0];
      S->res0 = sqrt(t[1]);
      S->res = S->res0;
      S->it = 0;
   }
}

template <class T>
__global__ void __launch_bounds__(kRedBlock) in_spmv(int64_t n, int64_t nslices,
                                                     const int32_t* __restrict__ sp,
                                                     const int32_t* __restrict__ scol,
                                                     const T* __restrict__ sval,
                                                     const float* __restrict__ p,
                                                     float* __restrict__ q, IRState* S,
                                                     double* partials, unsigned* counter,
                                                     const int* stop)
{
   if (*stop) return;
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < nslices * 32;
        row += stride) {
      const int64_t s = row >> 5;
      const int lane = (int)(row & 31);
      const int32_t beg = sp[s], end = sp[s + 1];
      float acc = 0.0f;
      for (int32_t k = beg + lane; k < end; k += 32) acc += to_f(sval[k]) * __ldg(p + scol[k]);
      if (row < n) {
         q[row] = acc;
         v[0] += (double)p[row] * (double)acc;
      }
   }
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t)) S->alpha = S->rho / t[0];
}

// d += alpha p, rr -= alpha q, z = D rr, rho' = (rr, z), ||rr||
__global__ void __launch_bounds__(kRedBlock) in_update(int64_t n, float* d,
                                                       const float* __restrict__ p, float* rr,
                                                       const float* __restrict__ q,
                                                       const float* __restrict__ dinv, IRState* S,
                                                       double* partials, unsigned* counter,
                                                       double inner_tol, int max_inner, int* stop)
{
   if (*stop) return;
   const float a = (float)S->alpha;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      d[i] += a * p[i];
      const float ri = rr[i] - a * q[i];
      rr[i] = ri;
      v[0] += (double)ri * (double)ri;
      v[1] += (double)ri * (double)(ri * dinv[i]);
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      S->res = sqrt(t[0]);
      S->it += 1;
      S->rho_old = S->rho;
      S->rho = t[1];
      if (S->res <= inner_tol * S->res0 || S->it >= max_inner) *stop = 1;
   }
}

__global__ void __launch_bounds__(kRedBlock) in_direction(int64_t n, const float* __restrict__ rr,
                                                          const float* __restrict__ dinv, float* p,
                                                          const IRState* S, const int* stop)
{
   if (*stop) return;
   const float beta = (float)(S->rho / S->rho_old);
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      p[i] = rr[i] * dinv[i] + beta * p[i];
}

__global__ void ir_correct(int64_t n, double* x, const float* __restrict__ d, const IRState* S)
{
   const double sc = S->rnorm;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      x[i] += sc * (double)d[i];
}

__global__ void inv_diag32(int64_t n, const int32_t* dpos, const double* val, float* dinv, int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const int32_t k = dpos[i];
      const double a = k >= 0 ? val[k] : 0.0;
      if (a == 0.0) atomicOr(bad, 1);
      dinv[i] = (float)(1.0 / a);
   }
}

}  // namespace

void solve_mixed(ofg_matrix* A, int prec_type, int inner_bits, const double* b, double* x,
                 int max_outer, int max_inner, double inner_tol, double tol, int* outer, int* inner,
                 double* true_res)
{
   OFG_REQUIRE(prec_type == OFG_DIAG || prec_type == OFG_IDENT, OFG_ERR_ARG,
               "mixed-precision inner solver supports DIAG and IDENT");
   OFG_REQUIRE(inner_bits == 32 || inner_bits == 16, OFG_ERR_ARG, "inner_bits must be 32 or 16");
   const int64_t n = A->n;
   ensure_sell(A);
   ensure_dpos(A);
   OFG_REQUIRE(A->dpos_complete, OFG_ERR_PIVOT, "a row has no diagonal entry");
   DBuf<__nv_bfloat16> v16;
   if (inner_bits == 32) ensure_sell32(A);
   else {
      v16.alloc(A->sell_val.n);
      cast_values<__nv_bfloat16><<<grid_for(A->sell_val.n, 256), 256, 0, stream()>>>(
         A->sell_val.n, A->sell_val.p, v16.p);
      count_launch();
   }
   DBuf<float> dinv(n), rr(n), p(n), q(n), d(n);
   DBuf<double> r(n), q64(n);
   DBuf<IRState> S(1);
   DBuf<int> stop(1), bad(1);
   bad.zero();
   DBuf<double> partials((size_t)grid_for(n, kRedBlock, 4) * 4 + 4);
   DBuf<unsigned> counter(1);
   counter.zero();
   if (prec_type == OFG_DIAG) {
      inv_diag32<<<grid_for(n, 256), 256, 0, stream()>>>(n, A->dpos.p, A->val.p, dinv.p, bad.p);
      count_launch();
      int h = 0;
      bad.download(&h, 1);
      OFG_REQUIRE(!h, OFG_ERR_PIVOT, "zero diagonal entry");
   }
   else {
      std::vector<float> ones(n, 1.0f);
      dinv.upload(ones.data(), n);
   }
   const unsigned g = grid_for(n, kRedBlock, 4);
   const unsigned gs = grid_for(A->nslices * 32, kRedBlock, 4);
   spmv_sell(A, x, q64.p);
   ir_residual<<<g, kRedBlock, 0, stream()>>>(n, b, q64.p, r.p, S.p, partials.p, counter.p, tol, 1);
   count_launch();
   OFG_LAUNCH_CHECK();
   IRState h{};
   S.download(&h, 1);
   int n_outer = 0, n_inner = 0;
   while (!h.done && n_outer < max_outer) {
      stop.zero();
      in_start<<<g, kRedBlock, 0, stream()>>>(n, r.p, dinv.p, rr.p, p.p, d.p, S.p, partials.p,
                                              counter.p);
      count_launch();
      int hs = 0;
      int batch = 8;
      for (;;) {
         // in_start left p = D rr; each step is spmv, update, new direction
         for (int k = 0; k < batch; ++k) {
            if (inner_bits == 32)
               in_spmv<float><<<gs, kRedBlock, 0, stream()>>>(n, A->nslices, A->sell_ptr.p,
                                                             A->sell_col.p, A->sell_val32.p, p.p,
                                                             q.p, S.p, partials.p, counter.p,
                                                             stop.p);
            else
               in_spmv<__nv_bfloat16><<<gs, kRedBlock, 0, stream()>>>(
                  n, A->nslices, A->sell_ptr.p, A->sell_col.p, v16.p, p.p, q.p, S.p, partials.p,
                  counter.p, stop.p);
            in_update<<<g, kRedBlock, 0, stream()>>>(n, d.p, p.p, rr.p, q.p, dinv.p, S.p,
                                                     partials.p, counter.p, inner_tol, max_inner,
                                                     stop.p);
            in_direction<<<g, kRedBlock, 0, stream()>>>(n, rr.p, dinv.p, p.p, S.p, stop.p);
            count_launch(3);
         }
         OFG_LAUNCH_CHECK();
         stop.download(&hs, 1);
         if (hs) break;
         batch = std::min(batch * 2, 64);
      }
      ir_correct<<<g, kRedBlock, 0, stream()>>>(n, x, d.p, S.p);
      count_launch();
      S.download(&h, 1);
      n_inner += h.it;
      n_outer++;
      spmv_sell(A, x, q64.p);
      ir_residual<<<g, kRedBlock, 0, stream()>>>(n, b, q64.p, r.p, S.p, partials.p, counter.p, tol,
                                                 0);
      count_launch();
      OFG_LAUNCH_CHECK();
      S.download(&h, 1);
   }
   *outer = n_outer;
   *inner = n_inner;
   *true_res = h.rel;
}

}  // namespace ofg

using namespace ofg;

extern "C" int ofg_solve_mixed(ofg_matrix* A, int prec_type, int inner_bits, const double* b,
                               double* x, int max_outer, int max_inner, double inner_tol,
                               double toler, int* outer, int* inner, double* true_res)
{
   return guarded("ofg_solve_mixed", [&] {
      OFG_REQUIRE(A && b && x && outer && inner && true_res, OFG_ERR_ARG, "null argument");
      In<double> db(b, A->n);
      InOut<double> dx(x, A->n, true);
      solve_mixed(A, prec_type, inner_bits, db.d, dx.d, max_outer, max_inner, inner_tol, toler,
                  outer, inner, true_res);
      dx.finish();
   });
}
