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
// is not thrown away at every refinement, so the iteration count stays that
// of FP64 CG).
// Mode 1 (classic restarted refinement): every refinement solves
// A d = r / ||r|| from d = 0 to `inner_tol` and adds ||r|| d.
//
// FP64 is used only for b - A x, the refinement update x += ..., and the
// accumulation of every Krylov dot product.  One FP32 CG iteration streams
// 8*nnz + 56*n bytes (6*nnz + 56*n with BF16 values) against 12*nnz + 112*n
// in FP64.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "internal.cuh"
#include "reduce.cuh"

namespace ofg {
namespace {

struct MixState {
   double bnorm, rel;                 // FP64 true residual
   double rho, rho_new, alpha, rn, rmark, res0;
   int it, pause, done, pad;
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

// r = b - q (FP64); ||r||, ||b|| (first call); convergence test
__global__ void __launch_bounds__(kRedBlock) mx_residual(int64_t n, const double* __restrict__ b,
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

// r_lo = (float)(r * scale); rho_new = (r_lo, D r_lo); ||r_lo||; optionally
// d = 0 and p = D r_lo (fresh start)
__global__ void __launch_bounds__(kRedBlock) mx_load_residual(int64_t n,
                                                              const double* __restrict__ r,
                                                              double scale,
                                                              const float* __restrict__ dinv,
                                                              float* rr, float* p, float* d,
                                                              int fresh, MixState* S,
                                                              double* partials, unsigned* counter)
{
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const float ri = (float)(r[i] * scale);
      const float zi = ri * dinv[i];
      rr[i] = ri;
      d[i] = 0.0f;
      if (fresh) p[i] = zi;
      v[0] += (double)ri * (double)zi;
      v[1] += (double)ri * (double)ri;
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      S->rho_new = t[0];
      if (fresh) S->rho = t[0];
      S->rn = sqrt(t[1]);
      S->rmark = S->rn;
      if (fresh) S->res0 = S->rn;
      S->pause = 0;
   }
}

template <class T>
__global__ void __launch_bounds__(kRedBlock) mx_spmv(int64_t n, int64_t nslices,
                                                     const int32_t* __restrict__ sp,
                                                     const int32_t* __restrict__ scol,
                                                     const T* __restrict__ sval,
                                                     const float* __restrict__ p,
                                                     float* __restrict__ q, MixState* S,
                                                     double* partials, unsigned* counter,
                                                     int* worked)
{
   if (S->pause) return;
   prof_mark(worked);
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

// d += alpha p, r -= alpha q; ||r||, (r, D r); decides when the host must
// refine (mode 0) or stop the inner solve (mode 1)
__global__ void __launch_bounds__(kRedBlock) mx_update(int64_t n, float* d,
                                                       const float* __restrict__ p, float* rr,
                                                       const float* __restrict__ q,
                                                       const float* __restrict__ dinv, MixState* S,
                                                       double* partials, unsigned* counter,
                                                       double delta, double tol, double scale,
                                                       int max_inner, int mode)
{
   if (S->pause) return;
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
      S->rn = sqrt(t[0]);
      S->rho_new = t[1];
      S->it += 1;
      if (mode == 0) {
         // refine when the residual fell by delta, or when the recurrence
         // says the FP64 target is reached
         if (S->rn <= delta * S->rmark || S->rn * scale <= tol * S->bnorm || S->it >= max_inner)
            S->pause = 1;
      }
      else if (S->rn <= delta * S->res0 || S->it >= max_inner) {
         S->pause = 1;
      }
   }
}

__global__ void __launch_bounds__(kRedBlock) mx_direction(int64_t n, const float* __restrict__ rr,
                                                          const float* __restrict__ dinv, float* p,
                                                          MixState* S)
{
   if (S->pause) return;
   const float beta = (float)(S->rho_new / S->rho);
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      p[i] = rr[i] * dinv[i] + beta * p[i];
}

// rho <- rho_new, after every block of mx_direction has read rho
__global__ void mx_rho_shift(MixState* S)
{
   if (S->pause) return;
   S->rho = S->rho_new;
}

// x += scale * d (FP64)
__global__ void mx_correct(int64_t n, double* x, const float* __restrict__ d, double scale)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      x[i] += scale * (double)d[i];
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

__global__ void fill_ones(int64_t n, float* p)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = 1.0f;
}

}  // namespace

void solve_mixed(ofg_matrix* A, int prec_type, int inner_bits, int mode, const double* b, double* x,
                 int max_outer, int max_inner, double inner_tol, double tol, int* outer, int* inner,
                 double* true_res)
{
   OFG_REQUIRE(prec_type == OFG_DIAG || prec_type == OFG_IDENT, OFG_ERR_ARG,
               "mixed-precision inner solver supports DIAG and IDENT");
   OFG_REQUIRE(inner_bits == 32 || inner_bits == 16, OFG_ERR_ARG, "inner_bits must be 32 or 16");
   OFG_REQUIRE(mode == 0 || mode == 1, OFG_ERR_ARG, "mode must be 0 or 1");
   OFG_REQUIRE(inner_tol > 0 && inner_tol < 1, OFG_ERR_ARG, "inner_tol must be in (0, 1)");
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
   DBuf<MixState> S(1);
   DBuf<int> bad(1);
   bad.zero();
   DBuf<double> partials(((size_t)grid_for(n, kRedBlock, 8) + 1) * 4 + 4);
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
      fill_ones<<<grid_for(n, 256), 256, 0, stream()>>>(n, dinv.p);
      count_launch();
   }
   const unsigned g = grid_for(n, kRedBlock, 8);
   const unsigned gs = grid_for(A->nslices * 32, kRedBlock, 8);
   auto true_residual = [&](int first) {
      spmv_sell(A, x, q64.p);
      mx_residual<<<g, kRedBlock, 0, stream()>>>(n, b, q64.p, r.p, S.p, partials.p, counter.p, tol,
                                                 first);
      count_launch();
      OFG_LAUNCH_CHECK();
   };
   MixState h{};
   true_residual(1);
   S.download(&h, 1);
   int n_outer = 0;
   // mode 1 solves for d in units of ||r||; mode 0 keeps absolute units
   double scale = 1.0;
   bool fresh = true;
   while (!h.done && n_outer < max_outer && h.it < max_inner) {
      if (mode == 1) {
         scale = h.rel * h.bnorm;
         fresh = true;
      }
      mx_load_residual<<<g, kRedBlock, 0, stream()>>>(n, r.p, 1.0 / scale, dinv.p, rr.p, p.p, d.p,
                                                      fresh ? 1 : 0, S.p, partials.p, counter.p);
      count_launch();
      if (!fresh) {
         mx_direction<<<g, kRedBlock, 0, stream()>>>(n, rr.p, dinv.p, p.p, S.p);
         mx_rho_shift<<<1, 1, 0, stream()>>>(S.p);
         count_launch(2);
      }
      fresh = false;
      int batch = 8;
      for (;;) {
         for (int k = 0; k < batch; ++k) {
            int* worked = prof_begin();
            if (inner_bits == 32)
               mx_spmv<float><<<gs, kRedBlock, 0, stream()>>>(n, A->nslices, A->sell_ptr.p,
                                                             A->sell_col.p, A->sell_val32.p, p.p,
                                                             q.p, S.p, partials.p, counter.p,
                                                             worked);
            else
               mx_spmv<__nv_bfloat16><<<gs, kRedBlock, 0, stream()>>>(
                  n, A->nslices, A->sell_ptr.p, A->sell_col.p, v16.p, p.p, q.p, S.p, partials.p,
                  counter.p, worked);
            prof_end(inner_bits == 32 ? PROF_SPMV32 : PROF_SPMV16,
                     (inner_bits == 32 ? 8.0 : 6.0) * A->nnz + 12.0 * n + 4.0);
            mx_update<<<g, kRedBlock, 0, stream()>>>(n, d.p, p.p, rr.p, q.p, dinv.p, S.p,
                                                     partials.p, counter.p, inner_tol, tol, scale,
                                                     max_inner, mode);
            mx_direction<<<g, kRedBlock, 0, stream()>>>(n, rr.p, dinv.p, p.p, S.p);
            mx_rho_shift<<<1, 1, 0, stream()>>>(S.p);
            count_launch(4);
         }
         OFG_LAUNCH_CHECK();
         S.download(&h, 1);
         if (h.pause) break;
         batch = std::min(batch * 2, 64);
      }
      // refinement step in FP64
      mx_correct<<<g, kRedBlock, 0, stream()>>>(n, x, d.p, scale);
      count_launch();
      true_residual(0);
      S.download(&h, 1);
      n_outer++;
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
                  toler, outer, inner, true_res);
      dx.finish();
   });
}
