// bicgstab.cu -- OFELI's BiCGStab(A, P, b, x, max_it, toler)
// (include/solvers/BiCGStab.h:87-161) on the device: the same recurrence and
// the same return convention (iterations; 2 when (rr, r) vanishes; 3 when
// omega vanishes; -(max_it + 1) when the loop runs out; the tests on ||s|| and
// ||r|| are strict, as in OFELI).  Scalars live in device memory; the host
// launches iterations in batches and reads the state between batches.  Every
// kernel of an iteration is a no-op once the state says done, and the
// preconditioner sweeps and SpMVs take the same flag.
//
// Per iteration: two preconditioner applications, two FP64 SpMVs, four
// reductions ((rr, r); (rr, v); ||s||; (t, s) with (t, t); ||r||), and the
// vector updates fused into the kernels that produce their inputs.
#include "internal.cuh"
#include "reduce.cuh"

namespace ofg {
namespace {

struct BiState {
   double nrm, res, rho1, rho2, alpha, omega, beta;
   int it, done, result, stop_s;
};

// r = b - q, rr = r, ||b||, ||r||; the test before the first iteration
__global__ void __launch_bounds__(kRedBlock, 8) bi_init(int64_t n, const double* __restrict__ b,
                                                     const double* __restrict__ q, double* r,
                                                     double* rr, BiState* S, double* partials,
                                                     unsigned* counter, double tol)
{
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double bi = b[i], ri = bi - q[i];
      r[i] = ri;
      rr[i] = ri;
      v[0] += bi * bi;
      v[1] += ri * ri;
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      double nrm = sqrt(t[0]);
      if (nrm == 0.0) nrm = 1.0;
      S->nrm = nrm;
      S->res = sqrt(t[1]) / nrm;
      S->it = 0;
      S->rho1 = S->rho2 = S->alpha = S->omega = S->beta = 0.0;
      S->stop_s = 0;
      S->done = S->res <= tol ? 1 : 0;
      S->result = 0;
   }
}

// rho1 = (rr, r); the next iteration number; the breakdown test; beta
__global__ void __launch_bounds__(kRedBlock, 8) bi_rho(int64_t n, const double* __restrict__ rr,
                                                    const double* __restrict__ r, BiState* S,
                                                    double* partials, unsigned* counter, int max_it)
{
   if (S->done) return;
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      v[0] += rr[i] * r[i];
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t)) {
      const int it = S->it + 1;
      S->it = it;
      if (it > max_it) {
         S->done = 1;
         S->result = -it;
         return;
      }
      S->rho1 = t[0];
      if (t[0] == 0.0) {
         S->done = 1;
         S->result = 2;
         return;
      }
      if (it > 1) S->beta = (t[0] / S->rho2) * (S->alpha / S->omega);
   }
}

// p = r (first iteration) or r + beta (p - omega v)
__global__ void bi_direction(int64_t n, const double* __restrict__ r, const double* __restrict__ v,
                             double* p, const BiState* S)
{
   if (S->done) return;
   const bool first = S->it == 1;
   const double beta = S->beta, omega = S->omega;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      p[i] = first ? r[i] : r[i] + beta * (p[i] - omega * v[i]);
}

// alpha = rho1 / (rr, v)
__global__ void __launch_bounds__(kRedBlock, 8) bi_alpha(int64_t n, const double* __restrict__ rr,
                                                      const double* __restrict__ v, BiState* S,
                                                      double* partials, unsigned* counter)
{
   if (S->done) return;
   double w[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      w[0] += rr[i] * v[i];
   double t[1];
   if (grid_reduce<1>(w, partials, counter, t)) S->alpha = S->rho1 / t[0];
}

// s = r - alpha v, ||s||; converged at s: done, and x += alpha pp follows
__global__ void __launch_bounds__(kRedBlock, 8) bi_s(int64_t n, const double* __restrict__ r,
                                                  const double* __restrict__ v, double* s,
                                                  BiState* S, double* partials, unsigned* counter,
                                                  double tol)
{
   if (S->done) return;
   const double alpha = S->alpha;
   double w[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double si = r[i] - alpha * v[i];
      s[i] = si;
      w[0] += si * si;
   }
   double t[1];
   if (grid_reduce<1>(w, partials, counter, t)) {
      const double res = sqrt(t[0]) / S->nrm;
      S->res = res;
      if (res < tol) {
         S->done = 1;
         S->result = S->it;
         S->stop_s = 1;
      }
   }
}

// x += alpha pp when the iteration stopped at s (once)
__global__ void bi_x_at_s(int64_t n, double* x, const double* __restrict__ pp, const BiState* S)
{
   if (!S->stop_s) return;
   const double alpha = S->alpha;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      x[i] += alpha * pp[i];
}

__global__ void bi_clear_stop(BiState* S) { S->stop_s = 0; }

// omega = (t, s) / (t, t)
__global__ void __launch_bounds__(kRedBlock, 8) bi_omega(int64_t n, const double* __restrict__ t,
                                                      const double* __restrict__ s, BiState* S,
                                                      double* partials, unsigned* counter)
{
   if (S->done) return;
   double w[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double ti = t[i];
      w[0] += ti * s[i];
      w[1] += ti * ti;
   }
   double tt[2];
   if (grid_reduce<2>(w, partials, counter, tt)) S->omega = tt[0] / tt[1];
}

// x += alpha pp + omega ss; r = s - omega t; ||r||; the end-of-iteration tests
__global__ void __launch_bounds__(kRedBlock, 8) bi_update(int64_t n, double* x,
                                                       const double* __restrict__ pp,
                                                       const double* __restrict__ ss,
                                                       const double* __restrict__ s,
                                                       const double* __restrict__ t, double* r,
                                                       BiState* S, double* partials,
                                                       unsigned* counter, double tol)
{
   if (S->done) return;
   const double alpha = S->alpha, omega = S->omega;
   double w[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      x[i] += alpha * pp[i] + omega * ss[i];
      const double ri = s[i] - omega * t[i];
      r[i] = ri;
      w[0] += ri * ri;
   }
   double tt[1];
   if (grid_reduce<1>(w, partials, counter, tt)) {
      S->rho2 = S->rho1;
      const double res = sqrt(tt[0]) / S->nrm;
      S->res = res;
      if (res < tol) {
         S->done = 1;
         S->result = S->it;
      }
      else if (omega == 0.0) {
         S->done = 1;
         S->result = 3;
      }
   }
}

__global__ void bi_copy(int64_t n, const double* __restrict__ a, double* b, const int* skip)
{
   if (*skip) return;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) b[i] = a[i];
}

}  // namespace

void bicgstab_solve(ofg_prec* P, const double* b, double* x, int max_it, double tol, int* result,
                    double* res)
{
   ofg_matrix* A = P->A;
   const int64_t n = A->n;
   ensure_sell(A);
   if (prec_stale(P)) prec_setup(P);
   DBuf<double> r(n), rr(n), p(n), pp(n), s(n), ss(n), t(n), v(n);
   DBuf<BiState> S(1);
   const unsigned g = grid_for(n, kRedBlock, 8), ge = grid_for(n, 256);
   DBuf<double> partials(((size_t)g + 1) * 2 + 4);
   DBuf<unsigned> counter(1);
   counter.zero();
   p.zero();
   v.zero();
   const bool sweep = P->type != OFG_IDENT && P->type != OFG_DIAG && P->type != OFG_LEARNED;
   if (sweep) {
      fill_sentinel(pp.p, n);
      fill_sentinel(ss.p, n);
   }
   spmv_sell(A, x, v.p);
   bi_init<<<g, kRedBlock, 0, stream()>>>(n, b, v.p, r.p, rr.p, S.p, partials.p, counter.p, tol);
   count_launch();
   OFG_LAUNCH_CHECK();
   const int* done = &S.p->done;
   auto apply = [&](const double* in, double* out) {
      if (P->type == OFG_IDENT) {
         bi_copy<<<ge, 256, 0, stream()>>>(n, in, out, done);
         count_launch();
      }
      else {
         prec_apply_device(P, in, out, nullptr, done);
      }
   };
   BiState h{};
   S.download(&h, 1);
   int batch = 2;
   while (!h.done) {
      for (int k = 0; k < batch; ++k) {
         bi_rho<<<g, kRedBlock, 0, stream()>>>(n, rr.p, r.p, S.p, partials.p, counter.p, max_it);
         bi_direction<<<ge, 256, 0, stream()>>>(n, r.p, v.p, p.p, S.p);
         count_launch(2);
         apply(p.p, pp.p);
         spmv_sell(A, pp.p, v.p, done);
         bi_alpha<<<g, kRedBlock, 0, stream()>>>(n, rr.p, v.p, S.p, partials.p, counter.p);
         bi_s<<<g, kRedBlock, 0, stream()>>>(n, r.p, v.p, s.p, S.p, partials.p, counter.p, tol);
         bi_x_at_s<<<ge, 256, 0, stream()>>>(n, x, pp.p, S.p);
         bi_clear_stop<<<1, 1, 0, stream()>>>(S.p);
         count_launch(4);
         apply(s.p, ss.p);
         spmv_sell(A, ss.p, t.p, done);
         bi_omega<<<g, kRedBlock, 0, stream()>>>(n, t.p, s.p, S.p, partials.p, counter.p);
         bi_update<<<g, kRedBlock, 0, stream()>>>(n, x, pp.p, ss.p, s.p, t.p, r.p, S.p, partials.p,
                                                  counter.p, tol);
         count_launch(2);
      }
      OFG_LAUNCH_CHECK();
      S.download(&h, 1);
      if (sweep) check_status(P);
      batch = std::min(batch * 2, 32);
   }
   *result = h.result;
   if (res) *res = h.res;
}

}  // namespace ofg

using namespace ofg;

extern "C" int ofg_bicgstab(ofg_prec* P, const double* b, double* x, int max_it, double toler,
                            int* result, double* res)
{
   return guarded("ofg_bicgstab", [&] {
      OFG_REQUIRE(P && b && x && result, OFG_ERR_ARG, "null argument");
      const int64_t n = P->A->n;
      if (n == 0) {
         *result = 0;
         if (res) *res = 0.0;
         return;
      }
      In<double> db(b, n);
      InOut<double> dx(x, n, true);
      bicgstab_solve(P, db.d, dx.d, max_it, toler, result, res);
      dx.finish();
   });
}
