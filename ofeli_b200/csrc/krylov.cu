// krylov.cu -- OFELI's CG and GMRes (include/solvers/CG.h:99-157,
// include/solvers/GMRes.h:67-241) on the device.
//
// All scalars of the recurrences (rho, alpha, beta, the Hessenberg column,
// the Givens rotations, the residual and the stopping test) live in device
// memory and are produced by the last block of the kernel that reduces them,
// so an iteration never waits for the host.  The host enqueues batches of
// iterations and reads back one small state struct per batch; kernels
// launched after convergence see the `done` flag and return at once.
//
// CG per iteration (DIAG / IDENT, the Jacobi application is folded into the
// vector kernels):
//   direction:  p = D r + beta p                      32 n bytes
//   spmv:       q = A p, (p, q) -> alpha               12 nnz + 20 n (SELL-32)
//   update:     x += alpha p, r -= alpha q, ||r||, (r, D r)   56 n
// D-ILU / SSOR: the backward sweep also returns (r, z), the direction kernel
// reads z.
#include <algorithm>
#include <cmath>

#include "internal.cuh"
#include "reduce.cuh"

namespace ofg {
namespace {

struct CGState {
   double nrm, rho, rho_old, alpha, res;
   int it, done, result, pad;
};

enum { PT_IDENT = 0, PT_DIAG = 1, PT_SWEEP = 2 };

template <int PT>
__device__ __forceinline__ double zval(int64_t i, const double* r, const double* piv, const double* z)
{
   if (PT == PT_DIAG) return r[i] * piv[i];
   if (PT == PT_IDENT) return r[i];
   return z[i];
}

template <int PT>
__global__ void __launch_bounds__(kRedBlock, 8) cg_init(int64_t n, const double* __restrict__ b,
                                                     const double* __restrict__ q, double* r,
                                                     const double* __restrict__ piv, CGState* S,
                                                     double* partials, unsigned* counter, double tol)
{
   double v[3] = {0.0, 0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double bi = b[i], ri = bi - q[i];
      r[i] = ri;
      v[0] += bi * bi;
      v[1] += ri * ri;
      if (PT == PT_DIAG) v[2] += ri * (ri * piv[i]);
      if (PT == PT_IDENT) v[2] += ri * ri;
   }
   double t[3];
   if (grid_reduce<3>(v, partials, counter, t)) {
      double nrm = sqrt(t[0]);
      if (nrm == 0.0) nrm = 1.0;
      S->nrm = nrm;
      S->res = sqrt(t[1]) / nrm;
      S->it = 0;
      S->rho = t[2];
      S->rho_old = 1.0;
      S->done = S->res <= tol ? 1 : 0;
      S->result = 0;
   }
}

template <int PT>
__global__ void __launch_bounds__(kRedBlock, 8) cg_direction(int64_t n, const double* __restrict__ r,
                                                          const double* __restrict__ piv,
                                                          const double* __restrict__ z, double* p,
                                                          const CGState* S)
{
   pdl_wait();
   pdl_release();
   if (S->done) return;
   const bool first = S->it == 0;
   const double beta = first ? 0.0 : S->rho / S->rho_old;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double zi = zval<PT>(i, r, piv, z);
      p[i] = first ? zi : zi + beta * p[i];
   }
}

__global__ void __launch_bounds__(kRedBlock, 8) cg_spmv(int64_t n, int64_t nslices,
                                                     const int32_t* __restrict__ sp,
                                                     const int32_t* __restrict__ scol,
                                                     const double* __restrict__ sval,
                                                     const double* __restrict__ p,
                                                     double* __restrict__ q, CGState* S,
                                                     double* partials, unsigned* counter,
                                                     int* worked)
{
   pdl_wait();
   pdl_release();
   if (S->done) return;
   prof_mark(worked);
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < nslices * 32;
        row += stride) {
      const int64_t s = row >> 5;
      const int lane = (int)(row & 31);
      const int32_t beg = sp[s], end = sp[s + 1];
      double acc = 0.0;
      for (int32_t k = beg + lane; k < end; k += 32) acc += sval[k] * __ldg(p + scol[k]);
      if (row < n) {
         q[row] = acc;
         v[0] += p[row] * acc;
      }
   }
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t)) S->alpha = S->rho / t[0];
}

template <int PT>
__global__ void __launch_bounds__(kRedBlock, 8) cg_update(int64_t n, double* x,
                                                       const double* __restrict__ p, double* r,
                                                       const double* __restrict__ q,
                                                       const double* __restrict__ piv, CGState* S,
                                                       double* partials, unsigned* counter,
                                                       double tol, int max_it, double* hist)
{
   pdl_wait();
   pdl_release();
   if (S->done) return;
   const double a = S->alpha;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      x[i] += a * p[i];
      const double ri = r[i] - a * q[i];
      r[i] = ri;
      v[0] += ri * ri;
      if (PT == PT_DIAG) v[1] += ri * (ri * piv[i]);
      if (PT == PT_IDENT) v[1] += ri * ri;
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      const double res = sqrt(t[0]) / S->nrm;
      const int it = S->it + 1;
      S->it = it;
      S->res = res;
      if (hist) hist[it] = res;
      if (res <= tol) {
         S->done = 1;
         S->result = it;
      }
      else if (it >= max_it) {
         S->done = 1;
         S->result = -(max_it + 1);
      }
      S->rho_old = S->rho;
      if (PT != PT_SWEEP) S->rho = t[1];
   }
}

// ---------------------------------------------------------------- GMRES --
struct GMState {
   double normb, beta, res;
   int it, done, stop, conv_i, result, pad;
};

__global__ void __launch_bounds__(kRedBlock, 8) gm_residual(int64_t n, const double* __restrict__ b,
                                                         const double* __restrict__ q, double* r,
                                                         GMState* S, double* partials,
                                                         unsigned* counter, int first)
{
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double bi = b[i];
      r[i] = bi - q[i];
      v[0] += bi * bi;
   }
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t))
      if (first) S->normb = sqrt(t[0]);
}

// beta = ||r||; first call: the initial convergence test of GMRes.h:169-179,
// later calls: the restart test of :222-233.
__global__ void __launch_bounds__(kRedBlock, 8) gm_beta(int64_t n, const double* __restrict__ r,
                                                     GMState* S, double* partials,
                                                     unsigned* counter, double tol, int first,
                                                     int max_it)
{
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      v[0] += r[i] * r[i];
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t)) {
      const double beta = sqrt(t[0]);
      S->beta = beta;
      if (first) {
         if (S->normb == 0.0) S->normb = 1.0;
         S->it = 1;
         S->res = beta / S->normb;
         S->done = S->res <= tol ? 1 : 0;
         S->result = 1;
      }
      else {
         S->res = beta / S->normb;
         if (S->res < tol) {
            S->done = 1;
            S->result = S->it;
         }
         else if (S->it > max_it) {
            S->done = 1;
            S->result = -S->it;
         }
      }
      S->stop = S->done;
      S->conv_i = -1;
   }
}

// v0 = r / beta, s = (beta, 0, ...)
__global__ void gm_start(int64_t n, const double* __restrict__ r, double* v0, double* s, int m,
                         const GMState* S)
{
   if (S->stop) return;
   const double sc = 1.0 / S->beta;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      v0[i] = sc * r[i];
   if (blockIdx.x == 0)
      for (int j = threadIdx.x; j <= m; j += blockDim.x) s[j] = j == 0 ? S->beta : 0.0;
}

// Modified Gram-Schmidt step k of column i: w -= h_{k-1} v_{k-1} (k > 0),
// then h_k = (w, v_k).  The chain gm_mgs(0..i), gm_mgs_last, gm_scale
// finishes each dot product in the next kernel: a kernel leaves its
// per-block partials in `pout`; the next one sums them (pin) in every block,
// in the order of a last-block reduction, and its block 0 stores the
// Hessenberg entry.
__global__ void __launch_bounds__(kRedBlock, 8) gm_mgs(int64_t n, double* w,
                                                    const double* __restrict__ vprev,
                                                    double* hprev,
                                                    const double* __restrict__ vk,
                                                    const double* __restrict__ pin, double* pout,
                                                    const GMState* S)
{
   if (S->stop) return;
   double h = 0.0;
   if (hprev) {
      double tot[1];
      partials_total<1>(pin, gridDim.x, tot);
      h = tot[0];
      if (blockIdx.x == 0 && threadIdx.x == 0) *hprev = h;
   }
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      double wi = w[i];
      if (hprev) {
         wi -= h * vprev[i];
         w[i] = wi;
      }
      v[0] += wi * vk[i];
   }
   block_partials<1>(v, pout);
}

// last projection w -= h_i v_i (h_i = H(i,i) from the partials of
// gm_mgs(i)); ||w||^2 left as partials for gm_scale
__global__ void __launch_bounds__(kRedBlock, 8) gm_mgs_last(int64_t n, double* w,
                                                         const double* __restrict__ vi, double* hi,
                                                         const double* __restrict__ pin,
                                                         double* pout, const GMState* S)
{
   if (S->stop) return;
   double tot[1];
   partials_total<1>(pin, gridDim.x, tot);
   const double h = tot[0];
   if (blockIdx.x == 0 && threadIdx.x == 0) *hi = h;
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double wi = w[i] - h * vi[i];
      w[i] = wi;
      v[0] += wi * wi;
   }
   block_partials<1>(v, pout);
}

// H(i+1,i) = ||w|| from the partials of gm_mgs_last; v_{i+1} = w / H(i+1,i)
__global__ void __launch_bounds__(kRedBlock, 8) gm_scale(int64_t n, const double* __restrict__ w,
                                                      double* vnext, double* h,
                                                      const double* __restrict__ pin,
                                                      const GMState* S)
{
   if (S->stop) return;
   double tot[1];
   partials_total<1>(pin, gridDim.x, tot);
   const double hn = sqrt(tot[0]);
   if (blockIdx.x == 0 && threadIdx.x == 0) *h = hn;
   const double sc = 1.0 / hn;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      vnext[i] = sc * w[i];
}

__device__ __forceinline__ void rotate(double& dx, double& dy, double cs, double sn)
{
   const double temp = cs * dx + sn * dy;
   dy = cs * dy - sn * dx;
   dx = temp;
}

// set_rotation (GMRes.h:98-115)
__device__ __forceinline__ void set_rotation(double dx, double dy, double& cs, double& sn)
{
   if (dy == 0.0) {
      cs = 1.0;
      sn = 0.0;
   }
   else if (fabs(dy) > fabs(dx)) {
      const double temp = dx / dy;
      sn = 1.0 / sqrt(1.0 + temp * temp);
      cs = temp * sn;
   }
   else {
      const double temp = dy / dx;
      cs = 1.0 / sqrt(1.0 + temp * temp);
      sn = temp * cs;
   }
}

// Givens rotations of Hessenberg column i and the convergence test
// (GMRes.h:200-217); advances the iteration counter like the inner for loop.
__global__ void gm_givens(double* H, double* s, double* cs, double* sn, int i, int m, GMState* S,
                          double tol, int max_it)
{
   if (S->stop || threadIdx.x != 0) return;
   const int ld = m + 1;
   for (int k = 0; k < i; ++k) rotate(H[k * ld + i], H[(k + 1) * ld + i], cs[k], sn[k]);
   set_rotation(H[i * ld + i], H[(i + 1) * ld + i], cs[i], sn[i]);
   rotate(H[i * ld + i], H[(i + 1) * ld + i], cs[i], sn[i]);
   rotate(s[i], s[i + 1], cs[i], sn[i]);
   const double res = fabs(s[i + 1]) / S->normb;
   S->res = res;
   if (res < tol) {
      S->conv_i = i;
      S->stop = 1;
      S->done = 1;
      S->result = S->it;
      return;
   }
   S->it += 1;
   if (S->it > max_it) S->stop = 1;
}

// update(x, k, H, s, v) (GMRes.h:78-94): back substitution for y
__global__ void gm_backsolve(const double* H, const double* s, double* y, int k, int m)
{
   if (threadIdx.x != 0 || blockIdx.x != 0) return;
   const int ld = m + 1;
   for (int j = 0; j <= m; ++j) y[j] = s[j];
   for (int i = k; i >= 0; --i) {
      y[i] /= H[i * ld + i];
      for (int j = i - 1; j >= 0; --j) y[j] -= H[j * ld + i] * y[i];
   }
}

__global__ void gm_update_x(int64_t n, double* x, const double* __restrict__ V,
                            const double* __restrict__ y, int k)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += stride) {
      double xl = x[l];
      for (int j = 0; j <= k; ++j) xl += V[(int64_t)j * n + l] * y[j];
      x[l] = xl;
   }
}

__global__ void __launch_bounds__(kRedBlock, 8) res_kernel(int64_t n, const double* __restrict__ b,
                                                        const double* __restrict__ q,
                                                        double* out, double* partials,
                                                        unsigned* counter)
{
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double bi = b[i], ri = bi - q[i];
      v[0] += ri * ri;
      v[1] += bi * bi;
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      double nb = sqrt(t[1]);
      *out = sqrt(t[0]) / (nb == 0.0 ? 1.0 : nb);
   }
}

unsigned red_grid(int64_t n) { return grid_for(n, kRedBlock, 8); }

// Scratch of one Krylov call: reduction partials, counter, state.
struct RedScratch {
   DBuf<double> partials;
   DBuf<unsigned> counter;
   explicit RedScratch(int64_t n)
   {
      partials.alloc(((size_t)red_grid(n) + 1) * 4 + 4);
      counter.alloc(1);
      counter.zero();
   }
};

template <int PT>
void cg_iteration(ofg_prec* P, int64_t n, double* x, double* r, double* p, double* q, double* z,
                  CGState* S, RedScratch& rs, double tol, int max_it, double* hist)
{
   ofg_matrix* A = P->A;
   const unsigned g = red_grid(n);
   if (PT == PT_SWEEP) prec_apply_device(P, r, z, &S->rho, &S->done);
   // programmatic dependent launch: each kernel's blocks start while the
   // previous kernel drains its reduction tail
   launch_pdl(cg_direction<PT>, g, kRedBlock, n, r, P->pivot.p, z, p, S);
   int* worked = prof_begin();
   launch_pdl(cg_spmv, grid_for(A->nslices * 32, kRedBlock, 8), kRedBlock, n, A->nslices,
              A->sell_ptr.p, A->sell_col.p, A->sell_val.p, p, q, S, rs.partials.p, rs.counter.p,
              worked);
   prof_end(PROF_SPMV64, 12.0 * A->nnz + 20.0 * A->n + 4.0);
   launch_pdl(cg_update<PT>, g, kRedBlock, n, x, p, r, q, P->pivot.p, S, rs.partials.p,
              rs.counter.p, tol, max_it, hist);
   OFG_LAUNCH_CHECK();
}

template <int PT>
void cg_run(ofg_prec* P, const double* b, double* x, int max_it, double tol, int* result,
            double* res, double* hist)
{
   ofg_matrix* A = P->A;
   const int64_t n = A->n;
   DBuf<double> r(n), p(n), q(n), z(PT == PT_SWEEP ? n : 1);
   DBuf<CGState> S(1);
   RedScratch rs(n);
   if (PT == PT_SWEEP) fill_sentinel(z.p, n);
   spmv_sell(A, x, q.p);
   cg_init<PT><<<red_grid(n), kRedBlock, 0, stream()>>>(n, b, q.p, r.p, P->pivot.p, S.p,
                                                        rs.partials.p, rs.counter.p, tol);
   count_launch();
   OFG_LAUNCH_CHECK();
   CGState h{};
   S.download(&h, 1);
   int batch = 4;
   while (!h.done) {
      if (max_it <= 0) {
         h.result = -(max_it + 1);
         break;
      }
      for (int k = 0; k < batch; ++k)
         cg_iteration<PT>(P, n, x, r.p, p.p, q.p, z.p, S.p, rs, tol, max_it, hist);
      S.download(&h, 1);
      if (PT == PT_SWEEP) check_status(P);
      batch = std::min(batch * 2, 64);
   }
   *result = h.result;
   if (res) *res = h.res;
}

}  // namespace

void cg_solve(ofg_prec* P, const double* b, double* x, int max_it, double tol, int* result,
              double* res, double* hist)
{
   ensure_sell(P->A);
   if (prec_stale(P)) prec_setup(P);
   switch (P->type) {
      case OFG_IDENT: cg_run<PT_IDENT>(P, b, x, max_it, tol, result, res, hist); break;
      case OFG_DIAG: cg_run<PT_DIAG>(P, b, x, max_it, tol, result, res, hist); break;
      default: cg_run<PT_SWEEP>(P, b, x, max_it, tol, result, res, hist); break;
   }
}

void gmres_solve(ofg_prec* P, const double* b, double* x, int m, int max_it, double tol,
                 int* result, double* res)
{
   ofg_matrix* A = P->A;
   ensure_sell(A);
   if (prec_stale(P)) prec_setup(P);
   const int64_t n = A->n;
   OFG_REQUIRE(m >= 1, OFG_ERR_ARG, "restart length must be >= 1");
   DBuf<double> r(n), w(n), q(n), V((size_t)(m + 1) * n);
   DBuf<double> H((size_t)(m + 1) * (m + 1)), s(m + 1), cs(m + 1), sn(m + 1), y(m + 1);
   H.zero();
   s.zero();
   cs.zero();
   sn.zero();
   DBuf<GMState> S(1);
   RedScratch rs(n);
   const unsigned g = red_grid(n);
   // the two partial buffers the Gram-Schmidt chain alternates between
   DBuf<double> gp(2 * (size_t)g);
   double* const gpb[2] = {gp.p, gp.p + g};
   const int ld = m + 1;
   auto precond_inplace = [&](double* v, const int* skip) {
      if (P->type == OFG_IDENT) return;
      prec_apply_device(P, v, v, nullptr, skip);
   };
   // r = P^{-1}(b - A x), beta, initial test
   spmv_sell(A, x, q.p);
   gm_residual<<<g, kRedBlock, 0, stream()>>>(n, b, q.p, r.p, S.p, rs.partials.p, rs.counter.p, 1);
   count_launch();
   precond_inplace(r.p, nullptr);
   gm_beta<<<g, kRedBlock, 0, stream()>>>(n, r.p, S.p, rs.partials.p, rs.counter.p, tol, 1, max_it);
   count_launch();
   OFG_LAUNCH_CHECK();
   GMState h{};
   S.download(&h, 1);
   if (P->type != OFG_IDENT && P->type != OFG_DIAG) check_status(P);
   while (!h.done) {
      gm_start<<<g, kRedBlock, 0, stream()>>>(n, r.p, V.p, s.p, m, S.p);
      count_launch();
      // the cycle's iterations go out in batches of 4, 8, 16, ... with one
      // read of the state after each: once gm_givens has stopped the cycle,
      // the kernels of its remaining iterations (which would all return at
      // once) are not launched
      int i = 0;
      for (int batch = 4; i < m; batch *= 2) {
         const int end = std::min(m, i + batch);
         for (; i < end; ++i) {
            double* vi = V.p + (size_t)i * n;
            spmv_sell(A, vi, w.p, &S.p->stop);
            precond_inplace(w.p, &S.p->stop);
            // gm_mgs(k) writes gpb[k & 1]; H(k-1,i) is stored by gm_mgs(k),
            // H(i,i) by gm_mgs_last, H(i+1,i) by gm_scale
            for (int k = 0; k <= i; ++k) {
               gm_mgs<<<g, kRedBlock, 0, stream()>>>(
                  n, w.p, k > 0 ? V.p + (size_t)(k - 1) * n : nullptr,
                  k > 0 ? H.p + (size_t)(k - 1) * ld + i : nullptr, V.p + (size_t)k * n,
                  gpb[(k + 1) & 1], gpb[k & 1], S.p);
            }
            gm_mgs_last<<<g, kRedBlock, 0, stream()>>>(n, w.p, vi, H.p + (size_t)i * ld + i,
                                                       gpb[i & 1], gpb[(i + 1) & 1], S.p);
            gm_scale<<<g, kRedBlock, 0, stream()>>>(n, w.p, V.p + (size_t)(i + 1) * n,
                                                    H.p + (size_t)(i + 1) * ld + i,
                                                    gpb[(i + 1) & 1], S.p);
            gm_givens<<<1, 32, 0, stream()>>>(H.p, s.p, cs.p, sn.p, i, m, S.p, tol, max_it);
            count_launch(i + 5);
            OFG_LAUNCH_CHECK();
         }
         if (i < m) {
            S.download(&h, 1);
            if (h.stop) break;
         }
      }
      S.download(&h, 1);
      if (P->type != OFG_IDENT && P->type != OFG_DIAG) check_status(P);
      const int k = h.done ? h.conv_i : m - 1;
      gm_backsolve<<<1, 32, 0, stream()>>>(H.p, s.p, y.p, k, m);
      gm_update_x<<<g, kRedBlock, 0, stream()>>>(n, x, V.p, y.p, k);
      count_launch(2);
      OFG_LAUNCH_CHECK();
      if (h.done) break;
      // restart: r = P^{-1}(b - A x), beta, tests
      spmv_sell(A, x, q.p);
      gm_residual<<<g, kRedBlock, 0, stream()>>>(n, b, q.p, r.p, S.p, rs.partials.p, rs.counter.p, 0);
      count_launch();
      precond_inplace(r.p, nullptr);
      gm_beta<<<g, kRedBlock, 0, stream()>>>(n, r.p, S.p, rs.partials.p, rs.counter.p, tol, 0,
                                             max_it);
      count_launch();
      OFG_LAUNCH_CHECK();
      S.download(&h, 1);
      if (P->type != OFG_IDENT && P->type != OFG_DIAG) check_status(P);
   }
   *result = h.result;
   if (res) *res = h.res;
}

double residual_device(const ofg_matrix* A, const double* b, const double* x)
{
   const int64_t n = A->n;
   ensure_sell(const_cast<ofg_matrix*>(A));
   DBuf<double> q(n), out(1);
   RedScratch rs(n);
   spmv_sell(A, x, q.p);
   res_kernel<<<red_grid(n), kRedBlock, 0, stream()>>>(n, b, q.p, out.p, rs.partials.p, rs.counter.p);
   count_launch();
   OFG_LAUNCH_CHECK();
   double h = 0;
   out.download(&h, 1);
   return h;
}

}  // namespace ofg

using namespace ofg;

extern "C" {

int ofg_cg(ofg_prec* P, const double* b, double* x, int max_it, double toler, int* result,
           double* res)
{
   return guarded("ofg_cg", [&] {
      OFG_REQUIRE(P && b && x && result, OFG_ERR_ARG, "null argument");
      const int64_t n = P->A->n;
      In<double> db(b, n);
      InOut<double> dx(x, n, true);
      cg_solve(P, db.d, dx.d, max_it, toler, result, res, nullptr);
      dx.finish();
   });
}

int ofg_cg_history(ofg_prec* P, const double* b, double* x, int max_it, double toler, int* result,
                   double* res, double* hist)
{
   return guarded("ofg_cg_history", [&] {
      OFG_REQUIRE(P && b && x && result && hist, OFG_ERR_ARG, "null argument");
      const int64_t n = P->A->n;
      In<double> db(b, n);
      InOut<double> dx(x, n, true);
      InOut<double> dh(hist, (size_t)max_it + 1, true);
      cg_solve(P, db.d, dx.d, max_it, toler, result, res, dh.d);
      dx.finish();
      dh.finish();
   });
}

int ofg_gmres(ofg_prec* P, const double* b, double* x, int m, int max_it, double toler, int* result,
              double* res)
{
   return guarded("ofg_gmres", [&] {
      OFG_REQUIRE(P && b && x && result, OFG_ERR_ARG, "null argument");
      const int64_t n = P->A->n;
      In<double> db(b, n);
      InOut<double> dx(x, n, true);
      gmres_solve(P, db.d, dx.d, m, max_it, toler, result, res);
      dx.finish();
   });
}

int ofg_residual(const ofg_matrix* A, const double* b, const double* x, double* rel)
{
   return guarded("ofg_residual", [&] {
      OFG_REQUIRE(A && b && x && rel, OFG_ERR_ARG, "null argument");
      In<double> db(b, A->n), dx(x, A->n);
      *rel = residual_device(A, db.d, dx.d);
   });
}

}  // extern "C"
