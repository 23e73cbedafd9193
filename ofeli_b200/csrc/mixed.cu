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
// accumulation of every Krylov dot product.  One Jacobi-preconditioned
// FP32 CG iteration streams (v + c)*nnz + 52*n bytes -- v = 4 (FP32) or 2
// (BF16) value bytes, c = 4 (int32 column), 2 (16-bit offset) or nearly 0
// (slices with uniform offsets) -- against 12*nnz + 108*n for a fused FP64
// iteration.
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
#include "sellq.cuh"

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

// BF16 copy of the values; *inexact = 1 when some value does not come back
// unchanged from BF16 (a NaN never does)
__global__ void cast_bf16_exact(int64_t total, const double* __restrict__ src, __nv_bfloat16* dst,
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
                                                              float* rr, float* p, float* d,
                                                              int fresh, MixState* S,
                                                              double* partials, unsigned* counter)
{
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

// When the host must refine (mode 0) or stop the inner solve (mode 1).
struct StopRule {
   double delta, tol, scale;
   int max_inner, mode;
};

// Decision after iteration `it` from ||r||^2: every block of the deciding
// kernel takes it from the same totals; block 0 records ||r||, the count
// and the pause for the host and the later kernels.
__device__ __forceinline__ bool decide_pause(MixState* S, double rr2, int it, const StopRule& st)
{
   const double rn = sqrt(rr2);
   bool stop;
   if (st.mode == 0)
      // refine when the residual fell by delta, or when the recurrence says
      // the FP64 target is reached
      stop = rn <= st.delta * S->rmark || rn * st.scale <= st.tol * S->bnorm || it >= st.max_inner;
   else
      stop = rn <= st.delta * S->res0 || it >= st.max_inner;
   if (blockIdx.x == 0 && threadIdx.x == 0) {
      S->rn = rn;
      S->it = it;
      if (stop) S->pause = 1;
   }
   return stop;
}

// q = A p over four rows per thread; (p, q) left as per-block partials for
// mx_update.  UNI: slices with uniform offsets (suni[s] >= 0) read one
// offset per position from stab and gather p with vector loads.
template <class T, class I, bool UNI = false>
__global__ void __launch_bounds__(kRedBlock, kQuadBlocks) mx_spmv(int64_t nquads, const int32_t* __restrict__ sp,
                                                     const I* __restrict__ scol,
                                                     const T* __restrict__ sval,
                                                     const float* __restrict__ p,
                                                     float* __restrict__ q, const MixState* S,
                                                     double* pq, int* worked,
                                                     const int32_t* __restrict__ suni = nullptr,
                                                     const int16_t* __restrict__ stab = nullptr)
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
      const T* vp = sval + beg + lane0;
      const int32_t u = UNI ? suni[s] : -1;
      if (u >= 0) {
         acc = uniform_quad(vp, stab + u, w, p, (int)r0);
      }
      else {
         const I* cp = scol + beg + lane0;
         auto step = [&](int32_t k) {
            const int4 c = load_cols(cp + k * 32, r0);
            const float4 a = load_vals(vp + k * 32);
            acc.x += a.x * __ldg(p + c.x);
            acc.y += a.y * __ldg(p + c.y);
            acc.z += a.z * __ldg(p + c.z);
            acc.w += a.w * __ldg(p + c.w);
         };
         // with uniform slices this path is the rare one: kept rolled so
         // that it does not set the kernel's register count
         if (UNI) {
#pragma unroll 1
            for (int32_t k = 0; k < w; ++k) step(k);
         }
         else {
#pragma unroll 8
            for (int32_t k = 0; k < w; ++k) step(k);
         }
      }
      *reinterpret_cast<float4*>(q + r0) = acc;
      const float4 pr = *reinterpret_cast<const float4*>(p + r0);
      v[0] += (double)pr.x * acc.x + (double)pr.y * acc.y + (double)pr.z * acc.z +
              (double)pr.w * acc.w;
   }
   block_partials<1>(v, pq);
}

// alpha = rho_it / (p, q) from the SpMV's partials (it = iterations done);
// r -= alpha q; ||r|| and, when JAC, (r, D r) left as partials for the
// kernel that decides (lg_lower or mx_direction).  The matching
// d += alpha p is made by the direction kernel, which reads p anyway (or by
// mx_flush_d when this iteration pauses the loop).
template <bool JAC>
__global__ void __launch_bounds__(kRedBlock, 8) mx_update(int64_t nquads, float* rr,
                                                       const float* __restrict__ q,
                                                       const float* __restrict__ dinv, MixState* S,
                                                       const double* __restrict__ pq,
                                                       double* rpart, int it)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   double pqt[1];
   partials_total<1>(pq, gridDim.x, pqt);
   const double alpha = S->rho[it & 1] / pqt[0];
   if (blockIdx.x == 0 && threadIdx.x == 0) S->alpha = alpha;
   const float a = (float)alpha;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   float4* r4 = reinterpret_cast<float4*>(rr);
   const float4* q4 = reinterpret_cast<const float4*>(q);
   const float4* m4 = reinterpret_cast<const float4*>(dinv);
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const float4 qi = q4[i];
      float4 ri = r4[i];
      ri.x -= a * qi.x; ri.y -= a * qi.y; ri.z -= a * qi.z; ri.w -= a * qi.w;
      r4[i] = ri;
      v[0] += (double)ri.x * ri.x + (double)ri.y * ri.y + (double)ri.z * ri.z + (double)ri.w * ri.w;
      if (JAC) {
         const float4 mi = m4[i];
         v[1] += (double)ri.x * (ri.x * mi.x) + (double)ri.y * (ri.y * mi.y) +
                 (double)ri.z * (ri.z * mi.z) + (double)ri.w * (ri.w * mi.w);
      }
   }
   block_partials<2>(v, rpart);
}

// d += alpha p with this iteration's alpha and p (upd_d), then the new
// direction
__device__ __forceinline__ void add_alpha_p(float4* d4, int64_t i, float a, const float4& pi)
{
   float4 di = d4[i];
   di.x += a * pi.x; di.y += a * pi.y; di.z += a * pi.z; di.w += a * pi.w;
   d4[i] = di;
}

// After iteration `it` (decide): the stop decision and rho_it = (r, D r)
// from mx_update's partials; then (d += alpha p;) p = D r + beta p,
// beta = rho_it / rho_{it-1}.  Right after a refinement (no decide) rho_it
// is the one mx_load_residual stored.
__global__ void __launch_bounds__(kRedBlock, 8) mx_direction(int64_t nquads,
                                                          const float* __restrict__ rr,
                                                          const float* __restrict__ dinv, float* p,
                                                          float* d, int upd_d, MixState* S,
                                                          const double* __restrict__ rpart, int it,
                                                          int decide, StopRule st)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   double rho;
   if (decide) {
      double tot[2];
      partials_total<2>(rpart, gridDim.x, tot);
      rho = tot[1];
      if (blockIdx.x == 0 && threadIdx.x == 0) S->rho[it & 1] = rho;
      if (decide_pause(S, tot[0], it, st)) return;
   }
   else {
      rho = S->rho[it & 1];
   }
   const float beta = (float)(rho / S->rho[(it + 1) & 1]);
   const float a = (float)S->alpha;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   float4* p4 = reinterpret_cast<float4*>(p);
   float4* d4 = reinterpret_cast<float4*>(d);
   const float4* r4 = reinterpret_cast<const float4*>(rr);
   const float4* m4 = reinterpret_cast<const float4*>(dinv);
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const float4 ri = r4[i], mi = m4[i];
      float4 pi = p4[i];
      if (upd_d) add_alpha_p(d4, i, a, pi);
      pi.x = ri.x * mi.x + beta * pi.x;
      pi.y = ri.y * mi.y + beta * pi.y;
      pi.z = ri.z * mi.z + beta * pi.z;
      pi.w = ri.w * mi.w + beta * pi.w;
      p4[i] = pi;
   }
}

// After iteration `it` (decide): the stop decision from mx_update's
// partials; then t = G r
template <class V, class I, bool UNI = false>
__global__ void __launch_bounds__(kRedBlock, kQuadBlocks) lg_lower(int64_t nquads, const int32_t* __restrict__ sp,
                                                      const I* __restrict__ scol,
                                                      const V* __restrict__ sval,
                                                      const float* __restrict__ r, float* t,
                                                      MixState* S, const double* __restrict__ rpart,
                                                      int it, int decide, StopRule st, int* worked,
                                                      const int32_t* __restrict__ suni = nullptr,
                                                      const int16_t* __restrict__ stab = nullptr)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   if (decide) {
      double tot[2];
      partials_total<2>(rpart, gridDim.x, tot);
      if (decide_pause(S, tot[0], it, st)) return;
   }
   prof_mark(worked);
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride)
      *reinterpret_cast<float4*>(t + i * 4) =
         sell_quad<V, I, UNI>(sp, scol, sval, r, i * 4, suni, stab);
}

// z = G^T t; (r, z) left as partials for lg_direction
template <class V, class I, bool UNI = false>
__global__ void __launch_bounds__(kRedBlock, kQuadBlocks) lg_upper(int64_t nquads, const int32_t* __restrict__ sp,
                                                      const I* __restrict__ scol,
                                                      const V* __restrict__ sval,
                                                      const float* __restrict__ t, float* z,
                                                      const float* __restrict__ r, const MixState* S,
                                                      double* cpart, int* worked,
                                                      const int32_t* __restrict__ suni = nullptr,
                                                      const int16_t* __restrict__ stab = nullptr)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   prof_mark(worked);
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const float4 zi = sell_quad<V, I, UNI>(sp, scol, sval, t, i * 4, suni, stab);
      *reinterpret_cast<float4*>(z + i * 4) = zi;
      const float4 ri = *reinterpret_cast<const float4*>(r + i * 4);
      v[0] += (double)ri.x * zi.x + (double)ri.y * zi.y + (double)ri.z * zi.z + (double)ri.w * zi.w;
   }
   block_partials<1>(v, cpart);
}

// rho_it = (r, z) from lg_upper's partials and beta = rho_it / rho_{it-1};
// then (d += alpha p;) p = z + beta p (p = z on a fresh start).  M = G^T G
// is one fixed linear operator within a solve, so the PCG beta applies (the
// flexible Polak-Ribiere form, -alpha (z, q) / rho_{it-1}, took 4566 instead
// of 3994 iterations at 2049^2 in FP32); right after a refinement replaced
// r the same beta keeps the direction.
__global__ void __launch_bounds__(kRedBlock, 8) lg_direction(int64_t nquads,
                                                          const float* __restrict__ z, float* p,
                                                          float* d, int upd_d, MixState* S,
                                                          const double* __restrict__ cpart, int it,
                                                          int fresh)
{
   pdl_wait();
   pdl_release();
   if (S->pause) return;
   double tot[1];
   partials_total<1>(cpart, gridDim.x, tot);
   const double old = S->rho[(it + 1) & 1];
   const double bd = tot[0] / old;
   if (blockIdx.x == 0 && threadIdx.x == 0) {
      S->rho[it & 1] = tot[0];
      S->beta = bd;
   }
   const float beta = fresh ? 0.f : (float)bd;
   const float a = (float)S->alpha;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   float4* p4 = reinterpret_cast<float4*>(p);
   float4* d4 = reinterpret_cast<float4*>(d);
   const float4* z4 = reinterpret_cast<const float4*>(z);
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
      const float4 zi = z4[i];
      if (fresh) {
         p4[i] = zi;
         continue;
      }
      float4 pi = p4[i];
      if (upd_d) add_alpha_p(d4, i, a, pi);
      pi.x = zi.x + beta * pi.x;
      pi.y = zi.y + beta * pi.y;
      pi.z = zi.z + beta * pi.z;
      pi.w = zi.w + beta * pi.w;
      p4[i] = pi;
   }
}

// d += alpha p for the iteration that paused the loop (its direction kernel
// returned early)
__global__ void mx_flush_d(int64_t nquads, float* d, const float* __restrict__ p,
                           const MixState* S)
{
   const float a = (float)S->alpha;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   float4* d4 = reinterpret_cast<float4*>(d);
   const float4* p4 = reinterpret_cast<const float4*>(p);
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride)
      add_alpha_p(d4, i, a, p4[i]);
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

// The uniform-slice kernels keep their per-entry path rolled (registers), so
// they pay off only when nearly every entry sits in a uniform slice: with
// 95 % (2-D square in natural order) a step took 16 % less time, with 72 %
// (3-D Kuhn cube, whose grid lines of 127 rows cut many slices) 13 % more.
bool mostly_uniform(const ofg_matrix* M)
{
   return M->utab_len > 0 && M->uni_nnz >= 0.9 * (double)M->nnz;
}

}  // namespace

void solve_mixed(ofg_matrix* A, int prec_type, int inner_bits, int mode, const double* b, double* x,
                 int max_outer, int max_inner, double inner_tol, double tol, int* outer, int* inner,
                 double* true_res, ofg_prec* LP, int* fell_back)
{
   const bool learned = LP != nullptr;
   OFG_REQUIRE(learned || prec_type == OFG_DIAG || prec_type == OFG_IDENT, OFG_ERR_ARG,
               "mixed-precision inner solver supports DIAG and IDENT");
   OFG_REQUIRE(inner_bits == 32 || inner_bits == 16 || inner_bits == 0, OFG_ERR_ARG,
               "inner_bits must be 32, 16 or 0 (automatic)");
   OFG_REQUIRE(mode == 0 || mode == 1, OFG_ERR_ARG, "mode must be 0 or 1");
   OFG_REQUIRE(inner_tol > 0 && inner_tol < 1, OFG_ERR_ARG, "inner_tol must be in (0, 1)");
   const int64_t n = A->n;
   // FP32 values asked for: both SELL copies of new values in one pass
   if (inner_bits == 32) ensure_sell32(A);
   else ensure_sell(A);
   ensure_dpos(A);
   OFG_REQUIRE(A->dpos_complete, OFG_ERR_PIVOT, "a row has no diagonal entry");
   bool g16 = false;
   if (learned) {
      if (prec_stale(LP)) prec_setup(LP);
      ensure_sell_bf16(LP->gl);
      ensure_sell_bf16(LP->gu);
      g16 = ensure_sell_d16(LP->gl) && ensure_sell_d16(LP->gu);
      OFG_REQUIRE(LP->gl->nslices == A->nslices && LP->gu->nslices == A->nslices, OFG_ERR_ARG,
                  "learned factor does not match the matrix");
      if (g16) {
         ensure_sell_uniform(LP->gl);
         ensure_sell_uniform(LP->gu);
      }
   }
   const bool luni = g16 && mostly_uniform(LP->gl), uuni = g16 && mostly_uniform(LP->gu);
   const int64_t npad = A->nslices * 32, nquads = npad / 4;
   // 16-bit column offsets when every |column - row| fits (banded orderings,
   // structured meshes): 2 bytes less per entry streamed by every SpMV
   const bool a16 = ensure_sell_d16(A);
   // slices whose rows share their offsets read one offset per position and
   // gather p with vector loads
   if (a16) ensure_sell_uniform(A);
   const bool auni = a16 && mostly_uniform(A);
   // index bytes streamed per product: 2 per entry outside the uniform
   // slices, the uniform slices' table
   auto index_bytes = [](const ofg_matrix* M, bool d16, bool uni) {
      if (!d16) return 4.0 * M->nnz;
      if (!uni) return 2.0 * M->nnz;
      return 2.0 * (M->nnz - M->uni_nnz) + 2.0 * M->utab_len;
   };
   // bad[0]: zero diagonal entry; bad[1]: a value of A is not exact in BF16
   DBuf<int> bad(2);
   bad.zero();
   DBuf<__nv_bfloat16> v16;
   if (inner_bits == 32) ensure_sell32(A);
   else if (inner_bits == 16) {
      v16.alloc(A->sell_val.n);
      cast_values<__nv_bfloat16><<<grid_for(A->sell_val.n, 256), 256, 0, stream()>>>(
         A->sell_val.n, A->sell_val.p, v16.p);
      count_launch();
   }
   else {
      // automatic: BF16 values only when the copy is lossless, so that the
      // inner iteration is the FP32 one with 2 bytes less per entry
      v16.alloc(A->sell_val.n);
      cast_bf16_exact<<<grid_for(A->sell_val.n, 256), 256, 0, stream()>>>(
         A->sell_val.n, A->sell_val.p, v16.p, bad.p + 1);
      count_launch();
   }
   const int64_t nv = npad > 0 ? npad : 4;
   // p, r and t are gathered: 8 elements of slack for quad_at
   DBuf<float> dinv(nv), rr(nv + 8), p(nv + 8), q(nv), d(nv);
   DBuf<float> tz(learned ? nv + 8 : 1), zz(learned ? nv : 1);
   DBuf<double> r(n > 0 ? n : 1), q64(n > 0 ? n : 1);
   DBuf<MixState> S(1);
   p.zero();
   q.zero();
   const unsigned g = grid_for(std::max<int64_t>(n, nquads), kRedBlock, 8);
   DBuf<double> partials(((size_t)g + 1) * 4 + 4);
   DBuf<unsigned> counter(1);
   counter.zero();
   inv_diag32<<<grid_for(nv, 256), 256, 0, stream()>>>(n, npad, A->dpos.p, A->val.p, dinv.p,
                                                        prec_type == OFG_IDENT ? 1 : 0, bad.p);
   count_launch();
   int hb[2] = {0, 0};
   bad.download(hb, 2);
   OFG_REQUIRE(!hb[0], OFG_ERR_PIVOT, "zero diagonal entry");
   int bits = inner_bits;
   if (inner_bits == 0) {
      bits = hb[1] ? 32 : 16;
      if (bits == 32) {
         v16.release();
         ensure_sell32(A);
      }
   }
   const float* jac = learned ? nullptr : dinv.p;
   const unsigned gq = grid_for(nquads, kRedBlock, kQuadBlocks);
   // per-block partials of the reductions that the next kernel finishes:
   // (p, q) of the SpMV, ||r||^2 and (r, D r) of the update, (r, z) of the
   // product with G^T
   DBuf<double> red(5 * (size_t)gq + 1);
   double* const pq = red.p;
   double* const rpart = red.p + gq;
   double* const cpart = red.p + 3 * (size_t)gq;
   const unsigned gn = grid_for(n, kRedBlock, 8);
   auto true_residual = [&](int first) {
      spmv_sell(A, x, q64.p);
      mx_residual<<<gn, kRedBlock, 0, stream()>>>(n, b, q64.p, r.p, S.p, partials.p, counter.p,
                                                  tol, first);
      count_launch();
      OFG_LAUNCH_CHECK();
   };
   // z = G^T G r, rho, beta, then the new direction
   // algorithmic bytes of the two factor products: BF16 value + column
   // index (2 or 4 bytes) per entry, the gathered input and the output (and
   // r, q for the reduction of the second)
   const double gl_bytes = learned ? 2.0 * LP->gl->nnz + index_bytes(LP->gl, g16, luni) : 0.0;
   const double gu_bytes = learned ? 2.0 * LP->gu->nnz + index_bytes(LP->gu, g16, uuni) : 0.0;
   auto learned_direction = [&](int fresh, int upd_d, int it, int decide, const StopRule& st) {
      using bf = __nv_bfloat16;
      const bf* vl = reinterpret_cast<const bf*>(learned ? LP->gl->sell_valbf.p : nullptr);
      const bf* vu = reinterpret_cast<const bf*>(learned ? LP->gu->sell_valbf.p : nullptr);
      int* worked = prof_begin();
      if (luni)
         launch_pdl(lg_lower<bf, int16_t, true>, gq, kRedBlock, nquads, LP->gl->sell_ptr.p,
                    LP->gl->sell_d16.p, vl, rr.p, tz.p, S.p, rpart, it, decide, st, worked,
                    LP->gl->sell_uni.p, LP->gl->sell_utab.p);
      else if (g16)
         launch_pdl(lg_lower<bf, int16_t>, gq, kRedBlock, nquads, LP->gl->sell_ptr.p,
                    LP->gl->sell_d16.p, vl, rr.p, tz.p, S.p, rpart, it, decide, st, worked,
                    nullptr, nullptr);
      else
         launch_pdl(lg_lower<bf, int32_t>, gq, kRedBlock, nquads, LP->gl->sell_ptr.p,
                    LP->gl->sell_col.p, vl, rr.p, tz.p, S.p, rpart, it, decide, st, worked,
                    nullptr, nullptr);
      prof_end(PROF_LEARNED_APPLY, gl_bytes + 8.0 * n);
      worked = prof_begin();
      if (uuni)
         launch_pdl(lg_upper<bf, int16_t, true>, gq, kRedBlock, nquads, LP->gu->sell_ptr.p,
                    LP->gu->sell_d16.p, vu, tz.p, zz.p, rr.p, S.p, cpart, worked,
                    LP->gu->sell_uni.p, LP->gu->sell_utab.p);
      else if (g16)
         launch_pdl(lg_upper<bf, int16_t>, gq, kRedBlock, nquads, LP->gu->sell_ptr.p,
                    LP->gu->sell_d16.p, vu, tz.p, zz.p, rr.p, S.p, cpart, worked, nullptr,
                    nullptr);
      else
         launch_pdl(lg_upper<bf, int32_t>, gq, kRedBlock, nquads, LP->gu->sell_ptr.p,
                    LP->gu->sell_col.p, vu, tz.p, zz.p, rr.p, S.p, cpart, worked, nullptr,
                    nullptr);
      prof_end(PROF_LEARNED_APPLY, gu_bytes + 12.0 * n);
      launch_pdl(lg_direction, gq, kRedBlock, nquads, zz.p, p.p, d.p, upd_d, S.p, cpart, it, fresh);
   };
   MixState h{};
   true_residual(1);
   S.download(&h, 1);
   int n_outer = 0;
   // mode 1 solves for d in units of ||r||; mode 0 keeps absolute units
   double scale = 1.0;
   bool fresh = true;
   // stagnation watch of the learned iteration: the recursive residual must
   // halve within kStallIters iterations and stay finite, and the true
   // residual must fall at every refinement
   constexpr int kStallIters = 2000;
   bool stalled = false;
   int no_gain = 0;
   double last_rel = h.rel;
   while (!h.done && n_outer < max_outer && h.it < max_inner && n > 0) {
      if (mode == 1) {
         scale = h.rel * h.bnorm;
         fresh = true;
      }
      mx_load_residual<<<gq, kRedBlock, 0, stream()>>>(n, npad, r.p, 1.0 / scale, jac, rr.p, p.p,
                                                       d.p, fresh ? 1 : 0, S.p, partials.p,
                                                       counter.p);
      count_launch();
      const StopRule st{inner_tol, tol, scale, max_inner, mode};
      if (learned) learned_direction(fresh ? 1 : 0, 0, h.it, 0, st);
      else if (!fresh) {
         mx_direction<<<gq, kRedBlock, 0, stream()>>>(nquads, rr.p, dinv.p, p.p, d.p, 0, S.p, rpart,
                                                      h.it, 0, st);
         count_launch();
      }
      fresh = false;
      int mark_it = h.it;
      double mark_rn = h.rel * h.bnorm / scale;
      int batch = 8;
      for (;;) {
         // iterations done when the batch starts; the kernels of the batch's
         // k-th iteration get it0 + k (and it0 + k + 1 once it is done)
         const int it0 = h.it;
         for (int k = 0; k < batch; ++k) {
            const int cur = it0 + k;
            // the kernels of an iteration chain with programmatic dependent
            // launch: each one's blocks start while the previous one drains
            // its reduction tail
            int* worked = prof_begin();
            const int32_t* su = A->sell_uni.p;
            const int16_t* st16 = A->sell_utab.p;
            if (bits == 32 && auni)
               launch_pdl(mx_spmv<float, int16_t, true>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_d16.p, A->sell_val32.p, p.p, q.p, S.p, pq, worked, su, st16);
            else if (bits == 32 && a16)
               launch_pdl(mx_spmv<float, int16_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_d16.p, A->sell_val32.p, p.p, q.p, S.p, pq, worked, nullptr,
                          nullptr);
            else if (bits == 32)
               launch_pdl(mx_spmv<float, int32_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_col.p, A->sell_val32.p, p.p, q.p, S.p, pq, worked, nullptr,
                          nullptr);
            else if (auni)
               launch_pdl(mx_spmv<__nv_bfloat16, int16_t, true>, gq, kRedBlock, nquads,
                          A->sell_ptr.p, A->sell_d16.p, v16.p, p.p, q.p, S.p, pq, worked, su,
                          st16);
            else if (a16)
               launch_pdl(mx_spmv<__nv_bfloat16, int16_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_d16.p, v16.p, p.p, q.p, S.p, pq, worked, nullptr, nullptr);
            else
               launch_pdl(mx_spmv<__nv_bfloat16, int32_t>, gq, kRedBlock, nquads, A->sell_ptr.p,
                          A->sell_col.p, v16.p, p.p, q.p, S.p, pq, worked, nullptr, nullptr);
            // algorithmic bytes: value (4 or 2 bytes) and column index (4, 2
            // as a 16-bit offset, or a uniform slice's table) per entry, p
            // gathered, q written, p read for the dot
            prof_end(bits == 32 ? PROF_SPMV32 : PROF_SPMV16,
                     (bits == 32 ? 4.0 : 2.0) * A->nnz + index_bytes(A, a16, auni) + 12.0 * n +
                        4.0);
            if (learned) {
               launch_pdl(mx_update<false>, gq, kRedBlock, nquads, rr.p, q.p, jac, S.p, pq,
                          rpart, cur);
               learned_direction(0, 1, cur + 1, 1, st);
            }
            else {
               launch_pdl(mx_update<true>, gq, kRedBlock, nquads, rr.p, q.p, dinv.p, S.p, pq,
                          rpart, cur);
               launch_pdl(mx_direction, gq, kRedBlock, nquads, rr.p, dinv.p, p.p, d.p, 1, S.p,
                          rpart, cur + 1, 1, st);
            }
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
      // the iteration that paused the loop skipped its direction kernel,
      // which would have made its d += alpha p
      mx_flush_d<<<gq, kRedBlock, 0, stream()>>>(nquads, d.p, p.p, S.p);
      count_launch();
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
      solve_mixed(A, OFG_DIAG, bits, mode, b, x, std::max(1, max_outer - n_outer),
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

// CG with the learned preconditioner in FP32 inside FP64 iterative
// refinement (mode 0; the name keeps the "f" of the flexible form it first
// had); falls back to the plain Jacobi iteration when the
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
