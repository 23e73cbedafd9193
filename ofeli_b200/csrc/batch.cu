// batch.cu -- many independent P1 problems of uneven size, assembled and
// solved in one persistent launch.
//
// The problems' meshes, patterns, element-to-CSR maps and node-to-element
// lists are concatenated once (ofg_batch_create).  One launch of
// batch_kernel then does, for every problem: Equation::build() (each node
// gathers its CSR row over its elements in ascending order, as the
// single-problem kernel does, so the values are OFELI's bit for bit), CG with the diagonal
// preconditioner in FP64 (OFELI's CG recurrence, include/solvers/CG.h:99-157)
// to the relative residual `toler`, a check of the FP64 true residual
// ||b - A x|| / ||b|| (the iteration continues from the true residual if the
// check fails), and insertBC into the nodal solution.
//
// Work is taken from a queue, most work first.  Without clusters a block owns
// one problem at a time, so all reductions are block-local.  With
// thread-block clusters (4 or 8 blocks) a problem larger than one block's
// fair share of the total is solved by the whole cluster -- rows, nonzeros
// and nodes split among its blocks, cluster barriers
// between the phases, dot products summed over the blocks in rank order
// through distributed shared memory -- and smaller problems are taken one
// per block of the cluster, so that the largest problems no longer set the
// length of the launch.  The launch shape -- threads per block, lanes per
// CSR row in the SpMV, blocks per cluster -- is picked by a measured
// autotuner (ofg_batch_tune) that first measures every problem's work (rows
// x iterations).  The launch (with the queue reset) is captured in a CUDA
// graph and replayed.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "element.cuh"

namespace ofg {
namespace {

using namespace elem;

struct BatchProblem {
   int64_t node_off, elem_off, row_off, rp_off, nnz_off, n2p_off, n2e_off;
   int32_t nn, ne, n, pad;
};

// a work item: `count` problems order[first ..] taken one per block of a
// cluster, or (big) one problem order[first] solved by the whole cluster
struct BatchItem {
   int32_t first, count, big, pad;
};

struct BatchArgs {
   int nprob, nitems;
   const BatchProblem* probs;
   const int32_t* order;
   const BatchItem* items;
   int* queue;
   // meshes
   const double* coords;
   const int32_t* elem;
   const int32_t* code;
   const int32_t* dof;
   const int32_t* n2e_ptr;   // node-to-element lists, per problem (nn + 1 entries)
   const int32_t* n2e;
   const int32_t* emap;
   // matrices and vectors
   const int32_t* row_ptr;
   const int32_t* col;
   const int32_t* dpos;
   double* val;
   double *b, *x, *r, *p, *q, *dinv;
   // inputs and outputs
   const double* kel;
   const double* f;
   const double* bc;
   double* u;
   int* iters;
   double* res;
   int* bad;
   int max_it;
   double tol;
   // mixed precision: FP32 values, 16-bit column offsets (or int32 columns
   // where an offset does not fit), FP32 inner vectors
   int mixed, offsets16;
   float* val32;
   const int16_t* d16;
   float *rl, *pl, *ql, *dl, *dinv32;
};

// sums NV values over the block; every thread receives the totals (fixed
// order: a shuffle tree within each warp, then the same tree over the warp
// sums in the first warp, whose result is broadcast through shared memory)
template <int NV, int THREADS>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*sh)[THREADS / 32])
{
   constexpr int NW = THREADS / 32;
   __shared__ double tot[NV];
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
   for (int i = 0; i < NV; ++i) {
      double s = warp_sum(v[i]);
      if (lane == 0) sh[i][w] = s;
   }
   __syncthreads();
   if (w == 0) {
#pragma unroll
      for (int i = 0; i < NV; ++i) {
         double s = warp_sum(lane < NW ? sh[i][lane] : 0.0);
         if (lane == 0) tot[i] = s;
      }
   }
   __syncthreads();
#pragma unroll
   for (int i = 0; i < NV; ++i) v[i] = tot[i];
}

// ---- thread-block clusters: rank, barrier, distributed shared memory loads
__device__ __forceinline__ unsigned cluster_rank()
{
   unsigned r;
   asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
   return r;
}

__device__ __forceinline__ void cluster_sync()
{
   asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t cluster_addr(const void* p, unsigned rank)
{
   uint32_t a = (uint32_t)__cvta_generic_to_shared(p), r;
   asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
   return r;
}

__device__ __forceinline__ double ld_cluster(const double* p, unsigned rank)
{
   double v;
   asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(cluster_addr(p, rank)) : "memory");
   return v;
}

__device__ __forceinline__ int ld_cluster(const int* p, unsigned rank)
{
   int v;
   asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(cluster_addr(p, rank)) : "memory");
   return v;
}

// The blocks working on one problem: one block (size 1: block barriers and
// block reductions), or the whole cluster (size > 1: each block owns a
// contiguous share of rows, nonzeros and nodes; cluster
// barriers; reductions summed over the blocks in rank order through
// distributed shared memory, double-buffered exchange slots).
template <int THREADS>
struct Team {
   int rank, size;
   double (*sh)[THREADS / 32];
   double (*xr)[4];
   int parity;
   __device__ __forceinline__ void bar()
   {
      if (size == 1) __syncthreads();
      else cluster_sync();
   }
   template <int NV>
   __device__ __forceinline__ void sum(double (&v)[NV])
   {
      block_sum<NV, THREADS>(v, sh);
      if (size > 1) {
         if (threadIdx.x == 0)
#pragma unroll
            for (int i = 0; i < NV; ++i) xr[parity][i] = v[i];
         cluster_sync();
#pragma unroll
         for (int i = 0; i < NV; ++i) {
            double s = 0.0;
            for (int r = 0; r < size; ++r) s += ld_cluster(&xr[parity][i], (unsigned)r);
            v[i] = s;
         }
         parity ^= 1;
      }
   }
   __device__ __forceinline__ int64_t lo(int64_t n) const { return n * rank / size; }
   __device__ __forceinline__ int64_t hi(int64_t n) const { return n * (rank + 1) / size; }
};

// y = A x over rows [r0, r1), LPR lanes per row; adds this thread's share of
// (w, y) to wy (w may be null) and, when b != null, of ||b - y||^2 to rr
// with b - y stored into rout
template <int THREADS, int LPR>
__device__ __forceinline__ void block_spmv(int r0, int r1, const int32_t* rp, const int32_t* col,
                                           const double* val, const double* x, double* y,
                                           const double* w, double& wy, const double* b,
                                           double* rout, double& rr)
{
   const int lane = threadIdx.x % LPR;
   for (int i0 = r0; i0 < r1; i0 += THREADS / LPR) {
      const int i = i0 + (int)threadIdx.x / LPR;
      double s = 0.0;
      if (i < r1)
         for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += val[k] * x[col[k]];
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LPR);
      if (i < r1 && lane == 0) {
         if (y) y[i] = s;
         if (w) wy += w[i] * s;
         if (b) {
            const double t = b[i] - s;
            rout[i] = t;
            rr += t * t;
         }
      }
   }
}

// q = A p over rows [r0, r1) with FP32 values and FP32 vectors, columns as
// 16-bit offsets from the row (d16) or absolute (col); adds this thread's
// share of (p, q) to pq
template <int THREADS, int LPR>
__device__ __forceinline__ void block_spmv32(int r0, int r1, const int32_t* rp, const int16_t* d16,
                                             const int32_t* col, const float* val, const float* x,
                                             float* y, double& pq)
{
   const int lane = threadIdx.x % LPR;
   for (int i0 = r0; i0 < r1; i0 += THREADS / LPR) {
      const int i = i0 + (int)threadIdx.x / LPR;
      float s = 0.f;
      if (i < r1) {
         if (d16)
            for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += val[k] * x[i + d16[k]];
         else
            for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += val[k] * x[col[k]];
      }
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LPR);
      if (i < r1 && lane == 0) {
         y[i] = s;
         pq += (double)x[i] * (double)s;
      }
   }
}

// CG + DIAG in FP32 inside FP64 refinement (the reliable-update form of the
// single-problem mixed solver): one FP32 recurrence; whenever its residual
// has fallen by 20x since the last refinement, or says the target is
// reached, x += d in FP64, r = b - A x with the FP64 values, r_lo = (float) r,
// and the recurrence continues with its direction kept.  Dot products are
// accumulated in FP64; convergence is declared on the FP64 true residual.
template <int THREADS, int LPR>
__device__ void cg_mixed(const BatchArgs& a, const BatchProblem& P, Team<THREADS>& T, int r0,
                         int r1, int& it_out, double& res_out, bool& done_out)
{
   const int tid = threadIdx.x;
   const int32_t* rp = a.row_ptr + P.rp_off;
   const int32_t* col = a.col + P.nnz_off;
   const double* val = a.val + P.nnz_off;
   const float* v32 = a.val32 + P.nnz_off;
   const int16_t* d16 = a.offsets16 ? a.d16 + P.nnz_off : nullptr;
   const double* b = a.b + P.row_off;
   double* x = a.x + P.row_off;
   double* r = a.r + P.row_off;
   float* rl = a.rl + P.row_off;
   float* pl = a.pl + P.row_off;
   float* ql = a.ql + P.row_off;
   float* dl = a.dl + P.row_off;
   float* m32 = a.dinv32 + P.row_off;
   double v[3] = {0.0, 0.0, 0.0};
   for (int i = r0 + tid; i < r1; i += THREADS) {
      const double bi = b[i];
      const float ri = (float)bi, mi = (float)(1.0 / val[a.dpos[P.row_off + i]]);
      const float zi = mi * ri;
      m32[i] = mi;
      x[i] = 0.0;
      r[i] = bi;
      rl[i] = ri;
      dl[i] = 0.f;
      pl[i] = zi;
      v[0] += bi * bi;
      v[1] += (double)ri * (double)zi;
      v[2] += (double)ri * (double)ri;
   }
   T.sum(v);
   double bnorm = sqrt(v[0]);
   if (bnorm == 0.0) bnorm = 1.0;
   double rho = v[1], rmark = sqrt(v[2]);
   double res = sqrt(v[0]) / bnorm;
   int it = 0;
   bool done = res <= a.tol;
   while (!done && it < a.max_it) {
      ++it;
      double w1[1] = {0.0};
      block_spmv32<THREADS, LPR>(r0, r1, rp, d16, col, v32, pl, ql, w1[0]);
      T.sum(w1);
      const float alpha = (float)(rho / w1[0]);
      double u2[2] = {0.0, 0.0};
      for (int i = r0 + tid; i < r1; i += THREADS) {
         dl[i] += alpha * pl[i];
         const float ri = rl[i] - alpha * ql[i];
         rl[i] = ri;
         u2[0] += (double)ri * ri;
         u2[1] += (double)ri * (ri * m32[i]);
      }
      T.sum(u2);
      const double rn = sqrt(u2[0]);
      double rz = u2[1];
      if (rn <= 0.05 * rmark || rn <= a.tol * bnorm) {
         // refinement in FP64
         for (int i = r0 + tid; i < r1; i += THREADS) {
            x[i] += (double)dl[i];
            dl[i] = 0.f;
         }
         T.bar();
         double w2[1] = {0.0}, d2 = 0.0;
         block_spmv<THREADS, LPR>(r0, r1, rp, col, val, x, nullptr, nullptr, d2, b, r, w2[0]);
         T.sum(w2);
         res = sqrt(w2[0]) / bnorm;
         if (res <= a.tol) {
            done = true;
            break;
         }
         double u3[2] = {0.0, 0.0};
         for (int i = r0 + tid; i < r1; i += THREADS) {
            const float ri = (float)r[i];
            rl[i] = ri;
            u3[0] += (double)ri * (ri * m32[i]);
            u3[1] += (double)ri * ri;
         }
         T.sum(u3);
         rz = u3[0];
         rmark = sqrt(u3[1]);
      }
      const float beta = (float)(rz / rho);
      rho = rz;
      for (int i = r0 + tid; i < r1; i += THREADS) pl[i] = m32[i] * rl[i] + beta * pl[i];
      T.bar();
   }
   if (!done && it > 0) {
      // ran out: fold the correction in and report the true residual
      for (int i = r0 + tid; i < r1; i += THREADS) {
         x[i] += (double)dl[i];
         dl[i] = 0.f;
      }
      T.bar();
      double w2[1] = {0.0}, d2 = 0.0;
      block_spmv<THREADS, LPR>(r0, r1, rp, col, val, x, nullptr, nullptr, d2, b, r, w2[0]);
      T.sum(w2);
      res = sqrt(w2[0]) / bnorm;
   }
   it_out = it;
   res_out = res;
   done_out = done;
}

// One problem: build(), CG + DIAG with the true-residual check, insertBC.
template <int NEN, int THREADS, int LPR>
__device__ void solve_problem(const BatchArgs& a, int pid, Team<THREADS>& T)
{
   const int tid = threadIdx.x;
   const BatchProblem P = a.probs[pid];
   const int n = P.n;
   const double* xy = a.coords + P.node_off * (NEN - 1);  // dim = NEN - 1 coordinates
   const int32_t* code = a.code + P.node_off;
   const int32_t* dof = a.dof + P.node_off;
   const int32_t* rp = a.row_ptr + P.rp_off;
   const int32_t* col = a.col + P.nnz_off;
   double* val = a.val + P.nnz_off;
   double* b = a.b + P.row_off;
   double* x = a.x + P.row_off;
   double* r = a.r + P.row_off;
   double* p = a.p + P.row_off;
   double* q = a.q + P.row_off;
   double* dinv = a.dinv + P.row_off;
   const int nnz = rp[n];
   const int r0 = (int)T.lo(n), r1 = (int)T.hi(n);

   // ---- Equation::build(): each node gathers its CSR row and RHS entry
   // over its elements in ascending order (the single-problem kernel's
   // arithmetic and order: OFELI's values bit for bit)
   {
      const int32_t* np = a.n2e_ptr + P.n2p_off;
      const int32_t* lists = a.n2e + P.n2e_off;
      const int32_t* elem = a.elem + P.elem_off * NEN;
      const int32_t* emap = a.emap + P.elem_off * NEN * NEN;
      const double* kel = a.kel ? a.kel + P.elem_off : nullptr;
      const double* f = a.f ? a.f + P.node_off : nullptr;
      const double* bc = a.bc ? a.bc + P.node_off : nullptr;
      auto report = [&](int64_t e) { atomicMin(a.bad, (int)(P.elem_off + e)); };
      for (int64_t i = T.lo(P.nn) + tid; i < T.hi(P.nn); i += THREADS) {
         const int32_t ri = dof[i];
         double bi;
         if constexpr (NEN == 3)
            bi = gather_node_rows(i, ri, np[i], np[i + 1], lists, elem, emap, rp,
                                  LaplaceT3{xy, code, kel, f, bc}, val, report);
         else
            bi = gather_node_rows(i, ri, np[i], np[i + 1], lists, elem, emap, rp,
                                  DiffusionT4{xy, code, kel, f, bc}, val, report);
         if (ri) b[ri - 1] = bi;
      }
      T.bar();
   }

   int it = 0;
   double res = 0.0;
   bool done = false;
   if (a.mixed) {
      for (int64_t k = T.lo(nnz) + tid; k < T.hi(nnz); k += THREADS) a.val32[P.nnz_off + k] = (float)val[k];
      T.bar();
      cg_mixed<THREADS, LPR>(a, P, T, r0, r1, it, res, done);
   }
   else {
      // ---- CG with the diagonal preconditioner (FP64)
      double v[2] = {0.0, 0.0};
      for (int i = r0 + tid; i < r1; i += THREADS) {
         const double d = 1.0 / val[a.dpos[P.row_off + i]];
         const double bi = b[i], zi = d * bi;
         dinv[i] = d;
         x[i] = 0.0;
         r[i] = bi;
         p[i] = zi;
         v[0] += bi * bi;
         v[1] += bi * zi;
      }
      T.sum(v);
      double bnorm = sqrt(v[0]);
      if (bnorm == 0.0) bnorm = 1.0;
      double rho = v[1];
      res = sqrt(v[0]) / bnorm;
      done = res <= a.tol;
      while (!done && it < a.max_it) {
         ++it;
         double w1[1] = {0.0}, dummy = 0.0;
         block_spmv<THREADS, LPR>(r0, r1, rp, col, val, p, q, p, w1[0], nullptr, nullptr, dummy);
         T.sum(w1);
         const double alpha = rho / w1[0];
         double u2[2] = {0.0, 0.0};
         for (int i = r0 + tid; i < r1; i += THREADS) {
            x[i] += alpha * p[i];
            const double ri = r[i] - alpha * q[i];
            r[i] = ri;
            u2[0] += ri * ri;
            u2[1] += ri * (dinv[i] * ri);
         }
         T.sum(u2);
         res = sqrt(u2[0]) / bnorm;
         double rz = u2[1];
         bool restart = false;
         if (res <= a.tol) {
            // FP64 true residual; r <- b - A x either way
            double w2[1] = {0.0}, d2 = 0.0;
            block_spmv<THREADS, LPR>(r0, r1, rp, col, val, x, nullptr, nullptr, d2, b, r, w2[0]);
            T.sum(w2);
            res = sqrt(w2[0]) / bnorm;
            if (res <= a.tol) {
               done = true;
               break;
            }
            restart = true;
            double u3[1] = {0.0};
            for (int i = r0 + tid; i < r1; i += THREADS) u3[0] += r[i] * (dinv[i] * r[i]);
            T.sum(u3);
            rz = u3[0];
         }
         const double beta = restart ? 0.0 : rz / rho;
         rho = rz;
         for (int i = r0 + tid; i < r1; i += THREADS) p[i] = dinv[i] * r[i] + beta * p[i];
         T.bar();
      }
      if (!done && it > 0) {
         // ran out: report the true residual
         double w2[1] = {0.0}, d2 = 0.0;
         block_spmv<THREADS, LPR>(r0, r1, rp, col, val, x, nullptr, nullptr, d2, b, q, w2[0]);
         T.sum(w2);
         res = sqrt(w2[0]) / bnorm;
      }
   }
   T.bar();
   // ---- insertBC into the nodal solution
   for (int64_t i = T.lo(P.nn) + tid; i < T.hi(P.nn); i += THREADS) {
      const int32_t dd = dof[i];
      a.u[P.node_off + i] = dd ? x[dd - 1] : (a.bc ? a.bc[P.node_off + i] : 0.0);
   }
   if (T.rank == 0 && tid == 0) {
      a.iters[pid] = done ? it : -it;
      a.res[pid] = res;
   }
}

// Persistent kernel: a block (CS == 1) or a cluster of CS blocks takes work
// items from the queue until it is empty.  An item is either up to CS small
// problems (one per block of the cluster) or one large problem that the
// whole cluster solves together.
template <int NEN, int THREADS, int LPR, int CS>
__global__ void __launch_bounds__(THREADS, 2048 / THREADS) batch_kernel(BatchArgs a)
{
   __shared__ int s_item;
   __shared__ double sh[3][THREADS / 32];
   __shared__ double xr[2][4];
   const int tid = threadIdx.x;
   const unsigned rank = CS > 1 ? cluster_rank() : 0u;
   Team<THREADS> T{0, 1, sh, xr, 0};
   for (;;) {
      int item;
      if constexpr (CS == 1) {
         if (tid == 0) s_item = atomicAdd(a.queue, 1);
         __syncthreads();
         item = s_item;
         __syncthreads();
      }
      else {
         if (rank == 0 && tid == 0) s_item = atomicAdd(a.queue, 1);
         cluster_sync();
         item = ld_cluster(&s_item, 0u);
         cluster_sync();
      }
      if (item >= a.nitems) break;
      const BatchItem w = a.items[item];
      if (w.big) {
         T.rank = (int)rank;
         T.size = CS;
         solve_problem<NEN, THREADS, LPR>(a, a.order[w.first], T);
      }
      else if ((int)rank < w.count) {
         T.rank = 0;
         T.size = 1;
         solve_problem<NEN, THREADS, LPR>(a, a.order[w.first + rank], T);
      }
      __syncthreads();
   }
}

// 16-bit column offsets (column - row, local numbering) of every problem;
// one block per problem; flags an offset that does not fit
__global__ void batch_offsets16(int nprob, const BatchProblem* probs, const int32_t* row_ptr,
                                const int32_t* col, int16_t* d16, int* wide)
{
   for (int p = blockIdx.x; p < nprob; p += gridDim.x) {
      const BatchProblem P = probs[p];
      const int32_t* rp = row_ptr + P.rp_off;
      for (int i = threadIdx.x; i < P.n; i += blockDim.x)
         for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            const int d = col[P.nnz_off + k] - i;
            if (d > 32767 || d < -32768) atomicOr(wide, 1);
            d16[P.nnz_off + k] = (int16_t)d;
         }
   }
}

struct Config {
   int threads, lpr, cs;
};
constexpr Config kConfigs[] = {
   {256, 1, 1},  {256, 2, 1},  {512, 1, 1},  {512, 2, 1},  {1024, 1, 1}, {1024, 2, 1},
   {256, 1, 4},  {256, 2, 4},  {512, 1, 4},  {512, 2, 4},  {1024, 1, 4}, {1024, 2, 4},
   {256, 1, 8},  {256, 2, 8},  {512, 1, 8},  {512, 2, 8},  {1024, 1, 8}, {1024, 2, 8}};
constexpr int kNumConfigs = sizeof(kConfigs) / sizeof(kConfigs[0]);

// blocks that run at once for a configuration (whole clusters)
template <int NEN, int T, int L, int CS>
int concurrent_blocks(int blocks_per_sm)
{
   if constexpr (CS == 1) {
      int occ = 0;
      OFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel<NEN, T, L, 1>, T, 0));
      occ = std::max(1, blocks_per_sm > 0 ? std::min(occ, blocks_per_sm) : occ);
      return occ * num_sms();
   }
   else {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(CS * num_sms());
      cfg.blockDim = dim3(T);
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = CS;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int nclusters = 0;
      OFG_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, batch_kernel<NEN, T, L, CS>, &cfg));
      int blocks = std::max(1, nclusters) * CS;
      if (blocks_per_sm > 0) blocks = std::min(blocks, std::max(CS, blocks_per_sm * num_sms() / CS * CS));
      return blocks;
   }
}

template <int NEN, int T, int L, int CS>
void launch_one(const BatchArgs& a, int blocks, cudaStream_t st)
{
   if constexpr (CS == 1) {
      batch_kernel<NEN, T, L, 1><<<std::max(1, blocks), T, 0, st>>>(a);
   }
   else {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(std::max(CS, blocks / CS * CS));
      cfg.blockDim = dim3(T);
      cfg.stream = st;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = CS;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      OFG_CUDA(cudaLaunchKernelEx(&cfg, batch_kernel<NEN, T, L, CS>, a));
   }
   count_launch();
}

// dispatch over the configuration table: concurrency (launch == false) or
// the launch itself
template <int NEN>
int for_config(int c, bool launch, const BatchArgs* a, int blocks, int blocks_per_sm,
               cudaStream_t st)
{
#define OFG_BATCH_CASE(idx, T, L, CS)                                        \
   case idx:                                                                 \
      if (launch) launch_one<NEN, T, L, CS>(*a, blocks, st);                 \
      else return concurrent_blocks<NEN, T, L, CS>(blocks_per_sm);           \
      return 0;
   switch (c) {
      OFG_BATCH_CASE(0, 256, 1, 1)
      OFG_BATCH_CASE(1, 256, 2, 1)
      OFG_BATCH_CASE(2, 512, 1, 1)
      OFG_BATCH_CASE(3, 512, 2, 1)
      OFG_BATCH_CASE(4, 1024, 1, 1)
      OFG_BATCH_CASE(5, 1024, 2, 1)
      OFG_BATCH_CASE(6, 256, 1, 4)
      OFG_BATCH_CASE(7, 256, 2, 4)
      OFG_BATCH_CASE(8, 512, 1, 4)
      OFG_BATCH_CASE(9, 512, 2, 4)
      OFG_BATCH_CASE(10, 1024, 1, 4)
      OFG_BATCH_CASE(11, 1024, 2, 4)
      OFG_BATCH_CASE(12, 256, 1, 8)
      OFG_BATCH_CASE(13, 256, 2, 8)
      OFG_BATCH_CASE(14, 512, 1, 8)
      OFG_BATCH_CASE(15, 512, 2, 8)
      OFG_BATCH_CASE(16, 1024, 1, 8)
      default: break;
   }
   if (launch) launch_one<NEN, 1024, 2, 8>(*a, blocks, st);
   else return concurrent_blocks<NEN, 1024, 2, 8>(blocks_per_sm);
   return 0;
#undef OFG_BATCH_CASE
}

}  // namespace
}  // namespace ofg

struct ofg_batch {
   int nprob = 0, dim = 2, nen = 3;
   int64_t nn = 0, ne = 0, nrows = 0, nnz = 0;
   std::vector<ofg::BatchProblem> probs;
   ofg::DBuf<ofg::BatchProblem> d_probs;
   ofg::DBuf<int32_t> order;
   ofg::DBuf<int> queue, bad, iters;
   ofg::DBuf<double> coords;
   ofg::DBuf<int32_t> elem, code, dof, n2e_ptr, n2e, emap, row_ptr, col, dpos;
   ofg::DBuf<double> val, b, x, r, p, q, dinv, kel, f, bc, u, res;
   bool have_bc = false;
   int config = 4;  // index into kConfigs
   int blocks_per_sm = 0;
   // work estimate per problem (rows x iterations once measured) and the
   // work items built from it for the current configuration
   std::vector<double> work;
   ofg::DBuf<ofg::BatchItem> items;
   int nitems = 0, items_config = -1, blocks = 1;
   bool work_measured = false;
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   cudaStream_t capture = nullptr;
   int graph_config = -1;
   int max_it = 0;
   double tol = 0.0;
   // mixed precision (bits 32): FP32 value copy, 16-bit offsets, FP32 vectors
   int bits = 64, offsets16 = 0;
   ofg::DBuf<float> val32, rl, pl, ql, dl, dinv32;
   ofg::DBuf<int16_t> d16;
   ~ofg_batch()
   {
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      if (capture) cudaStreamDestroy(capture);
   }
};

namespace ofg {
namespace {

BatchArgs args_of(ofg_batch* B)
{
   BatchArgs a{};
   a.nprob = B->nprob;
   a.nitems = B->nitems;
   a.probs = B->d_probs.p;
   a.order = B->order.p;
   a.items = B->items.p;
   a.queue = B->queue.p;
   a.coords = B->coords.p;
   a.elem = B->elem.p;
   a.code = B->code.p;
   a.dof = B->dof.p;
   a.n2e_ptr = B->n2e_ptr.p;
   a.n2e = B->n2e.p;
   a.emap = B->emap.p;
   a.row_ptr = B->row_ptr.p;
   a.col = B->col.p;
   a.dpos = B->dpos.p;
   a.val = B->val.p;
   a.b = B->b.p;
   a.x = B->x.p;
   a.r = B->r.p;
   a.p = B->p.p;
   a.q = B->q.p;
   a.dinv = B->dinv.p;
   a.kel = B->kel.p;
   a.f = B->f.p;
   a.bc = B->have_bc ? B->bc.p : nullptr;
   a.u = B->u.p;
   a.iters = B->iters.p;
   a.res = B->res.p;
   a.bad = B->bad.p;
   a.max_it = B->max_it;
   a.tol = B->tol;
   a.mixed = B->bits == 32;
   a.offsets16 = B->offsets16;
   a.val32 = B->val32.p;
   a.d16 = B->d16.p;
   a.rl = B->rl.p;
   a.pl = B->pl.p;
   a.ql = B->ql.p;
   a.dl = B->dl.p;
   a.dinv32 = B->dinv32.p;
   return a;
}

int concurrency(ofg_batch* B, int config)
{
   return B->nen == 3 ? for_config<3>(config, false, nullptr, 0, B->blocks_per_sm, nullptr)
                      : for_config<4>(config, false, nullptr, 0, B->blocks_per_sm, nullptr);
}

// Problem order (most work first) and work items for a configuration: with
// clusters, a problem whose work exceeds one block's fair share of the
// total gets the whole cluster; the others are grouped CS at a time in
// order, so a group holds problems of similar size.  Items run in
// decreasing order of their time per block.
void build_items(ofg_batch* B, int config)
{
   if (B->items_config == config) return;
   const int np = B->nprob, cs = kConfigs[config].cs;
   std::vector<int32_t> order(np);
   std::iota(order.begin(), order.end(), 0);
   std::stable_sort(order.begin(), order.end(),
                    [&](int32_t x, int32_t y) { return B->work[x] > B->work[y]; });
   const double total = std::accumulate(B->work.begin(), B->work.end(), 0.0);
   const double fair = total / std::max(1, concurrency(B, config));
   std::vector<BatchItem> items;
   std::vector<double> cost;
   for (int i = 0; i < np;) {
      const double w = B->work[order[i]];
      if (cs > 1 && w > fair) {
         items.push_back({i, 1, 1, 0});
         cost.push_back(w / cs);
         ++i;
      }
      else {
         const int c = std::min(cs, np - i);
         items.push_back({i, c, 0, 0});
         cost.push_back(w);
         i += c;
      }
   }
   std::vector<int> idx(items.size());
   std::iota(idx.begin(), idx.end(), 0);
   std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return cost[x] > cost[y]; });
   std::vector<BatchItem> sorted;
   for (int k : idx) sorted.push_back(items[k]);
   B->order.upload(order.data(), np);
   B->items.upload(sorted.data(), sorted.size());
   B->nitems = (int)sorted.size();
   B->blocks = (int)std::min<int64_t>(concurrency(B, config), (int64_t)B->nitems * cs);
   B->items_config = config;
   OFG_CUDA(cudaStreamSynchronize(stream()));
}

// the queue reset and the persistent launch, as stream work
void enqueue(ofg_batch* B, int config, cudaStream_t st)
{
   OFG_CUDA(cudaMemsetAsync(B->queue.p, 0, sizeof(int), st));
   const BatchArgs a = args_of(B);
   if (B->nen == 3) for_config<3>(config, true, &a, B->blocks, B->blocks_per_sm, st);
   else for_config<4>(config, true, &a, B->blocks, B->blocks_per_sm, st);
   OFG_LAUNCH_CHECK();
}

// per-problem work from the last solve's iteration counts
void measure_work(ofg_batch* B)
{
   std::vector<int> it(B->nprob);
   B->iters.download(it.data(), B->nprob);
   for (int p = 0; p < B->nprob; ++p)
      B->work[p] = (double)B->probs[p].n * (double)std::max(1, std::abs(it[p]));
   B->work_measured = true;
   B->items_config = -1;
}

// the same work through a CUDA graph, captured (on the batch's own capture
// stream) once per configuration and solver setting, launched on the
// library stream
void run_graph(ofg_batch* B)
{
   if (B->items_config != B->config) {
      build_items(B, B->config);
      B->graph_config = -1;
   }
   if (B->graph_config != B->config) {
      if (B->exec) cudaGraphExecDestroy(B->exec);
      if (B->graph) cudaGraphDestroy(B->graph);
      B->exec = nullptr;
      B->graph = nullptr;
      if (!B->capture) OFG_CUDA(cudaStreamCreateWithFlags(&B->capture, cudaStreamNonBlocking));
      OFG_CUDA(cudaStreamBeginCapture(B->capture, cudaStreamCaptureModeThreadLocal));
      try {
         enqueue(B, B->config, B->capture);
      }
      catch (...) {
         cudaGraph_t g = nullptr;
         cudaStreamEndCapture(B->capture, &g);
         if (g) cudaGraphDestroy(g);
         throw;
      }
      OFG_CUDA(cudaStreamEndCapture(B->capture, &B->graph));
      OFG_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
      B->graph_config = B->config;
   }
   OFG_CUDA(cudaGraphLaunch(B->exec, stream()));
   count_launch();  // the graph's kernel (the queue reset is a memset)
}

void check_bad(ofg_batch* B)
{
   int h = 0;
   B->bad.download(&h, 1);
   if (h != INT32_MAX) {
      int big = INT32_MAX;
      B->bad.upload(&big, 1);
      throw Error(OFG_ERR_JACOBIAN, "non-positive Jacobian determinant in batch element " +
                                        std::to_string(h + 1));
   }
}

template <class T>
void gather(DBuf<T>& dst, int64_t off, const T* src, int64_t count)
{
   if (count > 0)
      OFG_CUDA(cudaMemcpyAsync(dst.p + off, src, count * sizeof(T), cudaMemcpyDeviceToDevice,
                               stream()));
}

}  // namespace
}  // namespace ofg

using namespace ofg;

extern "C" {

int ofg_batch_create(int nprob, ofg_mesh* const* meshes, ofg_batch** out)
{
   return guarded("ofg_batch_create", [&] {
      OFG_REQUIRE(nprob > 0 && meshes && out, OFG_ERR_ARG, "bad arguments");
      auto B = new ofg_batch();
      try {
         B->nprob = nprob;
         B->dim = meshes[0]->dim;
         B->nen = meshes[0]->nen;
         std::vector<ofg_matrix*> mats(nprob, nullptr);
         for (int p = 0; p < nprob; ++p) {
            ofg_mesh* m = meshes[p];
            OFG_REQUIRE(m && m->dim == B->dim, OFG_ERR_ARG, "batch meshes must share one dimension");
            if (ofg_matrix_create_from_mesh(m, &mats[p]) != OFG_OK)
               throw Error(OFG_ERR_PATTERN, std::string("pattern of batch problem ") +
                                                std::to_string(p) + ": " + ofg_last_error());
            OFG_REQUIRE(m->nn < INT32_MAX && m->ne < INT32_MAX, OFG_ERR_SIZE, "problem too large");
            BatchProblem P{};
            P.node_off = B->nn;
            P.elem_off = B->ne;
            P.row_off = B->nrows;
            P.rp_off = B->nrows + p;
            P.nnz_off = B->nnz;
            P.n2p_off = B->nn + p;
            P.n2e_off = B->ne * m->nen;
            P.nn = (int32_t)m->nn;
            P.ne = (int32_t)m->ne;
            P.n = (int32_t)mats[p]->n;

            B->probs.push_back(P);
            B->nn += m->nn;
            B->ne += m->ne;
            B->nrows += mats[p]->n;
            B->nnz += mats[p]->nnz;

            ensure_dpos(mats[p]);
            OFG_REQUIRE(mats[p]->dpos_complete, OFG_ERR_PIVOT, "a row has no diagonal entry");
         }
         OFG_REQUIRE(B->nnz < INT32_MAX, OFG_ERR_SIZE, "batch nonzeros must be below 2^31");
         const int nen = B->nen, dim = B->dim;
         B->coords.alloc(B->nn * dim);
         B->elem.alloc(B->ne * nen);
         B->code.alloc(B->nn);
         B->dof.alloc(B->nn);
         B->n2e_ptr.alloc(B->nn + nprob);
         B->n2e.alloc(B->ne * nen);
         B->emap.alloc(B->ne * nen * nen);
         B->row_ptr.alloc(B->nrows + nprob);
         B->col.alloc(B->nnz);
         B->dpos.alloc(B->nrows);
         for (int p = 0; p < nprob; ++p) {
            ofg_mesh* m = meshes[p];
            ofg_matrix* A = mats[p];
            const BatchProblem& P = B->probs[p];
            gather(B->coords, P.node_off * dim, m->coords.p, m->nn * dim);
            gather(B->elem, P.elem_off * nen, m->elem.p, m->ne * nen);
            gather(B->code, P.node_off, m->code.p, m->nn);
            gather(B->dof, P.node_off, m->dof.p, m->nn);
            gather(B->n2e_ptr, P.n2p_off, m->n2e_ptr.p, m->nn + 1);
            gather(B->n2e, P.n2e_off, m->n2e.p, m->ne * nen);
            gather(B->emap, P.elem_off * nen * nen, A->emap.p, m->ne * nen * nen);
            gather(B->row_ptr, P.rp_off, A->row_ptr.p, A->n + 1);
            gather(B->col, P.nnz_off, A->col.p, A->nnz);
            gather(B->dpos, P.row_off, A->dpos.p, A->n);
         }
         OFG_CUDA(cudaStreamSynchronize(stream()));
         for (auto* A : mats) delete A;
         // work estimate until iteration counts are measured: rows x
         // rows^(1/2) (CG iterations grow like the mesh width in 2-D)
         B->work.resize(nprob);
         for (int p = 0; p < nprob; ++p)
            B->work[p] = (double)B->probs[p].n * std::sqrt((double)std::max(1, B->probs[p].n));
         B->order.alloc(nprob);
         B->items.alloc(nprob);
         B->d_probs.alloc(nprob);
         B->d_probs.upload(B->probs.data(), nprob);
         B->queue.alloc(1);
         B->bad.alloc(1);
         int big = INT32_MAX;
         B->bad.upload(&big, 1);
         B->iters.alloc(nprob);
         B->res.alloc(nprob);
         B->val.alloc(B->nnz);
         for (auto* v : {&B->b, &B->x, &B->r, &B->p, &B->q, &B->dinv}) v->alloc(B->nrows);
         B->kel.alloc(B->ne);
         B->f.alloc(B->nn);
         B->bc.alloc(B->nn);
         B->u.alloc(B->nn);
         B->kel.zero();
         B->f.zero();
         B->bc.zero();
         OFG_CUDA(cudaStreamSynchronize(stream()));
      }
      catch (...) {
         delete B;
         throw;
      }
      *out = B;
   });
}

int ofg_batch_destroy(ofg_batch* B)
{
   return guarded("ofg_batch_destroy", [&] {
      delete B;
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_batch_info(const ofg_batch* B, int* nprob, int64_t* nodes, int64_t* elements,
                   int64_t* rows, int64_t* nnz)
{
   return guarded("ofg_batch_info", [&] {
      OFG_REQUIRE(B, OFG_ERR_ARG, "null batch");
      if (nprob) *nprob = B->nprob;
      if (nodes) *nodes = B->nn;
      if (elements) *elements = B->ne;
      if (rows) *rows = B->nrows;
      if (nnz) *nnz = B->nnz;
   });
}

int ofg_batch_problem_info(const ofg_batch* B, int prob, int64_t* nodes, int64_t* elements,
                           int64_t* rows, int64_t* nnz)
{
   return guarded("ofg_batch_problem_info", [&] {
      OFG_REQUIRE(B && prob >= 0 && prob < B->nprob, OFG_ERR_ARG, "bad arguments");
      const BatchProblem& P = B->probs[prob];
      const int64_t next = prob + 1 < B->nprob ? B->probs[prob + 1].nnz_off : B->nnz;
      if (nodes) *nodes = P.nn;
      if (elements) *elements = P.ne;
      if (rows) *rows = P.n;
      if (nnz) *nnz = next - P.nnz_off;
   });
}

int ofg_batch_set_inputs(ofg_batch* B, const double* kel, const double* f, const double* bc)
{
   return guarded("ofg_batch_set_inputs", [&] {
      OFG_REQUIRE(B, OFG_ERR_ARG, "null batch");
      if (kel) B->kel.upload(kel, B->ne);
      else {
         // k = 1
         std::vector<double> ones(B->ne, 1.0);
         B->kel.upload(ones.data(), B->ne);
         OFG_CUDA(cudaStreamSynchronize(stream()));
      }
      if (f) B->f.upload(f, B->nn);
      else B->f.zero();
      B->have_bc = bc != nullptr;
      if (bc) B->bc.upload(bc, B->nn);
   });
}

int ofg_batch_solve(ofg_batch* B, int max_it, double toler)
{
   return guarded("ofg_batch_solve", [&] {
      OFG_REQUIRE(B && max_it >= 0, OFG_ERR_ARG, "bad arguments");
      if (B->max_it != max_it || B->tol != toler) {
         B->graph_config = -1;  // the captured launch holds the settings
         B->max_it = max_it;
         B->tol = toler;
      }
      run_graph(B);
      check_bad(B);
   });
}

int ofg_batch_get_results(const ofg_batch* B, double* u, int* iters, double* res)
{
   return guarded("ofg_batch_get_results", [&] {
      OFG_REQUIRE(B, OFG_ERR_ARG, "null batch");
      if (u) B->u.download(u, B->nn);
      if (iters) B->iters.download(iters, B->nprob);
      if (res) B->res.download(res, B->nprob);
   });
}

int ofg_batch_get_matrix(const ofg_batch* B, int prob, double* values, double* rhs)
{
   return guarded("ofg_batch_get_matrix", [&] {
      OFG_REQUIRE(B && prob >= 0 && prob < B->nprob, OFG_ERR_ARG, "bad arguments");
      const BatchProblem& P = B->probs[prob];
      int32_t nnz = 0, first = 0;
      OFG_CUDA(cudaMemcpyAsync(&first, B->row_ptr.p + P.rp_off, 4, cudaMemcpyDeviceToHost, stream()));
      OFG_CUDA(cudaMemcpyAsync(&nnz, B->row_ptr.p + P.rp_off + P.n, 4, cudaMemcpyDeviceToHost,
                               stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
      if (values)
         OFG_CUDA(cudaMemcpyAsync(values, B->val.p + P.nnz_off, (nnz - first) * sizeof(double),
                                  cudaMemcpyDefault, stream()));
      if (rhs)
         OFG_CUDA(cudaMemcpyAsync(rhs, B->b.p + P.row_off, P.n * sizeof(double), cudaMemcpyDefault,
                                  stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

// Measured autotuner: solves once to measure every problem's work, then runs
// the whole batch once per launch shape (threads per block x lanes per CSR
// row x blocks per cluster, with the work items built for that shape) on
// the current inputs, and keeps the fastest.
int ofg_batch_tune(ofg_batch* B, int max_it, double toler, int* chosen, float* times_ms)
{
   return guarded("ofg_batch_tune", [&] {
      OFG_REQUIRE(B, OFG_ERR_ARG, "null batch");
      B->max_it = max_it;
      B->tol = toler;
      cudaEvent_t e0, e1;
      OFG_CUDA(cudaEventCreate(&e0));
      OFG_CUDA(cudaEventCreate(&e1));
      float best = 1e30f;
      int best_c = B->config;
      // the per-problem work the items are built from: measured iterations
      build_items(B, B->config);
      enqueue(B, B->config, stream());
      OFG_CUDA(cudaStreamSynchronize(stream()));
      measure_work(B);
      for (int c = 0; c < kNumConfigs; ++c) {
         build_items(B, c);
         enqueue(B, c, stream());  // warm-up
         OFG_CUDA(cudaEventRecord(e0, stream()));
         enqueue(B, c, stream());
         OFG_CUDA(cudaEventRecord(e1, stream()));
         OFG_CUDA(cudaEventSynchronize(e1));
         float ms = 0.f;
         OFG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
         if (times_ms) times_ms[c] = ms;
         if (ms < best) {
            best = ms;
            best_c = c;
         }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      check_bad(B);
      B->config = best_c;
      B->items_config = -1;
      B->graph_config = -1;
      if (chosen) *chosen = best_c;
   });
}

int ofg_batch_set_precision(ofg_batch* B, int bits)
{
   return guarded("ofg_batch_set_precision", [&] {
      OFG_REQUIRE(B && (bits == 64 || bits == 32), OFG_ERR_ARG, "bits must be 64 or 32");
      if (bits == 32 && !B->val32.p) {
         B->val32.alloc(B->nnz);
         for (auto* v : {&B->rl, &B->pl, &B->ql, &B->dl, &B->dinv32}) v->alloc(B->nrows);
         B->d16.alloc(B->nnz);
         DBuf<int> wide(1);
         wide.zero();
         batch_offsets16<<<std::min(B->nprob, num_sms() * 4), 256, 0, stream()>>>(
            B->nprob, B->d_probs.p, B->row_ptr.p, B->col.p, B->d16.p, wide.p);
         count_launch();
         OFG_LAUNCH_CHECK();
         int h = 0;
         wide.download(&h, 1);
         B->offsets16 = h ? 0 : 1;
         if (!B->offsets16) B->d16.release();
      }
      if (B->bits != bits) {
         B->bits = bits;
         B->graph_config = -1;
      }
   });
}

int ofg_batch_set_config(ofg_batch* B, int config, int blocks_per_sm)
{
   return guarded("ofg_batch_set_config", [&] {
      OFG_REQUIRE(B && config >= 0 && config < kNumConfigs && blocks_per_sm >= 0, OFG_ERR_ARG,
                  "bad arguments");
      B->config = config;
      B->blocks_per_sm = blocks_per_sm;
      B->items_config = -1;
      B->graph_config = -1;
   });
}

int ofg_batch_config_shape(int config, int* threads, int* lanes_per_row, int* cluster)
{
   return guarded("ofg_batch_config_shape", [&] {
      OFG_REQUIRE(config >= 0 && config < kNumConfigs, OFG_ERR_ARG, "bad configuration");
      if (threads) *threads = kConfigs[config].threads;
      if (lanes_per_row) *lanes_per_row = kConfigs[config].lpr;
      if (cluster) *cluster = kConfigs[config].cs;
   });
}

}  // extern "C"
