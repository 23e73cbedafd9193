// batch.cu -- many independent P1 problems of uneven size, assembled and
// solved in one persistent launch.
//
// The problems' meshes, patterns, element-to-CSR maps and element colourings
// are concatenated once (ofg_batch_create).  One launch of batch_kernel then
// does, for every problem: Equation::build() (coloured, atomic-free element
// scatter, the colours separated by block barriers), CG with the diagonal
// preconditioner in FP64 (OFELI's CG recurrence, include/solvers/CG.h:99-157)
// to the relative residual `toler`, a check of the FP64 true residual
// ||b - A x|| / ||b|| (the iteration continues from the true residual if the
// check fails), and insertBC into the nodal solution.
//
// A block owns one problem at a time and takes the next one from a queue in
// decreasing order of nonzeros (longest first), so all reductions are
// block-local and nothing waits across blocks.  The launch shape -- threads
// per block and the lanes that share one CSR row in the SpMV -- is a template
// choice picked by a measured autotuner (ofg_batch_tune).  The launch (with
// the queue reset) is captured in a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "element.cuh"

namespace ofg {
namespace {

using namespace elem;

struct BatchProblem {
   int64_t node_off, elem_off, row_off, rp_off, nnz_off, color_base;
   int32_t nn, ne, n, ncolors;
};

struct BatchArgs {
   int nprob;
   const BatchProblem* probs;
   const int32_t* order;
   int* queue;
   // meshes
   const double* coords;
   const int32_t* elem;
   const int32_t* code;
   const int32_t* dof;
   const int64_t* color_ptr;
   const int32_t* color_elems;
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
};

// sums NV values over the block; every thread receives the totals (fixed
// order: warps in index order)
template <int NV, int THREADS>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*sh)[THREADS / 32])
{
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
   for (int i = 0; i < NV; ++i) {
      double s = warp_sum(v[i]);
      if (lane == 0) sh[i][w] = s;
   }
   __syncthreads();
#pragma unroll
   for (int i = 0; i < NV; ++i) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < THREADS / 32; ++k) s += sh[i][k];
      v[i] = s;
   }
   __syncthreads();
}

// y = A x over the problem's rows, LPR lanes per row; returns this thread's
// share of (w, y) (w may be null) and, when b != null, of ||b - y||^2 with
// b - y stored into rout
template <int THREADS, int LPR>
__device__ __forceinline__ void block_spmv(int n, const int32_t* rp, const int32_t* col,
                                           const double* val, const double* x, double* y,
                                           const double* w, double& wy, const double* b,
                                           double* rout, double& rr)
{
   const int lane = threadIdx.x % LPR;
   for (int i0 = 0; i0 < n; i0 += THREADS / LPR) {
      const int i = i0 + (int)threadIdx.x / LPR;
      double s = 0.0;
      if (i < n)
         for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += val[k] * x[col[k]];
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LPR);
      if (i < n && lane == 0) {
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

template <int NEN, int THREADS, int LPR>
__global__ void __launch_bounds__(THREADS) batch_kernel(BatchArgs a)
{
   __shared__ int s_slot;
   __shared__ double sh[3][THREADS / 32];
   const int tid = threadIdx.x;
   for (;;) {
      if (tid == 0) s_slot = atomicAdd(a.queue, 1);
      __syncthreads();
      const int slot = s_slot;
      __syncthreads();
      if (slot >= a.nprob) break;
      const int pid = a.order[slot];
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

      // ---- Equation::build(): zero, then one pass per element colour
      for (int k = tid; k < nnz; k += THREADS) val[k] = 0.0;
      for (int i = tid; i < n; i += THREADS) b[i] = 0.0;
      __syncthreads();
      for (int c = 0; c < P.ncolors; ++c) {
         const int64_t beg = a.color_ptr[P.color_base + c], end = a.color_ptr[P.color_base + c + 1];
         for (int64_t t = beg + tid; t < end; t += THREADS) {
            const int64_t e = a.color_elems[P.elem_off + t];
            const int32_t* ep = a.elem + (P.elem_off + e) * NEN;
            int32_t en[NEN];
#pragma unroll
            for (int i = 0; i < NEN; ++i) en[i] = ep[i];
            // Laplace2DT3::LHS (times k) + BodyRHS, or DC3DT4::Diffusion(k) +
            // BodyRHS: the operation order of the single-problem kernels
            double g[NEN][3], meas;
            bool ok;
            if constexpr (NEN == 3) ok = tri3(xy, en, g, meas);
            else ok = tet4(xy, en, g, meas);
            if (!ok) {
               atomicMin(a.bad, (int)(P.elem_off + e));
               continue;
            }
            const double k = a.kel ? a.kel[P.elem_off + e] : 1.0;
            double Ke[NEN][NEN], Fe[NEN];
            if constexpr (NEN == 3) {
#pragma unroll
               for (int i = 0; i < 3; ++i)
#pragma unroll
                  for (int j = 0; j < 3; ++j) Ke[i][j] = meas * dot3(g[i], g[j]) * k;
#pragma unroll
               for (int i = 0; i < 3; ++i) Fe[i] = a.f ? a.f[P.node_off + en[i]] * meas * kThird : 0.0;
            }
            else {
               const double c = k * meas;
#pragma unroll
               for (int i = 0; i < 4; ++i)
#pragma unroll
                  for (int j = 0; j < 4; ++j) Ke[i][j] = c * dot3(g[i], g[j]);
#pragma unroll
               for (int i = 0; i < 4; ++i) Fe[i] = a.f ? a.f[P.node_off + en[i]] * 0.25 * meas : 0.0;
            }
            if (a.bc) lift_bc<NEN>(en, code, a.bc + P.node_off, Ke, Fe);
            scatter<NEN>(P.elem_off + e, en, dof, a.emap, Ke, Fe, val, b);
         }
         __syncthreads();
      }

      // ---- CG with the diagonal preconditioner (FP64)
      double v[3] = {0.0, 0.0, 0.0};
      for (int i = tid; i < n; i += THREADS) {
         const double d = 1.0 / val[a.dpos[P.row_off + i]];
         const double bi = b[i], zi = d * bi;
         dinv[i] = d;
         x[i] = 0.0;
         r[i] = bi;
         p[i] = zi;
         v[0] += bi * bi;
         v[1] += bi * zi;
      }
      block_sum<3, THREADS>(v, sh);
      double bnorm = sqrt(v[0]);
      if (bnorm == 0.0) bnorm = 1.0;
      double rho = v[1];
      double res = sqrt(v[0]) / bnorm;
      int it = 0;
      bool done = res <= a.tol;
      while (!done && it < a.max_it) {
         ++it;
         double pq = 0.0, dummy = 0.0;
         block_spmv<THREADS, LPR>(n, rp, col, val, p, q, p, pq, nullptr, nullptr, dummy);
         double w1[1] = {pq};
         block_sum<1, THREADS>(w1, sh);
         const double alpha = rho / w1[0];
         double u2[3] = {0.0, 0.0, 0.0};
         for (int i = tid; i < n; i += THREADS) {
            x[i] += alpha * p[i];
            const double ri = r[i] - alpha * q[i];
            r[i] = ri;
            u2[0] += ri * ri;
            u2[1] += ri * (dinv[i] * ri);
         }
         block_sum<3, THREADS>(u2, sh);
         res = sqrt(u2[0]) / bnorm;
         double rz = u2[1];
         bool restart = false;
         if (res <= a.tol) {
            // FP64 true residual; r <- b - A x either way
            double tr = 0.0, d2 = 0.0;
            block_spmv<THREADS, LPR>(n, rp, col, val, x, nullptr, nullptr, d2, b, r, tr);
            double w2[1] = {tr};
            block_sum<1, THREADS>(w2, sh);
            res = sqrt(w2[0]) / bnorm;
            if (res <= a.tol) {
               done = true;
               break;
            }
            restart = true;
            double u3[3] = {0.0, 0.0, 0.0};
            for (int i = tid; i < n; i += THREADS) u3[0] += r[i] * (dinv[i] * r[i]);
            block_sum<3, THREADS>(u3, sh);
            rz = u3[0];
         }
         const double beta = restart ? 0.0 : rz / rho;
         rho = rz;
         for (int i = tid; i < n; i += THREADS) p[i] = dinv[i] * r[i] + beta * p[i];
         __syncthreads();
      }
      if (!done && it > 0) {
         // ran out: report the true residual
         double tr = 0.0, d2 = 0.0;
         block_spmv<THREADS, LPR>(n, rp, col, val, x, nullptr, nullptr, d2, b, q, tr);
         double w2[1] = {tr};
         block_sum<1, THREADS>(w2, sh);
         res = sqrt(w2[0]) / bnorm;
      }
      // ---- insertBC into the nodal solution
      for (int i = tid; i < P.nn; i += THREADS) {
         const int32_t dd = dof[i];
         a.u[P.node_off + i] = dd ? x[dd - 1] : (a.bc ? a.bc[P.node_off + i] : 0.0);
      }
      if (tid == 0) {
         a.iters[pid] = done ? it : -it;
         a.res[pid] = res;
      }
      __syncthreads();
   }
}

struct Config {
   int threads, lpr;
};
constexpr Config kConfigs[] = {{256, 1}, {256, 2}, {256, 4}, {256, 8}, {512, 1}, {512, 2},
                               {512, 4}, {512, 8}, {1024, 1}, {1024, 2}, {1024, 4}, {1024, 8}};
constexpr int kNumConfigs = sizeof(kConfigs) / sizeof(kConfigs[0]);

template <int NEN, int T, int L>
void launch_one(const BatchArgs& a, int blocks_per_sm, int nprob, cudaStream_t st)
{
   int occ = 0;
   OFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel<NEN, T, L>, T, 0));
   occ = std::max(1, blocks_per_sm > 0 ? std::min(occ, blocks_per_sm) : occ);
   const int grid = std::max(1, std::min(nprob, occ * num_sms()));
   batch_kernel<NEN, T, L><<<grid, T, 0, st>>>(a);
   count_launch();
}

template <int NEN>
void launch_cfg(int c, const BatchArgs& a, int blocks_per_sm, int nprob, cudaStream_t st)
{
   switch (c) {
      case 0: launch_one<NEN, 256, 1>(a, blocks_per_sm, nprob, st); break;
      case 1: launch_one<NEN, 256, 2>(a, blocks_per_sm, nprob, st); break;
      case 2: launch_one<NEN, 256, 4>(a, blocks_per_sm, nprob, st); break;
      case 3: launch_one<NEN, 256, 8>(a, blocks_per_sm, nprob, st); break;
      case 4: launch_one<NEN, 512, 1>(a, blocks_per_sm, nprob, st); break;
      case 5: launch_one<NEN, 512, 2>(a, blocks_per_sm, nprob, st); break;
      case 6: launch_one<NEN, 512, 4>(a, blocks_per_sm, nprob, st); break;
      case 7: launch_one<NEN, 512, 8>(a, blocks_per_sm, nprob, st); break;
      case 8: launch_one<NEN, 1024, 1>(a, blocks_per_sm, nprob, st); break;
      case 9: launch_one<NEN, 1024, 2>(a, blocks_per_sm, nprob, st); break;
      case 10: launch_one<NEN, 1024, 4>(a, blocks_per_sm, nprob, st); break;
      default: launch_one<NEN, 1024, 8>(a, blocks_per_sm, nprob, st); break;
   }
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
   ofg::DBuf<int32_t> elem, code, dof, color_elems, emap, row_ptr, col, dpos;
   ofg::DBuf<int64_t> color_ptr;
   ofg::DBuf<double> val, b, x, r, p, q, dinv, kel, f, bc, u, res;
   bool have_bc = false;
   int config = 2;  // index into kConfigs
   int blocks_per_sm = 0;
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   cudaStream_t capture = nullptr;
   int graph_config = -1;
   int max_it = 0;
   double tol = 0.0;
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
   a.probs = B->d_probs.p;
   a.order = B->order.p;
   a.queue = B->queue.p;
   a.coords = B->coords.p;
   a.elem = B->elem.p;
   a.code = B->code.p;
   a.dof = B->dof.p;
   a.color_ptr = B->color_ptr.p;
   a.color_elems = B->color_elems.p;
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
   return a;
}

// the queue reset and the persistent launch, as stream work
void enqueue(ofg_batch* B, int config, cudaStream_t st)
{
   OFG_CUDA(cudaMemsetAsync(B->queue.p, 0, sizeof(int), st));
   const BatchArgs a = args_of(B);
   if (B->nen == 3) launch_cfg<3>(config, a, B->blocks_per_sm, B->nprob, st);
   else launch_cfg<4>(config, a, B->blocks_per_sm, B->nprob, st);
   OFG_LAUNCH_CHECK();
}

// the same work through a CUDA graph, captured (on the batch's own capture
// stream) once per configuration and solver setting, launched on the
// library stream
void run_graph(ofg_batch* B)
{
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
         int64_t ncolor_tot = 0;
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
            P.color_base = ncolor_tot + p;
            P.nn = (int32_t)m->nn;
            P.ne = (int32_t)m->ne;
            P.n = (int32_t)mats[p]->n;
            P.ncolors = (int32_t)m->color_ptr.size() - 1;
            B->probs.push_back(P);
            B->nn += m->nn;
            B->ne += m->ne;
            B->nrows += mats[p]->n;
            B->nnz += mats[p]->nnz;
            ncolor_tot += P.ncolors;
            ensure_dpos(mats[p]);
            OFG_REQUIRE(mats[p]->dpos_complete, OFG_ERR_PIVOT, "a row has no diagonal entry");
         }
         OFG_REQUIRE(B->nnz < INT32_MAX, OFG_ERR_SIZE, "batch nonzeros must be below 2^31");
         const int nen = B->nen, dim = B->dim;
         B->coords.alloc(B->nn * dim);
         B->elem.alloc(B->ne * nen);
         B->code.alloc(B->nn);
         B->dof.alloc(B->nn);
         B->color_elems.alloc(B->ne);
         B->emap.alloc(B->ne * nen * nen);
         B->row_ptr.alloc(B->nrows + nprob);
         B->col.alloc(B->nnz);
         B->dpos.alloc(B->nrows);
         std::vector<int64_t> cptr;
         for (int p = 0; p < nprob; ++p) {
            ofg_mesh* m = meshes[p];
            ofg_matrix* A = mats[p];
            const BatchProblem& P = B->probs[p];
            gather(B->coords, P.node_off * dim, m->coords.p, m->nn * dim);
            gather(B->elem, P.elem_off * nen, m->elem.p, m->ne * nen);
            gather(B->code, P.node_off, m->code.p, m->nn);
            gather(B->dof, P.node_off, m->dof.p, m->nn);
            gather(B->color_elems, P.elem_off, m->color_elems.p, m->ne);
            gather(B->emap, P.elem_off * nen * nen, A->emap.p, m->ne * nen * nen);
            gather(B->row_ptr, P.rp_off, A->row_ptr.p, A->n + 1);
            gather(B->col, P.nnz_off, A->col.p, A->nnz);
            gather(B->dpos, P.row_off, A->dpos.p, A->n);
            cptr.insert(cptr.end(), m->color_ptr.begin(), m->color_ptr.end());
         }
         B->color_ptr.alloc(cptr.size());
         B->color_ptr.upload(cptr.data(), cptr.size());
         OFG_CUDA(cudaStreamSynchronize(stream()));
         for (auto* A : mats) delete A;
         // longest problems first
         std::vector<int32_t> order(nprob);
         std::iota(order.begin(), order.end(), 0);
         std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
            const int64_t na = B->probs[a].ne, nb = B->probs[b].ne;
            return na > nb;
         });
         B->order.alloc(nprob);
         B->order.upload(order.data(), nprob);
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

// Measured autotuner: runs the whole batch once per launch shape (threads
// per block x lanes per CSR row) on the current inputs, keeps the fastest.
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
      for (int c = 0; c < kNumConfigs; ++c) {
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
      B->graph_config = -1;
      if (chosen) *chosen = best_c;
   });
}

int ofg_batch_set_config(ofg_batch* B, int config, int blocks_per_sm)
{
   return guarded("ofg_batch_set_config", [&] {
      OFG_REQUIRE(B && config >= 0 && config < kNumConfigs && blocks_per_sm >= 0, OFG_ERR_ARG,
                  "bad arguments");
      B->config = config;
      B->blocks_per_sm = blocks_per_sm;
      B->graph_config = -1;
   });
}

int ofg_batch_config_shape(int config, int* threads, int* lanes_per_row)
{
   return guarded("ofg_batch_config_shape", [&] {
      OFG_REQUIRE(config >= 0 && config < kNumConfigs, OFG_ERR_ARG, "bad configuration");
      if (threads) *threads = kConfigs[config].threads;
      if (lanes_per_row) *lanes_per_row = kConfigs[config].lpr;
   });
}

}  // extern "C"
