// entries.cu -- SpMatrix's entry-level API on the device matrix:
//   SpMatrix::TMult (y += A^T x), SpMatrix::set(i,j,v) / add(i,j,v) in
//   batches.
//
// TMult (include/linear_algebra/SpMatrix_impl.h:760-767) accumulates
// y[col] += a * x[row] over the rows in ascending order, into y as given.
// OFELI's loop reads the column of the entry before the one it multiplies
// (col_ind[row_ptr[i] + j - 1], out of bounds at the first entry) and uses
// that 1-based column as a 0-based index; the intended product is
// implemented: a column-major copy of the pattern (built once per matrix,
// each column's entries in ascending row) lets one thread own each y entry
// and add its products in OFELI's row order, product and sum rounded
// separately as OFELI's loop does, so the result is the loop's bit for bit.
//
// set / add (SpMatrix_impl.h:785-802, _col_index :1009-1015) look an entry
// up by a linear search of its row and assign or add.  A batch is applied in
// its order by one device thread (entry edits are few: boundary terms,
// penalties); a pair outside the pattern stops the batch with OFG_ERR_ARG
// after the entries before it (OFELI's set throws there; its add writes
// into the previous row's last entry instead).
//
// The diagonal solve x_i = b_i / a_ii is the explicit step of TimeStepping's
// forward Euler scheme (src/solvers/TimeStepping.cpp:428-441: b(i) /=
// D(i), D the assembled diagonal of the scaled capacity), one correctly
// rounded division per row.
#include "internal.cuh"

namespace ofg {
namespace {

__global__ void col_count(int64_t nnz, const int32_t* __restrict__ col, int64_t* cnt)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride)
      atomicAdd(reinterpret_cast<unsigned long long*>(cnt + col[k]), 1ull);
}

__global__ void col_fill(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                         const int64_t* __restrict__ tp, int32_t* cursor, int32_t* trow,
                         int32_t* tpos)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t c = col[k];
         const int64_t slot = tp[c] + atomicAdd(cursor + c, 1);
         trow[slot] = (int32_t)i;
         tpos[slot] = k;
      }
}

// each column's entries into ascending row (insertion sort; columns of FEM
// patterns hold a few dozen entries)
__global__ void col_sort(int64_t n, const int64_t* __restrict__ tp, int32_t* trow, int32_t* tpos)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
      const int64_t b = tp[c], e = tp[c + 1];
      for (int64_t s = b + 1; s < e; ++s) {
         const int32_t r = trow[s], p = tpos[s];
         int64_t t = s - 1;
         while (t >= b && trow[t] > r) {
            trow[t + 1] = trow[t];
            tpos[t + 1] = tpos[t];
            --t;
         }
         trow[t + 1] = r;
         tpos[t + 1] = p;
      }
   }
}

__global__ void spmv_t_add(int64_t n, const int64_t* __restrict__ tp, const int32_t* __restrict__ trow,
                           const int32_t* __restrict__ tpos, const double* __restrict__ a,
                           const double* __restrict__ x, double* y)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
      double acc = y[c];
      for (int64_t s = tp[c]; s < tp[c + 1]; ++s)
         acc = __dadd_rn(acc, __dmul_rn(a[tpos[s]], x[trow[s]]));
      y[c] = acc;
   }
}

__global__ void apply_entries(int64_t count, const int64_t* __restrict__ ii,
                              const int64_t* __restrict__ jj, const double* __restrict__ v, int set,
                              int64_t n, const int32_t* __restrict__ rp,
                              const int32_t* __restrict__ col, double* a, int64_t* bad)
{
   if (blockIdx.x != 0 || threadIdx.x != 0) return;
   for (int64_t e = 0; e < count; ++e) {
      const int64_t i = ii[e], j = jj[e];
      if (i < 1 || i > n || j < 1 || j > n) {
         *bad = e;
         return;
      }
      int64_t found = -1;
      for (int32_t k = rp[i - 1]; k < rp[i]; ++k)
         if (col[k] == j - 1) {
            found = k;
            break;
         }
      if (found < 0) {
         *bad = e;
         return;
      }
      a[found] = set ? v[e] : __dadd_rn(a[found], v[e]);
   }
}

void ensure_transpose(ofg_matrix* A)
{
   if (A->t_ready) return;
   const int64_t n = A->n, nnz = A->nnz;
   DBuf<int64_t> cnt(n + 1);
   cnt.zero();
   A->t_ptr.alloc(n + 1);
   A->t_row.alloc(nnz > 0 ? nnz : 1);
   A->t_pos.alloc(nnz > 0 ? nnz : 1);
   if (nnz) {
      col_count<<<grid_for(nnz, 256), 256, 0, stream()>>>(nnz, A->col.p, cnt.p);
      count_launch();
   }
   scan_exclusive_i64(cnt.p, A->t_ptr.p, n + 1);
   DBuf<int32_t> cursor(n > 0 ? n : 1);
   cursor.zero();
   if (n) {
      col_fill<<<grid_for(n, 256), 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p, A->t_ptr.p,
                                                        cursor.p, A->t_row.p, A->t_pos.p);
      col_sort<<<grid_for(n, 256), 256, 0, stream()>>>(n, A->t_ptr.p, A->t_row.p, A->t_pos.p);
      count_launch(2);
   }
   OFG_LAUNCH_CHECK();
   OFG_CUDA(cudaStreamSynchronize(stream()));
   A->t_ready = true;
}

// x_i = b_i / a_ii; *bad = lowest row without a nonzero diagonal entry
__global__ void diag_divide(int64_t n, const int32_t* __restrict__ dpos,
                            const double* __restrict__ val, const double* __restrict__ b, double* x,
                            int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const int32_t d = dpos[i];
      const double a = d >= 0 ? val[d] : 0.0;
      if (a == 0.0) atomicMin(bad, (int)i);
      x[i] = b[i] / a;
   }
}

}  // namespace
}  // namespace ofg

using namespace ofg;

extern "C" {

int ofg_spmv_transpose_add(ofg_matrix* A, const double* x, double* y)
{
   return guarded("ofg_spmv_transpose_add", [&] {
      OFG_REQUIRE(A && x && y, OFG_ERR_ARG, "null argument");
      ensure_transpose(A);
      In<double> dx(x, A->n);
      InOut<double> dy(y, A->n, true);
      if (A->n) {
         spmv_t_add<<<grid_for(A->n, 256), 256, 0, stream()>>>(A->n, A->t_ptr.p, A->t_row.p,
                                                                A->t_pos.p, A->val.p, dx.d, dy.d);
         count_launch();
         OFG_LAUNCH_CHECK();
      }
      dy.finish();
   });
}

int ofg_matrix_edit(ofg_matrix* A, int64_t count, const int64_t* i, const int64_t* j,
                    const double* v, int set)
{
   return guarded("ofg_matrix_edit", [&] {
      OFG_REQUIRE(A && count >= 0 && (count == 0 || (i && j && v)), OFG_ERR_ARG, "bad arguments");
      if (!count) return;
      In<int64_t> di(i, count), dj(j, count);
      In<double> dv(v, count);
      DBuf<int64_t> bad(1);
      const int64_t none = -1;
      bad.upload(&none, 1);
      apply_entries<<<1, 32, 0, stream()>>>(count, di.d, dj.d, dv.d, set ? 1 : 0, A->n,
                                             A->row_ptr.p, A->col.p, A->val.p, bad.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      matrix_touch(A);
      int64_t h = -1;
      bad.download(&h, 1);
      if (h >= 0) {
         int64_t hi = 0, hj = 0;
         OFG_CUDA(cudaMemcpy(&hi, di.d + h, sizeof(int64_t), cudaMemcpyDefault));
         OFG_CUDA(cudaMemcpy(&hj, dj.d + h, sizeof(int64_t), cudaMemcpyDefault));
         throw Error(OFG_ERR_ARG, "Index pair (" + std::to_string(hi) + "," + std::to_string(hj) +
                                      ") not compatible with sparse storage (entry " +
                                      std::to_string(h) + " of the batch)");
      }
   });
}

int ofg_matrix_diag_solve(ofg_matrix* A, const double* b, double* x)
{
   return guarded("ofg_matrix_diag_solve", [&] {
      OFG_REQUIRE(A && b && x, OFG_ERR_ARG, "null argument");
      const int64_t n = A->n;
      ensure_dpos(A);
      In<double> db(b, n);
      InOut<double> dx(x, n, false);
      DBuf<int> bad(1);
      int big = INT32_MAX;
      bad.upload(&big, 1);
      if (n) {
         diag_divide<<<grid_for(n, 256), 256, 0, stream()>>>(n, A->dpos.p, A->val.p, db.d, dx.d,
                                                            bad.p);
         count_launch();
         OFG_LAUNCH_CHECK();
      }
      int h = 0;
      bad.download(&h, 1);
      OFG_REQUIRE(h == INT32_MAX, OFG_ERR_PIVOT,
                  "zero or missing diagonal entry in row " + std::to_string(h + 1));
      dx.finish();
   });
}

}  // extern "C"
