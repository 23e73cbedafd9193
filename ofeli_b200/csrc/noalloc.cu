// noalloc.cu -- a Jacobi-preconditioned CG that allocates no device memory.
//
// Some callers cannot call cudaMalloc once they are running: services that
// reserve their whole device-memory budget at start-up and forbid later
// driver allocations, or host frameworks that own the device allocator and
// hand the library only the buffers of one call.  ofg_cg_diag_noalloc serves
// them: the caller passes the CSR matrix and the vectors already on the
// device, and every scratch buffer the solve needs (the residual, direction
// and product vectors, the inverse diagonal, the reduction partials and the
// scalar state) lives in one file-scope __device__ array of fixed size,
// which each GPU that loads the library holds until the process exits.
//
// Limits and sharing: systems of at most kMaxRows rows (larger ones are
// rejected with OFG_ERR_SIZE before anything is launched).  All calls share
// the one array, so calls that overlap on the GPU (different streams, or
// host threads on one device) race and must be serialised by the caller.
// The array keeps the last call's contents; the parts that must start at
// zero (the reduction arrival counter) are cleared on every call.
//
// CUDA loads a library's device code and its __device__ arrays lazily, on
// first use, and that load takes device memory.  ofg_init(device) therefore
// does it up front for this file: it looks up the array's address (which
// places the array on the device) and queries every kernel here (which loads
// its code), with that device current.  A caller that must not allocate
// calls ofg_init for each device it uses before that phase begins, and
// before any stream capture.  Every call looks the address up again (a
// host-side table lookup once the code is loaded), so a context that was
// reset and rebuilt gets the array's new address.
#include <algorithm>
#include <cmath>

#include "internal.cuh"
#include "reduce.cuh"

namespace ofg {
namespace {

constexpr int64_t kMaxRows = 1 << 17;  // 131072 rows
constexpr int kMaxBlocks = 8 * 256;    // reduction partials cap (>= 8 blocks per SM)

struct NAState {
   double nrm, rho, rho_old, alpha, res;
   int it, done, result, bad;
};

// layout of the scratch: r, p, q, dinv (kMaxRows doubles each), partials
// (3 per block), the arrival counter, the state
constexpr size_t kVecBytes = sizeof(double) * kMaxRows;
constexpr size_t kPartialsOff = 4 * kVecBytes;
constexpr size_t kCounterOff = kPartialsOff + sizeof(double) * 3 * kMaxBlocks;
constexpr size_t kStateOff = kCounterOff + 256;
constexpr size_t kScratchBytes = kStateOff + 256;

__device__ __align__(256) unsigned char g_cg_scratch[kScratchBytes];

// device address of g_cg_scratch on the current device (in host code the
// symbol is only a stand-in for the device array, never a device address)
unsigned char* scratch_address()
{
   void* p = nullptr;
   OFG_CUDA(cudaGetSymbolAddress(&p, g_cg_scratch));
   return static_cast<unsigned char*>(p);
}

// 8 lanes per row on CSR; lane 0 of each group owns the row's result
template <class RowOp>
__device__ __forceinline__ void csr_rows8(int64_t n, const int32_t* __restrict__ rp,
                                          const int32_t* __restrict__ col,
                                          const double* __restrict__ val,
                                          const double* __restrict__ x, RowOp op)
{
   const int lane = threadIdx.x & 31;
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t base = warp * 4; base < n; base += nwarps * 4) {
      const int64_t row = base + (lane >> 3);
      double acc = 0.0;
      if (row < n)
         for (int32_t k = rp[row] + (lane & 7); k < rp[row + 1]; k += 8) acc += val[k] * x[col[k]];
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (row < n && (lane & 7) == 0) op(row, acc);
   }
}

// r = b - A x, dinv, ||b||, ||r||, (r, D r); flags a zero or missing diagonal
__global__ void __launch_bounds__(kRedBlock) na_init(int64_t n, const int32_t* rp,
                                                     const int32_t* col, const double* val,
                                                     const double* b, const double* x, double* r,
                                                     double* dinv, NAState* S, double* partials,
                                                     unsigned* counter, double tol)
{
   double v[3] = {0.0, 0.0, 0.0};
   int bad = 0;
   csr_rows8(n, rp, col, val, x, [&](int64_t row, double ax) {
      double d = 0.0;
      for (int32_t k = rp[row]; k < rp[row + 1]; ++k)
         if (col[k] == (int32_t)row) d = val[k];
      if (!(fabs(d) > 0.0)) bad = 1;  // zero, missing or NaN
      const double di = 1.0 / d, bi = b[row], ri = bi - ax;
      dinv[row] = di;
      r[row] = ri;
      v[0] += bi * bi;
      v[1] += ri * ri;
      v[2] += ri * (ri * di);
   });
   if (bad) atomicOr(&S->bad, 1);
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

__global__ void __launch_bounds__(kRedBlock) na_direction(int64_t n, const double* r,
                                                          const double* dinv, double* p,
                                                          const NAState* S)
{
   if (S->done) return;
   const bool first = S->it == 0;
   const double beta = first ? 0.0 : S->rho / S->rho_old;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double zi = r[i] * dinv[i];
      p[i] = first ? zi : zi + beta * p[i];
   }
}

__global__ void __launch_bounds__(kRedBlock) na_spmv(int64_t n, const int32_t* rp,
                                                     const int32_t* col, const double* val,
                                                     const double* p, double* q, NAState* S,
                                                     double* partials, unsigned* counter)
{
   if (S->done) return;
   double v[1] = {0.0};
   csr_rows8(n, rp, col, val, p, [&](int64_t row, double ap) {
      q[row] = ap;
      v[0] += p[row] * ap;
   });
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t)) S->alpha = S->rho / t[0];
}

__global__ void __launch_bounds__(kRedBlock) na_update(int64_t n, double* x, const double* p,
                                                       double* r, const double* q,
                                                       const double* dinv, NAState* S,
                                                       double* partials, unsigned* counter,
                                                       double tol, int max_it)
{
   if (S->done) return;
   const double a = S->alpha;
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      x[i] += a * p[i];
      const double ri = r[i] - a * q[i];
      r[i] = ri;
      v[0] += ri * ri;
      v[1] += ri * (ri * dinv[i]);
   }
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      const double res = sqrt(t[0]) / S->nrm;
      const int it = S->it + 1;
      S->it = it;
      S->res = res;
      if (res <= tol) {
         S->done = 1;
         S->result = it;
      }
      else if (it >= max_it) {
         S->done = 1;
         S->result = -(max_it + 1);
      }
      S->rho_old = S->rho;
      S->rho = t[1];
   }
}

}  // namespace

// Loads this file's device code and places g_cg_scratch on the current
// device, so that later calls of ofg_cg_diag_noalloc take no device memory.
void noalloc_prepare()
{
   scratch_address();
   cudaFuncAttributes fa;
   OFG_CUDA(cudaFuncGetAttributes(&fa, na_init));
   OFG_CUDA(cudaFuncGetAttributes(&fa, na_direction));
   OFG_CUDA(cudaFuncGetAttributes(&fa, na_spmv));
   OFG_CUDA(cudaFuncGetAttributes(&fa, na_update));
}

}  // namespace ofg

using namespace ofg;

extern "C" int ofg_cg_diag_noalloc(int64_t n, const int32_t* row_ptr, const int32_t* col,
                                   const double* val, const double* b, double* x, int max_it,
                                   double toler, int* result, double* res)
{
   return guarded("ofg_cg_diag_noalloc", [&] {
      OFG_REQUIRE(row_ptr && col && val && b && x && result, OFG_ERR_ARG, "null argument");
      OFG_REQUIRE(n >= 1, OFG_ERR_ARG, "need at least one row");
      OFG_REQUIRE(n <= kMaxRows, OFG_ERR_SIZE,
                  "ofg_cg_diag_noalloc handles at most 131072 rows (its scratch is a fixed "
                  "device array); use ofg_cg for larger systems");
      OFG_REQUIRE(is_device_ptr(row_ptr) && is_device_ptr(col) && is_device_ptr(val) &&
                     is_device_ptr(b) && is_device_ptr(x),
                  OFG_ERR_ARG, "all arrays must be device memory (nothing is staged)");
      unsigned char* base = scratch_address();
      double* r = reinterpret_cast<double*>(base);
      double* p = reinterpret_cast<double*>(base + kVecBytes);
      double* q = reinterpret_cast<double*>(base + 2 * kVecBytes);
      double* dinv = reinterpret_cast<double*>(base + 3 * kVecBytes);
      double* partials = reinterpret_cast<double*>(base + kPartialsOff);
      unsigned* counter = reinterpret_cast<unsigned*>(base + kCounterOff);
      NAState* S = reinterpret_cast<NAState*>(base + kStateOff);
      cudaStream_t st = stream();
      OFG_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), st));
      OFG_CUDA(cudaMemsetAsync(&S->bad, 0, sizeof(int), st));
      const unsigned g = std::min<unsigned>(grid_for(n, kRedBlock, 8), kMaxBlocks);
      const unsigned gs = std::min<unsigned>(grid_for(n * 8, kRedBlock, 8), kMaxBlocks);
      na_init<<<gs, kRedBlock, 0, st>>>(n, row_ptr, col, val, b, x, r, dinv, S, partials, counter,
                                        toler);
      count_launch();
      OFG_LAUNCH_CHECK();
      NAState h{};
      OFG_CUDA(cudaMemcpyAsync(&h, S, sizeof(NAState), cudaMemcpyDeviceToHost, st));
      OFG_CUDA(cudaStreamSynchronize(st));
      OFG_REQUIRE(!h.bad, OFG_ERR_PIVOT, "zero or missing diagonal entry");
      int batch = 4;
      while (!h.done) {
         if (max_it <= 0) {
            h.result = -(max_it + 1);
            break;
         }
         for (int k = 0; k < batch; ++k) {
            na_direction<<<g, kRedBlock, 0, st>>>(n, r, dinv, p, S);
            na_spmv<<<gs, kRedBlock, 0, st>>>(n, row_ptr, col, val, p, q, S, partials, counter);
            na_update<<<g, kRedBlock, 0, st>>>(n, x, p, r, q, dinv, S, partials, counter, toler,
                                               max_it);
            count_launch(3);
         }
         OFG_LAUNCH_CHECK();
         OFG_CUDA(cudaMemcpyAsync(&h, S, sizeof(NAState), cudaMemcpyDeviceToHost, st));
         OFG_CUDA(cudaStreamSynchronize(st));
         batch = std::min(batch * 2, 64);
      }
      *result = h.result;
      if (res) *res = h.res;
   });
}
