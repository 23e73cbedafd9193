// matrix.cu -- the device CSR matrix behind OFELI's SpMatrix<real_t>: pattern
// import/export in OFELI's layout, values, SELL-32 copy and the SpMV kernels.
//
// SpMV is memory bound: 12*nnz + 20*n bytes per FP64 product with int32
// column indices (values 8 B + column 4 B per entry, row pointer 4 B, x read
// and y written once per row).  Two kernels:
//   * spmv_sell_kernel: one thread per row over SELL-32 slices; every load of
//     a warp is one contiguous, 256-byte aligned line of values (128 B of
//     columns), so the matrix streams at full width; x gathers hit L2.
//   * spmv_csr_vec_kernel: L lanes per row straight on CSR (L = the power of
//     two covering the mean row length), used where no SELL copy exists.
#include <cuda_bf16.h>

#include <cstdint>
#include <vector>

#include "internal.cuh"

namespace ofg {

// --------------------------------------------------------------- scans ----
namespace {
constexpr int kScanBlock = 1024;

__global__ void scan_block_sums(const int64_t* in, int64_t* out, int64_t* sums, int64_t n)
{
   __shared__ int64_t sh[kScanBlock];
   int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
   int64_t v = i < n ? in[i] : 0;
   sh[threadIdx.x] = v;
   __syncthreads();
   for (int o = 1; o < kScanBlock; o <<= 1) {
      int64_t t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
   }
   if (i < n) out[i] = sh[threadIdx.x] - v;  // exclusive within the block
   if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = sh[threadIdx.x];
}

__global__ void scan_add_offsets(int64_t* out, const int64_t* offs, int64_t n)
{
   int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
   if (i < n) out[i] += offs[blockIdx.x];
}
}  // namespace

// out[i] = sum_{j<i} in[i]; recursion over block sums.
void scan_exclusive_i64(const int64_t* d_in, int64_t* d_out, int64_t n)
{
   if (n <= 0) return;
   int64_t nb = (n + kScanBlock - 1) / kScanBlock;
   DBuf<int64_t> sums(nb), offs(nb);
   scan_block_sums<<<(unsigned)nb, kScanBlock, 0, stream()>>>(d_in, d_out, sums.p, n);
   count_launch();
   OFG_LAUNCH_CHECK();
   if (nb > 1) {
      scan_exclusive_i64(sums.p, offs.p, nb);
      scan_add_offsets<<<(unsigned)nb, kScanBlock, 0, stream()>>>(d_out, offs.p, n);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
}

// -------------------------------------------------------- pattern import --
namespace {
__global__ void import_pattern(int64_t n, int64_t nnz, const int64_t* rp, const int64_t* ci,
                               int32_t* rp32, int32_t* col32, int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) {
      int64_t v = rp[i];
      if (v < 0 || v > nnz || (i == 0 && v != 0) || (i == n && v != nnz) ||
          (i < n && rp[i + 1] < v))
         atomicOr(bad, 1);
      rp32[i] = (int32_t)v;
   }
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
      int64_t c = ci[k];
      if (c < 1 || c > n) atomicOr(bad, 2);
      col32[k] = (int32_t)(c - 1);
   }
}

__global__ void export_pattern(int64_t n, int64_t nnz, const int32_t* rp32, const int32_t* col32,
                               int64_t* rp, int64_t* ci)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride)
      rp[i] = rp32[i];
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride)
      ci[k] = (int64_t)col32[k] + 1;
}

__global__ void find_diag(int64_t n, const int32_t* rp, const int32_t* col, int32_t* dpos,
                          int* missing)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      int32_t d = -1;
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
         if (col[k] == (int32_t)i) d = k;
      dpos[i] = d;
      if (d < 0) atomicOr(missing, 1);
   }
}

// ------------------------------------------------------------- SELL-32 --
__global__ void sell_widths(int64_t n, int64_t nslices, const int32_t* rp, int64_t* width32)
{
   int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   int lane = threadIdx.x & 31;
   if (s >= nslices) return;
   int64_t r = s * 32 + lane;
   int len = r < n ? rp[r + 1] - rp[r] : 0;
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
   if (lane == 0) width32[s] = (int64_t)len * 32;
}

__global__ void sell_fill(int64_t n, int64_t nslices, const int32_t* rp, const int32_t* col,
                          const int64_t* sp64, int32_t* sp, int32_t* scol, int32_t* ssrc)
{
   int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= nslices * 32) return;
   int64_t s = r >> 5;
   int lane = (int)(r & 31);
   int64_t beg = sp64[s], w = (sp64[s + 1] - beg) / 32;
   if (lane == 0) sp[s] = (int32_t)beg;
   if (r == nslices * 32 - 1) sp[nslices] = (int32_t)sp64[nslices];
   int len = r < n ? rp[r + 1] - rp[r] : 0;
   int32_t pad = r < n ? (int32_t)r : 0;
   for (int64_t k = 0; k < w; ++k) {
      int64_t idx = beg + k * 32 + lane;
      if (k < len) {
         scol[idx] = col[rp[r] + k];
         ssrc[idx] = rp[r] + (int32_t)k;
      }
      else {
         scol[idx] = pad;
         ssrc[idx] = -1;
      }
   }
}

template <class T>
__global__ void sell_values(int64_t total, const int32_t* ssrc, const double* val, T* sval)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
      int32_t s = ssrc[i];
      sval[i] = s >= 0 ? (T)val[s] : (T)0;
   }
}

// both SELL copies (FP64 and FP32) from one gather of the CSR values
__global__ void sell_values_both(int64_t total, const int32_t* ssrc, const double* val,
                                 double* sval, float* sval32)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
      const int32_t s = ssrc[i];
      const double v = s >= 0 ? val[s] : 0.0;
      sval[i] = v;
      sval32[i] = (float)v;
   }
}

__global__ void sell_values_bf16(int64_t total, const int32_t* ssrc, const double* val,
                                 uint16_t* sval)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
      int32_t s = ssrc[i];
      const __nv_bfloat16 v = __float2bfloat16(s >= 0 ? (float)val[s] : 0.0f);
      sval[i] = *reinterpret_cast<const uint16_t*>(&v);
   }
}

// column - row of every entry of SELL row r (0 for padding; padding rows of
// the last slice point at themselves), flagging any offset beyond 16 bits
__global__ void sell_offsets16(int64_t nslices, const int32_t* sp, const int32_t* scol,
                               const int32_t* ssrc, int16_t* d16, int* wide)
{
   int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= nslices * 32) return;
   const int64_t s = r >> 5;
   const int lane = (int)(r & 31);
   const int64_t beg = sp[s], w = (sp[s + 1] - beg) / 32;
   for (int64_t k = 0; k < w; ++k) {
      const int64_t idx = beg + k * 32 + lane;
      const int64_t d = ssrc[idx] >= 0 ? (int64_t)scol[idx] - r : 0;
      if (d > 32767 || d < -32768) atomicOr(wide, 1);
      d16[idx] = (int16_t)d;
   }
}

// one warp per slice: the slice's width w when all 32 rows have the same
// 16-bit offset at every position k, else -1; counts the nonzeros of the
// uniform slices
__global__ void sell_uniform_scan(int64_t nslices, const int32_t* __restrict__ sp,
                                  const int16_t* __restrict__ d16,
                                  const int32_t* __restrict__ ssrc, int32_t* width,
                                  unsigned long long* uni_nnz)
{
   const int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int lane = threadIdx.x & 31;
   if (s >= nslices) return;  // the whole warp shares s
   const int64_t beg = sp[s];
   const int w = (int)((sp[s + 1] - beg) >> 5);
   bool uni = true;
   int real = 0;
   for (int k = 0; k < w; ++k) {
      const int64_t idx = beg + (int64_t)k * 32 + lane;
      const int16_t d = d16[idx];
      const bool same = __all_sync(0xffffffffu, d == __shfl_sync(0xffffffffu, d, 0));
      uni = uni && same;
      real += ssrc[idx] >= 0 ? 1 : 0;
   }
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) real += __shfl_xor_sync(0xffffffffu, real, o);
   if (lane == 0) {
      width[s] = uni ? w : -1;
      if (uni) atomicAdd(uni_nnz, (unsigned long long)real);
   }
}

// the uniform slices' offsets, one per position k
__global__ void sell_uniform_fill(int64_t nslices, const int32_t* __restrict__ sp,
                                  const int16_t* __restrict__ d16,
                                  const int32_t* __restrict__ uni, int16_t* tab)
{
   const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (s >= nslices || uni[s] < 0) return;
   const int64_t beg = sp[s];
   const int w = (int)((sp[s + 1] - beg) >> 5);
   for (int k = 0; k < w; ++k) tab[uni[s] + k] = d16[beg + (int64_t)k * 32];
}

// ------------------------------------------------------------------ SpMV --
template <bool ADD>
__global__ void __launch_bounds__(256, 8) spmv_sell_kernel(int64_t n, int64_t nslices,
                                                        const int32_t* __restrict__ sp,
                                                        const int32_t* __restrict__ scol,
                                                        const double* __restrict__ sval,
                                                        const double* __restrict__ x,
                                                        double* __restrict__ y, const int* skip,
                                                        int* worked)
{
   if (skip && *skip) return;
   prof_mark(worked);
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nslices * 32; r += stride) {
      int64_t s = r >> 5;
      int lane = (int)(r & 31);
      int32_t beg = sp[s], end = sp[s + 1];
      double acc = 0.0;
      for (int32_t k = beg + lane; k < end; k += 32) acc += sval[k] * __ldg(x + scol[k]);
      if (r < n) y[r] = ADD ? y[r] + acc : acc;
   }
}

// ---------------------------------------------------- FP32 SELL variants --
// y = A x with FP32 values and vectors, four thread-to-row mappings over the
// same SELL-32 arrays:
//   kind 0: one row per thread (a warp = one slice, 128-byte lines);
//   kind 1: four adjacent rows per thread, float4/int4 loads;
//   kind 2: four rows per thread taken from four consecutive slices (one
//           row per slice, scalar loads, four independent chains);
//   kind 3: two adjacent rows per thread, float2/int2 loads.
// y and x must hold nslices*32 entries (padding rows produce 0).
__global__ void __launch_bounds__(256) spmv32_row(int64_t nslices, const int32_t* __restrict__ sp,
                                                  const int32_t* __restrict__ scol,
                                                  const float* __restrict__ sval,
                                                  const float* __restrict__ x, float* __restrict__ y)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nslices * 32; r += stride) {
      const int64_t s = r >> 5;
      const int lane = (int)(r & 31);
      const int32_t beg = sp[s], end = sp[s + 1];
      float acc = 0.f;
#pragma unroll 8
      for (int32_t k = beg + lane; k < end; k += 32) acc += sval[k] * __ldg(x + scol[k]);
      y[r] = acc;
   }
}

__global__ void __launch_bounds__(256) spmv32_vec4(int64_t nslices, const int32_t* __restrict__ sp,
                                                   const int32_t* __restrict__ scol,
                                                   const float* __restrict__ sval,
                                                   const float* __restrict__ x,
                                                   float* __restrict__ y)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nslices * 8; t += stride) {
      const int64_t r0 = t * 4, s = r0 >> 5;
      const int32_t beg = sp[s], w = (sp[s + 1] - beg) >> 5;
      const int32_t* cp = scol + beg + (r0 & 31);
      const float* vp = sval + beg + (r0 & 31);
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 8
      for (int32_t k = 0; k < w; ++k) {
         const int4 c = *reinterpret_cast<const int4*>(cp + k * 32);
         const float4 a = *reinterpret_cast<const float4*>(vp + k * 32);
         acc.x += a.x * __ldg(x + c.x);
         acc.y += a.y * __ldg(x + c.y);
         acc.z += a.z * __ldg(x + c.z);
         acc.w += a.w * __ldg(x + c.w);
      }
      *reinterpret_cast<float4*>(y + r0) = acc;
   }
}

__global__ void __launch_bounds__(256) spmv32_slices4(int64_t nslices,
                                                      const int32_t* __restrict__ sp,
                                                      const int32_t* __restrict__ scol,
                                                      const float* __restrict__ sval,
                                                      const float* __restrict__ x,
                                                      float* __restrict__ y)
{
   // warp w owns slices 4w .. 4w+3; lane l owns row l of each
   const int lane = threadIdx.x & 31;
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t s4 = warp * 4; s4 < nslices; s4 += nw * 4) {
      int32_t beg[4], w[4];
      float acc[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
         const int64_t s = min(s4 + q, nslices - 1);
         beg[q] = sp[s];
         w[q] = s4 + q < nslices ? (sp[s + 1] - beg[q]) >> 5 : 0;
         acc[q] = 0.f;
      }
      const int32_t wmax = max(max(w[0], w[1]), max(w[2], w[3]));
      for (int32_t k = 0; k < wmax; ++k) {
#pragma unroll
         for (int q = 0; q < 4; ++q)
            if (k < w[q]) {
               const int32_t idx = beg[q] + k * 32 + lane;
               acc[q] += sval[idx] * __ldg(x + scol[idx]);
            }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
         if (s4 + q < nslices) y[(s4 + q) * 32 + lane] = acc[q];
   }
}

__global__ void __launch_bounds__(256) spmv32_vec2(int64_t nslices, const int32_t* __restrict__ sp,
                                                   const int32_t* __restrict__ scol,
                                                   const float* __restrict__ sval,
                                                   const float* __restrict__ x,
                                                   float* __restrict__ y)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nslices * 16; t += stride) {
      const int64_t r0 = t * 2, s = r0 >> 5;
      const int32_t beg = sp[s], w = (sp[s + 1] - beg) >> 5;
      const int32_t* cp = scol + beg + (r0 & 31);
      const float* vp = sval + beg + (r0 & 31);
      float2 acc = make_float2(0.f, 0.f);
#pragma unroll 8
      for (int32_t k = 0; k < w; ++k) {
         const int2 c = *reinterpret_cast<const int2*>(cp + k * 32);
         const float2 a = *reinterpret_cast<const float2*>(vp + k * 32);
         acc.x += a.x * __ldg(x + c.x);
         acc.y += a.y * __ldg(x + c.y);
      }
      *reinterpret_cast<float2*>(y + r0) = acc;
   }
}

template <int L, bool ADD>
__global__ void __launch_bounds__(256) spmv_csr_vec_kernel(int64_t n, const int32_t* __restrict__ rp,
                                                           const int32_t* __restrict__ col,
                                                           const double* __restrict__ val,
                                                           const double* __restrict__ x,
                                                           double* __restrict__ y)
{
   constexpr int G = 32 / L;  // rows per warp
   int lane = threadIdx.x & 31;
   int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
   for (int64_t base = warp * G; base < n; base += nwarps * G) {
      int64_t row = base + lane / L;
      double acc = 0.0;
      if (row < n) {
         int32_t beg = rp[row], end = rp[row + 1];
         for (int32_t k = beg + (lane & (L - 1)); k < end; k += L) acc += val[k] * __ldg(x + col[k]);
      }
#pragma unroll
      for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (row < n && (lane & (L - 1)) == 0) y[row] = ADD ? y[row] + acc : acc;
   }
}

template <bool ADD>
void launch_csr_vec(const ofg_matrix* A, const double* x, double* y)
{
   int L = 32;
   while (L > 1 && L / 2 >= A->avg_row) L /= 2;
   if (L < 4) L = 4;
   unsigned grid = grid_for(A->n * L, 256, 16);
   switch (L) {
      case 4: spmv_csr_vec_kernel<4, ADD><<<grid, 256, 0, stream()>>>(A->n, A->row_ptr.p, A->col.p, A->val.p, x, y); break;
      case 8: spmv_csr_vec_kernel<8, ADD><<<grid, 256, 0, stream()>>>(A->n, A->row_ptr.p, A->col.p, A->val.p, x, y); break;
      case 16: spmv_csr_vec_kernel<16, ADD><<<grid, 256, 0, stream()>>>(A->n, A->row_ptr.p, A->col.p, A->val.p, x, y); break;
      default: spmv_csr_vec_kernel<32, ADD><<<grid, 256, 0, stream()>>>(A->n, A->row_ptr.p, A->col.p, A->val.p, x, y); break;
   }
   count_launch();
   OFG_LAUNCH_CHECK();
}

}  // namespace

void matrix_touch(ofg_matrix* A) { A->version++; }

void matrix_finish_pattern(ofg_matrix* A)
{
   std::vector<int32_t> rp = A->row_ptr.to_host(A->n + 1);
   int mx = 0;
   for (int64_t i = 0; i < A->n; ++i) mx = std::max(mx, rp[i + 1] - rp[i]);
   A->max_row = mx;
   A->avg_row = A->n ? double(A->nnz) / double(A->n) : 0.0;
}

void ensure_dpos(ofg_matrix* A)
{
   if (A->dpos_ready) return;
   A->dpos.alloc(A->n > 0 ? A->n : 1);
   DBuf<int> missing(1);
   missing.zero();
   if (A->n) {
      find_diag<<<grid_for(A->n, 256), 256, 0, stream()>>>(A->n, A->row_ptr.p, A->col.p, A->dpos.p,
                                                           missing.p);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
   int h = 0;
   missing.download(&h, 1);
   A->dpos_ready = true;
   A->dpos_complete = (h == 0);
}

void ensure_sell(ofg_matrix* A)
{
   if (!A->sell_ready) {
      A->nslices = (A->n + 31) / 32;
      DBuf<int64_t> w(A->nslices + 1), sp64(A->nslices + 1);
      w.zero();
      if (A->nslices) {
         sell_widths<<<(unsigned)((A->nslices * 32 + 255) / 256), 256, 0, stream()>>>(
            A->n, A->nslices, A->row_ptr.p, w.p);
         count_launch();
         OFG_LAUNCH_CHECK();
      }
      scan_exclusive_i64(w.p, sp64.p, A->nslices + 1);
      int64_t total = 0;
      OFG_CUDA(cudaMemcpyAsync(&total, sp64.p + A->nslices, sizeof(int64_t), cudaMemcpyDeviceToHost,
                               stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
      OFG_REQUIRE(total < (int64_t(1) << 31), OFG_ERR_PATTERN, "SELL copy exceeds 2^31 entries");
      A->sell_ptr.alloc(A->nslices + 1);
      A->sell_col.alloc(total > 0 ? total : 1);
      A->sell_src.alloc(total > 0 ? total : 1);
      if (total == 0) {
         // the one placeholder entry of an empty matrix is padding: the value
         // copies below read nothing through it
         OFG_CUDA(cudaMemsetAsync(A->sell_src.p, 0xFF, sizeof(int32_t), stream()));
         OFG_CUDA(cudaMemsetAsync(A->sell_col.p, 0, sizeof(int32_t), stream()));
      }
      if (A->nslices) {
         sell_fill<<<(unsigned)((A->nslices * 32 + 255) / 256), 256, 0, stream()>>>(
            A->n, A->nslices, A->row_ptr.p, A->col.p, sp64.p, A->sell_ptr.p, A->sell_col.p,
            A->sell_src.p);
         count_launch();
         OFG_LAUNCH_CHECK();
      }
      else {
         A->sell_ptr.zero();
      }
      A->sell_val.alloc(total > 0 ? total : 1);
      A->sell_ready = true;
      A->sell_version = 0;
      A->sell32_version = 0;
      OFG_CUDA(cudaStreamSynchronize(stream()));
   }
   if (A->sell_version != A->version) {
      int64_t total = A->sell_val.n;
      sell_values<double><<<grid_for(total, 256), 256, 0, stream()>>>(total, A->sell_src.p, A->val.p,
                                                                       A->sell_val.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      A->sell_version = A->version;
   }
}

void ensure_sell32(ofg_matrix* A)
{
   if (A->sell_ready && A->sell_version != A->version && A->sell_val32.n == A->sell_val.n) {
      // both copies stale (new values): one pass writes both
      const int64_t total = A->sell_val.n;
      sell_values_both<<<grid_for(total, 256), 256, 0, stream()>>>(total, A->sell_src.p, A->val.p,
                                                                   A->sell_val.p,
                                                                   A->sell_val32.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      A->sell_version = A->version;
      A->sell32_version = A->version;
      return;
   }
   ensure_sell(A);
   if (A->sell32_version != A->version || A->sell_val32.n != A->sell_val.n) {
      int64_t total = A->sell_val.n;
      A->sell_val32.reserve(total);
      sell_values<float><<<grid_for(total, 256), 256, 0, stream()>>>(total, A->sell_src.p, A->val.p,
                                                                      A->sell_val32.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      A->sell32_version = A->version;
   }
}

void ensure_sell_bf16(ofg_matrix* A)
{
   ensure_sell(A);
   if (A->sellbf_version != A->version || A->sell_valbf.n != A->sell_val.n) {
      int64_t total = A->sell_val.n;
      A->sell_valbf.reserve(total);
      sell_values_bf16<<<grid_for(total, 256), 256, 0, stream()>>>(total, A->sell_src.p, A->val.p,
                                                                   A->sell_valbf.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      A->sellbf_version = A->version;
   }
}

bool ensure_sell_d16(ofg_matrix* A)
{
   ensure_sell(A);
   if (A->idx16 < 0) {
      const int64_t total = A->sell_val.n;
      A->sell_d16.alloc(total);
      DBuf<int> wide(1);
      wide.zero();
      if (A->nslices) {
         sell_offsets16<<<(unsigned)((A->nslices * 32 + 255) / 256), 256, 0, stream()>>>(
            A->nslices, A->sell_ptr.p, A->sell_col.p, A->sell_src.p, A->sell_d16.p, wide.p);
         count_launch();
         OFG_LAUNCH_CHECK();
      }
      else {
         A->sell_d16.zero();
      }
      int h = 0;
      wide.download(&h, 1);
      A->idx16 = h ? 0 : 1;
      if (!A->idx16) A->sell_d16.release();
   }
   return A->idx16 == 1;
}

void ensure_sell_uniform(ofg_matrix* A)
{
   if (A->uni_ready) return;
   OFG_REQUIRE(A->idx16 == 1, OFG_ERR_ARG, "slice-uniform offsets need the 16-bit offsets");
   const int64_t ns = A->nslices;
   A->sell_uni.alloc(ns > 0 ? ns : 1);
   std::vector<int32_t> w((size_t)ns);
   unsigned long long hn = 0;
   if (ns > 0) {
      DBuf<unsigned long long> cnt(1);
      cnt.zero();
      sell_uniform_scan<<<(unsigned)((ns * 32 + 255) / 256), 256, 0, stream()>>>(
         ns, A->sell_ptr.p, A->sell_d16.p, A->sell_src.p, A->sell_uni.p, cnt.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      A->sell_uni.download(w.data(), (size_t)ns);
      cnt.download(&hn, 1);
   }
   // table positions: uniform slices in order, w offsets each
   int64_t pos = 0;
   for (int64_t s = 0; s < ns; ++s) {
      if (w[(size_t)s] < 0) continue;
      const int32_t ws = w[(size_t)s];
      w[(size_t)s] = (int32_t)pos;
      pos += ws;
   }
   OFG_REQUIRE(pos <= INT32_MAX, OFG_ERR_SIZE, "offset table too large");
   A->utab_len = pos;
   A->uni_nnz = (int64_t)hn;
   A->sell_utab.alloc(pos > 0 ? pos : 1);
   if (ns > 0) {
      A->sell_uni.upload(w.data(), (size_t)ns);
      sell_uniform_fill<<<(unsigned)((ns + 255) / 256), 256, 0, stream()>>>(
         ns, A->sell_ptr.p, A->sell_d16.p, A->sell_uni.p, A->sell_utab.p);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
   OFG_CUDA(cudaStreamSynchronize(stream()));
   A->uni_ready = true;
}

void spmv_csr(const ofg_matrix* A, const double* x, double* y, bool add)
{
   if (!A->n) return;
   if (add) launch_csr_vec<true>(A, x, y);
   else launch_csr_vec<false>(A, x, y);
}

void spmv_sell(const ofg_matrix* A, const double* x, double* y, const int* skip)
{
   if (!A->n) return;
   int* worked = prof_begin();
   spmv_sell_kernel<false><<<grid_for(A->nslices * 32, 256, 8), 256, 0, stream()>>>(
      A->n, A->nslices, A->sell_ptr.p, A->sell_col.p, A->sell_val.p, x, y, skip, worked);
   prof_end(PROF_SPMV64, 12.0 * A->nnz + 20.0 * A->n + 4.0);
   count_launch();
   OFG_LAUNCH_CHECK();
}

}  // namespace ofg

using namespace ofg;

namespace {
void finish_create(ofg_matrix* A, const int* bad_dev)
{
   int bad = 0;
   OFG_CUDA(cudaMemcpyAsync(&bad, bad_dev, sizeof(int), cudaMemcpyDeviceToHost, stream()));
   OFG_CUDA(cudaStreamSynchronize(stream()));
   OFG_REQUIRE(!(bad & 1), OFG_ERR_ARG, "row_ptr is not a valid 0-based CSR row pointer");
   OFG_REQUIRE(!(bad & 2), OFG_ERR_ARG, "col_ind entry outside [1, n]");
   matrix_finish_pattern(A);
}
}  // namespace

extern "C" {

int ofg_matrix_create(int64_t n, int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                      ofg_matrix** out)
{
   return guarded("ofg_matrix_create", [&] {
      OFG_REQUIRE(out && row_ptr && (col_ind || nnz == 0) && n >= 0 && nnz >= 0, OFG_ERR_ARG,
                  "null argument or negative size");
      OFG_REQUIRE(nnz < (int64_t(1) << 31) && n < (int64_t(1) << 31), OFG_ERR_PATTERN,
                  "n and nnz must be below 2^31");
      auto A = new ofg_matrix();
      try {
         A->n = n;
         A->nnz = nnz;
         A->row_ptr.alloc(n + 1);
         A->col.alloc(nnz > 0 ? nnz : 1);
         A->val.alloc(nnz > 0 ? nnz : 1);
         A->val.zero();
         In<int64_t> rp(row_ptr, n + 1), ci(col_ind, nnz);
         DBuf<int> bad(1);
         bad.zero();
         import_pattern<<<grid_for(std::max(n + 1, nnz), 256), 256, 0, stream()>>>(
            n, nnz, rp.d, ci.d, A->row_ptr.p, A->col.p, bad.p);
         count_launch();
         OFG_LAUNCH_CHECK();
         finish_create(A, bad.p);
      }
      catch (...) {
         delete A;
         throw;
      }
      *out = A;
   });
}

int ofg_matrix_destroy(ofg_matrix* A)
{
   return guarded("ofg_matrix_destroy", [&] {
      delete A;
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_matrix_info(const ofg_matrix* A, int64_t* n, int64_t* nnz)
{
   return guarded("ofg_matrix_info", [&] {
      OFG_REQUIRE(A, OFG_ERR_ARG, "null matrix");
      if (n) *n = A->n;
      if (nnz) *nnz = A->nnz;
   });
}

int ofg_matrix_get_pattern(const ofg_matrix* A, int64_t* row_ptr, int64_t* col_ind)
{
   return guarded("ofg_matrix_get_pattern", [&] {
      OFG_REQUIRE(A && row_ptr && col_ind, OFG_ERR_ARG, "null argument");
      InOut<int64_t> rp(row_ptr, A->n + 1, false), ci(col_ind, A->nnz, false);
      export_pattern<<<grid_for(std::max(A->n + 1, A->nnz), 256), 256, 0, stream()>>>(
         A->n, A->nnz, A->row_ptr.p, A->col.p, rp.d, ci.d);
      count_launch();
      OFG_LAUNCH_CHECK();
      rp.finish();
      ci.finish();
   });
}

int ofg_matrix_set_values(ofg_matrix* A, const double* a)
{
   return guarded("ofg_matrix_set_values", [&] {
      OFG_REQUIRE(A && (a || A->nnz == 0), OFG_ERR_ARG, "null argument");
      if (A->nnz)
         OFG_CUDA(cudaMemcpyAsync(A->val.p, a, A->nnz * sizeof(double), cudaMemcpyDefault, stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
      matrix_touch(A);
   });
}

int ofg_matrix_get_values(const ofg_matrix* A, double* a)
{
   return guarded("ofg_matrix_get_values", [&] {
      OFG_REQUIRE(A && (a || A->nnz == 0), OFG_ERR_ARG, "null argument");
      if (A->nnz)
         OFG_CUDA(cudaMemcpyAsync(a, A->val.p, A->nnz * sizeof(double), cudaMemcpyDefault, stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_matrix_device_arrays(const ofg_matrix* A, const int32_t** row_ptr, const int32_t** col,
                             double** values)
{
   return guarded("ofg_matrix_device_arrays", [&] {
      OFG_REQUIRE(A, OFG_ERR_ARG, "null matrix");
      if (row_ptr) *row_ptr = A->row_ptr.p;
      if (col) *col = A->col.p;
      if (values) {
         *values = A->val.p;
         const_cast<ofg_matrix*>(A)->version++;  // caller may write through it
      }
   });
}

int ofg_matrix_clear(ofg_matrix* A)
{
   return guarded("ofg_matrix_clear", [&] {
      OFG_REQUIRE(A, OFG_ERR_ARG, "null matrix");
      A->val.zero();
      matrix_touch(A);
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_spmv(const ofg_matrix* A, const double* x, double* y)
{
   return guarded("ofg_spmv", [&] {
      OFG_REQUIRE(A && x && y, OFG_ERR_ARG, "null argument");
      In<double> dx(x, A->n);
      InOut<double> dy(y, A->n, false);
      ensure_sell(const_cast<ofg_matrix*>(A));
      spmv_sell(A, dx.d, dy.d);
      dy.finish();
   });
}

int ofg_spmv_add(const ofg_matrix* A, const double* x, double* y)
{
   return guarded("ofg_spmv_add", [&] {
      OFG_REQUIRE(A && x && y, OFG_ERR_ARG, "null argument");
      In<double> dx(x, A->n);
      InOut<double> dy(y, A->n, true);
      spmv_csr(A, dx.d, dy.d, true);
      dy.finish();
   });
}

int ofg_spmv32_device(ofg_matrix* A, int kind, int blocks_per_sm, const float* d_x, float* d_y)
{
   return guarded("ofg_spmv32_device", [&] {
      OFG_REQUIRE(A && d_x && d_y, OFG_ERR_ARG, "null argument");
      OFG_REQUIRE(kind >= 0 && kind <= 3, OFG_ERR_ARG, "kind must be 0..3");
      ensure_sell32(A);
      if (!A->n) return;
      const int bps = blocks_per_sm > 0 ? blocks_per_sm : 8;
      const int64_t ns = A->nslices;
      int* worked = prof_begin();
      if (worked) OFG_CUDA(cudaMemsetAsync(worked, 1, sizeof(int), stream()));
      switch (kind) {
         case 0:
            spmv32_row<<<grid_for(ns * 32, 256, bps), 256, 0, stream()>>>(
               ns, A->sell_ptr.p, A->sell_col.p, A->sell_val32.p, d_x, d_y);
            break;
         case 1:
            spmv32_vec4<<<grid_for(ns * 8, 256, bps), 256, 0, stream()>>>(
               ns, A->sell_ptr.p, A->sell_col.p, A->sell_val32.p, d_x, d_y);
            break;
         case 2:
            spmv32_slices4<<<grid_for(ns * 8, 256, bps), 256, 0, stream()>>>(
               ns, A->sell_ptr.p, A->sell_col.p, A->sell_val32.p, d_x, d_y);
            break;
         default:
            spmv32_vec2<<<grid_for(ns * 16, 256, bps), 256, 0, stream()>>>(
               ns, A->sell_ptr.p, A->sell_col.p, A->sell_val32.p, d_x, d_y);
            break;
      }
      prof_end(PROF_SPMV32, 8.0 * A->nnz + 12.0 * A->n + 4.0);
      count_launch();
      OFG_LAUNCH_CHECK();
   });
}

int ofg_spmv_device(const ofg_matrix* A, int kind, const double* d_x, double* d_y)
{
   return guarded("ofg_spmv_device", [&] {
      OFG_REQUIRE(A && d_x && d_y, OFG_ERR_ARG, "null argument");
      if (kind == 1) {
         ensure_sell(const_cast<ofg_matrix*>(A));
         spmv_sell(A, d_x, d_y);
      }
      else {
         spmv_csr(A, d_x, d_y, false);
      }
   });
}

}  // extern "C"
