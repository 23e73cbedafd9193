// learned.cu -- a learned preconditioner: a message-passing network over the
// matrix graph predicts a factorised sparse approximate inverse
//     M = G^T G,   G lower triangular on the pattern of A,
// so that M r ~ A^{-1} r.  M is symmetric positive definite by construction
// (G has a positive diagonal), it is applied as two sparse products (no
// triangular solves, fully parallel), and the network runs once per matrix.
//
// Network (width 64, 4 message-passing layers, BF16 activations and GEMM
// operands, FP32 accumulation and FP32 master weights):
//   scaled graph  a~_ij = a_ij / sqrt(a_ii a_jj)  (off-diagonal), d_i = sqrt(a_ii)
//   node inputs   f_i = (1, deg_i/16, sum_j |a~_ij|, log a_ii - mean log a)
//   h0 = relu(f W_in + b_in)
//   layer l:      agg_i = sum_{j != i} a~_ij h_j
//                 h_l = relu([h_{l-1} | agg] W_l + b_l) + h_{l-1}
//   head          G^_ii = softplus(v . h_i + c),  G^_ij = a~_ij (u . (h_i o h_j)) (j < i)
//                 G_ij = G^_ij / d_j
// With u = v = 0 and softplus(c) = 1 the factor is G = D^{-1/2}: M is Jacobi.
// Training (Adam) runs on residual / error pairs (r_p = A e_p) with one of
// two objectives:
//   1 (default) the Kaporin number of MA, (tr(MA)/n) / det(MA)^(1/n), with
//     the trace estimated on the pairs: log of
//     (1/P) sum_p (G e_p . G r_p) n/||e_p||^2  minus  (2/n) sum_i log G_ii.
//     It is invariant to the scale of M and its minimiser over the pattern
//     is the factorised sparse approximate inverse; the pairs' errors should
//     be spectrally flat (e.g. x* - x0 for random starting guesses x0).
//   0 mean_p ||M r_p - e_p||^2 / ||e_p||^2 (the direct error-correction
//     fit; with errors taken from CG iterates, which are dominated by smooth
//     modes, it does not give a better CG preconditioner than Jacobi).
//
// The layer products [rows x 128] x [128 x 64] (forward; the 128 inputs are
// h and agg, read from their own arrays) and [rows x 64] x [64 x 128] (the
// backward data product) run on the tensor cores: tcgen05.mma kind::f16,
// BF16 x BF16 -> FP32 accumulators in tensor memory, operands staged in
// shared memory in the K-major core-matrix layout, one elected thread
// issues, the epilogue reads the accumulators with tcgen05.ld and applies
// bias / ReLU / residual in registers.  A CUDA-core version of the same
// product is kept as the checker (ofg_learned_gemm_check).  The weight
// gradient X^T dZ (a reduction over all rows: the rows are the MMA's K)
// runs on the tensor cores too (wgrad_tc), from the BF16 copy of dZ that
// the data product uses.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"
#include "mbar.cuh"
#include "reduce.cuh"

typedef __nv_bfloat16 bf16;

namespace ofg {
namespace {

constexpr int HID = 64;
constexpr int NFEAT = 4;
constexpr int NLAYER = 4;
// parameter offsets (floats)
constexpr int P_WIN = 0;                                  // NFEAT x HID
constexpr int P_BIN = P_WIN + NFEAT * HID;                // HID
constexpr int P_W = P_BIN + HID;                          // NLAYER x (2 HID x HID)
constexpr int P_B = P_W + NLAYER * 2 * HID * HID;         // NLAYER x HID
constexpr int P_U = P_B + NLAYER * HID;                   // HID
constexpr int P_V = P_U + HID;                            // HID
constexpr int P_C = P_V + HID;                            // 1
constexpr int NPARAM = P_C + 1;

__device__ __forceinline__ float bf2f(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_f(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_f(float v) { return v; }

// eight BF16 values <-> eight floats through one 16-byte access
__device__ __forceinline__ void load8(const bf16* p, float* f)
{
   const uint4 u = *reinterpret_cast<const uint4*>(p);
   const __nv_bfloat162* b = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
   for (int q = 0; q < 4; ++q) {
      const float2 t = __bfloat1622float2(b[q]);
      f[2 * q] = t.x;
      f[2 * q + 1] = t.y;
   }
}

__device__ __forceinline__ void store8(bf16* p, const float* f)
{
   uint4 u;
   __nv_bfloat162* b = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
   for (int q = 0; q < 4; ++q) b[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
   *reinterpret_cast<uint4*>(p) = u;
}

// ------------------------------------------------------------ graph prep --
// d_i = sqrt(|a_ii|)
__global__ void lp_scale(int64_t n, const double* val, const int32_t* dpos, float* dsq)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      dsq[i] = (float)sqrt(fabs(val[dpos[i]]));
}

// a~ (0 on the diagonal) and the node features
__global__ void lp_features(int64_t n, const int32_t* rp, const int32_t* col, const double* val,
                            const float* dsq, float* at, float* feat)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      float rs = 0.f;
      int deg = 0;
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         float a = 0.f;
         if (j != (int32_t)i) {
            a = (float)(val[k] / ((double)dsq[i] * (double)dsq[j]));
            rs += fabsf(a);
            deg++;
         }
         at[k] = a;
      }
      feat[i * NFEAT + 0] = 1.f;
      feat[i * NFEAT + 1] = deg / 16.f;
      feat[i * NFEAT + 2] = rs;
      feat[i * NFEAT + 3] = 2.f * logf(dsq[i]);  // centred below
   }
}

__global__ void __launch_bounds__(kRedBlock) lp_logmean(int64_t n, const float* feat, double* out,
                                                        double* partials, unsigned* counter)
{
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      v[0] += feat[i * NFEAT + 3];
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t)) *out = t[0] / (double)(n > 0 ? n : 1);
}

__global__ void lp_center(int64_t n, float* feat, const double* mean)
{
   const float m = (float)*mean;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      feat[i * NFEAT + 3] -= m;
}

// position of the transposed entry of every off-diagonal entry (the pattern
// is symmetric for these matrices; -1 otherwise)
__global__ void lp_transpose(int64_t n, const int32_t* rp, const int32_t* col, int32_t* tp)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         int32_t pos = -1;
         int32_t lo = rp[j], hi = rp[j + 1] - 1;
         while (lo <= hi) {
            const int32_t mid = (lo + hi) >> 1;
            const int32_t c = col[mid];
            if (c == (int32_t)i) { pos = mid; break; }
            if (c < (int32_t)i) lo = mid + 1;
            else hi = mid - 1;
         }
         tp[k] = pos;
      }
}

// ----------------------------------------------------------- layers (fwd) --
// h0 = relu(f W_in + b_in); also z0 (pre-activation) when z is given
__global__ void lp_embed(int64_t n, const float* feat, const float* P, bf16* h, bf16* z)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * HID; t += stride) {
      const int64_t i = t / HID;
      const int c = (int)(t % HID);
      float s = P[P_BIN + c];
#pragma unroll
      for (int q = 0; q < NFEAT; ++q) s += feat[i * NFEAT + q] * P[P_WIN + q * HID + c];
      if (z) z[t] = __float2bfloat16(s);
      h[t] = __float2bfloat16(fmaxf(s, 0.f));
   }
}

// agg_i = sum_{j != i} a~_ij h_j   (8 threads per row, 8 features each)
__global__ void lp_aggregate(int64_t n, const int32_t* rp, const int32_t* col, const float* at,
                             const bf16* h, bf16* agg)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * 8; t += stride) {
      const int64_t i = t >> 3;
      const int f0 = (int)(t & 7) * 8;
      float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const float a = at[k];
         if (a == 0.f) continue;
         float hv[8];
         load8(h + (int64_t)col[k] * HID + f0, hv);
#pragma unroll
         for (int q = 0; q < 8; ++q) acc[q] += a * hv[q];
      }
      store8(agg + i * HID + f0, acc);
   }
}

// ------------------------------------------------------- layer products ----
// The A operand of a product: row m is [a0[m, 0:k0] | a1[m, 0:K-k0]] (a1
// unused when k0 == K); row strides in elements.
struct GemmA {
   const bf16* a0;
   int64_t lda0;
   const bf16* a1;
   int64_t lda1;
   int k0;
   __device__ __forceinline__ const bf16* at(int64_t m, int k) const
   {
      return k < k0 ? a0 + m * lda0 + k : a1 + m * lda1 + (k - k0);
   }
};

// Epilogue of a forward layer, 16 columns of one row at a time:
// z = acc + b; h_new = relu(z) + h_old (BF16); z kept when asked for.
struct FwdFunctor {
   const float* bias;
   const bf16* h_old;
   bf16* z;  // may be null
   bf16* h_new;
   // h_new written, and z when kept (BF16); h_old, read too, is the first
   // half of the A operand and counted there
   int bytes_per_col() const { return z ? 4 : 2; }
   __device__ __forceinline__ void operator()(int64_t row, int c0, const float* v) const
   {
      float ho[16], zz[16], hh[16];
      load8(h_old + row * HID + c0, ho);
      load8(h_old + row * HID + c0 + 8, ho + 8);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
         zz[q] = v[q] + bias[c0 + q];
         hh[q] = fmaxf(zz[q], 0.f) + ho[q];
      }
      if (z) {
         store8(z + row * HID + c0, zz);
         store8(z + row * HID + c0 + 8, zz + 8);
      }
      store8(h_new + row * HID + c0, hh);
      store8(h_new + row * HID + c0 + 8, hh + 8);
   }
};

// Epilogue of the backward data product: dcat (FP32, 128 columns).
struct BwdFunctor {
   float* dcat;
   int bytes_per_col() const { return 4; }
   __device__ __forceinline__ void operator()(int64_t row, int c0, const float* v) const
   {
      float4* o = reinterpret_cast<float4*>(dcat + row * 2 * HID + c0);
#pragma unroll
      for (int q = 0; q < 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
   }
};

struct StoreFunctor {  // plain FP32 store, for the product check
   float* out;
   int ld;
   int bytes_per_col() const { return 4; }
   __device__ __forceinline__ void operator()(int64_t row, int c0, const float* v) const
   {
      float4* o = reinterpret_cast<float4*>(out + row * ld + c0);
#pragma unroll
      for (int q = 0; q < 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
   }
};

// CUDA-core product: C[rows x N] = A[rows x K] * Bt^T, Bt[N x K] row-major
// BF16, FP32 accumulation (the checker of the tensor-core path).
template <int K, int N, class Epi>
__global__ void __launch_bounds__(256) gemm_cc(int64_t rows, GemmA a, const bf16* Bt, Epi epi)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < rows * (N / 16);
        t += stride) {
      const int64_t row = t / (N / 16);
      const int c0 = (int)(t % (N / 16)) * 16;
      float acc[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) acc[q] = 0.f;
      for (int k = 0; k < K; ++k) {
         const float av = bf2f(*a.at(row, k));
#pragma unroll
         for (int q = 0; q < 16; ++q) acc[q] += av * bf2f(Bt[(c0 + q) * K + k]);
      }
      epi(row, c0, acc);
   }
}

// Tensor-core product.  One CTA (4 warps) per 128-row tile at a time
// (persistent over tiles).  Shared memory holds A (128 x K) and B (N x K) in
// the K-major core-matrix layout without swizzle: element (m, k) of an
// M-row operand at (k/8)*(M/8)*128 + m*16 + (k%8)*2 bytes, so one MMA
// (K = 16) reads two 8-column chunks LBO = M*16 bytes apart, with SBO = 128
// bytes between 8-row groups.  Thread t stages row t of the A tile, 32
// bytes at a time (one full sector), and a warp's stores cover 512
// contiguous bytes.  The accumulator (128 lanes x N FP32 columns) lives in
// tensor memory; thread 0 issues the MMAs and commits them to an mbarrier.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
   uint64_t d = 0;
   d |= (uint64_t)((saddr >> 4) & 0x3FFF);
   d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
   d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
   d |= (uint64_t)1 << 46;  // descriptor version for this architecture
   // base offset 0, legacy LBO mode, layout type 0 = no swizzle
   return d;
}

template <int N>
__host__ __device__ constexpr uint32_t instr_desc_bf16_f32()
{
   // c_format F32 (bit 4), a/b format BF16 (bits 7, 10), K-major A and B,
   // N >> 3 at bits 17..22, M >> 4 at bits 24..28 (M = 128)
   return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
}

template <int K, int N, class Epi>
__global__ void __launch_bounds__(128, 4) gemm_tc(int64_t rows, GemmA a,
                                                  const bf16* __restrict__ Bt, Epi epi, int* status,
                                                  int* worked)
{
   static_assert(K % 16 == 0 && N % 16 == 0 && N >= 32 && N <= 256, "tile shape");
   prof_mark(worked);
   extern __shared__ __align__(1024) unsigned char smem[];
   unsigned char* sA = smem;                   // 128*K*2 bytes
   unsigned char* sB = smem + 128 * K * 2;     // N*K*2 bytes
   uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + N * K * 2);
   uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
   const int tid = threadIdx.x, warp = tid >> 5;

   // B once per CTA: row nr of chunk c at c*N*16 + nr*16
   for (int piece = tid; piece < N * K / 8; piece += 128) {
      const int nr = piece % N, c = piece / N;
      const uint4 v = *reinterpret_cast<const uint4*>(Bt + (int64_t)nr * K + c * 8);
      *reinterpret_cast<uint4*>(sB + c * N * 16 + nr * 16) = v;
   }
   if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                      smem_u32(tslot)),
                   "r"(N)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
   }
   asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
   asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
   __syncthreads();
   asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
   const uint32_t tmem = *tslot;
   const uint32_t sa = smem_u32(sA), sb = smem_u32(sB);
   constexpr uint32_t idesc = instr_desc_bf16_f32<N>();
   uint32_t phase = 0;
   bool failed = false;
   const int64_t ntiles = (rows + 127) / 128;

   for (int64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
      const int64_t m0 = tile * 128;
      {
         const int64_t r = m0 + tid;
#pragma unroll
         for (int cp = 0; cp < K / 16; ++cp) {
            uint4 v0 = make_uint4(0, 0, 0, 0), v1 = v0;
            if (r < rows) {
               const bf16* src = a.at(r, cp * 16);
               v0 = *reinterpret_cast<const uint4*>(src);
               v1 = *reinterpret_cast<const uint4*>(src + 8);
            }
            *reinterpret_cast<uint4*>(sA + (2 * cp) * 2048 + tid * 16) = v0;
            *reinterpret_cast<uint4*>(sA + (2 * cp + 1) * 2048 + tid * 16) = v1;
         }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (tid == 0) {
#pragma unroll
         for (int kk = 0; kk < K / 16; ++kk) {
            const uint64_t ad = smem_desc(sa + kk * 2 * 2048, 2048, 128);
            const uint64_t bd = smem_desc(sb + kk * 2 * N * 16, N * 16, 128);
            const uint32_t acc = kk > 0 ? 1u : 0u;
            asm volatile(
               "{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
               "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
               : "memory");
         }
         asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
               smem_u32(mbar))
            : "memory");
      }
      // bounded wait for the MMAs of this tile; the outcome is made uniform
      // over the block so that every thread leaves the loop together
      if (__syncthreads_or(mbar_wait(smem_u32(mbar), phase) ? 0 : 1)) {
         failed = true;
         if (tid == 0) atomicOr(status, 1);
      }
      else {
         phase ^= 1;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (!failed) {
         const int64_t row = m0 + warp * 32 + (tid & 31);
#pragma unroll
         for (int cb = 0; cb < N; cb += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
            asm volatile(
               "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
               "%10, %11, %12, %13, %14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
            if (row < rows) epi(row, cb, v);
         }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
   }
   // after a wait that ran out, give the MMAs in flight one more bounded
   // wait before the tensor memory is released
   if (failed) mbar_wait(smem_u32(mbar), phase);
   __syncthreads();
   if (warp == 0)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(N)
                   : "memory");
}

// The forward layer product [h | agg] W (K = 128, N = 64) with the A tiles
// brought in by the tensor memory accelerator and two stages in flight.
// Each 128-row tile of A arrives as sixteen 2-D boxes of {8 elements, 128
// rows} (one per 8-column chunk of h or agg), so box c lands as chunk c of
// gemm_tc's K-major core-matrix layout (2048 bytes: row m at m*16).  Per
// tile k of the block: thread 0 issues the TMA loads of tile k+2 into the
// stage the MMAs of tile k have just released and the MMAs of tile k+1 (into
// the other tensor-memory accumulator), then all threads run the epilogue
// of tile k.  So the loads, the MMAs and the epilogue of three tiles
// overlap.  Loads complete on a `full` mbarrier per stage (transaction
// count), MMAs commit to a `done` mbarrier per stage; every wait is bounded,
// and a block whose wait ran out drains what it issued before it returns.
// The tensor maps cover this GPU's own buffers only; no multicast.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t mbar)
{
   asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

template <class Epi>
__global__ void __launch_bounds__(128, 2) gemm_tc_tma(int64_t rows,
                                                      const __grid_constant__ CUtensorMap t0,
                                                      const __grid_constant__ CUtensorMap t1,
                                                      const bf16* __restrict__ Bt, Epi epi,
                                                      int* status, int* worked)
{
   constexpr int K = 2 * HID, N = HID;
   constexpr uint32_t kTileBytes = 128 * K * 2;  // 32 KB
   prof_mark(worked);
   extern __shared__ __align__(1024) unsigned char smem[];
   unsigned char* sA = smem;                    // two stages of kTileBytes
   unsigned char* sB = smem + 2 * kTileBytes;   // N*K*2 bytes
   uint64_t* bars = reinterpret_cast<uint64_t*>(sB + N * K * 2);  // full[2], done[2]
   uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 4);
   __shared__ int fail_sh;
   const int tid = threadIdx.x, warp = tid >> 5;

   for (int piece = tid; piece < N * K / 8; piece += 128) {
      const int nr = piece % N, c = piece / N;
      const uint4 v = *reinterpret_cast<const uint4*>(Bt + (int64_t)nr * K + c * 8);
      *reinterpret_cast<uint4*>(sB + c * N * 16 + nr * 16) = v;
   }
   if (tid == 0) {
      for (int q = 0; q < 4; ++q)
         asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bars + q)), "r"(1)
                      : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      fail_sh = 0;
   }
   if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                      smem_u32(tslot)),
                   "r"(2 * N)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
   }
   asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
   asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
   __syncthreads();
   asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
   const uint32_t tmem = *tslot;
   const uint32_t sa = smem_u32(sA), sb = smem_u32(sB);
   constexpr uint32_t idesc = instr_desc_bf16_f32<N>();
   const int64_t ntiles = (rows + 127) / 128;
   const int64_t mine = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
   auto full = [&](int s) { return smem_u32(bars + s); };
   auto done = [&](int s) { return smem_u32(bars + 2 + s); };
   // thread 0 only
   auto issue_load = [&](int64_t k) {
      const int s = (int)(k & 1);
      const int y = (int)((blockIdx.x + k * gridDim.x) * 128);
      const uint32_t dst = sa + s * kTileBytes;
      mbar_expect_tx(full(s), kTileBytes);
#pragma unroll
      for (int c = 0; c < K / 8; ++c)
         tma_load_2d(dst + c * 2048, c < 8 ? &t0 : &t1, (c & 7) * 8, y, full(s));
   };
   auto issue_mma = [&](int64_t k) {
      const int s = (int)(k & 1);
      const uint32_t a0 = sa + s * kTileBytes;
#pragma unroll
      for (int kk = 0; kk < K / 16; ++kk) {
         const uint64_t ad = smem_desc(a0 + kk * 2 * 2048, 2048, 128);
         const uint64_t bd = smem_desc(sb + kk * 2 * N * 16, N * 16, 128);
         const uint32_t acc = kk > 0 ? 1u : 0u;
         asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
               tmem + (uint32_t)(s * N)),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
            : "memory");
      }
      asm volatile(
         "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done(s))
         : "memory");
   };
   // loads issued and waited for, per stage (for the drain after a failure)
   int64_t loads_issued = 0, loads_waited = 0, mmas_issued = 0, mmas_waited = 0;
   bool failed = false;
   if (tid == 0 && mine > 0) {
      issue_load(0);
      loads_issued = 1;
      if (mine > 1) {
         issue_load(1);
         loads_issued = 2;
      }
      if (mbar_wait(full(0), 0)) {
         loads_waited = 1;
         asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
         issue_mma(0);
         mmas_issued = 1;
      }
      else {
         fail_sh = 1;
      }
   }
   __syncthreads();
   failed = fail_sh != 0;
   for (int64_t k = 0; k < mine && !failed; ++k) {
      const int s = (int)(k & 1);
      // MMAs of tile k finished: its accumulator is ready, its stage free
      if (__syncthreads_or(mbar_wait(done(s), (uint32_t)((k >> 1) & 1)) ? 0 : 1)) {
         failed = true;
         if (tid == 0) atomicOr(status, 1);
         break;
      }
      if (tid == 0) mmas_waited = k + 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (tid == 0) {
         if (k + 2 < mine) {
            issue_load(k + 2);
            loads_issued = k + 3;
         }
         if (k + 1 < mine) {
            if (mbar_wait(full((int)((k + 1) & 1)), (uint32_t)(((k + 1) >> 1) & 1))) {
               loads_waited = k + 2;
               asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
               issue_mma(k + 1);
               mmas_issued = k + 2;
            }
            else {
               fail_sh = 1;
               atomicOr(status, 1);
            }
         }
      }
      // epilogue of tile k from its accumulator
      const int64_t row = (blockIdx.x + k * gridDim.x) * 128 + warp * 32 + (tid & 31);
#pragma unroll
      for (int cb = 0; cb < N; cb += 16) {
         uint32_t r[16];
         const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(s * N + cb);
         asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
         asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
         float v[16];
#pragma unroll
         for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
         if (row < rows) epi(row, cb, v);
      }
      // every thread is done with accumulator s before MMAs reuse it
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      failed = fail_sh != 0;
   }
   // after a wait that ran out: drain what was issued (bounded waits)
   if (failed && tid == 0) {
      for (int64_t q = loads_waited; q < loads_issued; ++q)
         mbar_wait(full((int)(q & 1)), (uint32_t)((q >> 1) & 1));
      for (int64_t q = mmas_waited; q < mmas_issued; ++q)
         mbar_wait(done((int)(q & 1)), (uint32_t)((q >> 1) & 1));
   }
   __syncthreads();
   if (warp == 0)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * N)
                   : "memory");
}

// Weight gradient on the tensor cores: part[block] = X^T dz over the
// block's 128-row tiles, X = [h | agg] (rows x 128, BF16) and dz (rows x 64,
// BF16).  The reduction runs over the rows, so the rows are the MMA's K:
// each tile stages X^T (M = 128 features x K = 128 rows) and dz^T (N = 64 x
// K) in the K-major core-matrix layout of gemm_tc (element (m, k) at
// (k/8)*(M/8)*128 + m*16 + (k%8)*2 bytes; thread t writes row t of the
// tile, transposed, two bytes at a time), one thread issues the tile's
// eight K = 16 MMAs into the block's tensor-memory accumulator (128 lanes x
// 64 FP32 columns, kept across the block's tiles), and the block writes its
// 128 x 64 partial at the end.  Waits are bounded as in gemm_tc.
__global__ void __launch_bounds__(128, 4) wgrad_tc(int64_t rows, GemmA a,
                                                   const bf16* __restrict__ dz, float* part,
                                                   int* status, int* worked)
{
   constexpr int M = 2 * HID, N = HID;
   prof_mark(worked);
   extern __shared__ __align__(1024) unsigned char smem[];
   unsigned char* sA = smem;                // M x 128 rows: 32 KB
   unsigned char* sB = smem + M * 128 * 2;  // N x 128 rows: 16 KB
   uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + N * 128 * 2);
   uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
   const int tid = threadIdx.x, warp = tid >> 5;
   if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                      smem_u32(tslot)),
                   "r"(N)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
   }
   asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
   __syncthreads();
   asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
   const uint32_t tmem = *tslot;
   const uint32_t sa = smem_u32(sA), sb = smem_u32(sB);
   constexpr uint32_t idesc = instr_desc_bf16_f32<N>();
   uint32_t phase = 0;
   bool failed = false, any = false;
   const int64_t ntiles = (rows + 127) / 128;
   bf16* pa = reinterpret_cast<bf16*>(sA + (tid >> 3) * (M / 8) * 128 + (tid & 7) * 2);
   bf16* pb = reinterpret_cast<bf16*>(sB + (tid >> 3) * (N / 8) * 128 + (tid & 7) * 2);

   for (int64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
      const int64_t r = tile * 128 + tid;  // this thread's row: K index tid of the tile
#pragma unroll 4
      for (int c = 0; c < M / 8; ++c) {
         uint4 v = make_uint4(0, 0, 0, 0);
         if (r < rows) v = *reinterpret_cast<const uint4*>(a.at(r, c * 8));
         const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
         for (int q = 0; q < 8; ++q) pa[(c * 8 + q) * 8] = e[q];  // (m = 8c + q) * 16 bytes
      }
#pragma unroll 4
      for (int c = 0; c < N / 8; ++c) {
         uint4 v = make_uint4(0, 0, 0, 0);
         if (r < rows) v = *reinterpret_cast<const uint4*>(dz + r * N + c * 8);
         const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
         for (int q = 0; q < 8; ++q) pb[(c * 8 + q) * 8] = e[q];
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (tid == 0) {
#pragma unroll
         for (int kk = 0; kk < 8; ++kk) {
            const uint64_t ad = smem_desc(sa + kk * 2 * (M * 16), M * 16, 128);
            const uint64_t bd = smem_desc(sb + kk * 2 * (N * 16), N * 16, 128);
            const uint32_t acc = (any || kk > 0) ? 1u : 0u;
            asm volatile(
               "{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
               "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
               : "memory");
         }
         asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
               smem_u32(mbar))
            : "memory");
      }
      any = true;
      // the tile's MMAs must finish before the next tile overwrites the
      // operands (bounded wait, outcome uniform over the block)
      if (__syncthreads_or(mbar_wait(smem_u32(mbar), phase) ? 0 : 1)) {
         failed = true;
         if (tid == 0) atomicOr(status, 1);
      }
      else {
         phase ^= 1;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
   }
   // the accumulator: lane m = input feature, column n = output
   float* out = part + (int64_t)blockIdx.x * M * N + (int64_t)(warp * 32 + (tid & 31)) * N;
   for (int cb = 0; cb < N; cb += 16) {
      uint32_t v[16];
      if (any && !failed) {
         const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
         asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
         asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      }
      else {
#pragma unroll
         for (int q = 0; q < 16; ++q) v[q] = 0u;
      }
      float4* o = reinterpret_cast<float4*>(out + cb);
#pragma unroll
      for (int q = 0; q < 4; ++q)
         o[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                            __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
   }
   if (failed) mbar_wait(smem_u32(mbar), phase);
   asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
   __syncthreads();
   if (warp == 0)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(N)
                   : "memory");
}

// ------------------------------------------------------------------ head --
// G (lower part incl. diagonal, stored at A's CSR positions; upper = 0).
// Eight lanes per row, eight features each; the dot products are reduced
// over the lane group with shuffles.
__global__ void lp_head(int64_t n, const int32_t* rp, const int32_t* col, const float* at,
                        const float* dsq, const bf16* h, const float* P, float* g)
{
   const int lane = threadIdx.x & 31, sub = lane & 7;
   const unsigned gmask = 0xFFu << (lane & 24);
   float u[8], v[8];
#pragma unroll
   for (int q = 0; q < 8; ++q) {
      u[q] = P[P_U + sub * 8 + q];
      v[q] = P[P_V + sub * 8 + q];
   }
   const float cc = P[P_C];
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * 8; t += stride) {
      const int64_t i = t >> 3;
      float hi[8];
      load8(h + i * HID + sub * 8, hi);
      float dv = 0.f;
#pragma unroll
      for (int q = 0; q < 8; ++q) dv += v[q] * hi[q];
      dv += __shfl_xor_sync(gmask, dv, 1);
      dv += __shfl_xor_sync(gmask, dv, 2);
      dv += __shfl_xor_sync(gmask, dv, 4);
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         float gv = 0.f;
         if (j == (int32_t)i) {
            const float s = cc + dv;
            const float sp = fmaxf(s > 20.f ? s : log1pf(expf(s)), 1e-20f);
            gv = sp / dsq[i];
         }
         else if (j < (int32_t)i && at[k] != 0.f) {
            float hj[8];
            load8(h + (int64_t)j * HID + sub * 8, hj);
            float s = 0.f;
#pragma unroll
            for (int q = 0; q < 8; ++q) s += u[q] * hi[q] * hj[q];
            s += __shfl_xor_sync(gmask, s, 1);
            s += __shfl_xor_sync(gmask, s, 2);
            s += __shfl_xor_sync(gmask, s, 4);
            gv = at[k] * s / dsq[j];
         }
         if (sub == 0) g[k] = gv;
      }
   }
}

// ------------------------------------------------------- apply M = G^T G --
// z = G r (lower rows), for P columns of n entries (training)
template <class T>
__global__ void lp_apply_lower(int64_t n, int64_t ncols, const int32_t* rp, const int32_t* col,
                               const float* g, const T* r, T* z)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * ncols; t += stride) {
      const int64_t i = t % n, p = t / n;
      double s = 0.0;
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         if (j > (int32_t)i) break;
         s += (double)g[k] * (double)r[p * n + j];
      }
      z[p * n + i] = (T)s;
   }
}

// y = G^T z: y_j = sum_{i >= j} G_ij z_i, read through the transposed
// positions of row j's upper entries
template <class T>
__global__ void lp_apply_upper(int64_t n, int64_t ncols, const int32_t* rp, const int32_t* col,
                               const int32_t* tp, const float* g, const T* z, T* y)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * ncols; t += stride) {
      const int64_t j = t % n, p = t / n;
      double s = 0.0;
      for (int32_t k = rp[j]; k < rp[j + 1]; ++k) {
         const int32_t i = col[k];
         if (i < (int32_t)j) continue;
         const int32_t q = (i == (int32_t)j) ? k : tp[k];
         if (q >= 0) s += (double)g[q] * (double)z[p * n + i];
      }
      y[p * n + j] = (T)s;
   }
}

}  // namespace
}  // namespace ofg

// ----------------------------------------------------------------- handle --
struct ofg_learned {
   ofg::DBuf<float> params, grads, m1, m2;
   ofg::DBuf<bf16> wt;  // per layer: W_l^T (64 x 128), the forward B operand
   ofg::DBuf<bf16> wb;  // per layer: W_l (128 x 64), the backward B operand
   int64_t step = 0;
   int use_tc = 1;
   int loss_kind = 1;  // 0: ||M r - e||^2 / ||e||^2, 1: Kaporin number
   ofg::DBuf<int> status;
};

namespace ofg {

// Inputs, activations and output of the network on one matrix.  Training
// keeps every layer's activations (the backward pass needs them); inference
// keeps two hidden-state buffers and one aggregate buffer.
struct LearnedGraph {
   int64_t n = 0, nnz = 0;
   bool train = false, tp_ready = false;
   DBuf<float> dsq, at, feat, g;
   DBuf<int32_t> tp;
   DBuf<double> mean, partials;
   DBuf<unsigned> counter;
   DBuf<bf16> h[NLAYER + 1], z[NLAYER + 1], agg[NLAYER];
   bf16* hbuf(int l) { return train ? h[l].p : h[l & 1].p; }
   bf16* aggbuf(int l) { return train ? agg[l].p : agg[0].p; }
   bf16* zbuf(int l) { return train ? z[l].p : nullptr; }
};

namespace {

__global__ void lp_init_params(float* P, uint64_t seed)
{
   // Xavier-uniform weights from a counter-based hash, zero biases, u = v = 0,
   // softplus(c) = 1
   for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < NPARAM; t += gridDim.x * blockDim.x) {
      uint64_t z = seed * 0x9E3779B97F4A7C15ULL + (uint64_t)(t + 1) * 0xD1B54A32D192ED03ULL;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
      z ^= z >> 31;
      const float u01 = (float)((z >> 40) * (1.0 / 16777216.0));
      float v = 0.f;
      if (t < P_BIN) v = (2.f * u01 - 1.f) * sqrtf(6.f / (NFEAT + HID));
      else if (t >= P_W && t < P_B) v = (2.f * u01 - 1.f) * sqrtf(6.f / (2 * HID + HID)) * 0.5f;
      else if (t == P_C) v = 0.54132485f;  // log(e - 1)
      P[t] = v;
   }
}

__global__ void lp_cast_weights(const float* P, bf16* wt, bf16* wb)
{
   // W_l is stored (2 HID) x HID row-major at P_W + l * 2 HID * HID
   const int per = 2 * HID * HID;
   for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < NLAYER * per; t += gridDim.x * blockDim.x) {
      const int l = t / per, e = t % per;
      const int kin = e / HID, nout = e % HID;  // W[kin][nout]
      const bf16 v = __float2bfloat16(P[P_W + t]);
      wb[l * per + kin * HID + nout] = v;        // B for dX: [N=128 x K=64] = W rows
      wt[l * per + nout * 2 * HID + kin] = v;    // B for forward: [N=64 x K=128] = W^T rows
   }
}

}  // namespace

// (re)computes the graph inputs for A's current values; the transposed
// positions only when the pattern is new
static void graph_prepare(ofg_matrix* A, LearnedGraph& G, bool train)
{
   const int64_t n = A->n;
   ensure_dpos(A);
   OFG_REQUIRE(A->dpos_complete, OFG_ERR_PIVOT, "a row has no diagonal entry");
   if (G.n != n || G.nnz != A->nnz || G.train != train) {
      G.tp_ready = false;
      G.n = n;
      G.nnz = A->nnz;
      G.train = train;
      G.dsq.alloc(n);
      G.at.alloc(A->nnz);
      G.feat.alloc(n * NFEAT);
      G.g.alloc(A->nnz);
      G.tp.alloc(A->nnz);
      G.mean.alloc(1);
      G.partials.alloc(((size_t)grid_for(n, kRedBlock, 8) + 1) * 2);
      G.counter.alloc(1);
      G.counter.zero();
      for (int l = 0; l <= NLAYER; ++l) {
         G.h[l].release();
         G.z[l].release();
         if (l < NLAYER) G.agg[l].release();
      }
      const int nh = train ? NLAYER + 1 : 2, na = train ? NLAYER : 1;
      for (int l = 0; l < nh; ++l) G.h[l].alloc(n * HID);
      for (int l = 0; l < na; ++l) G.agg[l].alloc(n * HID);
      if (train)
         for (int l = 0; l <= NLAYER; ++l) G.z[l].alloc(n * HID);
   }
   const unsigned gr = grid_for(n, 256);
   lp_scale<<<gr, 256, 0, stream()>>>(n, A->val.p, A->dpos.p, G.dsq.p);
   lp_features<<<gr, 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p, A->val.p, G.dsq.p, G.at.p,
                                         G.feat.p);
   lp_logmean<<<grid_for(n, kRedBlock, 8), kRedBlock, 0, stream()>>>(n, G.feat.p, G.mean.p,
                                                                     G.partials.p, G.counter.p);
   lp_center<<<gr, 256, 0, stream()>>>(n, G.feat.p, G.mean.p);
   count_launch(4);
   if (!G.tp_ready) {
      lp_transpose<<<gr, 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p, G.tp.p);
      count_launch();
      G.tp_ready = true;
   }
   OFG_LAUNCH_CHECK();
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link the driver library itself)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
   static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
   if (!fn) {
      void* p = nullptr;
      cudaDriverEntryPointQueryResult q;
      OFG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
      OFG_REQUIRE(q == cudaDriverEntryPointSuccess && p, OFG_ERR_CUDA,
                  "cuTensorMapEncodeTiled is not available");
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
   }
   return fn;
}

// 2-D map of a rows x 64 BF16 block with row stride ld elements, boxes of
// {8 elements, 128 rows} (rows past the end read as zeros)
static CUtensorMap half_map(const bf16* base, int64_t rows, int64_t ld)
{
   OFG_REQUIRE(((uintptr_t)base & 15) == 0 && (ld * 2) % 16 == 0, OFG_ERR_ARG,
               "layer operand not 16-byte aligned");
   CUtensorMap m;
   cuuint64_t dims[2] = {(cuuint64_t)HID, (cuuint64_t)rows};
   cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
   cuuint32_t box[2] = {8, 128};
   cuuint32_t estr[2] = {1, 1};
   const CUresult r = tensor_map_encoder()(
      &m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
   OFG_REQUIRE(r == CUDA_SUCCESS, OFG_ERR_CUDA,
               "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
   return m;
}

template <int K, int N, class Epi>
static void run_gemm(ofg_learned* L, int64_t rows, GemmA a, const bf16* Bt, Epi epi)
{
   if (rows <= 0) return;
   if constexpr (K == 2 * HID && N == HID) {
      if (L->use_tc && a.k0 == HID && rows < (int64_t(1) << 31)) {
         // the forward product: TMA-fed, two stages in flight
         constexpr int smem = 2 * 128 * K * 2 + N * K * 2 + 64;
         static bool attr_set = false;
         if (!attr_set) {
            OFG_CUDA(cudaFuncSetAttribute(gemm_tc_tma<Epi>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            attr_set = true;
         }
         const CUtensorMap t0 = half_map(a.a0, rows, a.lda0), t1 = half_map(a.a1, rows, a.lda1);
         const int64_t tiles = (rows + 127) / 128;
         const unsigned grid = (unsigned)std::min<int64_t>(tiles, (int64_t)num_sms() * 2);
         int* worked = prof_begin();
         gemm_tc_tma<Epi><<<grid, 128, smem, stream()>>>(rows, t0, t1, Bt, epi, L->status.p,
                                                         worked);
         prof_end(PROF_NET_GEMM, (double)rows * (K * 2 + N * epi.bytes_per_col()) + (double)N * K * 2);
         count_launch();
         OFG_LAUNCH_CHECK();
         return;
      }
   }
   if (L->use_tc) {
      // at least 48 KB of shared memory per block caps residency at four
      // blocks per SM, so the tensor-memory allocations (<= 128 columns
      // each) never exceed the SM's 512 columns and never wait
      const int smem = std::max(128 * K * 2 + N * K * 2 + 64, 48 * 1024);
      static bool attr_set = false;
      if (!attr_set) {
         OFG_CUDA(cudaFuncSetAttribute(gemm_tc<K, N, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem));
         attr_set = true;
      }
      const int64_t tiles = (rows + 127) / 128;
      const unsigned grid = (unsigned)std::min<int64_t>(tiles, (int64_t)num_sms() * 4);
      int* worked = prof_begin();
      gemm_tc<K, N, Epi><<<grid, 128, smem, stream()>>>(rows, a, Bt, epi, L->status.p, worked);
      // algorithmic bytes: the A operand, the weights, and the epilogue's
      // own reads and writes per output column
      prof_end(PROF_NET_GEMM, (double)rows * (K * 2 + N * epi.bytes_per_col()) + (double)N * K * 2);
   }
   else {
      gemm_cc<K, N, Epi><<<grid_for(rows * (N / 16), 256), 256, 0, stream()>>>(rows, a, Bt, epi);
   }
   count_launch();
   OFG_LAUNCH_CHECK();
}

// forward pass: the hidden states and the factor G
static void learned_forward(ofg_learned* L, ofg_matrix* A, LearnedGraph& G)
{
   const int64_t n = A->n;
   lp_embed<<<grid_for(n * HID, 256), 256, 0, stream()>>>(n, G.feat.p, L->params.p, G.hbuf(0),
                                                            G.zbuf(0));
   count_launch();
   for (int l = 0; l < NLAYER; ++l) {
      lp_aggregate<<<grid_for(n * 8, 256), 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p, G.at.p,
                                                                G.hbuf(l), G.aggbuf(l));
      count_launch();
      FwdFunctor f{L->params.p + P_B + l * HID, G.hbuf(l), G.zbuf(l + 1), G.hbuf(l + 1)};
      GemmA a{G.hbuf(l), HID, G.aggbuf(l), HID, HID};
      run_gemm<2 * HID, HID>(L, n, a, L->wt.p + (size_t)l * 2 * HID * HID, f);
   }
   lp_head<<<grid_for(n * 8, 256), 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p, G.at.p, G.dsq.p,
                                                        G.hbuf(NLAYER), L->params.p, G.g.p);
   count_launch();
   OFG_LAUNCH_CHECK();
}

}  // namespace ofg

// ============================================================ backward ====
namespace ofg {
namespace {

// loss of a batch: dY_p = (2/P)(Y_p - E_p)/||E_p||^2, loss = mean ||Y-E||^2/||E||^2
__global__ void __launch_bounds__(kRedBlock) lp_loss(int64_t n, int64_t P, const float* Y,
                                                     const float* E, const float* enorm2,
                                                     float* dY, double* loss, double* partials,
                                                     unsigned* counter)
{
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * P; t += stride) {
      const int64_t p = t / n;
      const float d = Y[t] - E[t];
      const float w = 1.f / (enorm2[p] * (float)P);
      dY[t] = 2.f * d * w;
      v[0] += (double)d * d * w;
   }
   double tt[1];
   if (grid_reduce<1>(v, partials, counter, tt)) *loss = tt[0];
}

// Kaporin objective over the pairs (the condition-number measure
// (tr(MA)/n) / det(MA)^(1/n), whose minimiser over the pattern is the
// factorised sparse approximate inverse): with w_p = n / ||e_p||^2,
//     T = (1/P) sum_p w_p (G e_p . G r_p)   (an estimate of tr(G A G^T))
//     loss = log(T / n) - (2/n) sum_i log G_ii           (+ const)
// out[0] = loss, out[1] = T.
__global__ void __launch_bounds__(kRedBlock) lp_kap_loss(int64_t n, int64_t P, const float* Z,
                                                         const float* GE, const float* enorm2,
                                                         const int32_t* dpos, const float* g,
                                                         double* out, double* partials,
                                                         unsigned* counter)
{
   double v[2] = {0.0, 0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * P; t += stride) {
      const int64_t p = t / n;
      v[0] += (double)Z[t] * (double)GE[t] * ((double)n / ((double)enorm2[p] * (double)P));
   }
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      v[1] += log((double)g[dpos[i]]);
   double t[2];
   if (grid_reduce<2>(v, partials, counter, t)) {
      out[1] = t[0];
      out[0] = log(t[0] / (double)n) - 2.0 * t[1] / (double)n;
   }
}

// upstream of the trace term: dY_p = w_p / (P T) e_p
__global__ void lp_kap_dy(int64_t n, int64_t P, const float* E, const float* enorm2,
                          const double* out, float* dY)
{
   const double T = out[1];
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * P; t += stride) {
      const int64_t p = t / n;
      dY[t] = (float)((double)E[t] * (double)n / ((double)enorm2[p] * (double)P * T));
   }
}

// the log-determinant term: dG_ii -= 2 / (n G_ii)
__global__ void lp_kap_diag(int64_t n, const int32_t* dpos, const float* g, float* dg)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const int32_t k = dpos[i];
      dg[k] -= 2.f / ((float)n * g[k]);
   }
}

__global__ void __launch_bounds__(kRedBlock) lp_sqnorms(int64_t n, int64_t P, const float* E,
                                                        float* out)
{
   // one block per pair
   const int64_t p = blockIdx.x;
   if (p >= P) return;
   float s = 0.f;
   for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += E[p * n + i] * E[p * n + i];
   __shared__ float sh[kRedBlock / 32];
   s = warp_sumf(s);
   if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
   __syncthreads();
   if (threadIdx.x == 0) {
      float tot = 0.f;
      for (int w = 0; w < kRedBlock / 32; ++w) tot += sh[w];
      out[p] = tot > 0.f ? tot : 1.f;
   }
}

// dG at the lower positions: sum_p dY_p[j] Z_p[i] + dZ_p[i] R_p[j]
__global__ void lp_dG(int64_t n, int64_t P, const int32_t* rp, const int32_t* col, const float* R,
                      const float* Z, const float* dY, const float* dZ, float* dg)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         float s = 0.f;
         if (j <= (int32_t)i)
            for (int64_t p = 0; p < P; ++p)
               s += dY[p * n + j] * Z[p * n + i] + dZ[p * n + i] * R[p * n + j];
         dg[k] = s;
      }
}

// dS (the head's bilinear score) at lower off-diagonal positions and the
// diagonal softplus derivative
__global__ void lp_dS(int64_t n, const int32_t* rp, const int32_t* col, const float* at,
                      const float* dsq, const bf16* h, const float* P, const float* dg, float* ds)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         float v = 0.f;
         if (j == (int32_t)i) {
            float s = P[P_C];
            for (int c = 0; c < HID; ++c) s += P[P_V + c] * bf2f(h[i * HID + c]);
            const float sig = 1.f / (1.f + expf(-s));
            v = dg[k] * sig / dsq[i];
         }
         else if (j < (int32_t)i) {
            v = dg[k] * at[k] / dsq[j];
         }
         ds[k] = v;
      }
}

// dh of the head (gather, no atomics): diagonal term + lower and upper
// neighbours through the transposed positions
__global__ void lp_head_back(int64_t n, const int32_t* rp, const int32_t* col, const int32_t* tp,
                             const bf16* h, const float* P, const float* ds, float* dh)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * HID; t += stride) {
      const int64_t i = t / HID;
      const int c = (int)(t % HID);
      float acc = 0.f;
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         if (j == (int32_t)i) acc += ds[k] * P[P_V + c];
         else if (j < (int32_t)i) acc += ds[k] * P[P_U + c] * bf2f(h[(int64_t)j * HID + c]);
         else {
            const int32_t q = tp[k];  // (j, i) in row j, a lower entry of row j
            if (q >= 0) acc += ds[q] * P[P_U + c] * bf2f(h[(int64_t)j * HID + c]);
         }
      }
      dh[t] = acc;
   }
}

// per-block partial sums of the head parameter gradients:
// du_c = sum_lower dS h_ic h_jc; dv_c = sum_i dsd_i h_ic; dc = sum_i dsd_i.
// Eight threads per row, eight features each; the block's threads are
// summed in a fixed order (the result does not depend on scheduling).
constexpr int HEADG = 2 * HID + 1;
__global__ void __launch_bounds__(256) lp_head_pgrad(int64_t n, const int32_t* rp, const int32_t* col,
                                                     const bf16* h, const float* ds, float* part)
{
   __shared__ float red[256][17];
   const int sub = threadIdx.x & 7;
   float du[8], dv[8], dc = 0.f;
#pragma unroll
   for (int q = 0; q < 8; ++q) du[q] = dv[q] = 0.f;
   for (int64_t i = (int64_t)blockIdx.x * (blockDim.x / 8) + (threadIdx.x >> 3); i < n;
        i += (int64_t)gridDim.x * (blockDim.x / 8)) {
      float hi[8];
      load8(h + i * HID + sub * 8, hi);
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         const float s = ds[k];
         if (s == 0.f || j > (int32_t)i) continue;
         if (j == (int32_t)i) {
#pragma unroll
            for (int q = 0; q < 8; ++q) dv[q] += s * hi[q];
            dc += s;
         }
         else {
            float hj[8];
            load8(h + (int64_t)j * HID + sub * 8, hj);
#pragma unroll
            for (int q = 0; q < 8; ++q) du[q] += s * hi[q] * hj[q];
         }
      }
   }
#pragma unroll
   for (int q = 0; q < 8; ++q) {
      red[threadIdx.x][q] = du[q];
      red[threadIdx.x][8 + q] = dv[q];
   }
   red[threadIdx.x][16] = sub == 0 ? dc : 0.f;
   __syncthreads();
   for (int o = threadIdx.x; o < HEADG; o += blockDim.x) {
      float s = 0.f;
      if (o < 2 * HID) {
         const int oo = o % HID, sb = oo / 8, q = oo % 8 + (o < HID ? 0 : 8);
         for (int t = sb; t < (int)blockDim.x; t += 8) s += red[t][q];
      }
      else {
         for (int t = 0; t < (int)blockDim.x; t += 8) s += red[t][16];
      }
      part[(int64_t)blockIdx.x * HEADG + o] = s;
   }
}

// grads[off + q] = sum over blocks of part[b * width + q]   (block order)
__global__ void lp_sum_parts(const float* part, int nblocks, int width, float* out)
{
   for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < width; q += gridDim.x * blockDim.x) {
      float s = 0.f;
      for (int b = 0; b < nblocks; ++b) s += part[(int64_t)b * width + q];
      out[q] = s;
   }
}

// dz = dH * (z > 0); also the BF16 copy for the data product
__global__ void lp_relu_back(int64_t total, const float* dH, const bf16* z, float* dz, bf16* dz16)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
      const float v = bf2f(z[t]) > 0.f ? dH[t] : 0.f;
      dz[t] = v;
      dz16[t] = __float2bfloat16(v);
   }
}

// dh_prev = dH (residual) + dcat[:, :64] + A~ dcat[:, 64:]
__global__ void lp_layer_back(int64_t n, const int32_t* rp, const int32_t* col, const float* at,
                              const float* dH, const float* dcat, float* dprev)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * HID; t += stride) {
      const int64_t i = t / HID;
      const int c = (int)(t % HID);
      float s = dH[t] + dcat[i * 2 * HID + c];
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const float a = at[k];
         if (a != 0.f) s += a * dcat[(int64_t)col[k] * 2 * HID + HID + c];
      }
      dprev[t] = s;
   }
}

// per-block partials of X^T dz with X = [x0 (k0 columns) | x1] and an
// implicit all-ones column KIN for the bias gradient: part[b][(KIN+1) x HID]
// (KIN = 0: the bias gradient alone)
template <int KIN, class XT, class ZT>
__global__ void __launch_bounds__(256) lp_wgrad(int64_t n, const XT* x0, int ld0, int k0,
                                                const XT* x1, int ld1, const ZT* dz, float* part)
{
   constexpr int W = (KIN + 1) * HID;
   float acc[(W + 255) / 256];
#pragma unroll
   for (int q = 0; q < (W + 255) / 256; ++q) acc[q] = 0.f;
   __shared__ float xs[KIN + 1];
   __shared__ float zs[HID];
   for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
      __syncthreads();
      for (int q = threadIdx.x; q < KIN; q += blockDim.x)
         xs[q] = q < k0 ? to_f(x0[i * ld0 + q]) : to_f(x1[i * ld1 + (q - k0)]);
      if (threadIdx.x == 0) xs[KIN] = 1.f;
      for (int q = threadIdx.x; q < HID; q += blockDim.x) zs[q] = to_f(dz[i * HID + q]);
      __syncthreads();
#pragma unroll
      for (int q = 0; q < (W + 255) / 256; ++q) {
         const int e = q * 256 + threadIdx.x;
         if (e < W) acc[q] += xs[e / HID] * zs[e % HID];
      }
   }
#pragma unroll
   for (int q = 0; q < (W + 255) / 256; ++q) {
      const int e = q * 256 + threadIdx.x;
      if (e < W) part[(int64_t)blockIdx.x * W + e] = acc[q];
   }
}

__global__ void lp_adam(float* P, const float* g, float* m1, float* m2, int np, float lr, float b1t,
                        float b2t)
{
   for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x) {
      const float gv = g[t];
      const float a = 0.9f * m1[t] + 0.1f * gv;
      const float b = 0.999f * m2[t] + 0.001f * gv * gv;
      m1[t] = a;
      m2[t] = b;
      P[t] -= lr * (a / (1.f - b1t)) / (sqrtf(b / (1.f - b2t)) + 1e-8f);
   }
}

}  // namespace

// backward pass for a batch of pairs, gradients into L->grads; returns loss
static double learned_backward(ofg_learned* L, ofg_matrix* A, LearnedGraph& G, const float* R,
                               const float* E, int64_t P)
{
   const int64_t n = A->n;
   const unsigned gr = grid_for(n, 256);
   const unsigned gp = grid_for(n * P, 256);
   DBuf<float> Z(n * P), Y(n * P), dY(n * P), dZ(n * P), en(P), dg(A->nnz), ds(A->nnz);
   DBuf<float> dH(n * HID), dprev(n * HID), dz(n * HID), dcat(n * 2 * HID);
   DBuf<bf16> dz16(n * HID);
   DBuf<double> loss(2), partials(((size_t)grid_for(std::max<int64_t>(n * P, n), kRedBlock, 8) + 1) * 2);
   DBuf<unsigned> counter(1);
   counter.zero();
   L->grads.zero();
   const int32_t* rp = A->row_ptr.p;
   const int32_t* col = A->col.p;
   lp_apply_lower<float><<<gp, 256, 0, stream()>>>(n, P, rp, col, G.g.p, R, Z.p);
   lp_sqnorms<<<(unsigned)P, kRedBlock, 0, stream()>>>(n, P, E, en.p);
   if (L->loss_kind == 0) {
      // mean_p ||G^T G r_p - e_p||^2 / ||e_p||^2
      lp_apply_upper<float><<<gp, 256, 0, stream()>>>(n, P, rp, col, G.tp.p, G.g.p, Z.p, Y.p);
      lp_loss<<<grid_for(n * P, kRedBlock, 8), kRedBlock, 0, stream()>>>(n, P, Y.p, E, en.p, dY.p,
                                                                         loss.p, partials.p,
                                                                         counter.p);
   }
   else {
      lp_apply_lower<float><<<gp, 256, 0, stream()>>>(n, P, rp, col, G.g.p, E, Y.p);  // G e
      lp_kap_loss<<<grid_for(std::max<int64_t>(n * P, n), kRedBlock, 8), kRedBlock, 0, stream()>>>(
         n, P, Z.p, Y.p, en.p, A->dpos.p, G.g.p, loss.p, partials.p, counter.p);
      lp_kap_dy<<<gp, 256, 0, stream()>>>(n, P, E, en.p, loss.p, dY.p);
   }
   lp_apply_lower<float><<<gp, 256, 0, stream()>>>(n, P, rp, col, G.g.p, dY.p, dZ.p);
   lp_dG<<<gr, 256, 0, stream()>>>(n, P, rp, col, R, Z.p, dY.p, dZ.p, dg.p);
   if (L->loss_kind != 0) lp_kap_diag<<<gr, 256, 0, stream()>>>(n, A->dpos.p, G.g.p, dg.p);
   const bf16* hN = G.hbuf(NLAYER);
   lp_dS<<<gr, 256, 0, stream()>>>(n, rp, col, G.at.p, G.dsq.p, hN, L->params.p, dg.p, ds.p);
   lp_head_back<<<grid_for(n * HID, 256), 256, 0, stream()>>>(n, rp, col, G.tp.p, hN, L->params.p,
                                                               ds.p, dH.p);
   const int nb = num_sms() * 2;
   {
      DBuf<float> part((size_t)nb * HEADG);
      lp_head_pgrad<<<nb, 256, 0, stream()>>>(n, rp, col, hN, ds.p, part.p);
      lp_sum_parts<<<1, 256, 0, stream()>>>(part.p, nb, HEADG, L->grads.p + P_U);
   }
   count_launch(11);
   // layers, last to first
   for (int l = NLAYER - 1; l >= 0; --l) {
      lp_relu_back<<<grid_for(n * HID, 256), 256, 0, stream()>>>(n * HID, dH.p, G.zbuf(l + 1), dz.p,
                                                                   dz16.p);
      BwdFunctor bf{dcat.p};
      GemmA a{dz16.p, HID, nullptr, 0, HID};
      run_gemm<HID, 2 * HID>(L, n, a, L->wb.p + (size_t)l * 2 * HID * HID, bf);
      {
         // weight and bias gradients from the BF16 copy of dz, the operand of
         // the data product: X^T dz on the tensor cores (or on CUDA cores, the
         // checker), the column sums of dz on CUDA cores
         constexpr int W = (2 * HID + 1) * HID;
         DBuf<float> tot(W);
         if (L->use_tc && n > 0) {
            const int smem = 2 * HID * 128 * 2 + HID * 128 * 2 + 64;
            static bool attr_set = false;
            if (!attr_set) {
               OFG_CUDA(cudaFuncSetAttribute(wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             smem));
               attr_set = true;
            }
            const unsigned gw =
               (unsigned)std::min<int64_t>((n + 127) / 128, (int64_t)num_sms() * 4);
            DBuf<float> pw((size_t)gw * 2 * HID * HID), pb((size_t)nb * HID);
            int* worked = prof_begin();
            wgrad_tc<<<gw, 128, smem, stream()>>>(n, GemmA{G.hbuf(l), HID, G.aggbuf(l), HID, HID},
                                                  dz16.p, pw.p, L->status.p, worked);
            prof_end(PROF_NET_GEMM, (double)n * (2 * HID * 2 + HID * 2) + 4.0 * gw * 2 * HID * HID);
            lp_wgrad<0, bf16, bf16><<<nb, 256, 0, stream()>>>(n, nullptr, 0, 0, nullptr, 0, dz16.p,
                                                              pb.p);
            lp_sum_parts<<<32, 256, 0, stream()>>>(pw.p, gw, 2 * HID * HID, tot.p);
            lp_sum_parts<<<1, 64, 0, stream()>>>(pb.p, nb, HID, tot.p + 2 * HID * HID);
            count_launch(2);
         }
         else {
            DBuf<float> part((size_t)nb * W);
            lp_wgrad<2 * HID, bf16, bf16><<<nb, 256, 0, stream()>>>(n, G.hbuf(l), HID, HID,
                                                                   G.aggbuf(l), HID, dz16.p,
                                                                   part.p);
            lp_sum_parts<<<32, 256, 0, stream()>>>(part.p, nb, W, tot.p);
         }
         // rows 0..127 -> W_l, row 128 -> b_l
         OFG_CUDA(cudaMemcpyAsync(L->grads.p + P_W + l * 2 * HID * HID, tot.p,
                                  sizeof(float) * 2 * HID * HID, cudaMemcpyDeviceToDevice, stream()));
         OFG_CUDA(cudaMemcpyAsync(L->grads.p + P_B + l * HID, tot.p + 2 * HID * HID,
                                  sizeof(float) * HID, cudaMemcpyDeviceToDevice, stream()));
      }
      lp_layer_back<<<grid_for(n * HID, 256), 256, 0, stream()>>>(n, rp, col, G.at.p, dH.p, dcat.p,
                                                                   dprev.p);
      std::swap(dH, dprev);
      count_launch(4);
   }
   // embedding
   lp_relu_back<<<grid_for(n * HID, 256), 256, 0, stream()>>>(n * HID, dH.p, G.zbuf(0), dz.p, dz16.p);
   {
      constexpr int W = (NFEAT + 1) * HID;
      DBuf<float> part((size_t)nb * W), tot(W);
      lp_wgrad<NFEAT, float, float><<<nb, 256, 0, stream()>>>(n, G.feat.p, NFEAT, NFEAT, G.feat.p,
                                                              NFEAT, dz.p, part.p);
      lp_sum_parts<<<4, 256, 0, stream()>>>(part.p, nb, W, tot.p);
      OFG_CUDA(cudaMemcpyAsync(L->grads.p + P_WIN, tot.p, sizeof(float) * NFEAT * HID,
                               cudaMemcpyDeviceToDevice, stream()));
      OFG_CUDA(cudaMemcpyAsync(L->grads.p + P_BIN, tot.p + NFEAT * HID, sizeof(float) * HID,
                               cudaMemcpyDeviceToDevice, stream()));
   }
   count_launch(3);
   OFG_LAUNCH_CHECK();
   double h = 0;
   loss.download(&h, 1);
   return h;
}

static void learned_check(ofg_learned* L)
{
   int h = 0;
   L->status.download(&h, 1);
   if (h) {
      L->status.zero();
      throw Error(OFG_ERR_TIMEOUT, "tensor-core GEMM wait ran out");
   }
}

static void cast_weights(ofg_learned* L)
{
   lp_cast_weights<<<64, 256, 0, stream()>>>(L->params.p, L->wt.p, L->wb.p);
   count_launch();
   OFG_LAUNCH_CHECK();
}

}  // namespace ofg

// ------------------------------------------------- the preconditioner -----
// G (lower rows, the diagonal included) and G^T (upper rows) become two
// matrices of their own on A's row count, so that both products run as
// SELL-32 SpMVs (FP64 values for the FP64 Krylov loops, FP32 for the mixed
// one).  The network's buffers for the matrix are kept with the
// preconditioner (the pattern-only parts are computed once).
namespace ofg {
namespace {

__global__ void lp_tri_counts(int64_t n, const int32_t* rp, const int32_t* col, int64_t* lenL,
                              int64_t* lenU)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      int64_t l = 0, u = 0;
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         l += col[k] <= (int32_t)i;
         u += col[k] >= (int32_t)i;
      }
      lenL[i] = l;
      lenU[i] = u;
   }
   if (blockIdx.x == 0 && threadIdx.x == 0) lenL[n] = lenU[n] = 0;
}

__global__ void lp_to_i32(int64_t n, const int64_t* a, int32_t* b)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      b[i] = (int32_t)a[i];
}

// values (and on the first call the columns) of G and G^T from the head's
// output g (stored at A's lower positions) and the transposed positions tp
__global__ void lp_tri_fill(int64_t n, const int32_t* rp, const int32_t* col, const int32_t* tp,
                            const float* g, const int32_t* rpL, int32_t* colL, double* valL,
                            const int32_t* rpU, int32_t* colU, double* valU)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      int32_t l = rpL[i], u = rpU[i];
      for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
         const int32_t j = col[k];
         if (j <= (int32_t)i) {
            colL[l] = j;
            valL[l++] = (double)g[k];
         }
         if (j >= (int32_t)i) {
            const int32_t q = (j == (int32_t)i) ? k : tp[k];
            colU[u] = j;
            valU[u++] = q >= 0 ? (double)g[q] : 0.0;
         }
      }
   }
}

__global__ void __launch_bounds__(kRedBlock) lp_dot(int64_t n, const double* a, const double* b,
                                                    double* out, double* partials,
                                                    unsigned* counter, const int* skip)
{
   if (skip && *skip) return;
   double v[1] = {0.0};
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      v[0] += a[i] * b[i];
   double t[1];
   if (grid_reduce<1>(v, partials, counter, t)) *out = t[0];
}

ofg_matrix* tri_matrix(int64_t n, const DBuf<int64_t>& len)
{
   auto M = new ofg_matrix();
   M->n = n;
   DBuf<int64_t> rp64(n + 1);
   scan_exclusive_i64(len.p, rp64.p, n + 1);
   M->row_ptr.alloc(n + 1);
   lp_to_i32<<<grid_for(n + 1, 256), 256, 0, stream()>>>(n + 1, rp64.p, M->row_ptr.p);
   count_launch();
   OFG_LAUNCH_CHECK();
   int64_t nnz = 0;
   OFG_CUDA(cudaMemcpyAsync(&nnz, rp64.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, stream()));
   OFG_CUDA(cudaStreamSynchronize(stream()));
   M->nnz = nnz;
   M->col.alloc(nnz > 0 ? nnz : 1);
   M->val.alloc(nnz > 0 ? nnz : 1);
   return M;
}

std::vector<std::pair<const ofg_prec*, LearnedGraph*>> g_graphs;

LearnedGraph* graph_of(const ofg_prec* P)
{
   for (auto& e : g_graphs)
      if (e.first == P) return e.second;
   g_graphs.push_back({P, new LearnedGraph()});
   return g_graphs.back().second;
}

}  // namespace

void learned_release(const ofg_prec* P)
{
   for (size_t q = 0; q < g_graphs.size(); ++q)
      if (g_graphs[q].first == P) {
         delete g_graphs[q].second;
         g_graphs.erase(g_graphs.begin() + q);
         return;
      }
}

void learned_setup(ofg_prec* P)
{
   OFG_REQUIRE(P->net, OFG_ERR_ARG, "learned preconditioner without a network");
   ofg_matrix* A = P->A;
   const int64_t n = A->n;
   LearnedGraph& G = *graph_of(P);
   graph_prepare(A, G, false);
   learned_forward(P->net, A, G);
   learned_check(P->net);
   const unsigned gr = grid_for(n, 256);
   if (!P->gl) {
      DBuf<int64_t> lenL(n + 1), lenU(n + 1);
      lp_tri_counts<<<gr, 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p, lenL.p, lenU.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      P->gl = tri_matrix(n, lenL);
      P->gu = tri_matrix(n, lenU);
      P->t.alloc(n > 0 ? n : 1);
      P->partials.alloc(((size_t)grid_for(n, kRedBlock, 8) + 1) * 2);
      P->counter.alloc(1);
      P->counter.zero();
   }
   lp_tri_fill<<<gr, 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p, G.tp.p, G.g.p, P->gl->row_ptr.p,
                                         P->gl->col.p, P->gl->val.p, P->gu->row_ptr.p,
                                         P->gu->col.p, P->gu->val.p);
   count_launch();
   OFG_LAUNCH_CHECK();
   P->gl->version++;
   P->gu->version++;
   ensure_sell(P->gl);
   ensure_sell(P->gu);
}

void learned_apply(ofg_prec* P, const double* r, double* z, double* rz, const int* skip)
{
   const int64_t n = P->A->n;
   spmv_sell(P->gl, r, P->t.p, skip);  // t = G r
   spmv_sell(P->gu, P->t.p, z, skip);  // z = G^T t
   if (rz && r != z) {
      lp_dot<<<grid_for(n, kRedBlock, 8), kRedBlock, 0, stream()>>>(n, r, z, rz, P->partials.p,
                                                                     P->counter.p, skip);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
}

}  // namespace ofg

using namespace ofg;

extern "C" {

int ofg_learned_create(uint64_t seed, ofg_learned** out)
{
   return guarded("ofg_learned_create", [&] {
      OFG_REQUIRE(out, OFG_ERR_ARG, "null argument");
      auto L = new ofg_learned();
      L->params.alloc(NPARAM);
      L->grads.alloc(NPARAM);
      L->m1.alloc(NPARAM);
      L->m2.alloc(NPARAM);
      L->m1.zero();
      L->m2.zero();
      L->grads.zero();
      L->wt.alloc((size_t)NLAYER * 2 * HID * HID);
      L->wb.alloc((size_t)NLAYER * 2 * HID * HID);
      L->status.alloc(1);
      L->status.zero();
      lp_init_params<<<64, 256, 0, stream()>>>(L->params.p, seed);
      count_launch();
      cast_weights(L);
      OFG_CUDA(cudaStreamSynchronize(stream()));
      *out = L;
   });
}

int ofg_learned_destroy(ofg_learned* L)
{
   return guarded("ofg_learned_destroy", [&] {
      delete L;
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_learned_num_params(void) { return NPARAM; }

int ofg_learned_get_params(const ofg_learned* L, float* params, float* adam_m, float* adam_v,
                           int64_t* step)
{
   return guarded("ofg_learned_get_params", [&] {
      OFG_REQUIRE(L && params, OFG_ERR_ARG, "null argument");
      L->params.download(params, NPARAM);
      if (adam_m) L->m1.download(adam_m, NPARAM);
      if (adam_v) L->m2.download(adam_v, NPARAM);
      if (step) *step = L->step;
   });
}

int ofg_learned_set_params(ofg_learned* L, const float* params, const float* adam_m,
                           const float* adam_v, int64_t step)
{
   return guarded("ofg_learned_set_params", [&] {
      OFG_REQUIRE(L && params, OFG_ERR_ARG, "null argument");
      L->params.upload(params, NPARAM);
      if (adam_m) L->m1.upload(adam_m, NPARAM);
      if (adam_v) L->m2.upload(adam_v, NPARAM);
      L->step = step;
      cast_weights(L);
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_learned_set_tensor_cores(ofg_learned* L, int on)
{
   return guarded("ofg_learned_set_tensor_cores", [&] {
      OFG_REQUIRE(L, OFG_ERR_ARG, "null argument");
      L->use_tc = on ? 1 : 0;
   });
}

int ofg_learned_set_loss(ofg_learned* L, int kind)
{
   return guarded("ofg_learned_set_loss", [&] {
      OFG_REQUIRE(L && (kind == 0 || kind == 1), OFG_ERR_ARG, "loss kind must be 0 or 1");
      L->loss_kind = kind;
   });
}

int ofg_learned_train(ofg_learned* L, ofg_matrix* A, const float* R, const float* E, int npairs,
                      int steps, int batch, float lr, float* loss_history)
{
   return guarded("ofg_learned_train", [&] {
      OFG_REQUIRE(L && A && R && E && npairs > 0 && batch > 0 && batch <= npairs && steps >= 0,
                  OFG_ERR_ARG, "bad training arguments");
      const int64_t n = A->n;
      In<float> dR(R, (size_t)npairs * n), dE(E, (size_t)npairs * n);
      LearnedGraph G;
      graph_prepare(A, G, true);
      const int nbatches = npairs / batch;
      for (int s = 0; s < steps; ++s) {
         const int64_t p0 = (int64_t)(s % nbatches) * batch;
         learned_forward(L, A, G);
         const double loss = learned_backward(L, A, G, dR.d + p0 * n, dE.d + p0 * n, batch);
         learned_check(L);
         L->step++;
         const float b1t = powf(0.9f, (float)L->step), b2t = powf(0.999f, (float)L->step);
         lp_adam<<<64, 256, 0, stream()>>>(L->params.p, L->grads.p, L->m1.p, L->m2.p, NPARAM, lr,
                                           b1t, b2t);
         count_launch();
         cast_weights(L);
         if (loss_history) loss_history[s] = (float)loss;
      }
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_learned_grad(ofg_learned* L, ofg_matrix* A, const float* R, const float* E, int npairs,
                     double* loss, float* grads, float* factor)
{
   return guarded("ofg_learned_grad", [&] {
      OFG_REQUIRE(L && A && R && E && loss && npairs > 0, OFG_ERR_ARG, "null argument");
      const int64_t n = A->n;
      In<float> dR(R, (size_t)npairs * n), dE(E, (size_t)npairs * n);
      LearnedGraph G;
      graph_prepare(A, G, true);
      learned_forward(L, A, G);
      *loss = learned_backward(L, A, G, dR.d, dE.d, npairs);
      learned_check(L);
      if (grads) L->grads.download(grads, NPARAM);
      if (factor) G.g.download(factor, A->nnz);
   });
}

int ofg_prec_create_learned(ofg_learned* L, ofg_matrix* A, ofg_prec** out)
{
   return guarded("ofg_prec_create_learned", [&] {
      OFG_REQUIRE(L && A && out, OFG_ERR_ARG, "null argument");
      auto P = new ofg_prec();
      P->A = A;
      P->type = OFG_LEARNED;
      P->net = L;
      try {
         prec_setup(P);
      }
      catch (...) {
         delete P;
         throw;
      }
      OFG_CUDA(cudaStreamSynchronize(stream()));
      *out = P;
   });
}

// The same layer product on the tensor cores and on CUDA cores, for the test
// of the tensor-core path: out_tc, out_cc (rows x 64 FP32) = X (rows x 128,
// BF16 bit patterns) times layer `layer`'s weights.
int ofg_learned_gemm_check(ofg_learned* L, int layer, int64_t rows, const uint16_t* X,
                           float* out_tc, float* out_cc)
{
   return guarded("ofg_learned_gemm_check", [&] {
      OFG_REQUIRE(L && X && out_tc && out_cc && rows > 0 && layer >= 0 && layer < NLAYER,
                  OFG_ERR_ARG, "bad arguments");
      In<uint16_t> dX(X, (size_t)rows * 2 * HID);
      DBuf<float> a(rows * HID), b(rows * HID);
      const int saved = L->use_tc;
      const bf16* w = L->wt.p + (size_t)layer * 2 * HID * HID;
      const bf16* x = reinterpret_cast<const bf16*>(dX.d);
      GemmA op{x, 2 * HID, x + HID, 2 * HID, HID};  // the two halves of each row
      L->use_tc = 1;
      run_gemm<2 * HID, HID>(L, rows, op, w, StoreFunctor{a.p, HID});
      L->use_tc = 0;
      run_gemm<2 * HID, HID>(L, rows, op, w, StoreFunctor{b.p, HID});
      L->use_tc = saved;
      learned_check(L);
      a.download(out_tc, rows * HID);
      b.download(out_cc, rows * HID);
   });
}

}  // extern "C"
