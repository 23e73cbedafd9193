// common.cuh -- runtime plumbing shared by the libofeli_gpu.so sources:
// status/error reporting, the per-device stream, device buffers, host/device
// pointer staging, launch accounting and small device helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ofeli_gpu.h"

namespace ofg {

// ----------------------------------------------------------------- errors --
struct Error : std::runtime_error {
   int code;
   Error(int c, const std::string& m) : std::runtime_error(m), code(c) { }
};

void set_last_error(const std::string& msg);

#define OFG_CUDA(call)                                                                   \
   do {                                                                                  \
      cudaError_t e_ = (call);                                                           \
      if (e_ != cudaSuccess)                                                             \
         throw ::ofg::Error(OFG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
   } while (0)

#define OFG_REQUIRE(cond, code, msg)                    \
   do {                                                 \
      if (!(cond)) throw ::ofg::Error((code), (msg));   \
   } while (0)

// Runs f, converting exceptions into a status code + last-error message.
template <class F>
int guarded(const char* fn, F&& f)
{
   try {
      f();
      return OFG_OK;
   }
   catch (const Error& e) {
      set_last_error(std::string(fn) + ": " + e.what());
      return e.code;
   }
   catch (const std::bad_alloc&) {
      set_last_error(std::string(fn) + ": host allocation failed");
      return OFG_ERR_NOMEM;
   }
   catch (const std::exception& e) {
      set_last_error(std::string(fn) + ": " + e.what());
      return OFG_ERR_ARG;
   }
}

// ----------------------------------------------------------- stream, count --
cudaStream_t stream();
// frees the mesh-file reader's pinned staging buffer (meshio.cu)
void meshio_release_staging();
int num_sms();
void count_launch(int n = 1);
// loads the no-allocation solver's code and scratch array on the current device
void noalloc_prepare();

#define OFG_LAUNCH_CHECK() OFG_CUDA(cudaGetLastError())

// Optional CUDA-event timing of kernel families (ofg_profile_enable):
// prof_begin() before a launch returns a device flag the kernel sets when it
// does work (kernels that can be skipped by a device-side stop flag), or
// nullptr when profiling is off; prof_end(kind, algorithmic bytes) after the
// launch.  Launches that found their stop flag set are not counted.
enum { PROF_SPMV64 = 0, PROF_SPMV32 = 1, PROF_SPMV16 = 2, PROF_SWEEP = 3, PROF_ASSEMBLY = 4,
       PROF_NET_GEMM = 5, PROF_LEARNED_APPLY = 6, PROF_ORTH = 7, kProfKinds = 8 };
bool prof_on();
int* prof_begin();
void prof_end(int kind, double bytes);
void prof_collect();

__device__ __forceinline__ void prof_mark(int* worked)
{
   if (worked && blockIdx.x == 0 && threadIdx.x == 0) *worked = 1;
}

// ---------------------------------------------------------------- buffers --
// Owning device allocation (stream-ordered on the library stream).
template <class T>
struct DBuf {
   T* p = nullptr;
   size_t n = 0;
   DBuf() = default;
   explicit DBuf(size_t count) { alloc(count); }
   DBuf(const DBuf&) = delete;
   DBuf& operator=(const DBuf&) = delete;
   DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
   DBuf& operator=(DBuf&& o) noexcept
   {
      if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
      return *this;
   }
   ~DBuf() { release(); }
   void alloc(size_t count)
   {
      release();
      n = count;
      if (count) OFG_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), stream()));
   }
   // grows (never shrinks); contents are not preserved
   void reserve(size_t count)
   {
      if (count > n) alloc(count);
   }
   void release()
   {
      if (p) cudaFreeAsync(p, stream());
      p = nullptr;
      n = 0;
   }
   void zero()
   {
      if (n) OFG_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), stream()));
   }
   void upload(const T* h, size_t count)
   {
      OFG_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyDefault, stream()));
   }
   void download(T* h, size_t count) const
   {
      OFG_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDefault, stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
   }
   std::vector<T> to_host(size_t count) const
   {
      std::vector<T> h(count);
      if (count) download(h.data(), count);
      return h;
   }
};

// True when p is memory the current device can address directly.
bool is_device_ptr(const void* p);

// Input view of a user vector: device pointers pass through, host data is
// copied to a scratch buffer.
template <class T>
struct In {
   const T* d = nullptr;
   DBuf<T> tmp;
   In(const T* user, size_t count)
   {
      if (!user) return;
      if (is_device_ptr(user)) { d = user; return; }
      tmp.alloc(count);
      tmp.upload(user, count);
      d = tmp.p;
   }
};

// In/out view of a user vector: host data is staged in and copied back by
// finish().
template <class T>
struct InOut {
   T* user;
   T* d = nullptr;
   size_t count;
   bool host = false;
   DBuf<T> tmp;
   InOut(T* u, size_t c, bool copy_in) : user(u), count(c)
   {
      if (!u) return;
      if (is_device_ptr(u)) { d = u; return; }
      host = true;
      tmp.alloc(c);
      if (copy_in) tmp.upload(u, c);
      d = tmp.p;
   }
   void finish()
   {
      if (host && count) tmp.download(user, count);
      else OFG_CUDA(cudaStreamSynchronize(stream()));
   }
};

// ----------------------------------------------- programmatic dependent launch
// A kernel launched with launch_pdl may start while the previous kernel of
// the stream drains; it must call pdl_wait() before touching anything the
// previous kernels write (pdl_wait returns once they completed and their
// memory is visible), and calls pdl_release() to let its own successor start.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;"); }

template <typename... KArgs, typename... Args>
void launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, Args... args)
{
   cudaLaunchConfig_t cfg = {};
   cfg.gridDim = dim3(grid);
   cfg.blockDim = dim3(block);
   cfg.dynamicSmemBytes = 0;
   cfg.stream = stream();
   cudaLaunchAttribute attr[1];
   attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
   attr[0].val.programmaticStreamSerializationAllowed = 1;
   cfg.attrs = attr;
   cfg.numAttrs = 1;
   OFG_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
   count_launch();
}

inline unsigned grid_for(int64_t work, int block, int max_blocks_per_sm = 8)
{
   int64_t g = (work + block - 1) / block;
   int64_t cap = (int64_t)num_sms() * max_blocks_per_sm;
   if (g > cap) g = cap;
   if (g < 1) g = 1;
   return (unsigned)g;
}

// ------------------------------------------------------- device helpers ---
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

__device__ __forceinline__ float warp_sumf(float v)
{
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

// Relaxed GPU-scope loads/stores that bypass the (non-coherent) L1.
__device__ __forceinline__ double ld_relaxed(const double* p)
{
   double v;
   asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
   return v;
}
__device__ __forceinline__ float ld_relaxed(const float* p)
{
   float v;
   asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
   return v;
}
__device__ __forceinline__ void st_relaxed(double* p, double v)
{
   asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(float* p, float v)
{
   asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

}  // namespace ofg
