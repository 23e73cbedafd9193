// runtime.cu -- last-error reporting, the library stream, launch accounting
// and host/device pointer classification.
#include <atomic>
#include <mutex>

#include "common.cuh"

namespace ofg {

namespace {
thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};
cudaStream_t g_user_stream = nullptr;
bool g_user_stream_set = false;
cudaStream_t g_own_stream[64] = {};
int g_sms[64] = {};
std::mutex g_mu;

int current_device()
{
   int d = 0;
   OFG_CUDA(cudaGetDevice(&d));
   if (d < 0 || d >= 64) throw Error(OFG_ERR_ARG, "device index out of range");
   return d;
}
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

cudaStream_t stream()
{
   if (g_user_stream_set) return g_user_stream;
   int d = current_device();
   if (!g_own_stream[d]) {
      std::lock_guard<std::mutex> lk(g_mu);
      if (!g_own_stream[d]) {
         // The pool keeps freed blocks so that per-call scratch allocations
         // are served without returning to the driver.
         cudaMemPool_t pool;
         OFG_CUDA(cudaDeviceGetDefaultMemPool(&pool, d));
         uint64_t keep = UINT64_MAX;
         OFG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
         OFG_CUDA(cudaStreamCreateWithFlags(&g_own_stream[d], cudaStreamNonBlocking));
      }
   }
   return g_own_stream[d];
}

int num_sms()
{
   int d = current_device();
   if (!g_sms[d]) OFG_CUDA(cudaDeviceGetAttribute(&g_sms[d], cudaDevAttrMultiProcessorCount, d));
   return g_sms[d];
}

void count_launch(int n) { g_launches += n; }

bool is_device_ptr(const void* p)
{
   cudaPointerAttributes at;
   cudaError_t e = cudaPointerGetAttributes(&at, p);
   if (e != cudaSuccess) {
      cudaGetLastError();
      return false;
   }
   return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

}  // namespace ofg

extern "C" {

const char* ofg_last_error(void) { return ofg::g_last_error.c_str(); }

const char* ofg_version(void) { return "ofeli_b200 0.1 (sm_100a)"; }

int ofg_set_stream(void* s)
{
   ofg::g_user_stream = (cudaStream_t)s;
   ofg::g_user_stream_set = s != nullptr;
   return OFG_OK;
}

void* ofg_get_stream(void)
{
   void* s = nullptr;
   ofg::guarded("ofg_get_stream", [&] { s = (void*)ofg::stream(); });
   return s;
}

int64_t ofg_launch_count(void) { return ofg::g_launches.load(); }

}  // extern "C"
