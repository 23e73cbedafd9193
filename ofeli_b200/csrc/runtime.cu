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
bool g_pool_ready[64] = {};
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

// The device's default pool keeps freed blocks, so that the per-call scratch
// allocations are served without returning memory to the driver at every
// synchronisation (and mapping it again at the next call).  Done once per
// device, whichever stream the library runs on.
static void configure_pool(int d)
{
   if (g_pool_ready[d]) return;
   std::lock_guard<std::mutex> lk(g_mu);
   if (g_pool_ready[d]) return;
   cudaMemPool_t pool;
   OFG_CUDA(cudaDeviceGetDefaultMemPool(&pool, d));
   uint64_t keep = UINT64_MAX;
   OFG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
   g_pool_ready[d] = true;
}

cudaStream_t stream()
{
   int d = current_device();
   configure_pool(d);
   if (g_user_stream_set) return g_user_stream;
   if (!g_own_stream[d]) {
      std::lock_guard<std::mutex> lk(g_mu);
      if (!g_own_stream[d])
         OFG_CUDA(cudaStreamCreateWithFlags(&g_own_stream[d], cudaStreamNonBlocking));
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

// ------------------------------------------------------------ profiling --
namespace {
struct ProfRec {
   int id;
   cudaEvent_t a, b;
   double bytes;
   int slot;
};
constexpr int kProfSlots = 8192;
int* g_flags = nullptr;  // device, one "did work" flag per pending launch
int g_open_slot = -1;
struct ProfTot {
   int64_t launches = 0;
   double ms = 0.0, bytes = 0.0;
};
bool g_prof = false;
std::vector<ProfRec> g_pending;
std::vector<cudaEvent_t> g_pool;
ProfTot g_tot[kProfKinds];
cudaEvent_t g_open_a = nullptr;

cudaEvent_t take_event()
{
   if (g_pool.empty()) {
      cudaEvent_t e;
      OFG_CUDA(cudaEventCreate(&e));
      return e;
   }
   cudaEvent_t e = g_pool.back();
   g_pool.pop_back();
   return e;
}
}  // namespace

bool prof_on() { return g_prof; }

int g_prof_every = 1;
int64_t g_prof_seen = 0;

int* prof_begin()
{
   if (!g_prof) return nullptr;
   if (g_prof_every > 1 && (g_prof_seen++ % g_prof_every) != 0) return nullptr;
   if (!g_flags) {
      OFG_CUDA(cudaMalloc(&g_flags, kProfSlots * sizeof(int)));
      OFG_CUDA(cudaMemset(g_flags, 0, kProfSlots * sizeof(int)));
   }
   if ((int)g_pending.size() >= kProfSlots) prof_collect();
   g_open_slot = (int)g_pending.size();
   OFG_CUDA(cudaMemsetAsync(g_flags + g_open_slot, 0, sizeof(int), stream()));
   g_open_a = take_event();
   OFG_CUDA(cudaEventRecord(g_open_a, stream()));
   return g_flags + g_open_slot;
}

void prof_end(int id, double bytes)
{
   if (!g_prof || !g_open_a) return;
   cudaEvent_t b = take_event();
   OFG_CUDA(cudaEventRecord(b, stream()));
   g_pending.push_back({id, g_open_a, b, bytes, g_open_slot});
   g_open_a = nullptr;
   g_open_slot = -1;
}

void prof_collect()
{
   if (g_pending.empty()) return;
   std::vector<int> flags(g_pending.size(), 0);
   OFG_CUDA(cudaStreamSynchronize(stream()));
   OFG_CUDA(cudaMemcpy(flags.data(), g_flags, flags.size() * sizeof(int), cudaMemcpyDeviceToHost));
   for (auto& r : g_pending) {
      float ms = 0.f;
      OFG_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
      if (flags[r.slot]) {
         g_tot[r.id].launches++;
         g_tot[r.id].ms += ms;
         g_tot[r.id].bytes += r.bytes;
      }
      g_pool.push_back(r.a);
      g_pool.push_back(r.b);
   }
   g_pending.clear();
}

static const char* kProfNames[kProfKinds] = {"spmv64",   "spmv32",       "spmv16",
                                             "sweep",    "assembly",     "network_gemm",
                                             "learned_apply", "gram_schmidt"};

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

int ofg_init(int device)
{
   return ofg::guarded("ofg_init", [&] {
      OFG_REQUIRE(device >= 0, OFG_ERR_ARG, "device must be >= 0");
      OFG_CUDA(cudaSetDevice(device));
      OFG_CUDA(cudaStreamSynchronize(ofg::stream()));
      ofg::noalloc_prepare();
   });
}

int ofg_shutdown(void)
{
   return ofg::guarded("ofg_shutdown", [&] {
      OFG_CUDA(cudaStreamSynchronize(ofg::stream()));
      ofg::prof_collect();
      ofg::meshio_release_staging();
   });
}

int ofg_profile_enable(int on)
{
   return ofg::guarded("ofg_profile_enable", [&] {
      ofg::prof_collect();
      for (auto& t : ofg::g_tot) t = ofg::ProfTot();
      ofg::g_prof = on != 0;
      ofg::g_prof_every = on > 1 ? on : 1;
      ofg::g_prof_seen = 0;
   });
}

int ofg_profile_read(const char* name, int64_t* launches, double* total_ms, double* bytes)
{
   return ofg::guarded("ofg_profile_read", [&] {
      OFG_REQUIRE(name, OFG_ERR_ARG, "null name");
      ofg::prof_collect();
      for (int i = 0; i < ofg::kProfKinds; ++i)
         if (std::string(name) == ofg::kProfNames[i]) {
            if (launches) *launches = ofg::g_tot[i].launches;
            if (total_ms) *total_ms = ofg::g_tot[i].ms;
            if (bytes) *bytes = ofg::g_tot[i].bytes;
            return;
         }
      throw ofg::Error(OFG_ERR_ARG, std::string("unknown kernel family ") + name);
   });
}

}  // extern "C"
