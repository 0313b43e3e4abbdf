// Status strings, thread-local error text and per-device twiddle tables.
#include <cmath>
#include <cstdarg>
#include <mutex>
#include <vector>

#include "sp_common.cuh"

namespace sp {

static thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

// Twiddle tables live in a file-scope device array: 64 KiB per device,
// uploaded once per CUDA context by cudaMemcpyToSymbol; nothing is allocated.
__device__ __align__(256) float2 g_twiddle[2 * kMaxN];

// Identity of the calling thread's current CUDA context, unique over the
// life of the process (cuCtxGetId), reached through the runtime's driver
// entry points so the library does not link libcuda.  0 if unavailable.
unsigned long long current_context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || ctx == nullptr || get_id(ctx, &id) != 0)
    return 0;
  return id;
}

// The tables are uploaded once per CUDA context (a context that is destroyed
// and created again, e.g. after cudaDeviceReset, gets a fresh module and is
// uploaded again); the address is looked up on every call.
static std::mutex g_tw_mutex;
static std::vector<unsigned long long> g_tw_contexts;

cudaError_t twiddles(const float2** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_twiddle);  // also creates the context if needed
  if (e != cudaSuccess) return e;
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  bool ready = false;
  for (unsigned long long c : g_tw_contexts) ready = ready || (ctx != 0 && c == ctx);
  if (!ready) {
    std::vector<float2> host(2 * kMaxN, make_float2(0.f, 0.f));
    for (int N = 2; N <= kMaxN; N *= 2) {
      for (int x = 0; x < N; ++x) {
        // exact-rounded float of exp(-2 pi i x/N): evaluate in long double
        long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)x / N;
        host[N + x] = make_float2((float)cosl(a), (float)sinl(a));
      }
    }
    e = cudaMemcpyToSymbol(g_twiddle, host.data(), sizeof(float2) * host.size());
    if (e != cudaSuccess) return e;
    if (ctx != 0) g_tw_contexts.push_back(ctx);
  }
  *out = static_cast<const float2*>(p);
  return cudaSuccess;
}

}  // namespace sp

extern "C" {

int sp_version(void) { return 100; }

const char* sp_status_string(int status) {
  switch (status) {
    case SP_OK: return "ok";
    case SP_ERR_INVALID: return "invalid argument";
    case SP_ERR_SIZE: return "unsupported size";
    case SP_ERR_CUDA: return "CUDA error";
    case SP_ERR_WORKSPACE: return "workspace too small";
    case SP_ERR_UNSUPPORTED: return "unsupported";
    case SP_ERR_NOT_FOUND: return "not found";
    default: return "unknown status";
  }
}

const char* sp_last_error(void) { return sp::g_last_error; }

int sp_device_init(void) {
  const float2* tw = nullptr;
  SP_CUDA_TRY(sp::twiddles(&tw));
  return SP_OK;
}

}  // extern "C"
