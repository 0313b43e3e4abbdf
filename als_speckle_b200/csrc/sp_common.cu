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
// uploaded once per device by cudaMemcpyToSymbol; nothing is allocated.
__device__ __align__(256) float2 g_twiddle[2 * kMaxN];

static std::mutex g_tw_mutex;
static bool g_tw_ready[256];
static const float2* g_tw_addr[256];

cudaError_t twiddles(const float2** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  if (!g_tw_ready[dev]) {
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
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_twiddle);
    if (e != cudaSuccess) return e;
    g_tw_addr[dev] = static_cast<const float2*>(p);
    g_tw_ready[dev] = true;
  }
  *out = g_tw_addr[dev];
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
