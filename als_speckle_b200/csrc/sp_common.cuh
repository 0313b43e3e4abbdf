// Shared host-side helpers of libspeckle_b200: status/error reporting and the
// per-device twiddle tables.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/speckle_b200.h"

namespace sp {

// Record a failure message for sp_last_error() (thread-local).
void set_error(const char* fmt, ...);

inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
inline int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

// Device address of the twiddle tables of the current device, uploading them
// on first use.  Table for size N (power of two, 2..4096) starts at entry N:
// tw[N + x] = exp(-2 pi i x / N), x in [0, N).
cudaError_t twiddles(const float2** out);

#define SP_CUDA_TRY(expr)                                                              \
  do {                                                                                 \
    cudaError_t _e = (expr);                                                           \
    if (_e != cudaSuccess) {                                                           \
      ::sp::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, \
                      __LINE__);                                                       \
      return SP_ERR_CUDA;                                                              \
    }                                                                                  \
  } while (0)

#define SP_CHECK(cond, status, ...)  \
  do {                               \
    if (!(cond)) {                   \
      ::sp::set_error(__VA_ARGS__);  \
      return (status);               \
    }                                \
  } while (0)

inline cudaStream_t as_stream(sp_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// The fused engine (sp_engine.cu); `concurrent` allows the per-size launch
// chains to run on forked auxiliary streams.
int engine_run(const sp_trial* trials, int n_trials, void* workspace_dev, size_t workspace_bytes,
               const sp_run_opts* opts, sp_stream_t stream, bool concurrent);

constexpr int kMaxN = 4096;
constexpr int kMinN = 8;
constexpr int kThreads = 256;  // every engine/FFT CTA
}  // namespace sp
