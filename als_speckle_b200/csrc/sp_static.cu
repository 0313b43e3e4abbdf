// sp_engine_run_static: the fused engine for callers that cannot allocate
// device memory.
//
// sp_engine_run needs a scratch workspace (descriptor tables and one Fourier
// work plane per trial) that the caller allocates.  Some callers cannot do
// that: code running inside a host framework that owns every device
// allocation and hands out only the buffers it created, plugins whose
// allocator is not reachable from the thread that drives the GPU, or callers
// that must not allocate after start-up for determinism.  For them this entry
// point takes its scratch from a fixed array in device memory that belongs to
// this library, and never allocates.
//
// The array is kStaticScratchBytes (48 MiB).  A device holds it from the
// moment this library's device code is loaded there -- at the latest the
// first sp_engine_run_static call on that device (with CUDA's default lazy
// module loading), at library load with CUDA_MODULE_LOADING=EAGER -- until
// the process exits.  Requests whose workspace would exceed it
// are rejected with SP_ERR_SIZE before any work is enqueued.
#include <cstring>

#include "sp_common.cuh"

namespace sp {

constexpr size_t kStaticScratchBytes = (size_t)48 << 20;

// The scratch itself.  Host code must not use this name as an address: on the
// host it is only a stand-in, so its device address is looked up with
// cudaGetSymbolAddress and that pointer is what gets passed on.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch in the current context, looked up on
// every call (cheap beside an engine run; a cached address would outlive a
// context that is reset and created again).
static cudaError_t static_scratch(void** out) {
  return cudaGetSymbolAddress(out, g_static_scratch);
}

}  // namespace sp

using namespace sp;

extern "C" int sp_engine_run_static(const sp_trial* trials, int n_trials, const sp_run_opts* opts,
                                    sp_stream_t stream) {
  SP_CHECK(n_trials >= 0, SP_ERR_INVALID, "n_trials < 0");
  if (n_trials == 0) return SP_OK;
  SP_CHECK(trials != nullptr, SP_ERR_INVALID, "trials is null");
  size_t need = 0;
  const int st = sp_engine_workspace_size(trials, n_trials, &need);
  if (st != SP_OK) return st;
  SP_CHECK(need <= kStaticScratchBytes, SP_ERR_SIZE,
           "sp_engine_run_static: these trials need %zu bytes of scratch, more than the "
           "%zu-byte static array; use sp_engine_run with a caller-allocated workspace",
           need, kStaticScratchBytes);
  void* scratch = nullptr;
  SP_CUDA_TRY(static_scratch(&scratch));
  // Eager launches only: the graphs cached by sp_engine_run are keyed by the
  // workspace address and are not wanted for this shared array.
  sp_run_opts o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  o.use_graph = 0;
  // Nothing in the scratch needs to start at zero: the descriptor tables are
  // written by sp_engine_run on every call and each work plane is written
  // before it is read.
  // The launch chains of different sizes stay on the caller's stream here
  // (concurrent chains would create auxiliary streams and events).
  return engine_run(trials, n_trials, scratch, kStaticScratchBytes, &o, stream, false);
}
