// Per-size engine kernels.  Each size N is compiled in its own translation
// unit (sp_engine_n<N>.cu) so register allocation is per (N, E) and the build
// parallelises; the host engine reaches them through launch_pass().
#pragma once
#include "sp_engine_kernels.cuh"

namespace sp {

struct PassArgs {
  const Slot* slots;
  const Item* items;
  int n_items;
  const int* tick_base;  // optional device counter added to tick_off
  int tick_off;
  const float2* tw;
};

// Copy one slot descriptor into shared memory (word by word).
__device__ __forceinline__ void load_slot(Slot* dst, const Slot* __restrict__ src) {
  static_assert(sizeof(Slot) % 4 == 0, "slot size");
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
  for (int w = threadIdx.x; w < (int)(sizeof(Slot) / 4); w += blockDim.x) d[w] = s[w];
}

// E = 32 keeps 64 registers of line data per thread plus the prefetched
// psi/support: one 256-thread CTA per SM with up to 255 registers.  E = 16
// halves that and runs two CTAs per SM.
constexpr int min_blocks_for(int E) { return E >= 32 ? 1 : 2; }

// Stage the N-entry twiddle table of this size in shared memory (once per
// persistent CTA); returns its address.
template <int N, int E>
__device__ __forceinline__ const float2* stage_twiddles(float2* smem, const float2* __restrict__ tw_all) {
  float2* tw = smem + item_smem_elems(N, E);  // = RowSmem::kTw = ColSmem::kTw
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_all[N + i];
  __syncthreads();
  return tw;
}

template <int N, int E>
__global__ void __launch_bounds__(kThreads, min_blocks_for(E)) row_pass_kernel(PassArgs a) {
  extern __shared__ float2 smem[];
  __shared__ Slot s;
  const int tick = (a.tick_base ? *a.tick_base : 0) + a.tick_off;
  const float2* tw = stage_twiddles<N, E>(smem, a.tw);
  for (int it = blockIdx.x; it < a.n_items; it += gridDim.x) {
    const Item item = a.items[it];
    __syncthreads();  // previous item is done with smem and s
    load_slot(&s, &a.slots[item.slot]);
    __syncthreads();
    const int step = tick - s.start_tick;
    if (step < 0 || step > s.n_iter) continue;
    row_item<N, E>(s, step, item.block, smem, tw);
  }
}

template <int N, int E>
__global__ void __launch_bounds__(kThreads, min_blocks_for(E)) col_pass_kernel(PassArgs a) {
  extern __shared__ float2 smem[];
  __shared__ Slot s;
  __shared__ double red[2 * kThreads / 32];
  const int tick = (a.tick_base ? *a.tick_base : 0) + a.tick_off;
  const float2* tw = stage_twiddles<N, E>(smem, a.tw);
  for (int it = blockIdx.x; it < a.n_items; it += gridDim.x) {
    const Item item = a.items[it];
    __syncthreads();
    load_slot(&s, &a.slots[item.slot]);
    __syncthreads();
    const int step = tick - s.start_tick;
    if (step < 0 || step > s.n_iter) continue;
    col_item<N, E>(s, step, item.block, smem, tw, red);
  }
}

template <int N, int E>
cudaError_t launch_pass_t(int which, int grid, cudaStream_t st, const PassArgs& a) {
  const size_t sm = (size_t)pass_smem_elems<N, E>() * sizeof(float2);
  if (which == 0)
    col_pass_kernel<N, E><<<grid, kThreads, sm, st>>>(a);
  else
    row_pass_kernel<N, E><<<grid, kThreads, sm, st>>>(a);
  return cudaGetLastError();
}

template <int N, int E>
cudaError_t pass_setup_t(int* occupancy) {
  const int sm = pass_smem_elems<N, E>() * (int)sizeof(float2);
  cudaError_t e;
  e = cudaFuncSetAttribute(col_pass_kernel<N, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(row_pass_kernel<N, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  int a = 0, b = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, col_pass_kernel<N, E>, kThreads, sm);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, row_pass_kernel<N, E>, kThreads, sm);
  if (e != cudaSuccess) return e;
  *occupancy = a < b ? a : b;
  return cudaSuccess;
}

// Per-size entry points (defined in sp_engine_n<N>.cu).  E is clamped to N.
#define SP_DECLARE_SIZE(N)                                                                  \
  cudaError_t launch_pass_n##N(int E, int which, int grid, cudaStream_t st, const PassArgs& a); \
  cudaError_t pass_setup_n##N(int E, int* occupancy);
SP_DECLARE_SIZE(8)
SP_DECLARE_SIZE(16)
SP_DECLARE_SIZE(32)
SP_DECLARE_SIZE(64)
SP_DECLARE_SIZE(128)
SP_DECLARE_SIZE(256)
SP_DECLARE_SIZE(512)
SP_DECLARE_SIZE(1024)
SP_DECLARE_SIZE(2048)
SP_DECLARE_SIZE(4096)

#define SP_DEFINE_SIZE(N)                                                                    \
  cudaError_t launch_pass_n##N(int E, int which, int grid, cudaStream_t st, const PassArgs& a) { \
    if (E >= 32 && N >= 32) return launch_pass_t<N, (N >= 32 ? 32 : N)>(which, grid, st, a);   \
    return launch_pass_t<N, (N >= 16 ? 16 : N)>(which, grid, st, a);                           \
  }                                                                                          \
  cudaError_t pass_setup_n##N(int E, int* occupancy) {                                       \
    if (E >= 32 && N >= 32) return pass_setup_t<N, (N >= 32 ? 32 : N)>(occupancy);            \
    return pass_setup_t<N, (N >= 16 ? 16 : N)>(occupancy);                                    \
  }

// E actually used for a requested E at size N
inline int effective_e(int N, int E) {
  if (E >= 32 && N >= 32) return 32;
  return N >= 16 ? 16 : N;
}

}  // namespace sp
