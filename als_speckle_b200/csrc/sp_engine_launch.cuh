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
// smallest E instantiated for size N (8, or N/256 when a line needs more threads)
constexpr int kSmallE(int N) { return (N / kThreads > 8) ? N / kThreads : (N >= 8 ? 8 : N); }

// Resident CTAs per SM each kernel is compiled for (registers per thread =
// 64K / (256 * this)): E = 32 needs ~240 registers, E = 16 fits 128 and E = 8
// fits 64 (four CTAs, 32 warps per SM).
constexpr int min_blocks_for(int E, bool row) {
  return E >= 32 ? 1 : (E >= 16 ? 2 : 4);
}

// Build this size's per-stage twiddle tables in shared memory (once per
// persistent CTA); returns their address.
template <int N, int E>
__device__ __forceinline__ const float2* stage_twiddles(float2* smem, const float2* __restrict__ tw_all) {
  float2* tw = smem + item_smem_elems(N, E);  // = RowSmem::kTw = ColSmem::kTw
  build_stage_twiddles<N, E>(tw, tw_all + N);
  __syncthreads();
  return tw;
}

template <int N, int E>
__global__ void __launch_bounds__(kThreads, min_blocks_for(E, true)) row_pass_kernel(PassArgs a) {
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
__global__ void __launch_bounds__(kThreads, min_blocks_for(E, false)) col_pass_kernel(PassArgs a) {
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
constexpr size_t col_smem_bytes() { return (size_t)ColSmem<N, E>::kTotal * sizeof(float2); }
template <int N, int E>
constexpr size_t row_smem_bytes() { return (size_t)RowSmem<N, E>::kTotal * sizeof(float2); }

template <int N, int E>
cudaError_t launch_pass_t(int which, int grid, cudaStream_t st, const PassArgs& a) {
  if (which == 0)
    col_pass_kernel<N, E><<<grid, kThreads, col_smem_bytes<N, E>(), st>>>(a);
  else
    row_pass_kernel<N, E><<<grid, kThreads, row_smem_bytes<N, E>(), st>>>(a);
  return cudaGetLastError();
}

// occupancy[0] = resident column-pass CTAs per SM, occupancy[1] = row-pass
template <int N, int E>
cudaError_t pass_setup_t(int* occupancy) {
  const int sc = (int)col_smem_bytes<N, E>(), sr = (int)row_smem_bytes<N, E>();
  cudaError_t e;
  e = cudaFuncSetAttribute(col_pass_kernel<N, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sc);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(row_pass_kernel<N, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sr);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy[0], col_pass_kernel<N, E>, kThreads, sc);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy[1], row_pass_kernel<N, E>, kThreads, sr);
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
    if (E >= 16 && N >= 16) return launch_pass_t<N, (N >= 16 ? 16 : N)>(which, grid, st, a);   \
    return launch_pass_t<N, kSmallE(N)>(which, grid, st, a);                                  \
  }                                                                                          \
  cudaError_t pass_setup_n##N(int E, int* occupancy) {                                       \
    if (E >= 32 && N >= 32) return pass_setup_t<N, (N >= 32 ? 32 : N)>(occupancy);            \
    if (E >= 16 && N >= 16) return pass_setup_t<N, (N >= 16 ? 16 : N)>(occupancy);            \
    return pass_setup_t<N, kSmallE(N)>(occupancy);                                            \
  }

// E actually used for a requested E at size N: 32, 16 or 8, at most N, and at
// least N/256 so that a line needs no more than the CTA's 256 threads
inline int effective_e(int N, int E) {
  int e = (E >= 32 && N >= 32) ? 32 : ((E >= 16 && N >= 16) ? 16 : (N >= 8 ? 8 : N));
  while (N / e > kThreads) e *= 2;
  return e;
}

}  // namespace sp
