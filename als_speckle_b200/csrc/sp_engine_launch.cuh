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
__device__ __forceinline__ const float2* stage_twiddles(float2* tw, const float2* __restrict__ tw_all) {
  build_stage_twiddles<N, E>(tw, tw_all + N);
  __syncthreads();
  return tw;
}

// Row pass: persistent CTAs walk their items; within a CTA each line group
// (RowGroup) walks them on its own, with its own copies of the slot
// descriptors and its own rows of every buffer, so no step of the loop waits
// for the whole block.  The group's rows of the next item's G are requested
// as soon as its psi rows of the current item have been consumed.
template <int N, int E>
__global__ void __launch_bounds__(kThreads, min_blocks_for(E, true)) row_pass_kernel(PassArgs a) {
  using SM = RowSmem<N, E>;
  using RG = RowGroup<N, E>;
  extern __shared__ float2 smem[];
  __shared__ Slot sl[2][RG::NG];
  const int tick = (a.tick_base ? *a.tick_base : 0) + a.tick_off;
  const float2* tw = stage_twiddles<N, E>(smem + SM::kTw, a.tw);  // block barrier
  float* sup_tile = reinterpret_cast<float*>(smem + SM::kSup);
  const int g = threadIdx.x / RG::GT;
  const int gtid = threadIdx.x - g * RG::GT;
  if (g >= RG::NG) return;  // no lines for this group (small N)
  const auto sync = RG::sync(g);
  int it = blockIdx.x;
  int par = 0;
  bool ready = false;
  if (it < a.n_items) {
    load_slot_by<RG::GT>(&sl[0][g], &a.slots[a.items[it].slot], gtid);
    sync();
    if (row_finishes(sl[0][g], tick)) {
      prefetch_row_tile<N, E>(sl[0][g], a.items[it].block, smem, g, gtid);
      asm volatile("cp.async.commit_group;" ::: "memory");
      ready = true;
    }
  }
  for (; it < a.n_items; it += gridDim.x) {
    const int nit = it + gridDim.x;
    sync();  // the group is done with its rows of both buffers and its slot copy
    if (nit < a.n_items) load_slot_by<RG::GT>(&sl[par ^ 1][g], &a.slots[a.items[nit].slot], gtid);
    sync();
    const Slot& s = sl[par][g];
    const int step = tick - s.start_tick;
    bool next_ready = false;
    if (step >= 0 && step <= s.n_iter) {
      next_ready = row_item<N, E>(s, step, a.items[it].block, smem + par * SM::kB,
                                  smem + (par ^ 1) * SM::kB, ready, sup_tile,
                                  nit < a.n_items ? &sl[par ^ 1][g] : nullptr,
                                  nit < a.n_items ? a.items[nit].block : 0, tick, tw, g, gtid);
    }
    if (!next_ready) {
      // nothing is in flight for the next item: it keeps its G rows where
      // they are (global memory) and the buffers need not swap
      cp_async_wait_all();
      ready = false;
      continue;
    }
    ready = true;
    par ^= 1;
  }
  cp_async_wait_all();
}

// Column pass: persistent CTAs walk their items with a two-stage pipeline.
// At the top of item i the CTA requests (cp.async) item i's modulus tile and
// then item i+gridDim's G tile into the buffer item i-gridDim used, so the
// G tile of every item after the first arrives while the previous one is
// transformed.
template <int N, int E>
__global__ void __launch_bounds__(kThreads, min_blocks_for(E, false)) col_pass_kernel(PassArgs a) {
  using SM = ColSmem<N, E>;
  extern __shared__ float2 smem[];
  __shared__ Slot sl[2];
  __shared__ double red[2 * kThreads / 32];
  const int tick = (a.tick_base ? *a.tick_base : 0) + a.tick_off;
  const float2* tw = stage_twiddles<N, E>(smem + SM::kTw, a.tw);
  float* mod_tile = reinterpret_cast<float*>(smem + SM::kMod);
  int it = blockIdx.x;
  int par = 0;
  bool ready = false;
  if (it < a.n_items) {
    load_slot(&sl[0], &a.slots[a.items[it].slot]);
    __syncthreads();
    if (col_projects(sl[0], tick)) {
      prefetch_col_tile<N, E>(sl[0], a.items[it].block, smem);
      ready = true;
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (; it < a.n_items; it += gridDim.x) {
    const int nit = it + gridDim.x;
    __syncthreads();  // the previous item is done with its buffer, the modulus tile and its slot
    if (nit < a.n_items) load_slot(&sl[par ^ 1], &a.slots[a.items[nit].slot]);
    __syncthreads();
    const Slot& s = sl[par];
    const int step = tick - s.start_tick;
    const bool live = step >= 0 && step <= s.n_iter && (step > 0 || s.init == SP_INIT_RANDOM_PHASE);
    if (live) stage_col_modulus<N, E>(s, a.items[it].block, mod_tile);
    asm volatile("cp.async.commit_group;" ::: "memory");
    bool next_ready = false;
    if (nit < a.n_items && col_projects(sl[par ^ 1], tick)) {
      prefetch_col_tile<N, E>(sl[par ^ 1], a.items[nit].block, smem + (par ^ 1) * SM::kB);
      next_ready = true;
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    if (live) col_item<N, E>(s, step, a.items[it].block, smem + par * SM::kB, ready, mod_tile, tw, red);
    ready = next_ready;
    par ^= 1;
  }
  cp_async_wait_all();
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
