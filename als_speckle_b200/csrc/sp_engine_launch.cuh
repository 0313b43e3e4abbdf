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
  int reverse;  // walk the item list from its end
};



// Copy one slot descriptor into shared memory (word by word).
__device__ __forceinline__ void load_slot(Slot* dst, const Slot* __restrict__ src) {
  static_assert(sizeof(Slot) % 4 == 0, "slot size");
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
  for (int w = threadIdx.x; w < (int)(sizeof(Slot) / 4); w += blockDim.x) d[w] = s[w];
}

// Request one slot descriptor into shared memory (8-byte cp.async by the
// first threads of the block); it lands with the caller's next commit group.
__device__ __forceinline__ void copy_slot(Slot* dst, const Slot* src) {
  static_assert(sizeof(Slot) % 8 == 0, "slot size");
  constexpr int W = sizeof(Slot) / 8;
  if (threadIdx.x < W)
    cp_async<8>(reinterpret_cast<char*>(dst) + 8 * threadIdx.x,
                reinterpret_cast<const char*>(src) + 8 * threadIdx.x);
}

// An item read ahead into registers (slot < 0: none).
__device__ __forceinline__ Item item_at(const PassArgs& a, int it) {
  return it < a.n_items ? a.items[a.reverse ? a.n_items - 1 - it : it] : Item{-1, 0};
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
// (RowGroup) walks them on its own, with its own ring of slot descriptors
// (items k, k+1, k+2) and its own rows of every buffer, so no step of the
// loop waits for the whole block.  The group's rows of the next item's G are
// requested as soon as its psi rows of the current item have been consumed,
// together with the descriptor of the item after that; the item list is read
// ahead into registers.
template <int N, int E>
__global__ void __launch_bounds__(kThreads, min_blocks_for(E, true)) row_pass_kernel(PassArgs a) {
  using SM = RowSmem<N, E>;
  using RG = RowGroup<N, E>;
  extern __shared__ float2 smem[];
  __shared__ __align__(16) Slot sl[3][RG::NG];
  pdl_allow_next();
  const int tick = (a.tick_base ? *a.tick_base : 0) + a.tick_off;
  const float2* tw = stage_twiddles<N, E>(smem + SM::kTw, a.tw);  // block barrier
  float* sup_tile = reinterpret_cast<float*>(smem + SM::kSup);
  const int g = threadIdx.x / RG::GT;
  const int gtid = threadIdx.x - g * RG::GT;
  int it = blockIdx.x;
  if (g >= RG::NG || it >= a.n_items) return;  // no lines for this group, or no items
  const auto sync = RG::sync(g);
  const int G = gridDim.x;
  Item i0 = item_at(a, it), i1 = item_at(a, it + G), i2 = item_at(a, it + 2 * G);
  load_slot_by<RG::GT>(&sl[0][g], &a.slots[i0.slot], gtid);
  if (i1.slot >= 0) load_slot_by<RG::GT>(&sl[1][g], &a.slots[i1.slot], gtid);
  sync();
  pdl_wait_prev();  // the planes are the previous pass's output
  bool ready = false;
  if (row_finishes(sl[0][g], tick)) {
    prefetch_row_tile<N, E>(sl[0][g], i0.block, smem, g, gtid);
    asm volatile("cp.async.commit_group;" ::: "memory");
    ready = true;
  }
  int par = 0;
  for (int k = 0; it < a.n_items; it += G, ++k) {
    const Item i3 = item_at(a, it + 3 * G);
    sync();  // the group is done with its rows of both buffers and with item k-1's slot entry
    const Slot& s = sl[k % 3][g];
    auto copy_ring = [&]() {  // item k+2's descriptor into item k-1's entry
      if (i2.slot >= 0) copy_slot_by(&sl[(k + 2) % 3][g], &a.slots[i2.slot], gtid);
    };
    const int step = tick - s.start_tick;
    bool next_ready = false;
    if (step >= 0 && step <= s.n_iter) {
      next_ready = row_item<N, E>(s, step, i0.block, smem + par * SM::kB, smem + (par ^ 1) * SM::kB,
                                  ready, sup_tile, i1.slot >= 0 ? &sl[(k + 1) % 3][g] : nullptr,
                                  i1.block, tick, tw, g, gtid, copy_ring);
    }
    if (next_ready) {
      ready = true;
      par ^= 1;
    } else {
      // nothing is in flight for the next item: it keeps its G rows where
      // they are (global memory) and the buffers need not swap
      copy_ring();
      asm volatile("cp.async.commit_group;" ::: "memory");
      cp_async_wait_all();
      ready = false;
    }
    i0 = i1;
    i1 = i2;
    i2 = i3;
  }
  cp_async_wait_all();
}

// Column pass: persistent CTAs walk their items with one block barrier per
// item.  At the top of item k (after waiting for its G tile and the barrier)
// the block reads the inputs of the last stage of item k-1's inverse
// transforms from the other buffer, requests item k+1's G tile into that
// buffer in the same mapping (each column's threads also request item k's
// modulus), then finishes item k-1 straight into global memory; item k's
// columns then run with no block-wide synchronisation.  Slot descriptors go
// round a ring of three (items k, k+1 and k+2, whose copy is requested during
// item k), and the item list is read ahead into registers, so no step of the
// loop waits on a global load.
template <int N, int E>
__global__ void __launch_bounds__(kThreads, min_blocks_for(E, false)) col_pass_kernel(PassArgs a) {
  using CS = ColSmem<N, E>;
  extern __shared__ float2 smem[];
  __shared__ __align__(16) Slot sl[3];
  pdl_allow_next();
  const int tick = (a.tick_base ? *a.tick_base : 0) + a.tick_off;
  const float2* tw = stage_twiddles<N, E>(smem + CS::kTw, a.tw);  // block barrier
  float* mod = reinterpret_cast<float*>(smem + CS::kMod);
  int it = blockIdx.x;
  if (it >= a.n_items) return;  // the whole block leaves together
  const int G = gridDim.x;
  // items k, k+1, k+2 held in registers; item k+3 is read during item k
  Item i0 = item_at(a, it), i1 = item_at(a, it + G), i2 = item_at(a, it + 2 * G);
  load_slot(&sl[0], &a.slots[i0.slot]);
  if (i1.slot >= 0) load_slot(&sl[1], &a.slots[i1.slot]);
  __syncthreads();
  pdl_wait_prev();  // the planes (and the transposed modulus) are earlier kernels' output
  copy_col_g<N, E>(sl[0], i0.block, tick, smem);
  asm volatile("cp.async.commit_group;" ::: "memory");
  float2* pend = nullptr;  // plane whose last stage is left in the other buffer
  int pend_block = 0;
  int b = 0;
  for (int k = 0; it < a.n_items; it += G, ++k, b ^= 1) {
    const Item i3 = item_at(a, it + 3 * G);
    cp_async_wait_all();  // this item's G tile and item k+1's slot descriptor
    __syncthreads();      // ... visible to all; the previous item is finished
    float2* other = smem + (b ^ 1) * CS::kB;
    const Slot& s = sl[k % 3];
    auto copies = [&]() {
      copy_col_mod<N, E>(s, i0.block, tick, mod);
      asm volatile("cp.async.commit_group;" ::: "memory");
      if (i1.slot >= 0) copy_col_g<N, E>(sl[(k + 1) % 3], i1.block, tick, other);
      if (i2.slot >= 0) copy_slot(&sl[(k + 2) % 3], &a.slots[i2.slot]);  // item k-1's entry
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (pend)
      col_last_stage<N, E>(pend, pend_block, other, tw, copies);
    else
      copies();
    pend = nullptr;
    if (col_live(s, tick)) {
      pend = col_item<N, E>(s, tick - s.start_tick, i0.block, smem + b * CS::kB, mod, tw);
      pend_block = i0.block;
    }
    i0 = i1;
    i1 = i2;
    i2 = i3;
  }
  __syncthreads();
  if (pend) col_last_stage<N, E>(pend, pend_block, smem + (b ^ 1) * CS::kB, tw, [] {});
  cp_async_wait_all();
}

// Single-buffered column pass: CTAs of kColSbThreads threads, each walking
// half items (C/2 columns; sub-item j is half j & 1 of item j >> 1), with one
// set of column strips (exchanges and the last stage's inputs) and one
// row-major staging buffer for the G tile (96 KB in all), so two CTAs share
// an SM where the pipelined form fits one.  Two per SM (8 warps, up to 255
// registers) run fastest: with the strips alone (55 KB), three per SM at 170
// registers and four at 128 were slower, giving up per-warp parallelism in
// registers for warps that do not make up for it.
// Per half item: wait for the tile and modulus, barrier, forward transform
// (its first stage reading the staging buffer), projection and inverse
// transform up to its last stage (col_item), barrier, then the last stage in
// the row mapping straight to global memory while the next half's modulus
// (into the strips it has finished with) and tile (into the staging buffer,
// 16-byte copies of whole row segments) are requested; the other CTA on the
// SM covers the copies.  Used where it measures faster (512^2 at E = 32; at
// 1024^2 and above its narrower tiles lose more than the extra warps gain).
constexpr int kColSbThreads = 128;
__host__ __device__ constexpr bool col_single_buffered(int N, int E) { return N == 512 && E == 32; }
// column-pass work units per item
__host__ __device__ constexpr int col_split(int N, int E) {
  return col_single_buffered(N, E) ? lines_per_item(N, E) / lines_per_item_t(N, E, kColSbThreads) : 1;
}

template <int N, int E>
__global__ void __launch_bounds__(kColSbThreads, 2) col_pass_sb_kernel(PassArgs a) {
  constexpr int TH = kColSbThreads;
  constexpr int SPLIT = col_split(N, E);
  using CS = ColSmem<N, E, TH, 1>;
  static_assert(SPLIT * CS::C == lines_per_item(N, E), "an item is SPLIT whole sub-items");
  extern __shared__ float2 smem[];
  __shared__ __align__(16) Slot sl[3];
  pdl_allow_next();
  const int tick = (a.tick_base ? *a.tick_base : 0) + a.tick_off;
  const float2* tw = stage_twiddles<N, E>(smem + CS::kTw, a.tw);  // block barrier
  float* mod = reinterpret_cast<float*>(smem + CS::kMod);
  float2* tile = smem + ColTile<N, E, TH>::kOff;
  const int n_sub = SPLIT * a.n_items;
  int it = blockIdx.x;
  if (it >= n_sub) return;  // the whole block leaves together
  const int G = gridDim.x;
  auto sub_at = [&](int j) -> Item {
    if (j >= n_sub) return Item{-1, 0};
    Item i = item_at(a, j / SPLIT);
    i.block = SPLIT * i.block + j % SPLIT;
    return i;
  };
  // sub-items k, k+1, k+2 held in registers; sub-item k+3 is read during k
  Item i0 = sub_at(it), i1 = sub_at(it + G), i2 = sub_at(it + 2 * G);
  load_slot(&sl[0], &a.slots[i0.slot]);
  if (i1.slot >= 0) load_slot(&sl[1], &a.slots[i1.slot]);
  __syncthreads();
  pdl_wait_prev();  // the planes (and the transposed modulus) are earlier kernels' output
  copy_col_mod<N, E, TH>(sl[0], i0.block, tick, mod);
  asm volatile("cp.async.commit_group;" ::: "memory");
  if (col_projects(sl[0], tick)) copy_col_tile<N, E, TH>(sl[0].g, i0.block, tile);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int k = 0; it < n_sub; it += G, ++k) {
    const Item i3 = sub_at(it + 3 * G);
    cp_async_wait_all();  // this sub-item's modulus and tile, sub-item k+1's descriptor
    __syncthreads();      // ... visible to all; the previous sub-item is finished
    const Slot& s = sl[k % 3];
    float2* pend = nullptr;
    if (col_live(s, tick))
      pend = col_item<N, E, TH, true>(s, tick - s.start_tick, i0.block, smem, mod, tw, tile);
    __syncthreads();  // last-stage inputs in the strips; the modulus strips and the tile consumed
    auto copies = [&]() {
      if (i1.slot >= 0) copy_col_mod<N, E, TH>(sl[(k + 1) % 3], i1.block, tick, mod);
      asm volatile("cp.async.commit_group;" ::: "memory");
      if (i1.slot >= 0 && col_projects(sl[(k + 1) % 3], tick))
        copy_col_tile<N, E, TH>(sl[(k + 1) % 3].g, i1.block, tile);
      if (i2.slot >= 0) copy_slot(&sl[(k + 2) % 3], &a.slots[i2.slot]);  // sub-item k-1's entry
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (pend)
      col_last_stage<N, E, TH>(pend, i0.block, smem, tw, copies);
    else
      copies();
    i0 = i1;
    i1 = i2;
    i2 = i3;
  }
  cp_async_wait_all();
}

template <int N, int E>
constexpr size_t col_smem_bytes() {
  if constexpr (col_single_buffered(N, E))
    return (size_t)ColTile<N, E, kColSbThreads>::kTotal * sizeof(float2);
  else
    return (size_t)ColSmem<N, E>::kTotal * sizeof(float2);
}
template <int N, int E>
constexpr size_t row_smem_bytes() { return (size_t)RowSmem<N, E>::kTotal * sizeof(float2); }

template <int N, int E>
cudaError_t launch_pass_t(int which, int grid, cudaStream_t st, const PassArgs& a) {
  if (which == 0) {
    if constexpr (col_single_buffered(N, E))
      return launch_pdl(col_pass_sb_kernel<N, E>, grid, kColSbThreads, col_smem_bytes<N, E>(), st, a);
    else
      return launch_pdl(col_pass_kernel<N, E>, grid, kThreads, col_smem_bytes<N, E>(), st, a);
  }
  return launch_pdl(row_pass_kernel<N, E>, grid, kThreads, row_smem_bytes<N, E>(), st, a);
}

// occupancy[0] = resident column-pass CTAs per SM, occupancy[1] = row-pass
// (the column pass's CTAs each take 1 / col_split(N, E) of an item)
template <int N, int E>
cudaError_t pass_setup_t(int* occupancy) {
  const int sc = (int)col_smem_bytes<N, E>(), sr = (int)row_smem_bytes<N, E>();
  cudaError_t e;
  if constexpr (col_single_buffered(N, E)) {
    e = cudaFuncSetAttribute(col_pass_sb_kernel<N, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sc);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy[0], col_pass_sb_kernel<N, E>,
                                                      kColSbThreads, sc);
  } else {
    e = cudaFuncSetAttribute(col_pass_kernel<N, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sc);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy[0], col_pass_kernel<N, E>, kThreads, sc);
  }
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(row_pass_kernel<N, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sr);
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
