// Device side of the fused iteration engine.
//
// One iteration of the reference (phasing.py:1088-1353) is
//     psi_out = IFFT2( M * FFT2(psi_in) / |FFT2(psi_in)| )      (_fourier_constraint)
//     psi_in  = update_alg(psi_in, psi_out, support)              (_hio/_er/...)
// Here it is split at the 2-D FFT's row/column boundary into two passes over
// a Fourier work plane G that holds "rows transformed, columns not":
//   column pass  G <- IFFT_cols( P_M( FFT_cols(G) ) )   (+ FP64 error sums)
//   row pass     psi_out = IFFT_rows(G); psi_in = update(...);
//                G <- FFT_rows(psi_in)                   (start of next iteration)
// Every transform runs in the forward direction: an inverse is done as
// IFFT(x) = conj(FFT(conj(x))), with the conjugates folded into the
// projection and the update, and G is stored conjugated between the column
// pass and the row pass.  So each kernel holds one transform instance, which
// keeps its code small.
// Each pass is one persistent kernel over a work list of (slot, block) items;
// a block is 256*E pixels of one trial (256*E/N rows, or 256*E/N columns),
// where E (values per thread, 16 or 32) is chosen per size by the autotuner.
// Which part of the schedule a slot is in
// comes from its own start tick, so trials of different sizes, algorithms and
// iteration counts advance together in the same launches.
#pragma once
#include <type_traits>

#include "sp_common.cuh"
#include "sp_fft.cuh"

namespace sp {

struct Slot {
  int32_t logn, n_iter, n_runs, init;
  int32_t run_alg[SP_MAX_RUNS];
  int32_t run_end[SP_MAX_RUNS];  // cumulative counts; run_end[n_runs-1] = period
  float beta;
  uint32_t seed, trial;
  int32_t r0, c0, rows, cols;
  int32_t start_tick;
  int32_t pad_;
  float2* psi;
  float2* g;   // Fourier work plane
  float2* g2;  // second plane for DM (projection of dm1(psi)), or null
  const float* modulus;
  const float* modulus_t;  // the modulus transposed (row c = column c), in the workspace
  const float* support;
  float2* save;
  double* err;
  const float2* ipsf;      // partial coherence: transform of the point spread, or null
  float2* w;               // divisor work plane of G's projection (partial coherence)
  float2* w2;              // ... of G2's (DM)
  const float* spec_r;     // energy spectrum: rescale factors, or null
  const float* spec_w;     // ... and weights
  float* p;                // squared-divisor plane of G's projection (spectrum)
  float* p2;               // ... of G2's (DM)
  int32_t spec_n;          // spectrum samples (0 = none)
  int32_t pad2_;
};

struct Item {
  int32_t slot, block;
};

__host__ __device__ constexpr int clamp_e(int N, int E) { return E < N ? E : N; }

// threads per line T = N / E, lines per item = min(threads / T, N) for a
// CTA of `threads` (kThreads = 256 unless a kernel says otherwise)
__host__ __device__ constexpr int lines_per_item_t(int N, int E, int threads) {
  return (threads / (N / clamp_e(N, E))) < N ? (threads / (N / clamp_e(N, E))) : N;
}
__host__ __device__ constexpr int lines_per_item(int N, int E) {
  return lines_per_item_t(N, E, kThreads);
}

// Algorithm of 1-based iteration i: order_list[(i-1) % period] (phasing.py:260-267)
__device__ __forceinline__ int slot_alg(const Slot& s, int i) {
  const int period = s.run_end[s.n_runs - 1];
  const int p = (i - 1) % period;
  int a = s.run_alg[0];
#pragma unroll
  for (int r = SP_MAX_RUNS - 1; r >= 0; --r) {
    if (r < s.n_runs && p < s.run_end[r]) a = s.run_alg[r];
  }
  return a;
}

// ---------------------------------------------------------------------------
// real-space updates
//
// Every update of the reference is linear in (psi_in, psi_out) with weights
// that are affine in the support value s:
//     new = pi * (a0 + a1 s) + po * (b0 + b1 s)        [ - s*beta*t for DM ]
//   hio  phasing_hio.cl:16-17   (1-s)(pi - b po) + s po        a=(1,-1)  b=(-b, 1+b)
//   er   phasing_er.cl:13-14    s po                           a=(0,0)   b=(0, 1)
//   raar phasing_raar.cl:19-20  (1-s)(b pi + (1-2b) po) + s po a=(b,-b)  b=(1-2b, 2b)
//   sf   phasing_sf.cl:16-17    (1-s)(-po) + s po              a=(0,0)   b=(-1, 2)
//   er (CPU branch, phasing.py:1257)  s pi                     a=(0,1)   b=(0, 0)
//   sf (CPU branch, phasing.py:1284)  (1-s)(-pi) + s po        a=(-1,1)  b=(0, 1)
//   dm   phasing_dm2.cl:21-28 with g = -1/b:
//        s(2po - b t + b((1+g)po - g pi)) + (1-s)(pi - b po)
//        = pi + po(-b + (1+2b) s) - s b t                      a=(1,0)   b=(-b, 1+2b)
// so one code path serves all of them.
// ---------------------------------------------------------------------------
struct UpdateCoef {
  float a0, a1, b0, b1;
  bool needs_pi;
};

__device__ __forceinline__ UpdateCoef update_coef(int alg, float b) {
  switch (alg) {
    case SP_HIO: return {1.f, -1.f, -b, 1.f + b, true};
    case SP_ER: return {0.f, 0.f, 0.f, 1.f, false};
    case SP_RAAR: return {b, -b, 1.f - 2.f * b, 2.f * b, true};
    case SP_SF: return {0.f, 0.f, -1.f, 2.f, false};
    case SP_ER_CPU: return {0.f, 1.f, 0.f, 0.f, true};
    case SP_SF_CPU: return {-1.f, 1.f, 0.f, 1.f, true};
    case SP_DM: return {1.f, 0.f, -b, 1.f + 2.f * b, true};
    default: return {1.f, 0.f, 0.f, 0.f, true};
  }
}

// dm1 (phasing_dm1.cl:16): -g (1-s) pi + s pi = pi (-g + (1+g) s), g = gamma_m = 1/b
__device__ __forceinline__ float dm1_weight(float b, float s) {
  const float g = 1.0f / b;
  return -g + (1.f + g) * s;
}

__device__ __forceinline__ uint32_t hash_u32(uint32_t seed, uint32_t trial, uint32_t idx) {
  uint32_t h = (seed * 0x9E3779B1u) ^ (trial * 0x85EBCA77u);
  h ^= idx * 0xC2B2AE3Du;
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}

// Streaming loads.  Pixel data is read once per pass, so it bypasses L1
// (keeping L1 for nothing else is pointless: twiddles live in shared memory).
// Read-only inputs (modulus, support) also take the non-coherent path.
__device__ __forceinline__ float2 ld_stream(const float2* p) { return __ldcg(p); }
__device__ __forceinline__ float ld_ro(const float* p) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}

// Programmatic dependent launch: an engine kernel lets the next kernel of its
// stream be scheduled as soon as all of its own CTAs run, and that kernel
// builds its twiddle tables and reads its descriptors (nothing an earlier
// kernel writes) while this one finishes, then waits for it to complete
// before touching any plane.  The wait is the hardware's grid dependency: it
// ends when the earlier grid has completed and its writes are visible.
__device__ __forceinline__ void pdl_allow_next() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait_prev() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Launch with programmatic stream serialization (see pdl_allow_next).
template <class Args>
cudaError_t launch_pdl(void (*kernel)(Args), int grid, int threads, size_t smem, cudaStream_t st,
                       const Args& a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, a);
}

// Asynchronous global -> shared copies (cp.async, no registers held): psi,
// support and modulus tiles are requested at the start of an item and land
// while the item's first FFT runs.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(sa), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copy ROWS rows of RB bytes (a multiple of 16) starting at gsrc with global
// row pitch GP bytes into shared memory with row pitch SP bytes, 16 bytes per
// cp.async, shared among NT threads of which this is number q0.  All geometry
// is compile-time, so each thread's chunk addresses are a base plus constants.
template <int ROWS, int RB, int GP, int SP, int NT>
__device__ __forceinline__ void cp_async_rows(void* sdst, const void* gsrc, int q0) {
  static_assert(RB % 16 == 0 && SP % 16 == 0 && GP % 16 == 0, "16-byte chunks");
  constexpr int PER_ROW = RB / 16;
  constexpr int CHUNKS = ROWS * PER_ROW;
  char* d = static_cast<char*>(sdst);
  const char* g = static_cast<const char*>(gsrc);
  if constexpr (PER_ROW % NT == 0) {
    // thread q0 (< NT) copies chunks q0 + j*NT: row j / (PER_ROW/NT), chunk
    // q0 + (j % (PER_ROW/NT))*NT of that row -- one per-thread base plus
    // compile-time offsets, no index arithmetic per copy
    constexpr int PER = PER_ROW / NT;
    d += q0 * 16;
    g += q0 * 16;
#pragma unroll
    for (int j = 0; j < CHUNKS / NT; ++j) {
      const int r = j / PER, c = (j % PER) * NT;
      cp_async<16>(d + r * SP + c * 16, g + (size_t)r * GP + c * 16);
    }
  } else {
#pragma unroll
    for (int j = 0; j < (CHUNKS + NT - 1) / NT; ++j) {
      const int q = q0 + j * NT;
      if (CHUNKS % NT == 0 || q < CHUNKS) {
        const int r = q / PER_ROW, c = q - r * PER_ROW;  // PER_ROW is a power of two
        cp_async<16>(d + r * SP + c * 16, g + (size_t)r * GP + c * 16);
      }
    }
  }
}

// Shared-memory plan of one pass item.  Row pass: exchange strips | twiddles |
// psi tile (L x N complex) | support tile (L rows of N + 16 floats).  Column
// pass: exchange tile | twiddles | modulus tile (N rows x C floats).
// Row pass: two buffers of L padded strips that swap roles every item (one
// holds the item's G rows and then serves as its exchange buffer, the other
// receives its psi rows and, once the update has read them, the next item's
// G rows) | twiddles | support tile (L rows of N + 16 floats).
template <int N, int E>
struct RowSmem {
  static constexpr int L = lines_per_item(N, E);
  // row pitch of both buffers: the padded line, rounded up to an even number
  // of complex values so every row starts 16-byte aligned (cp.async)
  static constexpr int kStrip = (padk(N, pad_shift(E)) + 1) & ~1;
  static constexpr int kB = L * kStrip;                  // float2 entries per buffer
  static constexpr int kTw = 2 * kB;                     // offset of the twiddle tables
  static constexpr int kSupPitch = N + 16;               // floats per support row
  static constexpr int kSup = kTw + tw_stage_total(N, E);  // offset (float2 units)
  static constexpr int kTotal = kSup + (L * kSupPitch + 1) / 2;
};
// smallest y >= x with y = r (mod m)
__host__ __device__ constexpr int next_congruent(int x, int r, int m) {
  return x + ((r - x) % m + m) % m;
}

// Column-pass geometry.  An item is C adjacent columns; for its FFTs thread
// tid works on column lc = tid / T at rows t + i*T (t = tid % T), so a column
// belongs to half a warp, a warp, or a line group of T/32 warps, and the
// exchanges of its transforms are warp (or line) synchronised.  Each column
// has a strip of shared memory (element a at padk(a), pitch SP complex) for
// its G values and exchanges, and a strip of its modulus (pitch MP floats),
// copied by the column's own threads from the transposed modulus.
//
// The G tile crosses between the column layout and global rows in the
// "row mapping" of the last Stockham stage: butterfly q = tid + u*256 of the
// item is (row j = q / C, column c = q % C) and touches rows j + r*NSL,
// r < RL, of column c (NSL, RL: the last stage's input stride and radix).  The
// next item's G tile is copied in that mapping (8-byte cp.async), and the
// last stage of the inverse transform runs in it one item later, straight
// into global memory, so a copy overwrites only strip entries that the same
// thread has just consumed.  With SP = 16/C (mod 16) for C <= 8 and SP odd
// for C >= 16, every half-warp of those accesses touches 16 distinct 8-byte
// bank pairs; MP staggers the modulus strips of columns that share a warp.
// TH is the CTA's thread count and NB its number of G buffers (two for the
// pipelined column pass, one for the single-buffered one).
template <int N, int E, int TH = kThreads, int NB = 2>
struct ColSmem {
  static constexpr int T = N / E;
  static constexpr int C = lines_per_item_t(N, E, TH);
  static constexpr int SH = pad_shift(E);
  static constexpr int SP = C >= 16 ? next_congruent(padk(N, SH), 1, 2)
                                    : next_congruent(padk(N, SH), 16 / C, 16);
  static constexpr int MP = T >= 32 ? N : N + (T >= 4 ? T : 4);
  static constexpr int NSL = last_ns(N, E);      // last stage: inputs j + r*NSL
  static constexpr int RL = N / NSL;             // last stage radix
  static constexpr int BF = C * NSL;             // last-stage butterflies per item
  static constexpr int kB = C * SP;              // float2 entries per G buffer
  static constexpr int kTw = NB * kB;            // offset of the twiddle tables
  static constexpr int kMod = kTw + tw_stage_total(N, E);  // offset of the modulus strips
  static constexpr int kTotal = kMod + (C * MP + 1) / 2;
  // line groups for the modulus copy: GT threads own CG columns
  static constexpr int GT = T < 32 ? 32 : T;
  static constexpr int CG = (GT / T) < C ? (GT / T) : C;
};

// Synchronise the threads of one line when a line spans T > 32 threads
// (whole warps): named barrier 1 + line, so lines do not wait for each other.
template <int T>
struct LineSync {
  int id;
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(T) : "memory");
  }
};

// Row-pass line groups.  The threads of a row item split into groups of
// GT = max(T, 32) threads (a warp, or the warps of one line when T > 32);
// group g owns lines [g*LPG, g*LPG + ROWS) of the item.  A group copies its
// own rows (G, psi, support) and its own slot descriptor, so every wait in
// the row pass is a warp or line barrier and the groups of a block run
// independently of one another.
template <int N, int E>
struct RowGroup {
  static constexpr int T = N / E;
  static constexpr int L = lines_per_item(N, E);
  static constexpr int GT = T < 32 ? 32 : T;
  static constexpr int LPG = GT / T;
  static constexpr int ROWS = LPG < L ? LPG : L;  // lines of every group that has any
  static constexpr int NG = (L + LPG - 1) / LPG;  // groups with lines
  static_assert(NG * GT <= kThreads && NG <= 15, "row groups");
  using Sync = typename std::conditional<(T <= 32), WarpSync, LineSync<T>>::type;
  __device__ static Sync sync(int g) {
    if constexpr (T <= 32) return Sync{};
    else return Sync{1 + g};
  }
};

// Copy one slot descriptor into shared memory, word by word, by the NT
// threads of a group (q0 = thread index within it).
template <int NT>
__device__ __forceinline__ void load_slot_by(Slot* dst, const Slot* __restrict__ src, int q0) {
  static_assert(sizeof(Slot) % 4 == 0, "slot size");
  const int* sp = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
#pragma unroll
  for (int w = q0; w < (int)(sizeof(Slot) / 4); w += NT) d[w] = sp[w];
}

// Request one slot descriptor into shared memory, 8 bytes per cp.async, by
// the first threads of a group (q0 = thread index within it).
__device__ __forceinline__ void copy_slot_by(Slot* dst, const Slot* src, int q0) {
  static_assert(sizeof(Slot) % 8 == 0, "slot size");
  constexpr int W = sizeof(Slot) / 8;
  if (q0 < W)
    cp_async<8>(reinterpret_cast<char*>(dst) + 8 * q0, reinterpret_cast<const char*>(src) + 8 * q0);
}

// Does this step of the slot start with a row inverse FFT of G?
__device__ __forceinline__ bool row_finishes(const Slot& s, int tick) {
  const int step = tick - s.start_tick;
  return step >= 1 && step <= s.n_iter;
}

// Copy group g's G rows of a row item into its padded strips of buf.
template <int N, int E>
__device__ __forceinline__ void prefetch_row_tile(const Slot& s, int block, float2* buf, int g,
                                                  int gtid) {
  using RG = RowGroup<N, E>;
  constexpr int P = RowSmem<N, E>::kStrip;
  const int l0 = g * RG::LPG;
  cp_async_rows<RG::ROWS, N * 8, N * 8, P * 8, RG::GT>(
      buf + l0 * P, s.g + ((size_t)block * RG::L + l0) * N, gtid);
}

// ---------------------------------------------------------------------------
// row pass for one item of a size-N slot, run by line group g (thread gtid of
// it); `s` and `nxt` are the group's own copies of the slot descriptors.
//
// On entry `gbuf` holds the group's G rows of this item if `ready` (cp.async
// group pending, the most recent one this thread committed); `pbuf` is free.
// The psi and support rows are requested at once and land while the inverse
// FFT runs.  After the update has consumed psi, the group's rows of the next
// item's G are requested into `pbuf` (unless DM needs it as private
// storage); returns whether it did (with the caller's `extra` copies in the
// same group), and the caller swaps the buffers.
// ---------------------------------------------------------------------------
template <int N, int E, class Extra>
__device__ __forceinline__ bool row_item(const Slot& s, int step, int block, float2* gbuf,
                                         float2* pbuf, bool ready, float* sup_tile,
                                         const Slot* nxt, int nxt_block, int tick,
                                         const float2* __restrict__ tw, int g, int gtid,
                                         Extra&& extra) {
  using RG = RowGroup<N, E>;
  constexpr int T = N / E;
  constexpr int L = lines_per_item(N, E);
  constexpr int SH = pad_shift(E);
  constexpr int P = RowSmem<N, E>::kStrip;
  constexpr int SPITCH = RowSmem<N, E>::kSupPitch;
  const int tid = threadIdx.x;
  constexpr bool kFull = (L * T == kThreads);  // every thread owns a line segment
  const int lrow = tid / T;
  const int t = tid - lrow * T;
  const bool active = kFull || lrow < L;
  const int lr = active ? lrow : 0;
  const int row = block * L + lr;
  const int l0 = g * RG::LPG;  // the group's first line
  const RowLayout<SH> lay{gbuf + lr * P};
  const typename RG::Sync sync = RG::sync(g);
  const float b = s.beta;
  const size_t roff = (size_t)row * N + t;
  const size_t grow0 = ((size_t)block * L + l0) * N;  // the group's first row in the plane
  float2* psi = s.psi + roff;
  const float2* gtile = gbuf + lr * P + t;    // this thread's G elements (unpadded row)
  float2* psi_s = pbuf + lr * P + t;           // this thread's psi elements
  const float* sup_s = sup_tile + lr * SPITCH + t;

  bool finish, start;
  int alg_f, alg_s;
  if (step == 0) {
    finish = (s.init == SP_INIT_RANDOM_PHASE);
    alg_f = SP_ER;
    start = true;
    alg_s = slot_alg(s, 1);
  } else {
    finish = true;
    alg_f = slot_alg(s, step);
    start = step < s.n_iter;
    alg_s = start ? slot_alg(s, step + 1) : SP_ER;
  }
  // the next item's G rows go into pbuf once psi has been read, unless DM
  // keeps private values there; `extra` adds the caller's copies to that
  // commit group.  (*nxt is read only here, after this item's first wait:
  // its own copy may have travelled with this item's G rows.)
  bool prefetched = false;
  auto prefetch_next = [&]() {
    if (nxt != nullptr && alg_f != SP_DM && alg_s != SP_DM && row_finishes(*nxt, tick)) {
      sync();  // the group is done with its part of pbuf
      prefetch_row_tile<N, E>(*nxt, nxt_block, pbuf, g, gtid);
      extra();
      asm volatile("cp.async.commit_group;" ::: "memory");
      prefetched = true;
    }
  };
  auto copy_support = [&]() {
    cp_async_rows<RG::ROWS, N * 4, N * 4, SPITCH * 4, RG::GT>(sup_tile + l0 * SPITCH,
                                                              s.support + grow0, gtid);
  };

  float2 v[E];
  UpdateCoef cf{};
  if (finish) {
    cf = update_coef(alg_f, b);
    if (cf.needs_pi)
      cp_async_rows<RG::ROWS, N * 8, N * 8, P * 8, RG::GT>(pbuf + l0 * P, s.psi + grow0, gtid);
    copy_support();
    asm volatile("cp.async.commit_group;" ::: "memory");
  } else {
    if (alg_s == SP_DM) {
      copy_support();
      asm volatile("cp.async.commit_group;" ::: "memory");
    }
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = ld_stream(psi + i * T);
    }
    if (alg_s == SP_DM) {
      cp_async_wait_all();
      sync();
    } else {
      prefetch_next();
    }
  }
  // Up to four transforms, one instance: finishing (G, and G2 for DM) and
  // starting (psi, and dm1(psi) for DM).  The column pass leaves the work
  // planes conjugated, so all of them run forward:
  // IFFT_rows(G) = conj(FFT_rows(conj G)), the outer conjugate folded into
  // the update.
  const int nf = finish ? (alg_f == SP_DM ? 2 : 1) : 0;
  const int nt = nf + (start ? (alg_s == SP_DM ? 2 : 1) : 0);
#pragma unroll 1
  for (int x = 0; x < nt; ++x) {
    const bool fin = x < nf;
    const int plane = fin ? x : x - nf;
    if (fin) {
      if (plane == 0) {
        if (ready) {
          asm volatile("cp.async.wait_group 1;" ::: "memory");  // this item's G rows
          sync();
          if (active) {
#pragma unroll
            for (int i = 0; i < E; ++i) v[i] = gtile[i * T];
          }
        } else if (active) {
#pragma unroll
          for (int i = 0; i < E; ++i) v[i] = ld_stream(s.g + roff + i * T);
        }
      } else if (active) {
        // t = IFFT_rows(G2) is DM's second projection
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = ld_stream(s.g2 + roff + i * T);
      }
    } else if (plane == 0) {
      if (alg_s == SP_DM && active) {
        // dm1(psi) waits in the psi tile while psi itself is transformed
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float w = dm1_weight(b, sup_s[i * T]);
          psi_s[i * T] = make_float2(v[i].x * w, v[i].y * w);
        }
      }
    } else if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = psi_s[i * T];
    }
    fft_line<N, E, -1>(v, lay, sync, active, t, tw);
    if (fin) {
      if (plane == 0) {
        // psi_out = conj(v)
        cp_async_wait_all();
        sync();
        if (active) {
          // two copies of the loop, so that no element carries a select
          // between psi and zero (ER and SF never read psi)
          if (cf.needs_pi) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
              const float sv = sup_s[i * T];
              const float wa = cf.a0 + cf.a1 * sv;
              const float wb = cf.b0 + cf.b1 * sv;
              const float2 pi = psi_s[i * T];
              v[i] = make_float2(pi.x * wa + v[i].x * wb, pi.y * wa - v[i].y * wb);
            }
          } else {
#pragma unroll
            for (int i = 0; i < E; ++i) {
              const float wb = cf.b0 + cf.b1 * sup_s[i * T];
              v[i] = make_float2(v[i].x * wb, -v[i].y * wb);
            }
          }
          // DM: the update without -s*b*t waits in the psi tile
          if (nf == 2) {
#pragma unroll
            for (int i = 0; i < E; ++i) psi_s[i * T] = v[i];
          }
        }
      } else if (active) {
        // t = conj(v)
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float w = sup_s[i * T] * b;
          const float2 p = psi_s[i * T];
          v[i] = make_float2(p.x - w * v[i].x, p.y + w * v[i].y);
        }
      }
      if (plane == nf - 1) {
        if (active) {
          // psi is read again only by the next step's update, and ER and SF
          // (GPU forms) do not read it: before one of those (not at the
          // run's last step) the store is skipped
          if (!start || update_coef(alg_s, b).needs_pi) {
#pragma unroll
            for (int i = 0; i < E; ++i) psi[i * T] = v[i];
          }
          if (!start && s.save != nullptr && row >= s.r0 && row < s.r0 + s.rows) {
            float2* dst = s.save + (size_t)(row - s.r0) * s.cols - s.c0;
#pragma unroll
            for (int i = 0; i < E; ++i) {
              const int col = t + i * T;
              if (col >= s.c0 && col < s.c0 + s.cols) dst[col] = v[i];
            }
          }
        }
        prefetch_next();
      }
    } else {
      float2* dst = (plane == 0 ? s.g : s.g2) + roff;
      if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) dst[i * T] = v[i];
      }
    }
  }
  return prefetched;
}

// ---------------------------------------------------------------------------
// column pass for one item of a size-N slot
// ---------------------------------------------------------------------------
// m_s[i * mstride] is the modulus of element i (shared memory).  The result
// is conjugated: the inverse column transform that follows runs as a
// forward transform of the conjugate (IFFT(x) = conj(FFT(conj(x)))), so one
// transform instance serves both directions.
template <int N, int E>
__device__ __forceinline__ void project_cols(float2 (&v)[E], const float* m_s, int mstride,
                                             bool active, double& e2, double& e1, bool want_err) {
  constexpr float inv = 1.0f / ((float)N * (float)N);
  if (!active) return;
  // per-thread partial sums of E terms in FP32, accumulated into FP64
  float f2 = 0.f, f1 = 0.f;
  float m[E];
#pragma unroll
  for (int i = 0; i < E; ++i) {
    m[i] = m_s[i * mstride];
    // The reference divides by |F| = 0 (phasing_fourier.cl:14); here F = 0
    // keeps M with zero phase, without a select: 2^-62 added to the real part
    // turns F = 0 into (2^-62, 0), whose |F|^2 = 2^-124 is still a normal
    // float, so the projection below gives (M/N^2, -0) through power-of-two
    // scalings and |F| - M = -M.  Real parts of magnitude >= 2^-37 do not
    // change (the addend is below half their ulp).
    const float x = v[i].x + 0x1p-62f;
    const float p2 = x * x + v[i].y * v[i].y;
    const float rs = rsqrtf(p2);
    const float d = p2 * rs - m[i];  // |F| - M
    f2 = fmaf(d, d, f2);
    f1 += fabsf(d);
    const float sc = m[i] * rs * inv;
    v[i] = make_float2(x * sc, v[i].y * -sc);
  }
  if (want_err) {
    e2 += (double)f2;
    e1 += (double)f1;
  }
}

// Is the slot live in the column pass at this tick (a projection, or the
// random-phase start), and does it project (and so want its G tile)?
// (Projections of partially coherent slots run in the sp_coherence kernels
// instead; the column pass only builds their random-phase start.)
__device__ __forceinline__ bool slot_partial(const Slot& s) {
  return s.ipsf != nullptr || s.spec_n > 0;
}
__device__ __forceinline__ bool col_live(const Slot& s, int tick) {
  const int step = tick - s.start_tick;
  return step >= 0 && step <= s.n_iter &&
         (step > 0 ? !slot_partial(s) : s.init == SP_INIT_RANDOM_PHASE);
}
__device__ __forceinline__ bool col_projects(const Slot& s, int tick) {
  const int step = tick - s.start_tick;
  return step >= 1 && step <= s.n_iter && !slot_partial(s);
}

// This thread's last-stage butterflies of a column item: butterfly u is row
// j(u) of column c, and pa(u, r) the strip offset of its row j(u) + r*NSL in
// a G buffer.
template <int N, int E, int TH = kThreads>
struct ColButterflies {
  using CS = ColSmem<N, E, TH>;
  static constexpr int C = CS::C, SH = CS::SH, P = 1 << SH;
  static constexpr int U = (CS::BF + TH - 1) / TH;
  static constexpr int JS = TH / C;  // row step between a thread's butterflies
  static constexpr bool LIN = (JS % P) == 0 && (CS::NSL % P) == 0;
  int c, j0, pj0;
  __device__ __forceinline__ ColButterflies()
      : c(threadIdx.x % C), j0(threadIdx.x / C), pj0(c * CS::SP + padk(j0, SH)) {}
  __device__ __forceinline__ bool valid(int u) const {
    return CS::BF % TH == 0 || j0 + u * JS < CS::NSL;
  }
  __device__ __forceinline__ int j(int u) const { return j0 + u * JS; }
  __device__ __forceinline__ int pa(int u, int r) const {
    if constexpr (LIN) return pj0 + u * (JS + JS / P) + r * (CS::NSL + CS::NSL / P);
    else return c * CS::SP + padk(j0 + u * JS + r * CS::NSL, SH);
  }
};

// Request the tile of a column item from the plane `plane`, in the row mapping.
template <int N, int E, int TH = kThreads>
__device__ __forceinline__ void copy_col_plane(const float2* plane, int block, float2* gbuf) {
  using CS = ColSmem<N, E, TH>;
  using BF = ColButterflies<N, E, TH>;
  const BF bf;
  // this thread's first row of the tile; every copy is that base plus a
  // compile-time offset of whole rows
  const float2* g = plane + block * CS::C + bf.c + (size_t)bf.j0 * N;
#pragma unroll
  for (int u = 0; u < BF::U; ++u) {
    if (bf.valid(u)) {
#pragma unroll
      for (int r = 0; r < CS::RL; ++r)
        cp_async<8>(gbuf + bf.pa(u, r), g + (size_t)(u * BF::JS + r * CS::NSL) * N);
    }
  }
}

// Request the G tile of a column item when it projects.
template <int N, int E, int TH = kThreads>
__device__ __forceinline__ void copy_col_g(const Slot& s, int block, int tick, float2* gbuf) {
  if (col_projects(s, tick)) copy_col_plane<N, E, TH>(s.g, block, gbuf);
}

// Row-major staging buffer for the G tile of the single-buffered column pass:
// row a of the item's C columns at a * kPitch (C + 2 entries: 80-byte rows,
// so the 16-byte copies and the first stage's reads, rows t + i*T of two
// columns per warp, use every bank pair no more than the minimum twice).
template <int N, int E, int TH>
struct ColTile {
  using CS = ColSmem<N, E, TH, 1>;
  static constexpr int kPitch = CS::C + 2;
  static constexpr int kOff = (CS::kTotal + 1) & ~1;  // float2 offset, 16-byte aligned
  static constexpr int kTotal = kOff + N * kPitch;
};

// Request a plane's tile of a column item into the staging buffer, 16 bytes
// per cp.async: thread q copies chunks q + j*TH (row (q + j*TH) / Q, chunk
// q % Q of the row's Q = C/2), so each warp covers whole 32-byte sectors of
// consecutive rows.  Every thread of the block takes part, and the caller
// makes sure the whole block has read the buffer's previous tile.
template <int N, int E, int TH>
__device__ __forceinline__ void copy_col_tile(const float2* plane, int block, float2* tile) {
  using CT = ColTile<N, E, TH>;
  constexpr int C = CT::CS::C, Q = C / 2, ROWS_PER = TH / Q;
  static_assert(C % 2 == 0 && TH % Q == 0 && N % ROWS_PER == 0, "16-byte chunks of the tile rows");
  const int q = threadIdx.x;
  const float2* src = plane + (size_t)block * C + 2 * (q % Q) + (size_t)(q / Q) * N;
  float2* dst = tile + (q / Q) * CT::kPitch + 2 * (q % Q);
#pragma unroll
  for (int j = 0; j < N / ROWS_PER; ++j)
    cp_async<16>(dst + j * ROWS_PER * CT::kPitch, src + (size_t)j * ROWS_PER * N);
}

// The last stage of the inverse column transforms of an item whose earlier
// stages left their (conjugated) outputs in gbuf, run in the row mapping as a
// forward stage.  Its result, the conjugate of the new work plane, is
// written to g as it is: the row pass transforms the conjugate (see
// row_item), so the plane stays conjugated between the column pass and the
// row pass.  All inputs are read first; `then()` runs before the
// arithmetic (the caller's next copies into gbuf go there: each overwrites
// only entries this thread has already read).
template <int N, int E, int TH = kThreads, class Then>
__device__ __forceinline__ void col_last_stage(float2* g, int block, const float2* gbuf,
                                               const float2* __restrict__ tw, Then&& then) {
  using CS = ColSmem<N, E, TH>;
  using BF = ColButterflies<N, E, TH>;
  constexpr int R = CS::RL, NS = CS::NSL;
  const float2* __restrict__ tws = tw + tw_stage_offset(N, E, NS);
  const BF bf;
  float2 x[BF::U][R];
#pragma unroll
  for (int u = 0; u < BF::U; ++u) {
    if (bf.valid(u)) {
#pragma unroll
      for (int r = 0; r < R; ++r) x[u][r] = gbuf[bf.pa(u, r)];
    }
  }
  then();
  // per-thread bases; the butterflies' rows and twiddles are compile-time offsets from them
  float2* dst = g + block * CS::C + bf.c + (size_t)bf.j0 * N;
  const float2* __restrict__ twj = tws + bf.j0;
#pragma unroll
  for (int u = 0; u < BF::U; ++u) {
    if (bf.valid(u)) {
#pragma unroll
      for (int r = 1; r < R; ++r) x[u][r] = cmul(x[u][r], twj[r * NS + u * BF::JS]);
      dft<R, -1>(x[u]);
#pragma unroll
      for (int r = 0; r < R; ++r) dst[(size_t)(u * BF::JS + r * NS) * N] = x[u][r];
    }
  }
}

// Each column's threads request their columns' modulus: rows of the
// transposed modulus, 16 bytes per cp.async, into the columns' strips.
template <int N, int E, int TH = kThreads>
__device__ __forceinline__ void copy_col_mod(const Slot& s, int block, int tick, float* mod) {
  using CS = ColSmem<N, E, TH>;
  if (!col_live(s, tick)) return;
  const int g = threadIdx.x / CS::GT;
  const int gtid = threadIdx.x - g * CS::GT;
  const int lc0 = g * (CS::GT / CS::T);  // the group's first column
  if (lc0 >= CS::C) return;
  constexpr int PER_COL = N / 4;
  constexpr int CHUNKS = CS::CG * PER_COL;
  const float* src = s.modulus_t + (size_t)(block * CS::C + lc0) * N;
  float* dst = mod + lc0 * CS::MP;
  if constexpr (PER_COL % CS::GT == 0) {
    // chunk gtid + k*GT is column k / (PER_COL/GT), offset gtid + (k % (PER_COL/GT))*GT:
    // a per-thread base plus compile-time offsets
    constexpr int PER = PER_COL / CS::GT;
    src += gtid * 4;
    dst += gtid * 4;
#pragma unroll
    for (int k = 0; k < CHUNKS / CS::GT; ++k) {
      const int cc = k / PER, off = (k % PER) * CS::GT * 4;
      cp_async<16>(dst + cc * CS::MP + off, src + (size_t)cc * N + off);
    }
  } else {
#pragma unroll
    for (int k = 0; k < (CHUNKS + CS::GT - 1) / CS::GT; ++k) {
      const int q = gtid + k * CS::GT;
      if (CHUNKS % CS::GT == 0 || q < CHUNKS) {
        const int cc = q / PER_COL, off = (q - cc * PER_COL) * 4;
        cp_async<16>(dst + cc * CS::MP + off, src + (size_t)cc * N + off);
      }
    }
  }
}

// One column item, run by every thread of the block with no block-wide
// barrier: each column's threads read their G elements from the column's
// strip, transform, project with the modulus from the column's modulus strip
// (the most recent cp.async group but one), and run the inverse transform up
// to its last stage.  Returns the plane that col_last_stage must complete
// (for DM the first plane is finished here and the second plane's tile
// brought into the strips, which its transforms need).
// With STAGED (the single-buffered pass), the first plane's G tile is read
// from the row-major staging buffer `tile` instead of the strips.
template <int N, int E, int TH = kThreads, bool STAGED = false>
__device__ __forceinline__ float2* col_item(const Slot& s, int step, int block, float2* gbuf,
                                            const float* mod, const float2* __restrict__ tw,
                                            const float2* tile = nullptr) {
  using CS = ColSmem<N, E, TH>;
  constexpr int T = CS::T;
  constexpr int C = CS::C;
  constexpr int SH = CS::SH, P = 1 << SH;
  constexpr float inv = 1.0f / ((float)N * (float)N);
  constexpr bool kFull = (C * T == TH);
  static_assert(!STAGED || kFull, "the staged tile is read by every thread");
  using Sync = typename std::conditional<(T <= 32), WarpSync, LineSync<T>>::type;
  const int tid = threadIdx.x;
  const int lcol = tid / T;
  const int t = tid - lcol * T;
  const bool active = kFull || lcol < C;
  const int lc = active ? lcol : 0;
  const int col = block * C + lc;
  const RowLayout<SH> lay{gbuf + lc * CS::SP};
  Sync sync{};
  if constexpr (T > 32) sync = Sync{1 + lc};
  const float* mod_s = mod + lc * CS::MP + t;
  auto wait_modulus = [&]() {
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    sync();
  };

  // One pass of the loop per plane (two for DM: G, then G2), so each
  // transform is instantiated once.  A plane other than the last is finished
  // here by the whole block, and the next plane's tile is brought into the
  // strips through the same row-mapped copies as a prefetch.
  const bool dm = step > 0 && slot_alg(s, step) == SP_DM;
  const bool want_err = step > 0 && s.err != nullptr;
  const int planes = dm ? 2 : 1;
  double e2 = 0.0, e1 = 0.0;
  float2 v[E];
#pragma unroll 1
  for (int plane = 0; plane < planes; ++plane) {
    if (step == 0) {
      // random-phase start: G = IFFT_cols(M exp(2 pi i u) / N^2), written
      // conjugated into the strip by a rolled loop (the hash and sincospif
      // stay out of the unrolled code)
      wait_modulus();
      if (active) {
#pragma unroll 1
        for (int i = 0; i < E; ++i) {
          const int k = t + i * T;
          const uint32_t h = hash_u32(s.seed, s.trial, (uint32_t)(k * N + col));
          const float u = (float)(h >> 8) * (1.0f / 16777216.0f);
          float sn, cs;
          sincospif(2.0f * u, &sn, &cs);
          const float mm = mod_s[i * T] * inv;
          lay.at(k) = make_float2(mm * cs, -mm * sn);
        }
      }
    }
    bool staged = false;
    if constexpr (STAGED) {
      if (plane == 0 && step > 0) {  // the tile in the row-major staging buffer
        constexpr int TP = ColTile<N, E, TH>::kPitch;
        const float2* tp = tile + t * TP + lc;
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = tp[i * T * TP];
        staged = true;
      }
    }
    if (!staged && active) {  // the plane's tile (or the start values), in the column's strip
      if constexpr (T % P == 0) {
        const int p0 = padk(t, SH);
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = lay.atp(p0 + i * (T + T / P));
      } else {
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = lay.at(t + i * T);
      }
    }
    // phase 0: forward transform and projection; phase 1: the inverse up to
    // its last stage, as a forward transform of the conjugate
#pragma unroll 1
    for (int phase = step == 0 ? 1 : 0; phase < 2; ++phase) {
      fft_line_head<N, E, -1>(v, lay, sync, active, t, tw);
      if (phase == 0) {
        fft_stages<N, E, -1, CS::NSL, false>(v, lay, sync, active, t, tw);  // its last stage
        if (plane == 0) wait_modulus();
        project_cols<N, E>(v, mod_s, T, active, e2, e1, want_err && plane == 0);
      }
    }
    if (plane + 1 < planes) {
      // finish G and bring in the G2 tile through the same strips (each
      // thread's copies overwrite only entries it has already read)
      __syncthreads();  // every column's last-stage inputs are in the strips
      col_last_stage<N, E, TH>(s.g, block, gbuf, tw, [&] {
        copy_col_plane<N, E, TH>(s.g2, block, gbuf);
        asm volatile("cp.async.commit_group;" ::: "memory");
      });
      cp_async_wait_all();
      __syncthreads();  // the G2 tile is in the strips
    }
  }
  if (want_err) {
    // warp sums of the FP64 partials, one atomic pair per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      e2 += __shfl_xor_sync(0xffffffffu, e2, o);
      e1 += __shfl_xor_sync(0xffffffffu, e1, o);
    }
    if ((tid & 31) == 0) {
      atomicAdd(&s.err[2 * (step - 1)], e2);
      atomicAdd(&s.err[2 * (step - 1) + 1], e1);
    }
  }
  return dm ? s.g2 : s.g;
}

// shared-memory entries of one item's exchange buffer (rows: L padded strips;
// cols: padded tile)
__host__ __device__ constexpr int item_smem_elems(int N, int E) {
  return lines_per_item(N, E) * padk(N, pad_shift(E));
}
template <int N, int E>
__host__ __device__ constexpr int pass_smem_elems() {
  return RowSmem<N, E>::kTotal > ColSmem<N, E>::kTotal ? RowSmem<N, E>::kTotal
                                                       : ColSmem<N, E>::kTotal;
}

}  // namespace sp
