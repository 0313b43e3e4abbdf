// Partially coherent projections: the modulus replacement of
// phasing.py:1187-1228 with the divisor built by _build_divisor
// (phasing.py:1109-1157, GPU branch):
//   ipsf (transverse coherence, load(ipsf=...)):
//       div = sqrt(|IFFT2(FFT2(|F|^2) * ipsf)|),    F = FFT2(psi)
//   spectrum (longitudinal coherence, load(spectrum=...)), after the above:
//       div = sqrt(radial_rescale(div^2))   (kernels/phasing_radial_rescale.cl)
// The divisor needs the whole 2-D |F|^2, so for these slots the engine's
// column pass is replaced by up to five launches per projection plane (G,
// and G2 for DM), each skipping the jobs it does not apply to:
//   A  (columns) F = FFT_cols(G), stored over G; then W = FFT_cols(|F|^2)
//                (ipsf) or P = |F|^2 (spectrum only)
//   W  (rows)    W = IFFT_rows(FFT_rows(W) * ipsf), unnormalised   [ipsf]
//   B1 (columns) P = |IFFT_cols(W)| / N^2                     [ipsf + spectrum]
//   R            W (as floats) = radial_rescale(P)                [spectrum]
//   B  (columns) div = sqrt(|IFFT_cols(W)|) / N (ipsf only) or sqrt(W floats)
//                (spectrum); P = M F / div; G = conj(IFFT_cols(P / N^2))
//                = FFT_cols(conj(P) / N^2)
// B leaves G conjugated, as the engine's row pass expects.  The lines are
// transformed with the engine's Stockham building blocks, E = min(16, N)
// values per thread, one item (C columns or L rows of one plane) per block
// iteration; work is a list of (slot, plane) jobs.
#pragma once
#include "sp_engine_kernels.cuh"

namespace sp {

struct PcArgs {
  const Slot* slots;
  const int2* jobs;  // (slot, plane)
  int n_jobs;
  int tick;
  const float2* tw;  // twiddle table of all sizes
};

constexpr int pc_e(int N) { return N < 16 ? N : 16; }

// Does job (slot, plane) project at this tick?
__device__ __forceinline__ bool pc_active(const Slot& s, int plane, int tick) {
  const int step = tick - s.start_tick;
  return step >= 1 && step <= s.n_iter && (plane == 0 || slot_alg(s, step) == SP_DM);
}

template <int N>
__host__ __device__ constexpr int pc_smem_elems() {
  return item_smem_elems(N, pc_e(N)) + tw_stage_total(N, pc_e(N));
}

// A: F = FFT_cols(G) over G, W = FFT_cols(|F|^2).
template <int N>
__global__ void __launch_bounds__(kThreads, 4) pc_cols_a_kernel(PcArgs a) {
  constexpr int E = pc_e(N), T = N / E, C = lines_per_item(N, E);
  extern __shared__ float2 smem[];
  float2* tw = smem + item_smem_elems(N, E);
  build_stage_twiddles<N, E>(tw, a.tw + N);
  const int tid = threadIdx.x, c = tid % C, t = tid / C;
  const bool active = t < T;
  const ColLayout<pad_shift(E), C> lay{smem + c};
  constexpr int PER = N / C;
  for (int it = blockIdx.x; it < a.n_jobs * PER; it += gridDim.x) {
    const int j = it / PER, blk = it - j * PER;
    const int2 job = a.jobs[j];
    const Slot& s = a.slots[job.x];
    if (!pc_active(s, job.y, a.tick)) continue;  // uniform over the block
    float2* g = job.y ? s.g2 : s.g;
    float2* w = job.y ? s.w2 : s.w;
    const size_t off = (size_t)(active ? t : 0) * N + blk * C + c;
    float2 v[E];
    __syncthreads();  // the previous item's exchanges are done
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = g[off + (size_t)i * T * N];
    }
    fft_line<N, E, -1>(v, lay, BlockSync{}, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) {
        g[off + (size_t)i * T * N] = v[i];
        v[i] = make_float2(v[i].x * v[i].x + v[i].y * v[i].y, 0.f);
      }
    }
    if (s.ipsf == nullptr) {  // spectrum only: the squared divisor is |F|^2
      float* pp = job.y ? s.p2 : s.p;
      if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) pp[off + (size_t)i * T * N] = v[i].x;
      }
      continue;
    }
    fft_line<N, E, -1>(v, lay, BlockSync{}, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) w[off + (size_t)i * T * N] = v[i];
    }
  }
}

// W: W = IFFT_rows(FFT_rows(W) * ipsf), unnormalised.
template <int N>
__global__ void __launch_bounds__(kThreads) pc_rows_w_kernel(PcArgs a) {
  constexpr int E = pc_e(N), T = N / E, L = lines_per_item(N, E), SH = pad_shift(E);
  using Sync = typename std::conditional<(T <= 32), WarpSync, BlockSync>::type;
  extern __shared__ float2 smem[];
  float2* tw = smem + item_smem_elems(N, E);
  build_stage_twiddles<N, E>(tw, a.tw + N);
  __syncthreads();
  const int tid = threadIdx.x, lrow = tid / T, t = tid - lrow * T;
  const bool active = lrow < L;
  const int lr = active ? lrow : 0;
  const RowLayout<SH> lay{smem + lr * padk(N, SH)};
  constexpr int PER = N / L;
  for (int it = blockIdx.x; it < a.n_jobs * PER; it += gridDim.x) {
    const int j = it / PER, blk = it - j * PER;
    const int2 job = a.jobs[j];
    const Slot& s = a.slots[job.x];
    if (!pc_active(s, job.y, a.tick) || s.ipsf == nullptr) continue;
    float2* w = job.y ? s.w2 : s.w;
    const size_t off = (size_t)(blk * L + lr) * N + t;
    float2 v[E];
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = w[off + i * T];
    }
    fft_line<N, E, -1>(v, lay, Sync{}, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = cmul(v[i], s.ipsf[off + i * T]);
    }
    fft_line<N, E, +1>(v, lay, Sync{}, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) w[off + i * T] = v[i];
    }
  }
}

// B: divisor from W, projection of F (stored in G), inverse column transform;
// FP64 error sums of |F| - M for plane 0, one atomic pair per warp.
template <int N>
__global__ void __launch_bounds__(kThreads, 4) pc_cols_b_kernel(PcArgs a) {
  constexpr int E = pc_e(N), T = N / E, C = lines_per_item(N, E);
  constexpr float inv = 1.0f / ((float)N * (float)N);
  extern __shared__ float2 smem[];
  float2* tw = smem + item_smem_elems(N, E);
  build_stage_twiddles<N, E>(tw, a.tw + N);
  const int tid = threadIdx.x, c = tid % C, t = tid / C;
  const bool active = t < T;
  const ColLayout<pad_shift(E), C> lay{smem + c};
  constexpr int PER = N / C;
  for (int it = blockIdx.x; it < a.n_jobs * PER; it += gridDim.x) {
    const int j = it / PER, blk = it - j * PER;
    const int2 job = a.jobs[j];
    const Slot& s = a.slots[job.x];
    if (!pc_active(s, job.y, a.tick)) continue;
    const int step = a.tick - s.start_tick;
    float2* g = job.y ? s.g2 : s.g;
    const float2* w = job.y ? s.w2 : s.w;
    const int col = blk * C + c;
    const size_t off = (size_t)(active ? t : 0) * N + col;
    float2 v[E];
    float dv[E];
    __syncthreads();
    const bool spec = s.spec_n > 0;
    if (!spec) {
      if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = w[off + (size_t)i * T * N];
      }
      fft_line<N, E, +1>(v, lay, BlockSync{}, active, t, tw);
    }
    float f2 = 0.f, f1 = 0.f;
    if (active) {
      // rdv = 1 / divisor (0 where the divisor is 0), from the reciprocal
      // square root: the divisor is sqrt(D) with D the squared divisor
      if (spec) {  // R left the rescaled squared divisor in W, read as floats
        const float* wf = reinterpret_cast<const float*>(w);
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float d2 = wf[off + (size_t)i * T * N];
          dv[i] = d2 > 0.f ? rsqrtf(d2) : 0.f;
        }
      } else {  // D = |IFFT_cols(W)| / N^2
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float p2 = v[i].x * v[i].x + v[i].y * v[i].y;
          dv[i] = p2 > 0.f ? rsqrtf(p2 * rsqrtf(p2)) * (float)N : 0.f;
        }
      }
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const float2 f = g[off + (size_t)i * T * N];
        const float m = s.modulus[off + (size_t)i * T * N];
        const float p2 = f.x * f.x + f.y * f.y;
        const float d = (p2 > 0.f ? p2 * rsqrtf(p2) : 0.f) - m;
        f2 = fmaf(d, d, f2);
        f1 += fabsf(d);
        // the reference divides by a zero divisor; keep M with zero phase there
        const float sc = m * dv[i] * inv;
        v[i] = dv[i] > 0.f ? make_float2(f.x * sc, f.y * -sc) : make_float2(m * inv, 0.f);
      }
    }
    fft_line<N, E, -1>(v, lay, BlockSync{}, active, t, tw);  // = conj(IFFT_cols(P))
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) g[off + (size_t)i * T * N] = v[i];
    }
    if (job.y == 0 && s.err != nullptr) {
      double e2 = f2, e1 = f1;
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
  }
}

// B1: P = |IFFT_cols(W)| / N^2, the squared ipsf divisor, for slots that
// also have a spectrum.
template <int N>
__global__ void __launch_bounds__(kThreads, 4) pc_cols_b1_kernel(PcArgs a) {
  constexpr int E = pc_e(N), T = N / E, C = lines_per_item(N, E);
  constexpr float inv = 1.0f / ((float)N * (float)N);
  extern __shared__ float2 smem[];
  float2* tw = smem + item_smem_elems(N, E);
  build_stage_twiddles<N, E>(tw, a.tw + N);
  const int tid = threadIdx.x, c = tid % C, t = tid / C;
  const bool active = t < T;
  const ColLayout<pad_shift(E), C> lay{smem + c};
  constexpr int PER = N / C;
  for (int it = blockIdx.x; it < a.n_jobs * PER; it += gridDim.x) {
    const int j = it / PER, blk = it - j * PER;
    const int2 job = a.jobs[j];
    const Slot& s = a.slots[job.x];
    if (!pc_active(s, job.y, a.tick) || s.ipsf == nullptr || s.spec_n == 0) continue;
    const float2* w = job.y ? s.w2 : s.w;
    float* pp = job.y ? s.p2 : s.p;
    const size_t off = (size_t)(active ? t : 0) * N + blk * C + c;
    float2 v[E];
    __syncthreads();
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = w[off + (size_t)i * T * N];
    }
    fft_line<N, E, +1>(v, lay, BlockSync{}, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const float p2 = v[i].x * v[i].x + v[i].y * v[i].y;
        pp[off + (size_t)i * T * N] = (p2 > 0.f ? p2 * rsqrtf(p2) : 0.f) * inv;
      }
    }
  }
}

// R: W (read as N*N floats) = radial_rescale(P)  -- phasing_radial_rescale.cl:
// out(x, y) = sum_k w_k * bilinear(P, x / r_k, y / r_k) with corner-centred
// coordinates (x = i or i - N for column i, y likewise for row j); taps at
// or beyond -N/2 and N/2 carry weight 0 (the reference reads them, possibly
// outside the array, and multiplies by 0; here they read an element inside
// the plane instead, times 0).
// The bilinear taps are separable: column i's two source columns and their
// weights depend only on (k, i), row j's only on (k, j).  A block takes a
// tile of TC columns x RB rows; each thread owns one column and RT of the
// tile's rows.  The row taps of up to RQ samples (their weights times w_k)
// are built once per tile in shared memory, a thread's column taps in
// registers, so a sample costs a pixel four loads and four FMAs:
//   out += (w_k wy1) (v11 wx1 + v21 wx2) + (w_k wy2) (v12 wx1 + v22 wx2).
struct RescaleTap {
  int i1, i2;    // source index of each tap (column, or row * N); 0 where the weight is 0
  float w1, w2;  // 1 - |tap - r| (times the spectral weight for rows)
};

// pixels of one rescale tile (TC columns x RB rows, below), for grid sizing
__host__ __device__ constexpr int rescale_tile_pixels(int N) {
  return (N < kThreads ? N : kThreads) *
         (N < 8 * (kThreads / (N < kThreads ? N : kThreads)) ? N : 8 * (kThreads / (N < kThreads ? N : kThreads)));
}

template <int N>
struct RescaleTile {
  static constexpr int TC = N < kThreads ? N : kThreads;  // columns, one per thread
  static constexpr int G = kThreads / TC;                 // row groups
  static constexpr int RB = N < 8 * G ? N : 8 * G;         // rows per tile
  static constexpr int RT = (RB + G - 1) / G;              // rows per thread
  static constexpr int RQ = 16;                            // samples per table fill
  static_assert(TC * RB == rescale_tile_pixels(N), "tile size");
};

// taps of coordinate c (corner-centred) at rescale r; `stride` scales the
// index and `w` the weights
__device__ __forceinline__ RescaleTap rescale_tap(int N, float c, float r, int stride, float w) {
  const int N2 = N / 2;
  const float rc = c / r;
  const int c1 = (int)floorf(rc), c2 = c1 + 1;
  const bool k1 = c1 > -N2 && c1 < N2, k2 = c2 > -N2 && c2 < N2;
  RescaleTap t;
  t.w1 = k1 ? (1.f - fabsf((float)c1 - rc)) * w : 0.f;
  t.w2 = k2 ? (1.f - fabsf((float)c2 - rc)) * w : 0.f;
  t.i1 = k1 ? (c1 < 0 ? c1 + N : c1) * stride : 0;
  t.i2 = k2 ? (c2 < 0 ? c2 + N : c2) * stride : 0;
  return t;
}

template <int N>
__global__ void __launch_bounds__(kThreads, 5) pc_rescale_kernel(PcArgs a) {
  using RT_ = RescaleTile<N>;
  constexpr int TC = RT_::TC, G = RT_::G, RB = RT_::RB, RT = RT_::RT, RQ = RT_::RQ;
  constexpr int N2 = N / 2;
  constexpr int TILES = (N / TC) * (N / RB);
  __shared__ RescaleTap yt[RQ][RB];
  __shared__ float rq[RQ];
  const int tc = threadIdx.x % TC, g = threadIdx.x / TC;
  for (int it = blockIdx.x; it < a.n_jobs * TILES; it += gridDim.x) {
    const int j = it / TILES, tile = it - j * TILES;
    const int2 job = a.jobs[j];
    const Slot& s = a.slots[job.x];
    if (!pc_active(s, job.y, a.tick) || s.spec_n == 0) continue;  // uniform over the block
    const float* __restrict__ pp = job.y ? s.p2 : s.p;
    float* out = reinterpret_cast<float*>(job.y ? s.w2 : s.w);
    const int c0 = (tile % (N / TC)) * TC, r0 = (tile / (N / TC)) * RB;
    const int col = c0 + tc;
    const float xc = (float)(col > N2 - 1 ? col - N : col);
    float cum[RT];
#pragma unroll
    for (int u = 0; u < RT; ++u) cum[u] = 0.f;
    for (int q0 = 0; q0 < s.spec_n; q0 += RQ) {
      const int nq = s.spec_n - q0 < RQ ? s.spec_n - q0 : RQ;
      __syncthreads();  // the previous tile or sample group is done with the tables
      for (int e = threadIdx.x; e < nq * RB; e += kThreads) {
        const int q = e / RB, r = r0 + e % RB;
        yt[q][e % RB] = rescale_tap(N, (float)(r > N2 - 1 ? r - N : r), s.spec_r[q0 + q], N,
                                    s.spec_w[q0 + q]);
      }
      if (threadIdx.x < nq) rq[threadIdx.x] = s.spec_r[q0 + threadIdx.x];
      __syncthreads();
      for (int q = 0; q < nq; ++q) {
        const RescaleTap x = rescale_tap(N, xc, rq[q], 1, 1.f);
#pragma unroll
        for (int u = 0; u < RT; ++u) {
          const int lr = g + u * G;
          if (RB % G == 0 || lr < RB) {
            const RescaleTap y = yt[q][lr];
            const float h1 = fmaf(pp[y.i1 + x.i2], x.w2, pp[y.i1 + x.i1] * x.w1);
            const float h2 = fmaf(pp[y.i2 + x.i2], x.w2, pp[y.i2 + x.i1] * x.w1);
            cum[u] = fmaf(y.w2, h2, fmaf(y.w1, h1, cum[u]));
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < RT; ++u) {
      const int lr = g + u * G;
      if (RB % G == 0 || lr < RB) out[(int64_t)(r0 + lr) * N + col] = cum[u];
    }
  }
}

// which: 0 = A, 1 = W, 2 = B1, 3 = R, 4 = B
template <int N>
cudaError_t launch_pc_t(int which, int grid, cudaStream_t st, const PcArgs& a) {
  const size_t sm = (size_t)pc_smem_elems<N>() * sizeof(float2);
  if (which == 0) pc_cols_a_kernel<N><<<grid, kThreads, sm, st>>>(a);
  else if (which == 1) pc_rows_w_kernel<N><<<grid, kThreads, sm, st>>>(a);
  else if (which == 2) pc_cols_b1_kernel<N><<<grid, kThreads, sm, st>>>(a);
  else if (which == 3) pc_rescale_kernel<N><<<grid, kThreads, 0, st>>>(a);
  else pc_cols_b_kernel<N><<<grid, kThreads, sm, st>>>(a);
  return cudaGetLastError();
}

template <int N>
cudaError_t pc_setup_t() {
  const int sm = pc_smem_elems<N>() * (int)sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(pc_cols_a_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(pc_rows_w_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(pc_cols_b1_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(pc_cols_b_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

// work items per job (columns blocks = row blocks)
template <int N>
constexpr int pc_items_per_job() { return N / lines_per_item(N, pc_e(N)); }

}  // namespace sp

namespace sp {
#define SP_DECLARE_PC(N)                                                              \
  cudaError_t launch_pc_n##N(int which, int grid, cudaStream_t st, const PcArgs& a); \
  cudaError_t pc_setup_n##N();
SP_DECLARE_PC(8)
SP_DECLARE_PC(16)
SP_DECLARE_PC(32)
SP_DECLARE_PC(64)
SP_DECLARE_PC(128)
SP_DECLARE_PC(256)
SP_DECLARE_PC(512)
SP_DECLARE_PC(1024)
SP_DECLARE_PC(2048)
SP_DECLARE_PC(4096)

#define SP_DEFINE_PC(N)                                                                \
  cudaError_t launch_pc_n##N(int which, int grid, cudaStream_t st, const PcArgs& a) { \
    return launch_pc_t<N>(which, grid, st, a);                                        \
  }                                                                                    \
  cudaError_t pc_setup_n##N() { return pc_setup_t<N>(); }
}  // namespace sp
