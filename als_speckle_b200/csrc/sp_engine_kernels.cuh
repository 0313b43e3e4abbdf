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
// Each pass is one persistent kernel over a work list of (slot, block) items;
// a block is 256*E pixels of one trial (256*E/N rows, or 256*E/N columns),
// where E (values per thread, 16 or 32) is chosen per size by the autotuner.  Which part of the schedule a slot is in
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
  const float* support;
  float2* save;
  double* err;
};

struct Item {
  int32_t slot, block;
};

__host__ __device__ constexpr int clamp_e(int N, int E) { return E < N ? E : N; }

// threads per line T = N / E, lines per item = min(256 / T, N)
__host__ __device__ constexpr int lines_per_item(int N, int E) {
  return (kThreads / (N / clamp_e(N, E))) < N ? (kThreads / (N / clamp_e(N, E))) : N;
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
// real-space updates, same operation order as the OpenCL kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 update_px(int alg, float b, float s, float2 pi, float2 po) {
  float re, im;
  switch (alg) {
    case SP_HIO:  // phasing_hio.cl:16-17
      re = (1 - s) * (pi.x - b * po.x) + s * po.x;
      im = (1 - s) * (pi.y - b * po.y) + s * po.y;
      break;
    case SP_ER:  // phasing_er.cl:13-14
      re = s * po.x;
      im = s * po.y;
      break;
    case SP_RAAR: {  // phasing_raar.cl:12,19-20
      const float b2 = 1 - 2 * b;
      re = (1 - s) * (b * pi.x + b2 * po.x) + s * po.x;
      im = (1 - s) * (b * pi.y + b2 * po.y) + s * po.y;
      break;
    }
    case SP_SF:  // phasing_sf.cl:16-17
      re = (1 - s) * (-1 * po.x) + s * po.x;
      im = (1 - s) * (-1 * po.y) + s * po.y;
      break;
    case SP_ER_CPU:  // phasing.py:1257
      re = s * pi.x;
      im = s * pi.y;
      break;
    case SP_SF_CPU:  // phasing.py:1284
      re = (1 - s) * (-1 * pi.x) + s * po.x;
      im = (1 - s) * (-1 * pi.y) + s * po.y;
      break;
    default:
      re = pi.x;
      im = pi.y;
      break;
  }
  return make_float2(re, im);
}

// psi_in <- update(psi_in, psi_out = v) for one line's E values
template <int ALG, int E, int T>
__device__ __forceinline__ void update_line(float2 (&v)[E], const Slot& s, size_t roff, float b) {
  // ER and SF (kernel forms) do not read psi_in
  constexpr bool kNeedsPsiIn = !(ALG == SP_ER || ALG == SP_SF);
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const float sp = __ldg(&s.support[roff + i * T]);
    const float2 pi = kNeedsPsiIn ? s.psi[roff + i * T] : make_float2(0.f, 0.f);
    v[i] = update_px(ALG, b, sp, pi, v[i]);
  }
}

// DM update without the -s*b*t term (phasing_dm2.cl:21-28, g = gamma_s = -1/b):
//   s*(2po + b((1+g)po - g pi)) + (1-s)(pi - b po)
__device__ __forceinline__ float2 dm_partial(float b, float s, float2 pi, float2 po) {
  const float g = -1.0f / b;
  const float t1r = 2 * po.x + b * ((1 + g) * po.x - g * pi.x);
  const float t1i = 2 * po.y + b * ((1 + g) * po.y - g * pi.y);
  const float t2r = pi.x - b * po.x;
  const float t2i = pi.y - b * po.y;
  return make_float2(s * t1r + (1 - s) * t2r, s * t1i + (1 - s) * t2i);
}
// dm1 (phasing_dm1.cl:16): -g (1-s) pi + s pi, g = gamma_m = 1/b
__device__ __forceinline__ float2 dm1_px(float b, float s, float2 pi) {
  const float g = 1.0f / b;
  return make_float2(-1 * g * (1 - s) * pi.x + s * pi.x, -1 * g * (1 - s) * pi.y + s * pi.y);
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

// ---------------------------------------------------------------------------
// row pass for one item of a size-N slot
// ---------------------------------------------------------------------------
template <int N, int E>
__device__ __forceinline__ void row_item(const Slot& s, int step, int block, float2* smem,
                                         const float2* __restrict__ tw_all) {
  constexpr int T = N / E;
  constexpr int L = lines_per_item(N, E);
  using Sync = typename std::conditional<(T <= 32), WarpSync, BlockSync>::type;
  const float2* __restrict__ tw = tw_all + N;
  const int tid = threadIdx.x;
  const int lrow = tid / T;
  const int t = tid - lrow * T;
  const bool active = lrow < L;
  const int row = block * L + (active ? lrow : 0);
  const RowLayout lay{smem + (active ? lrow : 0) * pad32(N)};
  const Sync sync{};
  const float b = s.beta;
  const size_t roff = (size_t)row * N + t;

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

  float2 v[E];
  if (finish) {
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = s.g[roff + i * T];
    }
    fft_line<N, E, +1>(v, lay, sync, active, t, tw);  // v = psi_out
    if (alg_f == SP_DM) {
      if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float sp = __ldg(&s.support[roff + i * T]);
          s.psi[roff + i * T] = dm_partial(b, sp, s.psi[roff + i * T], v[i]);
        }
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = s.g2[roff + i * T];
      }
      fft_line<N, E, +1>(v, lay, sync, active, t, tw);  // v = second projection
      if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float sp = __ldg(&s.support[roff + i * T]);
          const float2 p = s.psi[roff + i * T];
          v[i] = make_float2(p.x - sp * b * v[i].x, p.y - sp * b * v[i].y);
        }
      }
    } else if (active) {
      switch (alg_f) {
        case SP_HIO: update_line<SP_HIO, E, T>(v, s, roff, b); break;
        case SP_ER: update_line<SP_ER, E, T>(v, s, roff, b); break;
        case SP_RAAR: update_line<SP_RAAR, E, T>(v, s, roff, b); break;
        case SP_SF: update_line<SP_SF, E, T>(v, s, roff, b); break;
        case SP_ER_CPU: update_line<SP_ER_CPU, E, T>(v, s, roff, b); break;
        case SP_SF_CPU: update_line<SP_SF_CPU, E, T>(v, s, roff, b); break;
        default: break;
      }
    }
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) s.psi[roff + i * T] = v[i];
      if (!start && s.save != nullptr && row >= s.r0 && row < s.r0 + s.rows) {
        float2* dst = s.save + (size_t)(row - s.r0) * s.cols - s.c0;
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const int col = t + i * T;
          if (col >= s.c0 && col < s.c0 + s.cols) dst[col] = v[i];
        }
      }
    }
  } else if (active) {
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = s.psi[roff + i * T];
  }
  if (start) {
    fft_line<N, E, -1>(v, lay, sync, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) s.g[roff + i * T] = v[i];
    }
    if (alg_s == SP_DM) {
      if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float sp = __ldg(&s.support[roff + i * T]);
          v[i] = dm1_px(b, sp, s.psi[roff + i * T]);
        }
      }
      fft_line<N, E, -1>(v, lay, sync, active, t, tw);
      if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) s.g2[roff + i * T] = v[i];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// column pass for one item of a size-N slot
// ---------------------------------------------------------------------------
template <int N, int E>
__device__ __forceinline__ void project_cols(float2 (&v)[E], const float* __restrict__ mod,
                                             size_t coff, bool active, double& e2, double& e1,
                                             bool want_err) {
  constexpr int T = N / E;
  constexpr float inv = 1.0f / ((float)N * (float)N);
  if (!active) return;
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const float m = __ldg(&mod[coff + (size_t)i * T * N]);
    const float p2 = v[i].x * v[i].x + v[i].y * v[i].y;
    if (p2 > 0.f) {
      const float rs = rsqrtf(p2);
      if (want_err) {
        const float d = p2 * rs - m;
        e2 = fma((double)d, (double)d, e2);
        e1 += fabs((double)d);
      }
      const float sc = m * rs * inv;
      v[i] = make_float2(v[i].x * sc, v[i].y * sc);
    } else {
      // the reference divides by |F| = 0 here (phasing_fourier.cl:14); keep M, zero phase
      if (want_err) {
        e2 = fma((double)m, (double)m, e2);
        e1 += (double)m;
      }
      v[i] = make_float2(m * inv, 0.f);
    }
  }
}

template <int N, int E>
__device__ __forceinline__ void col_item(const Slot& s, int step, int block, float2* smem,
                                         const float2* __restrict__ tw_all, double* red) {
  constexpr int T = N / E;
  constexpr int C = lines_per_item(N, E);
  constexpr float inv = 1.0f / ((float)N * (float)N);
  const float2* __restrict__ tw = tw_all + N;
  const int tid = threadIdx.x;
  const int c = tid % C;
  const int t = tid / C;
  const bool active = t < T;
  const int col = block * C + c;
  const ColLayout lay{smem, C, c};
  const BlockSync sync{};
  const size_t coff = (size_t)(active ? t : 0) * N + col;  // element (t + i*T, col) at coff + i*T*N

  float2 v[E];
  if (step == 0) {
    if (s.init != SP_INIT_RANDOM_PHASE) return;  // uniform over the block
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const int k = t + i * T;
        const uint32_t h = hash_u32(s.seed, s.trial, (uint32_t)(k * N + col));
        const float u = (float)(h >> 8) * (1.0f / 16777216.0f);
        float sn, cs;
        sincospif(2.0f * u, &sn, &cs);
        const float m = __ldg(&s.modulus[coff + (size_t)i * T * N]) * inv;
        v[i] = make_float2(m * cs, m * sn);
      }
    }
    fft_line<N, E, +1>(v, lay, sync, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) s.g[coff + (size_t)i * T * N] = v[i];
    }
    return;
  }

  const bool dm = slot_alg(s, step) == SP_DM;
  const bool want_err = s.err != nullptr;
  double e2 = 0.0, e1 = 0.0;
  for (int plane = 0; plane < (dm ? 2 : 1); ++plane) {
    float2* g = plane ? s.g2 : s.g;
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = g[coff + (size_t)i * T * N];
    }
    fft_line<N, E, -1>(v, lay, sync, active, t, tw);
    project_cols<N, E>(v, s.modulus, coff, active, e2, e1, want_err && plane == 0);
    fft_line<N, E, +1>(v, lay, sync, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) g[coff + (size_t)i * T * N] = v[i];
    }
  }
  (void)inv;
  if (want_err) {
    // block reduction of the two FP64 partial sums, one atomic each per item
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      e2 += __shfl_xor_sync(0xffffffffu, e2, o);
      e1 += __shfl_xor_sync(0xffffffffu, e1, o);
    }
    const int warp = tid >> 5;
    __syncthreads();
    if ((tid & 31) == 0) {
      red[2 * warp] = e2;
      red[2 * warp + 1] = e1;
    }
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, bsum = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) {
        a += red[2 * w];
        bsum += red[2 * w + 1];
      }
      atomicAdd(&s.err[2 * (step - 1)], a);
      atomicAdd(&s.err[2 * (step - 1) + 1], bsum);
    }
  }
}

// shared-memory entries one item needs (rows: L padded strips; cols: padded tile)
__host__ __device__ constexpr int item_smem_elems(int N, int E) {
  return lines_per_item(N, E) * pad32(N);
}

}  // namespace sp
