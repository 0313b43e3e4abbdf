// Stockham FFT building blocks for sm_100a.
//
// A line of N complex64 values (N a power of two, 2..4096) is transformed by
// T = N/E threads that each hold E values in registers (E a power of two,
// E <= N; 16 or 32 in the engine, chosen per N by the autotuner).  Thread t
// always holds the elements with index t + i*T (i = 0..E-1): that is the input
// read pattern of every Stockham stage and the output pattern of the last one,
// so a forward transform, a pointwise operation and an inverse transform can be
// chained in registers with no extra exchange.  Stage 1 is a radix-E DFT on the
// registers; later stages (radix R <= E, E/R butterflies per thread) read from
// and write to shared memory with the Stockham autosort index map
//     out[(j/Ns)*Ns*R + (j%Ns) + r*Ns] = DFT_R( in[j + r*N/R] * W^(r*(j%Ns)) )
// (Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC 2008).  Shared-memory addresses are padded with one
// slot per 32 entries, which makes every exchange of the row and column layouts
// below conflict-free for 8-byte accesses.
//
// Sign convention follows numpy: forward exp(-2*pi*i*n*k/N), inverse
// exp(+2*pi*i*n*k/N), no scaling here (callers fold 1/N^2 into the projection).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sp {

// ---------------------------------------------------------------------------
// compile-time sin/cos (double precision Taylor series after octant reduction)
// ---------------------------------------------------------------------------
constexpr double kPi = 3.141592653589793238462643383279502884;

__host__ __device__ constexpr double taylor_sin(double x) {
  double term = x, sum = x, x2 = x * x;
  for (int n = 1; n < 14; ++n) {
    term *= -x2 / ((2.0 * n) * (2.0 * n + 1.0));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double taylor_cos(double x) {
  double term = 1.0, sum = 1.0, x2 = x * x;
  for (int n = 1; n < 14; ++n) {
    term *= -x2 / ((2.0 * n - 1.0) * (2.0 * n));
    sum += term;
  }
  return sum;
}
// cos(2*pi*k/R) and sin(2*pi*k/R) for integer k, R
__host__ __device__ constexpr double cos_frac(int k, int R) {
  k = ((k % R) + R) % R;
  // reduce to first quadrant by symmetry
  if (4 * k == R) return 0.0;
  if (2 * k == R) return -1.0;
  if (4 * k == 3 * R) return 0.0;
  if (k == 0) return 1.0;
  if (4 * k < R) return taylor_cos(2.0 * kPi * k / R);
  if (2 * k < R) return -taylor_cos(2.0 * kPi * (R - 2 * k) / (2.0 * R));
  if (4 * k < 3 * R) return -taylor_cos(2.0 * kPi * (2 * k - R) / (2.0 * R));
  return taylor_cos(2.0 * kPi * (R - k) / R);
}
__host__ __device__ constexpr double sin_frac(int k, int R) {
  return cos_frac(4 * k - R, 4 * R);  // sin(x) = cos(x - pi/2)
}

// Complex add and subtract as one packed FP32x2 instruction each (sm_100:
// add/sub.f32x2 work on a 64-bit register pair, both lanes IEEE round to
// nearest, flushed like the scalar code built with -ftz).  The butterflies are
// almost all complex adds, so this halves their instruction count; products
// stay scalar, where a packed form would need lane broadcasts or swaps.
__device__ __forceinline__ float2 operator+(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 ra, rb, rr;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.ftz.f32x2 rr, ra, rb;\n\tmov.b64 {%0, %1}, rr;}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 operator-(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 ra, rb, rr;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.ftz.f32x2 rr, ra, rb;\n\tmov.b64 {%0, %1}, rr;}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }

__device__ __forceinline__ float2 cmul(float2 a, float2 w) {
  return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}
// a * conj(w)
__device__ __forceinline__ float2 cmulc(float2 a, float2 w) {
  return make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}

// multiply by exp(DIR * 2*pi*i*K/R) with K, R compile-time constants
template <int R, int DIR, int K>
__device__ __forceinline__ float2 twiddle_const(float2 a) {
  if constexpr (K == 0) {
    return a;
  } else if constexpr (4 * K == R) {
    // DIR=-1: multiply by -i ; DIR=+1: multiply by +i
    if constexpr (DIR < 0) return make_float2(a.y, -a.x);
    else return make_float2(-a.y, a.x);
  } else {
    constexpr float c = (float)cos_frac(K, R);
    constexpr float s = (float)(DIR * sin_frac(K, R));
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

template <int R, int DIR, int K>
__device__ __forceinline__ void dft_combine(float2* v, const float2* e, const float2* o) {
  if constexpr (K < R / 2) {
    if constexpr (4 * K == R) {
      // twiddle -i (DIR < 0) or +i: a lane swap with a sign, folded into
      // scalar adds (a packed add would first need the swapped pair)
      const float2 a = e[K], b = o[K];
      if constexpr (DIR < 0) {
        v[K] = make_float2(a.x + b.y, a.y - b.x);
        v[K + R / 2] = make_float2(a.x - b.y, a.y + b.x);
      } else {
        v[K] = make_float2(a.x - b.y, a.y + b.x);
        v[K + R / 2] = make_float2(a.x + b.y, a.y - b.x);
      }
    } else {
      const float2 t = twiddle_const<R, DIR, K>(o[K]);
      v[K] = e[K] + t;
      v[K + R / 2] = e[K] - t;
    }
    dft_combine<R, DIR, K + 1>(v, e, o);
  }
}

// In-register DFT of size R (natural order in and out), radix-2 decimation in
// time with compile-time twiddles; fully unrolled.
template <int R, int DIR>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  } else if constexpr (R > 2) {
    float2 e[R / 2], o[R / 2];
#pragma unroll
    for (int k = 0; k < R / 2; ++k) {
      e[k] = v[2 * k];
      o[k] = v[2 * k + 1];
    }
    dft<R / 2, DIR>(e);
    dft<R / 2, DIR>(o);
    dft_combine<R, DIR, 0>(v, e, o);
  }
}

// Shared-memory padding: one spare slot per 2^SH entries.  SH = 5 for E = 32
// and SH = 4 for E <= 16 make every exchange of both layouts conflict-free for
// 8-byte accesses (checked against a bank model for N = 64..2048).
__host__ __device__ constexpr int pad_shift(int E) { return E >= 32 ? 5 : 4; }
__host__ __device__ __forceinline__ constexpr int padk(int a, int sh) { return a + (a >> sh); }
__host__ __device__ __forceinline__ constexpr int pad32(int a) { return a + (a >> 5); }

// Shared-memory layouts for a Stockham index a in [0, N).
// Rows: each line owns a contiguous padded strip.
// `at(a)` takes a Stockham index; `atp(p)` an index already padded, which lets
// callers build addresses as a per-thread base plus compile-time constants
// (padk(x + m 2^SH) = padk(x) + m (2^SH + 1)).
template <int SH>
struct RowLayout {
  static constexpr int kShift = SH;
  float2* base;
  __device__ __forceinline__ float2& at(int a) const { return base[padk(a, SH)]; }
  __device__ __forceinline__ float2& atp(int p) const { return base[p]; }
};
// Column tiles: C lines interleaved element by element (line c is the column).
template <int SH, int C>
struct ColLayout {
  static constexpr int kShift = SH;
  float2* base;  // already offset by the column index c
  __device__ __forceinline__ float2& at(int a) const { return base[padk(a, SH) * C]; }
  __device__ __forceinline__ float2& atp(int p) const { return base[p * C]; }
};

// Twiddles of every Stockham stage after the first, stored per stage as
// [r][k] = W_{NS*R}^(r*k) (r < R, k < NS), so that adjacent threads (adjacent
// k) read adjacent entries.  Offset of the table of the stage that starts
// with sub-transform size NS:
__host__ __device__ constexpr int tw_stage_offset(int N, int E, int NS_target) {
  int off = 0;
  for (int NS = E; NS < NS_target && NS < N;) {
    const int R = (N / NS) < E ? (N / NS) : E;
    off += R * NS;
    NS *= R;
  }
  return off;
}
__host__ __device__ constexpr int tw_stage_total(int N, int E) { return tw_stage_offset(N, E, N); }

// Build the stage tables of (N, E) at `dst` (shared memory) from the N-entry
// table tw_n[x] = exp(-2 pi i x / N).  All threads of the block take part;
// the caller synchronises afterwards.
template <int N, int E>
__device__ __forceinline__ void build_stage_twiddles(float2* dst, const float2* __restrict__ tw_n) {
  constexpr int total = tw_stage_total(N, E);
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    int off = 0, NS = E;
    float2 w = make_float2(1.f, 0.f);
    while (NS < N) {
      const int R = (N / NS) < E ? (N / NS) : E;
      if (q < off + R * NS) {
        const int r = (q - off) / NS, k = (q - off) - r * NS;
        w = tw_n[(r * k) * (N / (NS * R))];
        break;
      }
      off += R * NS;
      NS *= R;
    }
    dst[q] = w;
  }
}

struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// Stages 2.. of the Stockham transform.  NS = product of radices done so far.
// HEAD stops before the last stage, whose inputs are then in shared memory.
template <int N, int E, int DIR, int NS, bool HEAD, class Lay, class Sync>
__device__ __forceinline__ void fft_stages(float2 (&v)[E], const Lay& lay, const Sync& sync,
                                           bool active, int t, const float2* __restrict__ tw) {
  constexpr int T = N / E;
  constexpr int SH = Lay::kShift;
  constexpr int P = 1 << SH;
  constexpr int R_ = (N / NS) < E ? (N / NS) : E;
  if constexpr (NS < N && !(HEAD && NS * R_ == N)) {
    constexpr int R = R_;                           // radix of this stage
    constexpr int M = E / R;                        // butterflies per thread
    constexpr bool LAST = (NS * R == N);
    // element t + i*T: padded index padk(t) + i * TP when T is a multiple of P
    constexpr bool LIN_RD = (T % P) == 0;
    constexpr int TP = T + T / P;
    const int prd = padk(t, SH);
    auto rd = [&](int i) -> float2& { return LIN_RD ? lay.atp(prd + i * TP) : lay.at(t + i * T); };
    const float2* __restrict__ tws = tw + tw_stage_offset(N, E, NS);  // this stage's [r][k] table
    if constexpr (!LAST) {
      // read all of this stage's inputs (element t + i*T -> v[i]) before
      // anyone overwrites the buffer with this stage's outputs
      if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = rd(i);
      }
      sync();
    }
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int j = t + m * T;
      const int k = j & (NS - 1);
      float2 u[R];
      if constexpr (LAST) {
        // the last stage writes nothing back to shared memory, so each
        // butterfly reads its own inputs just before use (short live ranges)
        if (active) {
#pragma unroll
          for (int r = 0; r < R; ++r) u[r] = rd(m + r * M);
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = v[m + r * M];
      }
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const float2 w = tws[r * NS + k];
        u[r] = (DIR < 0) ? cmul(u[r], w) : cmulc(u[r], w);
      }
      dft<R, DIR>(u);
      if constexpr (LAST) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[m + r * M] = u[r];
      } else {
        // outputs at base + r*NS; NS >= E >= P is a multiple of P
        const int base = (j / NS) * NS * R + k;
        const int pb = padk(base, SH);
        constexpr int NSP = NS + NS / P;
        if (active) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if constexpr (NS % P == 0)
              lay.atp(pb + r * NSP) = u[r];
            else
              lay.at(base + r * NS) = u[r];
          }
        }
      }
    }
    if constexpr (!LAST) {
      sync();
      fft_stages<N, E, DIR, NS * R, HEAD, Lay, Sync>(v, lay, sync, active, t, tw);
    }
  }
}

// Full 1-D transform of one line held as v[i] = x[t + i*T]; on return
// v[i] = X[t + i*T].  `tw` points at the stage tables built by
// build_stage_twiddles<N, E>.
// Every thread of the block must call this (it synchronises); inactive threads
// pass active=false and skip all memory traffic.
template <int N, int E, int DIR, class Lay, class Sync>
__device__ __forceinline__ void fft_line(float2 (&v)[E], const Lay& lay, const Sync& sync,
                                         bool active, int t, const float2* __restrict__ tw) {
  static_assert(E <= N && (N % E) == 0, "E must divide N");
  constexpr int T = N / E;
  dft<E, DIR>(v);
  if constexpr (T > 1) {
    // stage-1 outputs go to out[t*E + r]
    constexpr int SH = Lay::kShift;
    constexpr bool LIN_WR = (E % (1 << SH)) == 0;
    const int pw = padk(t * E, SH);
    sync();  // previous readers of this shared buffer are done
    if (active) {
#pragma unroll
      for (int r = 0; r < E; ++r) {
        if constexpr (LIN_WR)
          lay.atp(pw + r + (r >> SH)) = v[r];
        else
          lay.at(t * E + r) = v[r];
      }
    }
    sync();
    fft_stages<N, E, DIR, E, false, Lay, Sync>(v, lay, sync, active, t, tw);
  }
}

// Product of the radices before the last stage (N when the transform is the
// single in-register stage, T = 1); the last stage has radix N / last_ns.
__host__ __device__ constexpr int last_ns(int N, int E) {
  int ns = E;
  while (ns < N) {
    const int r = (N / ns) < E ? (N / ns) : E;
    if (ns * r == N) return ns;
    ns *= r;
  }
  return N;
}

// fft_line without its last stage: on return the last stage's inputs are in
// shared memory (Stockham index a at lay.at(a)), synchronised within the line;
// with T = 1 the whole (in-register) transform is done and stored there.
template <int N, int E, int DIR, class Lay, class Sync>
__device__ __forceinline__ void fft_line_head(float2 (&v)[E], const Lay& lay, const Sync& sync,
                                              bool active, int t, const float2* __restrict__ tw) {
  static_assert(E <= N && (N % E) == 0, "E must divide N");
  constexpr int T = N / E;
  constexpr int SH = Lay::kShift;
  dft<E, DIR>(v);
  sync();  // previous readers of this shared buffer are done
  if constexpr (T == 1) {
    if (active) {
#pragma unroll
      for (int r = 0; r < E; ++r) lay.at(r) = v[r];
    }
    sync();
  } else {
    constexpr bool LIN_WR = (E % (1 << SH)) == 0;
    const int pw = padk(t * E, SH);
    if (active) {
#pragma unroll
      for (int r = 0; r < E; ++r) {
        if constexpr (LIN_WR)
          lay.atp(pw + r + (r >> SH)) = v[r];
        else
          lay.at(t * E + r) = v[r];
      }
    }
    sync();
    fft_stages<N, E, DIR, E, true, Lay, Sync>(v, lay, sync, active, t, tw);
  }
}

}  // namespace sp
