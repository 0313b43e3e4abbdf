// Subpixel registration of frames to a reference frame and their alignment:
// the "align global phase and subpixel shift to trial 0, then average" step
// of the batched-trials workload.  The reference aligns frames only by whole
// pixels (conditioning.align_frames, speckle/conditioning.py:316-430, with
// crosscorr.alignment_coordinates, speckle/crosscorr.py:526-568); this keeps
// its cross-correlation convention and answers at integer shifts and refines
// the peak by the single-step upsampled DFT of Guizar-Sicairos, Thurman &
// Fienup ("Efficient subpixel image registration algorithms", Opt. Lett. 33,
// 156-158, 2008):
//   1. F_f = FFT2(frame f embedded at the corner of N x N), R = the reference's
//   2. X_f = F_f conj(R); c_f = IFFT2(X_f); d0 = the argmax of the fftshifted
//      |c_f| (ties to the first index, as numpy's argmax), a signed shift
//   3. the cross-correlation upsampled by U on an M x M grid (M = ceil(1.5 U))
//      centred on d0: c(d0 + (p - h, q - h)/U) for p, q < M, h = M/2, as two
//      matrix products of X_f' = X_f exp(2 pi i k.d0/N) (signed frequencies)
//      with W[k][q] = exp(2 pi i k (q - h)/(U N)) -- rows first, then columns
//   4. d = d0 + (p* - h, q* - h)/U at the largest |c|, theta = arg c there
//   5. aligned_f = IFFT2(F_f exp(2 pi i k.d/N) exp(-i theta)), cropped: the
//      frame moved by d (aligned_f(y) = frame_f(y + d)) and rotated onto the
//      reference's global phase
// Every phase argument is an integer numerator over N or U N, reduced exactly
// in integers before the (float) sincospi.
#include <algorithm>
#include <cmath>

#include "sp_common.cuh"

namespace sp {

cudaError_t fft2_dispatch(const float2* in, float2* out, int N, int batch, int inverse,
                          cudaStream_t st);

static inline int upsampled_points(int U) { return (3 * U + 1) / 2; }  // ceil(1.5 U)

__device__ __forceinline__ int signed_freq(int k, int N) { return k >= N / 2 ? k - N : k; }

// exp(2 pi i num / den) with num reduced modulo den exactly first
__device__ __forceinline__ float2 turn(long long num, long long den) {
  long long r = num % den;
  if (r < 0) r += den;
  float s, c;
  sincospif(2.0f * (float)((double)r / (double)den), &s, &c);
  return make_float2(c, s);
}
// the same for a power-of-two denominator N: the residue is a mask (two's
// complement gives the non-negative residue of a negative numerator too)
__device__ __forceinline__ float2 turn_pow2(int num, int N) {
  float s, c;
  sincospif(2.0f * (float)(num & (N - 1)) / (float)N, &s, &c);
  return make_float2(c, s);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// frames (n, rows, cols) at the corner of zeroed N x N planes
__global__ void reg_embed_kernel(const float2* __restrict__ src, float2* __restrict__ dst, int n,
                                 int rows, int cols, int N) {
  const long long total = (long long)n * N * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const long long f = k / ((long long)N * N);
    const long long rem = k - f * N * N;
    const int r = (int)(rem / N), c = (int)(rem - (long long)r * N);
    dst[k] = (r < rows && c < cols) ? src[(f * rows + r) * cols + c] : make_float2(0.f, 0.f);
  }
}

// X_f = F_f conj(R)
__global__ void reg_cross_kernel(const float2* __restrict__ F, const float2* __restrict__ R,
                                 float2* __restrict__ X, int n, long long NN) {
  const long long total = (long long)n * NN;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x)
    X[k] = cmulc(F[k], R[k % NN]);
}

// per frame: max over the fftshifted |c_f|, keyed (|c| bits << 32 | ~index)
__global__ void reg_argmax_kernel(const float2* __restrict__ C, int N,
                                  unsigned long long* __restrict__ best) {
  const int f = blockIdx.y;
  const long long NN = (long long)N * N;
  const float2* c = C + f * NN;
  unsigned long long mine = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < NN;
       k += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(k / N), cc = (int)(k - (long long)r * N);
    const uint32_t sidx = (uint32_t)(((r + N / 2) % N) * N + (cc + N / 2) % N);
    const float2 v = c[k];
    const float m = sqrtf(v.x * v.x + v.y * v.y);
    const unsigned long long key = ((unsigned long long)__float_as_uint(m) << 32) | (0xffffffffu - sidx);
    mine = key > mine ? key : mine;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, mine, o);
    mine = other > mine ? other : mine;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(&best[f], mine);
}

// the signed coarse shift d0 of frame f from its argmax key
__device__ __forceinline__ int2 coarse_shift(unsigned long long key, int N) {
  const uint32_t sidx = 0xffffffffu - (uint32_t)(key & 0xffffffffu);
  return make_int2((int)(sidx / N) - N / 2, (int)(sidx % N) - N / 2);
}

// W[k][q] = exp(2 pi i k_s (q - h) / (U N)), k < N, q < M
__global__ void reg_kernel_table(float2* __restrict__ W, int N, int U, int M) {
  const int h = M / 2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * M; i += gridDim.x * blockDim.x) {
    const int k = i / M, q = i - k * M;
    W[i] = turn((long long)signed_freq(k, N) * (q - h), (long long)U * N);
  }
}

// T1[f][ky][q] = sum_kx X_f'[ky][kx] W[kx][q], X_f' = F_f conj(R) exp(2 pi i k.d0/N).
// CTA: 32 rows ky of one frame, all M columns; kx in chunks of 32 through
// shared memory.  The modulation is separable, exp(2 pi i ky d0y/N) times
// exp(2 pi i kx d0x/N): the CTA's row factors are made once, each chunk's
// column factors once per chunk.  Thread (tr, tq) accumulates the register
// tile of rows tr + 8 j (j < 4) and columns tq + 32 m (m < 8, up to M).
constexpr int kRegRows = 32, kRegK = 32, kRegThreads = 256;
__global__ void __launch_bounds__(kRegThreads) reg_upsample_rows_kernel(
    const float2* __restrict__ F, const float2* __restrict__ R, const float2* __restrict__ W,
    const unsigned long long* __restrict__ best, float2* __restrict__ T1, int N, int M) {
  extern __shared__ float2 sm[];
  float2* xs = sm;                           // [kRegRows][kRegK + 1]
  float2* ws = sm + kRegRows * (kRegK + 1);  // [kRegK][M]
  __shared__ float2 rowf[kRegRows], colf[kRegK];
  const int f = blockIdx.y;
  const int ky0 = blockIdx.x * kRegRows;
  const long long NN = (long long)N * N;
  const int2 d0 = coarse_shift(best[f], N);
  const float2* Ff = F + f * NN;
  if (threadIdx.x < kRegRows) rowf[threadIdx.x] = turn_pow2(signed_freq(ky0 + threadIdx.x, N) * d0.x, N);
  const int tr = threadIdx.x / 32, tq = threadIdx.x % 32;
  constexpr int MQ = 8;  // up to 256 columns
  float2 acc[4][MQ];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int m = 0; m < MQ; ++m) acc[j][m] = make_float2(0.f, 0.f);
  for (int kx0 = 0; kx0 < N; kx0 += kRegK) {
    __syncthreads();  // the previous chunk's tiles are consumed
    if (threadIdx.x < kRegK) colf[threadIdx.x] = turn_pow2(signed_freq(kx0 + threadIdx.x, N) * d0.y, N);
    __syncthreads();
    for (int i = threadIdx.x; i < kRegRows * kRegK; i += blockDim.x) {
      const int rr = i / kRegK, kk = i - rr * kRegK;
      const int ky = ky0 + rr, kx = kx0 + kk;
      float2 v = make_float2(0.f, 0.f);
      if (ky < N && kx < N) {
        const long long idx = (long long)ky * N + kx;
        v = cmul(cmul(cmulc(Ff[idx], R[idx]), rowf[rr]), colf[kk]);
      }
      xs[rr * (kRegK + 1) + kk] = v;
    }
    for (int i = threadIdx.x; i < kRegK * M; i += blockDim.x) {
      const int kk = i / M, q = i - kk * M;
      ws[i] = (kx0 + kk < N) ? W[(long long)(kx0 + kk) * M + q] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int kk = 0; kk < kRegK; ++kk) {
      float2 x[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) x[j] = xs[(tr + 8 * j) * (kRegK + 1) + kk];
#pragma unroll
      for (int m = 0; m < MQ; ++m) {
        const int q = tq + 32 * m;
        if (q < M) {
          const float2 w = ws[kk * M + q];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            acc[j][m].x = fmaf(x[j].x, w.x, fmaf(-x[j].y, w.y, acc[j][m].x));
            acc[j][m].y = fmaf(x[j].x, w.y, fmaf(x[j].y, w.x, acc[j][m].y));
          }
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int ky = ky0 + tr + 8 * j;
    if (ky >= N) continue;
#pragma unroll
    for (int m = 0; m < MQ; ++m) {
      const int q = tq + 32 * m;
      if (q < M) T1[((long long)f * N + ky) * M + q] = acc[j][m];
    }
  }
}

// c_f[p][q] = sum_ky W[ky][p] T1_f[ky][q]; CTA: 8 rows p of one frame, all
// M columns; the CTA's largest |c| goes into best_up[f] (ties to the first
// index p M + q).
__global__ void __launch_bounds__(kRegThreads) reg_upsample_cols_kernel(
    const float2* __restrict__ T1, const float2* __restrict__ W, int N, int M,
    unsigned long long* __restrict__ best_up) {
  const int f = blockIdx.y;
  const int p0 = blockIdx.x * 8;
  const int tp = threadIdx.x / 32, tq = threadIdx.x % 32;
  const int p = p0 + tp;
  constexpr int MQ = 8;
  float2 acc[MQ];
#pragma unroll
  for (int m = 0; m < MQ; ++m) acc[m] = make_float2(0.f, 0.f);
  const float2* t1 = T1 + (long long)f * N * M;
  if (p < M) {
    for (int ky = 0; ky < N; ++ky) {
      const float2 w = W[(long long)ky * M + p];
#pragma unroll
      for (int m = 0; m < MQ; ++m) {
        const int q = tq + 32 * m;
        if (q < M) {
          const float2 t = t1[(long long)ky * M + q];
          acc[m].x = fmaf(w.x, t.x, fmaf(-w.y, t.y, acc[m].x));
          acc[m].y = fmaf(w.x, t.y, fmaf(w.y, t.x, acc[m].y));
        }
      }
    }
  }
  unsigned long long mine = 0;
  if (p < M) {
#pragma unroll
    for (int m = 0; m < MQ; ++m) {
      const int q = tq + 32 * m;
      if (q < M) {
        const float mag = sqrtf(acc[m].x * acc[m].x + acc[m].y * acc[m].y);
        const unsigned long long key = ((unsigned long long)__float_as_uint(mag) << 32) |
                                       (0xffffffffu - (uint32_t)(p * M + q));
        mine = key > mine ? key : mine;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, mine, o);
    mine = other > mine ? other : mine;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(&best_up[f], mine);
}

// Per frame (one warp each): the refined shift d = d0 + (p* - h, q* - h)/U
// (as the integer numerators d U), the phase of c at the peak (recomputed in
// FP64 from T1), and the result record shifts[f] = (dy, dx, theta).
__global__ void reg_finish_kernel(const float2* __restrict__ T1, const float2* __restrict__ W,
                                  const unsigned long long* __restrict__ best,
                                  const unsigned long long* __restrict__ best_up, int n, int N,
                                  int U, int M, int2* __restrict__ num, double* __restrict__ shifts) {
  const int f = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (f >= n) return;
  const int2 d0 = coarse_shift(best[f], N);
  const uint32_t idx = 0xffffffffu - (uint32_t)(best_up[f] & 0xffffffffu);
  const int p = (int)(idx / M), q = (int)(idx % M), h = M / 2;
  const float2* t1 = T1 + (long long)f * N * M;
  double re = 0.0, im = 0.0;
  for (int ky = lane; ky < N; ky += 32) {
    const float2 w = W[(long long)ky * M + p], t = t1[(long long)ky * M + q];
    re += (double)w.x * t.x - (double)w.y * t.y;
    im += (double)w.x * t.y + (double)w.y * t.x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if (lane == 0) {
    const int ny = d0.x * U + (p - h), nx = d0.y * U + (q - h);
    num[f] = make_int2(ny, nx);
    shifts[3 * f] = (double)ny / U;
    shifts[3 * f + 1] = (double)nx / U;
    shifts[3 * f + 2] = atan2(im, re);
  }
}

// F_f <- F_f exp(2 pi i k.d/N) exp(-i theta), d = num / U.  With
// num = d0 U + (p - h) per axis the ramp factors into the whole-pixel turn
// exp(2 pi i k d0 / N) and the kernel-table entry W[k][p] = exp(2 pi i k (p - h)/(U N)).
__global__ void reg_shift_kernel(float2* __restrict__ F, int n, int N, int U, int M,
                                 const float2* __restrict__ W, const int2* __restrict__ num,
                                 const double* __restrict__ shifts) {
  const long long NN = (long long)N * N, total = (long long)n * NN;
  const int h = M / 2;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(k / NN);
    const long long rem = k - f * NN;
    const int ky = (int)(rem / N), kx = (int)(rem - (long long)ky * N);
    const int2 d = num[f];
    // floor division of the numerators by U: d = d0 U + (p - h), p - h in [-h, h]
    const int d0y = (d.x + h) >= 0 ? (d.x + h) / U : -((-(d.x + h) + U - 1) / U);
    const int d0x = (d.y + h) >= 0 ? (d.y + h) / U : -((-(d.y + h) + U - 1) / U);
    const int py = d.x - d0y * U + h, px = d.y - d0x * U + h;
    float2 w = turn_pow2(signed_freq(ky, N) * d0y + signed_freq(kx, N) * d0x, N);
    w = cmul(w, cmul(W[(long long)ky * M + py], W[(long long)kx * M + px]));
    const double th = shifts[3 * f + 2];
    F[k] = cmul(F[k], cmul(w, make_float2((float)cos(th), (float)-sin(th))));
  }
}

// crop the (corner) rows x cols of each N x N plane
__global__ void reg_crop_kernel(const float2* __restrict__ src, float2* __restrict__ dst, int n,
                                int rows, int cols, int N) {
  const long long total = (long long)n * rows * cols;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const long long f = k / ((long long)rows * cols);
    const long long rem = k - f * rows * cols;
    const int r = (int)(rem / cols), c = (int)(rem - (long long)r * cols);
    dst[k] = src[(f * N + r) * N + c];
  }
}

struct RegLayout {
  size_t F, X, W, best, best_up, num, total;
};
static RegLayout reg_layout(int n, int N, int U) {
  const int M = upsampled_points(U);
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  RegLayout L;
  const size_t NN = (size_t)N * N;
  L.F = 0;
  L.X = L.F + al(sizeof(float2) * (n + 1) * NN);  // frames and (last) the reference
  L.W = L.X + al(sizeof(float2) * (size_t)n * N * (size_t)(N > M ? N : M));
  L.best = L.W + al(sizeof(float2) * (size_t)N * M);
  L.best_up = L.best + al(sizeof(unsigned long long) * n);
  L.num = L.best_up + al(sizeof(unsigned long long) * n);
  L.total = L.num + al(sizeof(int2) * n);
  return L;
}

}  // namespace sp

using namespace sp;

extern "C" int sp_register_workspace_size(int n_frames, int N, int upsample, size_t* bytes) {
  SP_CHECK(bytes && n_frames > 0 && upsample >= 1 && upsample <= 170, SP_ERR_INVALID,
           "sp_register_workspace_size: bad argument");
  SP_CHECK(is_pow2(N) && N >= kMinN && N <= kMaxN, SP_ERR_SIZE, "sp_register: N=%d", N);
  *bytes = reg_layout(n_frames, N, upsample).total;
  return SP_OK;
}

extern "C" int sp_register_subpixel(const void* frames_dev, int n_frames, int rows, int cols,
                                    const void* ref_dev, int N, int upsample, void* work_dev,
                                    size_t work_bytes, double* shifts_dev, void* out_dev,
                                    sp_stream_t stream) {
  SP_CHECK(frames_dev && ref_dev && work_dev && shifts_dev && n_frames > 0, SP_ERR_INVALID,
           "sp_register_subpixel: bad argument");
  SP_CHECK(is_pow2(N) && N >= kMinN && N <= kMaxN, SP_ERR_SIZE, "sp_register_subpixel: N=%d", N);
  SP_CHECK(rows > 0 && cols > 0 && rows <= N && cols <= N, SP_ERR_INVALID,
           "sp_register_subpixel: frames of %d x %d do not fit N=%d", rows, cols, N);
  SP_CHECK(upsample >= 1 && upsample <= 170, SP_ERR_INVALID,
           "sp_register_subpixel: upsample=%d not in [1, 170]", upsample);
  SP_CHECK(n_frames <= 65535, SP_ERR_SIZE, "sp_register_subpixel: at most 65535 frames");
  const RegLayout L = reg_layout(n_frames, N, upsample);
  SP_CHECK(work_bytes >= L.total, SP_ERR_WORKSPACE, "sp_register_subpixel: %zu bytes given, %zu needed",
           work_bytes, L.total);
  const int U = upsample, M = upsampled_points(U);
  cudaStream_t st = as_stream(stream);
  char* ws = static_cast<char*>(work_dev);
  float2* F = reinterpret_cast<float2*>(ws + L.F);
  float2* Rf = F + (size_t)n_frames * N * N;
  float2* X = reinterpret_cast<float2*>(ws + L.X);
  float2* W = reinterpret_cast<float2*>(ws + L.W);
  auto* best = reinterpret_cast<unsigned long long*>(ws + L.best);
  auto* best_up = reinterpret_cast<unsigned long long*>(ws + L.best_up);
  int2* num = reinterpret_cast<int2*>(ws + L.num);
  const long long NN = (long long)N * N;
  auto grid = [](long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 16); };
  reg_embed_kernel<<<grid(n_frames * NN), 256, 0, st>>>((const float2*)frames_dev, F, n_frames, rows,
                                                        cols, N);
  reg_embed_kernel<<<grid(NN), 256, 0, st>>>((const float2*)ref_dev, Rf, 1, rows, cols, N);
  SP_CUDA_TRY(cudaGetLastError());
  SP_CUDA_TRY(fft2_dispatch(F, F, N, n_frames + 1, 0, st));
  reg_cross_kernel<<<grid(n_frames * NN), 256, 0, st>>>(F, Rf, X, n_frames, NN);
  SP_CUDA_TRY(cudaGetLastError());
  SP_CUDA_TRY(fft2_dispatch(X, X, N, n_frames, 1, st));
  SP_CUDA_TRY(cudaMemsetAsync(best, 0, sizeof(unsigned long long) * n_frames, st));
  SP_CUDA_TRY(cudaMemsetAsync(best_up, 0, sizeof(unsigned long long) * n_frames, st));
  {
    const int bx = (int)std::min<long long>((NN + 255) / 256, 32);
    reg_argmax_kernel<<<dim3(bx, n_frames), 256, 0, st>>>(X, N, best);
  }
  reg_kernel_table<<<grid((long long)N * M), 256, 0, st>>>(W, N, U, M);
  SP_CUDA_TRY(cudaGetLastError());
  const size_t smem = sizeof(float2) * ((size_t)kRegRows * (kRegK + 1) + (size_t)kRegK * M);
  SP_CUDA_TRY(cudaFuncSetAttribute(reg_upsample_rows_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  reg_upsample_rows_kernel<<<dim3((N + kRegRows - 1) / kRegRows, n_frames), kRegThreads, smem, st>>>(
      F, Rf, W, best, X, N, M);
  reg_upsample_cols_kernel<<<dim3((M + 7) / 8, n_frames), kRegThreads, 0, st>>>(X, W, N, M, best_up);
  reg_finish_kernel<<<(n_frames + 3) / 4, 128, 0, st>>>(X, W, best, best_up, n_frames, N, U, M,
                                                        num, shifts_dev);
  SP_CUDA_TRY(cudaGetLastError());
  if (out_dev) {
    reg_shift_kernel<<<grid(n_frames * NN), 256, 0, st>>>(F, n_frames, N, U, M, W, num, shifts_dev);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(fft2_dispatch(F, F, N, n_frames, 1, st));  // inverse, scaled by 1/N^2
    reg_crop_kernel<<<grid((long long)n_frames * rows * cols), 256, 0, st>>>(F, (float2*)out_dev,
                                                                            n_frames, rows, cols, N);
    SP_CUDA_TRY(cudaGetLastError());
  }
  return SP_OK;
}
