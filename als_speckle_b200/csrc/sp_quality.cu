// Trial-quality measures after phasing:
//  * RFTF (Marchesini et al.), the Fourier-error counterpart of the PRTF:
//    rftf (phasing.py:1521-1608, one estimate, numpy) and gpu_rftf
//    (phasing.py:1611-1708 with kernels/phasing_rftf_accumulate.cl,
//    common_abs2_f2_f2.cl, common_multiply_axis_f_f2.cl, common_sqrt_f2.cl);
//  * hot-pixel removal, 3 x 3 median with zero padding
//    (conditioning.remove_hot_pixels, conditioning.py:207-313, CPU branch);
//  * the pair-wise cross-correlation maxima of covar_results
//    (phasing.py:1817-1982): max |IFFT2(conj(D_a) D_b)| for pairs of
//    transformed reconstructions.
#include <cuda_runtime.h>

#include "sp_common.cuh"
#include "sp_fft2.cuh"

namespace sp {
namespace {

int grid_of(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return (int)(g < 1 ? 1 : g);
}

#define SP_GRID_STRIDE(i, n)                                                   \
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); \
       i += (int64_t)gridDim.x * blockDim.x)

// (|x|^2, 0)  -- common_abs2_f2_f2.cl
__global__ void abs2_kernel(const float2* in, float2* out, int64_t n) {
  SP_GRID_STRIDE(i, n) {
    const float2 a = in[i];
    out[i] = make_float2(a.x * a.x + a.y * a.y, 0.f);
  }
}

// principal complex square root  -- common_sqrt_f2.cl
__global__ void sqrt_f2_kernel(const float2* in, float2* out, int64_t n) {
  SP_GRID_STRIDE(i, n) {
    const float a = in[i].x, b = in[i].y;
    const float h = hypotf(a, b);
    const float sg = b > 0.f ? 1.f : (b < 0.f ? -1.f : 0.f);  // OpenCL sign()
    out[i] = make_float2(sqrtf((h + a) * 0.5f), sg * sqrtf((h - a) * 0.5f));
  }
}

// (sqrt(|x|), 0): numpy's np.sqrt(np.abs(.)) of the CPU rftf (phasing.py:1577)
__global__ void sqrt_abs_kernel(const float2* in, float2* out, int64_t n) {
  SP_GRID_STRIDE(i, n) {
    const float2 a = in[i];
    out[i] = make_float2(sqrtf(sqrtf(a.x * a.x + a.y * a.y)), 0.f);
  }
}

// out[f][k] = in1[k] * in2[f][k], in1 real  -- common_multiply_axis_f_f2.cl
__global__ void multiply_axis_kernel(int frames, const float* in1, const float2* in2, float2* out,
                                     int64_t plane) {
  SP_GRID_STRIDE(k, plane) {
    const float a = in1[k];
    for (int f = 0; f < frames; ++f) {
      const float2 b = in2[k + f * plane];
      out[k + f * plane] = make_float2(a * b.x, a * b.y);
    }
  }
}

// out = a * b, complex  -- common_multiply_f2_f2.cl
__global__ void multiply_f2_kernel(const float2* a, const float2* b, float2* out, int64_t n) {
  SP_GRID_STRIDE(i, n) {
    const float2 x = a[i], y = b[i];
    out[i] = make_float2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
  }
}

// RFTF over frames  -- phasing_rftf_accumulate.cl: mean over frames of
// 1/sqrt(1 + (g - F.x)^2 / g^2), summed as the kernel does (term / frames,
// float).  Written at the fftshifted position when shift != 0 (gpu_rftf
// shifts the result, phasing.py:1700).
__global__ void rftf_accumulate_kernel(int frames, const float* goal, float* acc,
                                       const float2* fourier, int N, int shift) {
  const int64_t plane = (int64_t)N * N;
  SP_GRID_STRIDE(k, plane) {
    const float g = goal[k];
    float cum = 0.f;
    for (int f = 0; f < frames; ++f) {
      const float d1 = g - fourier[k + f * plane].x;
      const float d = (d1 * d1) / (g * g);
      const float e = 1.f / sqrtf(1.f + d);
      cum = cum + e / (float)frames;
    }
    int64_t o = k;
    if (shift) {
      const int r = (int)(k / N), c = (int)(k % N);
      o = (int64_t)((r + N / 2) % N) * N + (c + N / 2) % N;
    }
    acc[o] = cum;
  }
}

// FP64 sums[0] = sum |F - g|, sums[1] = sum |shift(F) - g| (rftf's choice
// between a goal modulus centred at (0,0) and at (N/2,N/2), phasing.py:1583-1584);
// F is the real part of `fourier`.
__global__ void rftf_align_sums_kernel(const float2* fourier, const float* goal, int N,
                                       double* sums) {
  const int64_t plane = (int64_t)N * N;
  double s1 = 0.0, s2 = 0.0;
  SP_GRID_STRIDE(k, plane) {
    const int r = (int)(k / N), c = (int)(k % N);
    // shift(F)[r][c] = F[(r + N/2) % N][(c + N/2) % N]
    const int64_t src = (int64_t)((r + N / 2) % N) * N + (c + N / 2) % N;
    const float g = goal[k];
    s1 += fabs((double)(fourier[k].x - g));
    s2 += fabs((double)(fourier[src].x - g));
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sums[0], s1);
    atomicAdd(&sums[1], s2);
  }
}

// error map of rftf (phasing.py:1586-1591), in the centred layout:
//   goal at (0,0):   err = shift((F - g)^2 / g^2)
//   goal centred:    err = (shift(F) - g)^2 / g^2
__global__ void rftf_error_kernel(const float2* fourier, const float* goal, int N, int centred,
                                  float* err) {
  const int64_t plane = (int64_t)N * N;
  SP_GRID_STRIDE(k, plane) {
    const int r = (int)(k / N), c = (int)(k % N);
    const int64_t sk = (int64_t)((r + N / 2) % N) * N + (c + N / 2) % N;  // shifted partner
    float f, g;
    if (centred) {
      f = fourier[sk].x;
      g = goal[k];
    } else {
      f = fourier[sk].x;
      g = goal[sk];
    }
    const float d = f - g;
    err[k] = (d * d) / (g * g);
  }
}

// rftf = sqrt(1 / (1 + err)), optionally rescaled from [1/sqrt 2, 1] to [0, 1]
// (phasing.py:1597-1601)
__global__ void rftf_from_error_kernel(const float* err, float* out, int64_t n, int scale) {
  SP_GRID_STRIDE(i, n) {
    float v = sqrtf(1.f / (1.f + err[i]));
    if (scale) {
      const float x = 0.70710678118654752f;
      v = (v - x) / (1.f - x);
    }
    out[i] = v;
  }
}

// one pass of remove_hot_pixels' CPU branch (conditioning.py:304-305):
// median = medfilt3x3(frame) + 0.1 (zero padding), frame = median where
// frame / median > threshold
__device__ __forceinline__ void sort_swap(float& a, float& b) {
  const float lo = fminf(a, b), hi = fmaxf(a, b);
  a = lo;
  b = hi;
}
__global__ void hot_pixels_kernel(const float* in, float* out, int rows, int cols,
                                  float threshold) {
  const int64_t n = (int64_t)rows * cols;
  SP_GRID_STRIDE(k, n) {
    const int r = (int)(k / cols), c = (int)(k % cols);
    float w[9];
    int q = 0;
    for (int dr = -1; dr <= 1; ++dr)
      for (int dc = -1; dc <= 1; ++dc) {
        const int rr = r + dr, cc = c + dc;
        w[q++] = (rr >= 0 && rr < rows && cc >= 0 && cc < cols) ? in[(int64_t)rr * cols + cc] : 0.f;
      }
    // median of the nine (sorted by adjacent exchanges)
    for (int i = 0; i < 9; ++i)
      for (int j = 0; j < 8 - i; ++j) sort_swap(w[j], w[j + 1]);
    const float med = w[4] + 0.1f;
    const float v = in[k];
    out[k] = (v / med > threshold) ? med : v;
  }
}

// products conj(D_a) * D_b for a chunk of pairs (covar_results' conj_mult)
__global__ void covar_products_kernel(const float2* dfts, const int2* pairs, int n_pairs,
                                      int64_t plane, float2* out) {
  const int64_t total = plane * n_pairs;
  SP_GRID_STRIDE(i, total) {
    const int p = (int)(i / plane);
    const int64_t k = i - (int64_t)p * plane;
    const int2 pr = pairs[p];
    const float2 a = dfts[(int64_t)pr.x * plane + k], b = dfts[(int64_t)pr.y * plane + k];
    out[i] = make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
  }
}

// cc[p] = max |plane p| (one block per plane)
__global__ void plane_max_abs_kernel(const float2* in, int64_t plane, float* cc) {
  const float2* x = in + (int64_t)blockIdx.x * plane;
  float m = 0.f;
  for (int64_t k = threadIdx.x; k < plane; k += blockDim.x) m = fmaxf(m, hypotf(x[k].x, x[k].y));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float r = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmaxf(r, red[w]);
    cc[blockIdx.x] = r;
  }
}

}  // namespace
}  // namespace sp

using namespace sp;

#define SP_N_CHECK(N, who)                                                          \
  SP_CHECK(is_pow2(N) && (N) >= kMinN && (N) <= kMaxN, SP_ERR_SIZE,                 \
           "%s: N=%d must be a power of two in [%d, %d]", who, (int)(N), kMinN, kMaxN)

extern "C" {

int sp_abs2_f2_f2(const void* in, void* out, int64_t n, sp_stream_t stream) {
  SP_CHECK(in && out && n >= 0, SP_ERR_INVALID, "sp_abs2_f2_f2: bad argument");
  if (n == 0) return SP_OK;
  abs2_kernel<<<grid_of(n), 256, 0, as_stream(stream)>>>((const float2*)in, (float2*)out, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_sqrt_f2(const void* in, void* out, int64_t n, sp_stream_t stream) {
  SP_CHECK(in && out && n >= 0, SP_ERR_INVALID, "sp_sqrt_f2: bad argument");
  if (n == 0) return SP_OK;
  sqrt_f2_kernel<<<grid_of(n), 256, 0, as_stream(stream)>>>((const float2*)in, (float2*)out, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_sqrt_abs_f2(const void* in, void* out, int64_t n, sp_stream_t stream) {
  SP_CHECK(in && out && n >= 0, SP_ERR_INVALID, "sp_sqrt_abs_f2: bad argument");
  if (n == 0) return SP_OK;
  sqrt_abs_kernel<<<grid_of(n), 256, 0, as_stream(stream)>>>((const float2*)in, (float2*)out, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_multiply_axis_f_f2(int frames, const float* in1, const void* in2, void* out, int64_t plane,
                          sp_stream_t stream) {
  SP_CHECK(in1 && in2 && out && frames >= 0 && plane >= 0, SP_ERR_INVALID,
           "sp_multiply_axis_f_f2: bad argument");
  if (frames == 0 || plane == 0) return SP_OK;
  multiply_axis_kernel<<<grid_of(plane), 256, 0, as_stream(stream)>>>(
      frames, in1, (const float2*)in2, (float2*)out, plane);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_multiply_f2_f2(const void* a, const void* b, void* out, int64_t n, sp_stream_t stream) {
  SP_CHECK(a && b && out && n >= 0, SP_ERR_INVALID, "sp_multiply_f2_f2: bad argument");
  if (n == 0) return SP_OK;
  multiply_f2_kernel<<<grid_of(n), 256, 0, as_stream(stream)>>>((const float2*)a, (const float2*)b,
                                                                (float2*)out, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_rftf_accumulate(int frames, const float* goal, float* accumulation, const void* fourier,
                       int N, int shift, sp_stream_t stream) {
  SP_N_CHECK(N, "sp_rftf_accumulate");
  SP_CHECK(goal && accumulation && fourier && frames > 0, SP_ERR_INVALID,
           "sp_rftf_accumulate: bad argument");
  rftf_accumulate_kernel<<<grid_of((int64_t)N * N), 256, 0, as_stream(stream)>>>(
      frames, goal, accumulation, (const float2*)fourier, N, shift);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_rftf_map(const void* fourier, const float* goal, int N, int scale, double* sums,
                float* err, float* out, sp_stream_t stream) {
  SP_N_CHECK(N, "sp_rftf_map");
  SP_CHECK(fourier && goal && sums && err && out, SP_ERR_INVALID, "sp_rftf_map: null pointer");
  cudaStream_t st = as_stream(stream);
  const int64_t plane = (int64_t)N * N;
  SP_CUDA_TRY(cudaMemsetAsync(sums, 0, 2 * sizeof(double), st));
  rftf_align_sums_kernel<<<grid_of(plane), 256, 0, st>>>((const float2*)fourier, goal, N, sums);
  SP_CUDA_TRY(cudaGetLastError());
  double h[2];
  SP_CUDA_TRY(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, st));
  SP_CUDA_TRY(cudaStreamSynchronize(st));
  // the reference leaves `error` unbound when the two sums are equal; the
  // goal is then taken to be centred at (0,0)
  const int centred = h[0] > h[1] ? 1 : 0;
  rftf_error_kernel<<<grid_of(plane), 256, 0, st>>>((const float2*)fourier, goal, N, centred, err);
  SP_CUDA_TRY(cudaGetLastError());
  rftf_from_error_kernel<<<grid_of(plane), 256, 0, st>>>(err, out, plane, scale);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_rftf_from_error(const float* err, float* out, int64_t n, int scale, sp_stream_t stream) {
  SP_CHECK(err && out && n >= 0, SP_ERR_INVALID, "sp_rftf_from_error: bad argument");
  if (n == 0) return SP_OK;
  rftf_from_error_kernel<<<grid_of(n), 256, 0, as_stream(stream)>>>(err, out, n, scale);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_remove_hot_pixels(float* data, float* work, int frames, int rows, int cols, int iterations,
                         float threshold, sp_stream_t stream) {
  SP_CHECK(data && work && frames >= 0 && rows > 0 && cols > 0 && iterations > 0, SP_ERR_INVALID,
           "sp_remove_hot_pixels: bad argument");
  cudaStream_t st = as_stream(stream);
  const int64_t plane = (int64_t)rows * cols;
  for (int f = 0; f < frames; ++f) {
    float* x = data + f * plane;
    for (int it = 0; it < iterations; ++it) {
      hot_pixels_kernel<<<grid_of(plane), 256, 0, st>>>(x, work, rows, cols, threshold);
      SP_CUDA_TRY(cudaGetLastError());
      SP_CUDA_TRY(cudaMemcpyAsync(x, work, plane * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
  }
  return SP_OK;
}

int sp_covar_pairs(const void* dfts, int N, const int32_t* pairs, int n_pairs, void* work,
                   int work_planes, float* cc, sp_stream_t stream) {
  SP_N_CHECK(N, "sp_covar_pairs");
  SP_CHECK(dfts && pairs && work && cc && n_pairs >= 0 && work_planes > 0, SP_ERR_INVALID,
           "sp_covar_pairs: bad argument");
  cudaStream_t st = as_stream(stream);
  const int64_t plane = (int64_t)N * N;
  const int2* pr = reinterpret_cast<const int2*>(pairs);
  for (int p0 = 0; p0 < n_pairs; p0 += work_planes) {
    const int cnt = n_pairs - p0 < work_planes ? n_pairs - p0 : work_planes;
    covar_products_kernel<<<grid_of(plane * cnt), 256, 0, st>>>(
        (const float2*)dfts, pr + p0, cnt, plane, (float2*)work);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(fft2_dispatch((const float2*)work, (float2*)work, N, cnt, 1, st));
    plane_max_abs_kernel<<<cnt, 256, 0, st>>>((const float2*)work, plane, cc + p0);
    SP_CUDA_TRY(cudaGetLastError());
  }
  return SP_OK;
}

}  // extern "C"
