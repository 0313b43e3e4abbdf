// Estimating the coherence function from reconstructions
// (phasing.optimize_coherence, phasing.py:507-930):
//  * Richardson-Lucy deconvolution of the measured intensity by the
//    reconstruction's intensity (_opt_iter_rl, :702-738), batched over frames;
//  * the objective of the Gaussian fit (_opt_iter_g, :663-700): the speckle
//    of the autocorrelation damped by a Gaussian coherence function, against
//    the measured modulus.
// Elementwise kernels mirror kernels/common_divide_f2_f2.cl,
// common_flip_f2.cl and common_gaussian_f.cl.
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

__device__ __forceinline__ float2 cdiv(float2 x, float2 y) {  // common_divide_f2_f2.cl
  const float denom = y.x * y.x + y.y * y.y;
  return make_float2((x.x * y.x + x.y * y.y) / denom, (x.y * y.x - x.x * y.y) / denom);
}

__device__ __forceinline__ float2 cmulf(float2 x, float2 y) {
  return make_float2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
}

// out = in1 / in2 (complex), in1 broadcast over frames when bcast != 0
__global__ void divide_kernel(const float2* in1, const float2* in2, float2* out, int64_t n,
                              int64_t plane, int bcast) {
  SP_GRID_STRIDE(i, n) out[i] = cdiv(in1[bcast ? i % plane : i], in2[i]);
}

// out[i2][j2] = in[i][j], i2 = N-1-i, j2 = N-1-j, per plane  -- common_flip_f2.cl
__global__ void flip_kernel(const float2* in, float2* out, int N, int64_t n) {
  const int64_t plane = (int64_t)N * N;
  SP_GRID_STRIDE(k, n) {
    const int64_t p = k / plane, r = k - p * plane;
    const int i = (int)(r / N), j = (int)(r % N);
    out[p * plane + (int64_t)(N - 1 - i) * N + (N - 1 - j)] = in[k];
  }
}

// the Gaussian coherence function in corner-centred coordinates
// (common_gaussian_f.cl; also shape.gaussian fftshifted, phasing.py:807)
__device__ __forceinline__ float gauss_at(int64_t k, int N, float sx, float sy) {
  int i = (int)(k / N), j = (int)(k % N);
  if (i > N / 2) i -= N;
  if (j > N / 2) j -= N;
  const float fi = (float)i, fj = (float)j;
  return expf(-(fi * fi) / (2.f * sx * sx)) * expf(-(fj * fj) / (2.f * sy * sy));
}

__global__ void gaussian_kernel(void* out, int N, float sx, float sy, int complex_out) {
  const int64_t plane = (int64_t)N * N;
  SP_GRID_STRIDE(k, plane) {
    const float g = gauss_at(k, N, sx, sy);
    if (complex_out) static_cast<float2*>(out)[k] = make_float2(g, 0.f);
    else static_cast<float*>(out)[k] = g;
  }
}

// work = gaussian(sx, sy) * ac
__global__ void damp_kernel(const float2* ac, float2* work, int N, float sx, float sy) {
  const int64_t plane = (int64_t)N * N;
  SP_GRID_STRIDE(k, plane) {
    const float g = gauss_at(k, N, sx, sy);
    work[k] = make_float2(g * ac[k].x, g * ac[k].y);
  }
}

// sum += (sqrt(|x|) - m)^2 in FP64
__global__ void speckle_misfit_kernel(const float2* x, const float* m, int64_t n, double* sum) {
  double s = 0.0;
  SP_GRID_STRIDE(k, n) {
    const float d = sqrtf(hypotf(x[k].x, x[k].y)) - m[k];
    s += (double)(d * d);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(sum, s);
}

// out = a * b (complex), elementwise over n
__global__ void multiply_kernel(const float2* a, const float2* b, float2* out, int64_t n) {
  SP_GRID_STRIDE(i, n) out[i] = cmulf(a[i], b[i]);
}

}  // namespace
}  // namespace sp

using namespace sp;

#define SP_N_CHECK(N, who)                                                          \
  SP_CHECK(is_pow2(N) && (N) >= kMinN && (N) <= kMaxN, SP_ERR_SIZE,                 \
           "%s: N=%d must be a power of two in [%d, %d]", who, (int)(N), kMinN, kMaxN)

extern "C" {

int sp_divide_f2_f2(const void* in1, const void* in2, void* out, int64_t n, sp_stream_t stream) {
  SP_CHECK(in1 && in2 && out && n >= 0, SP_ERR_INVALID, "sp_divide_f2_f2: bad argument");
  if (n == 0) return SP_OK;
  divide_kernel<<<grid_of(n), 256, 0, as_stream(stream)>>>((const float2*)in1, (const float2*)in2,
                                                           (float2*)out, n, n, 0);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_flip_f2(const void* in, void* out, int N, int planes, sp_stream_t stream) {
  SP_CHECK(in && out && in != out && N > 0 && planes >= 0, SP_ERR_INVALID,
           "sp_flip_f2: bad argument (in and out must differ)");
  const int64_t n = (int64_t)N * N * planes;
  if (n == 0) return SP_OK;
  flip_kernel<<<grid_of(n), 256, 0, as_stream(stream)>>>((const float2*)in, (float2*)out, N, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_gaussian(void* out, int N, float sx, float sy, int complex_out, sp_stream_t stream) {
  SP_CHECK(out && N > 0, SP_ERR_INVALID, "sp_gaussian: bad argument");
  gaussian_kernel<<<grid_of((int64_t)N * N), 256, 0, as_stream(stream)>>>(out, N, sx, sy, complex_out);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_richardson_lucy(void* u, const void* p_hat, const void* ph_hat, const void* d, void* work,
                       int N, int frames, int iterations, sp_stream_t stream) {
  SP_N_CHECK(N, "sp_richardson_lucy");
  SP_CHECK(u && p_hat && ph_hat && d && work && frames >= 0 && iterations >= 0, SP_ERR_INVALID,
           "sp_richardson_lucy: bad argument");
  if (frames == 0) return SP_OK;
  cudaStream_t st = as_stream(stream);
  const int64_t plane = (int64_t)N * N, n = plane * frames;
  float2* U = static_cast<float2*>(u);
  float2* B = static_cast<float2*>(work);
  const float2* P = static_cast<const float2*>(p_hat);
  const float2* PH = static_cast<const float2*>(ph_hat);
  const float2* D = static_cast<const float2*>(d);
  const int g = grid_of(n);
  for (int it = 0; it < iterations; ++it) {
    // blur = IFFT(FFT(u) p_hat)
    SP_CUDA_TRY(fft2_dispatch(U, B, N, frames, 0, st));
    multiply_kernel<<<g, 256, 0, st>>>(B, P, B, n);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(fft2_dispatch(B, B, N, frames, 1, st));
    // blur = d / blur
    divide_kernel<<<g, 256, 0, st>>>(D, B, B, n, plane, 1);
    SP_CUDA_TRY(cudaGetLastError());
    // blur = IFFT(FFT(blur) ph_hat); u *= blur
    SP_CUDA_TRY(fft2_dispatch(B, B, N, frames, 0, st));
    multiply_kernel<<<g, 256, 0, st>>>(B, PH, B, n);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(fft2_dispatch(B, B, N, frames, 1, st));
    multiply_kernel<<<g, 256, 0, st>>>(U, B, U, n);
    SP_CUDA_TRY(cudaGetLastError());
  }
  return SP_OK;
}

int sp_coherence_misfit(const void* ac, const float* modulus, float sx, float sy, int N, void* work,
                        double* sum, sp_stream_t stream) {
  SP_N_CHECK(N, "sp_coherence_misfit");
  SP_CHECK(ac && modulus && work && sum, SP_ERR_INVALID, "sp_coherence_misfit: null pointer");
  cudaStream_t st = as_stream(stream);
  const int64_t plane = (int64_t)N * N;
  damp_kernel<<<grid_of(plane), 256, 0, st>>>((const float2*)ac, (float2*)work, N, sx, sy);
  SP_CUDA_TRY(cudaGetLastError());
  SP_CUDA_TRY(fft2_dispatch((const float2*)work, (float2*)work, N, 1, 0, st));
  SP_CUDA_TRY(cudaMemsetAsync(sum, 0, sizeof(double), st));
  speckle_misfit_kernel<<<grid_of(plane), 256, 0, st>>>((const float2*)work, modulus, plane, sum);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

}  // extern "C"
