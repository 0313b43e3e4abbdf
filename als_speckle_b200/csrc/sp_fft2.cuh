// Standalone batched 2-D FFT (sp_fft2) on the same Stockham line transform as
// the engine: a row kernel and a column kernel per size, E = min(16, N)
// values per thread.  Replaces pyfft's Plan.execute (phasing.py:1074-1075).
#pragma once
#include "sp_common.cuh"
#include "sp_engine_kernels.cuh"

namespace sp {

template <int N, int DIR>
__global__ void __launch_bounds__(kThreads) fft_rows_kernel(const float2* in,
                                                            float2* out, int batch,
                                                            const float2* __restrict__ tw_all) {
  constexpr int E = (N < 16 ? N : 16);
  constexpr int T = N / E;
  constexpr int L = lines_per_item(N, E);
  constexpr int SH = pad_shift(E);
  using Sync = typename std::conditional<(T <= 32), WarpSync, BlockSync>::type;
  extern __shared__ float2 smem[];
  float2* tw = smem + item_smem_elems(N, E);
  build_stage_twiddles<N, E>(tw, tw_all + N);
  __syncthreads();
  const int tid = threadIdx.x;
  const int lrow = tid / T;
  const int t = tid - lrow * T;
  const bool active = lrow < L;
  const RowLayout<SH> lay{smem + (active ? lrow : 0) * padk(N, SH)};
  const int items = batch * (N / L);
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const size_t row = (size_t)it * L + (active ? lrow : 0);  // global row over the batch
    const size_t off = row * N + t;
    float2 v[E];
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = in[off + i * T];
    }
    fft_line<N, E, DIR>(v, lay, Sync{}, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) out[off + i * T] = v[i];
    }
  }
}

template <int N, int DIR>
__global__ void __launch_bounds__(kThreads) fft_cols_kernel(const float2* in,
                                                            float2* out, int batch,
                                                            float scale,
                                                            const float2* __restrict__ tw_all) {
  constexpr int E = (N < 16 ? N : 16);
  constexpr int T = N / E;
  constexpr int C = lines_per_item(N, E);
  extern __shared__ float2 smem[];
  float2* tw = smem + item_smem_elems(N, E);
  build_stage_twiddles<N, E>(tw, tw_all + N);
  __syncthreads();
  const int tid = threadIdx.x;
  const int c = tid % C;
  const int t = tid / C;
  const bool active = t < T;
  const ColLayout<pad_shift(E), C> lay{smem + c};
  const int per_plane = N / C;
  const int items = batch * per_plane;
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const int plane = it / per_plane;
    const int col = (it - plane * per_plane) * C + c;
    const size_t off = (size_t)plane * N * N + (size_t)(active ? t : 0) * N + col;
    float2 v[E];
    __syncthreads();
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = in[off + (size_t)i * T * N];
    }
    fft_line<N, E, DIR>(v, lay, BlockSync{}, active, t, tw);
    if (active) {
#pragma unroll
      for (int i = 0; i < E; ++i) out[off + (size_t)i * T * N] = make_float2(v[i].x * scale, v[i].y * scale);
    }
  }
}

template <int N>
cudaError_t fft2_t(const float2* in, float2* out, int batch, int inverse, cudaStream_t st,
                   const float2* tw, int n_sms) {
  constexpr int E = (N < 16 ? N : 16);
  const int sm = (item_smem_elems(N, E) + tw_stage_total(N, E)) * (int)sizeof(float2);
  const int rows_items = batch * (N / lines_per_item(N, E));
  const int grid = rows_items < n_sms * 4 ? rows_items : n_sms * 4;
  const float scale = inverse ? 1.0f / ((float)N * (float)N) : 1.0f;
  cudaError_t e;
  if (inverse) {
    e = cudaFuncSetAttribute(fft_rows_kernel<N, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fft_cols_kernel<N, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    fft_rows_kernel<N, +1><<<grid, kThreads, sm, st>>>(in, out, batch, tw);
    fft_cols_kernel<N, +1><<<grid, kThreads, sm, st>>>(out, out, batch, scale, tw);
  } else {
    e = cudaFuncSetAttribute(fft_rows_kernel<N, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fft_cols_kernel<N, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    fft_rows_kernel<N, -1><<<grid, kThreads, sm, st>>>(in, out, batch, tw);
    fft_cols_kernel<N, -1><<<grid, kThreads, sm, st>>>(out, out, batch, scale, tw);
  }
  return cudaGetLastError();
}

cudaError_t fft2_dispatch(const float2* in, float2* out, int N, int batch, int inverse,
                          cudaStream_t st);

#define SP_DECLARE_FFT2(N) \
  cudaError_t fft2_n##N(const float2* in, float2* out, int batch, int inverse, cudaStream_t st, \
                        const float2* tw, int n_sms);
SP_DECLARE_FFT2(8)
SP_DECLARE_FFT2(16)
SP_DECLARE_FFT2(32)
SP_DECLARE_FFT2(64)
SP_DECLARE_FFT2(128)
SP_DECLARE_FFT2(256)
SP_DECLARE_FFT2(512)
SP_DECLARE_FFT2(1024)
SP_DECLARE_FFT2(2048)
SP_DECLARE_FFT2(4096)

#define SP_DEFINE_FFT2(N)                                                                     \
  cudaError_t fft2_n##N(const float2* in, float2* out, int batch, int inverse, cudaStream_t st, \
                        const float2* tw, int n_sms) {                                        \
    return fft2_t<N>(in, out, batch, inverse, st, tw, n_sms);                                 \
  }

}  // namespace sp
