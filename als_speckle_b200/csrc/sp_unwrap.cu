// Polar unwrap of an N x N float map with cubic B-spline interpolation, and
// its row mean: the `prtfq` / `rftfq` outputs of the reference
// (speckle/phasing.py:1454-1458, :1512-1516, :1603-1605, :1701-1705), which
// call wrapping.unwrap(array, (0, N/2, (N/2, N/2))) (wrapping.py:8-67,
// :131-176) and average each radius over its angles.
//
// wrapping.unwrap samples the map on a polar grid with
// scipy.ndimage.map_coordinates(order=3, mode='constant').  That is cubic
// B-spline interpolation: the map is first turned into B-spline coefficients
// by the recursive prefilter of Unser, Aldroubi & Eden ("B-spline signal
// processing: Part II", IEEE Trans. Signal Process. 41, 1993) along each
// axis, with the whole-sample mirror boundary f[-k] = f[k],
// f[N-1+k] = f[N-1-k] and its exact causal initialisation (Thevenaz, Blu &
// Unser, "Interpolation revisited", IEEE Trans. Med. Imaging 19, 2000);
// every sample is then sum_ij c[i][j] b3(y - i) b3(x - j) over its 4 x 4
// neighbours, the coefficient index mirrored the same way beyond the edges.
// Both steps run in FP64 here; each sample is rounded to float32 (the map's
// type, which map_coordinates keeps) before the row mean.
#include <cmath>

#include "sp_common.cuh"

namespace sp {

// The cubic B-spline's pole and the prefilter's gain (1 - z)(1 - 1/z) = 6.
constexpr double kZ3 = -0.267949192431122706472553658494127633;  // sqrt(3) - 2
constexpr double kGain3 = 6.0;

// Prefilter one line of n values: in[k * stride] (float map or FP64
// coefficients) -> out[k * stride] (FP64); in may equal out.  The recursions
// carry their running value in a register, so only the loads of the next
// inputs are on the critical path and they can be issued ahead.
template <class T>
__device__ void bspline3_line(const T* in, double* out, int n, long stride) {
  const double z = kZ3;
  if (n == 1) {
    out[0] = (double)in[0];
    return;
  }
  // causal initialisation: sum_j z^j x~[j] over one period (length 2n - 2)
  // of the mirrored line x~, divided by 1 - z^(2n-2):
  //   x[0] + z^(n-1) x[n-1] + sum_{k=1}^{n-2} (z^k + z^(2n-2-k)) x[k]
  // (powers by repeated products, which underflow to 0 harmlessly)
  const double zn1 = pow(z, (double)(n - 1));
  double head = 0.0, tail = 0.0, zk = z;
#pragma unroll 8
  for (int k = 1; k < n - 1; ++k) {
    head += zk * (double)in[k * stride];
    zk *= z;
  }
  zk = z;  // z^(n-1-k) for k = n-2 down to 1
#pragma unroll 8
  for (int k = n - 2; k >= 1; --k) {
    tail += zk * (double)in[k * stride];
    zk *= z;
  }
  const double x0 = (double)in[0], xl = (double)in[(long)(n - 1) * stride];
  // the gain (1 - z)(1 - 1/z) = 6 is applied to the inputs as they are read
  double prev = kGain3 * (x0 + zn1 * xl + head + zn1 * tail) / (1.0 - zn1 * zn1);
  out[0] = prev;
#pragma unroll 8
  for (int k = 1; k < n; ++k) {
    prev = kGain3 * (double)in[k * stride] + z * prev;
    out[k * stride] = prev;
  }
  // anti-causal initialisation for the mirror boundary, then the recursion
  double next = (z / (z * z - 1.0)) * (prev + z * out[(long)(n - 2) * stride]);
  out[(long)(n - 1) * stride] = next;
#pragma unroll 8
  for (int k = n - 2; k >= 0; --k) {
    next = z * (next - out[k * stride]);
    out[k * stride] = next;
  }
}

// Columns first (thread j walks column j: neighbouring threads touch
// neighbouring addresses), from the float map into the FP64 coefficients.
__global__ void spline_cols_kernel(const float* __restrict__ in, double* __restrict__ c, int N) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  bspline3_line(in + j, c + j, N, N);
}

// Then rows, in place.
__global__ void spline_rows_kernel(double* __restrict__ c, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  bspline3_line(c + (size_t)i * N, c + (size_t)i * N, N, 1);
}

__device__ __forceinline__ int mirror_index(int i, int n) {
  if (n == 1) return 0;
  const int p = 2 * n - 2;
  i %= p;
  if (i < 0) i += p;
  return i >= n ? p - i : i;
}

// Cubic B-spline weights of the taps floor(u) - 1 .. floor(u) + 2 for t = u - floor(u).
__device__ __forceinline__ void bspline3_weights(double t, double w[4]) {
  const double s = 1.0 - t;
  w[0] = s * s * s / 6.0;
  w[1] = (3.0 * t * t * t - 6.0 * t * t + 4.0) / 6.0;
  w[2] = (-3.0 * t * t * t + 3.0 * t * t + 3.0 * t + 1.0) / 6.0;
  w[3] = t * t * t / 6.0;
}

__device__ __forceinline__ double bspline3_at(const double* __restrict__ c, int N, double y, double x) {
  const double fy = floor(y), fx = floor(x);
  double wy[4], wx[4];
  bspline3_weights(y - fy, wy);
  bspline3_weights(x - fx, wx);
  const int iy = (int)fy - 1, ix = (int)fx - 1;
  int cols[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) cols[b] = mirror_index(ix + b, N);
  double acc = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const double* row = c + (size_t)mirror_index(iy + a, N) * N;
    double ra = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b) ra += wx[b] * row[cols[b]];
    acc += wy[a] * ra;
  }
  return acc;
}

// One block per radius r_in + blockIdx.x: the samples at the `cols` angles
// phi_k = 2 pi k / cols (wrapping.py:46-51 order of operations), written to
// `unwrapped` (row-major, radius by angle) if given, and their mean to `mean`.
__global__ void unwrap_kernel(const double* __restrict__ c, int N, int r_in, int cols, double cy,
                              double cx, float* __restrict__ unwrapped, float* __restrict__ mean) {
  constexpr double kPi = 3.141592653589793238462643383279502884;
  const int row = blockIdx.x;
  const double r = (double)(r_in + row);
  double part = 0.0;
  for (int k = threadIdx.x; k < cols; k += blockDim.x) {
    const double phi = (double)k * 2.0 * kPi / (double)cols;
    double sn, cs;
    sincos(phi, &sn, &cs);
    const float v = (float)bspline3_at(c, N, r * sn + cy, r * cs + cx);
    if (unwrapped) unwrapped[(size_t)row * cols + k] = v;
    part += (double)v;
  }
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0 && mean) mean[row] = (float)(s / (double)cols);
  }
}

}  // namespace sp

using namespace sp;

extern "C" int sp_unwrap(const float* in_dev, int N, int r_in, int r_out, double cy, double cx,
                         int columns, double* work_dev, float* unwrapped_dev, float* mean_dev,
                         sp_stream_t stream) {
  SP_CHECK(in_dev && work_dev, SP_ERR_INVALID, "sp_unwrap: input and work pointers are required");
  SP_CHECK(unwrapped_dev || mean_dev, SP_ERR_INVALID, "sp_unwrap: no output requested");
  SP_CHECK(N >= 1 && N <= 65536, SP_ERR_SIZE, "sp_unwrap: N=%d", N);
  SP_CHECK(r_in >= 0 && r_out > r_in, SP_ERR_INVALID, "sp_unwrap: radii %d..%d", r_in, r_out);
  if (columns <= 0) columns = (int)(2.0 * 3.141592653589793 * (double)r_out);
  SP_CHECK(columns >= 1, SP_ERR_INVALID, "sp_unwrap: %d columns", columns);
  // every sample must fall inside the map (the prtfq / rftfq grid, centre N/2
  // and radii below N/2, always does); nothing outside is interpolated
  const double rmax = (double)(r_out - 1);
  SP_CHECK(cy - rmax >= 0.0 && cy + rmax <= (double)(N - 1) && cx - rmax >= 0.0 &&
               cx + rmax <= (double)(N - 1),
           SP_ERR_INVALID, "sp_unwrap: radius %d about (%g, %g) leaves the %d x %d map", r_out - 1,
           cy, cx, N, N);
  cudaStream_t st = as_stream(stream);
  const int tb = 128, nb = (N + tb - 1) / tb;
  spline_cols_kernel<<<nb, tb, 0, st>>>(in_dev, work_dev, N);
  SP_CUDA_TRY(cudaGetLastError());
  spline_rows_kernel<<<nb, tb, 0, st>>>(work_dev, N);
  SP_CUDA_TRY(cudaGetLastError());
  unwrap_kernel<<<r_out - r_in, 256, 0, st>>>(work_dev, N, r_in, columns, cy, cx, unwrapped_dev,
                                               mean_dev);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
