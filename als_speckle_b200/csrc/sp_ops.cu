// Operator API (one entry per reference OpenCL kernel), the standalone 2-D
// FFT entry point, and the post-processing kernels of the phasing path:
// global-phase alignment, PRTF, shrinkwrap blur/threshold, averaging and the
// cross-correlation peak used by integer frame alignment.
#include <cmath>
#include <cstring>
#include <vector>

#include "sp_common.cuh"
#include "sp_fft2.cuh"

namespace sp {

static int n_sms_cached() {
  static int sms[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (sms[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    sms[dev] = v;
  }
  return sms[dev];
}

static inline int grid_for(int64_t n, int threads = 256) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)n_sms_cached() * 16;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

cudaError_t fft2_dispatch(const float2* in, float2* out, int N, int batch, int inverse,
                          cudaStream_t st) {
  const float2* tw = nullptr;
  cudaError_t e = twiddles(&tw);
  if (e != cudaSuccess) return e;
  const int sms = n_sms_cached();
  switch (N) {
    case 8: return fft2_n8(in, out, batch, inverse, st, tw, sms);
    case 16: return fft2_n16(in, out, batch, inverse, st, tw, sms);
    case 32: return fft2_n32(in, out, batch, inverse, st, tw, sms);
    case 64: return fft2_n64(in, out, batch, inverse, st, tw, sms);
    case 128: return fft2_n128(in, out, batch, inverse, st, tw, sms);
    case 256: return fft2_n256(in, out, batch, inverse, st, tw, sms);
    case 512: return fft2_n512(in, out, batch, inverse, st, tw, sms);
    case 1024: return fft2_n1024(in, out, batch, inverse, st, tw, sms);
    case 2048: return fft2_n2048(in, out, batch, inverse, st, tw, sms);
    case 4096: return fft2_n4096(in, out, batch, inverse, st, tw, sms);
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------
// elementwise operators (kernels/phasing_*.cl, common_abs_f2_f2.cl)
// ---------------------------------------------------------------------------
__global__ void hio_kernel(float b, const float* __restrict__ sup, const float2* pi_,
                           const float2* po_, float2* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sup[i];
    const float2 po = po_[i], pi = pi_[i];
    out[i] = make_float2((1 - s) * (pi.x - b * po.x) + s * po.x, (1 - s) * (pi.y - b * po.y) + s * po.y);
  }
}
__global__ void er_kernel(const float* __restrict__ sup, const float2* po_, float2* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sup[i];
    const float2 po = po_[i];
    out[i] = make_float2(s * po.x, s * po.y);
  }
}
__global__ void raar_kernel(float b, const float* __restrict__ sup, const float2* pi_,
                            const float2* po_, float2* out, int64_t n) {
  const float b2 = 1 - 2 * b;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sup[i];
    const float2 po = po_[i], pi = pi_[i];
    out[i] = make_float2((1 - s) * (b * pi.x + b2 * po.x) + s * po.x,
                         (1 - s) * (b * pi.y + b2 * po.y) + s * po.y);
  }
}
__global__ void sf_kernel(const float* __restrict__ sup, const float2* pi_, const float2* po_,
                          float2* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sup[i];
    const float2 po = po_[i];
    (void)pi_;
    out[i] = make_float2((1 - s) * (-1 * po.x) + s * po.x, (1 - s) * (-1 * po.y) + s * po.y);
  }
}
__global__ void dm1_kernel(float g, const float* __restrict__ sup, const float2* pi_, float2* out,
                           int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sup[i];
    const float2 pi = pi_[i];
    out[i] = make_float2(-1 * g * (1 - s) * pi.x + s * pi.x, -1 * g * (1 - s) * pi.y + s * pi.y);
  }
}
__global__ void dm2_kernel(float b, float g, const float* __restrict__ sup, const float2* pi_,
                           const float2* po_, const float2* dm_, float2* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sup[i];
    const float2 pi = pi_[i], po = po_[i], dm = dm_[i];
    const float t1r = 2 * po.x - b * dm.x + b * ((1 + g) * po.x - g * pi.x);
    const float t1i = 2 * po.y - b * dm.y + b * ((1 + g) * po.y - g * pi.y);
    const float t2r = pi.x - b * po.x;
    const float t2i = pi.y - b * po.y;
    out[i] = make_float2(s * t1r + (1 - s) * t2r, s * t1i + (1 - s) * t2i);
  }
}
__global__ void fourier_kernel(const float2* psi, const float2* div, const float* __restrict__ mod,
                               float2* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 p = psi[i];
    const float s = mod[i] / div[i].x;
    out[i] = make_float2(p.x * s, p.y * s);
  }
}
__global__ void abs_f2_f2_kernel(const float2* in, float2* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 a = in[i];
    out[i] = make_float2(sqrtf(a.x * a.x + a.y * a.y), 0.f);
  }
}
__global__ void copy_to_buffer_kernel(float2* dst, const float2* src, int c0, int r0, int frame,
                                      int N, int cols, int rows) {
  const int64_t total = (int64_t)rows * cols;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(k / cols), i = (int)(k - (int64_t)j * cols);
    dst[(int64_t)frame * total + k] = src[(int64_t)(j + r0) * N + (i + c0)];
  }
}
// phasing_prtf_accumulate2.cl:16-25: |sum_n F_n/|F_n|| / frames
__global__ void prtf_accumulate_kernel(int frames, const float2* __restrict__ fft,
                                       float* __restrict__ prtf, int N, int shift) {
  const int64_t NN = (int64_t)N * N;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < NN;
       k += (int64_t)gridDim.x * blockDim.x) {
    float cr = 0.f, ci = 0.f;
    for (int n = 0; n < frames; ++n) {
      const float2 v = fft[k + n * NN];
      const float h = hypotf(v.x, v.y);
      if (h > 0.f) {
        cr += v.x / h;
        ci += v.y / h;
      }
    }
    cr /= frames;
    ci /= frames;
    int64_t dst = k;
    if (shift) {  // np.fft.fftshift for even N
      const int r = (int)(k / N), c = (int)(k - (int64_t)r * N);
      dst = (int64_t)((r + N / 2) % N) * N + (c + N / 2) % N;
    }
    prtf[dst] = hypotf(cr, ci);
  }
}

// sum_n F_n/|F_n| in FP32 (phasing_prtf_accumulate2.cl:20-23), added to acc
__global__ void phasor_sum_kernel(int frames, const float2* __restrict__ fft, float2* __restrict__ acc,
                                  int N) {
  const int64_t NN = (int64_t)N * N;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < NN;
       k += (int64_t)gridDim.x * blockDim.x) {
    float cr = 0.f, ci = 0.f;
    for (int n = 0; n < frames; ++n) {
      const float2 v = fft[k + n * NN];
      const float h = hypotf(v.x, v.y);
      if (h > 0.f) {
        cr += v.x / h;
        ci += v.y / h;
      }
    }
    acc[k] = make_float2(acc[k].x + cr, acc[k].y + ci);
  }
}
// prtf = fftshift(|acc| / frames)
__global__ void prtf_finish_kernel(const float2* __restrict__ acc, int frames, float* __restrict__ prtf,
                                   int N) {
  const int64_t NN = (int64_t)N * N;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < NN;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / N), c = (int)(k - (int64_t)r * N);
    const float2 a = acc[k];
    prtf[(int64_t)((r + N / 2) % N) * N + (c + N / 2) % N] = hypotf(a.x / frames, a.y / frames);
  }
}

// embed (n, rows, cols) frames at the corner of zeroed N x N planes
__global__ void embed_kernel(const float2* __restrict__ src, float2* __restrict__ dst, int n,
                             int rows, int cols, int N) {
  const int64_t total = (int64_t)n * N * N;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = k / ((int64_t)N * N);
    const int64_t rem = k - f * N * N;
    const int r = (int)(rem / N), c = (int)(rem - (int64_t)r * N);
    dst[k] = (r < rows && c < cols) ? src[(f * rows + r) * cols + c] : make_float2(0.f, 0.f);
  }
}

// ---------------------------------------------------------------------------
// global phase: five FP64 sums per frame, then rotate (phasing.py:1355-1404)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void phase_sums_kernel(const float2* __restrict__ frames, int64_t elems,
                                  double* __restrict__ sums) {
  // grid: (blocks per frame, frames)
  const int f = blockIdx.y;
  const float2* fr = frames + (int64_t)f * elems;
  double a = 0, b = 0, c = 0, d = 0, e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < elems;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double re = fr[i].x, im = fr[i].y;
    a = fma(re, re, a);
    b = fma(re, im, b);
    c = fma(im, im, c);
    d += re;
    e += im;
  }
  __shared__ double red[5][8];
  a = warp_sum(a); b = warp_sum(b); c = warp_sum(c); d = warp_sum(d); e = warp_sum(e);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = a; red[1][w] = b; red[2][w] = c; red[3][w] = d; red[4][w] = e;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[threadIdx.x][k];
    atomicAdd(&sums[5 * f + threadIdx.x], s);
  }
}

__global__ void phase_rotate_kernel(float2* frames, int64_t elems, const double* __restrict__ sums,
                                    double* angles) {
  const int f = blockIdx.y;
  const double A = sums[5 * f], B = sums[5 * f + 1], C = sums[5 * f + 2];
  const double D = sums[5 * f + 3], F = sums[5 * f + 4];
  // argmin_p A sin^2 p + 2B sin p cos p + C cos^2 p ; sign rule picks p or p + pi
  double p = 0.5 * atan2(-2.0 * B, A - C);
  if (cos(p) * D - sin(p) * F < 0.0) p += 3.14159265358979323846;
  if (p < 0.0) p += 2.0 * 3.14159265358979323846;
  if (angles && blockIdx.x == 0 && threadIdx.x == 0) angles[f] = p;
  const float cp = (float)cos(p), sp = (float)sin(p);
  float2* fr = frames + (int64_t)f * elems;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < elems;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 v = fr[i];
    fr[i] = make_float2(v.x * cp - v.y * sp, v.x * sp + v.y * cp);
  }
}

// ---------------------------------------------------------------------------
// averaging
// ---------------------------------------------------------------------------
__global__ void mean_frames_kernel(const float2* __restrict__ frames, int n, int64_t elems,
                                   float2* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < elems;
       i += (int64_t)gridDim.x * blockDim.x) {
    double re = 0, im = 0;
    for (int f = 0; f < n; ++f) {
      const float2 v = frames[(int64_t)f * elems + i];
      re += v.x;
      im += v.y;
    }
    out[i] = make_float2((float)(re / n), (float)(im / n));
  }
}

// ---------------------------------------------------------------------------
// shrinkwrap: separable circular Gaussian blur of |avg| in FP64
// (phasing.py:1786-1790: ifft2(fft2(fftshift(g)/sum g) * fft2(|avg|)).real is a
// circular convolution with the separable kernel k_r (x) k_c), then thresholds
// ---------------------------------------------------------------------------
__global__ void blur_rows_kernel(const float2* __restrict__ avg, const double* __restrict__ kc,
                                 double* __restrict__ tmp, int rows, int cols) {
  const int64_t total = (int64_t)rows * cols;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / cols), c = (int)(k - (int64_t)r * cols);
    double s = 0;
    for (int j = 0; j < cols; ++j) {
      int cc = c - j;
      if (cc < 0) cc += cols;
      const float2 v = avg[(int64_t)r * cols + cc];
      s = fma(kc[j], (double)sqrtf(v.x * v.x + v.y * v.y), s);
    }
    tmp[k] = s;
  }
}
__global__ void blur_cols_kernel(const double* __restrict__ tmp, const double* __restrict__ kr,
                                 double* __restrict__ blurred, int rows, int cols) {
  const int64_t total = (int64_t)rows * cols;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / cols), c = (int)(k - (int64_t)r * cols);
    double s = 0;
    for (int i = 0; i < rows; ++i) {
      int rr = r - i;
      if (rr < 0) rr += rows;
      s = fma(kr[i], tmp[(int64_t)rr * cols + c], s);
    }
    blurred[k] = s;
  }
}
// per-label maxima of blurred and sums of |avg| (label 0 = global max), as
// order-preserving 64-bit keys for atomicMax
__device__ __forceinline__ unsigned long long dkey(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
  const unsigned long long u = (k & 0x8000000000000000ull) ? (k & ~0x8000000000000000ull) : ~k;
  return __longlong_as_double((long long)u);
}
__global__ void label_stats_kernel(const double* __restrict__ blurred, const float2* __restrict__ avg,
                                   const int* __restrict__ labels, int64_t total,
                                   unsigned long long* __restrict__ maxkey, double* __restrict__ sums) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const double b = blurred[k];
    atomicMax(&maxkey[0], dkey(b));
    const int l = labels ? labels[k] : 0;
    if (l > 0) {
      atomicMax(&maxkey[l], dkey(b));
      const float2 v = avg[k];
      atomicAdd(&sums[l], (double)sqrtf(v.x * v.x + v.y * v.y));
    }
  }
}
// refined = sum over parts of (b*part > max(b*part)*lt) times (b > max(b)*gt)
__global__ void threshold_kernel(const double* __restrict__ blurred, const int* __restrict__ labels,
                                 int64_t total, const unsigned long long* __restrict__ maxkey,
                                 double local_t, double global_t, int kill_label,
                                 float* __restrict__ refined) {
  const double gmax = dkey_inv(maxkey[0]);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const double b = blurred[k];
    const int l = labels[k];
    float r = 0.f;
    if (l > 0 && l != kill_label) {
      // current.max() over the whole array includes the zeros outside the part
      const double pmax = fmax(dkey_inv(maxkey[l]), 0.0);
      r = (b > pmax * local_t) ? 1.f : 0.f;
    }
    if (!(b > gmax * global_t)) r = 0.f;
    refined[k] = r;
  }
}

// ---------------------------------------------------------------------------
// cross-correlation peak: argmax over the fftshifted |cc| (crosscorr.py:556)
// keyed so that ties go to the first index in shifted order, as numpy's argmax
// ---------------------------------------------------------------------------
__global__ void xcorr_mul_kernel(const float2* __restrict__ fa, const float2* __restrict__ fb,
                                 float2* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 a = fa[i], b = fb[i];
    out[i] = make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);  // a * conj(b)
  }
}
__global__ void argmax_shifted_kernel(const float2* __restrict__ cc, int N,
                                      unsigned long long* __restrict__ best) {
  const int64_t NN = (int64_t)N * N;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < NN;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / N), c = (int)(k - (int64_t)r * N);
    const int sr = (r + N / 2) % N, sc = (c + N / 2) % N;  // position after fftshift
    const uint32_t sidx = (uint32_t)(sr * N + sc);
    const float2 v = cc[k];
    const float m = sqrtf(v.x * v.x + v.y * v.y);
    const unsigned long long key = ((unsigned long long)__float_as_uint(m) << 32) | (0xffffffffu - sidx);
    atomicMax(best, key);
  }
}
__global__ void abs_to_complex_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                      int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 a = in[i];
    out[i] = make_float2(sqrtf(a.x * a.x + a.y * a.y), 0.f);
  }
}
__global__ void roll_kernel(const float2* __restrict__ in, float2* __restrict__ out, int rows,
                            int cols, int dr, int dc) {
  const int64_t total = (int64_t)rows * cols;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / cols), c = (int)(k - (int64_t)r * cols);
    int sr = (r - dr) % rows, sc = (c - dc) % cols;
    if (sr < 0) sr += rows;
    if (sc < 0) sc += cols;
    out[k] = in[(int64_t)sr * cols + sc];
  }
}
// centre-of-mass sums of |img| per frame (phasing.py:1731-1735)
__global__ void com_sums_kernel(const float2* __restrict__ frames, int rows, int cols,
                                double* __restrict__ sums) {
  const int f = blockIdx.y;
  const int64_t total = (int64_t)rows * cols;
  const float2* fr = frames + (int64_t)f * total;
  double s = 0, sr = 0, sc = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / cols), c = (int)(k - (int64_t)r * cols);
    const double a = (double)sqrtf(fr[k].x * fr[k].x + fr[k].y * fr[k].y);
    s += a;
    sr = fma((double)r, a, sr);
    sc = fma((double)c, a, sc);
  }
  s = warp_sum(s); sr = warp_sum(sr); sc = warp_sum(sc);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sums[3 * f], s);
    atomicAdd(&sums[3 * f + 1], sr);
    atomicAdd(&sums[3 * f + 2], sc);
  }
}
__global__ void roll_accumulate_kernel(const float2* __restrict__ frames, int n, int rows, int cols,
                                       const int* __restrict__ shifts, float2* __restrict__ out) {
  const int64_t total = (int64_t)rows * cols;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / cols), c = (int)(k - (int64_t)r * cols);
    float re = 0.f, im = 0.f;
    for (int f = 0; f < n; ++f) {
      // roll by (-dr, -dc): out[r][c] = in[(r + dr) % rows][(c + dc) % cols]
      int sr = (r + shifts[2 * f]) % rows, sc = (c + shifts[2 * f + 1]) % cols;
      if (sr < 0) sr += rows;
      if (sc < 0) sc += cols;
      const float2 v = frames[(int64_t)f * total + (int64_t)sr * cols + sc];
      re += v.x;
      im += v.y;
    }
    out[k] = make_float2(re, im);
  }
}

}  // namespace sp

using namespace sp;

#define SP_ELEMENTWISE_CHECK(n, ...)                                         \
  SP_CHECK((n) >= 0, SP_ERR_INVALID, "negative element count");              \
  if ((n) == 0) return SP_OK;

extern "C" {

int sp_hio(float beta, const float* support, const void* psi_in, const void* psi_out, void* output,
           int64_t n, sp_stream_t stream) {
  SP_ELEMENTWISE_CHECK(n);
  SP_CHECK(support && psi_in && psi_out && output, SP_ERR_INVALID, "sp_hio: null pointer");
  hio_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(beta, support, (const float2*)psi_in,
                                                         (const float2*)psi_out, (float2*)output, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_er(const float* support, const void* psi_out, void* output, int64_t n, sp_stream_t stream) {
  SP_ELEMENTWISE_CHECK(n);
  SP_CHECK(support && psi_out && output, SP_ERR_INVALID, "sp_er: null pointer");
  er_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(support, (const float2*)psi_out,
                                                        (float2*)output, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_raar(float beta, const float* support, const void* psi_in, const void* psi_out, void* output,
            int64_t n, sp_stream_t stream) {
  SP_ELEMENTWISE_CHECK(n);
  SP_CHECK(support && psi_in && psi_out && output, SP_ERR_INVALID, "sp_raar: null pointer");
  raar_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(beta, support, (const float2*)psi_in,
                                                          (const float2*)psi_out, (float2*)output, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_sf(const float* support, const void* psi_in, const void* psi_out, void* output, int64_t n,
          sp_stream_t stream) {
  SP_ELEMENTWISE_CHECK(n);
  SP_CHECK(support && psi_out && output, SP_ERR_INVALID, "sp_sf: null pointer");
  sf_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(support, (const float2*)psi_in,
                                                        (const float2*)psi_out, (float2*)output, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_dm1(float gamma_m, const float* support, const void* psi_in, void* output, int64_t n,
           sp_stream_t stream) {
  SP_ELEMENTWISE_CHECK(n);
  SP_CHECK(support && psi_in && output, SP_ERR_INVALID, "sp_dm1: null pointer");
  dm1_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(gamma_m, support, (const float2*)psi_in,
                                                         (float2*)output, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_dm2(float beta, float gamma_s, const float* support, const void* psi_in, const void* psi_out,
           const void* dm_tmp, void* output, int64_t n, sp_stream_t stream) {
  SP_ELEMENTWISE_CHECK(n);
  SP_CHECK(support && psi_in && psi_out && dm_tmp && output, SP_ERR_INVALID, "sp_dm2: null pointer");
  dm2_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(beta, gamma_s, support, (const float2*)psi_in,
                                                         (const float2*)psi_out, (const float2*)dm_tmp,
                                                         (float2*)output, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_fourier(const void* psi, const void* div, const float* modulus, void* out, int64_t n,
               sp_stream_t stream) {
  SP_ELEMENTWISE_CHECK(n);
  SP_CHECK(psi && div && modulus && out, SP_ERR_INVALID, "sp_fourier: null pointer");
  fourier_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>((const float2*)psi, (const float2*)div,
                                                             modulus, (float2*)out, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_abs_f2_f2(const void* in, void* out, int64_t n, sp_stream_t stream) {
  SP_ELEMENTWISE_CHECK(n);
  SP_CHECK(in && out, SP_ERR_INVALID, "sp_abs_f2_f2: null pointer");
  abs_f2_f2_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>((const float2*)in, (float2*)out, n);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_copy_to_buffer_f2(void* dst, const void* src, int c0, int r0, int frame, int N, int cols,
                         int rows, sp_stream_t stream) {
  SP_CHECK(dst && src, SP_ERR_INVALID, "sp_copy_to_buffer_f2: null pointer");
  SP_CHECK(rows > 0 && cols > 0 && r0 >= 0 && c0 >= 0 && r0 + rows <= N && c0 + cols <= N &&
               frame >= 0,
           SP_ERR_INVALID, "sp_copy_to_buffer_f2: box outside the array");
  copy_to_buffer_kernel<<<grid_for((int64_t)rows * cols), 256, 0, as_stream(stream)>>>(
      (float2*)dst, (const float2*)src, c0, r0, frame, N, cols, rows);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}
int sp_prtf_accumulate(int frames, const void* fft, float* prtf, int N, sp_stream_t stream) {
  SP_CHECK(fft && prtf && frames > 0 && N > 0, SP_ERR_INVALID, "sp_prtf_accumulate: bad argument");
  prtf_accumulate_kernel<<<grid_for((int64_t)N * N), 256, 0, as_stream(stream)>>>(
      frames, (const float2*)fft, prtf, N, 0);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_fft2(const void* in, void* out, int N, int batch, int inverse, sp_stream_t stream) {
  SP_CHECK(in && out, SP_ERR_INVALID, "sp_fft2: null pointer");
  SP_CHECK(is_pow2(N) && N >= kMinN && N <= kMaxN, SP_ERR_SIZE,
           "sp_fft2: N=%d must be a power of two in [%d, %d]", N, kMinN, kMaxN);
  SP_CHECK(batch >= 0, SP_ERR_INVALID, "sp_fft2: batch < 0");
  if (batch == 0) return SP_OK;
  SP_CUDA_TRY(fft2_dispatch((const float2*)in, (float2*)out, N, batch, inverse, as_stream(stream)));
  return SP_OK;
}

int sp_align_global_phase(void* frames, int n_frames, int64_t frame_elems, double* angles,
                          double* sums, sp_stream_t stream) {
  SP_CHECK(frames && sums && n_frames >= 0 && frame_elems > 0, SP_ERR_INVALID,
           "sp_align_global_phase: bad argument");
  SP_CHECK(n_frames <= 65535, SP_ERR_SIZE, "sp_align_global_phase: at most 65535 frames");
  if (n_frames == 0) return SP_OK;
  cudaStream_t st = as_stream(stream);
  SP_CUDA_TRY(cudaMemsetAsync(sums, 0, sizeof(double) * 5 * n_frames, st));
  int bx = (int)((frame_elems + 255) / 256);
  if (bx > 64) bx = 64;
  phase_sums_kernel<<<dim3(bx, n_frames), 256, 0, st>>>((const float2*)frames, frame_elems, sums);
  phase_rotate_kernel<<<dim3(bx, n_frames), 256, 0, st>>>((float2*)frames, frame_elems, sums, angles);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_prtf(const void* frames, int n_frames, int rows, int cols, int N, void* work, float* prtf,
            sp_stream_t stream) {
  SP_CHECK(frames && work && prtf && n_frames > 0, SP_ERR_INVALID, "sp_prtf: bad argument");
  SP_CHECK(is_pow2(N) && N >= kMinN && N <= kMaxN, SP_ERR_SIZE, "sp_prtf: N=%d unsupported", N);
  SP_CHECK(rows > 0 && cols > 0 && rows <= N && cols <= N, SP_ERR_INVALID,
           "sp_prtf: frames larger than N");
  cudaStream_t st = as_stream(stream);
  const int64_t total = (int64_t)n_frames * N * N;
  embed_kernel<<<grid_for(total), 256, 0, st>>>((const float2*)frames, (float2*)work, n_frames, rows,
                                                cols, N);
  SP_CUDA_TRY(cudaGetLastError());
  SP_CUDA_TRY(fft2_dispatch((const float2*)work, (float2*)work, N, n_frames, 0, st));
  prtf_accumulate_kernel<<<grid_for((int64_t)N * N), 256, 0, st>>>(n_frames, (const float2*)work,
                                                                   prtf, N, 1);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_prtf_phasors(const void* frames, int n_frames, int rows, int cols, int N, void* work,
                    void* acc, sp_stream_t stream) {
  SP_CHECK(frames && work && acc && n_frames > 0, SP_ERR_INVALID, "sp_prtf_phasors: bad argument");
  SP_CHECK(is_pow2(N) && N >= kMinN && N <= kMaxN, SP_ERR_SIZE, "sp_prtf_phasors: N=%d unsupported", N);
  SP_CHECK(rows > 0 && cols > 0 && rows <= N && cols <= N, SP_ERR_INVALID,
           "sp_prtf_phasors: frames larger than N");
  cudaStream_t st = as_stream(stream);
  const int64_t total = (int64_t)n_frames * N * N;
  embed_kernel<<<grid_for(total), 256, 0, st>>>((const float2*)frames, (float2*)work, n_frames, rows,
                                                cols, N);
  SP_CUDA_TRY(cudaGetLastError());
  SP_CUDA_TRY(fft2_dispatch((const float2*)work, (float2*)work, N, n_frames, 0, st));
  phasor_sum_kernel<<<grid_for((int64_t)N * N), 256, 0, st>>>(n_frames, (const float2*)work,
                                                              (float2*)acc, N);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_prtf_finish(const void* acc, int n_frames, int N, float* prtf, sp_stream_t stream) {
  SP_CHECK(acc && prtf && n_frames > 0, SP_ERR_INVALID, "sp_prtf_finish: bad argument");
  SP_CHECK(is_pow2(N) && N >= kMinN && N <= kMaxN, SP_ERR_SIZE, "sp_prtf_finish: N=%d unsupported", N);
  prtf_finish_kernel<<<grid_for((int64_t)N * N), 256, 0, as_stream(stream)>>>((const float2*)acc,
                                                                             n_frames, prtf, N);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_mean_frames(const void* frames, int n_frames, int64_t frame_elems, void* out,
                   sp_stream_t stream) {
  SP_CHECK(frames && out && n_frames > 0 && frame_elems > 0, SP_ERR_INVALID,
           "sp_mean_frames: bad argument");
  mean_frames_kernel<<<grid_for(frame_elems), 256, 0, as_stream(stream)>>>(
      (const float2*)frames, n_frames, frame_elems, (float2*)out);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_shrinkwrap(const void* avg, int rows, int cols, const double* kr, const double* kc,
                  const int* labels, int n_labels, double local_t, double global_t, int kill_weakest,
                  void* work, double* blurred, float* refined, double* part_sums,
                  sp_stream_t stream) {
  SP_CHECK(avg && kr && kc && labels && work && blurred && refined && part_sums, SP_ERR_INVALID,
           "sp_shrinkwrap: null pointer");
  SP_CHECK(rows > 0 && cols > 0 && n_labels >= 0, SP_ERR_INVALID, "sp_shrinkwrap: bad size");
  cudaStream_t st = as_stream(stream);
  const int64_t total = (int64_t)rows * cols;
  double* tmp = static_cast<double*>(work);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(tmp + total);
  blur_rows_kernel<<<grid_for(total), 256, 0, st>>>((const float2*)avg, kc, tmp, rows, cols);
  blur_cols_kernel<<<grid_for(total), 256, 0, st>>>(tmp, kr, blurred, rows, cols);
  // keys start at the smallest order-preserving key (0 encodes -NaN, below all)
  SP_CUDA_TRY(cudaMemsetAsync(keys, 0, sizeof(unsigned long long) * (n_labels + 1), st));
  SP_CUDA_TRY(cudaMemsetAsync(part_sums, 0, sizeof(double) * (n_labels + 1), st));
  label_stats_kernel<<<grid_for(total), 256, 0, st>>>(blurred, (const float2*)avg, labels, total,
                                                      keys, part_sums);
  SP_CUDA_TRY(cudaGetLastError());
  int kill = -1;
  if (kill_weakest && n_labels > 0) {
    // the weakest part is chosen on the host from part_sums (phasing.py:1811-1813)
    std::vector<double> h(n_labels + 1);
    SP_CUDA_TRY(cudaMemcpyAsync(h.data(), part_sums, sizeof(double) * (n_labels + 1),
                                cudaMemcpyDeviceToHost, st));
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    kill = 1;
    for (int l = 2; l <= n_labels; ++l)
      if (h[l] < h[kill]) kill = l;
  }
  threshold_kernel<<<grid_for(total), 256, 0, st>>>(blurred, labels, total, keys, local_t, global_t,
                                                    kill, refined);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_xcorr_peak(const void* a, const void* b, int N, int use_mag_only, void* work,
                  unsigned long long* best, sp_stream_t stream) {
  SP_CHECK(a && b && work && best, SP_ERR_INVALID, "sp_xcorr_peak: null pointer");
  SP_CHECK(is_pow2(N) && N >= kMinN && N <= kMaxN, SP_ERR_SIZE, "sp_xcorr_peak: N=%d", N);
  cudaStream_t st = as_stream(stream);
  const int64_t NN = (int64_t)N * N;
  float2* fa = static_cast<float2*>(work);
  float2* fb = fa + NN;
  if (use_mag_only) {
    abs_to_complex_kernel<<<grid_for(NN), 256, 0, st>>>((const float2*)a, fa, NN);
    abs_to_complex_kernel<<<grid_for(NN), 256, 0, st>>>((const float2*)b, fb, NN);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(fft2_dispatch(fa, fa, N, 1, 0, st));
    SP_CUDA_TRY(fft2_dispatch(fb, fb, N, 1, 0, st));
  } else {
    SP_CUDA_TRY(fft2_dispatch((const float2*)a, fa, N, 1, 0, st));
    SP_CUDA_TRY(fft2_dispatch((const float2*)b, fb, N, 1, 0, st));
  }
  xcorr_mul_kernel<<<grid_for(NN), 256, 0, st>>>(fa, fb, fa, NN);
  SP_CUDA_TRY(cudaGetLastError());
  SP_CUDA_TRY(fft2_dispatch(fa, fa, N, 1, 1, st));
  SP_CUDA_TRY(cudaMemsetAsync(best, 0, sizeof(unsigned long long), st));
  argmax_shifted_kernel<<<grid_for(NN), 256, 0, st>>>(fa, N, best);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_roll(const void* in, void* out, int rows, int cols, int dr, int dc, sp_stream_t stream) {
  SP_CHECK(in && out && in != out && rows > 0 && cols > 0, SP_ERR_INVALID, "sp_roll: bad argument");
  roll_kernel<<<grid_for((int64_t)rows * cols), 256, 0, as_stream(stream)>>>(
      (const float2*)in, (float2*)out, rows, cols, dr, dc);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_com_sums(const void* frames, int n_frames, int rows, int cols, double* sums,
                sp_stream_t stream) {
  SP_CHECK(frames && sums && n_frames > 0 && rows > 0 && cols > 0, SP_ERR_INVALID,
           "sp_com_sums: bad argument");
  SP_CHECK(n_frames <= 65535, SP_ERR_SIZE, "sp_com_sums: at most 65535 frames");
  cudaStream_t st = as_stream(stream);
  SP_CUDA_TRY(cudaMemsetAsync(sums, 0, sizeof(double) * 3 * n_frames, st));
  int bx = (int)(((int64_t)rows * cols + 255) / 256);
  if (bx > 64) bx = 64;
  com_sums_kernel<<<dim3(bx, n_frames), 256, 0, st>>>((const float2*)frames, rows, cols, sums);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

int sp_roll_accumulate(const void* frames, int n_frames, int rows, int cols, const int* shifts,
                       void* out, sp_stream_t stream) {
  SP_CHECK(frames && shifts && out && n_frames > 0 && rows > 0 && cols > 0, SP_ERR_INVALID,
           "sp_roll_accumulate: bad argument");
  roll_accumulate_kernel<<<grid_for((int64_t)rows * cols), 256, 0, as_stream(stream)>>>(
      (const float2*)frames, n_frames, rows, cols, shifts, (float2*)out);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

}  // extern "C"
