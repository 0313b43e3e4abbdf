// The plain single-instance GPU path: the reference's GPU dataflow
// (phasing.py:1187-1353 with pyfft replaced by cuFFT), one elementwise kernel
// per step and a stream synchronisation after every launch, as gpu.py:349
// waits after each kernel.  It is the baseline the fused engine is compared
// with, not part of the engine.
#include <cufft.h>

#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "sp_common.cuh"

namespace sp {

__global__ void scale_kernel(float2* x, float s, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = make_float2(x[i].x * s, x[i].y * s);
}

}  // namespace sp

using namespace sp;

#define SP_CUFFT_TRY(expr)                                                  \
  do {                                                                      \
    cufftResult _r = (expr);                                                \
    if (_r != CUFFT_SUCCESS) {                                              \
      ::sp::set_error("%s failed: cufft status %d", #expr, (int)_r);        \
      return SP_ERR_CUDA;                                                   \
    }                                                                       \
  } while (0)

#define SP_PLAIN_SYNC(st)                                                   \
  do {                                                                      \
    cudaError_t _e = cudaGetLastError();                                    \
    if (_e == cudaSuccess) _e = cudaStreamSynchronize(st);                  \
    if (_e != cudaSuccess) {                                                \
      ::sp::set_error("plain path: %s", cudaGetErrorString(_e));            \
      return SP_ERR_CUDA;                                                   \
    }                                                                       \
  } while (0)

namespace {
// One cuFFT plan per (device, N), made on first use and kept, as the
// reference makes its FFT plan once when the data are loaded
// (phasing.py:1187-1230).  The lock is held for a whole call because the
// plan's stream is set per call.
std::mutex g_plan_mu;
std::map<std::pair<int, int>, cufftHandle> g_plans;

int plan_for(int N, cufftHandle* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    ::sp::set_error("plain path: cudaGetDevice failed");
    return SP_ERR_CUDA;
  }
  auto it = g_plans.find({dev, N});
  if (it != g_plans.end()) {
    *out = it->second;
    return SP_OK;
  }
  cufftHandle plan = 0;
  if (cufftPlan2d(&plan, N, N, CUFFT_C2C) != CUFFT_SUCCESS) {
    ::sp::set_error("cufftPlan2d(%d) failed", N);
    return SP_ERR_CUDA;
  }
  g_plans[{dev, N}] = plan;
  *out = plan;
  return SP_OK;
}
}  // namespace

extern "C" int sp_plain_iterate(int N, int n_iter, int n_runs, const int32_t* run_alg,
                                const int32_t* run_count, float beta, void* psi_dev,
                                const float* modulus_dev, const float* support_dev, void* work_dev,
                                sp_stream_t stream) {
  SP_CHECK(is_pow2(N) && N >= kMinN && N <= kMaxN, SP_ERR_SIZE, "sp_plain_iterate: N=%d", N);
  SP_CHECK(psi_dev && modulus_dev && support_dev && work_dev && run_alg && run_count,
           SP_ERR_INVALID, "sp_plain_iterate: null pointer");
  SP_CHECK(n_runs >= 1 && n_runs <= SP_MAX_RUNS && n_iter >= 0, SP_ERR_INVALID,
           "sp_plain_iterate: bad order");
  std::vector<int> order;
  for (int r = 0; r < n_runs; ++r) {
    SP_CHECK(run_alg[r] >= SP_HIO && run_alg[r] <= SP_SF_CPU && run_count[r] >= 0, SP_ERR_INVALID,
             "sp_plain_iterate: bad run %d", r);
    for (int k = 0; k < run_count[r]; ++k) order.push_back(run_alg[r]);
  }
  SP_CHECK(!order.empty(), SP_ERR_INVALID, "sp_plain_iterate: empty order");
  cudaStream_t st = as_stream(stream);
  const int64_t n = (int64_t)N * N;
  float2* psi_in = static_cast<float2*>(psi_dev);
  float2* psi_out = static_cast<float2*>(work_dev);
  float2* fourier = psi_out + n;
  float2* div = fourier + n;
  float2* tmp = div + n;  // DM modified estimate / second projection
  std::lock_guard<std::mutex> lock(g_plan_mu);
  cufftHandle plan = 0;
  if (int rc = plan_for(N, &plan); rc != SP_OK) return rc;
  SP_CUFFT_TRY(cufftSetStream(plan, st));
  const float inv = 1.0f / ((float)N * (float)N);
  auto project = [&](float2* in, float2* out) -> int {
    SP_CUFFT_TRY(cufftExecC2C(plan, (cufftComplex*)in, (cufftComplex*)fourier, CUFFT_FORWARD));
    SP_PLAIN_SYNC(st);
    if (sp_abs_f2_f2(fourier, div, n, stream) != SP_OK) return SP_ERR_CUDA;
    SP_PLAIN_SYNC(st);
    if (sp_fourier(fourier, div, modulus_dev, fourier, n, stream) != SP_OK) return SP_ERR_CUDA;
    SP_PLAIN_SYNC(st);
    SP_CUFFT_TRY(cufftExecC2C(plan, (cufftComplex*)fourier, (cufftComplex*)out, CUFFT_INVERSE));
    SP_PLAIN_SYNC(st);
    scale_kernel<<<256, 256, 0, st>>>(out, inv, n);
    SP_PLAIN_SYNC(st);
    return SP_OK;
  };
  for (int it = 0; it < n_iter; ++it) {
    const int alg = order[it % order.size()];
    int rc = project(psi_in, psi_out);
    if (rc != SP_OK) return rc;
    switch (alg) {
      case SP_HIO: rc = sp_hio(beta, support_dev, psi_in, psi_out, psi_in, n, stream); break;
      case SP_ER: rc = sp_er(support_dev, psi_out, psi_in, n, stream); break;
      case SP_RAAR: rc = sp_raar(beta, support_dev, psi_in, psi_out, psi_in, n, stream); break;
      case SP_SF: rc = sp_sf(support_dev, psi_in, psi_out, psi_in, n, stream); break;
      case SP_DM: {
        const float gm = 1.0f / beta, gs = -gm;
        rc = sp_dm1(gm, support_dev, psi_in, tmp, n, stream);
        if (rc != SP_OK) break;
        SP_PLAIN_SYNC(st);
        rc = project(tmp, tmp);
        if (rc != SP_OK) return rc;
        rc = sp_dm2(beta, gs, support_dev, psi_in, psi_out, tmp, psi_in, n, stream);
        break;
      }
      default:
        rc = SP_ERR_UNSUPPORTED;
        set_error("sp_plain_iterate: algorithm %d has no plain kernel", alg);
        break;
    }
    if (rc != SP_OK) return rc;
    SP_PLAIN_SYNC(st);
  }
  return SP_OK;
}
