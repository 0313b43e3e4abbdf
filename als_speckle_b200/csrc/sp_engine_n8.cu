// Engine kernels and standalone 2-D FFT for N = 8 (see sp_engine_launch.cuh
// and sp_fft2.cuh).
#include "sp_engine_launch.cuh"
#include "sp_fft2.cuh"
namespace sp {
SP_DEFINE_SIZE(8)
SP_DEFINE_FFT2(8)
}  // namespace sp
