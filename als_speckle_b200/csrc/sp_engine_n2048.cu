// Engine kernels and standalone 2-D FFT for N = 2048 (see sp_engine_launch.cuh
// and sp_fft2.cuh).
#include "sp_engine_launch.cuh"
#include "sp_fft2.cuh"
namespace sp {
SP_DEFINE_SIZE(2048)
SP_DEFINE_FFT2(2048)
}  // namespace sp
