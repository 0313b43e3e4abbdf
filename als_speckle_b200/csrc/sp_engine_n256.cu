// Engine kernels, standalone 2-D FFT and partial-coherence kernels for N = 256 (see
// sp_engine_launch.cuh, sp_fft2.cuh and sp_coherence.cuh).
#include "sp_engine_launch.cuh"
#include "sp_fft2.cuh"
#include "sp_coherence.cuh"
namespace sp {
SP_DEFINE_SIZE(256)
SP_DEFINE_FFT2(256)
SP_DEFINE_PC(256)
}  // namespace sp
