// Engine kernels, standalone 2-D FFT and partial-coherence kernels for N = 2048 (see
// sp_engine_launch.cuh, sp_fft2.cuh and sp_coherence.cuh).
#include "sp_engine_launch.cuh"
#include "sp_fft2.cuh"
#include "sp_coherence.cuh"
namespace sp {
SP_DEFINE_SIZE(2048)
SP_DEFINE_FFT2(2048)
SP_DEFINE_PC(2048)
}  // namespace sp
