// Engine kernels, standalone 2-D FFT and partial-coherence kernels for N = 8 (see
// sp_engine_launch.cuh, sp_fft2.cuh and sp_coherence.cuh).
#include "sp_engine_launch.cuh"
#include "sp_fft2.cuh"
#include "sp_coherence.cuh"
namespace sp {
SP_DEFINE_SIZE(8)
SP_DEFINE_FFT2(8)
SP_DEFINE_PC(8)
}  // namespace sp
