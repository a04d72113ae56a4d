// Serial-mode batch kernels instantiated for a 128 x 128 probe window.
// Complex additions and the middle-stage FFT twiddles on packed FP32 pairs; other
// products stay scalar (fft_engine.cuh).
#define QB_F32X2_ADD 1
#define QB_F32X2_S2 1
#include "launch_impl.cuh"

int qb_launch_serial_128(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  return qb::launch_serial<128>(a, adj, st);
}
