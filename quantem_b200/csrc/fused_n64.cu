// Serial-mode batch kernels instantiated for a 64 x 64 probe window.
// Complex arithmetic on packed FP32 pairs (fft_engine.cuh).
#define QB_F32X2_ADD 1
#define QB_F32X2_MUL 1
#include "launch_impl.cuh"

int qb_launch_serial_64(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  return qb::launch_serial<64>(a, adj, st);
}
