// Serial-mode batch kernels instantiated for a 96 x 96 probe window (mixed radix 3 x 2^k).
// Complex arithmetic on packed FP32 pairs (fft_engine.cuh).
#define QB_F32X2_ADD 1
#define QB_F32X2_MUL 1
#include "launch_impl.cuh"

int qb_launch_serial_96(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  return qb::launch_serial<96>(a, adj, st);
}
