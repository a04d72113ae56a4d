// Multi-dataset persistent batch kernel for a 64 x 64 probe window.
// Complex arithmetic on packed FP32 pairs (fft_engine.cuh).
#define QB_F32X2_ADD 1
#define QB_F32X2_MUL 1
#include "launch_impl.cuh"

int qb_launch_multi_64(const ptycho_batch_args* sets, int nsets, cudaStream_t st) {
  return qb::launch_multi<64>(sets, nsets, st);
}
