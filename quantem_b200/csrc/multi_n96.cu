// Multi-dataset persistent batch kernel for a 96 x 96 probe window.
// Complex arithmetic on packed FP32 pairs (fft_engine.cuh).
#define QB_F32X2_ADD 1
#define QB_F32X2_MUL 1
#include "launch_impl.cuh"

int qb_launch_multi_96(const ptycho_batch_args* sets, int nsets, cudaStream_t st) {
  return qb::launch_multi<96>(sets, nsets, st);
}
