// Multi-dataset persistent batch kernel for a 96 x 96 probe window.
#include "launch_impl.cuh"

int qb_launch_multi_96(const ptycho_batch_args* sets, int nsets, cudaStream_t st) {
  return qb::launch_multi<96>(sets, nsets, st);
}
