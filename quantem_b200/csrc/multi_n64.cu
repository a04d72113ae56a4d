// Multi-dataset persistent batch kernel for a 64 x 64 probe window.
#include "launch_impl.cuh"

int qb_launch_multi_64(const ptycho_batch_args* sets, int nsets, cudaStream_t st) {
  return qb::launch_multi<64>(sets, nsets, st);
}
