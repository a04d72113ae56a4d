// Multi-dataset persistent batch kernel for a 128 x 128 probe window.
#include "launch_impl.cuh"

int qb_launch_multi_128(const ptycho_batch_args* sets, int nsets, cudaStream_t st) {
  return qb::launch_multi<128>(sets, nsets, st);
}
