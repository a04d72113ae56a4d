// Serial-mode batch kernels instantiated for a 64 x 64 probe window.
#include "launch_impl.cuh"

int qb_launch_serial_64(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  return qb::launch_serial<64>(a, adj, st);
}
