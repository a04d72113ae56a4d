// Mode-parallel (thread-block cluster) batch kernels for a 128 x 128 probe window.
#include "launch_impl.cuh"

int qb_launch_cluster_128(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  return qb::launch_cluster<128>(a, adj, st);
}

int qb_max_clusters_128(const ptycho_batch_args* a, bool adj) { return qb::max_clusters<128>(a, adj); }
