// Mode-parallel (thread-block cluster) batch kernels for a 64 x 64 probe window.
#include "launch_impl.cuh"

int qb_launch_cluster_64(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  return qb::launch_cluster<64>(a, adj, st);
}

int qb_max_clusters_64(const ptycho_batch_args* a, bool adj) { return qb::max_clusters<64>(a, adj); }
