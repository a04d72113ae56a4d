// 256 x 256 probe windows: cluster batch kernel and cluster FFT launches.
// Complex arithmetic on packed FP32 pairs in this translation unit (fft_engine.cuh).
#define QB_F32X2_ADD 1
#define QB_F32X2_MUL 1
#include "cluster256_kernels.cuh"
#include "launch_impl.cuh"

namespace {

template <bool ADJ>
cudaLaunchConfig_t c256_config(int grid, size_t smem, cudaStream_t st, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3(qb::Fft256C::T, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = qb::C256_CLUSTER;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <bool ADJ>
void c256_attrs() {
  const int smem = (int)qb::c256_smem_bytes();
  cudaFuncSetAttribute(qb::cluster256_kernel<ADJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

}  // namespace

// Clusters of 4 CTAs of the 256^2 batch kernel resident at once (-1 on error).
int qb_max_clusters_256(bool adj) {
  cudaLaunchAttribute attr[1];
  int n = 0;
  cudaError_t e;
  if (adj) {
    c256_attrs<true>();
    cudaLaunchConfig_t cfg = c256_config<true>(qb::C256_CLUSTER, qb::c256_smem_bytes(), nullptr, attr);
    e = cudaOccupancyMaxActiveClusters(&n, qb::cluster256_kernel<true>, &cfg);
  } else {
    c256_attrs<false>();
    cudaLaunchConfig_t cfg = c256_config<false>(qb::C256_CLUSTER, qb::c256_smem_bytes(), nullptr, attr);
    e = cudaOccupancyMaxActiveClusters(&n, qb::cluster256_kernel<false>, &cfg);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return n;
}

int qb_launch_c256(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  const qb::BatchParams p = qb::to_params(a);
  cudaLaunchAttribute attr[1];
  cudaError_t e;
  if (adj) {
    c256_attrs<true>();
    cudaLaunchConfig_t cfg = c256_config<true>(a->grid, qb::c256_smem_bytes(), st, attr);
    e = cudaLaunchKernelEx(&cfg, qb::cluster256_kernel<true>, p);
  } else {
    c256_attrs<false>();
    cudaLaunchConfig_t cfg = c256_config<false>(a->grid, qb::c256_smem_bytes(), st, attr);
    e = cudaLaunchKernelEx(&cfg, qb::cluster256_kernel<false>, p);
  }
  return e == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_CUDA;
}

int qb_fft256(const void* in, void* out, int count, bool inverse, float scale, cudaStream_t st) {
  const int smem = (int)qb::fft256_smem_bytes();
  cudaFuncSetAttribute(qb::fft256_batch_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(qb::fft256_batch_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const int ncl = count < 32 ? count : 32;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ncl * qb::C256_CLUSTER), 1, 1);
  cfg.blockDim = dim3(qb::Fft256C::T, 1, 1);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = qb::C256_CLUSTER;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const float2* i2 = static_cast<const float2*>(in);
  float2* o2 = static_cast<float2*>(out);
  cudaError_t e = inverse ? cudaLaunchKernelEx(&cfg, qb::fft256_batch_kernel<true>, i2, o2, count, scale)
                          : cudaLaunchKernelEx(&cfg, qb::fft256_batch_kernel<false>, i2, o2, count, scale);
  return e == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_CUDA;
}
