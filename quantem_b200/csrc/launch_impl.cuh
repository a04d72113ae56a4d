// Host-side launch helpers shared by the per-size translation units.
#pragma once
#include <cuda_runtime.h>

#include "cluster_kernels.cuh"
#include "ptycho_b200.h"
#include "ptycho_kernels.cuh"

namespace qb {

inline BatchParams to_params(const ptycho_batch_args* a) {
  BatchParams p;
  p.obj = static_cast<const float2*>(a->obj);
  p.probe_hat = static_cast<const float2*>(a->probe_hat);
  p.prop = static_cast<const float2*>(a->prop);
  p.prop_r = static_cast<const float2*>(a->prop_r);
  p.prop_c = static_cast<const float2*>(a->prop_c);
  p.positions = a->positions;
  p.batch_idx = a->batch_idx;
  p.targets = a->targets;
  p.mask = a->mask;
  p.grad_obj = static_cast<float2*>(a->grad_obj);
  p.probe_grad_part = static_cast<float2*>(a->probe_grad_part);
  p.scratch = static_cast<float2*>(a->scratch);
  p.loss_part = a->loss_part;
  p.out_intensity = a->out_intensity;
  p.out_exit = static_cast<float2*>(a->out_exit);
  p.out_waves = static_cast<float2*>(a->out_waves);
  p.status = a->status;
  p.S = a->S;
  p.P = a->P;
  p.B = a->B;
  p.Ho = a->Ho;
  p.Wo = a->Wo;
  p.npos = a->npos;
  p.loss_scale = a->loss_scale;
  p.inv_mean_intensity = a->inv_mean_intensity;
  p.loss_type = a->loss_type;
  p.analytic = a->analytic;
  p.an_norm = a->an_norm;
  p.ckpt = a->recompute_every;
  p.grad_positions = a->grad_positions;
  p.descan = a->descan;
  p.grad_descan = a->grad_descan;
  p.grad_prop = a->grad_prop;
  return p;
}

template <int N>
size_t batch_smem(const ptycho_batch_args* a) {
  return a->prop_r ? fused_smem_bytes_sep<N>(a->S) : fused_smem_bytes<N>();
}

// the serial kernel with its optional extensions compiled in (descan, position / descan /
// propagator gradients)
inline bool wants_ext(const ptycho_batch_args* a) {
  return a->descan || a->grad_descan || a->grad_prop || a->grad_positions;
}

template <int N, bool ADJ>
void launch_ext(const BatchParams& p, int grid, size_t smem, cudaStream_t st) {
  cudaFuncSetAttribute(fused_batch_kernel<N, ADJ, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  if (ADJ)
    cudaFuncSetAttribute(fused_batch_kernel<N, ADJ, false, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)((smem + 1024) * 100 / (228 * 1024) + 1));
  fused_batch_kernel<N, ADJ, false, true><<<grid, Fft2<N>::T, smem, st>>>(p);
}

// one CTA per position, modes in sequence
template <int N>
int launch_serial(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  const BatchParams p = to_params(a);
  const size_t smem = adj ? batch_smem_bytes<N, true>(a->prop_r != nullptr, a->S)
                          : batch_smem_bytes<N, false>(a->prop_r != nullptr, a->S);
  if (wants_ext(a) && !a->analytic) {
    if (adj)
      launch_ext<N, true>(p, a->grid, smem, st);
    else
      launch_ext<N, false>(p, a->grid, smem, st);
    return cudaPeekAtLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_CUDA;
  }
  // the attribute is per device; setting it on every launch keeps multi-device
  // processes correct and costs far less than one launch
  if (adj && a->analytic) {
    cudaFuncSetAttribute(fused_batch_kernel<N, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(fused_batch_kernel<N, true, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)((smem + 1024) * 100 / (228 * 1024) + 1));
    fused_batch_kernel<N, true, true><<<a->grid, Fft2<N>::T, smem, st>>>(p);
  } else if (adj) {
    cudaFuncSetAttribute(fused_batch_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // smallest shared-memory carve-out that fits: the rest of the 256 KB is L1 for spills
    cudaFuncSetAttribute(fused_batch_kernel<N, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)((smem + 1024) * 100 / (228 * 1024) + 1));
    fused_batch_kernel<N, true><<<a->grid, Fft2<N>::T, smem, st>>>(p);
  } else {
    cudaFuncSetAttribute(fused_batch_kernel<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    fused_batch_kernel<N, false><<<a->grid, Fft2<N>::T, smem, st>>>(p);
  }
  return cudaPeekAtLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_CUDA;
}

// several datasets in one persistent launch (serial body, adjoint)
template <int N>
int launch_multi(const ptycho_batch_args* sets, int nsets, cudaStream_t st) {
  MultiParams mp;
  mp.nd = nsets;
  mp.begin[0] = 0;
  size_t smem = 0;
  for (int d = 0; d < nsets; ++d) {
    mp.d[d] = to_params(&sets[d]);
    mp.begin[d + 1] = mp.begin[d] + sets[d].grid;
    const size_t sd = batch_smem_bytes<N, true>(sets[d].prop_r != nullptr, sets[d].S);
    if (sd > smem) smem = sd;
  }
  cudaFuncSetAttribute(multi_batch_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(multi_batch_kernel<N, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)((smem + 1024) * 100 / (228 * 1024) + 1));
  multi_batch_kernel<N, true><<<mp.begin[nsets], Fft2<N>::T, smem, st>>>(mp);
  return cudaPeekAtLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_CUDA;
}

template <int N, bool ADJ>
cudaLaunchConfig_t cluster_config(const ptycho_batch_args* a, int grid, cudaStream_t st, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3(4 * N, 1, 1);
  cfg.dynamicSmemBytes = batch_smem<N>(a);
  cfg.stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)a->P;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Number of clusters of P CTAs that can be resident at once.
template <int N>
int max_clusters(const ptycho_batch_args* a, bool adj) {
  cudaLaunchAttribute attr[1];
  int n = 0;
  cudaError_t e;
  if (adj) {
    cudaFuncSetAttribute(cluster_batch_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)batch_smem<N>(a));
    cudaLaunchConfig_t cfg = cluster_config<N, true>(a, a->P, nullptr, attr);
    e = cudaOccupancyMaxActiveClusters(&n, cluster_batch_kernel<N, true>, &cfg);
  } else {
    cudaFuncSetAttribute(cluster_batch_kernel<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)batch_smem<N>(a));
    cudaLaunchConfig_t cfg = cluster_config<N, false>(a, a->P, nullptr, attr);
    e = cudaOccupancyMaxActiveClusters(&n, cluster_batch_kernel<N, false>, &cfg);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return n;
}

template <int N>
int launch_cluster(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  const BatchParams p = to_params(a);
  cudaLaunchAttribute attr[1];
  cudaError_t e;
  if (adj) {
    cudaFuncSetAttribute(cluster_batch_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)batch_smem<N>(a));
    cudaFuncSetAttribute(cluster_batch_kernel<N, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)((batch_smem<N>(a) + 1024) * 100 / (228 * 1024) + 1));
    cudaLaunchConfig_t cfg = cluster_config<N, true>(a, a->grid, st, attr);
    e = cudaLaunchKernelEx(&cfg, cluster_batch_kernel<N, true>, p);
  } else {
    cudaFuncSetAttribute(cluster_batch_kernel<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)batch_smem<N>(a));
    cudaLaunchConfig_t cfg = cluster_config<N, false>(a, a->grid, st, attr);
    e = cudaLaunchKernelEx(&cfg, cluster_batch_kernel<N, false>, p);
  }
  return e == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_CUDA;
}

}  // namespace qb
