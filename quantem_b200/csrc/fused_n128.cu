// Instantiation of the fused batch kernel for a 128 x 128 probe window.
#include <cuda_runtime.h>

#include "ptycho_b200.h"
#include "ptycho_kernels.cuh"

namespace {
template <int N>
int launch_batch(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  qb::BatchParams p;
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
  const size_t smem = a->prop_r ? qb::fused_smem_bytes_sep<N>(a->S) : qb::fused_smem_bytes<N>();
  // the attribute is per device; setting it on every launch keeps multi-device
  // processes correct and costs far less than one launch
  if (adj) {
    cudaFuncSetAttribute(qb::fused_batch_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    qb::fused_batch_kernel<N, true><<<a->grid, 4 * N, smem, st>>>(p);
  } else {
    cudaFuncSetAttribute(qb::fused_batch_kernel<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    qb::fused_batch_kernel<N, false><<<a->grid, 4 * N, smem, st>>>(p);
  }
  return cudaPeekAtLastError() == cudaSuccess ? PTYCHO_OK : PTYCHO_ERR_CUDA;
}

}  // namespace

int qb_launch_batch_128(const ptycho_batch_args* a, bool adj, cudaStream_t st) {
  return launch_batch<128>(a, adj, st);
}
