// Allocation-free variant of the forward model + loss launch.
//
// Some callers cannot allocate device memory themselves: host programs whose
// memory is owned by another framework's allocator or arena and that only hand
// over their own input and output buffers, plugin hosts that forbid driver
// allocations, and code that must not synchronise the device (cudaMalloc /
// cudaFree can).  ptycho_forward_loss_noalloc serves them: the per-CTA loss
// partials that ptycho_forward_loss expects in a caller-provided buffer live
// here, in a file-scope device array that the library owns.
//
// Limits and sharing:
//   * the array holds PTYCHO_NOALLOC_MAX_GRID doubles (8 KiB) on every GPU that
//     loads the library, for the life of the process;
//   * a call whose launch grid exceeds PTYCHO_NOALLOC_MAX_GRID is rejected;
//   * all calls on a device share the one array: two calls that overlap on the
//     GPU (different streams, no ordering between them) race on it.  Every CTA of
//     a call overwrites its own slot before the final sum reads it, so nothing
//     needs clearing between calls;
//   * the array's device address is looked up on a device's first call and
//     cached for the life of the process: a device reset (cudaDeviceReset, or a
//     new primary context) between calls is not supported.
#include <cuda_runtime.h>

#include <mutex>

#include "ptycho_b200.h"

// defined in ptycho_abi.cu: stores the message returned by ptycho_get_last_error
int qb_record_error(int code, const char* msg);

namespace {

static __device__ __align__(256) double g_noalloc_loss_part[PTYCHO_NOALLOC_MAX_GRID];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_part_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_loss_part on the current device.  In host code
// the array's name only stands in for the symbol; the address must come from
// cudaGetSymbolAddress, once per device, with that device current.
int noalloc_partials(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return PTYCHO_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return PTYCHO_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_part_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_loss_part);
    if (e != cudaSuccess || !p) return PTYCHO_ERR_CUDA;
    g_part_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_part_ptr[dev];
  return PTYCHO_OK;
}

}  // namespace

extern "C" int ptycho_forward_loss_noalloc(const ptycho_batch_args* a, float* out_loss, void* stream) {
  if (!a || !out_loss) return qb_record_error(PTYCHO_ERR_INVALID, "forward_loss_noalloc: args or out_loss is NULL");
  if (a->grid < 1 || a->grid > PTYCHO_NOALLOC_MAX_GRID)
    return qb_record_error(PTYCHO_ERR_INVALID,
                           "forward_loss_noalloc: grid must be in [1, PTYCHO_NOALLOC_MAX_GRID = 1024]");
  double* part = nullptr;
  int rc = noalloc_partials(&part);
  if (rc) return qb_record_error(rc, "forward_loss_noalloc: cudaGetSymbolAddress of the static partials failed");
  ptycho_batch_args b = *a;
  b.loss_part = part;
  rc = ptycho_forward_loss(&b, stream);
  if (rc) return rc;
  if (a->B == 0) return cudaMemsetAsync(out_loss, 0, sizeof(float), static_cast<cudaStream_t>(stream)) == cudaSuccess
                            ? PTYCHO_OK
                            : PTYCHO_ERR_CUDA;
  return ptycho_reduce_loss(part, a->grid, out_loss, stream);
}
