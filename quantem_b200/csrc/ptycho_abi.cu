// C ABI entry points of libptycho_b200 (declared in include/ptycho_b200.h) and the
// small element-wise / reduction kernels around the fused batch kernel.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "ptycho_b200.h"
#include "cluster256_kernels.cuh"
#include "launch_impl.cuh"
#include "ptycho_kernels.cuh"

namespace {

thread_local char g_last_error[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PTYCHO_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return PTYCHO_OK;
}

bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

constexpr int kReduceBlocks = 592;  // 4 x 148 SMs
constexpr int kReduceThreads = 256;

// ---------------------------------------------------------------------------
// object hard constraint (object_models.py:289-300) and its vector-Jacobian product
// ---------------------------------------------------------------------------
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  }
  return t;  // valid in thread 0
}

// Sum of a fixed-order list of partials, computed by every block (deterministic).
__device__ __forceinline__ double sum_partials(const double* part, int n, double* red, double* bcast) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
  double t = block_sum(v, red);
  if (threadIdx.x == 0) *bcast = t;
  __syncthreads();
  return *bcast;
}

__global__ void angle_sum_kernel(const float2* __restrict__ obj, int64_t n, double* part) {
  __shared__ double red[32];
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 o = obj[i];
    v += (double)atan2f(o.y, o.x);
  }
  double t = block_sum(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// PURE: pure-phase objects (amplitude fixed at 1, object_models.py:292-298)
template <bool PURE>
__global__ void constrain_apply_kernel(const float2* __restrict__ obj, float2* __restrict__ out, int64_t n,
                                       const double* part, int nparts) {
  __shared__ double red[32];
  __shared__ double bc;
  const float mean = (float)(sum_partials(part, nparts, red, &bc) / (double)n);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 o = obj[i];
    const float amp = PURE ? 1.0f : fminf(fmaxf(hypotf(o.x, o.y), 0.0f), 1.0f);
    const float ph = atan2f(o.y, o.x) - mean;
    float s, c;
    sincosf(ph, &s, &c);
    out[i] = make_float2(amp * c, amp * s);
  }
}

// g_theta = clamp(|o|) * Im(G conj(e^{i theta})) summed over the object
template <bool PURE>
__global__ void vjp_sum_kernel(const float2* __restrict__ obj, const float2* __restrict__ gc, int64_t n,
                               const double* part_fwd, int nparts, double* part) {
  __shared__ double red[32];
  __shared__ double bc;
  const float mean = (float)(sum_partials(part_fwd, nparts, red, &bc) / (double)n);
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 o = obj[i], g = gc[i];
    const float amp = PURE ? 1.0f : fminf(fmaxf(hypotf(o.x, o.y), 0.0f), 1.0f);
    float s, c;
    sincosf(atan2f(o.y, o.x) - mean, &s, &c);
    v += (double)(amp * (g.y * c - g.x * s));
  }
  double t = block_sum(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <bool PURE>
__global__ void vjp_apply_kernel(const float2* __restrict__ obj, const float2* __restrict__ gc,
                                 float2* __restrict__ gout, int64_t n, const double* part_fwd,
                                 const double* part_g, int nparts, const float* scale) {
  __shared__ double red[32];
  __shared__ double bc;
  const float mean = (float)(sum_partials(part_fwd, nparts, red, &bc) / (double)n);
  __syncthreads();
  const float gmean = (float)(sum_partials(part_g, nparts, red, &bc) / (double)n);
  const float sc = scale ? *scale : 1.0f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 o = obj[i], g = gc[i];
    const float mag = hypotf(o.x, o.y);
    const float amp = PURE ? 1.0f : fminf(fmaxf(mag, 0.0f), 1.0f);
    float s, c;
    sincosf(atan2f(o.y, o.x) - mean, &s, &c);
    const float g_amp = g.x * c + g.y * s;            // Re(G conj(e))
    const float g_th = amp * (g.y * c - g.x * s);      // amp * Im(G conj(e))
    const float g_ph = g_th - gmean;
    // the amplitude of a pure-phase object does not enter its transmission
    const float g_mag = (!PURE && mag >= 0.0f && mag <= 1.0f) ? g_amp : 0.0f;
    float2 r = make_float2(0.f, 0.f);
    if (mag != 0.0f) {
      const float inv = 1.0f / mag;
      // g_mag * o/|o| + g_ph * i o/|o|^2
      r.x = g_mag * o.x * inv - g_ph * o.y * inv * inv;
      r.y = g_mag * o.y * inv + g_ph * o.x * inv * inv;
    }
    gout[i] = make_float2(r.x * sc, r.y * sc);
  }
}

// ---------------------------------------------------------------------------
// potential objects (object_models.py:301-320, 252-256): V' = V - offset, clamped
// at 0 with positivity; transmission t = exp(i V').  The baseline offset (when
// fixed) is factor * min(V), detached from the gradient as in the reference.
// ---------------------------------------------------------------------------
__global__ void potential_min_kernel(const float* __restrict__ v, int64_t n, double* part) {
  __shared__ float red[32];
  float m = INFINITY;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = fminf(m, v[i]);
  for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) m = fminf(m, red[i]);
    part[blockIdx.x] = (double)fminf(m, red[0]);
  }
}

// offset of the potential: factor * min over the per-block minima (0 when not fixed)
__device__ __forceinline__ float potential_offset(const double* part, int nparts, float factor) {
  if (!part) return 0.0f;
  __shared__ float bc;
  if (threadIdx.x == 0) {
    double m = part[0];
    for (int i = 1; i < nparts; ++i) m = fmin(m, part[i]);
    bc = (float)m * factor;
  }
  __syncthreads();
  return bc;
}

__global__ void potential_apply_kernel(const float* __restrict__ v, float2* __restrict__ out, int64_t n,
                                       int positivity, const double* part, int nparts, float factor) {
  const float off = potential_offset(part, nparts, factor);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x = v[i] - off;
    if (positivity) x = fmaxf(x, 0.0f);
    float s, c;
    sincosf(x, &s, &c);
    out[i] = make_float2(c, s);
  }
}

// dL/dV = Re(conj(G) i t) where the clamp passes (V - offset >= 0, as torch.clamp's gradient)
__global__ void potential_vjp_kernel(const float* __restrict__ v, const float2* __restrict__ gc,
                                     float* __restrict__ gout, int64_t n, int positivity, const double* part,
                                     int nparts, float factor, const float* scale) {
  const float off = potential_offset(part, nparts, factor);
  const float sc = scale ? *scale : 1.0f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x = v[i] - off;
    const bool pass = !positivity || x >= 0.0f;
    if (positivity) x = fmaxf(x, 0.0f);
    float s, c;
    sincosf(x, &s, &c);
    const float2 g = gc[i];
    gout[i] = pass ? sc * (g.y * c - g.x * s) : 0.0f;
  }
}

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------
__global__ void reduce_partials_kernel(const float2* __restrict__ parts, float2* __restrict__ out, int nparts,
                                       int64_t count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    float2 a = make_float2(0.f, 0.f);
    for (int g = 0; g < nparts; ++g) {
      const float2 v = parts[(int64_t)g * count + i];
      a.x += v.x;
      a.y += v.y;
    }
    out[i] = a;
  }
}

__global__ void reduce_loss_kernel(const double* parts, int nparts, float* out) {
  __shared__ double red[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) v += parts[i];
  double t = block_sum(v, red);
  if (threadIdx.x == 0) out[0] = (float)t;
}

// ---------------------------------------------------------------------------
// optimisers (torch.optim semantics, real view of complex parameters)
// ---------------------------------------------------------------------------
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, const float* lr_dev, float b1, float b2,
                            float eps, float wd, int decoupled, float bc1, float bc2_sqrt) {
  const float lr_ = lr_dev ? *lr_dev : lr;
  const float step = lr_ / bc1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float pi = p[i];
    float gi = g[i];
    if (wd != 0.0f) {
      if (decoupled) pi *= 1.0f - lr_ * wd;
      else gi = fmaf(wd, pi, gi);
    }
    float mi = m[i];
    mi = mi + (1.0f - b1) * (gi - mi);
    float vi = v[i] * b2 + (1.0f - b2) * gi * gi;
    const float denom = sqrtf(vi) / bc2_sqrt + eps;
    pi = pi - step * (mi / denom);
    p[i] = pi;
    m[i] = mi;
    v[i] = vi;
  }
}

// Adam with the step count on the device (CUDA-graph replays advance it): the
// bias corrections 1 - beta^t are evaluated per launch from *step.
__global__ void adam_dev_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, int64_t n, const float* lr_dev, const float* step, float b1,
                                float b2, float eps, float wd, int decoupled) {
  const float t = *step;
  const float lr_ = *lr_dev;
  const float bc1 = 1.0f - powf(b1, t);
  const float bc2s = sqrtf(1.0f - powf(b2, t));
  const float stp = lr_ / bc1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float pi = p[i];
    float gi = g[i];
    if (wd != 0.0f) {
      if (decoupled) pi *= 1.0f - lr_ * wd;
      else gi = fmaf(wd, pi, gi);
    }
    float mi = m[i];
    mi = mi + (1.0f - b1) * (gi - mi);
    float vi = v[i] * b2 + (1.0f - b2) * gi * gi;
    pi = pi - stp * (mi / (sqrtf(vi) / bc2s + eps));
    p[i] = pi;
    m[i] = mi;
    v[i] = vi;
  }
}

__global__ void add_scalar_kernel(float* x, float v) { x[0] += v; }

__global__ void sgd_kernel(float* __restrict__ p, const float* __restrict__ g, int64_t n, float lr,
                           const float* lr_dev, float wd) {
  const float lr_ = lr_dev ? *lr_dev : lr;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float gi = g[i];
    if (wd != 0.0f) gi = fmaf(wd, p[i], gi);
    p[i] = p[i] - lr_ * gi;
  }
}

// torch.optim.Adam with amsgrad=True: the denominator takes the running maximum of the
// second moment (vmax), otherwise the same step as adam_kernel
__global__ void adam_amsgrad_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                    float* __restrict__ v, float* __restrict__ vmax, int64_t n, float lr,
                                    const float* lr_dev, float b1, float b2, float eps, float wd, int decoupled,
                                    float bc1, float bc2_sqrt) {
  const float lr_ = lr_dev ? *lr_dev : lr;
  const float step = lr_ / bc1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float pi = p[i];
    float gi = g[i];
    if (wd != 0.0f) {
      if (decoupled) pi *= 1.0f - lr_ * wd;
      else gi = fmaf(wd, pi, gi);
    }
    float mi = m[i];
    mi = mi + (1.0f - b1) * (gi - mi);
    const float vi = v[i] * b2 + (1.0f - b2) * gi * gi;
    const float vm = fmaxf(vmax[i], vi);
    const float denom = sqrtf(vm) / bc2_sqrt + eps;
    p[i] = pi - step * (mi / denom);
    m[i] = mi;
    v[i] = vi;
    vmax[i] = vm;
  }
}

// torch.optim.SGD with momentum (dampening, Nesterov): the first step seeds the buffer with
// the gradient, later ones take buf = momentum buf + (1 - dampening) g
__global__ void sgd_momentum_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ buf,
                                    int64_t n, float lr, const float* lr_dev, float wd, float momentum,
                                    float dampening, int nesterov, int first) {
  const float lr_ = lr_dev ? *lr_dev : lr;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float pi = p[i];
    float gi = g[i];
    if (wd != 0.0f) gi = fmaf(wd, pi, gi);
    const float b = first ? gi : fmaf(1.0f - dampening, gi, buf[i] * momentum);
    buf[i] = b;
    const float d = nesterov ? fmaf(momentum, b, gi) : b;
    p[i] = pi - lr_ * d;
  }
}

// ---------------------------------------------------------------------------
// analytic update finalisation (object_models.py:686-725, probe_models.py:774-783)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));  // ordered like floats for v >= 0
}

// max over (slice, position) of the summed |o|^2 of each object patch
__global__ void patch_energy_max_kernel(const float2* __restrict__ obj, const float* __restrict__ positions,
                                        const int64_t* __restrict__ batch_idx, int S, int Ho, int Wo, int n, int B,
                                        int npos, float* out) {
  __shared__ double red[32];
  for (int b = blockIdx.x; b < B; b += gridDim.x) {
    const int64_t gi = batch_idx[b];
    if (gi < 0 || gi >= npos) continue;
    const int r0 = qb::wrap_index((int)rintf(positions[2 * gi]), Ho);
    const int c0 = qb::wrap_index((int)rintf(positions[2 * gi + 1]), Wo);
    for (int s = 0; s < S; ++s) {
      double v = 0.0;
      for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
        const int r = i / n, c = i % n;
        const int row = qb::wrap_index(r0 + qb::fsigned(r, n), Ho);
        const int col = qb::wrap_index(c0 + qb::fsigned(c, n), Wo);
        v += (double)qb::cabs2(obj[((size_t)s * Ho + row) * Wo + col]);
      }
      const double t = block_sum(v, red);
      if (threadIdx.x == 0) atomic_max_nonneg(out, (float)t);
    }
  }
}

__global__ void plane_max_kernel(const float* __restrict__ a, int64_t plane, int planes, float* maxes) {
  const int pl = blockIdx.y;
  float v = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < plane; i += (int64_t)gridDim.x * blockDim.x)
    v = fmaxf(v, a[(int64_t)pl * plane + i]);
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(maxes + pl, v);
}

__global__ void analytic_obj_kernel(const float2* __restrict__ upd, const float* __restrict__ maxes, int P,
                                    int64_t plane, int S, float2* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)S * plane;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / plane);
    float nrm = 0.f;
    for (int q = 0; q < P; ++q) nrm += maxes[s * P + q];
    const float2 u = upd[i];
    out[i] = make_float2(-u.x / nrm, -u.y / nrm);
  }
}

__global__ void analytic_probe_kernel(float2* __restrict__ x, int64_t count, const float* __restrict__ obj_norm,
                                      float ortho_norm) {
  const float sc = -1.0f / (obj_norm[0] * ortho_norm);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = make_float2(x[i].x * sc, x[i].y * sc);
}

// FP32 FMA throughput probe: 16 independent dependent-FMA chains per thread.
__global__ void __launch_bounds__(512) fma_probe_kernel(float* out, int iters) {
  float a[16];
  const float b = 1.0000001f + threadIdx.x * 1e-9f, c = 1e-7f;
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = fmaf(a[k], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += a[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 4 * 148) b = 4 * 148;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

// Records `msg` as this host thread's last error (used by noalloc.cu).
int qb_record_error(int code, const char* msg) { return fail(code, "%s", msg); }

// defined in fused_n{64,128}.cu and cluster_n{64,128}.cu
int qb_launch_serial_64(const ptycho_batch_args* a, bool adj, cudaStream_t st);
int qb_launch_serial_128(const ptycho_batch_args* a, bool adj, cudaStream_t st);
// defined in fused_n96.cu / multi_n96.cu: 96 x 96 windows (serial variant only)
int qb_launch_serial_96(const ptycho_batch_args* a, bool adj, cudaStream_t st);
int qb_launch_multi_96(const ptycho_batch_args* sets, int nsets, cudaStream_t st);
int qb_launch_cluster_64(const ptycho_batch_args* a, bool adj, cudaStream_t st);
int qb_launch_cluster_128(const ptycho_batch_args* a, bool adj, cudaStream_t st);
int qb_launch_multi_64(const ptycho_batch_args* sets, int nsets, cudaStream_t st);
int qb_launch_multi_128(const ptycho_batch_args* sets, int nsets, cudaStream_t st);
int qb_max_clusters_64(const ptycho_batch_args* a, bool adj);
int qb_max_clusters_128(const ptycho_batch_args* a, bool adj);
// defined in c256.cu: 256 x 256 windows on clusters of 4 CTAs
int qb_max_clusters_256(bool adj);
int qb_launch_c256(const ptycho_batch_args* a, bool adj, cudaStream_t st);
int qb_fft256(const void* in, void* out, int count, bool inverse, float scale, cudaStream_t st);

namespace {

int validate_batch(const ptycho_batch_args* a, bool adj) {
  if (!a) return fail(PTYCHO_ERR_INVALID, "args is NULL");
  if (a->n != 64 && a->n != 96 && a->n != 128 && a->n != 256)
    return fail(PTYCHO_ERR_UNSUPPORTED, "probe window n=%d not built (64, 96, 128, 256)", a->n);
  if (a->n == 96 && a->variant == PTYCHO_VARIANT_CLUSTER)
    return fail(PTYCHO_ERR_UNSUPPORTED, "n=96 runs on the serial variant");
  if (a->n == 256) {
    if (a->analytic) return fail(PTYCHO_ERR_UNSUPPORTED, "the analytic update is built for n = 64, 96, 128");
    if (a->out_exit || a->out_waves)
      return fail(PTYCHO_ERR_UNSUPPORTED, "exit-wave / wave outputs are built for n = 64, 128");
    if (a->recompute_every < 0 || a->recompute_every > a->S)
      return fail(PTYCHO_ERR_INVALID, "recompute_every=%d outside [0, S=%d]", a->recompute_every, a->S);
    if (a->B > 0 && a->grid % 4 != 0) return fail(PTYCHO_ERR_INVALID, "n=256: grid %d is not a multiple of 4", a->grid);
  }
  if (a->S < 1 || a->P < 1 || a->B < 0 || a->Ho < 1 || a->Wo < 1 || a->npos < 1)
    return fail(PTYCHO_ERR_INVALID, "bad sizes S=%d P=%d B=%d Ho=%d Wo=%d npos=%d", a->S, a->P, a->B, a->Ho, a->Wo,
                a->npos);
  if (a->B > 0 && (a->grid < 1 || a->grid > 65535)) return fail(PTYCHO_ERR_INVALID, "bad grid %d", a->grid);
  if (!a->obj || !a->probe_hat || !a->positions || !a->batch_idx || !a->targets || !a->mask || !a->loss_part)
    return fail(PTYCHO_ERR_INVALID, "required pointer is NULL");
  if (a->S > 1 && !a->prop && !(a->prop_r && a->prop_c))
    return fail(PTYCHO_ERR_INVALID, "propagators are NULL with S > 1");
  if ((a->prop_r == nullptr) != (a->prop_c == nullptr))
    return fail(PTYCHO_ERR_INVALID, "prop_r and prop_c must be given together");
  if (a->prop_r && a->n != 256) {  // n = 256 reads the factors through the L1 cache
    const size_t need = (size_t)(a->n == 64 ? qb::fused_smem_bytes_sep<64>(a->S)
                                            : (a->n == 96 ? qb::fused_smem_bytes_sep<96>(a->S)
                                                          : qb::fused_smem_bytes_sep<128>(a->S)));
    if (need + 1024 > 232448)
      return fail(PTYCHO_ERR_UNSUPPORTED, "separable propagators of %d slices do not fit in shared memory; pass prop",
                  a->S);
  }
  if (adj && (!a->grad_obj || !a->probe_grad_part || !a->scratch))
    return fail(PTYCHO_ERR_INVALID, "adjoint buffers are NULL");
  const void* ptrs[] = {a->obj, a->probe_hat, a->prop, a->grad_obj, a->probe_grad_part, a->scratch, a->out_exit,
                        a->out_waves, a->prop_r, a->prop_c};
  for (const void* q : ptrs)
    if (q && !aligned(q, 8)) return fail(PTYCHO_ERR_INVALID, "complex buffer not 8-byte aligned");
  if (a->loss_type < 0 || a->loss_type > 4) return fail(PTYCHO_ERR_INVALID, "bad loss type %d", a->loss_type);
  if ((a->grad_descan || a->grad_prop) && (!adj || a->analytic))
    return fail(PTYCHO_ERR_UNSUPPORTED, "descan / propagator gradients come from the autograd adjoint launch");
  if (a->grad_descan && !a->descan) return fail(PTYCHO_ERR_INVALID, "grad_descan needs the descan shifts");
  if (a->grad_prop && a->S > 17)
    return fail(PTYCHO_ERR_UNSUPPORTED, "propagator gradients are built for up to 17 slices (S=%d)", a->S);
  if (a->descan && a->analytic) return fail(PTYCHO_ERR_UNSUPPORTED, "descan shifts with the analytic update");
  if (a->analytic) {
    if (!adj) return fail(PTYCHO_ERR_INVALID, "analytic is an adjoint-launch option");
    if (!a->an_norm) return fail(PTYCHO_ERR_INVALID, "analytic update needs an_norm");
    if (a->variant == PTYCHO_VARIANT_CLUSTER)
      return fail(PTYCHO_ERR_UNSUPPORTED, "the analytic update runs on the serial variant");
  }
  return PTYCHO_OK;
}

// PTYCHO_VARIANT_CLUSTER or PTYCHO_VARIANT_SERIAL for this configuration, or -1.
int resolve_variant(const ptycho_batch_args* a) {
  if (a->variant == PTYCHO_VARIANT_SERIAL) return PTYCHO_VARIANT_SERIAL;
  if (a->variant == PTYCHO_VARIANT_CLUSTER)
    return (a->n != 96 && a->P >= 1 && a->P <= 8) ? PTYCHO_VARIANT_CLUSTER : -1;
  // measured on B200 (8 slices, 4 modes, 128^2): serial 5.9 ms vs cluster 6.9 ms per 592 positions
  if (a->variant == PTYCHO_VARIANT_AUTO) return PTYCHO_VARIANT_SERIAL;
  return -1;
}

int run_batch(const ptycho_batch_args* a, void* stream, bool adj) {
  int rc = validate_batch(a, adj);
  if (rc) return rc;
  if (a->B == 0) return PTYCHO_OK;
  if (a->n == 256) {
    if (a->grad_positions)
      return fail(PTYCHO_ERR_UNSUPPORTED, "position gradients are not built for 256 x 256 windows");
    if (a->descan || a->grad_descan || a->grad_prop)
      return fail(PTYCHO_ERR_UNSUPPORTED, "descan shifts and propagator gradients are not built for 256 x 256 windows");
    const int lrc = qb_launch_c256(a, adj, static_cast<cudaStream_t>(stream));
    if (lrc) return fail(lrc, "cluster256_kernel launch: %s", cudaGetErrorString(cudaGetLastError()));
    return PTYCHO_OK;
  }
  if (a->grad_positions && (!adj || a->analytic))
    return fail(PTYCHO_ERR_UNSUPPORTED, "position gradients come from the autograd adjoint launch");
  // the extensions (descan, position / descan / propagator gradients) live in the serial kernel
  const int variant = (a->analytic || qb::wants_ext(a)) ? PTYCHO_VARIANT_SERIAL : resolve_variant(a);
  if (variant < 0) return fail(PTYCHO_ERR_UNSUPPORTED, "variant %d not available for P=%d", a->variant, a->P);
  if (variant == PTYCHO_VARIANT_CLUSTER && a->grid % a->P != 0)
    return fail(PTYCHO_ERR_INVALID, "cluster launch: grid %d is not a multiple of P=%d", a->grid, a->P);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool cl = variant == PTYCHO_VARIANT_CLUSTER;
  const int lrc = cl ? (a->n == 64 ? qb_launch_cluster_64(a, adj, st) : qb_launch_cluster_128(a, adj, st))
                     : (a->n == 64 ? qb_launch_serial_64(a, adj, st)
                                   : (a->n == 96 ? qb_launch_serial_96(a, adj, st) : qb_launch_serial_128(a, adj, st)));
  if (lrc) return fail(lrc, "fused_batch_kernel launch: %s", cudaGetErrorString(cudaGetLastError()));
  return PTYCHO_OK;
}

}  // namespace

extern "C" {

int ptycho_get_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return PTYCHO_ERR_INVALID;
  strncpy(buf, g_last_error, len - 1);
  buf[len - 1] = '\0';
  return PTYCHO_OK;
}

// 2: ptycho_batch_args.grad_positions; 3: descan, grad_descan, grad_prop
int ptycho_abi_version(void) { return 3; }

int ptycho_sm_count(int* out) {
  if (!out) return fail(PTYCHO_ERR_INVALID, "out is NULL");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(out, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return fail(PTYCHO_ERR_CUDA, "sm count: %s", cudaGetErrorString(e));
  return PTYCHO_OK;
}

int ptycho_workspace_elems(int n, int S, int P, int grid, int64_t* scratch_elems, int64_t* partial_elems) {
  if (n < 1 || S < 1 || P < 1 || grid < 1) return fail(PTYCHO_ERR_INVALID, "bad workspace sizes");
  const int64_t nn = (int64_t)n * n;
  if (scratch_elems) *scratch_elems = (int64_t)grid * (P * S + P + 1) * nn;
  if (partial_elems) *partial_elems = (int64_t)grid * P * nn;
  return PTYCHO_OK;
}

int ptycho_batch_plan(const ptycho_batch_args* a, int adjoint, int* variant, int* grid, int64_t* scratch_elems,
                      int64_t* partial_elems, int* partial_parts) {
  if (!a) return fail(PTYCHO_ERR_INVALID, "plan: args is NULL");
  if (a->n != 64 && a->n != 96 && a->n != 128 && a->n != 256)
    return fail(PTYCHO_ERR_UNSUPPORTED, "probe window n=%d not built (64, 96, 128, 256)", a->n);
  if (a->S < 1 || a->P < 1 || a->B < 0) return fail(PTYCHO_ERR_INVALID, "plan: bad sizes");
  if (a->n == 256) {  // one cluster of 4 CTAs per position; each CTA holds a quarter of every wave
    const int mc = qb_max_clusters_256(adjoint != 0);
    if (mc < 1) return fail(PTYCHO_ERR_UNSUPPORTED, "no cluster of 4 CTAs with %zu B shared memory fits",
                            qb::c256_smem_bytes());
    const int B1 = a->B > 0 ? a->B : 1;
    const int ncl = B1 < mc ? B1 : mc;
    const int64_t q = (int64_t)256 * 256 / 4;
    if (variant) *variant = PTYCHO_VARIANT_CLUSTER;
    if (grid) *grid = 4 * ncl;
    if (scratch_elems) *scratch_elems = adjoint ? (int64_t)4 * ncl * qb::c256_slots(a->S, a->P, a->recompute_every) * q : 0;
    if (partial_elems) *partial_elems = (int64_t)ncl * a->P * 256 * 256;
    if (partial_parts) *partial_parts = ncl;
    return PTYCHO_OK;
  }
  const int v = (a->analytic || qb::wants_ext(a)) ? PTYCHO_VARIANT_SERIAL : resolve_variant(a);
  if (v < 0) return fail(PTYCHO_ERR_UNSUPPORTED, "variant %d not available for P=%d", a->variant, a->P);
  int sms = 0, dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return fail(PTYCHO_ERR_CUDA, "plan: %s", cudaGetErrorString(e));
  const int64_t nn = (int64_t)a->n * a->n;
  const int B = a->B > 0 ? a->B : 1;
  int g, parts;
  int64_t scr, part;
  if (v == PTYCHO_VARIANT_CLUSTER) {
    int mc = a->n == 64 ? qb_max_clusters_64(a, adjoint != 0) : qb_max_clusters_128(a, adjoint != 0);
    if (mc < 1) return fail(PTYCHO_ERR_UNSUPPORTED, "no cluster of %d CTAs fits on this device", a->P);
    const int ncl = B < mc ? B : mc;
    g = ncl * a->P;
    parts = ncl;
    scr = (int64_t)g * a->S * nn;
    part = (int64_t)g * nn;
  } else {
    g = B < sms ? B : sms;
    parts = g;
    // waves, far fields, intensity tile (+ the Fourier waves after each propagation)
    scr = (int64_t)g * (a->P * a->S + a->P + 1 + (a->grad_prop ? a->P * (a->S - 1) : 0)) * nn;
    part = (int64_t)g * a->P * nn;
  }
  if (variant) *variant = v;
  if (grid) *grid = g;
  if (scratch_elems) *scratch_elems = scr;
  if (partial_elems) *partial_elems = part;
  if (partial_parts) *partial_parts = parts;
  return PTYCHO_OK;
}

int ptycho_forward_loss(const ptycho_batch_args* a, void* stream) { return run_batch(a, stream, false); }

int ptycho_forward_adjoint_multi(const ptycho_batch_args* sets, int nsets, void* stream) {
  if (!sets || nsets < 1 || nsets > PTYCHO_MAX_DATASETS)
    return fail(PTYCHO_ERR_INVALID, "multi: nsets must be in [1, %d]", PTYCHO_MAX_DATASETS);
  long total = 0;
  for (int d = 0; d < nsets; ++d) {
    const int rc = validate_batch(&sets[d], true);
    if (rc) {
      char why[512];
      strncpy(why, g_last_error, sizeof(why) - 1);
      why[sizeof(why) - 1] = '\0';
      return fail(rc, "multi: dataset %d: %s", d, why);
    }
    if (sets[d].n != sets[0].n) return fail(PTYCHO_ERR_INVALID, "multi: every dataset needs the same probe window");
    if (sets[d].n == 256 || sets[d].analytic)
      return fail(PTYCHO_ERR_UNSUPPORTED, "multi: datasets with n = 64 / 128 and the autograd adjoint only");
    if (qb::wants_ext(&sets[d]))
      return fail(PTYCHO_ERR_UNSUPPORTED,
                  "multi: descan shifts and position / descan / propagator gradients run on ptycho_forward_adjoint");
    if (sets[d].grid < 1) return fail(PTYCHO_ERR_INVALID, "multi: dataset %d has grid %d", d, sets[d].grid);
    total += sets[d].grid;
  }
  if (total > 65535) return fail(PTYCHO_ERR_INVALID, "multi: %ld CTAs in total", total);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int lrc = sets[0].n == 64 ? qb_launch_multi_64(sets, nsets, st)
                                   : (sets[0].n == 96 ? qb_launch_multi_96(sets, nsets, st)
                                                      : qb_launch_multi_128(sets, nsets, st));
  if (lrc) return fail(lrc, "multi_batch_kernel launch: %s", cudaGetErrorString(cudaGetLastError()));
  return PTYCHO_OK;
}

int ptycho_forward_adjoint(const ptycho_batch_args* a, void* stream) { return run_batch(a, stream, true); }

int ptycho_fft2(const void* in, void* out, int count, int n, int inverse, float scale, void* stream) {
  if (!in || !out || count < 0) return fail(PTYCHO_ERR_INVALID, "fft2: bad arguments");
  if (n != 64 && n != 96 && n != 128 && n != 256) return fail(PTYCHO_ERR_UNSUPPORTED, "fft2: n=%d not built", n);
  if (count == 0) return PTYCHO_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 256) {  // in place is safe: a cluster loads its transform before its first cluster barrier
    if (qb_fft256(in, out, count, inverse != 0, scale, st)) return check_launch("fft256_batch_kernel");
    return check_launch("fft256_batch_kernel");
  }
  const float2* i2 = static_cast<const float2*>(in);
  float2* o2 = static_cast<float2*>(out);
  const int grid = count < 148 ? count : 148;
  if (n == 64) {
    const size_t smem = qb::fft2_smem_bytes<64>();
    if (inverse) qb::fft2_batch_kernel<64, true><<<grid, 256, smem, st>>>(i2, o2, count, scale);
    else qb::fft2_batch_kernel<64, false><<<grid, 256, smem, st>>>(i2, o2, count, scale);
  } else if (n == 96) {
    const size_t smem = qb::fft2_smem_bytes<96>();
    cudaFuncSetAttribute(qb::fft2_batch_kernel<96, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(qb::fft2_batch_kernel<96, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (inverse) qb::fft2_batch_kernel<96, true><<<grid, qb::Fft2<96>::T, smem, st>>>(i2, o2, count, scale);
    else qb::fft2_batch_kernel<96, false><<<grid, qb::Fft2<96>::T, smem, st>>>(i2, o2, count, scale);
  } else {
    const size_t smem = qb::fft2_smem_bytes<128>();
    cudaFuncSetAttribute(qb::fft2_batch_kernel<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(qb::fft2_batch_kernel<128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (inverse) qb::fft2_batch_kernel<128, true><<<grid, 512, smem, st>>>(i2, o2, count, scale);
    else qb::fft2_batch_kernel<128, false><<<grid, 512, smem, st>>>(i2, o2, count, scale);
  }
  return check_launch("fft2_batch_kernel");
}

int ptycho_reduce_partials(const void* parts, void* out, int nparts, int64_t count, void* stream) {
  if (!parts || !out || nparts < 1 || count < 0) return fail(PTYCHO_ERR_INVALID, "reduce_partials: bad arguments");
  if (count == 0) return PTYCHO_OK;
  reduce_partials_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(parts), static_cast<float2*>(out), nparts, count);
  return check_launch("reduce_partials_kernel");
}

int ptycho_reduce_loss(const double* parts, int nparts, float* out, void* stream) {
  if (!parts || !out || nparts < 1) return fail(PTYCHO_ERR_INVALID, "reduce_loss: bad arguments");
  reduce_loss_kernel<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(parts, nparts, out);
  return check_launch("reduce_loss_kernel");
}

int ptycho_reduce_blocks(void) { return kReduceBlocks; }

int ptycho_obj_constrain(const void* obj, void* out, int64_t count, double* work, int nwork, void* stream) {
  if (!obj || !out || !work || count < 1) return fail(PTYCHO_ERR_INVALID, "obj_constrain: bad arguments");
  if (nwork < 2 * kReduceBlocks) return fail(PTYCHO_ERR_INVALID, "obj_constrain: work too small (%d)", nwork);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float2* o = static_cast<const float2*>(obj);
  angle_sum_kernel<<<kReduceBlocks, kReduceThreads, 0, st>>>(o, count, work);
  constrain_apply_kernel<false><<<kReduceBlocks, kReduceThreads, 0, st>>>(o, static_cast<float2*>(out), count, work,
                                                                          kReduceBlocks);
  return check_launch("obj_constrain");
}

int ptycho_obj_constrain_vjp(const void* obj, const void* grad_c, void* grad_raw, int64_t count, double* work,
                             int nwork, const float* scale, void* stream) {
  if (!obj || !grad_c || !grad_raw || !work || count < 1)
    return fail(PTYCHO_ERR_INVALID, "obj_constrain_vjp: bad arguments");
  if (nwork < 2 * kReduceBlocks) return fail(PTYCHO_ERR_INVALID, "obj_constrain_vjp: work too small");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float2* o = static_cast<const float2*>(obj);
  const float2* g = static_cast<const float2*>(grad_c);
  vjp_sum_kernel<false><<<kReduceBlocks, kReduceThreads, 0, st>>>(o, g, count, work, kReduceBlocks,
                                                                   work + kReduceBlocks);
  vjp_apply_kernel<false><<<kReduceBlocks, kReduceThreads, 0, st>>>(o, g, static_cast<float2*>(grad_raw), count, work,
                                                                    work + kReduceBlocks, kReduceBlocks, scale);
  return check_launch("obj_constrain_vjp");
}

int ptycho_obj_transmission(const void* obj, void* out, int64_t count, int obj_type, int positivity,
                            int fix_baseline, float baseline_factor, double* work, int nwork, void* stream) {
  if (!obj || !out || !work || count < 1) return fail(PTYCHO_ERR_INVALID, "obj_transmission: bad arguments");
  if (nwork < 2 * kReduceBlocks) return fail(PTYCHO_ERR_INVALID, "obj_transmission: work too small (%d)", nwork);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (obj_type) {
    case PTYCHO_OBJ_COMPLEX:
      return ptycho_obj_constrain(obj, out, count, work, nwork, stream);
    case PTYCHO_OBJ_PURE_PHASE: {
      const float2* o = static_cast<const float2*>(obj);
      angle_sum_kernel<<<kReduceBlocks, kReduceThreads, 0, st>>>(o, count, work);
      constrain_apply_kernel<true><<<kReduceBlocks, kReduceThreads, 0, st>>>(o, static_cast<float2*>(out), count,
                                                                             work, kReduceBlocks);
      return check_launch("obj_transmission (pure phase)");
    }
    case PTYCHO_OBJ_POTENTIAL: {
      const float* v = static_cast<const float*>(obj);
      if (fix_baseline) potential_min_kernel<<<kReduceBlocks, kReduceThreads, 0, st>>>(v, count, work);
      potential_apply_kernel<<<kReduceBlocks, kReduceThreads, 0, st>>>(
          v, static_cast<float2*>(out), count, positivity, fix_baseline ? work : nullptr, kReduceBlocks,
          baseline_factor);
      return check_launch("obj_transmission (potential)");
    }
    default:
      return fail(PTYCHO_ERR_INVALID, "obj_transmission: unknown object type %d", obj_type);
  }
}

int ptycho_obj_transmission_vjp(const void* obj, const void* grad_t, void* grad_raw, int64_t count, int obj_type,
                                int positivity, int fix_baseline, float baseline_factor, double* work, int nwork,
                                const float* scale, void* stream) {
  if (!obj || !grad_t || !grad_raw || !work || count < 1)
    return fail(PTYCHO_ERR_INVALID, "obj_transmission_vjp: bad arguments");
  if (nwork < 2 * kReduceBlocks) return fail(PTYCHO_ERR_INVALID, "obj_transmission_vjp: work too small");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float2* g = static_cast<const float2*>(grad_t);
  switch (obj_type) {
    case PTYCHO_OBJ_COMPLEX:
      return ptycho_obj_constrain_vjp(obj, grad_t, grad_raw, count, work, nwork, scale, stream);
    case PTYCHO_OBJ_PURE_PHASE: {
      const float2* o = static_cast<const float2*>(obj);
      vjp_sum_kernel<true><<<kReduceBlocks, kReduceThreads, 0, st>>>(o, g, count, work, kReduceBlocks,
                                                                     work + kReduceBlocks);
      vjp_apply_kernel<true><<<kReduceBlocks, kReduceThreads, 0, st>>>(o, g, static_cast<float2*>(grad_raw), count,
                                                                       work, work + kReduceBlocks, kReduceBlocks,
                                                                       scale);
      return check_launch("obj_transmission_vjp (pure phase)");
    }
    case PTYCHO_OBJ_POTENTIAL: {
      // `work` holds the per-block minima of the matching forward call when the baseline is fixed
      potential_vjp_kernel<<<kReduceBlocks, kReduceThreads, 0, st>>>(
          static_cast<const float*>(obj), g, static_cast<float*>(grad_raw), count, positivity,
          fix_baseline ? work : nullptr, kReduceBlocks, baseline_factor, scale);
      return check_launch("obj_transmission_vjp (potential)");
    }
    default:
      return fail(PTYCHO_ERR_INVALID, "obj_transmission_vjp: unknown object type %d", obj_type);
  }
}

int ptycho_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t count, float lr,
                     const float* lr_dev, float beta1, float beta2, float eps, float weight_decay, int decoupled,
                     float bc1, float bc2_sqrt, void* stream) {
  if (!param || !grad || !exp_avg || !exp_avg_sq || count < 0) return fail(PTYCHO_ERR_INVALID, "adam: bad arguments");
  if (count == 0) return PTYCHO_OK;
  adam_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      param, grad, exp_avg, exp_avg_sq, count, lr, lr_dev, beta1, beta2, eps, weight_decay, decoupled, bc1, bc2_sqrt);
  return check_launch("adam_kernel");
}

int ptycho_patch_energy_max(const void* obj, const float* positions, const int64_t* batch_idx, int S, int Ho,
                            int Wo, int n, int B, int npos, float* out, void* stream) {
  if (!obj || !positions || !batch_idx || !out || S < 1 || Ho < 1 || Wo < 1 || n < 1 || B < 0 || npos < 1)
    return fail(PTYCHO_ERR_INVALID, "patch_energy_max: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(out, 0, sizeof(float), st) != cudaSuccess) return check_launch("patch_energy_max memset");
  if (B == 0) return PTYCHO_OK;
  const int grid = B < kReduceBlocks ? B : kReduceBlocks;
  patch_energy_max_kernel<<<grid, 256, 0, st>>>(static_cast<const float2*>(obj), positions, batch_idx, S, Ho, Wo, n,
                                                B, npos, out);
  return check_launch("patch_energy_max_kernel");
}

int ptycho_analytic_obj_finalize(const void* upd, const float* norm, float* maxes, int S, int P, int64_t plane,
                                 void* out, void* stream) {
  if (!upd || !norm || !maxes || !out || S < 1 || P < 1 || plane < 1)
    return fail(PTYCHO_ERR_INVALID, "analytic_obj_finalize: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(maxes, 0, sizeof(float) * (size_t)S * P, st) != cudaSuccess)
    return check_launch("analytic_obj_finalize memset");
  int bx = (int)((plane + 255) / 256);
  if (bx > 64) bx = 64;
  plane_max_kernel<<<dim3(bx, S * P), 256, 0, st>>>(norm, plane, S * P, maxes);
  analytic_obj_kernel<<<grid_for((int64_t)S * plane, 256), 256, 0, st>>>(static_cast<const float2*>(upd), maxes, P,
                                                                          plane, S, static_cast<float2*>(out));
  return check_launch("analytic_obj_finalize");
}

int ptycho_analytic_probe_finalize(void* probe_grad, int64_t count, const float* obj_norm, float ortho_norm,
                                   void* stream) {
  if (!probe_grad || !obj_norm || count < 0) return fail(PTYCHO_ERR_INVALID, "analytic_probe_finalize: bad arguments");
  if (count == 0) return PTYCHO_OK;
  analytic_probe_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<float2*>(probe_grad), count, obj_norm, ortho_norm);
  return check_launch("analytic_probe_kernel");
}

int ptycho_fp32_fma_probe(float* out, int iters, int blocks, void* stream) {
  if (!out || iters < 1 || blocks < 1) return fail(PTYCHO_ERR_INVALID, "fma probe: bad arguments");
  fma_probe_kernel<<<blocks, 512, 0, static_cast<cudaStream_t>(stream)>>>(out, iters);
  return check_launch("fma_probe_kernel");
}

int ptycho_adam_step_dev(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t count,
                         const float* lr_dev, const float* step_dev, float beta1, float beta2, float eps,
                         float weight_decay, int decoupled, void* stream) {
  if (!param || !grad || !exp_avg || !exp_avg_sq || !lr_dev || !step_dev || count < 0)
    return fail(PTYCHO_ERR_INVALID, "adam_dev: bad arguments");
  if (count == 0) return PTYCHO_OK;
  adam_dev_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      param, grad, exp_avg, exp_avg_sq, count, lr_dev, step_dev, beta1, beta2, eps, weight_decay, decoupled);
  return check_launch("adam_dev_kernel");
}

int ptycho_add_scalar(float* x, float v, void* stream) {
  if (!x) return fail(PTYCHO_ERR_INVALID, "add_scalar: NULL");
  add_scalar_kernel<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(x, v);
  return check_launch("add_scalar_kernel");
}

int ptycho_sgd_step(float* param, const float* grad, int64_t count, float lr, const float* lr_dev,
                    float weight_decay, void* stream) {
  if (!param || !grad || count < 0) return fail(PTYCHO_ERR_INVALID, "sgd: bad arguments");
  if (count == 0) return PTYCHO_OK;
  sgd_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(param, grad, count, lr, lr_dev,
                                                                                   weight_decay);
  return check_launch("sgd_kernel");
}

int ptycho_adam_amsgrad_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq,
                             float* max_exp_avg_sq, int64_t count, float lr, const float* lr_dev, float beta1,
                             float beta2, float eps, float weight_decay, int decoupled, float bc1, float bc2_sqrt,
                             void* stream) {
  if (!param || !grad || !exp_avg || !exp_avg_sq || !max_exp_avg_sq || count < 0)
    return fail(PTYCHO_ERR_INVALID, "adam_amsgrad: bad arguments");
  if (count == 0) return PTYCHO_OK;
  adam_amsgrad_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      param, grad, exp_avg, exp_avg_sq, max_exp_avg_sq, count, lr, lr_dev, beta1, beta2, eps, weight_decay, decoupled,
      bc1, bc2_sqrt);
  return check_launch("adam_amsgrad_kernel");
}

int ptycho_sgd_momentum_step(float* param, const float* grad, float* momentum_buffer, int64_t count, float lr,
                             const float* lr_dev, float weight_decay, float momentum, float dampening, int nesterov,
                             int first_step, void* stream) {
  if (!param || !grad || !momentum_buffer || count < 0) return fail(PTYCHO_ERR_INVALID, "sgd_momentum: bad arguments");
  if (count == 0) return PTYCHO_OK;
  sgd_momentum_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      param, grad, momentum_buffer, count, lr, lr_dev, weight_decay, momentum, dampening, nesterov, first_step);
  return check_launch("sgd_momentum_kernel");
}

}  // extern "C"
