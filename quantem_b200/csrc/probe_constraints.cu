// Optional probe constraints (reference: ProbeConstraints, probe_models.py:430-482):
//
// * centre of mass (`center_probe`, probe_models.py:467-482): per mode, the centre of
//   mass of |psi|^2 on the fftshifted grid minus n / 2, and the mode Fourier-shifted by
//   minus that offset (fourier_shift_expand, ptycho_utils.py:128-139): out =
//   ifft2(fft2(psi) exp(2 pi i (k_r c_r + k_c c_c))) with k = fftfreq(n) in float32
//   (ptycho_utils.py:166-170).  An unshifted row y sits at (y + n / 2) mod n after the
//   fftshift.  The gradient adds to the adjoint of the fixed shift
//   (ifft2(fft2(g) conj(ramp))) the path through the centre of mass: dL/dc =
//   Re (1 / n^2) sum_k conj(fft2(g)) spec 2 pi i k, and dc/d|psi|^2 = (w - n / 2 - c) /
//   sum |psi|^2 with d|psi|^2 -> 2 psi (torch's complex-gradient convention).
// * total variation (`tv_weight`, probe_models.py:460-466): weight x (mean |diff along
//   columns| + mean |diff along rows|) over all modes, gradient d / |d| (0 at d = 0).
//
// The probe stack is small (P <= 16 modes of n^2 <= 256^2), so the centre-of-mass
// reductions run one 1024-thread CTA per mode in float64 (fixed order, deterministic);
// the transforms are the library's batched 2-D FFTs.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include "ptycho_b200.h"

int qb_record_error(int code, const char* msg);

namespace {

constexpr int kThreads = 1024;
constexpr int kTvBlocks = 296;  // 2 x 148 SMs
constexpr int kTvThreads = 256;
constexpr int kMaxModes = 16;

int fail(int code, const char* fmt, ...) {
  char buf[400];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return qb_record_error(code, buf);
}

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PTYCHO_OK : fail(PTYCHO_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// block sum of three doubles, the result in every thread (fixed order)
__device__ double3 block_sum3(double a, double b, double c, double3* red) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = make_double3(a, b, c);
  __syncthreads();
  double3 s = make_double3(0.0, 0.0, 0.0);
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
    s.x += red[i].x;
    s.y += red[i].y;
    s.z += red[i].z;
  }
  return s;
}

__device__ __forceinline__ float fftfreq_f(int k, int n) {  // numpy fftfreq(n)[k] rounded to float32
  return (float)((double)(k < (n + 1) / 2 ? k : k - n) / (double)n);
}

// meta[p] = (c_r, c_c, sum |psi|^2) of mode p
__global__ void __launch_bounds__(kThreads) probe_com_kernel(const float2* __restrict__ probe, int n,
                                                             double* __restrict__ meta) {
  __shared__ double3 red[kThreads / 32];
  const int p = blockIdx.x;
  const int64_t nn = (int64_t)n * n;
  const float2* x = probe + (int64_t)p * nn;
  double t = 0.0, sr = 0.0, sc = 0.0;
  for (int64_t i = threadIdx.x; i < nn; i += kThreads) {
    const int r = (int)(i / n), c = (int)(i % n);
    const double v = (double)x[i].x * x[i].x + (double)x[i].y * x[i].y;
    t += v;
    sr += v * (double)((r + n / 2) % n);
    sc += v * (double)((c + n / 2) % n);
  }
  const double3 s = block_sum3(t, sr, sc, red);
  if (threadIdx.x == 0) {
    meta[3 * p + 0] = s.y / s.x - (double)(n / 2);
    meta[3 * p + 1] = s.z / s.x - (double)(n / 2);
    meta[3 * p + 2] = s.x;
  }
}

// the shift ramp exp(2 pi i (k_r c_r + k_c c_c)) of mode p at (r, c), phases in float32
// like the reference's complex64 ramp
__device__ __forceinline__ float2 shift_ramp(const double* meta, int p, int r, int c, int n) {
  const float cr = (float)meta[3 * p], cc = (float)meta[3 * p + 1];
  float sr, crs, sc, ccs;
  sincospif(2.0f * fftfreq_f(r, n) * cr, &sr, &crs);
  sincospif(2.0f * fftfreq_f(c, n) * cc, &sc, &ccs);
  return make_float2(crs * ccs - sr * sc, crs * sc + sr * ccs);
}

__global__ void probe_ramp_kernel(float2* __restrict__ spec, int P, int n, const double* __restrict__ meta) {
  const int64_t nn = (int64_t)n * n, total = (int64_t)P * nn;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(i / nn);
    const int64_t k = i % nn;
    const float2 e = shift_ramp(meta, p, (int)(k / n), (int)(k % n), n);
    const float2 v = spec[i];
    spec[i] = make_float2(v.x * e.x - v.y * e.y, v.x * e.y + v.y * e.x);
  }
}

// per mode: dL/dc = Re (2 pi i / n^2) sum_k conj(G) spec k, then G *= conj(ramp) in place
__global__ void __launch_bounds__(kThreads) probe_center_dcom_kernel(float2* __restrict__ G,
                                                                     const float2* __restrict__ spec, int n,
                                                                     double* __restrict__ meta) {
  __shared__ double3 red[kThreads / 32];
  const int p = blockIdx.x;
  const int64_t nn = (int64_t)n * n;
  float2* g = G + (int64_t)p * nn;
  const float2* sp = spec + (int64_t)p * nn;
  double ar = 0.0, ac = 0.0;
  for (int64_t i = threadIdx.x; i < nn; i += kThreads) {
    const int r = (int)(i / n), c = (int)(i % n);
    // Re(i conj(G) S) = -Im(conj(G) S) = -(G.x S.y - G.y S.x)
    const double im = (double)g[i].x * sp[i].y - (double)g[i].y * sp[i].x;
    ar -= im * (double)fftfreq_f(r, n);
    ac -= im * (double)fftfreq_f(c, n);
  }
  const double3 s = block_sum3(ar, ac, 0.0, red);
  if (threadIdx.x == 0) {
    const double k = 6.283185307179586 / (double)nn;
    meta[3 * (kMaxModes + p) + 0] = k * s.x;
    meta[3 * (kMaxModes + p) + 1] = k * s.y;
  }
  for (int64_t i = threadIdx.x; i < nn; i += kThreads) {  // each thread rewrites only what it read
    const float2 e = shift_ramp(meta, p, (int)(i / n), (int)(i % n), n);
    const float2 v = g[i];
    g[i] = make_float2(v.x * e.x + v.y * e.y, v.y * e.x - v.x * e.y);  // v conj(e)
  }
}

__global__ void probe_center_finish_kernel(const float2* __restrict__ probe, float2* __restrict__ grad, int P, int n,
                                           const double* __restrict__ meta) {
  const int64_t nn = (int64_t)n * n, total = (int64_t)P * nn;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(i / nn);
    const int64_t k = i % nn;
    const int r = (int)(k / n), c = (int)(k % n);
    const double cr = meta[3 * p], cc = meta[3 * p + 1], tot = meta[3 * p + 2];
    const double dr = meta[3 * (kMaxModes + p)], dc = meta[3 * (kMaxModes + p) + 1];
    const double f = 2.0 * (dr * ((double)((r + n / 2) % n) - (double)(n / 2) - cr) +
                            dc * ((double)((c + n / 2) % n) - (double)(n / 2) - cc)) / tot;
    const float2 x = probe[i], g = grad[i];
    grad[i] = make_float2(g.x + (float)(f * x.x), g.y + (float)(f * x.y));
  }
}

__device__ __forceinline__ float2 unit_or_zero(float2 d) {
  const float a = sqrtf(d.x * d.x + d.y * d.y);
  return a > 0.f ? make_float2(d.x / a, d.y / a) : make_float2(0.f, 0.f);
}

// per-block partial of scale * sum (|d_col| + |d_row|); with grad, the gradient
// scale * (u_col(i-1) - u_col(i) + u_row(i-n) - u_row(i)), u = d / |d|
__global__ void __launch_bounds__(kTvThreads) probe_tv_kernel(const float2* __restrict__ x, int P, int n, float scale,
                                                              double* __restrict__ parts, float2* __restrict__ grad) {
  __shared__ double3 red[kTvThreads / 32];
  const int64_t nn = (int64_t)n * n, total = (int64_t)P * nn;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = i % nn;
    const int r = (int)(k / n), c = (int)(k % n);
    const float2 v = x[i];
    float2 gc = make_float2(0.f, 0.f);
    if (c < n - 1) {
      const float2 d = make_float2(x[i + 1].x - v.x, x[i + 1].y - v.y);
      acc += sqrt((double)d.x * d.x + (double)d.y * d.y);
      const float2 u = unit_or_zero(d);
      gc.x -= u.x;
      gc.y -= u.y;
    }
    if (r < n - 1) {
      const float2 d = make_float2(x[i + n].x - v.x, x[i + n].y - v.y);
      acc += sqrt((double)d.x * d.x + (double)d.y * d.y);
      const float2 u = unit_or_zero(d);
      gc.x -= u.x;
      gc.y -= u.y;
    }
    if (grad) {
      if (c > 0) {
        const float2 u = unit_or_zero(make_float2(v.x - x[i - 1].x, v.y - x[i - 1].y));
        gc.x += u.x;
        gc.y += u.y;
      }
      if (r > 0) {
        const float2 u = unit_or_zero(make_float2(v.x - x[i - n].x, v.y - x[i - n].y));
        gc.x += u.x;
        gc.y += u.y;
      }
      grad[i] = make_float2(scale * gc.x, scale * gc.y);
    }
  }
  const double3 s = block_sum3(acc, 0.0, 0.0, red);
  if (threadIdx.x == 0) parts[blockIdx.x] = (double)scale * s.x;
}

bool valid_n(int n) { return n == 64 || n == 96 || n == 128 || n == 256; }

}  // namespace

extern "C" {

int ptycho_fft2(const void* in, void* out, int count, int n, int inverse, float scale, void* stream);
int ptycho_reduce_loss(const double* parts, int nparts, float* out, void* stream);

int64_t ptycho_probe_center_work_elems(int P, int n) {
  // spectrum (P n^2) + fft2(g) scratch (P n^2) + float64 meta: (c_r, c_c, sum |psi|^2) and
  // (dL/dc_r, dL/dc_c, unused) per mode, 6 kMaxModes doubles = 6 kMaxModes float2 slots
  return 2 * (int64_t)P * n * n + 6 * kMaxModes;
}

int ptycho_probe_center(const void* probe, void* out, int P, int n, void* work, int64_t work_elems, void* stream) {
  if (!probe || !out || !work || P < 1 || P > kMaxModes)
    return fail(PTYCHO_ERR_INVALID, "probe_center: bad arguments (1 <= P <= %d)", kMaxModes);
  if (!valid_n(n)) return fail(PTYCHO_ERR_UNSUPPORTED, "probe_center: n=%d not built", n);
  if (work_elems < ptycho_probe_center_work_elems(P, n))
    return fail(PTYCHO_ERR_INVALID, "probe_center: work needs %lld complex elements",
                (long long)ptycho_probe_center_work_elems(P, n));
  if (probe == out || out == work) return fail(PTYCHO_ERR_INVALID, "probe_center: out must not alias probe or work");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t pn = (int64_t)P * n * n;
  float2* spec = static_cast<float2*>(work);
  double* meta = reinterpret_cast<double*>(spec + 2 * pn);
  probe_com_kernel<<<P, kThreads, 0, st>>>(static_cast<const float2*>(probe), n, meta);
  int rc = check_launch("probe_com_kernel");
  if (rc) return rc;
  if ((rc = ptycho_fft2(probe, spec, P, n, 0, 1.0f, stream))) return rc;
  probe_ramp_kernel<<<148, 256, 0, st>>>(spec, P, n, meta);
  if ((rc = check_launch("probe_ramp_kernel"))) return rc;
  return ptycho_fft2(spec, out, P, n, 1, 1.0f / (float)((int64_t)n * n), stream);
}

int ptycho_probe_center_vjp(const void* probe, const void* grad_out, void* grad_probe, int P, int n, void* work,
                            int64_t work_elems, void* stream) {
  if (!probe || !grad_out || !grad_probe || !work || P < 1 || P > kMaxModes)
    return fail(PTYCHO_ERR_INVALID, "probe_center_vjp: bad arguments (1 <= P <= %d)", kMaxModes);
  if (!valid_n(n)) return fail(PTYCHO_ERR_UNSUPPORTED, "probe_center_vjp: n=%d not built", n);
  if (work_elems < ptycho_probe_center_work_elems(P, n))
    return fail(PTYCHO_ERR_INVALID, "probe_center_vjp: work needs %lld complex elements",
                (long long)ptycho_probe_center_work_elems(P, n));
  if (grad_probe == probe || grad_probe == work)
    return fail(PTYCHO_ERR_INVALID, "probe_center_vjp: grad_probe must not alias probe or work");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t pn = (int64_t)P * n * n;
  float2* spec = static_cast<float2*>(work);
  float2* G = spec + pn;
  double* meta = reinterpret_cast<double*>(spec + 2 * pn);
  int rc = ptycho_fft2(grad_out, G, P, n, 0, 1.0f, stream);
  if (rc) return rc;
  probe_center_dcom_kernel<<<P, kThreads, 0, st>>>(G, spec, n, meta);
  if ((rc = check_launch("probe_center_dcom_kernel"))) return rc;
  if ((rc = ptycho_fft2(G, grad_probe, P, n, 1, 1.0f / (float)((int64_t)n * n), stream))) return rc;
  probe_center_finish_kernel<<<148, 256, 0, st>>>(static_cast<const float2*>(probe), static_cast<float2*>(grad_probe),
                                                  P, n, meta);
  return check_launch("probe_center_finish_kernel");
}

int ptycho_probe_tv_work_elems(void) { return kTvBlocks; }

int ptycho_probe_tv(const void* probe, int P, int n, float weight, float* loss, void* grad, double* work, int nwork,
                    void* stream) {
  if (!probe || !loss || !work || P < 1 || n < 2) return fail(PTYCHO_ERR_INVALID, "probe_tv: bad arguments");
  if (nwork < kTvBlocks) return fail(PTYCHO_ERR_INVALID, "probe_tv: work needs %d doubles", kTvBlocks);
  if (grad == probe) return fail(PTYCHO_ERR_INVALID, "probe_tv: grad must not alias probe");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // both axes hold P n (n - 1) differences
  const float scale = weight / (float)((double)P * n * (n - 1));
  probe_tv_kernel<<<kTvBlocks, kTvThreads, 0, st>>>(static_cast<const float2*>(probe), P, n, scale, work,
                                                     static_cast<float2*>(grad));
  const int rc = check_launch("probe_tv_kernel");
  if (rc) return rc;
  return ptycho_reduce_loss(work, kTvBlocks, loss, stream);
}

}  // extern "C"
