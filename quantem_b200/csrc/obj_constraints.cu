// Optional object constraints of the reference's object model and the probe-overlap
// FOV mask they use (object_models.py:273-480, ptychography_base.py:191-216):
//
//  * probe overlap: sum over positions of |probe mode 0|^2 placed at each patch window;
//  * hard constraint with the FOV mask (apply_fov_mask): complex / pure-phase objects
//    amp m exp(i (angle - mean angle) m) m, potentials (V - offset)+ m, the potential's
//    baseline offset taken from the mask's background (fix_potential_baseline);
//  * exp(i V) of a (filtered) potential;
//  * Gaussian blur (gaussian_sigma): zero-padded separable correlation, self-adjoint;
//  * identical slices: every slice replaced by the slice mean;
//  * soft constraints: TV of phase / amplitude / potential along z and in-plane, and the
//    surface-zero terms of the first and last slices, with their gradients.
//
// Every pass is an HBM-bound elementwise or stencil sweep over the (S, Ho, Wo) object;
// reductions go through fixed-order per-block partials, so every result repeats bit for bit.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "ptycho_b200.h"

int qb_record_error(int code, const char* msg);

namespace {

constexpr int kBlocks = 296;  // 2 x 148 SMs
constexpr int kThreads = 256;

__device__ __forceinline__ double block_sum_d(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;  // valid in thread 0
}

// fixed-order sum of n partials, broadcast to the whole block
__device__ __forceinline__ double partials_sum(const double* part, int n) {
  __shared__ double red[32];
  __shared__ double bc;
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
  const double t = block_sum_d(v, red);
  if (threadIdx.x == 0) bc = t;
  __syncthreads();
  return bc;
}

__device__ __forceinline__ int wrapi(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

__device__ __forceinline__ float sgnf(float x) { return (x > 0.f) - (x < 0.f); }

// ------------------------------------------------------------------ probe overlap
__global__ void probe_overlap_kernel(const float* __restrict__ inten, int n, const float* __restrict__ pos, int npos,
                                     int Ho, int Wo, float* __restrict__ out) {
  const int64_t nn = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn * npos; t += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / nn);
    const int k = (int)(t % nn);
    const int i = k / n, j = k % n;
    const int fi = i < (n + 1) / 2 ? i : i - n, fj = j < (n + 1) / 2 ? j : j - n;  // fftfreq index
    const int r = wrapi((int)rintf(pos[2 * b]) + fi, Ho);
    const int c = wrapi((int)rintf(pos[2 * b + 1]) + fj, Wo);
    atomicAdd(out + (int64_t)r * Wo + c, inten[k]);
  }
}

// ------------------------------------------------- hard constraint with the FOV mask
// work layout (doubles): [0, kBlocks) angle partials, [kBlocks, 2 kBlocks) gradient partials
__global__ void angle_partials_kernel(const float2* __restrict__ obj, int64_t n, double* part) {
  __shared__ double red[32];
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 o = obj[i];
    v += (double)atan2f(o.y, o.x);
  }
  const double t = block_sum_d(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// out = A exp(i theta m), A = amp m^2, theta = angle - mean angle (PURE: amp = 1)
template <bool PURE>
__global__ void fov_apply_kernel(const float2* __restrict__ obj, const float* __restrict__ mask, int64_t hw,
                                 float2* __restrict__ out, int64_t n, const double* part) {
  const float mean = (float)(partials_sum(part, kBlocks) / (double)n);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 o = obj[i];
    const float m = mask[i % hw];
    const float amp = PURE ? 1.0f : fminf(fmaxf(hypotf(o.x, o.y), 0.0f), 1.0f);
    const float A = amp * m * m;
    float s, c;
    sincosf((atan2f(o.y, o.x) - mean) * m, &s, &c);
    out[i] = make_float2(A * c, A * s);
  }
}

// g_theta = m A Im(conj(e) G), summed for the mean-phase term
template <bool PURE>
__global__ void fov_vjp_partials_kernel(const float2* __restrict__ obj, const float* __restrict__ mask, int64_t hw,
                                        const float2* __restrict__ g, int64_t n, const double* part_fwd,
                                        double* part) {
  __shared__ double red[32];
  const float mean = (float)(partials_sum(part_fwd, kBlocks) / (double)n);
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 o = obj[i], gg = g[i];
    const float m = mask[i % hw];
    const float amp = PURE ? 1.0f : fminf(fmaxf(hypotf(o.x, o.y), 0.0f), 1.0f);
    float s, c;
    sincosf((atan2f(o.y, o.x) - mean) * m, &s, &c);
    v += (double)(m * amp * m * m * (gg.y * c - gg.x * s));
  }
  const double t = block_sum_d(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <bool PURE>
__global__ void fov_vjp_apply_kernel(const float2* __restrict__ obj, const float* __restrict__ mask, int64_t hw,
                                     const float2* __restrict__ g, float2* __restrict__ gout, int64_t n,
                                     const double* part_fwd, const double* part_g) {
  const float mean = (float)(partials_sum(part_fwd, kBlocks) / (double)n);
  __syncthreads();
  const float gmean = (float)(partials_sum(part_g, kBlocks) / (double)n);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 o = obj[i], gg = g[i];
    const float m = mask[i % hw];
    const float mag = hypotf(o.x, o.y);
    const float amp = PURE ? 1.0f : fminf(fmaxf(mag, 0.0f), 1.0f);
    float s, c;
    sincosf((atan2f(o.y, o.x) - mean) * m, &s, &c);
    const float g_amp = m * m * (gg.x * c + gg.y * s);               // Re(conj(e) G) m^2
    const float g_ph = m * amp * m * m * (gg.y * c - gg.x * s) - gmean;  // mean-removed g_theta
    const float g_mag = (!PURE && mag >= 0.0f && mag <= 1.0f) ? g_amp : 0.0f;
    float2 r = make_float2(0.f, 0.f);
    if (mag != 0.0f) {
      const float inv = 1.0f / mag;
      r.x = g_mag * o.x * inv - g_ph * o.y * inv * inv;
      r.y = g_mag * o.y * inv + g_ph * o.x * inv * inv;
    }
    gout[i] = r;
  }
}

// ------------------------------------------------------------- potential base
// work layout: [0, kB) max of the mask (per block), [kB, 2kB) background sums,
// [2kB, 3kB) background counts, [3kB, 4kB) minima of V
__global__ void mask_max_kernel(const float* __restrict__ mask, int64_t hw, double* part) {
  __shared__ float red[32];
  float m = -INFINITY;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < hw; i += (int64_t)gridDim.x * blockDim.x)
    m = fmaxf(m, mask[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
    part[blockIdx.x] = (double)fmaxf(m, red[0]);
  }
}

__device__ __forceinline__ float partials_max(const double* part, int n) {
  __shared__ float bc;
  if (threadIdx.x == 0) {
    double m = part[0];
    for (int i = 1; i < n; ++i) m = fmax(m, part[i]);
    bc = (float)m;
  }
  __syncthreads();
  return bc;
}

__global__ void background_stats_kernel(const float* __restrict__ v, const float* __restrict__ mask, int64_t hw,
                                        int64_t n, double* work) {
  __shared__ double red[32];
  __shared__ float redm[32];
  const float mmax = mask ? partials_max(work, kBlocks) : 0.0f;
  double sum = 0.0, cnt = 0.0;
  float mn = INFINITY;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float x = v[i];
    mn = fminf(mn, x);
    if (mask && mask[i % hw] < 0.5f * mmax) {
      sum += (double)x;
      cnt += 1.0;
    }
  }
  const double ts = block_sum_d(sum, red);
  const double tc = block_sum_d(cnt, red);
  for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  if ((threadIdx.x & 31) == 0) redm[threadIdx.x >> 5] = mn;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mn = fminf(mn, redm[w]);
    work[kBlocks + blockIdx.x] = ts;
    work[2 * kBlocks + blockIdx.x] = tc;
    work[3 * kBlocks + blockIdx.x] = (double)fminf(mn, redm[0]);
  }
}

// offset = factor * (mean of V over the background, or min V without one); 0 when not fixed
__device__ __forceinline__ float potential_offset_bg(const double* work, int fix, float factor) {
  if (!fix) return 0.0f;
  const double s = partials_sum(work + kBlocks, kBlocks);
  __syncthreads();
  const double c = partials_sum(work + 2 * kBlocks, kBlocks);
  __shared__ float bc;
  if (threadIdx.x == 0) {
    double off;
    if (c > 0.0) {
      off = (double)(float)(s / c);
    } else {
      double m = work[3 * kBlocks];
      for (int i = 1; i < kBlocks; ++i) m = fmin(m, work[3 * kBlocks + i]);
      off = m;
    }
    bc = (float)off * factor;
  }
  __syncthreads();
  return bc;
}

__global__ void potential_base_kernel(const float* __restrict__ v, const float* __restrict__ mask, int64_t hw,
                                      float* __restrict__ out, int64_t n, int positivity, int fix, float factor,
                                      const double* work) {
  const float off = potential_offset_bg(work, fix, factor);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x = v[i] - off;
    if (positivity) x = fmaxf(x, 0.0f);
    out[i] = mask ? x * mask[i % hw] : x;
  }
}

// the offset is detached (as in the reference); the clamp passes where V - offset >= 0
__global__ void potential_base_vjp_kernel(const float* __restrict__ v, const float* __restrict__ mask, int64_t hw,
                                          const float* __restrict__ g, float* __restrict__ gout, int64_t n,
                                          int positivity, int fix, float factor, const double* work) {
  const float off = potential_offset_bg(work, fix, factor);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float x = v[i] - off;
    const bool pass = !positivity || x >= 0.0f;
    gout[i] = pass ? (mask ? g[i] * mask[i % hw] : g[i]) : 0.0f;
  }
}

// ------------------------------------------------------------------ exp(i V)
__global__ void phase_exp_kernel(const float* __restrict__ v, float2* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float s, c;
    sincosf(v[i], &s, &c);
    out[i] = make_float2(c, s);
  }
}

__global__ void phase_exp_vjp_kernel(const float* __restrict__ v, const float2* __restrict__ g, float* __restrict__ gout,
                                     int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float s, c;
    sincosf(v[i], &s, &c);
    gout[i] = g[i].y * c - g[i].x * s;  // Re(conj(G) i t)
  }
}

// --------------------------------------------------------------- Gaussian blur
// out[s, r, c, k] = sum_t taps[t] in[s, r + t - R, c, k] (AXIS 0) or along c (AXIS 1),
// zero outside; K floats per element (1 real, 2 complex)
template <int AXIS>
__global__ void blur_pass_kernel(const float* __restrict__ in, float* __restrict__ out, int S, int Ho, int Wo, int K,
                                 const float* __restrict__ taps, int ntaps) {
  __shared__ float st[256];
  for (int t = threadIdx.x; t < ntaps; t += blockDim.x) st[t] = taps[t];
  __syncthreads();
  const int R = ntaps / 2;
  const int64_t rowlen = (int64_t)Wo * K;
  const int64_t n = (int64_t)S * Ho * rowlen;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t plane = i / ((int64_t)Ho * rowlen);
    const int64_t rem = i % ((int64_t)Ho * rowlen);
    const int r = (int)(rem / rowlen);
    const int64_t ck = rem % rowlen;
    const int c = (int)(ck / K);
    const int k = (int)(ck % K);
    const float* base = in + plane * Ho * rowlen;
    float acc = 0.f;
    if (AXIS == 0) {
      for (int t = 0; t < ntaps; ++t) {
        const int rr = r + t - R;
        if (rr >= 0 && rr < Ho) acc = fmaf(st[t], base[(int64_t)rr * rowlen + ck], acc);
      }
    } else {
      for (int t = 0; t < ntaps; ++t) {
        const int cc = c + t - R;
        if (cc >= 0 && cc < Wo) acc = fmaf(st[t], base[(int64_t)r * rowlen + (int64_t)cc * K + k], acc);
      }
    }
    out[i] = acc;
  }
}

// ------------------------------------------------------------- identical slices
__global__ void slice_mean_kernel(const float* __restrict__ in, float* __restrict__ out, int S, int64_t plane) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < plane; p += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int s = 0; s < S; ++s) acc += (double)in[(int64_t)s * plane + p];
    const float m = (float)(acc / (double)S);
    for (int s = 0; s < S; ++s) out[(int64_t)s * plane + p] = m;
  }
}

// ------------------------------------------------------------ soft constraints
// KIND 0: complex (phase and amplitude terms), 1: pure phase (phase terms), 2: real potential.
// work: [0, kB) loss partials, [kB, 2kB) / [2kB, 3kB) sum |phase| of the first / last slice,
// [3kB, 4kB) / [4kB, 5kB) sum sign(u) of the first / last slice
template <int KIND>
__device__ __forceinline__ void values_at(const float* obj, int64_t i, float& ph, float& amp) {
  if (KIND == 2) {
    ph = obj[i];
    amp = 0.f;
  } else {
    const float2 o = reinterpret_cast<const float2*>(obj)[i];
    ph = atan2f(o.y, o.x);
    amp = hypotf(o.x, o.y);
  }
}

template <int KIND>
__global__ void surface_abs_phase_kernel(const float* __restrict__ obj, int S, int64_t hw, double* work) {
  __shared__ double red[32];
  double a0 = 0.0, a1 = 0.0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < hw; p += (int64_t)gridDim.x * blockDim.x) {
    float ph, amp;
    values_at<KIND>(obj, p, ph, amp);
    a0 += fabsf(ph);
    values_at<KIND>(obj, (int64_t)(S - 1) * hw + p, ph, amp);
    a1 += fabsf(ph);
  }
  const double t0 = block_sum_d(a0, red);
  const double t1 = block_sum_d(a1, red);
  if (threadIdx.x == 0) {
    work[kBlocks + blockIdx.x] = t0;
    work[2 * kBlocks + blockIdx.x] = t1;
  }
}

template <int KIND>
__global__ void surface_sign_kernel(const float* __restrict__ obj, int S, int64_t hw, double* work) {
  __shared__ double red[32];
  const float m0 = (float)(partials_sum(work + kBlocks, kBlocks) / (double)hw);
  __syncthreads();
  const float m1 = (float)(partials_sum(work + 2 * kBlocks, kBlocks) / (double)hw);
  double a0 = 0.0, a1 = 0.0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < hw; p += (int64_t)gridDim.x * blockDim.x) {
    float ph, amp;
    values_at<KIND>(obj, p, ph, amp);
    a0 += sgnf(fabsf(ph) - m0);
    values_at<KIND>(obj, (int64_t)(S - 1) * hw + p, ph, amp);
    a1 += sgnf(fabsf(ph) - m1);
  }
  const double t0 = block_sum_d(a0, red);
  const double t1 = block_sum_d(a1, red);
  if (threadIdx.x == 0) {
    work[3 * kBlocks + blockIdx.x] = t0;
    work[4 * kBlocks + blockIdx.x] = t1;
  }
}

template <int KIND>
__global__ void soft_loss_kernel(const float* __restrict__ obj, int S, int Ho, int Wo, float wz, float wxy,
                                 float wsurf, float* __restrict__ grad, double* work) {
  __shared__ double red[32];
  const int64_t hw = (int64_t)Ho * Wo, n = (int64_t)S * hw;
  const bool surf = wsurf > 0.f && S >= 3;
  float m0 = 0.f, m1 = 0.f, sg0 = 0.f, sg1 = 0.f;
  if (surf && KIND != 2) {
    m0 = (float)(partials_sum(work + kBlocks, kBlocks) / (double)hw);
    __syncthreads();
    m1 = (float)(partials_sum(work + 2 * kBlocks, kBlocks) / (double)hw);
    __syncthreads();
    sg0 = (float)(partials_sum(work + 3 * kBlocks, kBlocks) / (double)hw);
    __syncthreads();
    sg1 = (float)(partials_sum(work + 4 * kBlocks, kBlocks) / (double)hw);
  }
  // weighted dimensions (object_models.py:398-411): z with wz (3-D arrays, S > 1), rows and
  // columns with wxy; each term w mean|diff| divided by the number of weighted dimensions
  const float w0 = S > 1 ? wz : 0.f;
  const int nd = (w0 > 0.f) + 2 * (wxy > 0.f);
  const float c0 = nd && w0 > 0.f ? w0 / (nd * (float)((int64_t)(S - 1) * hw)) : 0.f;
  const float c1 = nd && wxy > 0.f ? wxy / (nd * (float)((int64_t)S * (Ho - 1) * Wo)) : 0.f;
  const float c2 = nd && wxy > 0.f ? wxy / (nd * (float)((int64_t)S * Ho * (Wo - 1))) : 0.f;
  const bool amp_terms = KIND == 0;
  double lacc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / hw);
    const int64_t p = i % hw;
    const int r = (int)(p / Wo), c = (int)(p % Wo);
    float ph, amp;
    values_at<KIND>(obj, i, ph, amp);
    float gph = 0.f, gamp = 0.f;
    // one stencil step per weighted dimension: the loss term of the diff to the next element,
    // the gradient from the diffs on both sides
    auto tv_dim = [&](float cw, bool has_lo, int64_t lo, bool has_hi, int64_t hi) {
      if (cw == 0.f) return;
      float q, qa;
      if (has_hi) {
        values_at<KIND>(obj, hi, q, qa);
        const float d = q - ph;
        lacc += (double)(cw * fabsf(d));
        gph -= cw * sgnf(d);
        if (amp_terms) {
          const float da = qa - amp;
          lacc += (double)(cw * fabsf(da));
          gamp -= cw * sgnf(da);
        }
      }
      if (has_lo) {
        values_at<KIND>(obj, lo, q, qa);
        gph += cw * sgnf(ph - q);
        if (amp_terms) gamp += cw * sgnf(amp - qa);
      }
    };
    tv_dim(c0, s > 0, i - hw, s < S - 1, i + hw);
    tv_dim(c1, r > 0, i - Wo, r < Ho - 1, i + Wo);
    tv_dim(c2, c > 0, i - 1, c < Wo - 1, i + 1);
    if (surf && (s == 0 || s == S - 1)) {
      const float inv = 1.0f / (float)hw;
      if (KIND == 2) {
        lacc += (double)(wsurf * fabsf(ph) * inv);
        gph += wsurf * sgnf(ph) * inv;
      } else {
        const float m = s == 0 ? m0 : m1, sgm = s == 0 ? sg0 : sg1;
        const float u = fabsf(ph) - m;
        lacc += (double)(wsurf * fabsf(u) * inv);
        gph += wsurf * (sgnf(u) - sgm) * inv * sgnf(ph);
        if (amp_terms) {
          lacc += (double)(wsurf * (1.0f - amp) * inv);
          gamp -= wsurf * inv;
        }
      }
    }
    if (KIND == 2) {
      grad[i] = gph;
    } else {
      const float2 o = reinterpret_cast<const float2*>(obj)[i];
      float2 gz = make_float2(0.f, 0.f);
      if (amp != 0.f) {  // G = g_amp z / |z| + i g_phase z / |z|^2 (zero at a zero pixel)
        const float inv = 1.0f / amp;
        gz.x = gamp * o.x * inv - gph * o.y * inv * inv;
        gz.y = gamp * o.y * inv + gph * o.x * inv * inv;
      }
      reinterpret_cast<float2*>(grad)[i] = gz;
    }
  }
  const double t = block_sum_d(lacc, red);
  if (threadIdx.x == 0) work[blockIdx.x] = t;
}

__global__ void loss_from_partials_kernel(const double* __restrict__ part, float* __restrict__ out) {
  const double t = partials_sum(part, kBlocks);
  if (threadIdx.x == 0) *out = (float)t;
}

int check(const char* what);
int grid_for(int64_t n);

// ---------------------------------------------------------------- Butterworth filter
// object_models.py:481-520: per slice, mean removed, ifft2(fft2(x) env), mean added back.
// The 2-D transform is a direct DFT along the rows, a transpose, a direct DFT along the
// (former) columns and a transpose back: O(H W (H + W)) per slice, exact for any object
// size (no object-sized FFT is built on this path); the twiddles come from a per-line
// table of w^j, j < n, indexed by (k c) mod n.

// per-slice mean of a complex (or real, REAL) plane, one block per slice
template <bool REAL>
__global__ void plane_mean_kernel(const float* __restrict__ in, int64_t hw, float2* __restrict__ means) {
  __shared__ double red[32];
  const int s = blockIdx.x;
  double re = 0.0, im = 0.0;
  for (int64_t p = threadIdx.x; p < hw; p += blockDim.x) {
    if (REAL) {
      re += (double)in[(int64_t)s * hw + p];
    } else {
      const float2 v = reinterpret_cast<const float2*>(in)[(int64_t)s * hw + p];
      re += (double)v.x;
      im += (double)v.y;
    }
  }
  const double tr = block_sum_d(re, red);
  const double ti = block_sum_d(im, red);
  if (threadIdx.x == 0) means[s] = make_float2((float)(tr / (double)hw), (float)(ti / (double)hw));
}

// out (complex) = in - mean of its slice
template <bool REAL>
__global__ void center_kernel(const float* __restrict__ in, int64_t hw, int64_t n, const float2* __restrict__ means,
                              float2* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 m = means[i / hw];
    const float2 v = REAL ? make_float2(in[i], 0.f) : reinterpret_cast<const float2*>(in)[i];
    out[i] = make_float2(v.x - m.x, v.y - m.y);
  }
}

// DFT of every line of length n (lines contiguous): out[l, k] = scale sum_c x[l, c] w^(+-k c)
template <bool INV>
__global__ void dft_lines_kernel(const float2* __restrict__ in, float2* __restrict__ out, int n, float scale) {
  extern __shared__ float2 sh[];
  float2* x = sh;
  float2* tw = sh + n;
  const int64_t line = blockIdx.x;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    x[j] = in[line * n + j];
    double sn, cs;
    sincospi((INV ? 2.0 : -2.0) * (double)j / (double)n, &sn, &cs);
    tw[j] = make_float2((float)cs, (float)sn);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    float ar = 0.f, ai = 0.f;
    int idx = 0;
    for (int c = 0; c < n; ++c) {
      const float2 v = x[c], w = tw[idx];
      ar = fmaf(v.x, w.x, fmaf(-v.y, w.y, ar));
      ai = fmaf(v.x, w.y, fmaf(v.y, w.x, ai));
      idx += k;
      if (idx >= n) idx -= n;
    }
    out[line * n + k] = make_float2(ar * scale, ai * scale);
  }
}

// (S, H, W) -> (S, W, H), 32 x 32 tiles through shared memory
__global__ void transpose_c_kernel(const float2* __restrict__ in, float2* __restrict__ out, int H, int W) {
  __shared__ float2 t[32][33];
  const int64_t s = blockIdx.z;
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int r = r0 + dy, c = c0 + threadIdx.x;
    if (r < H && c < W) t[dy][threadIdx.x] = in[(s * H + r) * W + c];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int c = c0 + dy, r = r0 + threadIdx.x;
    if (r < H && c < W) out[(s * W + c) * H + r] = t[threadIdx.x][dy];
  }
}

// x (S, W, H) transposed spectrum *= env[kh, kw]
__global__ void env_mul_t_kernel(float2* __restrict__ x, const float* __restrict__ env, int H, int W, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i % ((int64_t)H * W);
    const int kw = (int)(p / H), kh = (int)(p % H);
    const float e = env[(int64_t)kh * W + kw];
    x[i] = make_float2(x[i].x * e, x[i].y * e);
  }
}

// out = y + add[slice] - sub[slice] (the real part for REAL): forward y + mean(x), VJP
// y - mean(y) + mean(g)
template <bool REAL>
__global__ void butter_finish_kernel(const float2* __restrict__ y, int64_t hw, int64_t n,
                                     const float2* __restrict__ add, const float2* __restrict__ sub,
                                     float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = i / hw;
    float2 v = y[i];
    v.x += add[s].x - (sub ? sub[s].x : 0.f);
    v.y += add[s].y - (sub ? sub[s].y : 0.f);
    if (REAL)
      out[i] = v.x;
    else
      reinterpret_cast<float2*>(out)[i] = v;
  }
}

// y (in a) = ifft2(env fft2(a)) of (S, H, W) complex planes; b: scratch of the same size
int butter_core(float2* a, float2* b, int S, int H, int W, const float* env, cudaStream_t st) {
  const size_t smw = sizeof(float2) * 2 * (size_t)W, smh = sizeof(float2) * 2 * (size_t)H;
  cudaFuncSetAttribute(dft_lines_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(smw > smh ? smw : smh));
  cudaFuncSetAttribute(dft_lines_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(smw > smh ? smw : smh));
  const dim3 tb(32, 8);
  const dim3 tg_hw((W + 31) / 32, (H + 31) / 32, S), tg_wh((H + 31) / 32, (W + 31) / 32, S);
  const int64_t n = (int64_t)S * H * W;
  dft_lines_kernel<false><<<S * H, kThreads, smw, st>>>(a, b, W, 1.0f);       // along W
  transpose_c_kernel<<<tg_hw, tb, 0, st>>>(b, a, H, W);                     // (S, W, H)
  dft_lines_kernel<false><<<S * W, kThreads, smh, st>>>(a, b, H, 1.0f);       // along H
  env_mul_t_kernel<<<grid_for(n), kThreads, 0, st>>>(b, env, H, W, n);
  dft_lines_kernel<true><<<S * W, kThreads, smh, st>>>(b, a, H, 1.0f / (float)H);
  transpose_c_kernel<<<tg_wh, tb, 0, st>>>(a, b, W, H);                     // (S, H, W)
  dft_lines_kernel<true><<<S * H, kThreads, smw, st>>>(b, a, W, 1.0f / (float)W);
  return check("butterworth dft");
}

int check(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PTYCHO_OK : qb_record_error(PTYCHO_ERR_CUDA, what);
}

int grid_for(int64_t n) {
  const int64_t g = (n + kThreads - 1) / kThreads;
  return (int)(g < kBlocks ? (g < 1 ? 1 : g) : kBlocks);
}

}  // namespace

extern "C" {

int ptycho_obj_constraint_work_elems(void) { return 5 * kBlocks; }

int ptycho_probe_overlap(const float* intensity, int n, const float* positions, int npos, int Ho, int Wo, float* out,
                         void* stream) {
  if (!intensity || !positions || !out || n < 1 || npos < 0 || Ho < 1 || Wo < 1)
    return qb_record_error(PTYCHO_ERR_INVALID, "probe_overlap: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(out, 0, sizeof(float) * (size_t)Ho * Wo, st) != cudaSuccess)
    return qb_record_error(PTYCHO_ERR_CUDA, "probe_overlap: memset");
  if (npos == 0) return PTYCHO_OK;
  probe_overlap_kernel<<<4 * kBlocks, kThreads, 0, st>>>(intensity, n, positions, npos, Ho, Wo, out);
  return check("probe_overlap_kernel");
}

int ptycho_obj_constrain_fov(const void* obj, const float* mask, int64_t hw, void* out, int64_t count, int pure,
                             double* work, int nwork, void* stream) {
  if (!obj || !mask || !out || !work || count < 1 || hw < 1 || count % hw || nwork < 5 * kBlocks)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_constrain_fov: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float2* o = static_cast<const float2*>(obj);
  angle_partials_kernel<<<kBlocks, kThreads, 0, st>>>(o, count, work);
  if (pure)
    fov_apply_kernel<true><<<kBlocks, kThreads, 0, st>>>(o, mask, hw, static_cast<float2*>(out), count, work);
  else
    fov_apply_kernel<false><<<kBlocks, kThreads, 0, st>>>(o, mask, hw, static_cast<float2*>(out), count, work);
  return check("fov_apply_kernel");
}

int ptycho_obj_constrain_fov_vjp(const void* obj, const float* mask, int64_t hw, const void* grad_c, void* grad_raw,
                                 int64_t count, int pure, double* work, int nwork, void* stream) {
  if (!obj || !mask || !grad_c || !grad_raw || !work || count < 1 || hw < 1 || count % hw || nwork < 5 * kBlocks)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_constrain_fov_vjp: bad arguments");
  if (grad_raw == obj || grad_raw == grad_c)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_constrain_fov_vjp: grad_raw aliases an input");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float2* o = static_cast<const float2*>(obj);
  const float2* g = static_cast<const float2*>(grad_c);
  angle_partials_kernel<<<kBlocks, kThreads, 0, st>>>(o, count, work);
  if (pure) {
    fov_vjp_partials_kernel<true><<<kBlocks, kThreads, 0, st>>>(o, mask, hw, g, count, work, work + kBlocks);
    fov_vjp_apply_kernel<true><<<kBlocks, kThreads, 0, st>>>(o, mask, hw, g, static_cast<float2*>(grad_raw), count,
                                                             work, work + kBlocks);
  } else {
    fov_vjp_partials_kernel<false><<<kBlocks, kThreads, 0, st>>>(o, mask, hw, g, count, work, work + kBlocks);
    fov_vjp_apply_kernel<false><<<kBlocks, kThreads, 0, st>>>(o, mask, hw, g, static_cast<float2*>(grad_raw), count,
                                                              work, work + kBlocks);
  }
  return check("fov_vjp_apply_kernel");
}

int ptycho_obj_potential_base(const float* v, const float* baseline_mask, const float* apply_mask, int64_t hw,
                              float* out, int64_t count, int positivity, int fix_baseline, float factor,
                              double* work, int nwork, void* stream) {
  if (!v || !out || !work || count < 1 || hw < 1 || count % hw || nwork < 5 * kBlocks)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_potential_base: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (fix_baseline) {
    if (baseline_mask) mask_max_kernel<<<kBlocks, kThreads, 0, st>>>(baseline_mask, hw, work);
    background_stats_kernel<<<kBlocks, kThreads, 0, st>>>(v, baseline_mask, hw, count, work);
  }
  potential_base_kernel<<<kBlocks, kThreads, 0, st>>>(v, apply_mask, hw, out, count, positivity, fix_baseline, factor,
                                                      work);
  return check("potential_base_kernel");
}

int ptycho_obj_potential_base_vjp(const float* v, const float* baseline_mask, const float* apply_mask, int64_t hw,
                                  const float* grad_out, float* grad_v, int64_t count, int positivity,
                                  int fix_baseline, float factor, double* work, int nwork, void* stream) {
  if (!v || !grad_out || !grad_v || !work || count < 1 || hw < 1 || count % hw || nwork < 5 * kBlocks)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_potential_base_vjp: bad arguments");
  if (grad_v == v) return qb_record_error(PTYCHO_ERR_INVALID, "obj_potential_base_vjp: grad_v aliases v");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (fix_baseline) {
    if (baseline_mask) mask_max_kernel<<<kBlocks, kThreads, 0, st>>>(baseline_mask, hw, work);
    background_stats_kernel<<<kBlocks, kThreads, 0, st>>>(v, baseline_mask, hw, count, work);
  }
  potential_base_vjp_kernel<<<kBlocks, kThreads, 0, st>>>(v, apply_mask, hw, grad_out, grad_v, count, positivity,
                                                          fix_baseline, factor, work);
  return check("potential_base_vjp_kernel");
}

int ptycho_phase_exp(const float* v, void* out, int64_t count, void* stream) {
  if (!v || !out || count < 0) return qb_record_error(PTYCHO_ERR_INVALID, "phase_exp: bad arguments");
  if (count == 0) return PTYCHO_OK;
  phase_exp_kernel<<<grid_for(count), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(v, static_cast<float2*>(out),
                                                                                        count);
  return check("phase_exp_kernel");
}

int ptycho_phase_exp_vjp(const float* v, const void* grad_t, float* grad_v, int64_t count, void* stream) {
  if (!v || !grad_t || !grad_v || count < 0) return qb_record_error(PTYCHO_ERR_INVALID, "phase_exp_vjp: bad arguments");
  if (grad_v == v) return qb_record_error(PTYCHO_ERR_INVALID, "phase_exp_vjp: grad_v aliases v");
  if (count == 0) return PTYCHO_OK;
  phase_exp_vjp_kernel<<<grid_for(count), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      v, static_cast<const float2*>(grad_t), grad_v, count);
  return check("phase_exp_vjp_kernel");
}

int ptycho_obj_blur(const void* in, void* out, void* tmp, int S, int Ho, int Wo, int is_complex, const float* taps,
                    int ntaps, void* stream) {
  if (!in || !out || !tmp || !taps || S < 1 || Ho < 1 || Wo < 1 || ntaps < 1 || ntaps > 255 || ntaps % 2 == 0)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_blur: bad arguments (odd tap count <= 255)");
  if (tmp == in || tmp == out) return qb_record_error(PTYCHO_ERR_INVALID, "obj_blur: tmp aliases in or out");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int K = is_complex ? 2 : 1;
  blur_pass_kernel<0><<<4 * kBlocks, kThreads, 0, st>>>(static_cast<const float*>(in), static_cast<float*>(tmp), S, Ho,
                                                        Wo, K, taps, ntaps);
  blur_pass_kernel<1><<<4 * kBlocks, kThreads, 0, st>>>(static_cast<const float*>(tmp), static_cast<float*>(out), S,
                                                        Ho, Wo, K, taps, ntaps);
  return check("blur_pass_kernel");
}

int ptycho_obj_slice_mean(const void* in, void* out, int S, int64_t hw, int is_complex, void* stream) {
  if (!in || !out || S < 1 || hw < 1) return qb_record_error(PTYCHO_ERR_INVALID, "obj_slice_mean: bad arguments");
  const int64_t plane = hw * (is_complex ? 2 : 1);
  slice_mean_kernel<<<grid_for(plane), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float*>(in), static_cast<float*>(out), S, plane);
  return check("slice_mean_kernel");
}

int ptycho_obj_butterworth(const void* in, void* out, int S, int Ho, int Wo, int is_real, const float* env, void* tmp,
                           void* means, void* stream) {
  if (!in || !out || !env || !tmp || !means || S < 1 || Ho < 1 || Wo < 1 || Ho > 6144 || Wo > 6144)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_butterworth: bad arguments (object sides <= 6144)");
  if (tmp == in || tmp == out) return qb_record_error(PTYCHO_ERR_INVALID, "obj_butterworth: tmp aliases in or out");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t hw = (int64_t)Ho * Wo, n = (int64_t)S * hw;
  float2* a = static_cast<float2*>(tmp);
  float2* b = a + n;
  float2* mu = static_cast<float2*>(means);
  const float* x = static_cast<const float*>(in);
  if (is_real) {
    plane_mean_kernel<true><<<S, kThreads, 0, st>>>(x, hw, mu);
    center_kernel<true><<<grid_for(n), kThreads, 0, st>>>(x, hw, n, mu, a);
  } else {
    plane_mean_kernel<false><<<S, kThreads, 0, st>>>(x, hw, mu);
    center_kernel<false><<<grid_for(n), kThreads, 0, st>>>(x, hw, n, mu, a);
  }
  int rc = butter_core(a, b, S, Ho, Wo, env, st);
  if (rc) return rc;
  if (is_real)
    butter_finish_kernel<true><<<grid_for(n), kThreads, 0, st>>>(a, hw, n, mu, nullptr, static_cast<float*>(out));
  else
    butter_finish_kernel<false><<<grid_for(n), kThreads, 0, st>>>(a, hw, n, mu, nullptr, static_cast<float*>(out));
  return check("butter_finish_kernel");
}

int ptycho_obj_butterworth_vjp(const void* grad_out, void* grad_in, int S, int Ho, int Wo, int is_real,
                               const float* env, void* tmp, void* means, void* stream) {
  if (!grad_out || !grad_in || !env || !tmp || !means || S < 1 || Ho < 1 || Wo < 1 || Ho > 6144 || Wo > 6144)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_butterworth_vjp: bad arguments (object sides <= 6144)");
  if (tmp == grad_out || tmp == grad_in)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_butterworth_vjp: tmp aliases a gradient");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t hw = (int64_t)Ho * Wo, n = (int64_t)S * hw;
  float2* a = static_cast<float2*>(tmp);
  float2* b = a + n;
  float2* mg = static_cast<float2*>(means);  // mean of g
  float2* my = mg + S;                      // mean of P g (zero while g is copied into a)
  const float* g = static_cast<const float*>(grad_out);
  if (cudaMemsetAsync(my, 0, sizeof(float2) * (size_t)S, st) != cudaSuccess)
    return qb_record_error(PTYCHO_ERR_CUDA, "obj_butterworth_vjp: memset");
  if (is_real) {
    plane_mean_kernel<true><<<S, kThreads, 0, st>>>(g, hw, mg);
    center_kernel<true><<<grid_for(n), kThreads, 0, st>>>(g, hw, n, my, a);  // my zeroed below first
  } else {
    plane_mean_kernel<false><<<S, kThreads, 0, st>>>(g, hw, mg);
    center_kernel<false><<<grid_for(n), kThreads, 0, st>>>(g, hw, n, my, a);
  }
  int rc = butter_core(a, b, S, Ho, Wo, env, st);
  if (rc) return rc;
  plane_mean_kernel<false><<<S, kThreads, 0, st>>>(reinterpret_cast<const float*>(a), hw, my);
  if (is_real)
    butter_finish_kernel<true><<<grid_for(n), kThreads, 0, st>>>(a, hw, n, mg, my, static_cast<float*>(grad_in));
  else
    butter_finish_kernel<false><<<grid_for(n), kThreads, 0, st>>>(a, hw, n, mg, my, static_cast<float*>(grad_in));
  return check("butter_finish_kernel");
}

int ptycho_obj_soft_loss(const void* obj, int S, int Ho, int Wo, int kind, float tv_weight_z, float tv_weight_xy,
                         float surface_zero_weight, double* work, int nwork, float* loss, void* grad, void* stream) {
  if (!obj || !work || !loss || !grad || S < 1 || Ho < 2 || Wo < 2 || kind < 0 || kind > 2 || nwork < 5 * kBlocks)
    return qb_record_error(PTYCHO_ERR_INVALID, "obj_soft_loss: bad arguments");
  if (grad == obj) return qb_record_error(PTYCHO_ERR_INVALID, "obj_soft_loss: grad aliases obj");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float* o = static_cast<const float*>(obj);
  float* g = static_cast<float*>(grad);
  const int64_t hw = (int64_t)Ho * Wo;
  const bool surf = surface_zero_weight > 0.f && S >= 3;
  if (kind == 0) {
    if (surf) {
      surface_abs_phase_kernel<0><<<kBlocks, kThreads, 0, st>>>(o, S, hw, work);
      surface_sign_kernel<0><<<kBlocks, kThreads, 0, st>>>(o, S, hw, work);
    }
    soft_loss_kernel<0><<<kBlocks, kThreads, 0, st>>>(o, S, Ho, Wo, tv_weight_z, tv_weight_xy, surface_zero_weight, g,
                                                      work);
  } else if (kind == 1) {
    if (surf) {
      surface_abs_phase_kernel<1><<<kBlocks, kThreads, 0, st>>>(o, S, hw, work);
      surface_sign_kernel<1><<<kBlocks, kThreads, 0, st>>>(o, S, hw, work);
    }
    soft_loss_kernel<1><<<kBlocks, kThreads, 0, st>>>(o, S, Ho, Wo, tv_weight_z, tv_weight_xy, surface_zero_weight, g,
                                                      work);
  } else {
    soft_loss_kernel<2><<<kBlocks, kThreads, 0, st>>>(o, S, Ho, Wo, tv_weight_z, tv_weight_xy, surface_zero_weight, g,
                                                      work);
  }
  loss_from_partials_kernel<<<1, kThreads, 0, st>>>(work, loss);
  return check("soft_loss_kernel");
}

}  // extern "C"
