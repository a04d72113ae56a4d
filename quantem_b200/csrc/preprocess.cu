// Dataset preprocessing on the GPU: centre of mass of every diffraction pattern
// and the normalisation of the measured intensities into corner-centred target
// amplitudes (reference: PtychographyDatasetRaster._set_intensities_com
// dataset_models.py:1027-1112 and _normalize_diffraction_intensities
// dataset_models.py:1372-1480, whose per-position loop Fourier-shifts every
// amplitude by minus its fitted centre of mass, clips at zero and fftshifts).
//
// The Fourier shift itself uses ptycho_fft2 (forward, then these ramps, then the
// inverse); the kernels here are the element-wise and reduction steps around it.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include "ptycho_b200.h"

int qb_record_error(int code, const char* msg);

namespace {

int fail(int code, const char* fmt, ...) {
  char buf[400];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return qb_record_error(code, buf);
}
int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PTYCHO_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return PTYCHO_OK;
}

constexpr int kThreads = 256;
constexpr int kPartBlocks = 592;  // 4 x 148 SMs

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;  // thread 0
}

// com[p] = sum I r / sum I, com[npos + p] = sum I c / sum I (row / column pixel
// indices from 0), I optionally times the detector mask (dataset_models.py:1058-1073).
__global__ void pattern_com_kernel(const float* __restrict__ inten, const float* __restrict__ mask, int npos, int nr,
                                   int nc, double* __restrict__ com) {
  __shared__ double red[32];
  const int64_t nn = (int64_t)nr * nc;
  for (int p = blockIdx.x; p < npos; p += gridDim.x) {
    const float* src = inten + (int64_t)p * nn;
    double s = 0.0, sr = 0.0, sc = 0.0;
    for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) {
      double v = (double)src[i];
      if (mask) v *= (double)mask[i];
      s += v;
      sr += v * (double)(i / nc);
      sc += v * (double)(i % nc);
    }
    const double ts = block_sum(s, red);
    const double tr = block_sum(sr, red);
    const double tc = block_sum(sc, red);
    if (threadIdx.x == 0) {
      com[p] = tr / ts;
      com[npos + p] = tc / ts;
    }
  }
}

// I = max(I, 0); a = sqrt(I); complex copy of a for the Fourier shift; per-block
// partial sums of I and a (fixed order).
__global__ void pattern_prepare_kernel(const float* __restrict__ in, int64_t count, float* __restrict__ iout,
                                       float* __restrict__ aout, float2* __restrict__ ac, double* __restrict__ part) {
  __shared__ double red[32];
  double si = 0.0, sa = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = fmaxf(in[i], 0.0f);
    const float a = sqrtf(v);
    if (iout) iout[i] = v;
    if (aout) aout[i] = a;
    ac[i] = make_float2(a, 0.0f);
    si += v;
    sa += a;
  }
  const double ti = block_sum(si, red);
  const double ta = block_sum(sa, red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = ti;
    part[2 * blockIdx.x + 1] = ta;
  }
}

__global__ void sum_parts_kernel(const double* __restrict__ part, int nparts, double* __restrict__ sums) {
  __shared__ double red[32];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  const double ta = block_sum(a, red);
  const double tb = block_sum(b, red);
  if (threadIdx.x == 0) {
    sums[0] = ta;
    sums[1] = tb;
  }
}

// spec[p][kr][kc] *= exp(-2 pi i (cs_p qc + rs_p qr)), qr = fftfreq(n)[kr], qc = fftfreq(n)[kc]
// (ptycho_utils.py:264-271 with rs, cs the row / column shift of pattern p).
__global__ void pattern_shift_ramp_kernel(float2* __restrict__ spec, const double* __restrict__ shifts, int npos,
                                          int n) {
  const int64_t nn = (int64_t)n * n;
  const int64_t total = (int64_t)npos * nn;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(i / nn);
    const int k = (int)(i % nn);
    const int kr = k / n, kc = k % n;
    const double qr = (double)(kr < (n + 1) / 2 ? kr : kr - n) / n;
    const double qc = (double)(kc < (n + 1) / 2 ? kc : kc - n) / n;
    double s, c;
    sincospi(-2.0 * (shifts[npos + p] * qc + shifts[p] * qr), &s, &c);
    const float2 v = spec[i];
    spec[i] = make_float2((float)(v.x * c - v.y * s), (float)(v.x * s + v.y * c));
  }
}

// centred amplitude = fftshift(max(Re(shifted) * scale, 0)) and its square.
__global__ void pattern_center_kernel(const float2* __restrict__ sh, int npos, int n, float scale,
                                      float* __restrict__ camp, float* __restrict__ cint) {
  const int64_t nn = (int64_t)n * n;
  const int64_t total = (int64_t)npos * nn;
  const int h = n / 2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / nn;
    const int k = (int)(i % nn);
    const int r = k / n, c = k % n;
    const float v = fmaxf(sh[i].x * scale, 0.0f);
    const int64_t d = p * nn + (int64_t)((r + h) % n) * n + (c + h) % n;
    camp[d] = v;
    if (cint) cint[d] = v * v;
  }
}

// Bilinear centring (ptycho_utils.py:273-284 with dataset_models.py:1427-1435): the
// amplitude rolled by floor(shift) and blended with its neighbours one pixel further by the
// fractional parts (periodic), in float64 like the reference's numpy arithmetic, clipped at 0
// and written fftshifted; shifts (2, npos) = (row, column) shift of every pattern.
__global__ void pattern_bilinear_kernel(const float* __restrict__ amp, const double* __restrict__ shifts, int npos,
                                        int n, float* __restrict__ camp, float* __restrict__ cint) {
  const int64_t nn = (int64_t)n * n;
  const int64_t total = (int64_t)npos * nn;
  const int h = n / 2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / nn;
    const int k = (int)(i % nn);
    const int r = k / n, c = k % n;
    const double rs = shifts[p], cs = shifts[npos + p];
    const double rf = floor(rs), cf = floor(cs);
    const double wr = rs - rf, wc = cs - cf;
    const int ir = (int)(((int64_t)rf % n + n) % n), ic = (int)(((int64_t)cf % n + n) % n);
    const int r0 = (r - ir + n) % n, r1 = (r - ir - 1 + 2 * n) % n;
    const int c0 = (c - ic + n) % n, c1 = (c - ic - 1 + 2 * n) % n;
    const float* a = amp + p * nn;
    double v = (double)a[r0 * n + c0] * ((1.0 - wr) * (1.0 - wc));
    v += (double)a[r1 * n + c0] * (wr * (1.0 - wc));
    v += (double)a[r0 * n + c1] * ((1.0 - wr) * wc);
    v += (double)a[r1 * n + c1] * (wr * wc);
    v = v > 0.0 ? v : 0.0;
    const int64_t d = p * nn + (int64_t)((r + h) % n) * n + (c + h) % n;
    camp[d] = (float)v;
    if (cint) cint[d] = (float)(v * v);
  }
}

int blocks_for(int64_t n, int cap = kPartBlocks) {
  int64_t b = (n + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  return (int)(b < cap ? b : cap);
}

}  // namespace

extern "C" {

int ptycho_pattern_com(const float* intensities, const float* mask, int npos, int nr, int nc, double* com,
                       void* stream) {
  if (!intensities || !com || npos < 1 || nr < 1 || nc < 1) return fail(PTYCHO_ERR_INVALID, "pattern_com: bad arguments");
  const int grid = npos < kPartBlocks ? npos : kPartBlocks;
  pattern_com_kernel<<<grid, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(intensities, mask, npos, nr, nc, com);
  return check_launch("pattern_com_kernel");
}

int ptycho_pattern_prepare(const float* intensities, int64_t count, float* intensities_out, float* amplitudes_out,
                           void* amplitudes_c, double* work, int64_t work_elems, double* sums, void* stream) {
  if (!intensities || !amplitudes_c || !work || !sums || count < 1 || work_elems < 2 * kPartBlocks)
    return fail(PTYCHO_ERR_INVALID, "pattern_prepare: bad arguments (work >= %d doubles)", 2 * kPartBlocks);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int grid = blocks_for(count);
  pattern_prepare_kernel<<<grid, kThreads, 0, st>>>(intensities, count, intensities_out, amplitudes_out,
                                                    static_cast<float2*>(amplitudes_c), work);
  if (int rc = check_launch("pattern_prepare_kernel")) return rc;
  sum_parts_kernel<<<1, kThreads, 0, st>>>(work, grid, sums);
  return check_launch("sum_parts_kernel");
}

int ptycho_pattern_shift_ramp(void* spectra, const double* shifts, int npos, int n, void* stream) {
  if (!spectra || !shifts || npos < 1 || n < 1) return fail(PTYCHO_ERR_INVALID, "pattern_shift_ramp: bad arguments");
  pattern_shift_ramp_kernel<<<blocks_for((int64_t)npos * n * n, 148 * 16), kThreads, 0,
                              static_cast<cudaStream_t>(stream)>>>(static_cast<float2*>(spectra), shifts, npos, n);
  return check_launch("pattern_shift_ramp_kernel");
}

int ptycho_pattern_center(const void* shifted, int npos, int n, float scale, float* centered_amplitudes,
                          float* centered_intensities, void* stream) {
  if (!shifted || !centered_amplitudes || npos < 1 || n < 2 || (n & 1))
    return fail(PTYCHO_ERR_INVALID, "pattern_center: bad arguments (even n)");
  pattern_center_kernel<<<blocks_for((int64_t)npos * n * n, 148 * 16), kThreads, 0,
                          static_cast<cudaStream_t>(stream)>>>(static_cast<const float2*>(shifted), npos, n, scale,
                                                               centered_amplitudes, centered_intensities);
  return check_launch("pattern_center_kernel");
}

int ptycho_pattern_bilinear(const float* amplitudes, const double* shifts, int npos, int n,
                            float* centered_amplitudes, float* centered_intensities, void* stream) {
  if (!amplitudes || !shifts || !centered_amplitudes || npos < 0 || n < 2 || (n & 1))
    return fail(PTYCHO_ERR_INVALID, "pattern_bilinear: bad arguments (even n)");
  if (centered_amplitudes == amplitudes || centered_intensities == amplitudes)
    return fail(PTYCHO_ERR_INVALID, "pattern_bilinear: outputs must not alias the amplitudes");
  if (npos == 0) return PTYCHO_OK;
  pattern_bilinear_kernel<<<blocks_for((int64_t)npos * n * n, 148 * 16), kThreads, 0,
                            static_cast<cudaStream_t>(stream)>>>(amplitudes, shifts, npos, n, centered_amplitudes,
                                                                 centered_intensities);
  return check_launch("pattern_bilinear_kernel");
}

}  // extern "C"
