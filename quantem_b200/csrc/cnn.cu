// Learned-initialiser CNN: the tcgen05 BF16 GEMM launcher and the NHWC layer
// kernels around it (im2col with circular padding, transposed-convolution
// gather/scatter, batch-norm statistics and application, ReLU masks, 2x2 max
// pooling, transposes, casts, MSE loss).  Every function here is part of the C
// ABI declared in include/ptycho_b200.h.
//
// Layout: an activation of shape (B, C, H, W) is stored channels-last as a
// row-major matrix with R = B*H*W rows (row r = (b*H + y)*W + x) and a leading
// dimension ld >= C, so a channel slice of a wider buffer (skip concatenation)
// is addressed by a column offset and the wider ld.
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <mutex>

#include "gemm_tcgen05.cuh"
#include "ptycho_b200.h"

int qb_record_error(int code, const char* msg);

namespace {

using bf16 = __nv_bfloat16;

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
bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
int blocks_for(int64_t n, int threads, int cap = 148 * 16) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return static_cast<int>(b < cap ? b : cap);
}

// ---------------------------------------------------------------------------
// GEMM launcher
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

int encode_fn() {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  return g_encode ? PTYCHO_OK : fail(PTYCHO_ERR_CUDA, "gemm: cuTensorMapEncodeTiled is not available");
}

// K-major bf16 matrix [rows][ld] (first k columns used) -> 2-D tensor map with
// a box of 64 (k) x box_rows and the 128-byte swizzle.
int make_map(CUtensorMap* map, const void* base, int rows, int k, int ld, int box_rows) {
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(k), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(qb::gemm::BK), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? PTYCHO_OK : fail(PTYCHO_ERR_INVALID, "gemm: tensor map encode failed (%d)", (int)r);
}

template <int BN>
int launch_gemm(const CUtensorMap& ta, const CUtensorMap& tb, int M, int N, int K, int splits, int kb_per,
                const qb::gemm::Epilogue& epi, int* status, cudaStream_t st) {
  using L = qb::gemm::Smem<BN>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(qb::gemm::gemm_bf16_tn_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                L::BYTES);
  });
  if (attr != cudaSuccess) return fail(PTYCHO_ERR_CUDA, "gemm: smem attribute: %s", cudaGetErrorString(attr));
  dim3 grid((M + qb::gemm::BM - 1) / qb::gemm::BM, (N + BN - 1) / BN, splits);
  qb::gemm::gemm_bf16_tn_kernel<BN><<<grid, qb::gemm::THREADS, L::BYTES, st>>>(ta, tb, M, N, K, kb_per, epi, status);
  return check_launch("gemm_bf16_tn_kernel");
}

// ---------------------------------------------------------------------------
// layer kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// col[r][(ky*3 + kx)*C + c] = x[b, (y+ky-1) mod H, (x+kx-1) mod W, c]; 8 channels per thread.
__global__ void im2col3x3_kernel(const bf16* __restrict__ x, int B, int H, int W, int C, int ldx,
                                 bf16* __restrict__ col, int ldcol) {
  const int c8 = C >> 3;
  const int64_t total = (int64_t)B * H * W * 9 * c8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int cv = (int)(i % c8);
    int64_t t = i / c8;
    const int tap = (int)(t % 9);
    const int64_t r = t / 9;
    const int xx = (int)(r % W), yy = (int)((r / W) % H), b = (int)(r / ((int64_t)W * H));
    const int sy = wrap(yy + tap / 3 - 1, H), sx = wrap(xx + tap % 3 - 1, W);
    const uint4 v = *reinterpret_cast<const uint4*>(x + ((int64_t)(b * H + sy) * W + sx) * ldx + cv * 8);
    *reinterpret_cast<uint4*>(col + r * ldcol + tap * C + cv * 8) = v;
  }
}

// dx[b, y, x, c] (+)= sum_tap dcol[(b, (y-ky+1) mod H, (x-kx+1) mod W)][tap*C + c]; 4 channels per thread.
__global__ void col2im3x3_kernel(const float* __restrict__ dcol, int ldcol, int B, int H, int W, int C,
                                 float* __restrict__ dx, int ldx, int accumulate) {
  const int c4 = C >> 2;
  const int64_t total = (int64_t)B * H * W * c4;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int cv = (int)(i % c4);
    const int64_t r = i / c4;
    const int xx = (int)(r % W), yy = (int)((r / W) % H), b = (int)(r / ((int64_t)W * H));
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int sy = wrap(yy - tap / 3 + 1, H), sx = wrap(xx - tap % 3 + 1, W);
      const float4 v =
          *reinterpret_cast<const float4*>(dcol + ((int64_t)(b * H + sy) * W + sx) * ldcol + tap * C + cv * 4);
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
    float4* o = reinterpret_cast<float4*>(dx + r * ldx + cv * 4);
    if (accumulate) {
      const float4 p = *o;
      acc.x += p.x;
      acc.y += p.y;
      acc.z += p.z;
      acc.w += p.w;
    }
    *o = acc;
  }
}

// Transposed convolution 3x3, stride 2, padding 1, output padding 1 (zero padded):
// out[b, oy, ox, co] = bias[co] + sum over taps with oy = 2 iy - 1 + ky, ox = 2 ix - 1 + kx
// of colT[(b, iy, ix)][(ky*3 + kx)*Co + co].  Output (B, 2H, 2W, Co) in bf16.
__global__ void convT_gather_kernel(const float* __restrict__ colT, int ldcol, int B, int H, int W, int Co,
                                    const float* __restrict__ bias, bf16* __restrict__ out, int ldo) {
  const int H2 = 2 * H, W2 = 2 * W;
  const int64_t total = (int64_t)B * H2 * W2 * Co;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int co = (int)(i % Co);
    const int64_t r = i / Co;
    const int ox = (int)(r % W2), oy = (int)((r / W2) % H2), b = (int)(r / ((int64_t)W2 * H2));
    float acc = bias ? bias[co] : 0.0f;
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
      const int ty = oy + 1 - ky;
      if (ty < 0 || (ty & 1)) continue;
      const int iy = ty >> 1;
      if (iy >= H) continue;
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const int tx = ox + 1 - kx;
        if (tx < 0 || (tx & 1)) continue;
        const int ix = tx >> 1;
        if (ix >= W) continue;
        acc += colT[((int64_t)(b * H + iy) * W + ix) * ldcol + (ky * 3 + kx) * Co + co];
      }
    }
    out[r * ldo + co] = __float2bfloat16_rn(acc);
  }
}

// Backward of the transposed convolution's scatter:
// dcol[(b, iy, ix)][(ky*3+kx)*Co + co] = dout[b, 2iy-1+ky, 2ix-1+kx, co] (0 outside), bf16.
__global__ void convT_im2col_kernel(const float* __restrict__ dout, int ldo, int B, int H, int W, int Co,
                                    bf16* __restrict__ dcol, int ldcol) {
  const int H2 = 2 * H, W2 = 2 * W;
  const int64_t total = (int64_t)B * H * W * 9 * Co;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int co = (int)(i % Co);
    int64_t t = i / Co;
    const int tap = (int)(t % 9);
    const int64_t r = t / 9;
    const int ix = (int)(r % W), iy = (int)((r / W) % H), b = (int)(r / ((int64_t)W * H));
    const int oy = 2 * iy - 1 + tap / 3, ox = 2 * ix - 1 + tap % 3;
    float v = 0.0f;
    if (oy >= 0 && oy < H2 && ox >= 0 && ox < W2) v = dout[((int64_t)(b * H2 + oy) * W2 + ox) * ldo + co];
    dcol[r * ldcol + tap * Co + co] = __float2bfloat16_rn(v);
  }
}

template <typename T>
__device__ __forceinline__ float to_f(T v);
template <>
__device__ __forceinline__ float to_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f<bf16>(bf16 v) { return __bfloat162float(v); }
template <typename T>
__device__ __forceinline__ T from_f(float v);
template <>
__device__ __forceinline__ float from_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ bf16 from_f<bf16>(float v) { return __float2bfloat16_rn(v); }

// out[z][c][r] = in[z][r][c] (32 x 32 tiles through shared memory), batched over z.
template <typename Ti, typename To>
__global__ void transpose_kernel(const Ti* __restrict__ in, int R, int C, int ldi, int64_t zsi, To* __restrict__ out,
                                 int ldo, int64_t zso) {
  __shared__ float tile[32][33];
  in += blockIdx.z * zsi;
  out += blockIdx.z * zso;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    tile[j][threadIdx.x] = (r < R && c < C) ? to_f<Ti>(in[(int64_t)r * ldi + c]) : 0.0f;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    if (c < C && r < R) out[(int64_t)c * ldo + r] = from_f<To>(tile[threadIdx.x][j]);
  }
}

// Deterministic column reductions over the rows of an FP32 matrix, in two passes:
// per-chunk partials (double) then a fixed-order sum per column.
//   mode 0: s0 = sum a,        s1 = sum a^2                  (batch-norm statistics)
//   mode 1: s0 = sum a,        s1 = sum a * (b - mean) * rstd (batch-norm backward; a = dy, b = input)
//   mode 2: s0 = sum a                                        (bias gradient)
constexpr int kColThreads = 256;
__global__ void colsum_partial_kernel(int mode, const float* __restrict__ a, int lda, const float* __restrict__ b,
                                      int ldb, const float* __restrict__ mean, const float* __restrict__ rstd, int R,
                                      int C, int rows_per_chunk, double* __restrict__ part) {
  __shared__ double red0[kColThreads], red1[kColThreads];
  const int TC = C < kColThreads ? C : kColThreads;
  const int RP = kColThreads / TC;
  const int tx = threadIdx.x % TC, ty = threadIdx.x / TC;
  const int c = blockIdx.y * TC + tx;
  const int r0 = blockIdx.x * rows_per_chunk, r1 = min(R, r0 + rows_per_chunk);
  double s0 = 0.0, s1 = 0.0;
  if (ty < RP && c < C) {
    const float m = (mode == 1) ? mean[c] : 0.0f, rs = (mode == 1) ? rstd[c] : 0.0f;
    float f0 = 0.f, f1 = 0.f;
    int cnt = 0;
    for (int r = r0 + ty; r < r1; r += RP) {
      const float v = a[(int64_t)r * lda + c];
      f0 += v;
      if (mode == 0) f1 = fmaf(v, v, f1);
      else if (mode == 1) f1 = fmaf(v, (b[(int64_t)r * ldb + c] - m) * rs, f1);
      if (++cnt == 64) {  // flush to double every 64 rows
        s0 += f0;
        s1 += f1;
        f0 = f1 = 0.f;
        cnt = 0;
      }
    }
    s0 += f0;
    s1 += f1;
  }
  red0[threadIdx.x] = s0;
  red1[threadIdx.x] = s1;
  __syncthreads();
  if (ty == 0 && c < C) {
    for (int k = 1; k < RP; ++k) {
      s0 += red0[k * TC + tx];
      s1 += red1[k * TC + tx];
    }
    part[((int64_t)blockIdx.x * 2 + 0) * C + c] = s0;
    part[((int64_t)blockIdx.x * 2 + 1) * C + c] = s1;
  }
}

// Finishing pass.  mode 0 (batch-norm statistics): mean, rstd = 1/sqrt(var + eps) with the
// biased variance; running statistics updated with the unbiased one (nn.BatchNorm2d).
// mode 1 (batch-norm backward): o0 = dbeta = sum dy, o1 = dgamma = sum dy*xhat.
// mode 2: o0 = sum (bias gradient), written or accumulated.
__global__ void colsum_final_kernel(int mode, const double* __restrict__ part, int nchunks, int R, int C, float eps,
                                    float momentum, float* o0, float* o1, float* run_mean, float* run_var,
                                    int accumulate) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  double s0 = 0.0, s1 = 0.0;
  for (int k = 0; k < nchunks; ++k) {
    s0 += part[((int64_t)k * 2 + 0) * C + c];
    s1 += part[((int64_t)k * 2 + 1) * C + c];
  }
  if (mode == 0) {
    const double mean = s0 / R;
    double var = s1 / R - mean * mean;
    if (var < 0.0) var = 0.0;
    o0[c] = (float)mean;
    o1[c] = (float)(1.0 / sqrt(var + (double)eps));
    if (run_mean) {
      const double unb = R > 1 ? var * R / (R - 1) : var;
      run_mean[c] = (float)((1.0 - momentum) * run_mean[c] + momentum * mean);
      run_var[c] = (float)((1.0 - momentum) * run_var[c] + momentum * unb);
    }
  } else if (mode == 1) {
    if (accumulate) {
      o0[c] += (float)s0;
      o1[c] += (float)s1;
    } else {
      o0[c] = (float)s0;
      o1[c] = (float)s1;
    }
  } else {
    o0[c] = accumulate ? o0[c] + (float)s0 : (float)s0;
  }
}

// Eval-mode statistics: mean = running mean, rstd = 1/sqrt(running var + eps).
__global__ void bn_eval_stats_kernel(const float* run_mean, const float* run_var, int C, float eps, float* mean,
                                     float* rstd) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < C) {
    mean[c] = run_mean[c];
    rstd[c] = rsqrtf(run_var[c] + eps);
  }
}

// y = (x - mean) * rstd * gamma + beta (or x when mean is null), bf16 out.
__global__ void bn_apply_kernel(const float* __restrict__ x, int ldx, int R, int C, const float* __restrict__ mean,
                                const float* __restrict__ rstd, const float* __restrict__ gamma,
                                const float* __restrict__ beta, bf16* __restrict__ y, int ldy) {
  const int64_t total = (int64_t)R * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t r = i / C;
    float v = x[r * ldx + c];
    if (mean) v = (v - mean[c]) * rstd[c] * gamma[c] + beta[c];
    y[r * ldy + c] = __float2bfloat16_rn(v);
  }
}

// Batch-norm backward (training statistics) followed by the derivative of the activation
// that produced its input x: dx = act'(x) * gamma * rstd * (dy - s_dy/R - xhat * s_dyxhat/R);
// without batch norm (mean null) dx = act'(x) * dy.  act = qb::ACT_* (1 = ReLU: the mask
// [x > 0]; 0: none).  Writes FP32 and BF16 copies.
__global__ void bn_relu_backward_kernel(const float* __restrict__ dy, int lddy, const float* __restrict__ x, int ldx,
                                        int R, int C, const float* __restrict__ mean, const float* __restrict__ rstd,
                                        const float* __restrict__ gamma, const float* __restrict__ sdy,
                                        const float* __restrict__ sdyx, int act, float* __restrict__ dz32,
                                        bf16* __restrict__ dz16, int ldz) {
  const int64_t total = (int64_t)R * C;
  const float invR = 1.0f / (float)R;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t r = i / C;
    const float xv = x[r * ldx + c];
    float g = dy[r * lddy + c];
    if (mean) {
      const float xh = (xv - mean[c]) * rstd[c];
      g = gamma[c] * rstd[c] * (g - sdy[c] * invR - xh * sdyx[c] * invR);
    }
    if (act) g *= qb::act_grad_from_output(act, xv);
    if (dz32) dz32[r * ldz + c] = g;
    if (dz16) dz16[r * ldz + c] = __float2bfloat16_rn(g);
  }
}

// Eval-mode batch-norm backward is a per-channel scale: dx = dy * gamma * rstd (then act').
__global__ void bn_eval_backward_kernel(const float* __restrict__ dy, int lddy, const float* __restrict__ x, int ldx,
                                        int R, int C, const float* __restrict__ rstd, const float* __restrict__ gamma,
                                        int act, float* __restrict__ dz32, bf16* __restrict__ dz16, int ldz) {
  const int64_t total = (int64_t)R * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t r = i / C;
    float g = dy[r * lddy + c] * gamma[c] * rstd[c];
    if (act) g *= qb::act_grad_from_output(act, x[r * ldx + c]);
    if (dz32) dz32[r * ldz + c] = g;
    if (dz16) dz16[r * ldz + c] = __float2bfloat16_rn(g);
  }
}

// 2x2 max pool, stride 2 (H, W even); argmax code (dy*2 + dx) of the first maximum in
// row-major window order, as torch's max_pool2d picks it.
__global__ void maxpool2_kernel(const bf16* __restrict__ in, int ldi, int B, int H, int W, int C,
                                bf16* __restrict__ out, int ldo, uint8_t* __restrict__ arg) {
  const int Ho = H / 2, Wo = W / 2;
  const int64_t total = (int64_t)B * Ho * Wo * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t r = i / C;
    const int ox = (int)(r % Wo), oy = (int)((r / Wo) % Ho), b = (int)(r / ((int64_t)Wo * Ho));
    float best = -INFINITY;
    int code = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int y = 2 * oy + (k >> 1), x = 2 * ox + (k & 1);
      const float v = __bfloat162float(in[((int64_t)(b * H + y) * W + x) * ldi + c]);
      if (k == 0 || v > best) {
        best = v;
        code = k;
      }
    }
    out[r * ldo + c] = __float2bfloat16_rn(best);
    arg[r * C + c] = (uint8_t)code;
  }
}

// din[b, y, x, c] (+)= dout[b, y/2, x/2, c] if (y, x) held the window maximum, else 0.
__global__ void maxpool2_backward_kernel(const float* __restrict__ dout, int lddo, const uint8_t* __restrict__ arg,
                                         int B, int H, int W, int C, float* __restrict__ din, int lddi,
                                         int accumulate) {
  const int Wo = W / 2, Ho = H / 2;
  const int64_t total = (int64_t)B * H * W * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t r = i / C;
    const int x = (int)(r % W), y = (int)((r / W) % H), b = (int)(r / ((int64_t)W * H));
    const int64_t ro = (int64_t)(b * Ho + y / 2) * Wo + x / 2;
    const float g = (arg[ro * C + c] == (uint8_t)(((y & 1) << 1) | (x & 1))) ? dout[ro * lddo + c] : 0.0f;
    float* o = din + r * lddi + c;
    *o = accumulate ? *o + g : g;
  }
}

__global__ void cast_bf16_kernel(const float* __restrict__ in, bf16* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

// Mean squared error over n values: partial sums of (p - t)^2 per block (double) and
// dp = 2 (p - t) / n in FP32 and BF16.
__global__ void mse_kernel(const float* __restrict__ p, const float* __restrict__ t, int64_t n,
                           double* __restrict__ part, float* __restrict__ dp32, bf16* __restrict__ dp16) {
  __shared__ double red[256];
  double s = 0.0;
  const float sc = 2.0f / (float)n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float d = p[i] - t[i];
    s += (double)d * d;
    if (dp32) dp32[i] = sc * d;
    if (dp16) dp16[i] = __float2bfloat16_rn(sc * d);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}
__global__ void mse_final_kernel(const double* part, int nparts, int64_t n, float* loss) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < nparts; ++i) s += part[i];
    *loss = (float)(s / (double)n);
  }
}

// Network input features from diffraction data: per scan position p and bin (u, v)
// of a bin x bin block, f = sqrt(norm * sum of the block's intensities) (amplitudes
// are squared first), then (f - mean[u*nb + v]) * scale, written as BF16 row p.
__global__ void bin_features_kernel(const float* __restrict__ pat, int npos, int n, int bin, int amplitudes,
                                    float norm, const float* __restrict__ mean, float scale, bf16* __restrict__ out,
                                    int ldo) {
  const int nb = n / bin;
  const int64_t total = (int64_t)npos * nb * nb;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % (nb * nb));
    const int64_t p = i / (nb * nb);
    const int u = c / nb, v = c % nb;
    const float* src = pat + p * n * n + (int64_t)(u * bin) * n + v * bin;
    float s = 0.0f;
    for (int a = 0; a < bin; ++a)
      for (int b = 0; b < bin; ++b) {
        const float x = src[a * n + b];
        s += amplitudes ? x * x : x;
      }
    float f = sqrtf(fmaxf(s * norm, 0.0f));
    if (mean) f -= mean[c];
    out[p * ldo + c] = __float2bfloat16_rn(f * scale);
  }
}

constexpr int kMseBlocks = 296;

int colsum(int mode, const float* a, int lda, const float* b, int ldb, const float* mean, const float* rstd, int R,
           int C, double* work, int64_t work_elems, float eps, float momentum, float* o0, float* o1, float* run_mean,
           float* run_var, int accumulate, cudaStream_t st) {
  const int TC = C < kColThreads ? C : kColThreads;
  const int RP = kColThreads / TC;
  int chunks = (R + RP * 16 - 1) / (RP * 16);
  if (chunks > 592) chunks = 592;
  if ((int64_t)chunks * 2 * C > work_elems) chunks = (int)(work_elems / (2 * (int64_t)C));
  if (chunks < 1) return fail(PTYCHO_ERR_INVALID, "cnn: reduction workspace too small (%lld doubles for C=%d)",
                              (long long)work_elems, C);
  const int rpc = (R + chunks - 1) / chunks;
  chunks = (R + rpc - 1) / rpc;
  dim3 grid(chunks, (C + TC - 1) / TC);
  colsum_partial_kernel<<<grid, kColThreads, 0, st>>>(mode, a, lda, b, ldb, mean, rstd, R, C, rpc, work);
  if (int rc = check_launch("colsum_partial_kernel")) return rc;
  colsum_final_kernel<<<(C + 127) / 128, 128, 0, st>>>(mode, work, chunks, R, C, eps, momentum, o0, o1, run_mean,
                                                       run_var, accumulate);
  return check_launch("colsum_final_kernel");
}

}  // namespace

// Dropout (nn.Dropout, blocks.py:134-135): x *= keep / (1 - p) with keep = u >= p, u a
// uniform draw per element from a counter-based hash of (seed, row * C + column) -- the
// SplitMix64 finaliser (Steele, Lea and Flood, 2014) -- so the backward regenerates the
// forward's mask from the same seed instead of storing it.
__device__ __forceinline__ float dropout_uniform(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (float)(z >> 40) * (1.0f / 16777216.0f);  // 24 random bits in [0, 1)
}

template <typename T>
__global__ void dropout_kernel(T* __restrict__ x, int R, int C, int ld, float p, float scale, uint64_t seed) {
  const int64_t total = (int64_t)R * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / C;
    const int c = (int)(i % C);
    const bool keep = dropout_uniform(seed, (uint64_t)i) >= p;
    T* e = x + r * ld + c;
    if constexpr (sizeof(T) == 4) {
      *e = keep ? *e * scale : 0.0f;
    } else {
      *e = keep ? __float2bfloat16_rn(__bfloat162float(*e) * scale) : __float2bfloat16_rn(0.0f);
    }
  }
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int ptycho_gemm_bf16(const void* A, int lda, const void* B, int ldb, void* C, int ldc, int M, int N, int K,
                     const float* bias, int flags, int splits, int* status, void* stream) {
  using namespace qb::gemm;
  if (!A || !B || !C || M < 1 || N < 1 || K < 1 || lda < K || ldb < K || ldc < N)
    return fail(PTYCHO_ERR_INVALID, "gemm: bad sizes (M=%d N=%d K=%d lda=%d ldb=%d ldc=%d)", M, N, K, lda, ldb, ldc);
  if ((lda & 7) || (ldb & 7) || !al16(A) || !al16(B))
    return fail(PTYCHO_ERR_INVALID, "gemm: A/B must be 16-byte aligned with leading dimensions a multiple of 8");
  if (flags & ~(EPI_BF16 | EPI_RELU | EPI_ATOMIC | EPI_ACT_MASK))
    return fail(PTYCHO_ERR_INVALID, "gemm: unknown flags %d", flags);
  int act = (flags & EPI_ACT_MASK) >> EPI_ACT_SHIFT;
  if (act >= qb::ACT_COUNT || ((flags & EPI_RELU) && act && act != qb::ACT_RELU))
    return fail(PTYCHO_ERR_INVALID, "gemm: bad activation in flags %d", flags);
  if (flags & EPI_RELU) act = qb::ACT_RELU;
  const int nkb = (K + BK - 1) / BK;
  if (splits < 1) splits = 1;
  if (splits > nkb) splits = nkb;
  const bool accumulate = (flags & EPI_ATOMIC) != 0;  // add into C as it is
  if (splits > 1) flags |= EPI_ATOMIC;
  if ((flags & EPI_ATOMIC) && ((flags & EPI_BF16) || act))
    return fail(PTYCHO_ERR_INVALID, "gemm: split-K / atomic output needs FP32 output without an activation");
  if (int rc = encode_fn()) return rc;
  const int kb_per = (nkb + splits - 1) / splits;
  splits = (nkb + kb_per - 1) / kb_per;  // every split gets >= 1 k-block
  const int BN = N <= 32 ? 32 : (N <= 64 ? 64 : 128);
  CUtensorMap ta, tb;
  if (int rc = make_map(&ta, A, M, K, lda, BM)) return rc;
  if (int rc = make_map(&tb, B, N, K, ldb, BN)) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!accumulate && splits > 1) {
    if (cudaMemset2DAsync(C, (size_t)ldc * 4, 0, (size_t)N * 4, (size_t)M, st) != cudaSuccess)
      return check_launch("gemm: clear split-K output");
  }
  Epilogue epi{C, bias, ldc, flags, act};
  switch (BN) {
    case 32: return launch_gemm<32>(ta, tb, M, N, K, splits, kb_per, epi, status, st);
    case 64: return launch_gemm<64>(ta, tb, M, N, K, splits, kb_per, epi, status, st);
    default: return launch_gemm<128>(ta, tb, M, N, K, splits, kb_per, epi, status, st);
  }
}

int ptycho_cnn_im2col3x3(const void* x, int B, int H, int W, int C, int ldx, void* col, int ldcol, void* stream) {
  if (!x || !col || B < 1 || H < 1 || W < 1 || C < 8 || (C & 7) || (ldx & 7) || (ldcol & 7) || ldx < C ||
      ldcol < 9 * C || !al16(x) || !al16(col))
    return fail(PTYCHO_ERR_INVALID, "im2col3x3: bad arguments (C and leading dims multiples of 8, 16-byte aligned)");
  const int64_t n = (int64_t)B * H * W * 9 * (C / 8);
  im2col3x3_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const bf16*>(x), B, H, W, C, ldx, static_cast<bf16*>(col), ldcol);
  return check_launch("im2col3x3_kernel");
}

int ptycho_cnn_col2im3x3(const float* dcol, int ldcol, int B, int H, int W, int C, float* dx, int ldx, int accumulate,
                         void* stream) {
  if (!dcol || !dx || B < 1 || H < 1 || W < 1 || C < 4 || (C & 3) || (ldcol & 3) || (ldx & 3) || ldcol < 9 * C ||
      ldx < C || !al16(dcol) || !al16(dx))
    return fail(PTYCHO_ERR_INVALID, "col2im3x3: bad arguments (C and leading dims multiples of 4, 16-byte aligned)");
  const int64_t n = (int64_t)B * H * W * (C / 4);
  col2im3x3_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(dcol, ldcol, B, H, W, C, dx, ldx,
                                                                                       accumulate);
  return check_launch("col2im3x3_kernel");
}

int ptycho_cnn_convT_gather(const float* colT, int ldcol, int B, int H, int W, int Co, const float* bias, void* out,
                            int ldo, void* stream) {
  if (!colT || !out || B < 1 || H < 1 || W < 1 || Co < 1 || ldcol < 9 * Co || ldo < Co)
    return fail(PTYCHO_ERR_INVALID, "convT_gather: bad arguments");
  const int64_t n = (int64_t)B * 4 * H * W * Co;
  convT_gather_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      colT, ldcol, B, H, W, Co, bias, static_cast<bf16*>(out), ldo);
  return check_launch("convT_gather_kernel");
}

int ptycho_cnn_convT_im2col(const float* dout, int ldo, int B, int H, int W, int Co, void* dcol, int ldcol,
                            void* stream) {
  if (!dout || !dcol || B < 1 || H < 1 || W < 1 || Co < 1 || ldo < Co || ldcol < 9 * Co)
    return fail(PTYCHO_ERR_INVALID, "convT_im2col: bad arguments");
  const int64_t n = (int64_t)B * H * W * 9 * Co;
  convT_im2col_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dout, ldo, B, H, W, Co, static_cast<bf16*>(dcol), ldcol);
  return check_launch("convT_im2col_kernel");
}

// dtypes: 0 = FP32, 1 = BF16.
int ptycho_cnn_transpose(const void* in, int in_dtype, int R, int C, int ldi, int64_t batch_stride_in, void* out,
                         int out_dtype, int ldo, int64_t batch_stride_out, int batch, void* stream) {
  if (!in || !out || R < 1 || C < 1 || ldi < C || ldo < R || batch < 1 || batch > 65535 || in_dtype < 0 ||
      in_dtype > 1 || out_dtype < 0 || out_dtype > 1)
    return fail(PTYCHO_ERR_INVALID, "transpose: bad arguments");
  dim3 grid((C + 31) / 32, (R + 31) / 32, batch), block(32, 8);
  if ((C + 31) / 32 > 2147483647 || (R + 31) / 32 > 65535) return fail(PTYCHO_ERR_INVALID, "transpose: too many rows");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (in_dtype == 0 && out_dtype == 1)
    transpose_kernel<float, bf16><<<grid, block, 0, st>>>(static_cast<const float*>(in), R, C, ldi, batch_stride_in,
                                                          static_cast<bf16*>(out), ldo, batch_stride_out);
  else if (in_dtype == 1 && out_dtype == 1)
    transpose_kernel<bf16, bf16><<<grid, block, 0, st>>>(static_cast<const bf16*>(in), R, C, ldi, batch_stride_in,
                                                         static_cast<bf16*>(out), ldo, batch_stride_out);
  else if (in_dtype == 0 && out_dtype == 0)
    transpose_kernel<float, float><<<grid, block, 0, st>>>(static_cast<const float*>(in), R, C, ldi, batch_stride_in,
                                                           static_cast<float*>(out), ldo, batch_stride_out);
  else
    transpose_kernel<bf16, float><<<grid, block, 0, st>>>(static_cast<const bf16*>(in), R, C, ldi, batch_stride_in,
                                                          static_cast<float*>(out), ldo, batch_stride_out);
  return check_launch("transpose_kernel");
}

int ptycho_cnn_bn_forward(const float* x, int ldx, int R, int C, const float* gamma, const float* beta,
                          float* run_mean, float* run_var, float momentum, float eps, int training, float* mean,
                          float* rstd, double* work, int64_t work_elems, void* out, int ldo, void* stream) {
  if (!x || !out || R < 1 || C < 1 || ldx < C || ldo < C) return fail(PTYCHO_ERR_INVALID, "bn_forward: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool bn = gamma != nullptr;
  if (bn) {
    if (!beta || !mean || !rstd || (!training && (!run_mean || !run_var)))
      return fail(PTYCHO_ERR_INVALID, "bn_forward: missing statistics buffers");
    if (training) {
      if (int rc = colsum(0, x, ldx, nullptr, 0, nullptr, nullptr, R, C, work, work_elems, eps, momentum, mean, rstd,
                          run_mean, run_var, 0, st))
        return rc;
    } else {
      bn_eval_stats_kernel<<<(C + 127) / 128, 128, 0, st>>>(run_mean, run_var, C, eps, mean, rstd);
      if (int rc = check_launch("bn_eval_stats_kernel")) return rc;
    }
  }
  bn_apply_kernel<<<blocks_for((int64_t)R * C, 256), 256, 0, st>>>(x, ldx, R, C, bn ? mean : nullptr, rstd, gamma,
                                                                    beta, static_cast<bf16*>(out), ldo);
  return check_launch("bn_apply_kernel");
}

int ptycho_cnn_bn_backward(const float* dy, int lddy, const float* x, int ldx, int R, int C, const float* gamma,
                           const float* mean, const float* rstd, int training, int act, float* dgamma, float* dbeta,
                           double* work, int64_t work_elems, float* dz32, void* dz16, int ldz, void* stream) {
  if (!dy || !x || R < 1 || C < 1 || lddy < C || ldx < C || ldz < C || (!dz32 && !dz16) || act < 0 ||
      act >= qb::ACT_COUNT)
    return fail(PTYCHO_ERR_INVALID, "bn_backward: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int g = blocks_for((int64_t)R * C, 256);
  if (gamma) {
    if (!mean || !rstd || !dgamma || !dbeta) return fail(PTYCHO_ERR_INVALID, "bn_backward: missing buffers");
    if (int rc = colsum(1, dy, lddy, x, ldx, mean, rstd, R, C, work, work_elems, 0.f, 0.f, dbeta, dgamma, nullptr,
                        nullptr, 0, st))
      return rc;
    if (training)
      bn_relu_backward_kernel<<<g, 256, 0, st>>>(dy, lddy, x, ldx, R, C, mean, rstd, gamma, dbeta, dgamma, act, dz32,
                                                 static_cast<bf16*>(dz16), ldz);
    else
      bn_eval_backward_kernel<<<g, 256, 0, st>>>(dy, lddy, x, ldx, R, C, rstd, gamma, act, dz32,
                                                 static_cast<bf16*>(dz16), ldz);
  } else {
    bn_relu_backward_kernel<<<g, 256, 0, st>>>(dy, lddy, x, ldx, R, C, nullptr, nullptr, nullptr, nullptr, nullptr,
                                               act, dz32, static_cast<bf16*>(dz16), ldz);
  }
  return check_launch("bn_backward");
}

int ptycho_cnn_colsum(const float* a, int lda, int R, int C, float* out, int accumulate, double* work,
                      int64_t work_elems, void* stream) {
  if (!a || !out || R < 1 || C < 1 || lda < C) return fail(PTYCHO_ERR_INVALID, "colsum: bad arguments");
  return colsum(2, a, lda, nullptr, 0, nullptr, nullptr, R, C, work, work_elems, 0.f, 0.f, out, nullptr, nullptr,
                nullptr, accumulate, static_cast<cudaStream_t>(stream));
}

int ptycho_cnn_maxpool2(const void* in, int ldi, int B, int H, int W, int C, void* out, int ldo, void* argmax,
                        void* stream) {
  if (!in || !out || !argmax || B < 1 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || ldi < C || ldo < C)
    return fail(PTYCHO_ERR_INVALID, "maxpool2: bad arguments (H, W even)");
  const int64_t n = (int64_t)B * (H / 2) * (W / 2) * C;
  maxpool2_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const bf16*>(in), ldi, B, H, W, C, static_cast<bf16*>(out), ldo, static_cast<uint8_t*>(argmax));
  return check_launch("maxpool2_kernel");
}

int ptycho_cnn_maxpool2_backward(const float* dout, int lddo, const void* argmax, int B, int H, int W, int C,
                                 float* din, int lddi, int accumulate, void* stream) {
  if (!dout || !argmax || !din || B < 1 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || lddo < C || lddi < C)
    return fail(PTYCHO_ERR_INVALID, "maxpool2_backward: bad arguments");
  const int64_t n = (int64_t)B * H * W * C;
  maxpool2_backward_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dout, lddo, static_cast<const uint8_t*>(argmax), B, H, W, C, din, lddi, accumulate);
  return check_launch("maxpool2_backward_kernel");
}

int ptycho_cnn_cast_bf16(const float* in, void* out, int64_t n, void* stream) {
  if (!in || !out || n < 0) return fail(PTYCHO_ERR_INVALID, "cast_bf16: bad arguments");
  if (n == 0) return PTYCHO_OK;
  cast_bf16_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(in, static_cast<bf16*>(out), n);
  return check_launch("cast_bf16_kernel");
}

int ptycho_cnn_mse(const float* pred, const float* target, int64_t n, float* loss, float* dpred32, void* dpred16,
                   double* work, int64_t work_elems, void* stream) {
  if (!pred || !target || !loss || n < 1 || !work || work_elems < kMseBlocks)
    return fail(PTYCHO_ERR_INVALID, "mse: bad arguments (workspace >= %d doubles)", kMseBlocks);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  mse_kernel<<<kMseBlocks, 256, 0, st>>>(pred, target, n, work, dpred32, static_cast<bf16*>(dpred16));
  if (int rc = check_launch("mse_kernel")) return rc;
  mse_final_kernel<<<1, 32, 0, st>>>(work, kMseBlocks, n, loss);
  return check_launch("mse_final_kernel");
}

int ptycho_cnn_bin_features(const float* patterns, int npos, int n, int bin, int amplitudes, float norm,
                            const float* mean, float scale, void* out, int ldo, void* stream) {
  if (!patterns || !out || npos < 1 || n < 1 || bin < 1 || n % bin || ldo < (n / bin) * (n / bin))
    return fail(PTYCHO_ERR_INVALID, "bin_features: bad arguments (n divisible by bin, ldo >= (n/bin)^2)");
  const int64_t total = (int64_t)npos * (n / bin) * (n / bin);
  bin_features_kernel<<<blocks_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      patterns, npos, n, bin, amplitudes, norm, mean, scale, static_cast<bf16*>(out), ldo);
  return check_launch("bin_features_kernel");
}

int ptycho_cnn_dropout(void* x, int dtype, int R, int C, int ld, float p, uint64_t seed, void* stream) {
  if (!x || R < 1 || C < 1 || ld < C || !(p >= 0.0f && p <= 1.0f) || (dtype != 0 && dtype != 1))
    return fail(PTYCHO_ERR_INVALID, "dropout: bad arguments");
  const float scale = p < 1.0f ? 1.0f / (1.0f - p) : 0.0f;  // p = 1 drops everything
  const int g = blocks_for((int64_t)R * C, 256);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == 0)
    dropout_kernel<float><<<g, 256, 0, st>>>(static_cast<float*>(x), R, C, ld, p, scale, seed);
  else
    dropout_kernel<bf16><<<g, 256, 0, st>>>(static_cast<bf16*>(x), R, C, ld, p, scale, seed);
  return check_launch("dropout_kernel");
}

}  // extern "C"
