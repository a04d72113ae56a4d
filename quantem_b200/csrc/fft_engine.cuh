// Register-resident 2-D FFT engine for one N x N complex64 wave per CTA (sm_100a).
//
// A CTA of T = 4N threads holds the wave in registers, E = N/4 complex values per
// thread.  The 2-D transform is factored into three register stages that each
// consume a subset of the 2*log2(N) index bits, with one shared-memory exchange
// between consecutive stages:
//
//   columns c = cB + B*cA  (N = A*B),   rows r = rD + D*rC  (N = C*D)
//   S1 : A-point DFT over cA            for fixed (r, cB)          -> kA
//   S2 : twiddle w_N^(cB*kA); B-point DFT over cB; C-point DFT over rC;
//        twiddle w_N^(rD*kC)            for fixed (rD, kA)         -> (kB, kC)
//   S3 : D-point DFT over rD            for fixed (kC, column)     -> kD
//
// The forward output of S3 is in natural frequency order: register (g, e) of a
// thread holds X[kC_g + C*e][col].  The inverse runs S3' -> S2' -> S1' with
// conjugate twiddles, so a forward transform, an elementwise multiply in Fourier
// space and an inverse transform need no exchange between S3 and S3'; likewise
// an inverse, a real-space multiply and a forward transform meet in S1 without
// an exchange.  One multislice step (FFT, propagator, IFFT, transmission) costs
// four exchanges.
//
// Shared-memory layout: float2 sm[N][N+1] (one padding column).  With the lane
// assignments below every stage's 32 lanes touch each bank pair at most twice,
// i.e. two wavefronts per 256-byte warp access, the minimum for 8-byte words.
//
// Supported N: 64 (A=16,B=4,C=4,D=16, 256 threads) and 128 (A=32,B=4,C=8,D=16,
// 512 threads); 96 is a specialisation at the end of this file (192 threads,
// mixed radix 3 x 2^k).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qb {

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
// Complex arithmetic.  With QB_F32X2_ADD / QB_F32X2_MUL set (per translation unit,
// before this header) it runs on sm_100's packed FP32 pairs, one instruction for the
// real and imaginary parts, with the same roundings as the scalar forms
//   a * b       = (fma(a.x, b.x, -(a.y b.y)), fma(a.x, b.y, a.y b.x))
//   a * conj(b) = (fma(a.x, b.x, a.y b.y),    fma(a.y, b.x, -(a.x b.y)))
// so results are bit-identical either way.  The packed operands live in aligned
// register pairs, which costs registers: packed products pay in the 64^2, 96^2 and
// 256^2 kernels but not in the 128^2 batch kernel, whose 512 threads already sit at
// 128 registers (it packs only its additions).
#ifndef QB_F32X2_ADD
#define QB_F32X2_ADD 0
#endif
#ifndef QB_F32X2_MUL
#define QB_F32X2_MUL 0
#endif
#if QB_F32X2_ADD
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
#else
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
#endif
#if QB_F32X2_MUL
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return __ffma2_rn(make_float2(a.x, a.x), b, __fmul2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x)));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return __ffma2_rn(a, make_float2(b.x, b.x), __fmul2_rn(make_float2(a.y, -a.x), make_float2(b.y, b.y)));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
#else
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
#endif
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// Packed products whatever the switches above say; QB_F32X2_S2 uses them for the
// twiddle multiplies of the 2-D engine's middle stage only (no extra spills in the
// 128^2 batch kernel, unlike packed products everywhere).
__device__ __forceinline__ float2 pcmul(float2 a, float2 b) {
  return __ffma2_rn(make_float2(a.x, a.x), b, __fmul2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x)));
}
__device__ __forceinline__ float2 pcmulc(float2 a, float2 b) {
  return __ffma2_rn(a, make_float2(b.x, b.x), __fmul2_rn(make_float2(a.y, -a.x), make_float2(b.y, b.y)));
}
#ifndef QB_F32X2_S2
#define QB_F32X2_S2 0
#endif
__device__ __forceinline__ float cabs2(float2 a) { return fmaf(a.x, a.x, a.y * a.y); }

// cos(2*pi*m/64) for m = 0..16 (first quadrant), IEEE double rounded to float.
__device__ __forceinline__ float qcos64(int m) {
  switch (m) {
    case 0: return 1.0f;
    case 1: return 0.99518472667219693f;
    case 2: return 0.98078528040323043f;
    case 3: return 0.95694033573220882f;
    case 4: return 0.92387953251128674f;
    case 5: return 0.88192126434835505f;
    case 6: return 0.83146961230254524f;
    case 7: return 0.77301045336273699f;
    case 8: return 0.70710678118654757f;
    case 9: return 0.63439328416364549f;
    case 10: return 0.55557023301960229f;
    case 11: return 0.47139673682599781f;
    case 12: return 0.38268343236508984f;
    case 13: return 0.29028467725446233f;
    case 14: return 0.19509032201612833f;
    case 15: return 0.09801714032956077f;
    default: return 0.0f;
  }
}

// Multiply by w_64^m (forward: exp(-2 pi i m/64); inverse: conjugate), m a
// compile-time constant after unrolling.  Quarter turns are exact.
template <bool INV>
__device__ __forceinline__ float2 twmul64(float2 a, int m) {
  m &= 63;
  if (m == 0) return a;
  if (m == 16) return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
  if (m == 32) return make_float2(-a.x, -a.y);
  if (m == 48) return INV ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
  const int q = m >> 4, r = m & 15;
  float c, s;  // cos/sin(2 pi m / 64)
  if (q == 0) { c = qcos64(r); s = qcos64(16 - r); }
  else if (q == 1) { c = -qcos64(16 - r); s = qcos64(r); }
  else if (q == 2) { c = -qcos64(r); s = -qcos64(16 - r); }
  else { c = qcos64(16 - r); s = -qcos64(r); }
  if (!INV) s = -s;
  return cmul(a, make_float2(c, s));
}

__host__ __device__ constexpr int bitrev(int k, int n) {
  int r = 0;
  for (int i = 1; i < n; i <<= 1) { r = (r << 1) | (k & 1); k >>= 1; }
  return r;
}

// In-register N-point DFT (N <= 64, power of two) on x[OFF + STRIDE*i], natural
// order in and out.  Radix-2 decimation in frequency, then a register rename.
template <int N, bool INV, int STRIDE = 1, int OFF = 0, int LEN>
__device__ __forceinline__ void dft_reg(float2 (&x)[LEN]) {
  if constexpr (N == 1) {
    return;
  } else if constexpr (N == 2) {
    float2 a = x[OFF], b = x[OFF + STRIDE];
    x[OFF] = cadd(a, b);
    x[OFF + STRIDE] = csub(a, b);
  } else {
#pragma unroll
    for (int half = N / 2; half >= 1; half >>= 1) {
#pragma unroll
      for (int blk = 0; blk < N; blk += 2 * half) {
#pragma unroll
        for (int j = 0; j < half; ++j) {
          const int i0 = OFF + STRIDE * (blk + j), i1 = OFF + STRIDE * (blk + j + half);
          float2 a = x[i0], b = x[i1];
          x[i0] = cadd(a, b);
          x[i1] = twmul64<INV>(csub(a, b), j * (64 / (2 * half)));
        }
      }
    }
    float2 y[N];
#pragma unroll
    for (int k = 0; k < N; ++k) y[k] = x[OFF + STRIDE * bitrev(k, N)];
#pragma unroll
    for (int k = 0; k < N; ++k) x[OFF + STRIDE * k] = y[k];
  }
}

// ---------------------------------------------------------------------------
// 2-D engine
// ---------------------------------------------------------------------------
template <int N> struct FftCfg;
template <> struct FftCfg<64> { static constexpr int A = 16, B = 4, C = 4, D = 16; };
template <> struct FftCfg<128> { static constexpr int A = 32, B = 4, C = 8, D = 16; };

template <int N>
struct Fft2 {
  static constexpr int A = FftCfg<N>::A, B = FftCfg<N>::B, C = FftCfg<N>::C, D = FftCfg<N>::D;
  static constexpr int T = 4 * N;        // threads per CTA
  static constexpr int E = N / 4;        // complex registers per thread
  static constexpr int G3 = E / D;       // S3 groups per thread
  static constexpr int PITCH = N + 1;    // shared-memory row pitch (float2)
  static constexpr int SM_FLOAT2 = N * PITCH;
  static_assert(A * B == N && C * D == N, "bad factorisation");
  static_assert(B * C == E && G3 * D == E && A == E, "stage sizes must match");

  // stage coordinates of this thread
  int s1_r, s1_cB;       // S1: row, column residue
  int s2_rD, s2_kA;      // S2
  int s3_c, s3_kC0;      // S3: column, first kC (group g adds 4*g)

  __device__ __forceinline__ void init(int tid) {
    const int lane = tid & 31, w = tid >> 5;
    s1_cB = lane & 3;
    s1_r = (w & 3) + 4 * (lane >> 2) + 32 * (w >> 2);
    s2_rD = lane & 15;
    s2_kA = (lane >> 4) + 2 * w;
    constexpr int CW = N / 32;  // warps per 32-column strip
    s3_c = lane + 32 * (w % CW);
    s3_kC0 = w / CW;
  }
  __device__ __forceinline__ int s3_kC(int g) const { return s3_kC0 + (T / 32 / (N / 32)) * g; }
  // natural (row, col) of S1 register e
  __device__ __forceinline__ int s1_col(int e) const { return s1_cB + B * e; }
  // frequency row of S3 register (g, e)
  __device__ __forceinline__ int s3_row(int g, int e) const { return s3_kC(g) + C * e; }

  // ---- exchanges (caller guarantees all prior reads of sm are complete) ----
  __device__ __forceinline__ void write_s1(float2* sm, const float2 (&x)[E]) const {
#pragma unroll
    for (int e = 0; e < A; ++e) sm[s1_r * PITCH + s1_cB + B * e] = x[e];
  }
  __device__ __forceinline__ void read_s1(const float2* sm, float2 (&x)[E]) const {
#pragma unroll
    for (int e = 0; e < A; ++e) x[e] = sm[s1_r * PITCH + s1_cB + B * e];
  }
  // S2 input layout (cB, rC): element (rD + D rC, cB + B kA)
  __device__ __forceinline__ void read_s2_in(const float2* sm, float2 (&x)[E]) const {
#pragma unroll
    for (int cB = 0; cB < B; ++cB)
#pragma unroll
      for (int rC = 0; rC < C; ++rC) x[cB * C + rC] = sm[(s2_rD + D * rC) * PITCH + cB + B * s2_kA];
  }
  __device__ __forceinline__ void write_s2_in(float2* sm, const float2 (&x)[E]) const {
#pragma unroll
    for (int cB = 0; cB < B; ++cB)
#pragma unroll
      for (int rC = 0; rC < C; ++rC) sm[(s2_rD + D * rC) * PITCH + cB + B * s2_kA] = x[cB * C + rC];
  }
  // S2 output layout (kB, kC): element (rD + D kC, kA + A kB)
  __device__ __forceinline__ void write_s2_out(float2* sm, const float2 (&x)[E]) const {
#pragma unroll
    for (int kB = 0; kB < B; ++kB)
#pragma unroll
      for (int kC = 0; kC < C; ++kC) sm[(s2_rD + D * kC) * PITCH + s2_kA + A * kB] = x[kB * C + kC];
  }
  __device__ __forceinline__ void read_s2_out(const float2* sm, float2 (&x)[E]) const {
#pragma unroll
    for (int kB = 0; kB < B; ++kB)
#pragma unroll
      for (int kC = 0; kC < C; ++kC) x[kB * C + kC] = sm[(s2_rD + D * kC) * PITCH + s2_kA + A * kB];
  }
  // S3 layout (g, e): element (e + D kC_g, col)
  __device__ __forceinline__ void read_s3(const float2* sm, float2 (&x)[E]) const {
#pragma unroll
    for (int g = 0; g < G3; ++g)
#pragma unroll
      for (int e = 0; e < D; ++e) x[g * D + e] = sm[(e + D * s3_kC(g)) * PITCH + s3_c];
  }
  __device__ __forceinline__ void write_s3(float2* sm, const float2 (&x)[E]) const {
#pragma unroll
    for (int g = 0; g < G3; ++g)
#pragma unroll
      for (int e = 0; e < D; ++e) sm[(e + D * s3_kC(g)) * PITCH + s3_c] = x[g * D + e];
  }

  // ---- register stages ----
  template <bool INV>
  __device__ __forceinline__ void s1(float2 (&x)[E]) const { dft_reg<A, INV, 1, 0>(x); }

  template <bool INV>
  __device__ __forceinline__ void s3(float2 (&x)[E]) const {
#pragma unroll
    for (int g = 0; g < G3; ++g) {
      if (g == 0) dft_reg<D, INV, 1, 0>(x);
      else dft_reg<D, INV, 1, D>(x);  // G3 <= 2 for the supported sizes
    }
  }

  // S2 forward: x holds (cB, rC) on entry, (kB, kC) on exit.  tw = w_N^k table.
  __device__ __forceinline__ void s2_fwd(float2 (&x)[E], const float2* tw) const {
#pragma unroll
    for (int cB = 1; cB < B; ++cB) {
      const float2 w = tw[(cB * s2_kA) & (N - 1)];
#pragma unroll
      for (int rC = 0; rC < C; ++rC) x[cB * C + rC] = QB_F32X2_S2 ? pcmul(x[cB * C + rC], w) : cmul(x[cB * C + rC], w);
    }
    s2_core<false>(x);
#pragma unroll
    for (int kC = 1; kC < C; ++kC) {
      const float2 w = tw[(s2_rD * kC) & (N - 1)];
#pragma unroll
      for (int kB = 0; kB < B; ++kB) x[kB * C + kC] = QB_F32X2_S2 ? pcmul(x[kB * C + kC], w) : cmul(x[kB * C + kC], w);
    }
  }
  // S2 inverse: (kB, kC) on entry, (cB, rC) on exit.
  __device__ __forceinline__ void s2_inv(float2 (&x)[E], const float2* tw) const {
#pragma unroll
    for (int kC = 1; kC < C; ++kC) {
      const float2 w = tw[(s2_rD * kC) & (N - 1)];
#pragma unroll
      for (int kB = 0; kB < B; ++kB) x[kB * C + kC] = QB_F32X2_S2 ? pcmulc(x[kB * C + kC], w) : cmulc(x[kB * C + kC], w);
    }
    s2_core<true>(x);
#pragma unroll
    for (int cB = 1; cB < B; ++cB) {
      const float2 w = tw[(cB * s2_kA) & (N - 1)];
#pragma unroll
      for (int rC = 0; rC < C; ++rC) x[cB * C + rC] = QB_F32X2_S2 ? pcmulc(x[cB * C + rC], w) : cmulc(x[cB * C + rC], w);
    }
  }
  // B-point DFT along index 0 (stride C) and C-point DFT along index 1 (stride 1).
  template <bool INV>
  __device__ __forceinline__ void s2_core(float2 (&x)[E]) const {
    s2_bdft<INV, 0>(x);
    s2_cdft<INV, 0>(x);
  }
  template <bool INV, int RC>
  __device__ __forceinline__ void s2_bdft(float2 (&x)[E]) const {
    if constexpr (RC < C) {
      dft_reg<B, INV, C, RC>(x);
      s2_bdft<INV, RC + 1>(x);
    }
  }
  template <bool INV, int KB>
  __device__ __forceinline__ void s2_cdft(float2 (&x)[E]) const {
    if constexpr (KB < B) {
      dft_reg<C, INV, 1, KB * C>(x);
      s2_cdft<INV, KB + 1>(x);
    }
  }

  // ---- whole transforms between layouts (each exchange brackets with barriers) ----
  // Forward: registers in S1 layout -> registers in S3 layout (unnormalised).
  __device__ __forceinline__ void forward(float2 (&x)[E], float2* sm, const float2* tw) const {
    s1<false>(x);
    __syncthreads();
    write_s1(sm, x);
    __syncthreads();
    read_s2_in(sm, x);
    s2_fwd(x, tw);
    __syncthreads();
    write_s2_out(sm, x);
    __syncthreads();
    read_s3(sm, x);
    s3<false>(x);
  }
  // Inverse: registers in S3 layout -> registers in S1 layout (unnormalised).
  __device__ __forceinline__ void inverse(float2 (&x)[E], float2* sm, const float2* tw) const {
    s3<true>(x);
    __syncthreads();
    write_s3(sm, x);
    __syncthreads();
    read_s2_out(sm, x);
    s2_inv(x, tw);
    __syncthreads();
    write_s2_in(sm, x);
    __syncthreads();
    read_s1(sm, x);
    s1<true>(x);
  }
};

// ---------------------------------------------------------------------------
// mixed radix (N = 3 * 2^k) for 96 x 96 windows
// ---------------------------------------------------------------------------
// cos(2*pi*m/96) for m = 0..24 (first quadrant), IEEE double rounded to float.
__device__ __forceinline__ float qcos96(int m) {
  switch (m) {
    case 0: return 1.0f;
    case 1: return 0.9978589232386035f;
    case 2: return 0.9914448613738104f;
    case 3: return 0.9807852804032304f;
    case 4: return 0.9659258262890683f;
    case 5: return 0.9469301294951057f;
    case 6: return 0.9238795325112867f;
    case 7: return 0.8968727415326884f;
    case 8: return 0.8660254037844387f;
    case 9: return 0.8314696123025452f;
    case 10: return 0.7933533402912352f;
    case 11: return 0.7518398074789774f;
    case 12: return 0.7071067811865476f;
    case 13: return 0.6593458151000688f;
    case 14: return 0.6087614290087207f;
    case 15: return 0.5555702330196024f;
    case 16: return 0.5000000000000001f;
    case 17: return 0.44228869021900125f;
    case 18: return 0.38268343236508984f;
    case 19: return 0.3214394653031617f;
    case 20: return 0.25881904510252074f;
    case 21: return 0.19509032201612833f;
    case 22: return 0.1305261922200517f;
    case 23: return 0.06540312923014327f;
    default: return 0.0f;
  }
}
// Multiply by w_96^m (forward exp(-2 pi i m/96), inverse its conjugate); m a
// compile-time constant after unrolling, quarter turns exact.
template <bool INV>
__device__ __forceinline__ float2 twmul96(float2 a, int m) {
  m %= 96;
  if (m < 0) m += 96;
  if (m == 0) return a;
  if (m == 24) return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
  if (m == 48) return make_float2(-a.x, -a.y);
  if (m == 72) return INV ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
  const int q = m / 24, r = m % 24;
  float c, s;  // cos / sin(2 pi m / 96)
  if (q == 0) { c = qcos96(r); s = qcos96(24 - r); }
  else if (q == 1) { c = -qcos96(24 - r); s = qcos96(r); }
  else if (q == 2) { c = -qcos96(r); s = -qcos96(24 - r); }
  else { c = qcos96(24 - r); s = -qcos96(r); }
  if (!INV) s = -s;
  return cmul(a, make_float2(c, s));
}
// 3-point DFT in place: (a, b, c) -> (X0, X1, X2), w3 = exp(-+2 pi i / 3).
template <bool INV>
__device__ __forceinline__ void dft3(float2& a, float2& b, float2& c) {
  const float h = 0.8660254037844386f;  // sin(pi / 3)
  const float2 t1 = cadd(b, c);
  const float2 t2 = make_float2(fmaf(-0.5f, t1.x, a.x), fmaf(-0.5f, t1.y, a.y));
  const float2 d = csub(b, c);
  // forward: -i * sin(pi/3) * (b - c); inverse: +i * sin(pi/3) * (b - c)
  const float2 t3 = INV ? make_float2(-h * d.y, h * d.x) : make_float2(h * d.y, -h * d.x);
  a = cadd(a, t1);
  b = cadd(t2, t3);
  c = csub(t2, t3);
}
// In-register N-point DFT for N = 3*M (M a power of two) or a power of two, on
// x[OFF + STRIDE*i], natural order in and out: three M-point DFTs over the
// residues of i mod 3, twiddles w_N^(r*k), M three-point DFTs, register rename.
template <int N, bool INV, int STRIDE = 1, int OFF = 0, int LEN>
__device__ __forceinline__ void dft_reg_n(float2 (&x)[LEN]) {
  if constexpr ((N & (N - 1)) == 0) {
    dft_reg<N, INV, STRIDE, OFF>(x);
  } else {
    static_assert(N % 3 == 0 && ((N / 3) & (N / 3 - 1)) == 0 && 96 % N == 0, "N = 3 * 2^k dividing 96");
    constexpr int M = N / 3;
    dft_reg<M, INV, 3 * STRIDE, OFF>(x);
    dft_reg<M, INV, 3 * STRIDE, OFF + STRIDE>(x);
    dft_reg<M, INV, 3 * STRIDE, OFF + 2 * STRIDE>(x);
#pragma unroll
    for (int k = 1; k < M; ++k) {
      x[OFF + STRIDE * (3 * k + 1)] = twmul96<INV>(x[OFF + STRIDE * (3 * k + 1)], (96 / N) * k);
      x[OFF + STRIDE * (3 * k + 2)] = twmul96<INV>(x[OFF + STRIDE * (3 * k + 2)], (96 / N) * 2 * k);
    }
#pragma unroll
    for (int k = 0; k < M; ++k)
      dft3<INV>(x[OFF + STRIDE * (3 * k)], x[OFF + STRIDE * (3 * k + 1)], x[OFF + STRIDE * (3 * k + 2)]);
    float2 y[N];  // X[k + M j] sits at position 3k + j
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) y[k + M * j] = x[OFF + STRIDE * (3 * k + j)];
#pragma unroll
    for (int i = 0; i < N; ++i) x[OFF + STRIDE * i] = y[i];
  }
}

// 96 x 96 engine: T = 192 threads (6 warps), E = 48 complex registers each.
//   columns c = cB + 2*cA (A = 48, B = 2), rows r = rD + 4*rC (C = 24, D = 4)
//   S1: 48-point DFT over cA for fixed (r, cB)               -> kA
//   S2: twiddle w96^(cB*kA); 2-point over cB; 24-point over rC; twiddle w96^(rD*kC)
//   S3: 4-point DFT over rD for 12 (kC, column) groups        -> kD
// Exchange layouts (float2 index): stage 1<->2 element (r, cB, kA) at r + 100 kA + 4800 cB,
// stage 2<->3 element (row, col) at 104 row + col; both verified to give two wavefronts per
// warp access with the lane maps of init().
template <>
struct Fft2<96> {
  static constexpr int N = 96, A = 48, B = 2, C = 24, D = 4;
  static constexpr int T = 192;
  static constexpr int E = 48;
  static constexpr int G3 = 12;
  static constexpr int SM_FLOAT2 = 9976;

  int s1_r, s1_cB;
  int s2_rD, s2_kA;
  int s3_c, s3_kC0;

  __device__ __forceinline__ void init(int tid) {
    const int lane = tid & 31, w = tid >> 5;
    s1_r = (lane & 15) + 16 * w;
    s1_cB = lane >> 4;
    s2_rD = lane & 3;
    s2_kA = (lane >> 2) + 8 * w;
    s3_c = lane + 32 * (w % 3);
    s3_kC0 = w / 3;
  }
  __device__ __forceinline__ int s3_kC(int g) const { return s3_kC0 + 2 * g; }
  __device__ __forceinline__ int s1_col(int e) const { return s1_cB + B * e; }
  __device__ __forceinline__ int s3_row(int g, int e) const { return s3_kC(g) + C * e; }

  __device__ __forceinline__ void write_s1(float2* sm, const float2 (&x)[E]) const {
    float2* w = sm + s1_r + 4800 * s1_cB;
#pragma unroll
    for (int e = 0; e < A; ++e) w[100 * e] = x[e];
  }
  __device__ __forceinline__ void read_s1(const float2* sm, float2 (&x)[E]) const {
    const float2* r = sm + s1_r + 4800 * s1_cB;
#pragma unroll
    for (int e = 0; e < A; ++e) x[e] = r[100 * e];
  }
  // S2 input layout (cB, rC): element (rD + 4 rC, cB, kA)
  __device__ __forceinline__ void read_s2_in(const float2* sm, float2 (&x)[E]) const {
    const float2* r = sm + s2_rD + 100 * s2_kA;
#pragma unroll
    for (int cB = 0; cB < B; ++cB)
#pragma unroll
      for (int rC = 0; rC < C; ++rC) x[cB * C + rC] = r[4 * rC + 4800 * cB];
  }
  __device__ __forceinline__ void write_s2_in(float2* sm, const float2 (&x)[E]) const {
    float2* w = sm + s2_rD + 100 * s2_kA;
#pragma unroll
    for (int cB = 0; cB < B; ++cB)
#pragma unroll
      for (int rC = 0; rC < C; ++rC) w[4 * rC + 4800 * cB] = x[cB * C + rC];
  }
  // S2 output layout (kB, kC): element (row rD + 4 kC, col kA + 48 kB)
  __device__ __forceinline__ void write_s2_out(float2* sm, const float2 (&x)[E]) const {
    float2* w = sm + 104 * s2_rD + s2_kA;
#pragma unroll
    for (int kB = 0; kB < B; ++kB)
#pragma unroll
      for (int kC = 0; kC < C; ++kC) w[416 * kC + 48 * kB] = x[kB * C + kC];
  }
  __device__ __forceinline__ void read_s2_out(const float2* sm, float2 (&x)[E]) const {
    const float2* r = sm + 104 * s2_rD + s2_kA;
#pragma unroll
    for (int kB = 0; kB < B; ++kB)
#pragma unroll
      for (int kC = 0; kC < C; ++kC) x[kB * C + kC] = r[416 * kC + 48 * kB];
  }
  // S3 layout (g, e): element (row e + 4 kC_g, col)
  __device__ __forceinline__ void read_s3(const float2* sm, float2 (&x)[E]) const {
    const float2* r = sm + 104 * 4 * s3_kC0 + s3_c;
#pragma unroll
    for (int g = 0; g < G3; ++g)
#pragma unroll
      for (int e = 0; e < D; ++e) x[g * D + e] = r[104 * (e + 8 * g)];
  }
  __device__ __forceinline__ void write_s3(float2* sm, const float2 (&x)[E]) const {
    float2* w = sm + 104 * 4 * s3_kC0 + s3_c;
#pragma unroll
    for (int g = 0; g < G3; ++g)
#pragma unroll
      for (int e = 0; e < D; ++e) w[104 * (e + 8 * g)] = x[g * D + e];
  }

  template <bool INV>
  __device__ __forceinline__ void s1(float2 (&x)[E]) const { dft_reg_n<A, INV, 1, 0>(x); }
  template <bool INV, int G>
  __device__ __forceinline__ void s3_groups(float2 (&x)[E]) const {
    if constexpr (G < G3) {
      dft_reg<D, INV, 1, G * D>(x);
      s3_groups<INV, G + 1>(x);
    }
  }
  template <bool INV>
  __device__ __forceinline__ void s3(float2 (&x)[E]) const { s3_groups<INV, 0>(x); }

  template <bool INV>
  __device__ __forceinline__ void s2_core(float2 (&x)[E]) const {
#pragma unroll
    for (int rC = 0; rC < C; ++rC) {  // 2-point DFT over cB
      const float2 a = x[rC], b = x[C + rC];
      x[rC] = cadd(a, b);
      x[C + rC] = csub(a, b);
    }
    dft_reg_n<C, INV, 1, 0>(x);
    dft_reg_n<C, INV, 1, C>(x);
  }
  __device__ __forceinline__ void s2_fwd(float2 (&x)[E], const float2* tw) const {
    const float2 w1 = tw[s2_kA];  // w96^(1 * kA)
#pragma unroll
    for (int rC = 0; rC < C; ++rC) x[C + rC] = cmul(x[C + rC], w1);
    s2_core<false>(x);
#pragma unroll
    for (int kC = 1; kC < C; ++kC) {
      const float2 w = tw[s2_rD * kC];  // rD * kC <= 69 < 96
#pragma unroll
      for (int kB = 0; kB < B; ++kB) x[kB * C + kC] = cmul(x[kB * C + kC], w);
    }
  }
  __device__ __forceinline__ void s2_inv(float2 (&x)[E], const float2* tw) const {
#pragma unroll
    for (int kC = 1; kC < C; ++kC) {
      const float2 w = tw[s2_rD * kC];
#pragma unroll
      for (int kB = 0; kB < B; ++kB) x[kB * C + kC] = cmulc(x[kB * C + kC], w);
    }
    s2_core<true>(x);
    const float2 w1 = tw[s2_kA];
#pragma unroll
    for (int rC = 0; rC < C; ++rC) x[C + rC] = cmulc(x[C + rC], w1);
  }

  __device__ __forceinline__ void forward(float2 (&x)[E], float2* sm, const float2* tw) const {
    s1<false>(x);
    __syncthreads();
    write_s1(sm, x);
    __syncthreads();
    read_s2_in(sm, x);
    s2_fwd(x, tw);
    __syncthreads();
    write_s2_out(sm, x);
    __syncthreads();
    read_s3(sm, x);
    s3<false>(x);
  }
  __device__ __forceinline__ void inverse(float2 (&x)[E], float2* sm, const float2* tw) const {
    s3<true>(x);
    __syncthreads();
    write_s3(sm, x);
    __syncthreads();
    read_s2_out(sm, x);
    s2_inv(x, tw);
    __syncthreads();
    write_s2_in(sm, x);
    __syncthreads();
    read_s1(sm, x);
    s1<true>(x);
  }
};

}  // namespace qb
