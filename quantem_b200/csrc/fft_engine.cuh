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
// 512 threads).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qb {

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
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
      for (int rC = 0; rC < C; ++rC) x[cB * C + rC] = cmul(x[cB * C + rC], w);
    }
    s2_core<false>(x);
#pragma unroll
    for (int kC = 1; kC < C; ++kC) {
      const float2 w = tw[(s2_rD * kC) & (N - 1)];
#pragma unroll
      for (int kB = 0; kB < B; ++kB) x[kB * C + kC] = cmul(x[kB * C + kC], w);
    }
  }
  // S2 inverse: (kB, kC) on entry, (cB, rC) on exit.
  __device__ __forceinline__ void s2_inv(float2 (&x)[E], const float2* tw) const {
#pragma unroll
    for (int kC = 1; kC < C; ++kC) {
      const float2 w = tw[(s2_rD * kC) & (N - 1)];
#pragma unroll
      for (int kB = 0; kB < B; ++kB) x[kB * C + kC] = cmulc(x[kB * C + kC], w);
    }
    s2_core<true>(x);
#pragma unroll
    for (int cB = 1; cB < B; ++cB) {
      const float2 w = tw[(cB * s2_kA) & (N - 1)];
#pragma unroll
      for (int rC = 0; rC < C; ++rC) x[cB * C + rC] = cmulc(x[cB * C + rC], w);
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

}  // namespace qb
