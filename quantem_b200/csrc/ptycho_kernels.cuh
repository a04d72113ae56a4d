// Multislice mixed-probe ptychography kernels for sm_100a.
//
// fused_batch_kernel<N, ADJ>: one CTA per scan position at a time (persistent
// grid-stride loop).  For every probe mode the CTA builds the sub-pixel shifted
// probe from the Fourier-space probe and a separable phase ramp, runs the
// multislice recursion (transmission by the gathered object patch, Fresnel
// propagation by FFT * propagator * IFFT), forms the far field with an
// orthonormal FFT and accumulates |Psi|^2 over modes in shared memory.  The loss
// and dL/dI follow in the same pass.  With ADJ the CTA then runs the adjoint for
// every mode: back-projection through the detector FFT, reverse slices with
// conjugate transmission / propagator, scatter-add of the object gradient
// (float2 atomics) and accumulation of the Fourier-space probe gradient into a
// per-CTA partial.  Incoming waves of every slice are kept in a per-CTA scratch
// slot between forward and adjoint.
//
// Reference behaviour (quantem.diffractive_imaging):
//   probe shift      ptycho_utils.py:128-176, probe_models.py:718-720
//   patch gather     object_models.py:252-265, dataset_models.py:514-535,1487-1490
//   multislice       ptychography_base.py:934-947, 970-989
//   detector         detector_models.py:22-30
//   loss             ptychography_base.py:908-932
//   autograd         ptychography.py:326-332 (torch complex-gradient convention)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_engine.cuh"

namespace qb {

enum LossType : int {
  LOSS_L2_AMPLITUDE = 0,
  LOSS_L1_AMPLITUDE = 1,
  LOSS_L2_INTENSITY = 2,
  LOSS_L1_INTENSITY = 3,
  LOSS_POISSON = 4,
};

struct BatchParams {
  const float2* obj;          // constrained object (S, Ho, Wo)
  const float2* probe_hat;    // fft2 of the orthogonalised probes (P, N, N)
  const float2* prop;         // propagators (S-1, N, N), used when prop_r is null
  const float2* prop_r;       // separable propagator row factors (S-1, N) or null
  const float2* prop_c;       // separable propagator column factors (S-1, N)
  const float* positions;     // (npos, 2) scan positions [px]
  const int64_t* batch_idx;   // (B,) indices into positions / targets
  const float* targets;       // (npos, N, N) detector (centred) layout
  const float* mask;          // (N, N) detector layout
  float2* grad_obj;           // (S, Ho, Wo) accumulated, ADJ only
  float2* probe_grad_part;    // (grid, P, N, N) per-CTA Fourier partials, ADJ only
  float2* scratch;            // (grid, P*S + P, N*N), ADJ only
  double* loss_part;          // (grid,) per-CTA loss partial sums
  float* out_intensity;       // optional (B, N, N) detector layout
  float2* out_exit;           // optional (P, B, N, N) exit waves
  float2* out_waves;          // optional (S, P, B, N, N) incoming wave of each slice
  int* status;                // optional non-finite counter
  int S, P, B, Ho, Wo, npos;
  float loss_scale;           // num_gpts / (B * mean_intensity)
  float inv_mean_intensity;   // 1 / mean_intensity (poisson)
  int loss_type;
  int analytic;               // 0: autograd adjoint; 1: analytic update (ptychography.py:339-372), serial kernel
  float* an_norm;             // (S, P, Ho, Wo) scatter of |psi|^2 for the analytic normalisation
  int ckpt;                   // 256^2 cluster kernel: checkpoint interval of the adjoint (0 = keep all waves)
  float* grad_positions;      // optional (B, 2) dL/d(position), serial autograd adjoint only
  const float* descan;        // optional (npos, 2) descan shifts [px] applied to the exit wave
  float* grad_descan;         // optional (B, 2) dL/d(descan), serial autograd adjoint only
  float* grad_prop;           // optional (S-1, 2) propagator sensitivities, serial autograd adjoint only
};

// Status word of the batch kernels: bits 0-19 count non-finite predicted
// intensities, bits 20-30 count batch indices outside [0, npos).  Each field
// saturates at its maximum instead of carrying into the next one (a NaN object at
// thousands of positions x 128^2 pixels would otherwise overflow the first field
// into the second).  A bounded compare-and-swap loop; it runs only on error paths.
constexpr int kStatusNonfiniteBits = 20;
constexpr int kStatusInvalidShift = 20;
constexpr int kStatusInvalidBits = 11;
__device__ __forceinline__ void status_add(int* st, int shift, int bits, int n) {
  if (!st || n <= 0) return;
  const unsigned fmask = (1u << bits) - 1u;
  unsigned old = *reinterpret_cast<volatile unsigned*>(st);
  for (int it = 0; it < 4096; ++it) {
    const unsigned cur = (old >> shift) & fmask;
    const unsigned add = (unsigned)n < fmask - cur ? (unsigned)n : fmask - cur;
    if (add == 0) return;
    const unsigned want = old + (add << shift);
    const unsigned seen = atomicCAS(reinterpret_cast<unsigned*>(st), old, want);
    if (seen == old) return;
    old = seen;
  }
}
__device__ __forceinline__ void status_add_nonfinite(int* st, int n) { status_add(st, 0, kStatusNonfiniteBits, n); }
__device__ __forceinline__ void status_add_invalid(int* st, int n) {
  status_add(st, kStatusInvalidShift, kStatusInvalidBits, n);
}

__device__ __forceinline__ int fsigned(int k, int n) { return k < n / 2 ? k : k - n; }
__device__ __forceinline__ int wrap_index(int x, int n) {
  x %= n;
  return x < 0 ? x + n : x;
}

// Object patches are re-read by every mode and slice of a position and by the
// neighbouring positions of the batch: keep them in L2 (evict-last policy) while the
// saved waves and the measured targets stream through it.  Measured on the full
// 4096-position batch: 29.58 -> 29.29 ms (with the reversed adjoint mode order).
__device__ __forceinline__ uint64_t evict_last_policy() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// saved data read back once: skip L1 allocation so the object lines stay resident there
__device__ __forceinline__ float4 ld_stream4(const float4* ptr) {
  float4 v;
  asm volatile("ld.global.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(ptr));
  return v;
}
__device__ __forceinline__ float2 ld_obj(const float2* ptr, uint64_t pol) {
  float2 v;
  asm("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(ptr), "l"(pol));
  return v;
}

// Saved per-thread register arrays (waves, far fields, checkpoints) are stored
// thread-major with the register pair (e, e+1) packed into one 16-byte word:
// element e of thread tid lives in word (e / 2) * T + tid, so a warp moves 512
// contiguous bytes per access and a thread issues E / 2 vector accesses.
template <int E, int T>
__device__ __forceinline__ void store_pairs(float2* dst, int tid, const float2 (&x)[E]) {
  float4* d = reinterpret_cast<float4*>(dst) + tid;
#pragma unroll
  for (int e = 0; e < E; e += 2)
    asm volatile("st.global.L1::no_allocate.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(d + (e >> 1) * T),
                 "f"(x[e].x), "f"(x[e].y), "f"(x[e + 1].x), "f"(x[e + 1].y) : "memory");
}
template <int E, int T>
__device__ __forceinline__ void load_pairs(const float2* src, int tid, float2 (&x)[E]) {
  const float4* s = reinterpret_cast<const float4*>(src) + tid;
#pragma unroll
  for (int e = 0; e < E; e += 2) {
    const float4 v = s[(e >> 1) * T];
    x[e] = make_float2(v.x, v.y);
    x[e + 1] = make_float2(v.z, v.w);
  }
}

// shared-memory bytes used by fused_batch_kernel<N, *> (without the separable
// propagator factors, which add 2 * N * (S-1) float2 when used)
template <int N>
constexpr size_t fused_smem_bytes() {
  return sizeof(float2) * (size_t)(Fft2<N>::SM_FLOAT2 + 3 * N) + sizeof(float) * (size_t)N * N +
         sizeof(int) * (size_t)(2 * N);
}
template <int N>
constexpr size_t fused_smem_bytes_sep(int S) {
  return fused_smem_bytes<N>() + sizeof(float2) * (size_t)2 * N * (size_t)(S > 1 ? S - 1 : 0);
}
// The adjoint kernel keeps its intensity / dL/dI tile in its global scratch slot
// (L2-resident, 64 KB per CTA at 128^2) instead of shared memory; the 64 KB left
// to the L1 cache hold the register spills of the 512-thread CTA.
template <int N, bool ADJ>
constexpr size_t batch_smem_bytes(bool sep, int S) {
  return (sep ? fused_smem_bytes_sep<N>(S) : fused_smem_bytes<N>()) - (ADJ ? sizeof(float) * (size_t)N * N : 0);
}

template <int N>
__device__ __forceinline__ void loss_elem(const BatchParams& p, float I, float t, float m,
                                          double& acc, float& dldi) {
  switch (p.loss_type) {
    case LOSS_L2_AMPLITUDE: {
      const float a = sqrtf(I + 1e-9f);
      const float d = a * m - t * m;
      acc += (double)d * d;
      dldi = p.loss_scale * d * m / a;
      break;
    }
    case LOSS_L1_AMPLITUDE: {
      const float a = sqrtf(I + 1e-9f);
      const float d = a * m - t * m;
      acc += fabs((double)d);
      const float sg = d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f);
      dldi = p.loss_scale * sg * m * 0.5f / a;
      break;
    }
    case LOSS_L2_INTENSITY: {
      const float d = I * m - t * m;
      acc += (double)d * d;
      dldi = p.loss_scale * 2.f * d * m;
      break;
    }
    case LOSS_L1_INTENSITY: {
      const float d = I * m - t * m;
      acc += fabs((double)d);
      const float sg = d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f);
      dldi = p.loss_scale * sg * m;
      break;
    }
    default: {  // poisson: sum(I - t log(I + 1e-6)) / mean_I
      acc += (double)I - (double)t * log((double)I + 1e-6);
      dldi = p.inv_mean_intensity * (1.f - t / (I + 1e-6f));
      break;
    }
  }
}

// x (S3 layout, Fourier space) *= K_s (CONJ: conj(K_s)), separable factors from
// shared memory or the full (S-1, N, N) array from global memory.
template <int N, bool CONJ>
__device__ __forceinline__ void apply_prop(const Fft2<N>& f, float2 (&x)[Fft2<N>::E], const BatchParams& p, int s,
                                           bool sep, const float2* sKr, const float2* sKc) {
  constexpr int D = Fft2<N>::D, G3 = Fft2<N>::G3;
  if (sep) {
#pragma unroll
    for (int g = 0; g < G3; ++g) {
      const float2 kc = sKc[s * N + f.s3_c];
#pragma unroll
      for (int e = 0; e < D; ++e) {
        const float2 k = cmul(sKr[s * N + f.s3_row(g, e)], kc);
        x[g * D + e] = CONJ ? cmulc(x[g * D + e], k) : cmul(x[g * D + e], k);
      }
    }
  } else {
    const float2* pr = p.prop + (size_t)s * N * N;
#pragma unroll
    for (int g = 0; g < G3; ++g)
#pragma unroll
      for (int e = 0; e < D; ++e) {
        const float2 k = __ldg(pr + (size_t)f.s3_row(g, e) * N + f.s3_c);
        x[g * D + e] = CONJ ? cmulc(x[g * D + e], k) : cmul(x[g * D + e], k);
      }
  }
}

// x (S1 layout) *= o (CONJ: conj(o)) for the object row orow_ptr, columns through
// colmap.  Loads go in batches of 8 so that a batch is in flight at once while
// the wave occupies half of the register file.
template <int N, bool CONJ>
__device__ __forceinline__ void gather_mul(const Fft2<N>& f, float2 (&x)[Fft2<N>::E], const float2* orow_ptr,
                                           const int* colmap, uint64_t pol) {
  constexpr int E = Fft2<N>::E;
#pragma unroll
  for (int e0 = 0; e0 < E; e0 += 8) {
    float2 ob[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) ob[j] = ld_obj(orow_ptr + colmap[f.s1_col(e0 + j)], pol);
#pragma unroll
    for (int j = 0; j < 8; ++j) x[e0 + j] = CONJ ? cmulc(x[e0 + j], ob[j]) : cmul(x[e0 + j], ob[j]);
  }
}

// Descan (ptychography_base.py:903-905): the exit wave (S1 layout) times the
// translation ramp of the descan shift (dr, dc) evaluated on the real-space grid,
// exp(-2 pi i (fftfreq(r) dr + fftfreq(c) dc)) (ptycho_utils.py:156-176); CONJ: its
// conjugate, for the adjoint.
template <int N, bool CONJ>
__device__ __forceinline__ void descan_mul(const Fft2<N>& f, float2 (&x)[Fft2<N>::E], float dr, float dc) {
  constexpr int E = Fft2<N>::E;
  const float ar = (float)fsigned(f.s1_r, N) * dr;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    float sn, cs;
    sincospif(-2.0f * (ar + (float)fsigned(f.s1_col(e), N) * dc) / (float)N, &sn, &cs);
    x[e] = CONJ ? cmulc(x[e], make_float2(cs, sn)) : cmul(x[e], make_float2(cs, sn));
  }
}

// Fourier-space probe-gradient partial (S3 layout): pg += conj(ramp) * x, batched RMW.
template <int N>
__device__ __forceinline__ void accumulate_probe_grad(const Fft2<N>& f, const float2 (&x)[Fft2<N>::E], float2* pg,
                                                      const float2* rowf, const float2* colf) {
  constexpr int D = Fft2<N>::D, G3 = Fft2<N>::G3;
  constexpr int BT = D < 8 ? D : 8;  // batch of read-modify-writes within one D-point group
  static_assert(D % BT == 0, "batch must divide the group");
#pragma unroll
  for (int g = 0; g < G3; ++g)
#pragma unroll
    for (int e0 = 0; e0 < D; e0 += BT) {
      float2 old[BT];
#pragma unroll
      for (int j = 0; j < BT; ++j) old[j] = pg[(size_t)f.s3_row(g, e0 + j) * N + f.s3_c];
#pragma unroll
      for (int j = 0; j < BT; ++j) {
        const int kr = f.s3_row(g, e0 + j), kc = f.s3_c;
        pg[(size_t)kr * N + kc] = cadd(old[j], cmulc(x[g * D + e0 + j], cmul(rowf[kr], colf[kc])));
      }
    }
}

// Body of the serial batch kernel for one dataset: CTA `cta` of the `ncta` CTAs
// that work on this dataset's positions.
// EXT: the optional extensions (descan shifts, position / descan / propagator gradients)
// are compiled in; the default kernel carries none of their code or registers.
template <int N, bool ADJ, bool AN = false, bool EXT = false>
__device__ __forceinline__ void serial_body(const BatchParams& p, const int cta, const int ncta) {
  // AN (compile time): analytic update directions instead of the autograd adjoint,
  // so the autograd kernel carries none of the analytic code or live values
  using F = Fft2<N>;
  constexpr int E = F::E, D = F::D, G3 = F::G3, T = F::T;
  static_assert(E % 8 == 0, "gathers and scatters go in batches of 8 registers");
  extern __shared__ float4 smem_raw[];
  float2* sm = reinterpret_cast<float2*>(smem_raw);
  float2* tw = sm + F::SM_FLOAT2;
  float2* rowf = tw + N;
  float2* colf = rowf + N;
  // intensity / dL/dI tile: shared memory (forward-only) or the CTA's scratch slot (ADJ)
  float* inten_sm = reinterpret_cast<float*>(colf + N);
  int* rowmap = reinterpret_cast<int*>(ADJ ? reinterpret_cast<float*>(colf + N) : inten_sm + N * N);
  int* colmap = rowmap + N;
  // separable propagators K_s[kr][kc] = Kr_s[kr] * Kc_s[kc] (probe_models.py:376-427
  // builds exp(-i pi lambda dz (kr^2 + kc^2)) times per-axis tilt ramps)
  float2* sKr = reinterpret_cast<float2*>(colmap + N);
  float2* sKc = sKr + (size_t)N * (p.S > 1 ? p.S - 1 : 0);
  const bool sep = p.prop_r != nullptr;
  const uint64_t pol = evict_last_policy();
  __shared__ double red[32];
  __shared__ int nfred[32];  // per-warp non-finite counts
  __shared__ float posred[32][2];  // per-warp position / descan gradient partials
  __shared__ float propred[2 * 16];  // EXT: this CTA's propagator sensitivities (S <= 17)

  const int tid = threadIdx.x;
  F f;
  f.init(tid);
  for (int k = tid; k < N; k += T) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)N, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
  if (sep) {
    for (int k = tid; k < (p.S - 1) * N; k += T) {
      sKr[k] = p.prop_r[k];
      sKc[k] = p.prop_c[k];
    }
  }
  const float inv_n = 1.0f / (float)N;
  const float inv_n2 = inv_n * inv_n;
  const size_t NN = (size_t)N * N;
  const int S = p.S, P = p.P;
  const size_t HoWo = (size_t)p.Ho * p.Wo;
  // scratch slots per CTA: P*S incident waves, P far fields, the intensity tile and (EXT
  // with propagator sensitivities) the P*(S-1) Fourier-space waves after each propagation
  const bool want_prop = EXT && ADJ && p.grad_prop != nullptr;
  const size_t nslot = (size_t)(P * S + P + 1) + (want_prop ? (size_t)P * (S - 1) : 0);
  float2* slot = ADJ ? p.scratch + (size_t)cta * nslot * NN : nullptr;
  float2* zslot = want_prop ? slot + (size_t)(P * S + P + 1) * NN : nullptr;
  if (want_prop) {
    for (int k = tid; k < 2 * 16; k += T) propred[k] = 0.f;
  }
  float* inten = ADJ ? reinterpret_cast<float*>(slot + (size_t)(P * S + P) * NN) : inten_sm;
  // Per-thread saved data (waves, far fields, intensities) is thread-major with the
  // register pair (e, e+1) packed into one word: one 16-byte (waves) or 8-byte
  // (intensities) access per pair.  Element e of this thread lives in pair word
  // (e / 2) * T + tid, half e % 2.
  float2* inten2 = reinterpret_cast<float2*>(inten);
  float2* pgrad = ADJ ? p.probe_grad_part + (size_t)cta * (size_t)P * NN : nullptr;
  if (ADJ) {
    for (int m = 0; m < P; ++m)
#pragma unroll
      for (int g = 0; g < G3; ++g)
#pragma unroll
        for (int e = 0; e < D; ++e)
          pgrad[(size_t)m * NN + (size_t)f.s3_row(g, e) * N + f.s3_c] = make_float2(0.f, 0.f);
  }
  double loss_acc = 0.0;
  int nonfinite = 0;

  // each CTA takes a contiguous block of the batch: positions processed at the same
  // time are far apart in the batch order, so raster-ordered batches do not pile
  // the object-gradient atomics of neighbouring windows onto the same addresses
  const int bchunk = (p.B + ncta - 1) / ncta;
  const int bend = min(p.B, (cta + 1) * bchunk);
  for (int b = cta * bchunk; b < bend; ++b) {
    const int64_t gi = p.batch_idx[b];
    if (gi < 0 || gi >= p.npos) {  // invalid index: skip the position and report it
      if (tid == 0) status_add_invalid(p.status, 1);
      continue;
    }
    const float py = p.positions[2 * gi], px = p.positions[2 * gi + 1];
    const float ry = rintf(py), rx = rintf(px);  // round half to even
    const float fy = py - ry, fx = px - rx;
    const int r0 = wrap_index((int)ry, p.Ho), c0 = wrap_index((int)rx, p.Wo);
    __syncthreads();  // previous position finished with rowf/colf/maps
    for (int k = tid; k < 2 * N; k += T) {
      const int kk = k < N ? k : k - N;
      const float fq = (float)fsigned(kk, N) * inv_n;         // fftfreq(N) in float32
      const float a = -6.283185307179586f * fq;                // -2 pi k
      float s, c;
      sincosf(a * (k < N ? fy : fx), &s, &c);
      if (k < N) {
        rowf[kk] = make_float2(c, s);
        rowmap[kk] = wrap_index(r0 + fsigned(kk, N), p.Ho);
      } else {
        colf[kk] = make_float2(c, s);
        colmap[kk] = wrap_index(c0 + fsigned(kk, N), p.Wo);
      }
    }
    __syncthreads();
    const int orow = rowmap[f.s1_r];

    // One loop with a single inverse and a single forward transform site walks
    // the forward chains of all modes, the loss, and (ADJ) the reverse chains.
    // x always enters the loop top in S3 (Fourier) layout.
    float2 x[E];
    auto load_probe = [&](int mm) {
      const float2* ph = p.probe_hat + (size_t)mm * NN;
#pragma unroll
      for (int g = 0; g < G3; ++g)
#pragma unroll
        for (int e = 0; e < D; ++e) {
          const int kr = f.s3_row(g, e), kc = f.s3_c;
          x[g * D + e] = cmul(cmul(__ldg(ph + (size_t)kr * N + kc), rowf[kr]), colf[kc]);
        }
    };
    // start of the reverse chain of mode mm, in S3 layout: autograd seeds the far
    // field times 2 dL/dI; the analytic update seeds the Fourier projection
    // m(Psi) - Psi = Psi (f - 1) + fix (ptychography.py:357-372), f and fix
    // stored by the loss step
    float* tile2 = ADJ ? inten + NN : nullptr;
    auto load_far_seed = [&](int mm) {
      const float2* fw = slot + (size_t)(P * S + mm) * NN;
      if (AN) {
#pragma unroll
        for (int e = 0; e < E; e += 2) {
          const float4 v = ld_stream4(reinterpret_cast<const float4*>(fw) + (e >> 1) * T + tid);
          const float2 in = inten2[(e >> 1) * T + tid];
          const float2 fx = reinterpret_cast<const float2*>(tile2)[(e >> 1) * T + tid];
          const float fm0 = in.x - 1.0f, fm1 = in.y - 1.0f;
          x[e] = make_float2(fmaf(v.x, fm0, fx.x), v.y * fm0);
          x[e + 1] = make_float2(fmaf(v.z, fm1, fx.y), v.w * fm1);
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; e += 2) {
          const float4 v = ld_stream4(reinterpret_cast<const float4*>(fw) + (e >> 1) * T + tid);
          const float2 in = inten2[(e >> 1) * T + tid];
          x[e] = make_float2(v.x * 2.0f * in.x, v.y * 2.0f * in.x);
          x[e + 1] = make_float2(v.z * 2.0f * in.y, v.w * 2.0f * in.y);
        }
      }
    };
    int m = 0, s = 0;
    bool bwd = false, first_bwd = false;
    load_probe(0);
    while (true) {
      f.inverse(x, sm, tw);
      // ---------------- real space (S1 layout) ----------------
      const float2* orow_ptr = p.obj + (size_t)s * HoWo + (size_t)orow * p.Wo;
      if (!bwd) {
#pragma unroll
        for (int e = 0; e < E; ++e) x[e] = cscale(x[e], inv_n2);
        if (ADJ) {
          float2* wv = slot + (size_t)(m * S + s) * NN;
          store_pairs<E, T>(wv, tid, x);
        }
        if (p.out_waves) {
          float2* ow = p.out_waves + (((size_t)s * P + m) * p.B + b) * NN + (size_t)f.s1_r * N;
#pragma unroll
          for (int e = 0; e < E; ++e) ow[f.s1_col(e)] = x[e];
        }
        gather_mul<N, false>(f, x, orow_ptr, colmap, pol);
        if (EXT && s == S - 1 && p.descan) descan_mul<N, false>(f, x, __ldg(p.descan + 2 * gi), __ldg(p.descan + 2 * gi + 1));
        if (s == S - 1 && p.out_exit) {
          float2* oe = p.out_exit + ((size_t)m * p.B + b) * NN + (size_t)f.s1_r * N;
#pragma unroll
          for (int e = 0; e < E; ++e) oe[f.s1_col(e)] = x[e];
        }
      } else {
        const float sc = first_bwd ? inv_n : inv_n2;  // adjoint of the orthonormal FFT, or of a propagation
        const float2* wv = slot + (size_t)(m * S + s) * NN;
        float2* grow = p.grad_obj + (size_t)s * HoWo + (size_t)orow * p.Wo;
        // the exit wave carries the descan ramp: its gradient times conj(ramp) is the
        // gradient of the last slice's transmitted wave
        if (EXT && first_bwd && p.descan)
          descan_mul<N, true>(f, x, __ldg(p.descan + 2 * gi), __ldg(p.descan + 2 * gi + 1));
#pragma unroll
        for (int e0 = 0; e0 < E; e0 += 8) {
          float2 ps[8], ob[8];
          int col[8];
#pragma unroll
          for (int j = 0; j < 8; j += 2) {
            const float4 v = ld_stream4(reinterpret_cast<const float4*>(wv) + ((e0 + j) >> 1) * T + tid);
            ps[j] = make_float2(v.x, v.y);
            ps[j + 1] = make_float2(v.z, v.w);
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            col[j] = colmap[f.s1_col(e0 + j)];
            ob[j] = ld_obj(orow_ptr + col[j], pol);
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const float2 g = cscale(x[e0 + j], sc);
            atomicAdd(grow + col[j], cmulc(g, ps[j]));  // conj(psi) * g
            x[e0 + j] = cmulc(g, ob[j]);                 // conj(o) * g
          }
          if (AN) {  // sum_patches(|psi|^2) of this slice and mode (object_models.py:701-703)
            float* nrow = p.an_norm + ((size_t)s * P + m) * HoWo + (size_t)orow * p.Wo;
#pragma unroll
            for (int j = 0; j < 8; ++j) atomicAdd(nrow + col[j], cabs2(ps[j]));
          }
        }
        if (EXT && first_bwd && p.grad_descan) {
          // x = dL/dw of the last slice's incident wave w, so conj(x) w = conj(dL/dE) E for the
          // exit wave E: dL/d(descan) = (2 pi / N) sum fftfreq_index Im(conj(x) w), summed over the modes
          float gr = 0.f, gc = 0.f;
#pragma unroll
          for (int e = 0; e < E; e += 2) {
            const float4 v = reinterpret_cast<const float4*>(wv)[(e >> 1) * T + tid];
            const float im0 = x[e].x * v.y - x[e].y * v.x;
            const float im1 = x[e + 1].x * v.w - x[e + 1].y * v.z;
            gc = fmaf((float)fsigned(f.s1_col(e), N), im0, gc);
            gc = fmaf((float)fsigned(f.s1_col(e + 1), N), im1, gc);
            gr += im0 + im1;
          }
          gr *= (float)fsigned(f.s1_r, N);
          for (int o = 16; o > 0; o >>= 1) {
            gr += __shfl_xor_sync(0xffffffffu, gr, o);
            gc += __shfl_xor_sync(0xffffffffu, gc, o);
          }
          if ((tid & 31) == 0) {
            posred[tid >> 5][0] = gr;
            posred[tid >> 5][1] = gc;
          }
          __syncthreads();
          if (tid == 0) {  // fixed-order sum over warps, accumulated over the modes of this position
            float sr = 0.f, scc = 0.f;
            for (int w = 0; w < T / 32; ++w) {
              sr += posred[w][0];
              scc += posred[w][1];
            }
            const float k = 6.283185307179586f / (float)N;
            float* out = p.grad_descan + 2 * (size_t)b;
            const bool first = m == P - 1;  // the reverse chains run last mode first
            out[0] = (first ? 0.f : out[0]) + k * sr;
            out[1] = (first ? 0.f : out[1]) + k * scc;
          }
          __syncthreads();
        }
        if (AN && s == 0) {
          // analytic probe update: sum over positions of the back-propagated
          // gradient at the probe plane, no inverse shift (probe_models.py:774-783)
          float2* pg = pgrad + (size_t)m * NN + (size_t)f.s1_r * N;
#pragma unroll
          for (int e0 = 0; e0 < E; e0 += 8) {
            float2 old[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) old[j] = pg[f.s1_col(e0 + j)];
#pragma unroll
            for (int j = 0; j < 8; ++j) pg[f.s1_col(e0 + j)] = cadd(old[j], x[e0 + j]);
          }
          if (m > 0) {
            --m;
            s = S - 1;
            first_bwd = true;
            load_far_seed(m);
            continue;
          }
          break;
        }
      }
      f.forward(x, sm, tw);
      // ---------------- Fourier space (S3 layout) ----------------
      if (!bwd) {
        if (s < S - 1) {
          apply_prop<N, false>(f, x, p, s, sep, sKr, sKc);
          if (want_prop) store_pairs<E, T>(zslot + (size_t)(m * (S - 1) + s) * NN, tid, x);  // Z_s = K_s fft2(chi_s)
          ++s;
          continue;
        }
#pragma unroll
        for (int e = 0; e < E; ++e) x[e] = cscale(x[e], inv_n);  // orthonormal detector FFT
        if (ADJ) {
          float2* fw = slot + (size_t)(P * S + m) * NN;
          store_pairs<E, T>(fw, tid, x);
        }
#pragma unroll
        for (int e = 0; e < E; e += 2) {
          const float2 old = m == 0 ? make_float2(0.f, 0.f) : inten2[(e >> 1) * T + tid];
          inten2[(e >> 1) * T + tid] = make_float2(old.x + cabs2(x[e]), old.y + cabs2(x[e + 1]));
        }
        if (ADJ && AN) {  // sum_p |Psi_p + 1e-9|^2 (ptychography_base.py:958)
          float2* t2 = reinterpret_cast<float2*>(tile2);
#pragma unroll
          for (int e = 0; e < E; e += 2) {
            const float2 old = m == 0 ? make_float2(0.f, 0.f) : t2[(e >> 1) * T + tid];
            t2[(e >> 1) * T + tid] = make_float2(old.x + cabs2(make_float2(x[e].x + 1e-9f, x[e].y)),
                                                 old.y + cabs2(make_float2(x[e + 1].x + 1e-9f, x[e + 1].y)));
          }
        }
        if (m < P - 1) {
          ++m;
          s = 0;
          load_probe(m);
          continue;
        }
        // loss over the mode-summed intensity (each thread owns its S3 slots)
        {
          const float* tg = p.targets + (size_t)gi * NN;
#pragma unroll
          for (int g = 0; g < G3; ++g)
#pragma unroll
            for (int e = 0; e < D; ++e) {
              const int kr = f.s3_row(g, e), kc = f.s3_c;
              const int di = ((kr + N / 2) % N) * N + ((kc + N / 2) % N);
              const int li = 2 * (((g * D + e) >> 1) * T + tid) + ((g * D + e) & 1);
              const float I = inten[li];
              if (!isfinite(I)) ++nonfinite;
              float dldi;
              const float tv = __ldcs(tg + di);  // targets stream through L2 once per iteration
              loss_elem<N>(p, I, tv, __ldg(p.mask + di), loss_acc, dldi);
              if (ADJ && AN) {
                // factor f and additive fix of the Fourier projection seed
                if (P == 1) {
                  dldi = I > 0.f ? tv / sqrtf(I) : 0.f;   // t exp(i angle(Psi)) = Psi t / |Psi|
                  tile2[li] = I > 0.f ? 0.f : tv;        // angle(0) = 0
                } else {
                  const float A = sqrtf(tile2[li]);
                  dldi = A > 0.f ? tv / A : 0.f;         // zero estimate -> infinity -> factor 0
                  tile2[li] = 0.f;
                }
              }
              inten[li] = dldi;
              if (p.out_intensity) p.out_intensity[(size_t)b * NN + di] = I;
            }
        }
        if (!ADJ) break;
        bwd = true;
        first_bwd = true;
        m = P - 1;  // last mode first: its far field and deepest waves are the most recent in L2
        s = S - 1;
        load_far_seed(m);
        continue;
      }
      first_bwd = false;
      if (s > 0) {
        if (want_prop) {
          // x = N^2 dL/dZ for Z = K_{s-1} fft2(chi_{s-1}) (w_s = ifft2(Z)): sum over this thread's
          // frequencies of fftfreq_index * Im(conj(dL/dZ) Z), the sensitivity of the loss to a
          // phase ramp of the propagator along each axis (the probe tilt, probe_models.py:418-425)
          const float2* zw = zslot + (size_t)(m * (S - 1) + s - 1) * NN;
          float gr = 0.f, gc = 0.f;
#pragma unroll
          for (int g = 0; g < G3; ++g)
#pragma unroll
            for (int e = 0; e < D; e += 2) {
              const int i = g * D + e;
              const float4 v = reinterpret_cast<const float4*>(zw)[(i >> 1) * T + tid];
              const float im0 = x[i].x * v.y - x[i].y * v.x;
              const float im1 = x[i + 1].x * v.w - x[i + 1].y * v.z;
              gr = fmaf((float)fsigned(f.s3_row(g, e), N), im0, gr);
              gr = fmaf((float)fsigned(f.s3_row(g, e + 1), N), im1, gr);
              gc += im0 + im1;
            }
          gc *= (float)fsigned(f.s3_c, N);
          for (int o = 16; o > 0; o >>= 1) {
            gr += __shfl_xor_sync(0xffffffffu, gr, o);
            gc += __shfl_xor_sync(0xffffffffu, gc, o);
          }
          if ((tid & 31) == 0) {
            atomicAdd(&propred[2 * (s - 1)], gr * inv_n2);
            atomicAdd(&propred[2 * (s - 1) + 1], gc * inv_n2);
          }
        }
        apply_prop<N, true>(f, x, p, s - 1, sep, sKr, sKc);
        --s;
        continue;
      }
      accumulate_probe_grad<N>(f, x, pgrad + (size_t)m * NN, rowf, colf);
      if (EXT && p.grad_positions) {
        // positions enter through the probe shift Y = probe_hat * ramp(frac) only; x = N^2 dL/dY
        // here, so dL/dfrac = (2 pi / N^2) sum_k fftfreq(k) Im(conj(x_k) Y_k), summed over the modes
        const float2* ph = p.probe_hat + (size_t)m * NN;
        float gr = 0.f, gc = 0.f;
#pragma unroll
        for (int g = 0; g < G3; ++g)
#pragma unroll
          for (int e = 0; e < D; ++e) {
            const int kr = f.s3_row(g, e), kc = f.s3_c;
            const float2 y = cmul(cmul(__ldg(ph + (size_t)kr * N + kc), rowf[kr]), colf[kc]);
            const float2 xv = x[g * D + e];
            const float im = xv.x * y.y - xv.y * y.x;
            gr = fmaf((float)fsigned(kr, N), im, gr);
            gc = fmaf((float)fsigned(kc, N), im, gc);
          }
        for (int o = 16; o > 0; o >>= 1) {
          gr += __shfl_xor_sync(0xffffffffu, gr, o);
          gc += __shfl_xor_sync(0xffffffffu, gc, o);
        }
        if ((tid & 31) == 0) {
          posred[tid >> 5][0] = gr;
          posred[tid >> 5][1] = gc;
        }
        __syncthreads();
        if (tid == 0) {  // fixed-order sum over warps, accumulated over the modes of this position
          float sr = 0.f, sc = 0.f;
          for (int w = 0; w < T / 32; ++w) {
            sr += posred[w][0];
            sc += posred[w][1];
          }
          const float k = 6.283185307179586f / ((float)N * (float)N * (float)N);  // 2 pi / N^2, fftfreq = k / N
          float* out = p.grad_positions + 2 * (size_t)b;
          const bool first = m == P - 1;  // the reverse chains run last mode first
          out[0] = (first ? 0.f : out[0]) + k * sr;
          out[1] = (first ? 0.f : out[1]) + k * sc;
        }
        __syncthreads();
      }
      if (m > 0) {
        --m;
        s = S - 1;
        first_bwd = true;
        load_far_seed(m);
        continue;
      }
      break;
    }
  }

  // ------------------------------ loss reduction ------------------------------
  for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xffffffffu, loss_acc, o);
  // one status update per CTA: per-thread updates of a shared word contend and can drop counts
  const int nf_warp = __reduce_add_sync(0xffffffffu, nonfinite);
  if ((tid & 31) == 0) {
    red[tid >> 5] = loss_acc;
    nfred[tid >> 5] = nf_warp;
  }
  __syncthreads();
  if (tid == 0) {
    int nf = 0;
    for (int w = 0; w < T / 32; ++w) nf += nfred[w];
    status_add_nonfinite(p.status, nf);
    double t = 0.0;
    for (int w = 0; w < T / 32; ++w) t += red[w];
    // l1/l2: sum / (B / num_gpts) / mean_I ; poisson: sum / mean_I
    p.loss_part[cta] = t * (double)(p.loss_type == LOSS_POISSON ? p.inv_mean_intensity : p.loss_scale);
  }
  if (want_prop && tid < 2 * (S - 1)) atomicAdd(p.grad_prop + tid, propred[tid]);  // after the barrier above
}

template <int N, bool ADJ, bool AN = false, bool EXT = false>
__global__ void __launch_bounds__(Fft2<N>::T, 1) fused_batch_kernel(const BatchParams p) {
  serial_body<N, ADJ, AN, EXT>(p, blockIdx.x, gridDim.x);
}

// Several independent datasets (same probe window N; any S, P, object size,
// scan size) in one persistent launch: CTAs [begin[d], begin[d+1]) work on
// dataset d.  The descriptors stay in the launch's parameter space
// (__grid_constant__), indexed by the CTA's uniform dataset id.
constexpr int kMaxDatasets = 16;
struct MultiParams {
  int nd;
  int begin[kMaxDatasets + 1];
  BatchParams d[kMaxDatasets];
};

template <int N, bool ADJ>
__global__ void __launch_bounds__(Fft2<N>::T, 1) multi_batch_kernel(const __grid_constant__ MultiParams mp) {
  int d = 0;
  while (d + 1 < mp.nd && (int)blockIdx.x >= mp.begin[d + 1]) ++d;
  serial_body<N, ADJ>(mp.d[d], (int)blockIdx.x - mp.begin[d], mp.begin[d + 1] - mp.begin[d]);
}

// Batched 2-D FFT of (count, N, N) arrays, one CTA per transform, natural layout
// in and out, result multiplied by `scale`.
template <int N, bool INV>
__global__ void __launch_bounds__(Fft2<N>::T, 1) fft2_batch_kernel(const float2* in, float2* out, int count,
                                                             float scale) {
  using F = Fft2<N>;
  constexpr int E = F::E, D = F::D, G3 = F::G3, T = F::T;
  extern __shared__ float4 smem_raw[];
  float2* sm = reinterpret_cast<float2*>(smem_raw);
  float2* tw = sm + F::SM_FLOAT2;
  const int tid = threadIdx.x;
  F f;
  f.init(tid);
  for (int k = tid; k < N; k += T) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)N, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
  __syncthreads();
  const size_t NN = (size_t)N * N;
  for (int t = blockIdx.x; t < count; t += gridDim.x) {
    const float2* src = in + (size_t)t * NN;
    float2* dst = out + (size_t)t * NN;
    float2 x[E];
    if (!INV) {
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = src[(size_t)f.s1_r * N + f.s1_col(e)];
      f.forward(x, sm, tw);
#pragma unroll
      for (int g = 0; g < G3; ++g)
#pragma unroll
        for (int e = 0; e < D; ++e) dst[(size_t)f.s3_row(g, e) * N + f.s3_c] = cscale(x[g * D + e], scale);
    } else {
#pragma unroll
      for (int g = 0; g < G3; ++g)
#pragma unroll
        for (int e = 0; e < D; ++e) x[g * D + e] = src[(size_t)f.s3_row(g, e) * N + f.s3_c];
      f.inverse(x, sm, tw);
#pragma unroll
      for (int e = 0; e < E; ++e) dst[(size_t)f.s1_r * N + f.s1_col(e)] = cscale(x[e], scale);
    }
    __syncthreads();
  }
}

template <int N>
constexpr size_t fft2_smem_bytes() {
  return sizeof(float2) * (size_t)(Fft2<N>::SM_FLOAT2 + N);
}

}  // namespace qb
