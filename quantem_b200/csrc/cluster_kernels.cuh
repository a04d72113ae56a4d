// Mode-parallel batch kernel: one thread-block cluster of P CTAs per scan
// position, CTA rank m computing probe mode m (sm_100a, cluster size P <= 8).
//
// Compared with fused_batch_kernel (one CTA, modes in sequence) this kernel
//  * sums the mode intensities |Psi_m|^2 across the cluster through distributed
//    shared memory (each CTA reads the P intensity tiles),
//  * sums the object-gradient contributions conj(psi_{s,m}) g_{s,m} of the P
//    modes in distributed shared memory before one float2 atomic scatter per
//    slice, i.e. P times fewer global atomics,
//  * keeps only its own mode's S incoming waves in its scratch slot (the far
//    field stays in registers through the loss), so the scratch in flight is S
//    waves per SM instead of P*(S+1).
// Everything else (probe shift, multislice, detector, loss, probe-gradient
// partials) is the same arithmetic as fused_batch_kernel, reference behaviour
// cited there.
#pragma once
#include <cooperative_groups.h>

#include "ptycho_kernels.cuh"

namespace qb {

template <int N, bool ADJ>
__global__ void __launch_bounds__(4 * N, 1) cluster_batch_kernel(const BatchParams p) {
  namespace cg = cooperative_groups;
  using F = Fft2<N>;
  constexpr int E = F::E, D = F::D, G3 = F::G3, T = F::T, PITCH = F::PITCH;
  cg::cluster_group cluster = cg::this_cluster();
  const int P = p.P;  // == cluster size
  const int m = (int)cluster.block_rank();
  const int cid = blockIdx.x / P, ncl = gridDim.x / P;

  extern __shared__ float4 smem_raw[];
  float2* sm = reinterpret_cast<float2*>(smem_raw);
  float2* tw = sm + F::SM_FLOAT2;
  float2* rowf = tw + N;
  float2* colf = rowf + N;
  float* inten = reinterpret_cast<float*>(colf + N);
  int* rowmap = reinterpret_cast<int*>(inten + N * N);
  int* colmap = rowmap + N;
  float2* sKr = reinterpret_cast<float2*>(colmap + N);
  float2* sKc = sKr + (size_t)N * (p.S > 1 ? p.S - 1 : 0);
  const bool sep = p.prop_r != nullptr;
  __shared__ double red[32];
  __shared__ int nfred[32];  // per-warp non-finite counts

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
  const int S = p.S;
  const size_t HoWo = (size_t)p.Ho * p.Wo;
  float2* slot = ADJ ? p.scratch + (size_t)blockIdx.x * (size_t)S * NN : nullptr;
  float2* pgrad = ADJ ? p.probe_grad_part + (size_t)blockIdx.x * NN : nullptr;
  if (ADJ) {
#pragma unroll
    for (int g = 0; g < G3; ++g)
#pragma unroll
      for (int e = 0; e < D; ++e) pgrad[(size_t)f.s3_row(g, e) * N + f.s3_c] = make_float2(0.f, 0.f);
  }
  // rows of the summed object-gradient tile this CTA scatters
  const int row_lo = (m * N) / P, row_hi = ((m + 1) * N) / P;
  double loss_acc = 0.0;
  int nonfinite = 0;

  const int bchunk = (p.B + ncl - 1) / ncl;  // contiguous block of the batch per cluster
  const int bend = min(p.B, (cid + 1) * bchunk);
  for (int b = cid * bchunk; b < bend; ++b) {
    const int64_t gi = p.batch_idx[b];
    if (gi < 0 || gi >= p.npos) {  // uniform across the cluster: every CTA skips it
      if (m == 0 && tid == 0) status_add_invalid(p.status, 1);
      continue;
    }
    const float py = p.positions[2 * gi], px = p.positions[2 * gi + 1];
    const float ry = rintf(py), rx = rintf(px);
    const float fy = py - ry, fx = px - rx;
    const int r0 = wrap_index((int)ry, p.Ho), c0 = wrap_index((int)rx, p.Wo);
    __syncthreads();
    for (int k = tid; k < 2 * N; k += T) {
      const int kk = k < N ? k : k - N;
      const float fq = (float)fsigned(kk, N) * inv_n;
      const float a = -6.283185307179586f * fq;
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
    // the whole chain of mode m: probe shift, S slices, detector, loss and (ADJ)
    // the reverse chain.  Keeping one copy of each unrolled transform keeps the
    // kernel inside the instruction caches.
    float2 x[E];
    {
      const float2* ph = p.probe_hat + (size_t)m * NN;
#pragma unroll
      for (int g = 0; g < G3; ++g)
#pragma unroll
        for (int e = 0; e < D; ++e) {
          const int kr = f.s3_row(g, e), kc = f.s3_c;
          x[g * D + e] = cmul(cmul(__ldg(ph + (size_t)kr * N + kc), rowf[kr]), colf[kc]);
        }
    }
    int s = 0;
    bool bwd = false, first_bwd = false;
    while (true) {
      f.inverse(x, sm, tw);
      // ---------------- real space (S1 layout) ----------------
      const float2* orow_ptr = p.obj + (size_t)s * HoWo + (size_t)orow * p.Wo;
      if (!bwd) {
#pragma unroll
        for (int e = 0; e < E; ++e) x[e] = cscale(x[e], inv_n2);
        if (ADJ) {
          float2* wv = slot + (size_t)s * NN;
#pragma unroll
          for (int e = 0; e < E; ++e) wv[e * T + tid] = x[e];
        }
        if (p.out_waves) {
          float2* ow = p.out_waves + (((size_t)s * P + m) * p.B + b) * NN + (size_t)f.s1_r * N;
#pragma unroll
          for (int e = 0; e < E; ++e) ow[f.s1_col(e)] = x[e];
        }
        gather_mul<N, false>(f, x, orow_ptr, colmap, evict_last_policy());
        if (s == S - 1 && p.out_exit) {
          float2* oe = p.out_exit + ((size_t)m * p.B + b) * NN + (size_t)f.s1_r * N;
#pragma unroll
          for (int e = 0; e < E; ++e) oe[f.s1_col(e)] = x[e];
        }
      } else {
        const float sc = first_bwd ? inv_n : inv_n2;  // adjoint of the orthonormal FFT, or of a propagation
#pragma unroll
        for (int e = 0; e < E; ++e) x[e] = cscale(x[e], sc);
        const float2* wv = slot + (size_t)s * NN;
        __syncthreads();  // exchange buffer free (the inverse finished reading it)
#pragma unroll
        for (int e0 = 0; e0 < E; e0 += 8) {
          float2 ps[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) ps[j] = wv[(e0 + j) * T + tid];
#pragma unroll
          for (int j = 0; j < 8; ++j) sm[f.s1_r * PITCH + f.s1_col(e0 + j)] = cmulc(x[e0 + j], ps[j]);
        }
        cluster.sync();  // every mode's contribution tile is in place
        float2* grow_s = p.grad_obj + (size_t)s * HoWo;
        const int nel = (row_hi - row_lo) * N;
        for (int i = tid; i < nel; i += T) {
          const int r = row_lo + i / N, c = i % N;
          float2 a = make_float2(0.f, 0.f);
          for (int q = 0; q < P; ++q) a = cadd(a, cluster.map_shared_rank(sm, q)[r * PITCH + c]);
          atomicAdd(grow_s + (size_t)rowmap[r] * p.Wo + colmap[c], a);
        }
        cluster.sync();  // all tiles read before any exchange buffer is reused
        gather_mul<N, true>(f, x, orow_ptr, colmap, evict_last_policy());
      }
      f.forward(x, sm, tw);
      // ---------------- Fourier space (S3 layout) ----------------
      if (!bwd) {
        if (s < S - 1) {
          apply_prop<N, false>(f, x, p, s, sep, sKr, sKc);
          ++s;
          continue;
        }
        // detector: orthonormal far field, mode intensities summed over the cluster
#pragma unroll
        for (int e = 0; e < E; ++e) {
          x[e] = cscale(x[e], inv_n);
          inten[e * T + tid] = cabs2(x[e]);
        }
        cluster.sync();  // every mode's |Psi|^2 tile is complete
        const float* tg = p.targets + (size_t)gi * NN;
#pragma unroll
        for (int g = 0; g < G3; ++g)
#pragma unroll
          for (int e = 0; e < D; ++e) {
            const int kr = f.s3_row(g, e), kc = f.s3_c;
            const int di = ((kr + N / 2) & (N - 1)) * N + ((kc + N / 2) & (N - 1));
            const int li = (g * D + e) * T + tid;
            float I = 0.f;
            for (int q = 0; q < P; ++q) I += cluster.map_shared_rank(inten, q)[li];
            float dldi;
            double acc = 0.0;
            loss_elem<N>(p, I, __ldg(tg + di), __ldg(p.mask + di), acc, dldi);
            if (m == 0) {
              loss_acc += acc;
              if (!isfinite(I)) ++nonfinite;
              if (p.out_intensity) p.out_intensity[(size_t)b * NN + di] = I;
            }
            x[g * D + e] = cscale(x[g * D + e], 2.0f * dldi);
          }
        if (!ADJ) {
          cluster.sync();  // intensity tiles read before the next position overwrites them
          break;
        }
        bwd = true;
        first_bwd = true;
        continue;
      }
      first_bwd = false;
      if (s > 0) {
        apply_prop<N, true>(f, x, p, s - 1, sep, sKr, sKc);
        --s;
        continue;
      }
      // probe-shift adjoint: conj(ramp) * fft2(g0) into this CTA's partial
      accumulate_probe_grad<N>(f, x, pgrad, rowf, colf);
      break;
    }
  }

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
    p.loss_part[blockIdx.x] = t * (double)(p.loss_type == LOSS_POISSON ? p.inv_mean_intensity : p.loss_scale);
  }
  cluster.sync();  // no CTA exits while another may still read its shared memory
}

}  // namespace qb
