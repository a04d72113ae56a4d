// 256 x 256 multislice mixed-probe batch kernel: one thread-block cluster of four
// CTAs per scan position (persistent over positions), the 2-D FFTs staged
// across the cluster through distributed shared memory (fft256_cluster.cuh).
//
// Same computation and reference behaviour as serial_body in ptycho_kernels.cuh
// (probe shift ptycho_utils.py:128-176, patch gather object_models.py:252-265,
// multislice ptychography_base.py:934-947 / 970-989, detector
// detector_models.py:22-30, loss ptychography_base.py:908-932, autograd adjoint
// ptychography.py:326-332).  Each CTA owns a quarter of every wave: 64 object
// rows in real space, 64 spectral columns in Fourier space.
//
// Adjoint memory: with p.ckpt == 0 every slice's incident wave is kept (P*S
// quarter-waves per CTA).  With p.ckpt = k > 0 only the Fourier-space wave
// entering every k-th slice is kept; the reverse sweep saves its back-propagated
// wave, recomputes the k incident waves of the next segment from its checkpoint
// into a k-slot buffer, restores the saved wave and continues (recompute in the
// adjoint: P*ceil(S/k) + k slots instead of P*S, at the cost of S - S/k extra
// propagation steps per mode).
#pragma once
#include "fft256_cluster.cuh"
#include "ptycho_kernels.cuh"

namespace qb {

constexpr int C256_CLUSTER = 4;

// dynamic shared memory of cluster256_kernel: exchange buffer, twiddles, shift
// ramps, wrap maps and the CTA's quarter of the intensity / dL/dI tile
constexpr size_t c256_smem_bytes() {
  return sizeof(float2) * (size_t)(Fft256C::SM_FLOAT2 + Fft256C::TW_FLOAT2 + 2 * 256) + sizeof(int) * 512 +
         sizeof(float) * (size_t)Fft256C::T * Fft256C::E;
}
// scratch slots (each T*E float2) per CTA
__host__ __device__ inline int c256_slots(int S, int P, int ck) {
  return ck <= 0 ? P * S + P : P * ((S + ck - 1) / ck) + P + ck + 1;
}

template <bool ADJ>
__global__ void __launch_bounds__(512, 1) cluster256_kernel(const BatchParams p) {
  using F = Fft256C;
  constexpr int N = 256, E = F::E, T = F::T;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float4 smem_raw[];
  float2* sm = reinterpret_cast<float2*>(smem_raw);
  float2* tw = sm + F::SM_FLOAT2;
  float2* rowf = tw + F::TW_FLOAT2;
  float2* colf = rowf + N;
  int* rowmap = reinterpret_cast<int*>(colf + N);
  int* colmap = rowmap + N;
  float* inten = reinterpret_cast<float*>(colmap + N);
  __shared__ double red[32];
  __shared__ int nfred[32];  // per-warp non-finite counts

  const int tid = threadIdx.x;
  const int q = (int)cl.block_rank();
  const int cid = blockIdx.x / C256_CLUSTER, ncl = gridDim.x / C256_CLUSTER;
  F f;
  f.init(tid, q);
  F::fill_twiddles(tw, tid, T);
  const float inv_n = 1.0f / (float)N;
  const float inv_n2 = inv_n * inv_n;
  const size_t NN = (size_t)N * N;
  const int S = p.S, P = p.P, ck = p.ckpt;
  const size_t HoWo = (size_t)p.Ho * p.Wo;
  const size_t QW = (size_t)T * E;
  const int nck = ck > 0 ? (S + ck - 1) / ck : 0;
  float2* base = ADJ ? p.scratch + (size_t)blockIdx.x * (size_t)c256_slots(S, P, ck) * QW : nullptr;
  // slot layout: store-all: waves (m*S + s), far fields (P*S + m)
  //              checkpoints: ckpt (m*nck + j), far (P*nck + m), segment (P*nck + P + i), saved wave (last)
  auto wave_slot = [&](int m, int s) { return base + (size_t)(m * S + s) * QW; };
  auto ckpt_slot = [&](int m, int j) { return base + (size_t)(m * nck + j) * QW; };
  auto far_slot = [&](int m) { return base + (size_t)((ck > 0 ? P * nck : P * S) + m) * QW; };
  auto seg_slot = [&](int i) { return base + (size_t)(P * nck + P + i) * QW; };
  float2* gsave = ADJ && ck > 0 ? base + (size_t)(P * nck + P + ck) * QW : nullptr;
  float2* pgrad = ADJ ? p.probe_grad_part + (size_t)cid * P * NN : nullptr;
  const int kc = f.b_kc();
  if (ADJ) {
    for (int m = 0; m < P; ++m)
#pragma unroll
      for (int i = 0; i < E; ++i) pgrad[(size_t)m * NN + (size_t)f.b_kr(i) * N + kc] = make_float2(0.f, 0.f);
  }
  cl.sync();  // every CTA of the cluster runs before any distributed-shared-memory access
  double loss_acc = 0.0;
  int nonfinite = 0;

  // each cluster takes a contiguous block of the batch (concurrent positions far apart)
  const int bchunk = (p.B + ncl - 1) / ncl;
  const int bend = min(p.B, (cid + 1) * bchunk);
  for (int b = cid * bchunk; b < bend; ++b) {
    const int64_t gi = p.batch_idx[b];
    if (gi < 0 || gi >= p.npos) {  // the whole cluster skips the position (same b)
      if (tid == 0 && q == 0) status_add_invalid(p.status, 1);
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
    const int orow = rowmap[f.a_row()];

    float2 x[E];
    auto load_probe = [&](int mm) {
      const float2* ph = p.probe_hat + (size_t)mm * NN;
      const float2 cf = colf[kc];
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const int kr = f.b_kr(i);
        x[i] = cmul(cmul(__ldg(ph + (size_t)kr * N + kc), rowf[kr]), cf);
      }
    };
    auto load_far_seed = [&](int mm) {
      const float2* fw = far_slot(mm);
      load_pairs<E, T>(fw, tid, x);
#pragma unroll
      for (int i = 0; i < E; ++i) x[i] = cscale(x[i], 2.0f * inten[i * T + tid]);
    };
    auto apply_prop = [&](int s, bool conj) {
      if (p.prop_r) {
        const float2 kcf = __ldg(p.prop_c + (size_t)s * N + kc);
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float2 k = cmul(__ldg(p.prop_r + (size_t)s * N + f.b_kr(i)), kcf);
          x[i] = conj ? cmulc(x[i], k) : cmul(x[i], k);
        }
      } else {
        const float2* pr = p.prop + (size_t)s * NN;
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float2 k = __ldg(pr + (size_t)f.b_kr(i) * N + kc);
          x[i] = conj ? cmulc(x[i], k) : cmul(x[i], k);
        }
      }
    };
    auto gather_mul = [&](int s) {
      const float2* orow_ptr = p.obj + (size_t)s * HoWo + (size_t)orow * p.Wo;
#pragma unroll
      for (int e0 = 0; e0 < E; e0 += 8) {
        float2 ob[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) ob[j] = __ldg(orow_ptr + colmap[f.a_col(e0 + j)]);
#pragma unroll
        for (int j = 0; j < 8; ++j) x[e0 + j] = cmul(x[e0 + j], ob[j]);
      }
    };

    int m = 0, s = 0;
    bool bwd = false, first_bwd = false, rec = false;
    int seg_lo = 1, seg_hi = 0, srec = 0;  // segment of recomputed waves (empty)
    load_probe(0);
    while (true) {
      if (ADJ && ck > 0) {
        if (!bwd && s % ck == 0) {  // Fourier checkpoint of the wave entering slice s
          float2* cp = ckpt_slot(m, s / ck);
          store_pairs<E, T>(cp, tid, x);
        } else if (bwd && !rec && (s < seg_lo || s > seg_hi)) {
          // recompute the incident waves of the segment that ends at slice s
          store_pairs<E, T>(gsave, tid, x);
          seg_lo = (s / ck) * ck;
          seg_hi = s;
          srec = seg_lo;
          rec = true;
          const float2* cp = ckpt_slot(m, s / ck);
          load_pairs<E, T>(cp, tid, x);
        }
      }
      f.inverse(x, sm, tw, cl);
      // ---------------- real space (layout A) ----------------
      if (!bwd || rec) {
#pragma unroll
        for (int e = 0; e < E; ++e) x[e] = cscale(x[e], inv_n2);
        if (ADJ) {
          float2* wv = rec ? seg_slot(srec - seg_lo) : (ck == 0 ? wave_slot(m, s) : nullptr);
          if (wv) {
            store_pairs<E, T>(wv, tid, x);
          }
          if (rec && srec == seg_hi) {  // segment complete: resume the reverse sweep at slice seg_hi
            load_pairs<E, T>(gsave, tid, x);
            rec = false;
            continue;
          }
        }
        gather_mul(rec ? srec : s);
      } else {
        const float sc = first_bwd ? inv_n : inv_n2;
        const float2* wv = ck == 0 ? wave_slot(m, s) : seg_slot(s - seg_lo);
        const float2* orow_ptr = p.obj + (size_t)s * HoWo + (size_t)orow * p.Wo;
        float2* grow = p.grad_obj + (size_t)s * HoWo + (size_t)orow * p.Wo;
#pragma unroll
        for (int e0 = 0; e0 < E; e0 += 4) {
          float2 ps[4], ob[4];
          int col[4];
#pragma unroll
          for (int j = 0; j < 4; j += 2) {
            const float4 v = reinterpret_cast<const float4*>(wv)[((e0 + j) >> 1) * T + tid];
            ps[j] = make_float2(v.x, v.y);
            ps[j + 1] = make_float2(v.z, v.w);
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            col[j] = colmap[f.a_col(e0 + j)];
            ob[j] = __ldg(orow_ptr + col[j]);
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const float2 g = cscale(x[e0 + j], sc);
            atomicAdd(grow + col[j], cmulc(g, ps[j]));
            x[e0 + j] = cmulc(g, ob[j]);
          }
        }
      }
      f.forward(x, sm, tw, cl);
      // ---------------- Fourier space (layout B) ----------------
      if (rec) {
        apply_prop(srec, false);
        ++srec;
        continue;
      }
      if (!bwd) {
        if (s < S - 1) {
          apply_prop(s, false);
          ++s;
          continue;
        }
#pragma unroll
        for (int i = 0; i < E; ++i) x[i] = cscale(x[i], inv_n);  // orthonormal detector FFT
        if (ADJ) {
          float2* fw = far_slot(m);
          store_pairs<E, T>(fw, tid, x);
        }
#pragma unroll
        for (int i = 0; i < E; ++i) inten[i * T + tid] = (m == 0 ? 0.f : inten[i * T + tid]) + cabs2(x[i]);
        if (m < P - 1) {
          ++m;
          s = 0;
          load_probe(m);
          continue;
        }
        {
          // detector (centred) index of (kr, kc): kr = 4tl + a + 32kB shifts to 4tl + a + 32((kB + 4) % 8)
          const int dbase = 4 * f.tl * N + ((kc + N / 2) & (N - 1));
          const float* tg = p.targets + (size_t)gi * NN + dbase;
          const float* mk = p.mask + dbase;
          float* oi = p.out_intensity ? p.out_intensity + (size_t)b * NN + dbase : nullptr;
#pragma unroll
          for (int i = 0; i < E; ++i) {
            const int doff = ((i >> 3) + 32 * (((i & 7) + 4) & 7)) * N;
            const float I = inten[i * T + tid];
            if (!isfinite(I)) ++nonfinite;
            float dldi;
            loss_elem<N>(p, I, __ldg(tg + doff), __ldg(mk + doff), loss_acc, dldi);
            inten[i * T + tid] = dldi;
            if (oi) oi[doff] = I;
          }
        }
        if (!ADJ) break;
        bwd = true;
        first_bwd = true;
        m = 0;
        s = S - 1;
        seg_lo = 1;
        seg_hi = 0;
        load_far_seed(0);
        continue;
      }
      first_bwd = false;
      if (s > 0) {
        apply_prop(s - 1, true);
        --s;
        continue;
      }
      {  // Fourier-space probe gradient: conj(ramp) * x
        float2* pg = pgrad + (size_t)m * NN;
        const float2 cf = colf[kc];
#pragma unroll
        for (int i0 = 0; i0 < E; i0 += 8) {
          float2 old[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) old[j] = pg[(size_t)f.b_kr(i0 + j) * N + kc];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int kr = f.b_kr(i0 + j);
            pg[(size_t)kr * N + kc] = cadd(old[j], cmulc(x[i0 + j], cmul(rowf[kr], cf)));
          }
        }
      }
      if (m < P - 1) {
        ++m;
        s = S - 1;
        first_bwd = true;
        seg_lo = 1;
        seg_hi = 0;
        load_far_seed(m);
        continue;
      }
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
    // l1/l2: sum / (B / num_gpts) / mean_I ; poisson: sum / mean_I
    p.loss_part[blockIdx.x] = t * (double)(p.loss_type == LOSS_POISSON ? p.inv_mean_intensity : p.loss_scale);
  }
  cl.sync();  // no CTA leaves while a peer may still write into its shared memory
}

// count 256 x 256 transforms in natural layout, one cluster per transform
template <bool INV>
__global__ void __launch_bounds__(512, 1) fft256_batch_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                             int count, float scale) {
  using F = Fft256C;
  constexpr int N = 256, E = F::E, T = F::T;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float4 smem_raw[];
  float2* sm = reinterpret_cast<float2*>(smem_raw);
  float2* tw = sm + F::SM_FLOAT2;
  const int tid = threadIdx.x;
  F f;
  f.init(tid, (int)cl.block_rank());
  F::fill_twiddles(tw, tid, T);
  cl.sync();
  const int cid = blockIdx.x / C256_CLUSTER, ncl = gridDim.x / C256_CLUSTER;
  const size_t NN = (size_t)N * N;
  float2 x[E];
  for (int t = cid; t < count; t += ncl) {
    const float2* src = in + (size_t)t * NN;
    float2* dst = out + (size_t)t * NN;
    if (!INV) {
      const int r = f.a_row();
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = src[(size_t)r * N + f.a_col(e)];
      f.forward(x, sm, tw, cl);
      const int kc = f.b_kc();
#pragma unroll
      for (int i = 0; i < E; ++i) dst[(size_t)f.b_kr(i) * N + kc] = cscale(x[i], scale);
    } else {
      const int kc = f.b_kc();
#pragma unroll
      for (int i = 0; i < E; ++i) x[i] = src[(size_t)f.b_kr(i) * N + kc];
      f.inverse(x, sm, tw, cl);
      const int r = f.a_row();
#pragma unroll
      for (int e = 0; e < E; ++e) dst[(size_t)r * N + f.a_col(e)] = cscale(x[e], scale);
    }
  }
  cl.sync();
}

constexpr size_t fft256_smem_bytes() { return sizeof(float2) * (size_t)(Fft256C::SM_FLOAT2 + Fft256C::TW_FLOAT2); }

}  // namespace qb
