// Mixed-state probe orthogonalisation and its gradient (reference:
// ProbePixelated._probe_orthogonalization_constraint, probe_models.py:484-525):
// modified Gram-Schmidt over the P modes with the running vector, each mode
// rescaled to its original norm, modes sorted by descending real-space intensity.
//
// P is small (<= 16) and a mode has N*N elements, so one CTA of 1024 threads runs
// the whole sequential algorithm: every projection coefficient and norm is a
// block reduction in float64 over a pass through one or two modes (L2-resident),
// and the gradient replays the same steps backwards.  Replaces some fifty tiny
// tensor-op launches of the forward and about three times as many in autograd's
// backward.
//
// Work buffer (float2 view, caller-owned, reused by the gradient):
//   q    [P * nn]      orthonormal modes (unsorted)
//   gq   [P * nn]      gradient scratch of q
//   meta               c[P*P] (complex, row i: coefficients of mode i), then per mode
//                      n0, nrm, nrm_c as float2 (x = value) and the sort order
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include "ptycho_b200.h"

int qb_record_error(int code, const char* msg);

namespace {

constexpr int kThreads = 1024;
constexpr int kMaxModes = 16;

int fail(int code, const char* fmt, ...) {
  char buf[400];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return qb_record_error(code, buf);
}

struct Z {
  double re, im;
};

// sum over the block of (re, im); every thread gets the result
__device__ Z block_sum2(double re, double im, double2* red) {
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();  // red is free
  if (l == 0) red[w] = make_double2(re, im);
  __syncthreads();
  double sr = 0.0, si = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {  // fixed order, every thread
    sr += red[i].x;
    si += red[i].y;
  }
  return {sr, si};
}

__device__ __forceinline__ float2 cmul_(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconjmul(float2 a, float2 b) {  // conj(a) * b
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

struct Meta {
  float2* c;     // P*P
  float2* norm;  // P: (n0, nrm), P: (nrm_c, 0)
  int* order;    // P
};
__device__ __forceinline__ Meta meta_of(float2* work, int P, int64_t nn) {
  Meta m;
  m.c = work + 2 * (int64_t)P * nn;
  m.norm = m.c + P * P;
  m.order = reinterpret_cast<int*>(m.norm + 2 * P);
  return m;
}

__global__ void __launch_bounds__(kThreads, 1)
    probe_ortho_kernel(const float2* __restrict__ in, float2* __restrict__ out, int P, int64_t nn, float2* work) {
  __shared__ double2 red[kThreads / 32];
  __shared__ float inten[kMaxModes];
  float2* q = work;
  const Meta m = meta_of(work, P, nn);
  const int tid = threadIdx.x;
  for (int i = 0; i < P; ++i) {
    const float2* pi = in + (int64_t)i * nn;
    float2* qi = q + (int64_t)i * nn;
    double s = 0.0;
    for (int64_t k = tid; k < nn; k += kThreads) {
      const float2 v = pi[k];
      qi[k] = v;  // running vector u, in place
      s += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double n0 = sqrt(block_sum2(s, 0.0, red).re);
    for (int j = 0; j < i; ++j) {  // c = sum conj(q_j) u ; u -= c q_j
      const float2* qj = q + (int64_t)j * nn;
      double cr = 0.0, ci = 0.0;
      for (int64_t k = tid; k < nn; k += kThreads) {
        const float2 t = cconjmul(qj[k], qi[k]);
        cr += t.x;
        ci += t.y;
      }
      const Z c = block_sum2(cr, ci, red);
      const float2 cf = make_float2((float)c.re, (float)c.im);
      if (tid == 0) m.c[i * P + j] = cf;
      for (int64_t k = tid; k < nn; k += kThreads) {
        const float2 t = cmul_(cf, qj[k]);
        qi[k] = make_float2(qi[k].x - t.x, qi[k].y - t.y);
      }
    }
    double s2 = 0.0;
    for (int64_t k = tid; k < nn; k += kThreads) s2 += (double)qi[k].x * qi[k].x + (double)qi[k].y * qi[k].y;
    const double nrm = sqrt(block_sum2(s2, 0.0, red).re);
    const double nrm_c = nrm > 1e-12 ? nrm : 1e-12;
    const float inv = (float)(1.0 / nrm_c);
    double s3 = 0.0;
    for (int64_t k = tid; k < nn; k += kThreads) {
      const float2 v = make_float2(qi[k].x * inv, qi[k].y * inv);
      qi[k] = v;
      const float ox = v.x * (float)n0, oy = v.y * (float)n0;
      s3 += (double)ox * ox + (double)oy * oy;
    }
    const double it = block_sum2(s3, 0.0, red).re;
    if (tid == 0) {
      m.norm[i] = make_float2((float)n0, (float)nrm);
      m.norm[P + i] = make_float2((float)nrm_c, 0.f);
      inten[i] = (float)it;
    }
  }
  __syncthreads();
  if (tid == 0) {  // stable descending order of the intensities
    for (int i = 0; i < P; ++i) m.order[i] = i;
    for (int i = 1; i < P; ++i)
      for (int j = i; j > 0 && inten[m.order[j]] > inten[m.order[j - 1]]; --j) {
        const int t = m.order[j];
        m.order[j] = m.order[j - 1];
        m.order[j - 1] = t;
      }
  }
  __syncthreads();
  for (int r = 0; r < P; ++r) {
    const int i = m.order[r];
    const float n0 = m.norm[i].x;
    const float2* qi = q + (int64_t)i * nn;
    float2* o = out + (int64_t)r * nn;
    for (int64_t k = tid; k < nn; k += kThreads) o[k] = make_float2(qi[k].x * n0, qi[k].y * n0);
  }
}

// Reverse of probe_ortho_kernel (torch convention: the gradient of a real loss
// with respect to z is dL/dRe z + i dL/dIm z).
__global__ void __launch_bounds__(kThreads, 1)
    probe_ortho_vjp_kernel(const float2* __restrict__ in, const float2* __restrict__ grad_sorted,
                           float2* __restrict__ grad_in, int P, int64_t nn, float2* work) {
  __shared__ double2 red[kThreads / 32];
  const float2* q = work;
  float2* gq = work + (int64_t)P * nn;
  const Meta m = meta_of(work, P, nn);
  const int tid = threadIdx.x;
  // g_q = g_out n0 ; g_in = in / n0 * Re<q, g_out>
  for (int r = 0; r < P; ++r) {
    const int i = m.order[r];
    const float n0 = m.norm[i].x;
    const float2* go = grad_sorted + (int64_t)r * nn;
    const float2* qi = q + (int64_t)i * nn;
    double s = 0.0;
    for (int64_t k = tid; k < nn; k += kThreads) {
      const float2 g = go[k];
      gq[(int64_t)i * nn + k] = make_float2(g.x * n0, g.y * n0);
      s += (double)qi[k].x * g.x + (double)qi[k].y * g.y;
    }
    const double gn0 = block_sum2(s, 0.0, red).re;
    const float f = (float)(n0 > 0.f ? gn0 / (double)n0 : 0.0);
    const float2* pi = in + (int64_t)i * nn;
    float2* gi = grad_in + (int64_t)i * nn;
    for (int64_t k = tid; k < nn; k += kThreads) gi[k] = make_float2(pi[k].x * f, pi[k].y * f);
  }
  __syncthreads();
  for (int i = P - 1; i >= 0; --i) {
    const float nrm = m.norm[i].y, nrm_c = m.norm[P + i].x;
    const float2* qi = q + (int64_t)i * nn;
    float2* gqi = gq + (int64_t)i * nn;
    // u = q_i nrm_c ; g_u = g_q / nrm_c (+ u / nrm * g_nrm), kept in gqi
    double s = 0.0;
    for (int64_t k = tid; k < nn; k += kThreads)
      s += ((double)qi[k].x * gqi[k].x + (double)qi[k].y * gqi[k].y) * nrm_c;  // Re<u, g_q>
    const double sdot = block_sum2(s, 0.0, red).re;
    const bool live = nrm >= 1e-12f;
    const float gnrm = live ? (float)(-sdot / ((double)nrm_c * nrm_c)) : 0.f;
    const float a = 1.f / nrm_c, bq = live ? gnrm * nrm_c / nrm : 0.f;  // g_u = a g_q + bq q
    for (int64_t k = tid; k < nn; k += kThreads)
      gqi[k] = make_float2(a * gqi[k].x + bq * qi[k].x, a * gqi[k].y + bq * qi[k].y);
    // u^(i) = q_i nrm_c; walk j = i-1 .. 0 with u^(j) = u^(j+1) + c_ij q_j (u^(j) = u_prev of step j)
    for (int j = i - 1; j >= 0; --j) {
      const float2 cij = m.c[i * P + j];
      const float2* qj = q + (int64_t)j * nn;
      float2* gqj = gq + (int64_t)j * nn;
      double gr = 0.0, gim = 0.0;
      for (int64_t k = tid; k < nn; k += kThreads) {
        const float2 t = cconjmul(qj[k], gqi[k]);  // conj(q_j) g_u
        gr += t.x;
        gim += t.y;
      }
      const Z gcs = block_sum2(gr, gim, red);
      const float2 gc = make_float2((float)-gcs.re, (float)-gcs.im);  // g_c = -sum conj(q_j) g_u
      for (int64_t k = tid; k < nn; k += kThreads) {
        // u_prev = u^(j) = q_i nrm_c + sum_{l >= j} c_il q_l, rebuilt here from the saved q's
        float2 up = make_float2(qi[k].x * nrm_c, qi[k].y * nrm_c);
        for (int l = j; l < i; ++l) {
          const float2 t = cmul_(m.c[i * P + l], q[(int64_t)l * nn + k]);
          up.x += t.x;
          up.y += t.y;
        }
        const float2 gu = gqi[k];
        // g_q_j += -conj(c) g_u + conj(g_c) u_prev
        const float2 t1 = cconjmul(cij, gu);
        const float2 t2 = cconjmul(gc, up);
        gqj[k] = make_float2(gqj[k].x - t1.x + t2.x, gqj[k].y - t1.y + t2.y);
        // g_u_prev = g_u + q_j g_c
        const float2 t3 = cmul_(qj[k], gc);
        gqi[k] = make_float2(gu.x + t3.x, gu.y + t3.y);
      }
      __syncthreads();
    }
    float2* gi = grad_in + (int64_t)i * nn;
    for (int64_t k = tid; k < nn; k += kThreads) gi[k] = make_float2(gi[k].x + gqi[k].x, gi[k].y + gqi[k].y);
    __syncthreads();
  }
}

}  // namespace

extern "C" {

int64_t ptycho_probe_ortho_work_elems(int P, int64_t nn) {
  // q, gq, c, norms (float2 units) + the order (ints, rounded up to float2)
  return 2 * (int64_t)P * nn + (int64_t)P * P + 2 * P + (P + 1) / 2;
}

int ptycho_probe_orthogonalize(const void* probe, void* out, int P, int64_t nn, void* work, int64_t work_elems,
                               void* stream) {
  if (!probe || !out || !work || P < 1 || P > kMaxModes || nn < 1)
    return fail(PTYCHO_ERR_INVALID, "probe_orthogonalize: bad arguments (1 <= P <= %d)", kMaxModes);
  if (work_elems < ptycho_probe_ortho_work_elems(P, nn))
    return fail(PTYCHO_ERR_INVALID, "probe_orthogonalize: work needs %lld complex elements",
                (long long)ptycho_probe_ortho_work_elems(P, nn));
  if (probe == out) return fail(PTYCHO_ERR_INVALID, "probe_orthogonalize: out must not alias the input");
  probe_ortho_kernel<<<1, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(probe), static_cast<float2*>(out), P, nn, static_cast<float2*>(work));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PTYCHO_OK : fail(PTYCHO_ERR_CUDA, "probe_ortho_kernel: %s", cudaGetErrorString(e));
}

int ptycho_probe_orthogonalize_vjp(const void* probe, const void* grad_sorted, void* grad_probe, int P, int64_t nn,
                                   void* work, int64_t work_elems, void* stream) {
  if (!probe || !grad_sorted || !grad_probe || !work || P < 1 || P > kMaxModes || nn < 1)
    return fail(PTYCHO_ERR_INVALID, "probe_orthogonalize_vjp: bad arguments (1 <= P <= %d)", kMaxModes);
  if (work_elems < ptycho_probe_ortho_work_elems(P, nn))
    return fail(PTYCHO_ERR_INVALID, "probe_orthogonalize_vjp: work needs %lld complex elements",
                (long long)ptycho_probe_ortho_work_elems(P, nn));
  // the kernel reads probe and grad_sorted while it writes grad_probe (restrict pointers)
  if (grad_probe == probe || grad_probe == grad_sorted || grad_probe == work)
    return fail(PTYCHO_ERR_INVALID, "probe_orthogonalize_vjp: grad_probe must not alias probe, grad_sorted or work");
  probe_ortho_vjp_kernel<<<1, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(probe), static_cast<const float2*>(grad_sorted), static_cast<float2*>(grad_probe), P,
      nn, static_cast<float2*>(work));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PTYCHO_OK : fail(PTYCHO_ERR_CUDA, "probe_ortho_vjp_kernel: %s", cudaGetErrorString(e));
}

}  // extern "C"
