// 256 x 256 complex 2-D FFT staged across a cluster of 4 CTAs (sm_100a).
//
// A 256^2 complex64 wave (512 KB) does not fit one SM, so four CTAs of a
// thread-block cluster hold a quarter each (512 threads x 32 registers).
//
//   Layout A (real space / row slab): CTA q holds rows r = 64q + line,
//     thread (line = tid/8, tl = tid%8) holds columns c = tl + 8e, e = 0..31.
//   Layout B (spectrum / column slab): CTA q holds spectral columns
//     kc = 64q + line; after the column transform thread (line, g = tl) holds
//     kr = 4g + a + 32kB in register a*8 + kB.
//
// Each 256-point 1-D transform is local to a CTA: a 32-point register DFT over
// e, the twiddle w256^(tl*k1), a shared-memory exchange inside the line, and
// four 8-point register DFTs (k = k1 + 32*k2, natural order).  Between the row
// and column transforms the slabs are redistributed across the cluster: every
// thread stores its values straight into the owning CTA's shared memory
// (distributed shared memory), bracketed by cluster barriers.  A 2-D FFT thus
// costs two local exchanges and one cluster exchange.  All shared-memory
// accesses (local and remote) use XOR-swizzled indices chosen so that each warp
// access splits into the minimum two 128-byte wavefronts.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "fft_engine.cuh"

namespace qb {

namespace cg = cooperative_groups;

struct Fft256C {
  static constexpr int N = 256;
  static constexpr int T = 512;
  static constexpr int E = 32;
  static constexpr int LINES = 64;
  static constexpr int SM_FLOAT2 = 17536;  // >= the largest of the three layouts below (63*274 + 271)
  // twiddle table: tw[t*33 + k1] = w256^(t*k1), t < 8, k1 < 32 (row padding 33 keeps the
  // eight t rows on distinct banks)
  static constexpr int TW_FLOAT2 = 8 * 33;
  static __device__ __forceinline__ void fill_twiddles(float2* tw, int tid, int nthreads) {
    for (int k = tid; k < 8 * 32; k += nthreads) {
      const int t = k >> 5, k1 = k & 31;
      double s, c;
      sincospi(-2.0 * (double)(t * k1) / 256.0, &s, &c);
      tw[t * 33 + k1] = make_float2((float)c, (float)s);
    }
  }

  int q;     // cluster rank (0..3)
  int line;  // tid / 8
  int tl;    // tid % 8

  __device__ __forceinline__ void init(int tid, int rank) {
    q = rank;
    line = tid >> 3;
    tl = tid & 7;
  }
  // Buffer layouts (float2 index).  Padding is additive, so every access is a
  // per-thread base plus a compile-time offset (one address register per loop);
  // the paddings were chosen by exhaustive search so that each warp access of
  // every exchange touches each of the 16 float2 bank pairs at most twice.
  //   line-local exchange, element (k1, t) of line ln:  ln*264 + 33*(k1/4) + 8*(k1%4) + t
  //   column slab, element (kc_local, r):               kcl*260 + 2*(kcl/4) + r
  //   row slab spectrum, element (r_local, kc):         rl*274 + kc + kc/16
  // (row lengths cover each padded row: 262 < 264, 256 < 260, 271 < 274)
  static constexpr int LP = 264, BP = 260, AP = 274;
  __device__ __forceinline__ int lx(int ln, int k1, int t) const { return ln * LP + 33 * (k1 >> 2) + 8 * (k1 & 3) + t; }
  __device__ __forceinline__ int bx(int kcl, int r) const { return kcl * BP + 2 * (kcl >> 2) + r; }
  __device__ __forceinline__ int ax(int rl, int kc) const { return rl * AP + kc + (kc >> 4); }

  // coordinates
  __device__ __forceinline__ int a_row() const { return 64 * q + line; }     // layout A row
  __device__ __forceinline__ int a_col(int e) const { return tl + 8 * e; }   // layout A column
  __device__ __forceinline__ int b_kc() const { return 64 * q + line; }      // layout B spectral column
  __device__ __forceinline__ int b_kr(int i) const { return 4 * tl + (i >> 3) + 32 * (i & 7); }  // register i = a*8+kB

  // four 8-point DFTs on registers a*8 .. a*8+7 (compile-time offsets keep x in registers)
  template <bool INV, int A>
  __device__ __forceinline__ void dft8_groups(float2 (&x)[E]) const {
    if constexpr (A < 4) {
      dft_reg<8, INV, 1, A * 8>(x);
      dft8_groups<INV, A + 1>(x);
    }
  }

  // Split cluster barrier: the first barrier of a cluster exchange only has to
  // order every CTA's last reads of its own buffer before the peers' remote
  // stores, so each thread arrives right after those reads and waits just before
  // its own remote stores; the register work in between hides the barrier.
  static __device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  }
  static __device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
  }

  // ---- 256-point transform along the line: x[e] = element tl + 8e in, natural
  //      frequency k = 4*tl + a + 32*kB in register a*8 + kB out ----
  // ARRIVE: arrive on the cluster barrier after the last read of the buffer
  template <bool INV, bool ARRIVE = false>
  __device__ __forceinline__ void line_fwd(float2 (&x)[E], float2* sm, const float2* tw) const {
    dft_reg<32, INV>(x);
    {
      const float2* twr = tw + 33 * tl;
#pragma unroll
      for (int k1 = 1; k1 < 32; ++k1) x[k1] = INV ? cmulc(x[k1], twr[k1]) : cmul(x[k1], twr[k1]);
    }
    __syncthreads();
    {
      float2* w = sm + line * LP + tl;  // + lx offset of (k1, 0)
#pragma unroll
      for (int k1 = 0; k1 < 32; ++k1) w[33 * (k1 >> 2) + 8 * (k1 & 3)] = x[k1];
    }
    __syncthreads();
    {
      const float2* r = sm + line * LP + 33 * tl;  // group g = tl: k1 = 4g + a
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int t = 0; t < 8; ++t) x[a * 8 + t] = r[8 * a + t];
    }
    if (ARRIVE) cluster_arrive();
    dft8_groups<INV, 0>(x);
  }
  // inverse direction of line_fwd's data flow: frequency distribution in,
  // element tl + 8e out (INV selects the conjugate transform)
  template <bool INV, bool ARRIVE = false>
  __device__ __forceinline__ void line_bwd(float2 (&x)[E], float2* sm, const float2* tw) const {
    dft8_groups<INV, 0>(x);
    __syncthreads();
    {
      float2* w = sm + line * LP + 33 * tl;
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int t = 0; t < 8; ++t) w[8 * a + t] = x[a * 8 + t];
    }
    __syncthreads();
    {
      const float2* r = sm + line * LP + tl;
#pragma unroll
      for (int k1 = 0; k1 < 32; ++k1) x[k1] = r[33 * (k1 >> 2) + 8 * (k1 & 3)];
    }
    if (ARRIVE) cluster_arrive();
    {
      const float2* twr = tw + 33 * tl;
#pragma unroll
      for (int k1 = 1; k1 < 32; ++k1) x[k1] = INV ? cmulc(x[k1], twr[k1]) : cmul(x[k1], twr[k1]);
    }
    dft_reg<32, INV>(x);
  }

  // ---- cluster exchanges ----
  // 32-bit shared::cluster address of `local` in the CTA of cluster rank `rank`
  static __device__ __forceinline__ uint32_t peer_addr(const void* local, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(r)
                 : "r"((uint32_t)__cvta_generic_to_shared(local)), "r"(rank));
    return r;
  }
  static __device__ __forceinline__ void st_peer(uint32_t addr, float2 v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
  }
  // A (row spectrum, register a*8+kB holds kc = 4tl + a + 32kB of row a_row())
  //   -> B (column slab, register e holds r = tl + 8e of spectral column b_kc())
  // (the caller arrived on the cluster barrier after its last read of sm)
  __device__ __forceinline__ void a_to_b(float2 (&x)[E], float2* sm, cg::cluster_group& cl) const {
    cluster_wait();  // every CTA of the cluster is done reading its buffer
    // bx(4tl + a + 32x, 64q + line) = [1042 tl + 64q + line] + 260a + 8336x
    const float2* mine = sm + 1042 * tl + 64 * q + line;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      const uint32_t dst = peer_addr(mine, (uint32_t)d);
#pragma unroll
      for (int xb = 0; xb < 2; ++xb)
#pragma unroll
        for (int a = 0; a < 4; ++a) st_peer(dst + 8u * (uint32_t)(260 * a + 8336 * xb), x[a * 8 + 2 * d + xb]);
    }
    cl.sync();
    const float2* r = sm + BP * line + 2 * (line >> 2) + tl;
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = r[8 * e];
  }
  // B (column slab, register e holds r = tl + 8e of spectral column b_kc())
  //   -> A (row spectrum distribution of row a_row())
  __device__ __forceinline__ void b_to_a(float2 (&x)[E], float2* sm, cg::cluster_group& cl) const {
    cluster_wait();  // arrived after the caller's last read of sm
    // ax(tl + 8j, 64q + line) = [274 tl + 68q + line + line/16] + 2192 j
    const float2* mine = sm + AP * tl + 68 * q + line + (line >> 4);
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      const uint32_t dst = peer_addr(mine, (uint32_t)d);
#pragma unroll
      for (int j = 0; j < 8; ++j) st_peer(dst + 8u * (uint32_t)(8 * AP * j), x[8 * d + j]);
    }
    cl.sync();
    // ax(line, 4tl + a + 32kB) = [274 line + 4tl + tl/4] + a + 34kB
    const float2* r = sm + AP * line + 4 * tl + (tl >> 2);
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int kB = 0; kB < 8; ++kB) x[a * 8 + kB] = r[a + 34 * kB];
  }

  // ---- whole 2-D transforms (unnormalised) ----
  // layout A real space -> layout B spectrum
  __device__ __forceinline__ void forward(float2 (&x)[E], float2* sm, const float2* tw, cg::cluster_group& cl) const {
    line_fwd<false, true>(x, sm, tw);
    a_to_b(x, sm, cl);
    line_fwd<false>(x, sm, tw);
  }
  // layout B spectrum -> layout A real space
  __device__ __forceinline__ void inverse(float2 (&x)[E], float2* sm, const float2* tw, cg::cluster_group& cl) const {
    line_bwd<true, true>(x, sm, tw);
    b_to_a(x, sm, cl);
    line_bwd<true>(x, sm, tw);
  }
};

}  // namespace qb
