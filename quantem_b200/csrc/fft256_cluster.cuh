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
  static constexpr int PITCH = 264;  // == 8 (mod 16) float2: line pairs fall on opposite bank halves
  static constexpr int SM_FLOAT2 = LINES * PITCH;

  int q;     // cluster rank (0..3)
  int line;  // tid / 8
  int tl;    // tid % 8

  __device__ __forceinline__ void init(int tid, int rank) {
    q = rank;
    line = tid >> 3;
    tl = tid & 7;
  }
  // line-local exchange between the 32-point and the 8-point stage: element
  // (k1, t) of a line
  __device__ __forceinline__ int lx(int ln, int k1, int t) const { return ln * PITCH + 8 * k1 + (t ^ (k1 >> 2)); }
  // column-slab buffer: element (kc_local, r)
  __device__ __forceinline__ int bx(int kcl, int r) const { return kcl * PITCH + (r ^ (((kcl >> 2) & 3) << 2)); }
  // row-slab spectrum buffer: element (r_local, kc)
  __device__ __forceinline__ int ax(int rl, int kc) const {
    return rl * PITCH + (kc ^ ((kc >> 4) & 3) ^ (((rl >> 1) & 3) << 2));
  }

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

  // ---- 256-point transform along the line: x[e] = element tl + 8e in, natural
  //      frequency k = 4*tl + a + 32*kB in register a*8 + kB out ----
  template <bool INV>
  __device__ __forceinline__ void line_fwd(float2 (&x)[E], float2* sm, const float2* tw) const {
    dft_reg<32, INV>(x);
#pragma unroll
    for (int k1 = 1; k1 < 32; ++k1) {
      const float2 w = tw[(tl * k1) & 255];
      x[k1] = INV ? cmulc(x[k1], w) : cmul(x[k1], w);
    }
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) sm[lx(line, k1, tl)] = x[k1];
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int t = 0; t < 8; ++t) x[a * 8 + t] = sm[lx(line, 4 * tl + a, t)];
    dft8_groups<INV, 0>(x);
  }
  // inverse direction of line_fwd's data flow: frequency distribution in,
  // element tl + 8e out (INV selects the conjugate transform)
  template <bool INV>
  __device__ __forceinline__ void line_bwd(float2 (&x)[E], float2* sm, const float2* tw) const {
    dft8_groups<INV, 0>(x);
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int t = 0; t < 8; ++t) sm[lx(line, 4 * tl + a, t)] = x[a * 8 + t];
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) x[k1] = sm[lx(line, k1, tl)];
#pragma unroll
    for (int k1 = 1; k1 < 32; ++k1) {
      const float2 w = tw[(tl * k1) & 255];
      x[k1] = INV ? cmulc(x[k1], w) : cmul(x[k1], w);
    }
    dft_reg<32, INV>(x);
  }

  // ---- cluster exchanges ----
  // A (row spectrum, register a*8+kB holds kc = 4tl + a + 32kB of row a_row())
  //   -> B (column slab, register e holds r = tl + 8e of spectral column b_kc())
  __device__ __forceinline__ void a_to_b(float2 (&x)[E], float2* sm, cg::cluster_group& cl) const {
    cl.sync();  // every CTA of the cluster is done reading its buffer
    const int r = a_row();
#pragma unroll
    for (int kB = 0; kB < 8; ++kB) {
      float2* dst = cl.map_shared_rank(sm, (unsigned)(kB >> 1));
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int kcl = 4 * tl + a + 32 * (kB & 1);
        dst[bx(kcl, r)] = x[a * 8 + kB];
      }
    }
    cl.sync();
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = sm[bx(line, tl + 8 * e)];
  }
  // B (column slab, register e holds r = tl + 8e of spectral column b_kc())
  //   -> A (row spectrum distribution of row a_row())
  __device__ __forceinline__ void b_to_a(float2 (&x)[E], float2* sm, cg::cluster_group& cl) const {
    cl.sync();
    const int kc = b_kc();
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      float2* dst = cl.map_shared_rank(sm, (unsigned)d);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int e = 8 * d + j;
        dst[ax(tl + 8 * j, kc)] = x[e];  // r = tl + 8e, local row r - 64d = tl + 8j
      }
    }
    cl.sync();
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int kB = 0; kB < 8; ++kB) x[a * 8 + kB] = sm[ax(line, 4 * tl + a + 32 * kB)];
  }

  // ---- whole 2-D transforms (unnormalised) ----
  // layout A real space -> layout B spectrum
  __device__ __forceinline__ void forward(float2 (&x)[E], float2* sm, const float2* tw, cg::cluster_group& cl) const {
    line_fwd<false>(x, sm, tw);
    a_to_b(x, sm, cl);
    line_fwd<false>(x, sm, tw);
  }
  // layout B spectrum -> layout A real space
  __device__ __forceinline__ void inverse(float2 (&x)[E], float2* sm, const float2* tw, cg::cluster_group& cl) const {
    line_bwd<true>(x, sm, tw);
    b_to_a(x, sm, cl);
    line_bwd<true>(x, sm, tw);
  }
};

}  // namespace qb
