// ntt_fast.cuh - specialised transform passes for the two-pass (N > 2^13) path.
//
// Same arithmetic and level order as ntt_core.cuh (radix-2 Gentleman-Sande DIF
// forward, Cooley-Tukey DIT inverse, grouped four levels per register pass),
// but every index is a compile-time function of the tile shape, the first
// group reads global memory straight into registers (16 or 32 independent
// loads in flight per thread) and the last group writes global memory straight
// from registers, so a pass costs one shared-memory round trip per middle group
// only.  Shared memory is XOR-swizzled so that every group's access pattern is
// free of bank conflicts.
#pragma once
#include "field.cuh"

namespace fpx_dev {

// ---------------------------------------------------------------------------
// Register butterfly groups.
// x holds 2^G points p0 + i*s (s = 2^S) of a block of length 2^LL; base = p0
// mod s.  Forward: levels len = 2^LL .. 2^(LL-G+1); inverse: the reverse.
// Twiddle index for level l, pair j: (len/2) + base + j*s.
// ---------------------------------------------------------------------------
template <int G, int LL, bool INV, int NA, bool ZB = false, bool ZH = false>
__device__ __forceinline__ void bf_group(uint32_t (&x)[2][1 << G], const uint2* __restrict__ tw, int base,
                                         const Fp& f) {
  // ZB: base == 0 (the last group of a transform), so every j == 0 twiddle is 1
  // and its butterfly needs no multiplication.
  // ZH (forward only): the upper half x[E/2..E) is zero (zero-padded input), so
  // the first level is u' = u, v' = u * w and x[E/2..E) need not hold anything.
  constexpr int E = 1 << G;
  constexpr int S = LL - G;
  uint2 w[E];  // w[hs + j]: twiddle of pair j at the level with pair distance hs
#pragma unroll
  for (int hs = 1; hs < E; hs <<= 1) {
#pragma unroll
    for (int j = 0; j < hs; ++j) {
      if (ZB && j == 0) continue;
      w[hs + j] = __ldg(&tw[(hs << S) + base + (j << S)]);
    }
  }
  if (!INV) {
    if constexpr (ZH) {
#pragma unroll
      for (int i = 0; i < E / 2; ++i)
#pragma unroll
        for (int a = 0; a < NA; ++a) x[a][i + E / 2] = (ZB && i == 0) ? x[a][i] : shoup(x[a][i], w[E / 2 + i], f.p);
    }
#pragma unroll
    for (int hs = ZH ? E / 4 : E / 2; hs >= 1; hs >>= 1) {
#pragma unroll
      for (int i = 0; i < E; ++i)
        if (!(i & hs)) {
          const int j = i & (hs - 1);
#pragma unroll
          for (int a = 0; a < NA; ++a) {
            if (ZB && j == 0) dif_bf1(x[a][i], x[a][i + hs], f);
            else dif_bf(x[a][i], x[a][i + hs], w[hs + j], f);
          }
        }
    }
  } else {
#pragma unroll
    for (int hs = 1; hs < E; hs <<= 1) {
#pragma unroll
      for (int i = 0; i < E; ++i)
        if (!(i & hs)) {
          const int j = i & (hs - 1);
#pragma unroll
          for (int a = 0; a < NA; ++a) {
            if (ZB && j == 0) dit_bf1(x[a][i], x[a][i + hs], f);
            else dit_bf(x[a][i], x[a][i + hs], w[hs + j], f);
          }
        }
    }
  }
}

__device__ __forceinline__ uint32_t brev_c(uint32_t t, int logn) { return logn ? (__brev(t) >> (32 - logn)) : 0u; }

// ---------------------------------------------------------------------------
// Row pass, C = 2^12, 256 threads, 16 points per thread per group.
//   group A: len 4096..512, thread t holds t + 256 i
//   group B: len 256..32,   thread t holds 256 (t>>4) + (t&15) + 16 i
//   group C: len 16..2,     thread t holds 16 t + i      (contiguous)
// Padded layout pad12(a) = a + 4 (a >> 5) + 16 (a >> 8): every pattern is free
// of bank conflicts, patterns A and B are a per-thread base plus compile-time
// offsets (304 i and 16 i + 4 (i >> 1)), and pattern C stays contiguous, so it
// moves with 128-bit accesses.
// ---------------------------------------------------------------------------
constexpr int kRowWords = 4096 + 512 + 256;
__device__ __forceinline__ int pad12(int a) { return a + 4 * (a >> 5) + 16 * (a >> 8); }
__device__ __forceinline__ int baseA(int t) { return pad12(t); }
__device__ __forceinline__ int baseB(int t) { return 304 * (t >> 4) + (t & 15); }
__device__ __forceinline__ int baseC(int t) { return pad12(t << 4); }
__host__ __device__ constexpr int offA(int i) { return 304 * i; }
__host__ __device__ constexpr int offB(int i) { return 16 * i + 4 * (i >> 1); }
__device__ __forceinline__ int posA(int t, int i) { return t + (i << 8); }
__device__ __forceinline__ int posC(int t, int i) { return (t << 4) + i; }

// Column pass tile: W = 2^LOGW adjacent columns x R = 2^LOGR rows, element
// (row t, col c) at smem word a = t*W + c, XOR-swizzled for the last group's
// pattern (instances one group-length apart):
//   a ^ (((a >> (GL+LOGW)) & (32/W - 1)) << LOGW).
// A padded layout would make every offset a compile-time constant, but its
// extra 1/8 of shared memory moves three resident CTAs past the 196 KB carveout
// and halves the L1 left for the twiddle tables, which costs more than the
// address arithmetic saves.
template <int LOGR, int LOGW, int GL>
struct ColSwz {
  static constexpr bool ON = GL + LOGW >= 5 && LOGW < 5;
  static constexpr int SH = GL + LOGW;         // the XOR key is a >> SH
  static constexpr int MB = ON ? 5 - LOGW : 0;  // key bits
  __host__ __device__ static constexpr int at(int a) {
    if constexpr (ON) {
      return a ^ (((a >> SH) & ((1 << MB) - 1)) << LOGW);
    } else {
      return a;
    }
  }
  // Addresses of the 2^G points of one group instance, element i at unswizzled
  // word a0 + (i << SS): the XOR key is periodic in i with period P, so
  // at(a_{kP+r}) = at(a_r) + k (P << SS) and a thread computes P swizzled bases
  // per instance, the rest being compile-time offsets.
  template <int SS, int G>
  struct Group {
    static constexpr int P0 = !ON ? 1 : (SS >= SH + MB ? 1 : (SS >= SH ? 1 << (SH + MB - SS) : 1 << MB));
    static constexpr int P = P0 < (1 << G) ? P0 : (1 << G);
    __device__ __forceinline__ static void bases(int a0, int (&b)[P]) {
#pragma unroll
      for (int r = 0; r < P; ++r) b[r] = at(a0 + (r << SS));
    }
    __device__ __forceinline__ static int addr(const int (&b)[P], int i) { return b[i % P] + (i / P) * (P << SS); }
  };
};

// Asynchronous global -> shared copies (cp.async), zero-filling past src_bytes.
__device__ __forceinline__ void cp_async16(uint32_t* smem, const uint32_t* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async4(uint32_t* smem, const uint32_t* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Group sizes of an R = 2^LOGR point column transform, largest first.
template <int LOGR>
struct ColGroups {
  static constexpr int K = (LOGR + 3) / 4;
  __host__ __device__ static constexpr int size(int k) { return LOGR / K + (k < LOGR % K ? 1 : 0); }
  __host__ __device__ static constexpr int top(int k) {  // log2 of the group's first block length
    int t = LOGR;
    for (int i = 0; i < k; ++i) t -= size(i);
    return t;
  }
};

}  // namespace fpx_dev
