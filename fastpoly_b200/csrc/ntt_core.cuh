// ntt_core.cuh - CTA-level transform building blocks.
//
// A CTA holds a tile of W interleaved transforms of R = 2^logR points each in
// shared memory: point `pos` of transform `c` lives at smem[pad(pos*W + c)].
// The transform runs as groups of up to four radix-2 levels; a thread loads
// the 2^G points of one butterfly group into registers, runs all G levels
// there, and writes them back.  Forward = Gentleman-Sande DIF from the largest
// block down (no bit reversal, spectrum left in bit-reversed order);
// inverse = Cooley-Tukey DIT from the smallest block up, the exact transpose.
// Both match the reference's radix-4 DIF/DIT pair level for level
// (ntt.hpp:859-946: a radix-4 stage is two radix-2 levels with these
// twiddles), so the spectrum permutation is the reference's.
//
// Twiddles come from one per-prime table `tw` with tw[h + k] = w_{2h}^k
// (w_len = g^((p-1)/len)) for every block length 2h <= 2^13, stored as
// (value, Shoup quotient) pairs; the inverse table holds w_{2h}^-k.
#pragma once
#include "field.cuh"

namespace fpx_dev {

constexpr int kSmallLog = 13;  // largest per-prime twiddle table: block length 2^13

__device__ __forceinline__ int pad(int a) { return a + (a >> 5); }
__host__ __device__ constexpr int padded_words(int n) { return n + (n >> 5) + 1; }

// One group of G DIF levels.  The group's first level has block length
// L = 2^lL; the thread's points are p0 + i*s with s = L >> G.
template <int G, bool INVERSE>
__device__ __forceinline__ void group_pass(uint32_t* __restrict__ sm, int logR, int logW, int lL,
                                           const uint2* __restrict__ tw, const Fp f, int tid, int nt) {
  constexpr int E = 1 << G;
  const int s_log = lL - G;
  const int s = 1 << s_log;
  const int ninst = 1 << (logR - G + logW);
  const int wmask = (1 << logW) - 1;
  for (int inst = tid; inst < ninst; inst += nt) {
    const int c = inst & wmask;
    const int rest = inst >> logW;
    const int base = rest & (s - 1);
    const int p0 = ((rest >> s_log) << lL) + base;
    uint32_t x[E];
#pragma unroll
    for (int i = 0; i < E; ++i) x[i] = sm[pad(((p0 + (i << s_log)) << logW) + c)];
    if (!INVERSE) {
#pragma unroll
      for (int l = 0; l < G; ++l) {
        const int hs = 1 << (G - 1 - l);
        const int half = 1 << (lL - 1 - l);
        uint2 w[E / 2];
#pragma unroll
        for (int j = 0; j < hs; ++j) w[j] = __ldg(&tw[half + base + (j << s_log)]);
#pragma unroll
        for (int i = 0; i < E; ++i)
          if (!(i & hs)) dif_bf(x[i], x[i + hs], w[i & (hs - 1)], f);
      }
    } else {
#pragma unroll
      for (int l = G - 1; l >= 0; --l) {
        const int hs = 1 << (G - 1 - l);
        const int half = 1 << (lL - 1 - l);
        uint2 w[E / 2];
#pragma unroll
        for (int j = 0; j < hs; ++j) w[j] = __ldg(&tw[half + base + (j << s_log)]);
#pragma unroll
        for (int i = 0; i < E; ++i)
          if (!(i & hs)) dit_bf(x[i], x[i + hs], w[i & (hs - 1)], f);
      }
    }
#pragma unroll
    for (int i = 0; i < E; ++i) sm[pad(((p0 + (i << s_log)) << logW) + c)] = x[i];
  }
}

template <bool INVERSE>
__device__ __forceinline__ void run_group(int G, uint32_t* sm, int logR, int logW, int lL, const uint2* tw,
                                          const Fp& f, int tid, int nt) {
  switch (G) {
    case 4: group_pass<4, INVERSE>(sm, logR, logW, lL, tw, f, tid, nt); break;
    case 3: group_pass<3, INVERSE>(sm, logR, logW, lL, tw, f, tid, nt); break;
    case 2: group_pass<2, INVERSE>(sm, logR, logW, lL, tw, f, tid, nt); break;
    default: group_pass<1, INVERSE>(sm, logR, logW, lL, tw, f, tid, nt); break;
  }
}

// Full forward DIF over the tile (groups of four levels from the top).
// Caller synchronises before (tile loaded) and after (tile complete).
__device__ __forceinline__ void tile_dif(uint32_t* sm, int logR, int logW, const uint2* tw, const Fp& f,
                                         int tid, int nt) {
  int lL = logR;
  while (lL > 0) {
    const int G = lL >= 4 ? 4 : lL;
    run_group<false>(G, sm, logR, logW, lL, tw, f, tid, nt);
    lL -= G;
    if (lL > 0) __syncthreads();
  }
}

// Full inverse DIT over the tile: the same groups in reverse order.
__device__ __forceinline__ void tile_dit(uint32_t* sm, int logR, int logW, const uint2* tw, const Fp& f,
                                         int tid, int nt) {
  // Group boundaries as in tile_dif (lL = logR, logR-4, ...), visited bottom-up.
  const int ng = (logR + 3) / 4;
  for (int gi = ng - 1; gi >= 0; --gi) {
    const int lL = logR - 4 * gi;
    run_group<true>(lL >= 4 ? 4 : lL, sm, logR, logW, lL, tw, f, tid, nt);
    if (gi > 0) __syncthreads();
  }
}

}  // namespace fpx_dev
