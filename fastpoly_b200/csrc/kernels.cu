// kernels.cu - sm_100a kernels for the NTT path and their host launchers.
//
// Transform decomposition (the reference's NttPlan, ntt.hpp:86-994, re-designed
// for one GPU):
//   * N <= 2^13: one CTA per transform, the whole DIF/DIT in shared memory
//     (k_small); pointwise product, scaling and the output window are fused.
//   * N  > 2^13: N = R x C, C = 2^12 (2^13 for N >= 2^24), R <= 2^12.
//       pass A (k_colfwd):  R-point DIF down each of the C columns (stride C),
//                           then the Bailey twiddle w_N^(j * bitrev_R(t));
//       pass B (k_rows):    C-point DIF along each contiguous row; optionally the
//                           second operand's rows, the pointwise product and the
//                           C-point DIT of the product, all while the row is in
//                           shared memory;
//       pass A' (k_colinv): inverse Bailey twiddle (1/N folded in), R-point DIT
//                           down the columns, and the caller's output window.
//     The spectrum of this factorisation sits at position t*C+u as
//     X[bitrev_R(t) + R*bitrev_C(u)] = X[bitrev_N(t*C+u)]: exactly the
//     reference's bit-reversed DIF order.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

#include "field.cuh"
#include "kernels.h"
#include "ntt_core.cuh"

using namespace fpx_dev;

namespace {

// Programmatic dependent launch.  Every kernel of this file is launched with
// programmatic stream serialization (pdl_launch), so the GPU may schedule it
// while the stream's previous kernel is still running: its launch latency
// hides behind the previous kernel's last wave.  The kernel lets its own
// dependents launch at once, then waits until the previous kernel has
// completed and its writes are visible before touching global memory; nothing
// before pdl_enter() reads or writes global memory.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Which launches take the attribute, by grid size in CTAs: measured on B200,
// back-to-back products gain 15-25 % with it at grids of up to 32 CTAs
// (transforms up to 2^17 points) and 5-13 % at grids of two waves and more
// (2^21 points and up), but lose 10-20 % at the grids in between (2^18-2^20
// points: 64-256 CTAs), so those launch without it.  FPX_PDL=0 in the
// environment turns it off everywhere; FPX_PDL_SMALL / FPX_PDL_LARGE move the
// two bounds (for measurements).
struct PdlPolicy {
  bool on = true;
  unsigned small = 32, large = 296;
};
const PdlPolicy& pdl_policy() {
  static const PdlPolicy pol = [] {
    PdlPolicy r;
    const char* e = std::getenv("FPX_PDL");
    r.on = !(e && e[0] == '0');
    if (const char* v = std::getenv("FPX_PDL_SMALL")) r.small = (unsigned)std::strtoul(v, nullptr, 10);
    if (const char* v = std::getenv("FPX_PDL_LARGE")) r.large = (unsigned)std::strtoul(v, nullptr, 10);
    return r;
  }();
  return pol;
}
bool pdl_for(dim3 grid) {
  const PdlPolicy& pol = pdl_policy();
  const unsigned ctas = grid.x * grid.y * grid.z;
  return pol.on && (ctas <= pol.small || ctas >= pol.large);
}

template <typename... KA, typename... A>
cudaError_t pdl_launch(void (*k)(KA...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_for(grid) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

struct Ptab {
  const uint2* fwd;
  const uint2* inv;
  Fp f;
  uint32_t q1;
};

Ptab dev_tab(const fpx::PrimeTables& pt) {
  return Ptab{reinterpret_cast<const uint2*>(pt.fwd), reinterpret_cast<const uint2*>(pt.inv), make_fp(pt.p), pt.q1};
}

struct InD {
  const uint32_t* ptr;
  uint32_t count;
  int reduce;
};
struct EpiD {
  uint32_t* out;
  uint32_t lo, hi;
  uint2 scale;
  const uint32_t* mul_mont;
  int negate;
  const uint32_t* sub_from;
  uint32_t sub_len;
  int accumulate;
};

InD dev_in(const fpx::InOp& x) { return InD{x.ptr, x.count, x.reduce}; }
EpiD dev_epi(const fpx::Epi& e) {
  return EpiD{e.out, e.lo, e.hi, make_uint2(e.scale.w, e.scale.q), e.mul_mont, e.negate, e.sub_from, e.sub_len,
              e.accumulate};
}

__device__ __forceinline__ uint32_t load_in(const InD& in, uint32_t i, const Fp& f, uint32_t q1) {
  if (i >= in.count) return 0u;
  uint32_t v = __ldg(in.ptr + i);
  return in.reduce ? reduce_any(v, q1, f) : v;
}

// Writes natural-order output x (lazy, < 4p) at global index gi through the epilogue.
__device__ __forceinline__ void epi_store(const EpiD& e, uint32_t gi, uint32_t x, const Fp& f) {
  if (gi < e.lo || gi >= e.hi) return;
  const uint32_t j = gi - e.lo;
  uint32_t v = e.scale.x ? shoup(x, e.scale, f.p) : red(x, f.p2);
  if (e.mul_mont) v = mont(v, __ldg(e.mul_mont + j), f);
  v = red(v, f.p);
  if (e.negate) v = v ? f.p - v : 0u;
  if (e.sub_from) {
    const uint32_t s = j < e.sub_len ? __ldg(e.sub_from + j) : 0u;
    v = s >= v ? s - v : s + f.p - v;
  }
  if (e.accumulate) v = red(v + e.out[j], f.p);
  e.out[j] = v;
}

// The plain epilogue (no scale, table, negation, subtraction or accumulation):
// canonical value into the window.
template <bool PLAIN>
__device__ __forceinline__ void epi_store_t(const EpiD& e, uint32_t gi, uint32_t x, const Fp& f) {
  if constexpr (PLAIN) {
    if (gi < e.lo || gi >= e.hi) return;
    e.out[gi - e.lo] = red(red(x, f.p2), f.p);
  } else {
    epi_store(e, gi, x, f);
  }
}
// Two adjacent outputs gi, gi + 1 of the plain epilogue: one 64-bit store when
// both fall in the window and the destination is 8-byte aligned.
template <bool PLAIN>
__device__ __forceinline__ void epi_store_pair(const EpiD& e, uint32_t gi, uint32_t x0, uint32_t x1, const Fp& f) {
  if constexpr (PLAIN) {
    if (gi >= e.lo && gi + 1 < e.hi) {
      uint32_t* o = e.out + (gi - e.lo);
      const uint32_t y0 = red(red(x0, f.p2), f.p), y1 = red(red(x1, f.p2), f.p);
      if (((uintptr_t)o & 7u) == 0) {
        *reinterpret_cast<uint2*>(o) = make_uint2(y0, y1);
      } else {
        o[0] = y0;
        o[1] = y1;
      }
      return;
    }
  }
  epi_store_t<PLAIN>(e, gi, x0, f);
  epi_store_t<PLAIN>(e, gi + 1, x1, f);
}
bool host_epi_plain(const fpx::Epi& e) {
  return e.scale.w == 0 && !e.mul_mont && !e.negate && !e.sub_from && !e.accumulate;
}


// ---------------------------------------------------------------------------
// Single-CTA transforms (N <= 2^13).
// ---------------------------------------------------------------------------
struct SmallD {
  InD x, y;
  int forward, ymode, inverse;
  const uint32_t* yspec;
  uint32_t* yspec_out;
  uint32_t* spec_x;
  EpiD epi;
};

__device__ __forceinline__ void small_body(const SmallD& job, const Ptab& pt, int logN) {
  extern __shared__ uint32_t sm[];
  const int N = 1 << logN, tid = threadIdx.x, nt = blockDim.x;
  uint32_t* X = sm;
  uint32_t* Y = sm + padded_words(N);
  const Fp f = pt.f;
  for (int i = tid; i < N; i += nt) X[pad(i)] = job.forward ? load_in(job.x, i, f, pt.q1) : __ldg(job.x.ptr + i);
  if (job.ymode == 1)
    for (int i = tid; i < N; i += nt) Y[pad(i)] = load_in(job.y, i, f, pt.q1);
  else if (job.ymode == 2)
    for (int i = tid; i < N; i += nt) Y[pad(i)] = __ldg(job.yspec + i);
  __syncthreads();
  if (job.forward) {
    tile_dif(X, logN, 0, pt.fwd, f, tid, nt);
    __syncthreads();
  }
  if (job.ymode == 1) {
    tile_dif(Y, logN, 0, pt.fwd, f, tid, nt);
    __syncthreads();
    if (job.yspec_out)
      for (int i = tid; i < N; i += nt) job.yspec_out[i] = red(Y[pad(i)], f.p);
  }
  if (job.ymode == 1 || job.ymode == 2) {
    for (int i = tid; i < N; i += nt) X[pad(i)] = mont(X[pad(i)], Y[pad(i)], f);
  } else if (job.ymode == 3) {
    for (int i = tid; i < N; i += nt) { const uint32_t v = X[pad(i)]; X[pad(i)] = mont(v, v, f); }
  }
  if (!job.inverse) {
    for (int i = tid; i < N; i += nt) job.spec_x[i] = red(X[pad(i)], f.p);
    return;
  }
  __syncthreads();
  tile_dit(X, logN, 0, pt.inv, f, tid, nt);
  __syncthreads();
  const uint32_t hi = job.epi.hi < (uint32_t)N ? job.epi.hi : (uint32_t)N;
  for (uint32_t i = job.epi.lo + tid; i < hi; i += nt) epi_store(job.epi, i, X[pad(i)], f);
}

__global__ void __launch_bounds__(512) k_small(SmallD job, Ptab pt, int logN) { pdl_enter(); small_body(job, pt, logN); }

// ---------------------------------------------------------------------------
// Pass A forward (columns).
// ---------------------------------------------------------------------------
struct ColOps {
  InD in[3];
  uint32_t* out[3];
};
struct BigD {
  int logR, logC, logW;
  const uint2* lo;   // w_N^y, y < 256
  const uint2* mid;  // w_N^(256 y), y < 256
  const uint2* hi;   // w_N^(65536 y), y < max(1, N / 65536)
  const uint4* cf;   // column factors of a column pair (BigTables::cf_fwd / cf_inv), or nullptr
  uint2 r32;         // 2^32 mod p with its Shoup quotient
};

// Bailey twiddle w_N^ex from the three small tables (5 KiB for N = 2^23, L1
// resident next to the per-prime table): three Shoup products.
__device__ __forceinline__ uint32_t bailey_mul(uint32_t x, uint32_t ex, const BigD& bt, const Fp& f) {
  x = shoup(x, __ldg(bt.lo + (ex & 255u)), f.p);
  x = shoup(x, __ldg(bt.mid + ((ex >> 8) & 255u)), f.p);
  return shoup(x, __ldg(bt.hi + (ex >> 16)), f.p);
}

// ---------------------------------------------------------------------------
// Pass B (rows), optionally fused with the second operand, the pointwise
// product and the row inverse.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_rows(uint32_t* x, const uint32_t* y, int ymode, uint32_t* y_spec_out,
                                               int forward, int inverse, int logC, Ptab pt) {
  pdl_enter();
  extern __shared__ uint32_t sm[];
  const int tid = threadIdx.x, nt = blockDim.x, C = 1 << logC;
  uint32_t* X = sm;
  uint32_t* Y = sm + padded_words(C);
  const size_t row = (size_t)blockIdx.x << logC;
  const Fp f = pt.f;
  for (int i = tid; i < C; i += nt) X[pad(i)] = x[row + i];
  if (ymode == 1 || ymode == 2)
    for (int i = tid; i < C; i += nt) Y[pad(i)] = __ldg(y + row + i);
  __syncthreads();
  if (forward) {
    tile_dif(X, logC, 0, pt.fwd, f, tid, nt);
    __syncthreads();
  }
  if (ymode == 1) {
    tile_dif(Y, logC, 0, pt.fwd, f, tid, nt);
    __syncthreads();
    if (y_spec_out)
      for (int i = tid; i < C; i += nt) y_spec_out[row + i] = red(Y[pad(i)], f.p);
  }
  if (ymode == 1 || ymode == 2) {
    for (int i = tid; i < C; i += nt) X[pad(i)] = mont(X[pad(i)], Y[pad(i)], f);
  } else if (ymode == 3) {
    for (int i = tid; i < C; i += nt) { const uint32_t v = X[pad(i)]; X[pad(i)] = mont(v, v, f); }
  }
  if (inverse) {
    __syncthreads();
    tile_dit(X, logC, 0, pt.inv, f, tid, nt);
  }
  __syncthreads();
  if (inverse) {
    for (int i = tid; i < C; i += nt) x[row + i] = X[pad(i)];
  } else {  // a spectrum leaves canonical (lazy values stay inside the transform)
    for (int i = tid; i < C; i += nt) x[row + i] = red(X[pad(i)], f.p);
  }
}


// ---------------------------------------------------------------------------
// Elementwise kernels.
// ---------------------------------------------------------------------------
__global__ void k_pointwise(Fp f, uint32_t* a, const uint32_t* b, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    a[i] = mont(a[i], b[i], f);
}

// Sum of pointwise products of spectra, the spectral side of a blocked
// product: acc[i] (+)= sum_t x_t[i] y_t[i] * 2^-32 mod p, canonical; inputs
// lazy below 4p.  Four words per thread per step (16-byte loads).
constexpr int kMacPairs = 16;
struct MacPairs {
  const uint4* x[kMacPairs];
  const uint4* y[kMacPairs];
  int n;
};
__device__ __forceinline__ uint32_t mac1(uint32_t acc, uint32_t x, uint32_t y, const Fp& f) {
  return red(acc + red(mont(canon4(x, f), canon4(y, f), f), f.p), f.p);
}
__global__ void k_spec_mac(Fp f, MacPairs pr, uint4* acc, size_t n4, int accumulate) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    uint4 s = accumulate ? acc[i] : make_uint4(0u, 0u, 0u, 0u);
    for (int t = 0; t < pr.n; ++t) {
      const uint4 x = __ldg(pr.x[t] + i), y = __ldg(pr.y[t] + i);
      s.x = mac1(s.x, x.x, y.x, f);
      s.y = mac1(s.y, x.y, y.y, f);
      s.z = mac1(s.z, x.z, y.z, f);
      s.w = mac1(s.w, x.w, y.w, f);
    }
    acc[i] = s;
  }
}

struct GarnerC {
  uint32_t P1, P2, P3;
  uint2 inv12;      // P1^-1 mod P2 (Shoup)
  uint2 p1_in3;     // P1 mod P3
  uint2 inv123;     // (P1 P2)^-1 mod P3
  uint32_t t;       // target modulus
  uint32_t t_q1;    // floor(2^32 / t)
  uint2 p1_t;       // P1 mod t
  uint2 p12_t;      // P1 P2 mod t
};

__device__ __forceinline__ uint32_t redc_any(uint32_t x, uint32_t m) { return min(x, x - m); }

// One coefficient from its residues r1, r2, r3 (mod P1, P2, P3; the first
// `primes` of them), reduced into the target field.
__device__ __forceinline__ uint32_t garner_one(const GarnerC& g, int primes, uint32_t x1, uint32_t r2, uint32_t r3) {
  uint32_t v = x1 - __umulhi(x1, g.t_q1) * g.t;
  v = redc_any(v, g.t);
  if (primes >= 2) {
    uint32_t x2 = redc_any(shoup(r2 + g.P2 - x1, g.inv12, g.P2), g.P2);
    uint32_t v2 = redc_any(shoup(x2, g.p1_t, g.t), g.t);
    v = redc_any(v + v2, g.t);
    if (primes == 3) {
      const uint32_t y = redc_any(shoup(x2, g.p1_in3, g.P3), g.P3);
      const uint32_t x12 = redc_any(x1 + y, g.P3);  // x1 + P1*x2 mod P3
      const uint32_t x3 = redc_any(shoup(r3 + g.P3 - x12, g.inv123, g.P3), g.P3);
      const uint32_t v3 = redc_any(shoup(x3, g.p12_t, g.t), g.t);
      v = redc_any(v + v3, g.t);
    }
  }
  return v;
}
// The epilogue of output i: the Montgomery table factor, negation, accumulation, store.
__device__ __forceinline__ void garner_put(const GarnerC& g, uint32_t v, uint32_t* out, size_t i, int accumulate,
                                           const uint32_t* post_mont, int negate, uint32_t tpinv) {
  if (post_mont) {  // Montgomery table product in the target field (odd target)
    const Fp ft{g.t, 2 * g.t, tpinv};
    v = red(mont(v, __ldg(post_mont + i), ft), g.t);
  }
  if (negate && v) v = g.t - v;
  if (accumulate) v = redc_any(v + out[i], g.t);
  out[i] = v;
}

__device__ __forceinline__ void garner_body(const GarnerC& g, int primes, const uint32_t* c1, const uint32_t* c2,
                                            const uint32_t* c3, uint32_t* out, size_t n, int accumulate,
                                            const uint32_t* post_mont = nullptr, int negate = 0,
                                            uint32_t tpinv = 0, size_t first = 0, size_t span = ~size_t(0)) {
  // outputs [first, min(n, first + span)), grid-stride over the whole range when span is unbounded
  const bool whole = span == ~size_t(0);
  const size_t end = whole ? n : (first + span < n ? first + span : n);
  const size_t step = whole ? (size_t)gridDim.x * blockDim.x : blockDim.x;
  for (size_t i = (whole ? blockIdx.x * (size_t)blockDim.x : first) + threadIdx.x; i < end; i += step) {
    const uint32_t v = garner_one(g, primes, c1[i], primes >= 2 ? c2[i] : 0u, primes == 3 ? c3[i] : 0u);
    garner_put(g, v, out, i, accumulate, post_mont, negate, tpinv);
  }
}

__global__ void k_garner(GarnerC g, int primes, const uint32_t* c1, const uint32_t* c2, const uint32_t* c3,
                         uint32_t* out, size_t n, int accumulate) {
  pdl_enter();
  garner_body(g, primes, c1, c2, c3, out, n, accumulate);
}

// The same over 16-byte aligned residues, four consecutive outputs per thread
// (16-byte loads, four independent chains), grid-stride.
__global__ void k_garner4(GarnerC g, int primes, const uint32_t* c1, const uint32_t* c2, const uint32_t* c3,
                          uint32_t* out, size_t n, int accumulate) {
  pdl_enter();
  const size_t stride = 4 * (size_t)gridDim.x * blockDim.x;
  for (size_t i = 4 * (blockIdx.x * (size_t)blockDim.x + threadIdx.x); i < n; i += stride) {
    if (i + 4 <= n) {
      const uint4 a = *reinterpret_cast<const uint4*>(c1 + i);
      const uint4 b = primes >= 2 ? *reinterpret_cast<const uint4*>(c2 + i) : make_uint4(0u, 0u, 0u, 0u);
      const uint4 c = primes == 3 ? *reinterpret_cast<const uint4*>(c3 + i) : make_uint4(0u, 0u, 0u, 0u);
      const uint32_t v0 = garner_one(g, primes, a.x, b.x, c.x), v1 = garner_one(g, primes, a.y, b.y, c.y);
      const uint32_t v2 = garner_one(g, primes, a.z, b.z, c.z), v3 = garner_one(g, primes, a.w, b.w, c.w);
      garner_put(g, v0, out, i, accumulate, nullptr, 0, 0);
      garner_put(g, v1, out, i + 1, accumulate, nullptr, 0, 0);
      garner_put(g, v2, out, i + 2, accumulate, nullptr, 0, 0);
      garner_put(g, v3, out, i + 3, accumulate, nullptr, 0, 0);
    } else {
      for (size_t t = i; t < n; ++t)
        garner_put(g, garner_one(g, primes, c1[t], primes >= 2 ? c2[t] : 0u, primes == 3 ? c3[t] : 0u), out, t,
                   accumulate, nullptr, 0, 0);
    }
  }
}

__global__ void k_from_mont(Fp f, const uint32_t* in, uint32_t* out, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = red(mont(in[i], 1u, f), f.p);
}
__global__ void k_bits2(const uint32_t* in, uint32_t* out, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[i] & 1u;
}
__global__ void k_scale(uint32_t p, const uint32_t* in, uint32_t* out, size_t n, uint2 c) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = redc_any(shoup(in[i], c, p), p);
}

__device__ uint32_t mont_pow(uint32_t base_m, uint32_t e, uint32_t one_m, const Fp& f) {
  uint32_t r = one_m, b = base_m;
  while (e) {
    if (e & 1) r = red(mont(r, b, f), f.p);
    b = red(mont(b, b, f), f.p);
    e >>= 1;
  }
  return r;
}

// tab[i] = (1/i) * 2^32 mod p for 1 <= i <= n (i < p), tab[0] = 0.
__global__ void k_inv_table(Fp f, uint2 r_sh, uint2 r2_sh, uint32_t* tab, size_t n) {
  pdl_enter();
  const uint32_t one_m = red(shoup(1u, r_sh, f.p), f.p);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i <= n; i += (size_t)gridDim.x * blockDim.x) {
    if (i == 0) { tab[0] = 0; continue; }
    const uint32_t im = red(shoup((uint32_t)i, r_sh, f.p), f.p);  // i * 2^32 mod p
    tab[i] = mont_pow(im, f.p - 2, one_m, f);                        // (1/i) * 2^32
  }
}

__global__ void k_derivative(Fp f, uint32_t q1, uint2 r_sh, const uint32_t* a, uint32_t* r, size_t cnt1) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cnt1; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t k = reduce_any((uint32_t)(i + 1), q1, f);
    const uint32_t t = red(mont(a[i + 1], k, f), f.p);   // a*k/R
    r[i] = red(shoup(t, r_sh, f.p), f.p);                // * R
  }
}

// Direct product window (short operand a, la <= 40):
// out[i] = sum_j a[j] * b[i + off - j].
__device__ __forceinline__ void direct_body(uint32_t p, const Fp& f, const uint32_t* a, int la, const uint32_t* b,
                                            size_t lb, size_t off, size_t cnt, uint32_t* out, int accumulate,
                                            const uint32_t* post_mont = nullptr, int negate = 0,
                                            size_t first = 0, size_t span = ~size_t(0)) {
  __shared__ uint32_t am[64];
  if (threadIdx.x < la) {
    const uint32_t v = a[threadIdx.x];
    am[threadIdx.x] = (p == 2) ? v : (uint32_t)(((uint64_t)v << 32) % p);  // Montgomery form of a[j]
  }
  __syncthreads();
  // outputs [first, min(cnt, first + span)), grid-stride over the whole range when span is unbounded
  const bool whole = span == ~size_t(0);
  const size_t end = whole ? cnt : (first + span < cnt ? first + span : cnt);
  const size_t step = whole ? (size_t)gridDim.x * blockDim.x : blockDim.x;
  for (size_t i = (whole ? blockIdx.x * (size_t)blockDim.x : first) + threadIdx.x; i < end; i += step) {
    const size_t k = i + off;
    uint64_t acc = 0;
    uint32_t bits = 0;
    const int jlo = k >= lb ? (int)(k - lb + 1) : 0;
    const int jhi = (int)((size_t)la - 1 < k ? (size_t)la - 1 : k);
    for (int j = jlo; j <= jhi; ++j) {
      const uint32_t bv = __ldg(b + (k - j));
      if (p == 2) bits ^= am[j] & bv;
      else acc += mont(am[j], bv, f);
    }
    uint32_t v = (p == 2) ? (bits & 1u) : (uint32_t)(acc % p);
    if (post_mont) v = red(mont(v, __ldg(post_mont + i), f), f.p);
    if (negate && v) v = p - v;
    if (accumulate) {
      const uint64_t s = (uint64_t)v + out[i];
      v = (uint32_t)(s >= p ? s - p : s);
    }
    out[i] = v;
  }
}

__global__ void k_direct(uint32_t p, Fp f, uint2 r_sh, const uint32_t* a, int la, const uint32_t* b, size_t lb,
                         size_t off, size_t cnt, uint32_t* out, int accumulate) {
  pdl_enter();
  direct_body(p, f, a, la, b, lb, off, cnt, out, accumulate);
}

int grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  return b ? (int)b : 1;
}

uint2 shoup_const(uint32_t w, uint32_t p) { return make_uint2(w, (uint32_t)(((uint64_t)w << 32) / p)); }

// ---------------------------------------------------------------------------
// Newton inverse at the small sizes in one CTA.  The doubling steps k -> 2k of
// the series inverse (inverse.hpp:18-65) with 2k <= 2^13 points run back to
// back in shared memory: per step the middle product h = -(a c)[k, 2k) and the
// product (h c) mod x^(2k-k) as cyclic products of 2k points (wrap-free for
// these windows), exactly what the per-step launches compute, with no launch,
// global round trip or host step between them.  c[0, k0) holds the seed.
// ---------------------------------------------------------------------------
constexpr int kNewtonThreads = 512;
constexpr int kNewtonMaxLog = kSmallLog;  // 2k <= 2^13: the per-prime twiddle table
constexpr int kNewtonPW = padded_words(1 << kNewtonMaxLog);
constexpr int kNewtonSmemWords = 2 * kNewtonPW + (1 << kNewtonMaxLog) + (1 << (kNewtonMaxLog - 1));

struct NewtonInvD {
  const uint32_t* a;  // the series (canonical, a[0] != 0), la terms
  uint32_t la;
  uint32_t* c;        // its inverse: c[0, k0) on entry (k0 = 0: computed here), c[0, K) on return
  uint32_t k0, K;     // k0 0 or a power of two, K <= 2^13
  uint32_t r1, r2;    // 2^32 and 2^64 mod p
  uint2 scale_r[kNewtonMaxLog + 1];  // Shoup constants of 2^32 / 2^l mod p (undo N and the Montgomery factor)
};

// X[0, N) <- src[0, len), zero beyond (plain loads: global or shared memory).
__device__ __forceinline__ void cta_load(uint32_t* X, const uint32_t* src, uint32_t len, uint32_t N, int tid,
                                         int nt) {
  for (uint32_t i = tid; i < N; i += nt) X[pad(i)] = i < len ? src[i] : 0u;
}

// Forward (DIF) groups of the one-CTA products, with the pointwise product
// folded into the last group: after its butterflies a thread holds final
// spectrum values and multiplies them at once (Montgomery; DIF outputs are in
// [0, 2p), so every product is below p 2^32), saving a shared-memory pass and
// a barrier per product.  Modes: kNtMulSpec X <- DIF(X) * S (S a spectrum);
// kNtPair Y <- DIF(Y) and X <- DIF(X) * DIF(Y), both transforms in one pass per
// group (the same positions, so the same twiddles and the products in
// registers); kNtSquare X <- DIF(X)^2.  Grouping and butterflies are those of
// tile_dif, so every value is the one tile_dif and a separate pointwise pass
// give.
enum { kNtMulSpec = 1, kNtPair = 2, kNtSquare = 3 };

template <int G, int MODE>
__device__ __forceinline__ void nt_group(uint32_t* X, uint32_t* Y, const uint32_t* S, int logN, int lL, bool last,
                                         const uint2* __restrict__ tw, const Fp& f, int tid, int nt) {
  constexpr int E = 1 << G;
  constexpr bool PAIR = MODE == kNtPair;
  const int s_log = lL - G;
  const int ninst = 1 << (logN - G);
  for (int inst = tid; inst < ninst; inst += nt) {
    const int base = inst & ((1 << s_log) - 1);
    const int p0 = ((inst >> s_log) << lL) + base;
    uint32_t x[E], y[PAIR ? E : 1];
#pragma unroll
    for (int i = 0; i < E; ++i) {
      x[i] = X[pad(p0 + (i << s_log))];
      if constexpr (PAIR) y[i] = Y[pad(p0 + (i << s_log))];
    }
#pragma unroll
    for (int l = 0; l < G; ++l) {
      const int hs = 1 << (G - 1 - l);
      const int half = 1 << (lL - 1 - l);
      uint2 w[E / 2];
#pragma unroll
      for (int j = 0; j < hs; ++j) w[j] = __ldg(&tw[half + base + (j << s_log)]);
#pragma unroll
      for (int i = 0; i < E; ++i)
        if (!(i & hs)) {
          dif_bf(x[i], x[i + hs], w[i & (hs - 1)], f);
          if constexpr (PAIR) dif_bf(y[i], y[i + hs], w[i & (hs - 1)], f);
        }
    }
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int q = pad(p0 + (i << s_log));
      if constexpr (PAIR) Y[q] = y[i];
      if (last) {
        const uint32_t m = MODE == kNtPair ? y[PAIR ? i : 0] : (MODE == kNtMulSpec ? S[q] : x[i]);
        X[q] = mont(x[i], m, f);
      } else {
        X[q] = x[i];
      }
    }
  }
}

// The forward transform(s) of `nt_group` over N = 2^logN points; returns
// synchronised.
template <int MODE>
__device__ __forceinline__ void nt_fwd_mul(uint32_t* X, uint32_t* Y, const uint32_t* S, int logN, const Ptab& pt,
                                           int tid, int nt) {
  if (logN == 0) {  // one point: the pointwise product alone
    if (tid == 0) X[0] = mont(X[0], MODE == kNtPair ? Y[0] : (MODE == kNtMulSpec ? S[0] : X[0]), pt.f);
    __syncthreads();
    return;
  }
  int lL = logN;
  while (lL > 0) {
    const int G = lL >= 4 ? 4 : lL;
    const bool last = lL == G;
    switch (G) {
      case 4: nt_group<4, MODE>(X, Y, S, logN, lL, last, pt.fwd, pt.f, tid, nt); break;
      case 3: nt_group<3, MODE>(X, Y, S, logN, lL, last, pt.fwd, pt.f, tid, nt); break;
      case 2: nt_group<2, MODE>(X, Y, S, logN, lL, last, pt.fwd, pt.f, tid, nt); break;
      default: nt_group<1, MODE>(X, Y, S, logN, lL, last, pt.fwd, pt.f, tid, nt); break;
    }
    lL -= G;
    __syncthreads();
  }
}

// X <- DIT(DIF(X) * Y) over N = 2^logN points, Y a spectrum (Montgomery
// pointwise; the caller scales by 2^32 / N).  Call after X is loaded and
// synchronised; returns synchronised.
__device__ __forceinline__ void cta_mul(uint32_t* X, const uint32_t* Y, int logN, const Ptab& pt, int tid, int nt) {
  nt_fwd_mul<kNtMulSpec>(X, nullptr, Y, logN, pt, tid, nt);
  tile_dit(X, logN, 0, pt.inv, pt.f, tid, nt);
  __syncthreads();
}

// Y <- DIF(Y), X <- DIT(DIF(X) * DIF(Y)): both operands loaded and
// synchronised; Y keeps its spectrum for later products.
__device__ __forceinline__ void cta_mul2(uint32_t* X, uint32_t* Y, int logN, const Ptab& pt, int tid, int nt) {
  nt_fwd_mul<kNtPair>(X, Y, nullptr, logN, pt, tid, nt);
  tile_dit(X, logN, 0, pt.inv, pt.f, tid, nt);
  __syncthreads();
}

// X <- DIT(DIF(X)^2) over N = 2^logN points (the caller scales by 2^32 / N).
__device__ __forceinline__ void cta_mul_self(uint32_t* X, int logN, const Ptab& pt, int tid, int nt) {
  nt_fwd_mul<kNtSquare>(X, nullptr, nullptr, logN, pt, tid, nt);
  tile_dit(X, logN, 0, pt.inv, pt.f, tid, nt);
  __syncthreads();
}

// One doubling step of the series inverse: Cs[k, want) from Cs[0, k) and the
// first aw terms of the series (want <= 2k), at N = 2k points: h = -(a c)[k, want),
// then c[k + i] = (h c)[i].  Y holds c's spectrum afterwards.  gc: optional
// global copy of the new terms.
__device__ __forceinline__ void cta_inv_step(const uint32_t* series, uint32_t aw, uint32_t* Cs, uint32_t* gc,
                                             uint32_t k, uint32_t want, uint32_t* X, uint32_t* Y, uint32_t* H,
                                             const uint2* scale_r, const Ptab& pt, int tid, int nt) {
  const Fp f = pt.f;
  const uint32_t hl = want - k;
  const int logN = 32 - __clz(2 * k - 1);
  const uint32_t N = 1u << logN;
  const uint2 sc = scale_r[logN];
  cta_load(X, series, aw, N, tid, nt);
  cta_load(Y, Cs, k, N, tid, nt);
  __syncthreads();
  cta_mul2(X, Y, logN, pt, tid, nt);
  for (uint32_t i = tid; i < hl; i += nt) {
    const uint32_t v = red(shoup(X[pad(k + i)], sc, f.p), f.p);
    H[i] = v ? f.p - v : 0u;
  }
  __syncthreads();
  cta_load(X, H, hl, N, tid, nt);
  __syncthreads();
  cta_mul(X, Y, logN, pt, tid, nt);
  for (uint32_t i = tid; i < hl; i += nt) {
    const uint32_t v = red(shoup(X[pad(i)], sc, f.p), f.p);
    Cs[k + i] = v;
    if (gc) gc[k + i] = v;
  }
  __syncthreads();
}

__device__ __forceinline__ void newton_inv_body(const NewtonInvD& d, const Ptab& pt) {
  extern __shared__ uint32_t smn[];
  uint32_t* X = smn;                      // transform buffer, padded
  uint32_t* Y = smn + kNewtonPW;          // spectrum of c[0, k), padded
  uint32_t* Cs = smn + 2 * kNewtonPW;     // c[0, K)
  uint32_t* H = Cs + (1 << kNewtonMaxLog);  // h, < 2^12 terms
  const int tid = threadIdx.x, nt = blockDim.x;
  const Fp f = pt.f;
  uint32_t k = d.k0;
  if (k == 0) {
    // c[0] = a[0]^(p-2) mod p by Montgomery square-and-multiply
    if (tid == 0) {
      const uint32_t am = mont(__ldg(d.a), d.r2, f);
      uint32_t r = d.r1;
      for (int b = 31 - __clz(f.p - 2); b >= 0; --b) {
        r = mont(r, r, f);
        if (((f.p - 2) >> b) & 1u) r = mont(r, am, f);
      }
      const uint32_t c0 = red(mont(r, 1u, f), f.p);
      Cs[0] = c0;
      d.c[0] = c0;
    }
    k = 1;
  } else {
    for (uint32_t i = tid; i < k; i += nt) Cs[i] = d.c[i];
  }
  __syncthreads();
  for (; k < d.K; k <<= 1) {
    const uint32_t want = min(2 * k, d.K);
    cta_inv_step(d.a, min(d.la, want), Cs, d.c, k, want, X, Y, H, d.scale_r, pt, tid, nt);
  }
}

__global__ void __launch_bounds__(kNewtonThreads) k_newton_inv(NewtonInvD d, Ptab pt) {
  pdl_enter();
  newton_inv_body(d, pt);
}

// ---------------------------------------------------------------------------
// Newton exponential at the small sizes in one CTA (exponential.hpp:107-207):
// from b = 1, c = 1/b = 1, each step m -> m2 = min(2m, K) extends c to
// m2 - m terms (inverse doubling on b), then with N = 2m points
//   t1 = (a' b)[m-1, m2-1),  t2 = (t1 c) mod x^(m2-m) times 1/(m+i),
//   b[m + i] = (t2 b)[i],
// the same products as the per-step launches (wrap-free windows at N = 2m).
// ---------------------------------------------------------------------------
constexpr int kNewtonExpSmemWords = 3 * kNewtonPW + (1 << kNewtonMaxLog) + 2 * (1 << (kNewtonMaxLog - 1));

struct NewtonExpD {
  const uint32_t* ap;   // a' (canonical), lap terms
  uint32_t lap;
  const uint32_t* tab;  // 1/i in Montgomery form, i < K
  uint32_t* b;          // exp(a): b[0, K)
  uint32_t* c;          // 1/b: c[0, cs) on return (cs as the host computes it)
  uint32_t K;           // <= 2^13
  uint2 scale_r[kNewtonMaxLog + 1];
};

__device__ __forceinline__ void newton_exp_body(const NewtonExpD& d, const Ptab& pt) {
  extern __shared__ uint32_t smn[];
  uint32_t* X = smn;
  uint32_t* Y = smn + kNewtonPW;
  uint32_t* S = smn + 2 * kNewtonPW;        // spectrum of b[0, m)
  uint32_t* B = smn + 3 * kNewtonPW;        // b[0, K)
  uint32_t* Cs = B + (1 << kNewtonMaxLog);  // c, < 2^12 terms
  uint32_t* T = Cs + (1 << (kNewtonMaxLog - 1));
  const int tid = threadIdx.x, nt = blockDim.x;
  const Fp f = pt.f;
  if (tid == 0) {
    B[0] = 1u;
    Cs[0] = 1u;
    d.b[0] = 1u;
  }
  __syncthreads();
  uint32_t m = 1, cs = 1;
  while (m < d.K) {
    const uint32_t m2 = min(2 * m, d.K), hl = m2 - m;
    while (cs < hl) {
      const uint32_t want = min(2 * cs, hl);
      cta_inv_step(B, min(m, want), Cs, nullptr, cs, want, X, Y, T, d.scale_r, pt, tid, nt);
      cs = want;
    }
    const int logN = 32 - __clz(2 * m - 1);
    const uint32_t N = 1u << logN;
    const uint2 sc = d.scale_r[logN];
    // t1 = (a' b)[m-1, m-1+hl)
    cta_load(X, d.ap, min(d.lap, m2 - 1), N, tid, nt);
    cta_load(S, B, m, N, tid, nt);
    __syncthreads();
    cta_mul2(X, S, logN, pt, tid, nt);
    for (uint32_t i = tid; i < hl; i += nt) T[i] = red(shoup(X[pad(m - 1 + i)], sc, f.p), f.p);
    __syncthreads();
    // t2 = (t1 c) mod x^hl, times 1/(m+i)
    cta_load(X, T, hl, N, tid, nt);
    cta_load(Y, Cs, cs, N, tid, nt);
    __syncthreads();
    cta_mul2(X, Y, logN, pt, tid, nt);
    for (uint32_t i = tid; i < hl; i += nt)
      T[i] = red(mont(shoup(X[pad(i)], sc, f.p), __ldg(d.tab + m + i), f), f.p);
    __syncthreads();
    // b[m + i] = (t2 b)[i]
    cta_load(X, T, hl, N, tid, nt);
    __syncthreads();
    cta_mul(X, S, logN, pt, tid, nt);
    for (uint32_t i = tid; i < hl; i += nt) {
      const uint32_t v = red(shoup(X[pad(i)], sc, f.p), f.p);
      B[m + i] = v;
      d.b[m + i] = v;
    }
    __syncthreads();
    m = m2;
  }
  for (uint32_t i = tid; i < cs; i += nt) d.c[i] = Cs[i];
}

__global__ void __launch_bounds__(kNewtonThreads) k_newton_exp(NewtonExpD d, Ptab pt) {
  pdl_enter();
  newton_exp_body(d, pt);
}

// Many small Newton inverses and exponentials (batches), one CTA per job.
struct NewtonJobB {
  int kind;  // 0 inverse, 1 exponential
  Ptab pt;
  NewtonInvD inv;
  NewtonExpD exp;
};
__global__ void __launch_bounds__(kNewtonThreads) k_newton_b(const NewtonJobB* __restrict__ jobs) {
  pdl_enter();
  const NewtonJobB& j = jobs[blockIdx.x];
  if (j.kind == 0) newton_inv_body(j.inv, j.pt);
  else newton_exp_body(j.exp, j.pt);
}

// ---------------------------------------------------------------------------
// Newton square root at the small sizes in one CTA (square_root.hpp:12-112):
// from b = root of u[0] and c = 1/b, each step m -> m2 = min(2m, K) extends c
// to m2 - m terms, then with N = 2m points
//   t = u[m+i] - (b^2)[m+i],  b[m + i] = (t c)[i] / 2,
// the same products as the per-step launches (wrap-free windows at N = 2m).
// ---------------------------------------------------------------------------
constexpr int kNewtonSqrtSmemWords = 2 * kNewtonPW + (1 << kNewtonMaxLog) + 2 * (1 << (kNewtonMaxLog - 1));

struct NewtonSqrtD {
  const uint32_t* u;  // the series with u[0] a nonzero square (canonical), ulen terms
  uint32_t ulen;
  uint32_t* b;        // sqrt(u): b[0, K)
  uint32_t* c;        // 1/b: c[0, cs) on return (cs as for the exponential)
  uint32_t K;         // <= 2^13
  uint32_t root, root_inv;  // b[0] and 1/b[0]
  uint2 scale_r[kNewtonMaxLog + 1];
};

__global__ void __launch_bounds__(kNewtonThreads) k_newton_sqrt(NewtonSqrtD d, Ptab pt) {
  pdl_enter();
  extern __shared__ uint32_t smn[];
  uint32_t* X = smn;
  uint32_t* Y = smn + kNewtonPW;
  uint32_t* B = smn + 2 * kNewtonPW;        // b[0, K)
  uint32_t* Cs = B + (1 << kNewtonMaxLog);  // c, < 2^12 terms
  uint32_t* T = Cs + (1 << (kNewtonMaxLog - 1));
  const int tid = threadIdx.x, nt = blockDim.x;
  const Fp f = pt.f;
  if (tid == 0) {
    B[0] = d.root;
    Cs[0] = d.root_inv;
    d.b[0] = d.root;
  }
  __syncthreads();
  uint32_t m = 1, cs = 1;
  while (m < d.K) {
    const uint32_t m2 = min(2 * m, d.K), hl = m2 - m;
    while (cs < hl) {
      const uint32_t want = min(2 * cs, hl);
      cta_inv_step(B, min(m, want), Cs, nullptr, cs, want, X, Y, T, d.scale_r, pt, tid, nt);
      cs = want;
    }
    const int logN = 32 - __clz(2 * m - 1);
    const uint32_t N = 1u << logN;
    const uint2 sc = d.scale_r[logN];
    // t = u[m + i] - (b^2)[m + i]
    cta_load(X, B, m, N, tid, nt);
    __syncthreads();
    cta_mul_self(X, logN, pt, tid, nt);
    for (uint32_t i = tid; i < hl; i += nt) {
      const uint32_t v = red(shoup(X[pad(m + i)], sc, f.p), f.p);
      const uint32_t su = m + i < d.ulen ? d.u[m + i] : 0u;
      T[i] = su >= v ? su - v : su + f.p - v;
    }
    __syncthreads();
    // b[m + i] = (t c)[i] / 2
    cta_load(X, T, hl, N, tid, nt);
    cta_load(Y, Cs, cs, N, tid, nt);
    __syncthreads();
    cta_mul2(X, Y, logN, pt, tid, nt);
    for (uint32_t i = tid; i < hl; i += nt) {
      const uint32_t v = red(shoup(X[pad(i)], sc, f.p), f.p);
      const uint32_t h = (v & 1u) ? (v + f.p) >> 1 : v >> 1;  // v / 2 mod p (p odd)
      B[m + i] = h;
      d.b[m + i] = h;
    }
    __syncthreads();
    m = m2;
  }
  for (uint32_t i = tid; i < cs; i += nt) d.c[i] = Cs[i];
}

// ---------------------------------------------------------------------------
// Newton inverse, exponential and square root at the small sizes for a prime
// modulus P without the roots of unity (1e9+7, 2^31-1, small primes), on a
// cluster of three CTAs, one per transform prime 167772161, 469762049,
// 754974721: the doubling steps of inverse.hpp:18-65, exponential.hpp:107-207
// and square_root.hpp:12-112, every product a three-prime CRT product
// (crt_convolution.hpp:25-127).  For a product each CTA lifts the operands into
// its prime and runs the cyclic product of 2k points in shared memory; after a
// cluster barrier every CTA reads the three residue windows (its own and,
// through distributed shared memory, the other two) and runs Garner back to P,
// so each CTA holds the product's terms for the next one.  Two residue buffers
// alternate, so one cluster barrier per product suffices: a CTA overwrites a
// buffer only after the next product's barrier, which every CTA reaches after
// reading it.  The windows are the per-step path's (wrap-free at 2k points)
// and every coefficient is below 2^13 (P-1)^2 < 2^75, inside the three primes'
// product, so the terms are the same.
// ---------------------------------------------------------------------------
constexpr int kNewtonCrtSmemWords = 2 * kNewtonPW + (1 << kNewtonMaxLog) + 4 * (1 << (kNewtonMaxLog - 1));
constexpr uint32_t kCrtHW = 1u << (kNewtonMaxLog - 1);

struct CrtCl {
  Ptab q[3];  // 167772161, 469762049, 754974721
  uint2 scale_r[3][kNewtonMaxLog + 1];
  GarnerC g;      // Garner constants with target P
  uint32_t P;     // the modulus, prime
  uint32_t pinv;  // P^-1 mod 2^32 (Montgomery products in the target field, P odd)
};

struct NewtonCrtD {
  const uint32_t* a;  // the series (canonical mod P, a[0] != 0), la terms
  uint32_t la;
  uint32_t* c;        // its inverse mod P: c[0, K) on return
  uint32_t K;         // <= 2^13
  CrtCl cc;
};
struct NewtonExpCrtD {
  const uint32_t* ap;   // a' (canonical), lap terms
  uint32_t lap;
  const uint32_t* tab;  // 1/i mod P in Montgomery form, i < K
  uint32_t* b;          // exp(a): b[0, K)
  uint32_t* c;          // 1/b: c[0, cs) on return (cs as the host computes it)
  uint32_t K;
  CrtCl cc;
};
struct NewtonSqrtCrtD {
  const uint32_t* u;  // the series with u[0] a nonzero square (canonical), ulen terms
  uint32_t ulen;
  uint32_t* b;        // sqrt(u): b[0, K)
  uint32_t* c;        // 1/b: c[0, cs) on return
  uint32_t K;
  uint32_t root, root_inv;
  CrtCl cc;
};

// X[0, N) <- src[0, len) mod the transform prime q, zero beyond.
__device__ __forceinline__ void crt_lift_load(uint32_t* X, const uint32_t* src, uint32_t len, uint32_t N,
                                              const Ptab& q, int tid, int nt) {
  for (uint32_t i = tid; i < N; i += nt) X[pad(i)] = i < len ? reduce_any(src[i], q.q1, q.f) : 0u;
}

// out[i] = (x y)[off + i] mod P for i < hl (negated, or times post[i] in
// Montgomery form, on request), x = x[0, xl), y = y[0, yl), at N = 2^logN
// points; out in every CTA's shared memory.  All of the cluster's CTAs call it
// with the same arguments.
__device__ __forceinline__ void crt_cl_window(const CrtCl& cc, const uint32_t* x, uint32_t xl, const uint32_t* y,
                                             uint32_t yl, uint32_t off, uint32_t hl, int logN, uint32_t* X,
                                             uint32_t* Y, uint32_t* R2, int& par, uint32_t* out, int negate,
                                             const uint32_t* post, int tid, int nt) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned qi = cl.block_rank();
  const Ptab q = cc.q[qi];
  uint32_t* R = R2 + par * kCrtHW;
  const uint32_t N = 1u << logN;
  crt_lift_load(X, x, xl, N, q, tid, nt);
  crt_lift_load(Y, y, yl, N, q, tid, nt);
  __syncthreads();
  cta_mul2(X, Y, logN, q, tid, nt);
  const uint2 sc = cc.scale_r[qi][logN];
  for (uint32_t i = tid; i < hl; i += nt) R[i] = red(shoup(X[pad(off + i)], sc, q.f.p), q.f.p);
  cl.sync();
  garner_body(cc.g, 3, cl.map_shared_rank(R, 0), cl.map_shared_rank(R, 1), cl.map_shared_rank(R, 2), out, hl, 0,
              post, negate, cc.pinv, 0, hl);
  __syncthreads();
  par ^= 1;
}

// One doubling step of the series inverse: Cs[k, want) from Cs[0, k) and the
// first aw terms of the series (H: scratch of want - k words).
__device__ __forceinline__ void crt_cl_inv_step(const CrtCl& cc, const uint32_t* series, uint32_t aw, uint32_t* Cs,
                                               uint32_t k, uint32_t want, uint32_t* X, uint32_t* Y, uint32_t* H,
                                               uint32_t* R2, int& par, int tid, int nt) {
  const uint32_t hl = want - k;
  const int logN = 32 - __clz(2 * k - 1);
  crt_cl_window(cc, series, aw, Cs, k, k, hl, logN, X, Y, R2, par, H, 1, nullptr, tid, nt);  // -(a c)[k, want)
  crt_cl_window(cc, H, hl, Cs, k, 0, hl, logN, X, Y, R2, par, Cs + k, 0, nullptr, tid, nt);  // (h c) mod x^hl
}

__device__ __forceinline__ void newton_inv_crt_body(const NewtonCrtD& d) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ uint32_t smn[];
  uint32_t* X = smn;
  uint32_t* Y = smn + kNewtonPW;
  uint32_t* Cs = smn + 2 * kNewtonPW;       // c[0, K)
  uint32_t* H = Cs + (1 << kNewtonMaxLog);  // h, < 2^12 terms
  uint32_t* R2 = H + kCrtHW;                // two residue buffers
  const int tid = threadIdx.x, nt = blockDim.x;
  const bool lead = cl.block_rank() == 0;
  if (tid == 0) {  // c[0] = a[0]^(P-2) mod P
    const uint64_t P = d.cc.P;
    uint64_t r = 1 % P, b = __ldg(d.a) % P;
    for (uint32_t e = d.cc.P - 2; e; e >>= 1) {
      if (e & 1u) r = r * b % P;
      b = b * b % P;
    }
    Cs[0] = (uint32_t)r;
    if (lead) d.c[0] = (uint32_t)r;
  }
  __syncthreads();
  int par = 0;
  for (uint32_t k = 1; k < d.K; k <<= 1) {
    const uint32_t want = min(2 * k, d.K);
    crt_cl_inv_step(d.cc, d.a, min(d.la, want), Cs, k, want, X, Y, H, R2, par, tid, nt);
    if (lead)
      for (uint32_t i = k + tid; i < want; i += nt) d.c[i] = Cs[i];
  }
  cl.sync();  // no CTA leaves while another may still read its residues
}

__device__ __forceinline__ void newton_exp_crt_body(const NewtonExpCrtD& d) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ uint32_t smn[];
  uint32_t* X = smn;
  uint32_t* Y = smn + kNewtonPW;
  uint32_t* B = smn + 2 * kNewtonPW;        // b[0, K)
  uint32_t* Cs = B + (1 << kNewtonMaxLog);  // c, < 2^12 terms
  uint32_t* T = Cs + kCrtHW;
  uint32_t* R2 = T + kCrtHW;
  const int tid = threadIdx.x, nt = blockDim.x;
  const bool lead = cl.block_rank() == 0;
  if (tid == 0) {
    B[0] = 1u;
    Cs[0] = 1u;
    if (lead) d.b[0] = 1u;
  }
  __syncthreads();
  int par = 0;
  uint32_t m = 1, cs = 1;
  while (m < d.K) {
    const uint32_t m2 = min(2 * m, d.K), hl = m2 - m;
    while (cs < hl) {
      const uint32_t want = min(2 * cs, hl);
      crt_cl_inv_step(d.cc, B, min(m, want), Cs, cs, want, X, Y, T, R2, par, tid, nt);
      cs = want;
    }
    const int logN = 32 - __clz(2 * m - 1);
    // t1 = (a' b)[m-1, m-1+hl); t2 = (t1 c) mod x^hl times 1/(m+i); b[m + i] = (t2 b)[i]
    crt_cl_window(d.cc, d.ap, min(d.lap, m2 - 1), B, m, m - 1, hl, logN, X, Y, R2, par, T, 0, nullptr, tid, nt);
    crt_cl_window(d.cc, T, hl, Cs, cs, 0, hl, logN, X, Y, R2, par, T, 0, d.tab + m, tid, nt);
    crt_cl_window(d.cc, T, hl, B, m, 0, hl, logN, X, Y, R2, par, B + m, 0, nullptr, tid, nt);
    if (lead)
      for (uint32_t i = tid; i < hl; i += nt) d.b[m + i] = B[m + i];
    m = m2;
  }
  if (lead)
    for (uint32_t i = tid; i < cs; i += nt) d.c[i] = Cs[i];
  cl.sync();
}

__global__ void __launch_bounds__(kNewtonThreads) k_newton_inv_crt(NewtonCrtD d) {
  pdl_enter();
  newton_inv_crt_body(d);
}

__global__ void __launch_bounds__(kNewtonThreads) k_newton_exp_crt(NewtonExpCrtD d) {
  pdl_enter();
  newton_exp_crt_body(d);
}

// Many small CRT Newton inverses and exponentials (batches): one cluster of
// three CTAs per job, the job's descriptor read from global memory.
struct NewtonCrtJobB {
  int kind;  // 0 inverse, 1 exponential
  NewtonCrtD inv;
  NewtonExpCrtD exp;
};
__global__ void __launch_bounds__(kNewtonThreads) k_newton_crt_b(const NewtonCrtJobB* __restrict__ jobs) {
  pdl_enter();
  const NewtonCrtJobB& j = jobs[blockIdx.x / 3];
  if (j.kind == 0) newton_inv_crt_body(j.inv);
  else newton_exp_crt_body(j.exp);
}

__global__ void __launch_bounds__(kNewtonThreads) k_newton_sqrt_crt(NewtonSqrtCrtD d) {
  pdl_enter();
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ uint32_t smn[];
  uint32_t* X = smn;
  uint32_t* Y = smn + kNewtonPW;
  uint32_t* B = smn + 2 * kNewtonPW;        // b[0, K)
  uint32_t* Cs = B + (1 << kNewtonMaxLog);  // c, < 2^12 terms
  uint32_t* T = Cs + kCrtHW;
  uint32_t* R2 = T + kCrtHW;
  const int tid = threadIdx.x, nt = blockDim.x;
  const bool lead = cl.block_rank() == 0;
  const uint32_t P = d.cc.P;
  if (tid == 0) {
    B[0] = d.root;
    Cs[0] = d.root_inv;
    if (lead) d.b[0] = d.root;
  }
  __syncthreads();
  int par = 0;
  uint32_t m = 1, cs = 1;
  while (m < d.K) {
    const uint32_t m2 = min(2 * m, d.K), hl = m2 - m;
    while (cs < hl) {
      const uint32_t want = min(2 * cs, hl);
      crt_cl_inv_step(d.cc, B, min(m, want), Cs, cs, want, X, Y, T, R2, par, tid, nt);
      cs = want;
    }
    const int logN = 32 - __clz(2 * m - 1);
    // t = u[m + i] - (b^2)[m + i];  b[m + i] = (t c)[i] / 2
    crt_cl_window(d.cc, B, m, B, m, m, hl, logN, X, Y, R2, par, T, 0, nullptr, tid, nt);
    for (uint32_t i = tid; i < hl; i += nt) {
      const uint32_t v = T[i];
      const uint32_t su = m + i < d.ulen ? d.u[m + i] : 0u;
      T[i] = su >= v ? su - v : su + P - v;
    }
    __syncthreads();
    crt_cl_window(d.cc, T, hl, Cs, cs, 0, hl, logN, X, Y, R2, par, B + m, 0, nullptr, tid, nt);
    for (uint32_t i = tid; i < hl; i += nt) {
      const uint32_t v = B[m + i];
      const uint32_t h = (v & 1u) ? (uint32_t)(((uint64_t)v + P) >> 1) : v >> 1;  // v / 2 mod P (P odd)
      B[m + i] = h;
      if (lead) d.b[m + i] = h;
    }
    __syncthreads();
    m = m2;
  }
  if (lead)
    for (uint32_t i = tid; i < cs; i += nt) d.c[i] = Cs[i];
  cl.sync();
}

}  // namespace

namespace fpx {

int small_kernel_max_log() { return kSmallLog; }

cudaError_t kernels_fast_init();
cudaError_t kernels_batch_init();
cudaError_t launch_rows_generic(const PrimeTables& pt, const BigTables& bt, uint32_t* x, const uint32_t* y, int ymode,
                                uint32_t* y_spec_out, int forward, int inverse, cudaStream_t s);

// Opt-in shared-memory limits; per device, called once per context.
cudaError_t kernels_init() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* fn, int bytes) {
    const cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (r != cudaSuccess) e = r;
  };
  set((const void*)k_small, 2 * padded_words(1 << kSmallLog) * 4);
  set((const void*)k_rows, 2 * padded_words(1 << 13) * 4);
  set((const void*)k_newton_inv, kNewtonSmemWords * 4);
  set((const void*)k_newton_exp, kNewtonExpSmemWords * 4);
  set((const void*)k_newton_b, kNewtonExpSmemWords * 4);
  set((const void*)k_newton_sqrt, kNewtonSqrtSmemWords * 4);
  set((const void*)k_newton_inv_crt, kNewtonCrtSmemWords * 4);
  set((const void*)k_newton_exp_crt, kNewtonCrtSmemWords * 4);
  set((const void*)k_newton_sqrt_crt, kNewtonCrtSmemWords * 4);
  set((const void*)k_newton_crt_b, kNewtonCrtSmemWords * 4);
  const cudaError_t r = kernels_fast_init();
  const cudaError_t r2 = kernels_batch_init();
  const cudaError_t r3 = kernels_cyc_init();
  return e != cudaSuccess ? e : (r != cudaSuccess ? r : (r2 != cudaSuccess ? r2 : r3));
}

cudaError_t launch_small(const PrimeTables& pt, int logN, const SmallJob& job, cudaStream_t s) {
  SmallD d;
  d.x = dev_in(job.x);
  d.y = dev_in(job.y);
  d.forward = job.forward;
  d.ymode = job.ymode;
  d.inverse = job.inverse;
  d.yspec = job.yspec;
  d.yspec_out = job.yspec_out;
  d.spec_x = job.spec_x;
  d.epi = dev_epi(job.epi);
  const int N = 1 << logN;
  int nt = N / 16;
  if (nt < 32) nt = 32;
  if (nt > 512) nt = 512;
  const size_t smem = (size_t)2 * padded_words(N) * 4;
  (void)pdl_launch(k_small, 1, nt, smem, s, d, dev_tab(pt), logN);
  return cudaGetLastError();
}

cudaError_t launch_rows_generic(const PrimeTables& pt, const BigTables& bt, uint32_t* x, const uint32_t* y, int ymode,
                                uint32_t* y_spec_out, int forward, int inverse, cudaStream_t s) {
  const int C = 1 << bt.logC;
  const size_t smem = (size_t)2 * padded_words(C) * 4;
  const int nt = C / 16 > 512 ? 512 : C / 16;
  (void)pdl_launch(k_rows, 1u << bt.logR, nt, smem, s, x, y, ymode, y_spec_out, forward, inverse, bt.logC, dev_tab(pt));
  return cudaGetLastError();
}


cudaError_t launch_pointwise(uint32_t p, uint32_t* a, const uint32_t* b, size_t n, cudaStream_t s) {
  (void)pdl_launch(k_pointwise, grid_for(n, 256), 256, 0, s, make_fp(p), a, b, n);
  return cudaGetLastError();
}

namespace {
__global__ void k_add_into(uint32_t p, uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t v = dst[i] + __ldg(src + i);
    dst[i] = v >= p ? v - p : v;
  }
}
}  // namespace

cudaError_t launch_add_into(uint32_t p, uint32_t* dst, const uint32_t* src, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  (void)pdl_launch(k_add_into, grid_for(n, 256), 256, 0, s, p, dst, src, n);
  return cudaGetLastError();
}

cudaError_t launch_spec_mac(uint32_t p, const uint32_t* const* x, const uint32_t* const* y, int npairs, uint32_t* acc,
                            size_t n, int accumulate, cudaStream_t s) {
  if (n % 4 || npairs < 1) return cudaErrorInvalidValue;
  for (int t0 = 0; t0 < npairs; t0 += kMacPairs) {
    MacPairs pr{};
    pr.n = std::min(kMacPairs, npairs - t0);
    for (int t = 0; t < pr.n; ++t) {
      pr.x[t] = reinterpret_cast<const uint4*>(x[t0 + t]);
      pr.y[t] = reinterpret_cast<const uint4*>(y[t0 + t]);
    }
    (void)pdl_launch(k_spec_mac, grid_for(n / 4, 256), 256, 0, s, make_fp(p), pr, reinterpret_cast<uint4*>(acc), n / 4,
                     (accumulate || t0) ? 1 : 0);
  }
  return cudaGetLastError();
}

cudaError_t launch_garner(uint32_t target, int primes, const uint32_t* c1, const uint32_t* c2, const uint32_t* c3,
                          uint32_t* out, size_t n, int accumulate, cudaStream_t s) {
  const uint64_t P1 = 167772161u, P2 = 469762049u, P3 = 754974721u;
  auto powm = [](uint64_t a, uint64_t e, uint64_t m) {
    uint64_t r = 1 % m;
    a %= m;
    for (; e; e >>= 1, a = a * a % m)
      if (e & 1) r = r * a % m;
    return r;
  };
  GarnerC g;
  g.P1 = (uint32_t)P1; g.P2 = (uint32_t)P2; g.P3 = (uint32_t)P3;
  g.inv12 = shoup_const((uint32_t)powm(P1 % P2, P2 - 2, P2), (uint32_t)P2);
  g.p1_in3 = shoup_const((uint32_t)(P1 % P3), (uint32_t)P3);
  g.inv123 = shoup_const((uint32_t)powm((P1 * P2) % P3, P3 - 2, P3), (uint32_t)P3);
  g.t = target;
  g.t_q1 = (uint32_t)((((uint64_t)1) << 32) / target);
  g.p1_t = shoup_const((uint32_t)(P1 % target), target);
  g.p12_t = shoup_const((uint32_t)((P1 * P2) % target), target);
  const uintptr_t al = reinterpret_cast<uintptr_t>(c1) | reinterpret_cast<uintptr_t>(primes >= 2 ? c2 : c1) |
                       reinterpret_cast<uintptr_t>(primes == 3 ? c3 : c1);
  if (al & 15u)
    (void)pdl_launch(k_garner, grid_for(n, 256), 256, 0, s, g, primes, c1, c2, c3, out, n, accumulate);
  else
    (void)pdl_launch(k_garner4, grid_for((n + 3) / 4, 256), 256, 0, s, g, primes, c1, c2, c3, out, n, accumulate);
  return cudaGetLastError();
}

cudaError_t launch_from_mont(uint32_t p, const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (p == 2) (void)pdl_launch(k_bits2, grid_for(n, 256), 256, 0, s, in, out, n);
  else (void)pdl_launch(k_from_mont, grid_for(n, 256), 256, 0, s, make_fp(p), in, out, n);
  return cudaGetLastError();
}

cudaError_t launch_to_mont(uint32_t p, const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (p == 2) (void)pdl_launch(k_bits2, grid_for(n, 256), 256, 0, s, in, out, n);
  else (void)pdl_launch(k_scale, grid_for(n, 256), 256, 0, s, p, in, out, n, shoup_const((uint32_t)((((uint64_t)1) << 32) % p), p));
  return cudaGetLastError();
}

cudaError_t launch_scale(uint32_t p, const uint32_t* a, uint32_t* out, size_t n, uint32_t c, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  (void)pdl_launch(k_scale, grid_for(n, 256), 256, 0, s, p, a, out, n, shoup_const(c % p, p));
  return cudaGetLastError();
}

cudaError_t launch_inv_table(uint32_t p, uint32_t* tab, size_t n, cudaStream_t s) {
  const uint32_t r = (uint32_t)((((uint64_t)1) << 32) % p);
  const uint32_t r2 = (uint32_t)((uint64_t)r * r % p);
  (void)pdl_launch(k_inv_table, grid_for(n + 1, 256), 256, 0, s, make_fp(p), shoup_const(r, p), shoup_const(r2, p), tab, n);
  return cudaGetLastError();
}

cudaError_t launch_derivative(uint32_t p, const uint32_t* a, uint32_t* r, size_t cnt, cudaStream_t s) {
  if (cnt <= 1) return cudaSuccess;
  const uint32_t rr = (uint32_t)((((uint64_t)1) << 32) % p);
  const uint32_t q1 = (uint32_t)((((uint64_t)1) << 32) / p);
  (void)pdl_launch(k_derivative, grid_for(cnt - 1, 256), 256, 0, s, make_fp(p), q1, shoup_const(rr, p), a, r, cnt - 1);
  return cudaGetLastError();
}

cudaError_t launch_direct_product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t off,
                                  size_t cnt, uint32_t* out, int accumulate, cudaStream_t s) {
  if (cnt == 0) return cudaSuccess;
  const Fp f = (p & 1u) ? make_fp(p) : Fp{p, 2 * p, 1};
  const uint32_t r = (uint32_t)((((uint64_t)1) << 32) % p);
  (void)pdl_launch(k_direct, grid_for(cnt, 256), 256, 0, s, p, f, shoup_const(r, p), a, (int)la, b, lb, off, cnt, out, accumulate);
  return cudaGetLastError();
}

}  // namespace fpx

// ---------------------------------------------------------------------------
// Series helpers: seeds (O(32^2) recurrences), scans, reversal, subtraction.
// Generic 64-bit arithmetic: any prime 2 <= p < 2^31.
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ uint32_t mm64(uint32_t a, uint32_t b, uint32_t p) { return (uint32_t)((uint64_t)a * b % p); }
__device__ uint32_t pow64(uint32_t a, uint64_t e, uint32_t p) {
  uint32_t r = 1 % p, b = a % p;
  for (; e; e >>= 1) {
    if (e & 1) r = mm64(r, b, p);
    b = mm64(b, b, p);
  }
  return r;
}
__device__ __forceinline__ uint32_t inv64(uint32_t a, uint32_t p) { return p == 2 ? a : pow64(a, p - 2, p); }


// kind 0: inverse seed   c[i] = -(sum_{j=1..i, j<la} a[j] c[i-j]) * c[0], c[0] = 1/a[0]
// kind 1: exp seed       b[i] = (sum_{j=1..min(i,la)} a[j-1] b[i-j]) / i,   b[0] = 1   (a = a')
// kind 2: sqrt seed      b[i] = (u[i] - sum_{j=1..i-1} b[j] b[i-j]) * w,     b[0] = r0, w = 1/(2 r0)
// One warp; n <= 64.  Writes out[0..n).  The operands (in Montgomery form for
// odd p) and, for exp, the inverses 1/i are staged in shared memory by all
// lanes first; each step is then lane-parallel Montgomery products and a
// 32-bit modular warp sum.
__device__ __forceinline__ void seed_body(int kind, uint32_t p, const uint32_t* a, size_t la, uint32_t* out, int n,
                                          uint32_t r0) {
  __shared__ uint32_t c[64], cm[64], am[64], iv[64];
  const int lane = threadIdx.x;
  const bool odd = (p & 1u) != 0;
  const Fp f{p, 2 * p, odd ? inv_mod_2_32(p) : 1u};
  const uint32_t R = (uint32_t)((((uint64_t)1) << 32) % p);
  for (int i = lane; i < 64; i += 32) {
    const uint32_t v = (size_t)i < la && i < n ? a[i] % p : 0u;
    am[i] = odd ? mm64(v, R, p) : v;
    iv[i] = (kind == 1 && i > 0 && i < n) ? inv64((uint32_t)i % p, p) : 0u;
  }
  uint32_t w = 0;
  if (lane == 0) {
    if (kind == 0) c[0] = inv64(a[0] % p, p);
    else if (kind == 1) c[0] = 1 % p;
    else { c[0] = r0; w = inv64(mm64(2 % p, r0, p), p); }
    cm[0] = odd ? mm64(c[0], R, p) : c[0];
  }
  w = __shfl_sync(0xffffffffu, w, 0);
  __syncwarp();
  for (int i = 1; i < n; ++i) {
    uint32_t part = 0;
    for (int j = 1 + lane; j <= i; j += 32) {
      uint32_t t = 0;
      if (kind == 0) t = (size_t)j < la ? (odd ? red(mont(am[j], c[i - j], f), p) : mm64(am[j], c[i - j], p)) : 0u;
      else if (kind == 1) t = (size_t)j <= la ? (odd ? red(mont(am[j - 1], c[i - j], f), p) : mm64(am[j - 1], c[i - j], p)) : 0u;
      else t = j < i ? (odd ? red(mont(cm[j], c[i - j], f), p) : mm64(c[j], c[i - j], p)) : 0u;
      part = red(part + t, p);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) part = red(part + __shfl_xor_sync(0xffffffffu, part, o), p);
    if (lane == 0) {
      const uint32_t sm_ = part;
      uint32_t v;
      if (kind == 0) v = mm64(sm_ ? p - sm_ : 0u, c[0], p);
      else if (kind == 1) v = mm64(sm_, iv[i], p);
      else {
        const uint32_t u = (size_t)i < la ? a[i] % p : 0u;
        v = mm64(u >= sm_ ? u - sm_ : u + p - sm_, w, p);
      }
      c[i] = v;
      cm[i] = odd ? mm64(v, R, p) : v;
    }
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) out[i] = c[i];
}

__global__ void k_seed(int kind, uint32_t p, const uint32_t* a, size_t la, uint32_t* out, int n, uint32_t r0) {
  pdl_enter();
  seed_body(kind, p, a, la, out, n, r0);
}

// exp / log preparation (exponential.hpp:85-139): out = out0 + 0x + ..., ap = a'
// (first cnt coefficients of a); blockIdx.y = job.
struct ExpPrepB {
  Fp f;
  uint32_t q1;
  uint2 r_sh;
  const uint32_t* a;
  size_t cnt;  // min(la, n)
  uint32_t* ap;
  uint32_t* out;
  size_t n;
  uint32_t out0;
};
__global__ void k_exp_prep_b(const ExpPrepB* __restrict__ jobs) {
  pdl_enter();
  const ExpPrepB& j = jobs[blockIdx.y];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < j.n; i += (size_t)gridDim.x * blockDim.x) {
    j.out[i] = i == 0 ? j.out0 : 0u;
    if (i + 1 < j.cnt) {
      const uint32_t k = reduce_any((uint32_t)(i + 1), j.q1, j.f);
      j.ap[i] = red(shoup(red(mont(j.a[i + 1], k, j.f), j.f.p), j.r_sh, j.f.p), j.f.p);
    }
  }
}

// First (mode 0) or last (mode 1) index in [0, n) with a[i] != 0; n if none.
// Each thread keeps its own first / last hit, the block reduces them, and one
// atomic per block updates *res (dense inputs would otherwise serialise on a
// single address).  Mode 1 reports 0 both for "index 0" and "none"; the caller
// tells them apart.
__global__ void __launch_bounds__(256) k_find_nonzero(const uint32_t* a, size_t n, int mode, unsigned long long* res) {
  pdl_enter();
  unsigned long long hit = 0;  // index + 1, 0 = none
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    if (a[i]) {
      hit = i + 1;
      if (mode == 0) break;  // a thread's indices only grow
    }
  }
  __shared__ unsigned long long red_sm[8];
  unsigned long long v = hit ? hit - 1 : (mode == 0 ? ~0ull : 0ull);
  for (int o = 16; o; o >>= 1) {
    const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
    v = mode == 0 ? (u < v ? u : v) : (u > v ? u : v);
  }
  if ((threadIdx.x & 31) == 0) red_sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      v = mode == 0 ? (red_sm[w] < v ? red_sm[w] : v) : (red_sm[w] > v ? red_sm[w] : v);
    if (mode == 0 && v != ~0ull) atomicMin(res, v);
    if (mode == 1 && v != 0) atomicMax(res, v);
  }
}

__global__ void k_reverse(const uint32_t* a, uint32_t* r, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    r[i] = a[n - 1 - i];
}

// r[i] = a[i] - b[i] (mod p), b missing beyond lb.
__global__ void k_sub(uint32_t p, const uint32_t* a, const uint32_t* b, size_t lb, uint32_t* r, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = a[i], y = i < lb ? b[i] : 0u;
    r[i] = x >= y ? x - y : x + (p - y);
  }
}

// Characteristic two square root (square_root.hpp:14-23): out[i/2] = a[i] for even i.
__global__ void k_sqrt_char2(const uint32_t* a, size_t cnt, uint32_t* out, unsigned long long* odd_flag) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t v = a[i] & 1u;
    if (i & 1) { if (v) atomicMax(odd_flag, 1ull); }
    else out[i / 2] = v;
  }
}

// Elementwise Montgomery-table product: out[i] = a[i] * tab[i] (tab in Montgomery form).
__global__ void k_mul_mont_tab(Fp f, const uint32_t* a, const uint32_t* tab, uint32_t* out, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = red(mont(a[i], tab[i], f), f.p);
}

}  // namespace

namespace fpx {

cudaError_t launch_seed(int kind, uint32_t p, const uint32_t* a, size_t la, uint32_t* out, int n, uint32_t r0,
                        cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  (void)pdl_launch(k_seed, 1, 32, 0, s, kind, p, a, la, out, n, r0);
  return cudaGetLastError();
}

int newton_inv_max_log() { return kNewtonMaxLog; }

cudaError_t launch_newton_inv(const PrimeTables& pt, const uint32_t* a, size_t la, uint32_t* c, size_t k0, size_t K,
                              cudaStream_t s) {
  // the last step k -> K transforms 2^ceil(log2 K) points
  if (K > (size_t(1) << kNewtonMaxLog) || (k0 & (k0 - 1)) || k0 > K || (size_t(1) << pt.small_log) < K ||
      !(pt.p & 1u) || pt.p >= (1u << 30))
    return cudaErrorInvalidValue;
  if (K == k0) return cudaSuccess;
  NewtonInvD d;
  d.r1 = (uint32_t)((uint64_t(1) << 32) % pt.p);
  d.r2 = (uint32_t)((uint64_t)d.r1 * d.r1 % pt.p);
  d.a = a;
  d.la = (uint32_t)std::min<size_t>(la, K);
  d.c = c;
  d.k0 = (uint32_t)k0;
  d.K = (uint32_t)K;
  for (int l = 0; l <= kNewtonMaxLog; ++l) d.scale_r[l] = shoup_const(l <= pt.small_log ? pt.inv_pow2_r[l] : 0u, pt.p);
  (void)pdl_launch(k_newton_inv, 1, kNewtonThreads, (size_t)kNewtonSmemWords * 4, s, d, dev_tab(pt));
  return cudaGetLastError();
}

cudaError_t launch_newton_exp(const PrimeTables& pt, const uint32_t* ap, size_t lap, const uint32_t* tab, uint32_t* b,
                              uint32_t* c, size_t K, cudaStream_t s) {
  if (K < 2 || K > (size_t(1) << kNewtonMaxLog) || (size_t(1) << pt.small_log) < K || !(pt.p & 1u) ||
      pt.p >= (1u << 30))
    return cudaErrorInvalidValue;
  NewtonExpD d;
  d.ap = ap;
  d.lap = (uint32_t)std::min<size_t>(lap, K);
  d.tab = tab;
  d.b = b;
  d.c = c;
  d.K = (uint32_t)K;
  for (int l = 0; l <= kNewtonMaxLog; ++l) d.scale_r[l] = shoup_const(l <= pt.small_log ? pt.inv_pow2_r[l] : 0u, pt.p);
  (void)pdl_launch(k_newton_exp, 1, kNewtonThreads, (size_t)kNewtonExpSmemWords * 4, s, d, dev_tab(pt));
  return cudaGetLastError();
}

namespace {
void fill_newton_inv(NewtonInvD& d, const PrimeTables& pt, const uint32_t* a, size_t la, uint32_t* c, size_t K) {
  d.a = a;
  d.la = (uint32_t)std::min<size_t>(la, K);
  d.c = c;
  d.k0 = 0;
  d.K = (uint32_t)K;
  d.r1 = (uint32_t)((uint64_t(1) << 32) % pt.p);
  d.r2 = (uint32_t)((uint64_t)d.r1 * d.r1 % pt.p);
  for (int l = 0; l <= kNewtonMaxLog; ++l) d.scale_r[l] = shoup_const(l <= pt.small_log ? pt.inv_pow2_r[l] : 0u, pt.p);
}
void fill_newton_exp(NewtonExpD& d, const PrimeTables& pt, const uint32_t* ap, size_t lap, const uint32_t* tab,
                     uint32_t* b, uint32_t* c, size_t K) {
  d.ap = ap;
  d.lap = (uint32_t)std::min<size_t>(lap, K);
  d.tab = tab;
  d.b = b;
  d.c = c;
  d.K = (uint32_t)K;
  for (int l = 0; l <= kNewtonMaxLog; ++l) d.scale_r[l] = shoup_const(l <= pt.small_log ? pt.inv_pow2_r[l] : 0u, pt.p);
}
}  // namespace

size_t batch_newton_bytes(size_t jobs) {
  return jobs * std::max(sizeof(NewtonJobB), sizeof(NewtonCrtJobB)) + 512;
}

// The CRT jobs of a batch (defined with the cluster launchers below).
cudaError_t fill_newton_crt_batch(const std::vector<const NewtonJob*>& jobs, void* host);
cudaError_t launch_newton_crt_b(const void* dev, size_t count, cudaStream_t s);

cudaError_t launch_newton_batch(const std::vector<NewtonJob>& jobs, void* host_staging, void* dev_desc,
                                cudaStream_t s, cudaEvent_t staged) {
  if (jobs.empty()) return cudaSuccess;
  std::vector<const NewtonJob*> crt;
  for (const NewtonJob& x : jobs)
    if (x.aux) crt.push_back(&x);
  std::vector<NewtonJobB> v(jobs.size() - crt.size());
  for (size_t i = 0, vi = 0; i < jobs.size(); ++i) {
    const NewtonJob& x = jobs[i];
    if (x.aux) continue;
    const PrimeTables& pt = *x.pt;
    if (x.K < 1 || x.K > (size_t(1) << kNewtonMaxLog) || (size_t(1) << pt.small_log) < x.K || !(pt.p & 1u) ||
        pt.p >= (1u << 30) || (x.kind == 1 && x.K < 2))
      return cudaErrorInvalidValue;
    NewtonJobB& j = v[vi++];
    std::memset(&j, 0, sizeof j);
    j.kind = x.kind;
    j.pt = dev_tab(pt);
    if (x.kind == 0) fill_newton_inv(j.inv, pt, x.a, x.la, x.out, x.K);
    else fill_newton_exp(j.exp, pt, x.a, x.la, x.tab, x.out, x.c, x.K);
  }
  // descriptors: the one-CTA jobs, then (256-byte aligned) the cluster jobs
  const size_t off = (v.size() * sizeof(NewtonJobB) + 255) & ~size_t(255);
  std::memcpy(host_staging, v.data(), v.size() * sizeof(NewtonJobB));
  cudaError_t e = cudaSuccess;
  if (!crt.empty() && (e = fill_newton_crt_batch(crt, static_cast<char*>(host_staging) + off)) != cudaSuccess)
    return e;
  const size_t bytes = crt.empty() ? v.size() * sizeof(NewtonJobB) : off + crt.size() * sizeof(NewtonCrtJobB);
  e = cudaMemcpyAsync(dev_desc, host_staging, bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  if (staged && (e = cudaEventRecord(staged, s)) != cudaSuccess) return e;
  if (!v.empty())
    (void)pdl_launch(k_newton_b, (unsigned)v.size(), kNewtonThreads, (size_t)kNewtonExpSmemWords * 4, s,
                     static_cast<const NewtonJobB*>(dev_desc));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (!crt.empty()) return launch_newton_crt_b(static_cast<const char*>(dev_desc) + off, crt.size(), s);
  return cudaSuccess;
}

cudaError_t launch_newton_sqrt(const PrimeTables& pt, const uint32_t* u, size_t ulen, uint32_t root, uint32_t root_inv,
                               uint32_t* b, uint32_t* c, size_t K, cudaStream_t s) {
  if (K < 1 || K > (size_t(1) << kNewtonMaxLog) || (size_t(1) << pt.small_log) < K || !(pt.p & 1u) ||
      pt.p >= (1u << 30))
    return cudaErrorInvalidValue;
  NewtonSqrtD d;
  d.u = u;
  d.ulen = (uint32_t)std::min<size_t>(ulen, K);
  d.b = b;
  d.c = c;
  d.K = (uint32_t)K;
  d.root = root;
  d.root_inv = root_inv;
  for (int l = 0; l <= kNewtonMaxLog; ++l) d.scale_r[l] = shoup_const(l <= pt.small_log ? pt.inv_pow2_r[l] : 0u, pt.p);
  (void)pdl_launch(k_newton_sqrt, 1, kNewtonThreads, (size_t)kNewtonSqrtSmemWords * 4, s, d, dev_tab(pt));
  return cudaGetLastError();
}

cudaError_t launch_find_nonzero(const uint32_t* a, size_t n, int mode, unsigned long long* res, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  (void)pdl_launch(k_find_nonzero, grid_for(n, 256), 256, 0, s, a, n, mode, res);
  return cudaGetLastError();
}

cudaError_t launch_reverse(const uint32_t* a, uint32_t* r, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  (void)pdl_launch(k_reverse, grid_for(n, 256), 256, 0, s, a, r, n);
  return cudaGetLastError();
}

cudaError_t launch_sub(uint32_t p, const uint32_t* a, const uint32_t* b, size_t lb, uint32_t* r, size_t n,
                       cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  (void)pdl_launch(k_sub, grid_for(n, 256), 256, 0, s, p, a, b, lb, r, n);
  return cudaGetLastError();
}

cudaError_t launch_sqrt_char2(const uint32_t* a, size_t cnt, uint32_t* out, unsigned long long* odd_flag,
                              cudaStream_t s) {
  if (cnt == 0) return cudaSuccess;
  (void)pdl_launch(k_sqrt_char2, grid_for(cnt, 256), 256, 0, s, a, cnt, out, odd_flag);
  return cudaGetLastError();
}

cudaError_t launch_mul_mont_tab(uint32_t p, const uint32_t* a, const uint32_t* tab, uint32_t* out, size_t n,
                                cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  (void)pdl_launch(k_mul_mont_tab, grid_for(n, 256), 256, 0, s, make_fp(p), a, tab, out, n);
  return cudaGetLastError();
}

}  // namespace fpx

// ===========================================================================
// Specialised two-pass kernels (ntt_fast.cuh): the row pass for C = 2^12 and
// the column passes for every R = 2^2 .. 2^12.
// ===========================================================================
#include "ntt_fast.cuh"

namespace {

// Row pass, C = 4096.  Modes as k_rows: forward (DIF of x, and of y when
// ymode == 1), pointwise product (ymode 1 raw y, 2 y spectrum, 3 square),
// inverse (DIT).  The forward's last group, the product and the inverse's first
// group all act on the same 16 positions per thread, in registers.
__device__ __forceinline__ void lds16(const uint32_t* p, uint32_t (&v)[16]) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint4 u = q[k];
    v[4 * k] = u.x; v[4 * k + 1] = u.y; v[4 * k + 2] = u.z; v[4 * k + 3] = u.w;
  }
}
__device__ __forceinline__ void sts16(uint32_t* p, const uint32_t (&v)[16]) {
  uint4* q = reinterpret_cast<uint4*>(p);
#pragma unroll
  for (int k = 0; k < 4; ++k) q[k] = make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

__device__ __forceinline__ void rows12_body(uint32_t* __restrict__ x, const uint32_t* __restrict__ y, int ymode,
                                            uint32_t* __restrict__ y_spec_out, int forward, int inverse,
                                            const Ptab& pt, unsigned row_index) {
  __shared__ __align__(16) uint32_t sX[kRowWords];
  __shared__ __align__(16) uint32_t sY[kRowWords];
  const int t = threadIdx.x;
  const int bA = baseA(t), bB = baseB(t), bC = baseC(t);
  const size_t row = (size_t)row_index << 12;
  const Fp f = pt.f;
  uint32_t v[2][16];
  if (forward) {
    if (ymode == 1) {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        v[0][i] = x[row + posA(t, i)];
        v[1][i] = __ldg(y + row + posA(t, i));
      }
      bf_group<4, 12, false, 2>(v, pt.fwd, t, f);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        sX[bA + offA(i)] = v[0][i];
        sY[bA + offA(i)] = v[1][i];
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        v[0][i] = sX[bB + offB(i)];
        v[1][i] = sY[bB + offB(i)];
      }
      bf_group<4, 8, false, 2>(v, pt.fwd, t & 15, f);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        sX[bB + offB(i)] = v[0][i];
        sY[bB + offB(i)] = v[1][i];
      }
      __syncthreads();
      lds16(sX + bC, v[0]);
      lds16(sY + bC, v[1]);
      bf_group<4, 4, false, 2, true>(v, pt.fwd, 0, f);
      if (y_spec_out) {
        uint4* o = reinterpret_cast<uint4*>(y_spec_out + row + posC(t, 0));
#pragma unroll
        for (int q = 0; q < 4; ++q)
          o[q] = make_uint4(red(v[1][4 * q], f.p), red(v[1][4 * q + 1], f.p), red(v[1][4 * q + 2], f.p),
                            red(v[1][4 * q + 3], f.p));
      }
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) v[0][i] = x[row + posA(t, i)];
      bf_group<4, 12, false, 1>(v, pt.fwd, t, f);
#pragma unroll
      for (int i = 0; i < 16; ++i) sX[bA + offA(i)] = v[0][i];
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 16; ++i) v[0][i] = sX[bB + offB(i)];
      bf_group<4, 8, false, 1>(v, pt.fwd, t & 15, f);
#pragma unroll
      for (int i = 0; i < 16; ++i) sX[bB + offB(i)] = v[0][i];
      __syncthreads();
      lds16(sX + bC, v[0]);
      bf_group<4, 4, false, 1, true>(v, pt.fwd, 0, f);
    }
  } else {
    const uint4* in = reinterpret_cast<const uint4*>(x + row + posC(t, 0));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 u = in[q];
      v[0][4 * q] = u.x; v[0][4 * q + 1] = u.y; v[0][4 * q + 2] = u.z; v[0][4 * q + 3] = u.w;
    }
  }
  if (ymode == 1) {
#pragma unroll
    for (int i = 0; i < 16; ++i) v[0][i] = mont(v[0][i], v[1][i], f);
  } else if (ymode == 2) {
    const uint4* ys = reinterpret_cast<const uint4*>(y + row + posC(t, 0));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 u = __ldg(ys + q);
      v[0][4 * q] = mont(v[0][4 * q], u.x, f);
      v[0][4 * q + 1] = mont(v[0][4 * q + 1], u.y, f);
      v[0][4 * q + 2] = mont(v[0][4 * q + 2], u.z, f);
      v[0][4 * q + 3] = mont(v[0][4 * q + 3], u.w, f);
    }
  } else if (ymode == 3) {
#pragma unroll
    for (int i = 0; i < 16; ++i) v[0][i] = mont(v[0][i], v[0][i], f);
  }
  if (!inverse) {
    uint4* o = reinterpret_cast<uint4*>(x + row + posC(t, 0));
#pragma unroll
    for (int q = 0; q < 4; ++q)
      o[q] = make_uint4(red(v[0][4 * q], f.p), red(v[0][4 * q + 1], f.p), red(v[0][4 * q + 2], f.p),
                        red(v[0][4 * q + 3], f.p));
    return;
  }
  bf_group<4, 4, true, 1, true>(v, pt.inv, 0, f);
  sts16(sX + bC, v[0]);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 16; ++i) v[0][i] = sX[bB + offB(i)];
  bf_group<4, 8, true, 1>(v, pt.inv, t & 15, f);
#pragma unroll
  for (int i = 0; i < 16; ++i) sX[bB + offB(i)] = v[0][i];
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 16; ++i) v[0][i] = sX[bA + offA(i)];
  bf_group<4, 12, true, 1>(v, pt.inv, t, f);
#pragma unroll
  for (int i = 0; i < 16; ++i) x[row + posA(t, i)] = v[0][i];
}

__global__ void __launch_bounds__(256, 3) k_rows12(uint32_t* __restrict__ x, const uint32_t* __restrict__ y,
                                                  int ymode, uint32_t* __restrict__ y_spec_out, int forward,
                                                  int inverse, Ptab pt) {
  pdl_enter();
  rows12_body(x, y, ymode, y_spec_out, forward, inverse, pt, blockIdx.x);
}

// Default tile width: 2^LOGW columns with R * W = 2^13 words (32 KiB) up to
// R = 2^10 and 2^14 words (64 KiB) above, so that three CTAs fit on an SM.
__host__ __device__ constexpr int col_logw(int logr) { return logr >= 11 ? 14 - logr : 13 - logr; }

// Threads of a column-pass CTA and the resident CTAs per SM it is compiled for
// (80 registers a thread; shared memory also allows three 64 KB tiles).  512
// threads in two CTAs (64 registers) measured 5-9 % slower from 2^21 points up.
constexpr int kColNT = 256;
constexpr int kColMinBlocks = 3;

template <int LOGR, int LW = col_logw(LOGR)>
struct ColCfg {
  static constexpr int LOGW = LW;
  static constexpr int W = 1 << LOGW;
  static constexpr int TE = 1 << (LOGR + LOGW);
  static constexpr int K = ColGroups<LOGR>::K;
  static constexpr int GL = ColGroups<LOGR>::size(K - 1);
  using P = ColSwz<LOGR, LOGW, GL>;
  static constexpr int SMEM_WORDS = TE;
};

// Loads the W x R column tile (rows t, columns j0..j0+W) into shared memory
// with cp.async: all copies in flight at once, no register staging, zero
// beyond `count`.  16-byte copies when the source is 16-byte aligned.
template <int LOGR, int LOGW, bool HALF = false>
__device__ __forceinline__ void col_tile_load(uint32_t* sm, const uint32_t* src, uint32_t count, int j0, int logC,
                                              int tid) {
  // HALF: only rows t < R/2 (the rest are known zeros, never read as such)
  using C = ColCfg<LOGR, LOGW>;
  constexpr int TL = HALF ? C::TE / 2 : C::TE;
  if (src == nullptr || count == 0) {
    for (int e = tid; e < C::SMEM_WORDS; e += kColNT) sm[e] = 0u;
    return;
  }
  if (C::W >= 4 && ((uintptr_t)src & 15u) == 0) {
    constexpr int CPR = C::W >= 4 ? C::W / 4 : 1;  // 16-byte chunks per row segment
#pragma unroll 4
    for (int q = tid; q < TL / 4; q += kColNT) {
      const int t = q / CPR, cc = (q % CPR) * 4;
      const uint32_t gi = ((uint32_t)t << logC) + j0 + cc;
      const int valid = gi < count ? (int)min(4u, count - gi) : 0;
      cp_async16(sm + C::P::at((t << C::LOGW) + cc), src + (valid ? gi : 0), valid * 4);
    }
  } else {
#pragma unroll 4
    for (int e = tid; e < TL; e += kColNT) {
      const int t = e >> C::LOGW, c = e & (C::W - 1);
      const uint32_t gi = ((uint32_t)t << logC) + j0 + c;
      const bool v = gi < count;
      cp_async4(sm + C::P::at(e), src + (v ? gi : 0), v ? 4 : 0);
    }
  }
  cp_async_wait_all();
}

// Every thread works on two adjacent columns c, c+1 (c even) of the tile: the
// pair shares its twiddles, its swizzled addresses and its loop, and moves
// through shared memory as one 64-bit access (the swizzle never touches the
// low LOGW bits, so pairs stay adjacent and 8-byte aligned).
__device__ __forceinline__ void lds_pair(const uint32_t* p, uint32_t& a, uint32_t& b) {
  const uint2 v = *reinterpret_cast<const uint2*>(p);
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void sts_pair(uint32_t* p, uint32_t a, uint32_t b) {
  *reinterpret_cast<uint2*>(p) = make_uint2(a, b);
}

// One group over the tile, shared -> registers -> shared.  REDUCE: inputs may be
// any 32-bit value (CRT lift), reduce them on the way in (first forward group).
template <int LOGR, int LOGW, int KG, bool INV, bool REDUCE, bool ZH = false>
__device__ __forceinline__ void col_group_smem(uint32_t* sm, const uint2* tw, const Fp& f, uint32_t q1, int tid) {
  using C = ColCfg<LOGR, LOGW>;
  constexpr int G = ColGroups<LOGR>::size(KG);
  constexpr int T = ColGroups<LOGR>::top(KG);
  constexpr int S = T - G;
  constexpr int LP = C::LOGW - 1;  // column pairs per row: 2^LP
  constexpr int NINST = C::TE >> (G + 1);
#pragma unroll 1
  for (int inst = tid; inst < NINST; inst += kColNT) {
    const int c = (inst & ((1 << LP) - 1)) << 1;
    const int rest = inst >> LP;
    const int base = rest & ((1 << S) - 1);
    const int p0 = ((rest >> S) << T) + base;
    using A = typename C::P::template Group<S + C::LOGW, G>;
    int ab[A::P];
    A::bases((p0 << C::LOGW) + c, ab);
    uint32_t v[2][1 << G];
#pragma unroll
    for (int i = 0; i < (ZH ? (1 << G) / 2 : (1 << G)); ++i) {
      uint32_t x0, x1;
      lds_pair(sm + A::addr(ab, i), x0, x1);
      v[0][i] = REDUCE ? reduce_any(x0, q1, f) : x0;
      v[1][i] = REDUCE ? reduce_any(x1, q1, f) : x1;
    }
    bf_group<G, T, INV, 2, false, ZH>(v, tw, base, f);
#pragma unroll
    for (int i = 0; i < (1 << G); ++i) sts_pair(sm + A::addr(ab, i), v[0][i], v[1][i]);
  }
}

// Forward groups 0 .. K-2 (the last group is the caller's).
template <int LOGR, int LOGW, int KG, bool ZH = false>
__device__ __forceinline__ void col_fwd_groups(uint32_t* sm, const Ptab& pt, bool reduce, int tid) {
  if constexpr (KG < ColGroups<LOGR>::K - 1) {
    constexpr bool Z = ZH && KG == 0;
    if (KG == 0 && reduce) col_group_smem<LOGR, LOGW, KG, false, true, Z>(sm, pt.fwd, pt.f, pt.q1, tid);
    else col_group_smem<LOGR, LOGW, KG, false, false, Z>(sm, pt.fwd, pt.f, pt.q1, tid);
    __syncthreads();
    col_fwd_groups<LOGR, LOGW, KG + 1>(sm, pt, reduce, tid);
  }
}

// Inverse groups K-2 .. 1 (the first, smallest group and the last, group 0, are the caller's).
template <int LOGR, int LOGW, int KG>
__device__ __forceinline__ void col_inv_groups(uint32_t* sm, const Ptab& pt, int tid) {
  if constexpr (KG >= 1) {
    col_group_smem<LOGR, LOGW, KG, true, false>(sm, pt.inv, pt.f, pt.q1, tid);
    __syncthreads();
    col_inv_groups<LOGR, LOGW, KG - 1>(sm, pt, tid);
  }
}

// Bailey twiddle w_N^{j * bitrev_R(t)} of column j, row t = 2^G b + i (i < 2^G):
// exponent eb + js * bitrev_G(i).
struct BaileyCol {
  uint32_t eb, js;
  __device__ __forceinline__ BaileyCol(uint32_t j, int b, int logr, int g)
      : eb(j * brev_c(b, logr - g)), js(j << (logr - g)) {}
  __device__ __forceinline__ uint32_t apply(uint32_t x, int i, int g, const BigD& bt, const Fp& f) const {
    return bailey_mul(x, eb + js * brev_c(i, g), bt, f);
  }
};

// Factored form of the same twiddle: w_N^eb (the block's part, the same for
// all 2^G rows of the block) once per block in Montgomery form, times the
// column factor U_j^bitrev_G(i) from the table.  A point then costs one Shoup
// product by the factor and one Montgomery product by the block's part, both
// lazy in [0, 2p) (the Montgomery product needs a*b < p 2^32: 2p * 2p is, for
// p < 2^30), instead of three Shoup products and three table loads.
static_assert(ColGroups<5>::size(ColGroups<5>::K - 1) == 5 / ((5 + 3) / 4), "col_last_group_log");
static_assert(ColGroups<9>::size(ColGroups<9>::K - 1) == 9 / ((9 + 3) / 4), "col_last_group_log");
static_assert(ColGroups<11>::size(ColGroups<11>::K - 1) == 11 / ((11 + 3) / 4), "col_last_group_log");
static_assert(ColGroups<12>::size(ColGroups<12>::K - 1) == 12 / ((12 + 3) / 4), "col_last_group_log");
__device__ __forceinline__ uint32_t col_block_factor(uint32_t j, int b, int logr, int g, const BigD& bt,
                                                     const Fp& f) {
  return shoup(bailey_mul(1u, j * brev_c(b, logr - g), bt, f), bt.r32, f.p);
}

template <int LOGR, int LOGW>
__device__ __forceinline__ void colfwd_body(const InD& in, uint32_t* __restrict__ out, const BigD& bt, const Ptab& pt,
                                            int j0) {
  using C = ColCfg<LOGR, LOGW>;
  constexpr int K = ColGroups<LOGR>::K;
  constexpr int G = C::GL;
  constexpr int LP = C::LOGW - 1;
  extern __shared__ uint32_t sm[];
  const int tid = threadIdx.x, logC = bt.logC;
  const Fp f = pt.f;
  // zero-padded input (count <= N/2, every conv operand): the lower half of
  // each column is never loaded and the first level needs no additions
  const bool half = K > 1 && in.ptr != nullptr && in.count != 0 && in.count <= (1u << (LOGR - 1 + logC));
  if (half) {
    col_tile_load<LOGR, LOGW, true>(sm, in.ptr, in.count, j0, logC, tid);
    __syncthreads();
    col_fwd_groups<LOGR, LOGW, 0, true>(sm, pt, in.reduce != 0, tid);
  } else {
    col_tile_load<LOGR, LOGW>(sm, in.ptr, in.count, j0, logC, tid);
    __syncthreads();
    col_fwd_groups<LOGR, LOGW, 0>(sm, pt, in.reduce != 0, tid);
  }
  // last group: shared -> registers -> Bailey twiddle -> global (64-bit stores)
  constexpr int NINST = C::TE >> (G + 1);
  const bool reduce_here = K == 1 && in.reduce;
#pragma unroll 1
  for (int inst = tid; inst < NINST; inst += kColNT) {
    const int c = (inst & ((1 << LP) - 1)) << 1;
    const int b = inst >> LP;
    const int p0 = b << G;
    const uint32_t j = j0 + c;
    const bool fact = LOGR >= 9 && bt.cf != nullptr;
    uint32_t a0 = 0, a1 = 0;
    if (fact) {  // the block's factors first: their table loads overlap the butterflies
      a0 = col_block_factor(j, b, LOGR, G, bt, f);
      a1 = col_block_factor(j + 1, b, LOGR, G, bt, f);
    }
    using A = typename C::P::template Group<C::LOGW, G>;
    int ab[A::P];
    A::bases((p0 << C::LOGW) + c, ab);
    uint32_t v[2][1 << G];
#pragma unroll
    for (int i = 0; i < (1 << G); ++i) {
      uint32_t x0, x1;
      lds_pair(sm + A::addr(ab, i), x0, x1);
      v[0][i] = reduce_here ? reduce_any(x0, pt.q1, f) : x0;
      v[1][i] = reduce_here ? reduce_any(x1, pt.q1, f) : x1;
    }
    bf_group<G, G, false, 2, true>(v, pt.fwd, 0, f);
    if (fact) {
      const uint4* tp = bt.cf + ((size_t)(j >> 1) << G);
#pragma unroll
      for (int i = 0; i < (1 << G); ++i) {
        const uint4 t = __ldg(tp + i);
        *reinterpret_cast<uint2*>(out + ((size_t)(p0 + i) << logC) + j) =
            make_uint2(mont(shoup(v[0][i], t.x, t.y, f.p), a0, f), mont(shoup(v[1][i], t.z, t.w, f.p), a1, f));
      }
    } else {
      const BaileyCol w0(j, b, LOGR, G), w1(j + 1, b, LOGR, G);
#pragma unroll
      for (int i = 0; i < (1 << G); ++i)
        *reinterpret_cast<uint2*>(out + ((size_t)(p0 + i) << logC) + j) =
            make_uint2(w0.apply(v[0][i], i, G, bt, f), w1.apply(v[1][i], i, G, bt, f));
    }
  }
}

// Tiles of a column pass.  The first `nbig` tiles of every operand are 2^LW1
// columns wide, the remaining `nsmall` are 2^LW2 wide; blocks run through the
// wide tiles of all operands first (operand-major), then the narrow ones.  With
// the wide tiles filling whole waves of resident CTAs, the grid ends on narrow
// tiles instead of a partial wave of wide ones (148 SMs never divide a power of
// two).  LW1 == LW2: every tile is wide (nsmall = 0).
struct ColSplit {
  int nbig, nsmall, nops;
};
__device__ __forceinline__ bool col_tile_of(const ColSplit& sp, int lw1, int lw2, int& op, int& j0) {
  int b = (int)blockIdx.x;
  const int nb = sp.nbig * sp.nops;
  if (b < nb) {
    op = b / sp.nbig;
    j0 = (b - op * sp.nbig) << lw1;
    return true;
  }
  b -= nb;
  op = b / sp.nsmall;
  j0 = (sp.nbig << lw1) + ((b - op * sp.nsmall) << lw2);
  return false;
}

template <int LOGR, int LW1, int LW2>
__global__ void __launch_bounds__(kColNT, kColMinBlocks) k_colfwd_t(ColOps ops, BigD bt, Ptab pt, ColSplit sp) {
  pdl_enter();
  int op, j0;
  const bool wide = col_tile_of(sp, LW1, LW2, op, j0);
  const InD in = op == 0 ? ops.in[0] : (op == 1 ? ops.in[1] : ops.in[2]);
  uint32_t* out = op == 0 ? ops.out[0] : (op == 1 ? ops.out[1] : ops.out[2]);
  if constexpr (LW1 == LW2) {
    colfwd_body<LOGR, LW1>(in, out, bt, pt, j0);
  } else {
    if (wide) colfwd_body<LOGR, LW1>(in, out, bt, pt, j0);
    else colfwd_body<LOGR, LW2>(in, out, bt, pt, j0);
  }
}

template <int LOGR, int LOGW, bool PLAIN>
__device__ __forceinline__ void colinv_body(const uint32_t* __restrict__ in, const BigD& bt, const Ptab& pt,
                                            const EpiD& epi, int j0) {
  using C = ColCfg<LOGR, LOGW>;
  constexpr int K = ColGroups<LOGR>::K;
  constexpr int LP = C::LOGW - 1;
  extern __shared__ uint32_t sm[];
  const int tid = threadIdx.x, logC = bt.logC;
  const Fp f = pt.f;
  col_tile_load<LOGR, LOGW>(sm, in, 0xffffffffu, j0, logC, tid);
  __syncthreads();
  // first: the smallest blocks (Bailey twiddle on the way in), in place
  {
    constexpr int G = C::GL;
    constexpr int NINST = C::TE >> (G + 1);
#pragma unroll 1
    for (int inst = tid; inst < NINST; inst += kColNT) {
      const int c = (inst & ((1 << LP) - 1)) << 1;
      const int b = inst >> LP;
      const int p0 = b << G;
      const uint32_t j = j0 + c;
      using A = typename C::P::template Group<C::LOGW, G>;
      int ab[A::P];
      A::bases((p0 << C::LOGW) + c, ab);
      uint32_t v[2][1 << G];
      // Factored twiddle: the column factors on the way in, the block's factor
      // (the same for the block's 2^G rows) after the block's butterflies, which
      // are linear, so that its table loads overlap them.  Made canonical: it
      // multiplies DIT outputs in [0, 4p), and 4p * p < p 2^32.
      const bool fact = LOGR >= 9 && bt.cf != nullptr;
      uint32_t a0 = 0, a1 = 0;
      if (fact) {
        a0 = red(col_block_factor(j, b, LOGR, G, bt, f), f.p);
        a1 = red(col_block_factor(j + 1, b, LOGR, G, bt, f), f.p);
        const uint4* tp = bt.cf + ((size_t)(j >> 1) << G);
#pragma unroll
        for (int i = 0; i < (1 << G); ++i) {
          uint32_t x0, x1;
          lds_pair(sm + A::addr(ab, i), x0, x1);
          const uint4 t = __ldg(tp + i);
          v[0][i] = shoup(x0, t.x, t.y, f.p);
          v[1][i] = shoup(x1, t.z, t.w, f.p);
        }
      } else {
        const BaileyCol w0(j, b, LOGR, G), w1(j + 1, b, LOGR, G);
#pragma unroll
        for (int i = 0; i < (1 << G); ++i) {
          uint32_t x0, x1;
          lds_pair(sm + A::addr(ab, i), x0, x1);
          v[0][i] = w0.apply(x0, i, G, bt, f);
          v[1][i] = w1.apply(x1, i, G, bt, f);
        }
      }
      bf_group<G, G, true, 2, true>(v, pt.inv, 0, f);
      if (fact) {
#pragma unroll
        for (int i = 0; i < (1 << G); ++i) {
          v[0][i] = mont(v[0][i], a0, f);
          v[1][i] = mont(v[1][i], a1, f);
        }
      }
      if constexpr (K == 1) {
#pragma unroll
        for (int i = 0; i < (1 << G); ++i)
          epi_store_pair<PLAIN>(epi, (uint32_t)(((p0 + i) << logC) + j), v[0][i], v[1][i], f);
      } else {
#pragma unroll
        for (int i = 0; i < (1 << G); ++i) sts_pair(sm + A::addr(ab, i), v[0][i], v[1][i]);
      }
    }
  }
  if constexpr (K > 1) {
    __syncthreads();
    col_inv_groups<LOGR, LOGW, K - 2>(sm, pt, tid);
    // last: the full column blocks, shared -> registers -> epilogue (global)
    constexpr int G = ColGroups<LOGR>::size(0);
    constexpr int S = LOGR - G;
    constexpr int NINST = C::TE >> (G + 1);
#pragma unroll 1
    for (int inst = tid; inst < NINST; inst += kColNT) {
      const int c = (inst & ((1 << LP) - 1)) << 1;
      const int base = inst >> LP;
      using A = typename C::P::template Group<S + C::LOGW, G>;
      int ab[A::P];
      A::bases((base << C::LOGW) + c, ab);
      uint32_t v[2][1 << G];
#pragma unroll
      for (int i = 0; i < (1 << G); ++i) lds_pair(sm + A::addr(ab, i), v[0][i], v[1][i]);
      bf_group<G, LOGR, true, 2>(v, pt.inv, base, f);
#pragma unroll
      for (int i = 0; i < (1 << G); ++i)
        epi_store_pair<PLAIN>(epi, (uint32_t)(((base + (i << S)) << logC) + j0 + c), v[0][i], v[1][i], f);
    }
  }
}

template <int LOGR, bool PLAIN, int LW1, int LW2>
__global__ void __launch_bounds__(kColNT, kColMinBlocks) k_colinv_t(const uint32_t* __restrict__ in, BigD bt, Ptab pt, EpiD epi,
                                                     ColSplit sp) {
  pdl_enter();
  int op, j0;
  const bool wide = col_tile_of(sp, LW1, LW2, op, j0);
  if constexpr (LW1 == LW2) {
    colinv_body<LOGR, LW1, PLAIN>(in, bt, pt, epi, j0);
  } else {
    if (wide) colinv_body<LOGR, LW1, PLAIN>(in, bt, pt, epi, j0);
    else colinv_body<LOGR, LW2, PLAIN>(in, bt, pt, epi, j0);
  }
}

using ColFwdFn = void (*)(ColOps, BigD, Ptab, ColSplit);
using ColInvFn = void (*)(const uint32_t*, BigD, Ptab, EpiD, ColSplit);

// One compiled column-pass shape: R = 2^LOGR points per column, wide tiles of
// 2^LW1 columns, narrow tiles of 2^LW2 (LW1 == LW2: a single width).
template <int LOGR, int LW1, int LW2>
struct ColK {};

template <class... K>
struct ColTable;
template <int... R, int... A, int... B>
struct ColTable<ColK<R, A, B>...> {
  static ColFwdFn fwd(int logR, int lw1, int lw2) {
    ColFwdFn r = nullptr;
    ((logR == R && lw1 == A && lw2 == B ? (r = k_colfwd_t<R, A, B>, 0) : 0), ...);
    return r;
  }
  static ColInvFn inv(int logR, int lw1, int lw2, bool plain) {
    ColInvFn r = nullptr;
    ((logR == R && lw1 == A && lw2 == B ? (r = plain ? k_colinv_t<R, true, A, B> : k_colinv_t<R, false, A, B>, 0)
                                        : 0),
     ...);
    return r;
  }
  static cudaError_t init() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* fn, int bytes) {
      const cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      if (r != cudaSuccess) e = r;
    };
    (set((const void*)k_colfwd_t<R, A, B>, ColCfg<R, A>::SMEM_WORDS * 4), ...);
    (set((const void*)k_colinv_t<R, true, A, B>, ColCfg<R, A>::SMEM_WORDS * 4), ...);
    (set((const void*)k_colinv_t<R, false, A, B>, ColCfg<R, A>::SMEM_WORDS * 4), ...);
    return e;
  }
};
template <int L>
using ColD = ColK<L, col_logw(L), col_logw(L)>;
// Default widths for every R, and narrower tiles the tuner chooses from: for
// R <= 2^8 (transforms of at most 2^20 points, grids below one wave) tiles of
// 1/2, 1/4 and 1/8 the default width, more CTAs with less work each; for
// R = 2^9 .. 2^12 (2^21 .. 2^24 points, grids of several waves) half-width
// tiles and the split grids.  Narrow tiles keep 2^LW >= 4 columns below
// R = 2^12: at two columns the swizzle leaves 4-way bank conflicts there.
template <int L, int K>
using ColN = ColK<L, col_logw(L) - K, col_logw(L) - K>;
using Cols = ColTable<ColD<2>, ColN<2, 1>, ColN<2, 2>, ColN<2, 3>, ColD<3>, ColN<3, 1>, ColN<3, 2>, ColN<3, 3>,
                      ColD<4>, ColN<4, 1>, ColN<4, 2>, ColN<4, 3>, ColD<5>, ColN<5, 1>, ColN<5, 2>, ColN<5, 3>,
                      ColD<6>, ColN<6, 1>, ColN<6, 2>, ColN<6, 3>, ColD<7>, ColN<7, 1>, ColN<7, 2>, ColN<7, 3>,
                      ColD<8>, ColN<8, 1>, ColN<8, 2>, ColN<8, 3>,
                      ColD<9>, ColK<9, 3, 3>, ColK<9, 4, 3>, ColK<9, 4, 2>,
                      ColD<10>, ColK<10, 2, 2>, ColK<10, 3, 2>,
                      ColD<11>, ColK<11, 2, 2>, ColK<11, 3, 2>,
                      ColD<12>, ColK<12, 1, 1>, ColK<12, 2, 1>>;

}  // namespace

namespace fpx {

cudaError_t kernels_fast_init() { return Cols::init(); }

int col_shape_candidates(int logR, bool inverse, ColShape* out, int max) {
  const int d = col_logw(logR);
  int n = 0;
  auto add = [&](int lw1, int lw2) {
    if (n >= max) return;
    ColShape sh;
    sh.lw1 = lw1;
    sh.lw2 = lw2;
    sh.split = lw2 != lw1;
    if (sh.split) {
      const void* fn = inverse ? (const void*)Cols::inv(logR, lw1, lw2, true) : (const void*)Cols::fwd(logR, lw1, lw2);
      int dev = 0, sms = 0, per_sm = 0;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kColNT, (size_t(4) << (logR + lw1))) !=
              cudaSuccess) {
        cudaGetLastError();
        return;
      }
      sh.slots = sms * per_sm;
    }
    out[n++] = sh;
  };
  add(d, d);
  for (int a = d; a >= 1; --a)
    for (int b = a; b >= 1; --b)
      if ((a != d || b != d) && Cols::fwd(logR, a, b)) add(a, b);
  return n;
}

namespace {
// Tiles per operand of one column pass with shape `sh` (see ColSplit).
ColSplit col_split(const BigTables& bt, const ColShape& sh, int nops, int& lw1, int& lw2) {
  lw1 = sh.lw1 ? sh.lw1 : col_logw(bt.logR);
  lw2 = sh.lw1 && sh.split ? sh.lw2 : lw1;
  const int tiles = 1 << (bt.logC - lw1);
  ColSplit sp{tiles, 0, nops};
  if (lw2 < lw1 && sh.slots > 0) {
    const int nbig = (nops * tiles / sh.slots) * sh.slots / nops;  // whole waves of wide tiles
    if (nbig > 0 && nbig < tiles) {
      sp.nbig = nbig;
      sp.nsmall = (tiles - nbig) << (lw1 - lw2);
    }
  }
  return sp;
}

// Bailey tables of one column pass.  The inverse pass scales by 1/N, or by
// 2^32/N after a Montgomery pointwise product (mont_scaled), on its lo table.
BigD big_d(const BigTables& bt, int lw, bool inverse, bool mont_scaled, uint32_t p) {
  const uint32_t r = (uint32_t)((uint64_t(1) << 32) % p);
  const uint2 r32 = make_uint2(r, (uint32_t)(((uint64_t)r << 32) / p));
  if (!inverse)
    return BigD{bt.logR, bt.logC, lw, reinterpret_cast<const uint2*>(bt.lo_fwd),
                reinterpret_cast<const uint2*>(bt.mid_fwd), reinterpret_cast<const uint2*>(bt.hi_fwd),
                reinterpret_cast<const uint4*>(bt.cf_fwd), r32};
  return BigD{bt.logR, bt.logC, lw, reinterpret_cast<const uint2*>(mont_scaled ? bt.lo_inv_r : bt.lo_inv),
              reinterpret_cast<const uint2*>(bt.mid_inv), reinterpret_cast<const uint2*>(bt.hi_inv),
              reinterpret_cast<const uint4*>(bt.cf_inv), r32};
}
}  // namespace

cudaError_t launch_colfwd(const PrimeTables& pt, const BigTables& bt, int nops, const InOp* in,
                               uint32_t* const* out, cudaStream_t s) {
  ColOps ops{};
  for (int i = 0; i < nops; ++i) {
    ops.in[i] = dev_in(in[i]);
    ops.out[i] = out[i];
  }
  const ColShape sh = bt.shapes ? (nops == 1 ? bt.shapes->fwd1 : bt.shapes->fwd2) : ColShape{};
  int lw1, lw2;
  const ColSplit sp = col_split(bt, sh, nops, lw1, lw2);
  ColFwdFn fn = Cols::fwd(bt.logR, lw1, lw2);
  if (!fn || lw1 > bt.logC || nops < 1 || nops > 3) return cudaErrorInvalidValue;
  const BigD d = big_d(bt, lw1, false, false, pt.p);
  (void)pdl_launch(fn, (unsigned)(nops * (sp.nbig + sp.nsmall)), kColNT, size_t(4) << (bt.logR + lw1), s, ops, d, dev_tab(pt), sp);
  return cudaGetLastError();
}

cudaError_t launch_colinv(const PrimeTables& pt, const BigTables& bt, const uint32_t* in, int mont_scaled,
                               const Epi& epi, cudaStream_t s) {
  const ColShape sh = bt.shapes ? bt.shapes->inv : ColShape{};
  int lw1, lw2;
  const ColSplit sp = col_split(bt, sh, 1, lw1, lw2);
  ColInvFn fn = Cols::inv(bt.logR, lw1, lw2, host_epi_plain(epi));
  if (!fn || lw1 > bt.logC) return cudaErrorInvalidValue;
  const BigD d = big_d(bt, lw1, true, mont_scaled != 0, pt.p);
  (void)pdl_launch(fn, (unsigned)(sp.nbig + sp.nsmall), kColNT, size_t(4) << (bt.logR + lw1), s, in, d, dev_tab(pt), dev_epi(epi),
                                                                                 sp);
  return cudaGetLastError();
}

cudaError_t launch_rows(const PrimeTables& pt, const BigTables& bt, uint32_t* x, const uint32_t* y, int ymode,
                             uint32_t* y_spec_out, int forward, int inverse, cudaStream_t s) {
  if (bt.logC != 12) return launch_rows_generic(pt, bt, x, y, ymode, y_spec_out, forward, inverse, s);
  (void)pdl_launch(k_rows12, 1u << bt.logR, 256, 0, s, x, y, ymode, y_spec_out, forward, inverse, dev_tab(pt));
  return cudaGetLastError();
}

}  // namespace fpx

// ===========================================================================
// Batched execution: many independent products per launch.  Each CTA reads its
// job's descriptor (prime tables, operands, scratch, epilogue) from device
// memory, so one launch covers any mix of primes and polynomials of the same
// transform size; different sizes go to different launches.
// ===========================================================================
namespace {

struct SmallJobB {
  SmallD d;
  Ptab pt;
};
struct BigJobB {
  Ptab pt;
  BigD bf, bi;
  InD in[2];
  uint32_t* t[2];
  int nops, ymode;
  const uint32_t* yspec;
  uint32_t* yspec_out;
  EpiD epi;
};
struct DirectJobB {
  uint32_t p;
  Fp f;
  const uint32_t* a;
  int la;
  const uint32_t* b;
  size_t lb, off, cnt;
  uint32_t* out;
  int accumulate;
  const uint32_t* post_mont;
  int negate;
};
struct GarnerJobB {
  GarnerC g;
  int primes;
  const uint32_t *c1, *c2, *c3;
  uint32_t* out;
  size_t n;
  int accumulate;
  const uint32_t* post_mont;
  int negate;
  uint32_t tpinv;
};


template <int LOGR>
__global__ void __launch_bounds__(kColNT, kColMinBlocks) k_colfwd_b(const BigJobB* __restrict__ jobs) {
  pdl_enter();
  const BigJobB& j = jobs[blockIdx.z];
  if ((int)blockIdx.y >= j.nops) return;
  colfwd_body<LOGR, col_logw(LOGR)>(j.in[blockIdx.y], j.t[blockIdx.y], j.bf, j.pt, blockIdx.x << col_logw(LOGR));
}

__global__ void __launch_bounds__(256, 3) k_rows12_b(const BigJobB* __restrict__ jobs) {
  pdl_enter();
  const BigJobB& j = jobs[blockIdx.y];
  rows12_body(j.t[0], j.ymode == 1 ? j.t[1] : j.yspec, j.ymode, j.yspec_out, 1, 1, j.pt, blockIdx.x);
}

template <int LOGR, bool PLAIN>
__global__ void __launch_bounds__(kColNT, kColMinBlocks) k_colinv_b(const BigJobB* __restrict__ jobs) {
  pdl_enter();
  const BigJobB& j = jobs[blockIdx.y];
  colinv_body<LOGR, col_logw(LOGR), PLAIN>(j.t[0], j.bi, j.pt, j.epi, blockIdx.x << col_logw(LOGR));
}

// Batched direct products and Garner reconstructions: block b covers outputs
// [map[b].first, map[b].first + kOutSpan) of job map[b].job, so blocks follow
// each job's own length rather than the longest job's.
constexpr size_t kOutSpan = 2048;
struct OutBlock {
  uint32_t job;
  uint32_t first;
};
__global__ void k_direct_b(const DirectJobB* __restrict__ jobs, const OutBlock* __restrict__ map) {
  pdl_enter();
  const OutBlock m = map[blockIdx.x];
  const DirectJobB& j = jobs[m.job];
  direct_body(j.p, j.f, j.a, j.la, j.b, j.lb, j.off, j.cnt, j.out, j.accumulate, j.post_mont, j.negate, m.first,
              kOutSpan);
}

// Newton seeds for many jobs (k_seed per block): blockIdx.x = job.
struct SeedJobB {
  int kind;
  uint32_t p;
  const uint32_t* a;
  size_t la;
  uint32_t* out;
  int n;
  uint32_t r0;
};
__global__ void k_seed_b(const SeedJobB* __restrict__ jobs) {
  pdl_enter();
  const SeedJobB& j = jobs[blockIdx.x];
  seed_body(j.kind, j.p, j.a, j.la, j.out, j.n, j.r0);
}

// Four consecutive outputs per thread: 16-byte residue loads and four
// independent Garner chains (the residue buffers are 16-byte aligned, and
// every block starts at a multiple of kOutSpan); stores stay 32-bit, the
// caller's output having any alignment.  Unaligned residues: one per thread.
__global__ void k_garner_b(const GarnerJobB* __restrict__ jobs, const OutBlock* __restrict__ map) {
  pdl_enter();
  const OutBlock m = map[blockIdx.x];
  const GarnerJobB& j = jobs[m.job];
  const uintptr_t al = reinterpret_cast<uintptr_t>(j.c1) | reinterpret_cast<uintptr_t>(j.c2) |
                       reinterpret_cast<uintptr_t>(j.c3);
  if (al & 15u) {
    garner_body(j.g, j.primes, j.c1, j.c2, j.c3, j.out, j.n, j.accumulate, j.post_mont, j.negate, j.tpinv, m.first,
                kOutSpan);
    return;
  }
  const size_t end = m.first + kOutSpan < j.n ? m.first + kOutSpan : j.n;
  for (size_t i = m.first + 4 * (size_t)threadIdx.x; i < end; i += 4 * (size_t)blockDim.x) {
    if (i + 4 <= end) {
      const uint4 a = *reinterpret_cast<const uint4*>(j.c1 + i);
      const uint4 b = j.primes >= 2 ? *reinterpret_cast<const uint4*>(j.c2 + i) : make_uint4(0u, 0u, 0u, 0u);
      const uint4 c = j.primes == 3 ? *reinterpret_cast<const uint4*>(j.c3 + i) : make_uint4(0u, 0u, 0u, 0u);
      const uint32_t v0 = garner_one(j.g, j.primes, a.x, b.x, c.x), v1 = garner_one(j.g, j.primes, a.y, b.y, c.y);
      const uint32_t v2 = garner_one(j.g, j.primes, a.z, b.z, c.z), v3 = garner_one(j.g, j.primes, a.w, b.w, c.w);
      garner_put(j.g, v0, j.out, i, j.accumulate, j.post_mont, j.negate, j.tpinv);
      garner_put(j.g, v1, j.out, i + 1, j.accumulate, j.post_mont, j.negate, j.tpinv);
      garner_put(j.g, v2, j.out, i + 2, j.accumulate, j.post_mont, j.negate, j.tpinv);
      garner_put(j.g, v3, j.out, i + 3, j.accumulate, j.post_mont, j.negate, j.tpinv);
    } else {
      for (size_t t = i; t < end; ++t)
        garner_put(j.g, garner_one(j.g, j.primes, j.c1[t], j.primes >= 2 ? j.c2[t] : 0u, j.primes == 3 ? j.c3[t] : 0u),
                   j.out, t, j.accumulate, j.post_mont, j.negate, j.tpinv);
    }
  }
}

using BatchFn = void (*)(const BigJobB*);

template <int... L>
struct ColBatch {
  static BatchFn fwd(int logR) {
    BatchFn r = nullptr;
    ((logR == L ? (r = k_colfwd_b<L>, 0) : 0), ...);
    return r;
  }
  static BatchFn inv(int logR, bool plain) {
    BatchFn r = nullptr;
    ((logR == L ? (r = plain ? k_colinv_b<L, true> : k_colinv_b<L, false>, 0) : 0), ...);
    return r;
  }
  static cudaError_t launch(int logR, dim3 grid, const BigJobB* jobs, int smem, cudaStream_t s) {
    BatchFn fn = fwd(logR);
    if (!fn) return cudaErrorInvalidValue;
    (void)pdl_launch(fn, grid, kColNT, smem, s, jobs);
    return cudaGetLastError();
  }
  static cudaError_t launch_inv(int logR, bool plain, dim3 grid, const BigJobB* jobs, int smem, cudaStream_t s) {
    BatchFn fn = inv(logR, plain);
    if (!fn) return cudaErrorInvalidValue;
    (void)pdl_launch(fn, grid, kColNT, smem, s, jobs);
    return cudaGetLastError();
  }
  static cudaError_t init() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* fn, int bytes) {
      const cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      if (r != cudaSuccess) e = r;
    };
    (set((const void*)k_colfwd_b<L>, ColCfg<L>::SMEM_WORDS * 4), ...);
    (set((const void*)k_colinv_b<L, true>, ColCfg<L>::SMEM_WORDS * 4), ...);
    (set((const void*)k_colinv_b<L, false>, ColCfg<L>::SMEM_WORDS * 4), ...);
    return e;
  }
};
using ColsB = ColBatch<2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12>;


GarnerC garner_consts(uint32_t target) {
  const uint64_t P1 = 167772161u, P2 = 469762049u, P3 = 754974721u;
  auto powm = [](uint64_t a, uint64_t e, uint64_t m) {
    uint64_t r = 1 % m;
    a %= m;
    for (; e; e >>= 1, a = a * a % m)
      if (e & 1) r = r * a % m;
    return r;
  };
  GarnerC g;
  g.P1 = (uint32_t)P1; g.P2 = (uint32_t)P2; g.P3 = (uint32_t)P3;
  g.inv12 = shoup_const((uint32_t)powm(P1 % P2, P2 - 2, P2), (uint32_t)P2);
  g.p1_in3 = shoup_const((uint32_t)(P1 % P3), (uint32_t)P3);
  g.inv123 = shoup_const((uint32_t)powm((P1 * P2) % P3, P3 - 2, P3), (uint32_t)P3);
  g.t = target;
  g.t_q1 = (uint32_t)((((uint64_t)1) << 32) / target);
  g.p1_t = shoup_const((uint32_t)(P1 % target), target);
  g.p12_t = shoup_const((uint32_t)((P1 * P2) % target), target);
  return g;
}

struct BatchGroup {
  int logN;
  bool big;
  size_t off;
  int count;
  bool plain;  // every job's epilogue is plain
};
inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

__global__ void __launch_bounds__(256) k_cyc4096_b(const SmallJobB* __restrict__ jobs);  // defined below
cudaError_t launch_cyc_small_batch(int logN, unsigned count, const SmallJobB* jobs, cudaStream_t s);  // below

}  // namespace

namespace fpx {

cudaError_t kernels_batch_init() { return ColsB::init(); }

static size_t out_blocks(size_t n) { return n ? (n + kOutSpan - 1) / kOutSpan : 0; }

size_t batch_descriptor_bytes(const BatchPlan& b) {
  size_t blocks = 0;
  for (const DirectJob& x : b.direct) blocks += out_blocks(x.cnt);
  for (const GarnerJob& x : b.garner) blocks += out_blocks(x.n);
  return b.xjobs.size() * std::max(sizeof(SmallJobB), sizeof(BigJobB)) + b.direct.size() * sizeof(DirectJobB) +
         b.garner.size() * sizeof(GarnerJobB) + blocks * sizeof(OutBlock) + 256 * 40;  // sections 256-byte aligned
}

cudaError_t launch_batch(const BatchPlan& b, void* host_staging, void* dev_desc, cudaStream_t s,
                         cudaEvent_t staged) {
  // Layout: [small jobs by logN][big jobs by logN][direct][garner], each section 256-byte aligned.
  std::vector<int> order;
  order.reserve(b.xjobs.size());
  for (int lg = 0; lg <= 31; ++lg)  // stable bucket order by transform size
    for (size_t i = 0; i < b.xjobs.size(); ++i)
      if (b.xjobs[i].logN == lg) order.push_back((int)i);
  char* h = static_cast<char*>(host_staging);
  char* d = static_cast<char*>(dev_desc);
  size_t off = 0;
  std::vector<BatchGroup> groups;
  for (size_t k = 0; k < order.size();) {
    const int logN = b.xjobs[order[k]].logN;
    size_t e = k;
    while (e < order.size() && b.xjobs[order[e]].logN == logN) ++e;
    const bool big = logN > kSmallLog;
    off = align256(off);
    BatchGroup grp;
    grp.logN = logN;
    grp.big = big;
    grp.off = off;
    grp.count = (int)(e - k);
    grp.plain = true;
    for (size_t q = k; q < e; ++q) grp.plain = grp.plain && host_epi_plain(b.xjobs[order[q]].epi);
    groups.push_back(grp);
    for (size_t q = k; q < e; ++q) {
      const XJob& x = b.xjobs[order[q]];
      const Ptab pt = dev_tab(*x.pt);
      if (!big) {
        SmallJobB j{};
        j.pt = pt;
        j.d.x = dev_in(x.x);
        j.d.y = dev_in(x.y);
        j.d.forward = 1;
        j.d.ymode = x.ymode;
        j.d.inverse = 1;
        j.d.yspec = x.yspec;
        j.d.yspec_out = x.yspec_out;
        j.d.spec_x = nullptr;
        j.d.epi = dev_epi(x.epi);
        std::memcpy(h + off, &j, sizeof j);
        off += sizeof j;
      } else {
        const BigTables& bt = *x.bt;
        BigJobB j{};
        j.pt = pt;
        j.bf = big_d(bt, col_logw(bt.logR), false, false, pt.f.p);
        j.bi = big_d(bt, col_logw(bt.logR), true, x.ymode != 0, pt.f.p);
        j.in[0] = dev_in(x.x);
        j.in[1] = dev_in(x.y);
        j.t[0] = x.t1;
        j.t[1] = x.t2;
        j.nops = x.ymode == 1 ? 2 : 1;
        j.ymode = x.ymode;
        j.yspec = x.yspec;
        j.yspec_out = x.yspec_out;
        j.epi = dev_epi(x.epi);
        std::memcpy(h + off, &j, sizeof j);
        off += sizeof j;
      }
    }
    k = e;
  }
  off = align256(off);
  const size_t off_direct = off;
  for (const DirectJob& x : b.direct) {
    DirectJobB j;
    j.p = x.p;
    if (x.p & 1u) {
      j.f = make_fp(x.p);
    } else {
      j.f.p = x.p;
      j.f.p2 = 2 * x.p;
      j.f.pinv = 1;
    }
    j.a = x.a;
    j.la = (int)x.la;
    j.b = x.b;
    j.lb = x.lb;
    j.off = x.off;
    j.cnt = x.cnt;
    j.out = x.out;
    j.accumulate = x.accumulate;
    j.post_mont = x.post_mont;
    j.negate = x.negate;
    std::memcpy(h + off, &j, sizeof j);
    off += sizeof j;
  }
  off = align256(off);
  const size_t off_garner = off;
  for (const GarnerJob& x : b.garner) {
    GarnerJobB j;
    j.g = garner_consts(x.target);
    j.primes = x.primes;
    j.c1 = x.c1;
    j.c2 = x.c2;
    j.c3 = x.c3;
    j.out = x.out;
    j.n = x.n;
    j.accumulate = x.accumulate;
    j.post_mont = x.post_mont;
    j.negate = x.negate;
    j.tpinv = 1u;
    if (x.target & 1u) j.tpinv = inv_mod_2_32(x.target);
    std::memcpy(h + off, &j, sizeof j);
    off += sizeof j;
  }
  // block maps of the direct and Garner launches
  off = align256(off);
  const size_t off_dmap = off;
  for (size_t q = 0; q < b.direct.size(); ++q)
    for (size_t f0 = 0; f0 < b.direct[q].cnt; f0 += kOutSpan) {
      const OutBlock m{(uint32_t)q, (uint32_t)f0};
      std::memcpy(h + off, &m, sizeof m);
      off += sizeof m;
    }
  const size_t n_dmap = (off - off_dmap) / sizeof(OutBlock);
  off = align256(off);
  const size_t off_gmap = off;
  for (size_t q = 0; q < b.garner.size(); ++q)
    for (size_t f0 = 0; f0 < b.garner[q].n; f0 += kOutSpan) {
      const OutBlock m{(uint32_t)q, (uint32_t)f0};
      std::memcpy(h + off, &m, sizeof m);
      off += sizeof m;
    }
  const size_t n_gmap = (off - off_gmap) / sizeof(OutBlock);
  if (off == 0) return cudaSuccess;
  cudaError_t e = cudaMemcpyAsync(d, h, off, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  if (staged && (e = cudaEventRecord(staged, s)) != cudaSuccess) return e;
  // grid.y / grid.z hold at most 65535 jobs per launch
  constexpr size_t kMaxY = 65535;
  // block maps are at most 2^31 blocks; grid.x takes them in chunks
  constexpr size_t kMaxX = size_t(1) << 30;
  for (size_t k = 0; k < n_dmap; k += kMaxX) {
    (void)pdl_launch(k_direct_b, (unsigned)std::min(kMaxX, n_dmap - k), 256, 0, s, 
        reinterpret_cast<const DirectJobB*>(d + off_direct), reinterpret_cast<const OutBlock*>(d + off_dmap) + k);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  for (const BatchGroup& g : groups) {
    if (!g.big && g.logN == 12) {
      (void)pdl_launch(k_cyc4096_b, g.count, 256, 0, s, reinterpret_cast<const SmallJobB*>(d + g.off));
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      continue;
    }
    if (!g.big) {
      e = launch_cyc_small_batch(g.logN, (unsigned)g.count, reinterpret_cast<const SmallJobB*>(d + g.off), s);
      if (e != cudaSuccess) return e;
      continue;
    }
    const int logC = 12, logR = g.logN - logC;
    const int logW = col_logw(logR);
    const int smem = 4 << (logR + logW);
    for (size_t k = 0; k < (size_t)g.count; k += kMaxY) {
      const BigJobB* jobs = reinterpret_cast<const BigJobB*>(d + g.off) + k;
      const unsigned cnt = (unsigned)std::min(kMaxY, (size_t)g.count - k);
      e = ColsB::launch(logR, dim3(1u << (logC - logW), 2, cnt), jobs, smem, s);
      if (e != cudaSuccess) return e;
      (void)pdl_launch(k_rows12_b, dim3(1u << logR, cnt), 256, 0, s, jobs);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      e = ColsB::launch_inv(logR, g.plain, dim3(1u << (logC - logW), cnt), jobs, smem, s);
      if (e != cudaSuccess) return e;
    }
  }
  for (size_t k = 0; k < n_gmap; k += kMaxX) {
    (void)pdl_launch(k_garner_b, (unsigned)std::min(kMaxX, n_gmap - k), 256, 0, s, 
        reinterpret_cast<const GarnerJobB*>(d + off_garner), reinterpret_cast<const OutBlock*>(d + off_gmap) + k);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace fpx

namespace fpx {

cudaError_t launch_seeds_batch(const std::vector<SeedJob>& jobs, void* host_staging, void* dev_desc, cudaStream_t s,
                               cudaEvent_t staged) {
  if (jobs.empty()) return cudaSuccess;
  std::vector<SeedJobB> v;
  v.reserve(jobs.size());
  for (const SeedJob& x : jobs) v.push_back(SeedJobB{x.kind, x.p, x.a, x.la, x.out, x.n, x.r0});
  std::memcpy(host_staging, v.data(), v.size() * sizeof(SeedJobB));
  cudaError_t e = cudaMemcpyAsync(dev_desc, host_staging, v.size() * sizeof(SeedJobB), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  if (staged && (e = cudaEventRecord(staged, s)) != cudaSuccess) return e;
  (void)pdl_launch(k_seed_b, (unsigned)v.size(), 32, 0, s, static_cast<const SeedJobB*>(dev_desc));
  return cudaGetLastError();
}

cudaError_t launch_exp_prep_batch(const std::vector<ExpPrep>& jobs, void* host_staging, void* dev_desc,
                                  cudaStream_t s, cudaEvent_t staged) {
  if (jobs.empty()) return cudaSuccess;
  std::vector<ExpPrepB> v;
  size_t maxn = 0;
  for (const ExpPrep& x : jobs) {
    const uint32_t r = (uint32_t)((((uint64_t)1) << 32) % x.p);
    v.push_back(ExpPrepB{make_fp(x.p), (uint32_t)((((uint64_t)1) << 32) / x.p), shoup_const(r, x.p), x.a, x.cnt,
                         x.ap, x.out, x.n, x.out0});
    maxn = std::max(maxn, x.n);
  }
  std::memcpy(host_staging, v.data(), v.size() * sizeof(ExpPrepB));
  cudaError_t e = cudaMemcpyAsync(dev_desc, host_staging, v.size() * sizeof(ExpPrepB), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  if (staged && (e = cudaEventRecord(staged, s)) != cudaSuccess) return e;
  dim3 grid((unsigned)std::min<size_t>((maxn + 255) / 256, 256), (unsigned)v.size());
  (void)pdl_launch(k_exp_prep_b, grid, 256, 0, s, static_cast<const ExpPrepB*>(dev_desc));
  return cudaGetLastError();
}

size_t batch_aux_bytes(size_t jobs) { return jobs * std::max(sizeof(SeedJobB), sizeof(ExpPrepB)) + 256; }

}  // namespace fpx

namespace {
__global__ void k_gather_first(const uint32_t* const* __restrict__ ptrs, uint32_t* __restrict__ out, int n) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = ptrs[i] ? *ptrs[i] : 0u;
}

struct ReprSegB {
  Fp f;
  uint2 r_sh;  // 2^32 mod p as a Shoup constant
  uint32_t* ptr;
  size_t n;
  int to_mont;
};
__global__ void k_repr_b(const ReprSegB* __restrict__ segs) {
  pdl_enter();
  const ReprSegB& g = segs[blockIdx.y];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < g.n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = g.ptr[i];
    uint32_t y;
    if (g.f.p == 2) y = x & 1u;
    else if (g.to_mont) y = redc_any(shoup(x, g.r_sh, g.f.p), g.f.p);
    else y = red(mont(x, 1u, g.f), g.f.p);
    g.ptr[i] = y;
  }
}
}  // namespace

namespace fpx {
size_t repr_batch_bytes(size_t segs) { return segs * sizeof(ReprSegB) + 256; }

cudaError_t launch_repr_batch(const std::vector<ReprSeg>& segs, void* host_staging, void* dev_desc, cudaStream_t s,
                              cudaEvent_t staged) {
  std::vector<ReprSegB> v;
  size_t maxn = 0;
  for (const ReprSeg& x : segs) {
    if (x.n == 0) continue;
    ReprSegB b{};
    if (x.p == 2) {
      b.f.p = 2;
      b.f.p2 = 4;
      b.f.pinv = 1;
    } else {
      b.f = make_fp(x.p);
      b.r_sh = shoup_const((uint32_t)((((uint64_t)1) << 32) % x.p), x.p);
    }
    b.ptr = x.ptr;
    b.n = x.n;
    b.to_mont = x.to_mont;
    v.push_back(b);
    maxn = std::max(maxn, x.n);
  }
  if (v.empty()) return cudaSuccess;
  std::memcpy(host_staging, v.data(), v.size() * sizeof(ReprSegB));
  cudaError_t e = cudaMemcpyAsync(dev_desc, host_staging, v.size() * sizeof(ReprSegB), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  if (staged && (e = cudaEventRecord(staged, s)) != cudaSuccess) return e;
  for (size_t k = 0; k < v.size(); k += 65535) {  // grid.y limit
    const unsigned cnt = (unsigned)std::min<size_t>(65535, v.size() - k);
    dim3 grid((unsigned)std::min<size_t>((maxn + 255) / 256, 128), cnt);
    (void)pdl_launch(k_repr_b, grid, 256, 0, s, static_cast<const ReprSegB*>(dev_desc) + k);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace fpx

namespace fpx {
// out_host[i] = *ptrs[i] (0 for null) for many device pointers: one H2D of the
// pointer list, one kernel, one D2H; the caller synchronises the stream.
namespace {
constexpr int kScanThreads = 256, kScanPerThread = 4;
// Block b: the last nonzero word of segment b, scanning windows of
// kScanThreads * kScanPerThread words from the end (one window, as a rule: a
// remainder's top words are zero only by chance).
__global__ void __launch_bounds__(kScanThreads) k_last_nonzero_b(const Segment* __restrict__ segs,
                                                                 unsigned long long* __restrict__ out) {
  pdl_enter();
  const Segment g = segs[blockIdx.x];
  constexpr size_t W = (size_t)kScanThreads * kScanPerThread;
  size_t hi = g.n;
  unsigned long long found = g.n;
  while (hi > 0) {
    const size_t lo = hi > W ? hi - W : 0;
    long long best = -1;
#pragma unroll
    for (int k = 0; k < kScanPerThread; ++k) {
      const size_t i = lo + (size_t)k * kScanThreads + threadIdx.x;
      if (i < hi && g.ptr[i] != 0u) best = (long long)i;
    }
    // the largest index found in this window, if any
    __shared__ unsigned long long top;
    if (threadIdx.x == 0) top = 0;
    __syncthreads();
    if (best >= 0) atomicMax(&top, (unsigned long long)best + 1);
    __syncthreads();
    const unsigned long long t = top;
    __syncthreads();
    if (t) {
      found = t - 1;
      break;
    }
    hi = lo;
  }
  if (threadIdx.x == 0) out[blockIdx.x] = found;
}
}  // namespace

size_t last_nonzero_results_offset(size_t segs) { return (segs * sizeof(Segment) + 255) & ~size_t(255); }
size_t last_nonzero_batch_bytes(size_t segs) { return last_nonzero_results_offset(segs) + segs * 8 + 256; }

cudaError_t launch_last_nonzero_batch(const std::vector<Segment>& segs, void* host_staging, void* dev_buf,
                                      cudaStream_t s) {
  if (segs.empty()) return cudaSuccess;
  const size_t bytes = segs.size() * sizeof(Segment), roff = last_nonzero_results_offset(segs.size());
  std::memcpy(host_staging, segs.data(), bytes);
  char* d = static_cast<char*>(dev_buf);
  cudaError_t e = cudaMemcpyAsync(d, host_staging, bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  auto* dres = reinterpret_cast<unsigned long long*>(d + roff);
  (void)pdl_launch(k_last_nonzero_b, (unsigned)segs.size(), kScanThreads, 0, s,
                   reinterpret_cast<const Segment*>(d), dres);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return cudaMemcpyAsync(static_cast<char*>(host_staging) + roff, dres, segs.size() * 8, cudaMemcpyDeviceToHost, s);
}

cudaError_t launch_gather_first(const std::vector<const uint32_t*>& ptrs, void* host_staging, void* dev_buf,
                                uint32_t* host_out, cudaStream_t s) {
  if (ptrs.empty()) return cudaSuccess;
  const size_t bytes = ptrs.size() * sizeof(void*);
  std::memcpy(host_staging, ptrs.data(), bytes);
  char* d = static_cast<char*>(dev_buf);
  cudaError_t e = cudaMemcpyAsync(d, host_staging, bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  uint32_t* dout = reinterpret_cast<uint32_t*>(d + ((bytes + 255) & ~size_t(255)));
  (void)pdl_launch(k_gather_first, (unsigned)((ptrs.size() + 255) / 256), 256, 0, s, reinterpret_cast<const uint32_t* const*>(d),
                                                                         dout, (int)ptrs.size());
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return cudaMemcpyAsync(host_out, dout, ptrs.size() * 4, cudaMemcpyDeviceToHost, s);
}
}  // namespace fpx

// ===========================================================================
// One cyclic product of exactly 4096 points in one CTA: the row pass's
// register groups (three groups of four levels, padded conflict-free shared
// layout, twiddles loaded per group up front) for the forward transform(s),
// pointwise product and inverse, with the small-transform epilogue.  Replaces
// the generic one-CTA kernel at this size (13.2 us against 16.4 us for the
// generic kernel at half the size, one conv per call on B200).
//
// A thread-block-cluster version that spread 2^13..2^16-point products over
// 2..16 CTAs, exchanging the cross-chunk butterfly levels through distributed
// shared memory, was built and measured: 26 / 33 / 40 / 47 us against about
// 25 us for the three two-pass launches (each cross-chunk level cost a remote
// round trip and two cluster barriers), so those sizes stay two-pass.
// ===========================================================================
namespace {

__device__ __forceinline__ void cyc4096_body(const SmallD& job, const Ptab& pt) {
  __shared__ __align__(16) uint32_t sX[kRowWords];
  __shared__ __align__(16) uint32_t sY[kRowWords];
  const int t = threadIdx.x;
  const int bA = baseA(t), bB = baseB(t), bC = baseC(t);
  const Fp f = pt.f;
  const int ymode = job.ymode;
  uint32_t v[2][16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    v[0][i] = load_in(job.x, posA(t, i), f, pt.q1);
    if (ymode == 1) v[1][i] = load_in(job.y, posA(t, i), f, pt.q1);
  }
  if (ymode == 1) {
    bf_group<4, 12, false, 2>(v, pt.fwd, t, f);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      sX[bA + offA(i)] = v[0][i];
      sY[bA + offA(i)] = v[1][i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      v[0][i] = sX[bB + offB(i)];
      v[1][i] = sY[bB + offB(i)];
    }
    bf_group<4, 8, false, 2>(v, pt.fwd, t & 15, f);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      sX[bB + offB(i)] = v[0][i];
      sY[bB + offB(i)] = v[1][i];
    }
    __syncthreads();
    lds16(sX + bC, v[0]);
    lds16(sY + bC, v[1]);
    bf_group<4, 4, false, 2, true>(v, pt.fwd, 0, f);
    if (job.yspec_out) {
      uint4* o = reinterpret_cast<uint4*>(job.yspec_out + posC(t, 0));
#pragma unroll
      for (int q = 0; q < 4; ++q)
        o[q] = make_uint4(red(v[1][4 * q], f.p), red(v[1][4 * q + 1], f.p), red(v[1][4 * q + 2], f.p),
                          red(v[1][4 * q + 3], f.p));
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) v[0][i] = mont(v[0][i], v[1][i], f);
  } else {
    bf_group<4, 12, false, 1>(v, pt.fwd, t, f);
#pragma unroll
    for (int i = 0; i < 16; ++i) sX[bA + offA(i)] = v[0][i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 16; ++i) v[0][i] = sX[bB + offB(i)];
    bf_group<4, 8, false, 1>(v, pt.fwd, t & 15, f);
#pragma unroll
    for (int i = 0; i < 16; ++i) sX[bB + offB(i)] = v[0][i];
    __syncthreads();
    lds16(sX + bC, v[0]);
    bf_group<4, 4, false, 1, true>(v, pt.fwd, 0, f);
    if (ymode == 2) {
      const uint4* ys = reinterpret_cast<const uint4*>(job.yspec + posC(t, 0));
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint4 u = __ldg(ys + q);
        v[0][4 * q] = mont(v[0][4 * q], u.x, f);
        v[0][4 * q + 1] = mont(v[0][4 * q + 1], u.y, f);
        v[0][4 * q + 2] = mont(v[0][4 * q + 2], u.z, f);
        v[0][4 * q + 3] = mont(v[0][4 * q + 3], u.w, f);
      }
    } else if (ymode == 3) {
#pragma unroll
      for (int i = 0; i < 16; ++i) v[0][i] = mont(v[0][i], v[0][i], f);
    }
  }
  bf_group<4, 4, true, 1, true>(v, pt.inv, 0, f);
  sts16(sX + bC, v[0]);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 16; ++i) v[0][i] = sX[bB + offB(i)];
  bf_group<4, 8, true, 1>(v, pt.inv, t & 15, f);
#pragma unroll
  for (int i = 0; i < 16; ++i) sX[bB + offB(i)] = v[0][i];
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 16; ++i) v[0][i] = sX[bA + offA(i)];
  bf_group<4, 12, true, 1>(v, pt.inv, t, f);
#pragma unroll
  for (int i = 0; i < 16; ++i) epi_store(job.epi, posA(t, i), v[0][i], f);
}

__global__ void __launch_bounds__(256) k_cyc4096(SmallD job, Ptab pt) { pdl_enter(); cyc4096_body(job, pt); }
// Batched: one CTA per job (descriptors as the batched one-CTA kernel's).
__global__ void __launch_bounds__(256) k_cyc4096_b(const SmallJobB* __restrict__ jobs) {
  pdl_enter();
  const SmallJobB& j = jobs[blockIdx.x];
  cyc4096_body(j.d, j.pt);
}

}  // namespace

namespace fpx {

cudaError_t launch_cyc4096(const PrimeTables& pt, const SmallJob& job, cudaStream_t s) {
  SmallD d;
  d.x = dev_in(job.x);
  d.y = dev_in(job.y);
  d.forward = 1;
  d.ymode = job.ymode;
  d.inverse = 1;
  d.yspec = job.yspec;
  d.yspec_out = job.yspec_out;
  d.spec_x = nullptr;
  d.epi = dev_epi(job.epi);
  (void)pdl_launch(k_cyc4096, 1, 256, 0, s, d, dev_tab(pt));
  return cudaGetLastError();
}

}  // namespace fpx

// ===========================================================================
// Cyclic products of N = 2^LOGN <= 2^13 points in one CTA with compile-time
// structure: groups of at most four levels (sizes as the column passes'),
// every group's twiddles loaded up front, both operands of a product in the
// same register pass (twiddles shared), shared memory padded one word per 32.
// Replaces the generic one-CTA kernel for products (the raw transform keeps
// the generic one).
// ===========================================================================
namespace {

template <int LOGN, int KG, bool INV, int NA>
__device__ __forceinline__ void cyc_group(uint32_t* const (&S)[2], const uint2* __restrict__ tw, const Fp& f,
                                          int tid, int nt) {
  using Gs = ColGroups<LOGN>;
  constexpr int G = Gs::size(KG);
  constexpr int T = Gs::top(KG);
  constexpr int SS = T - G;
  constexpr int NINST = (1 << LOGN) >> G;
#pragma unroll 1
  for (int inst = tid; inst < NINST; inst += nt) {
    const int base = inst & ((1 << SS) - 1);
    const int p0 = ((inst >> SS) << T) + base;
    uint32_t v[2][1 << G];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int i = 0; i < (1 << G); ++i) v[a][i] = S[a][pad(p0 + (i << SS))];
    bf_group<G, T, INV, NA>(v, tw, base, f);
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int i = 0; i < (1 << G); ++i) S[a][pad(p0 + (i << SS))] = v[a][i];
  }
}

template <int LOGN, int KG, int NA>
__device__ __forceinline__ void cyc_fwd(uint32_t* const (&S)[2], const uint2* tw, const Fp& f, int tid, int nt) {
  if constexpr (KG < ColGroups<LOGN>::K) {
    cyc_group<LOGN, KG, false, NA>(S, tw, f, tid, nt);
    __syncthreads();
    cyc_fwd<LOGN, KG + 1, NA>(S, tw, f, tid, nt);
  }
}

template <int LOGN, int KG>
__device__ __forceinline__ void cyc_inv(uint32_t* const (&S)[2], const uint2* tw, const Fp& f, int tid, int nt) {
  if constexpr (KG >= 0) {
    cyc_group<LOGN, KG, true, 1>(S, tw, f, tid, nt);
    __syncthreads();
    cyc_inv<LOGN, KG - 1>(S, tw, f, tid, nt);
  }
}

template <int LOGN>
__device__ __forceinline__ void cyc_small_body(const SmallD& job, const Ptab& pt) {
  extern __shared__ uint32_t sm[];
  constexpr int N = 1 << LOGN;
  const int tid = threadIdx.x, nt = blockDim.x;
  uint32_t* const S[2] = {sm, sm + padded_words(N)};
  const Fp f = pt.f;
  const int ymode = job.ymode;
  for (int i = tid; i < N; i += nt) {
    S[0][pad(i)] = load_in(job.x, i, f, pt.q1);
    if (ymode == 1) S[1][pad(i)] = load_in(job.y, i, f, pt.q1);
    else if (ymode == 2) S[1][pad(i)] = __ldg(job.yspec + i);
  }
  __syncthreads();
  if (ymode == 1) {
    cyc_fwd<LOGN, 0, 2>(S, pt.fwd, f, tid, nt);
    if (job.yspec_out)
      for (int i = tid; i < N; i += nt) job.yspec_out[i] = red(S[1][pad(i)], f.p);
  } else {
    cyc_fwd<LOGN, 0, 1>(S, pt.fwd, f, tid, nt);
  }
  if (ymode == 1 || ymode == 2) {
    for (int i = tid; i < N; i += nt) S[0][pad(i)] = mont(S[0][pad(i)], S[1][pad(i)], f);
  } else if (ymode == 3) {
    for (int i = tid; i < N; i += nt) {
      const uint32_t v = S[0][pad(i)];
      S[0][pad(i)] = mont(v, v, f);
    }
  }
  __syncthreads();
  cyc_inv<LOGN, ColGroups<LOGN>::K - 1>(S, pt.inv, f, tid, nt);
  const uint32_t hi = job.epi.hi < (uint32_t)N ? job.epi.hi : (uint32_t)N;
  for (uint32_t i = job.epi.lo + tid; i < hi; i += nt) epi_store(job.epi, i, S[0][pad(i)], f);
}

template <int LOGN>
__global__ void __launch_bounds__(512) k_cyc_small(SmallD job, Ptab pt) {
  pdl_enter();
  cyc_small_body<LOGN>(job, pt);
}
template <int LOGN>
__global__ void __launch_bounds__(512) k_cyc_small_b(const SmallJobB* __restrict__ jobs) {
  pdl_enter();
  const SmallJobB& j = jobs[blockIdx.x];
  cyc_small_body<LOGN>(j.d, j.pt);
}

using CycFn = void (*)(SmallD, Ptab);
using CycBFn = void (*)(const SmallJobB*);

template <int... L>
struct CycTable {
  static CycFn one(int logN) {
    CycFn r = nullptr;
    ((logN == L ? (r = k_cyc_small<L>, 0) : 0), ...);
    return r;
  }
  static CycBFn batch(int logN) {
    CycBFn r = nullptr;
    ((logN == L ? (r = k_cyc_small_b<L>, 0) : 0), ...);
    return r;
  }
  static cudaError_t init() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* fn, int bytes) {
      const cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      if (r != cudaSuccess) e = r;
    };
    (set((const void*)k_cyc_small<L>, 2 * padded_words(1 << L) * 4), ...);
    (set((const void*)k_cyc_small_b<L>, 2 * padded_words(1 << L) * 4), ...);
    return e;
  }
};
using Cyc = CycTable<1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13>;

int cyc_threads(int logN) {
  const int n = (1 << logN) / 16;
  return n < 32 ? 32 : (n > 512 ? 512 : n);
}

}  // namespace

namespace fpx {

cudaError_t kernels_cyc_init() { return Cyc::init(); }

cudaError_t launch_cyc_small(const PrimeTables& pt, int logN, const SmallJob& job, cudaStream_t s) {
  CycFn fn = Cyc::one(logN);
  if (!fn) return cudaErrorInvalidValue;
  SmallD d;
  d.x = dev_in(job.x);
  d.y = dev_in(job.y);
  d.forward = 1;
  d.ymode = job.ymode;
  d.inverse = 1;
  d.yspec = job.yspec;
  d.yspec_out = job.yspec_out;
  d.spec_x = nullptr;
  d.epi = dev_epi(job.epi);
  (void)pdl_launch(fn, 1, cyc_threads(logN), (size_t)2 * padded_words(1 << logN) * 4, s, d, dev_tab(pt));
  return cudaGetLastError();
}

}  // namespace fpx

namespace {
cudaError_t launch_cyc_small_batch(int logN, unsigned count, const SmallJobB* jobs, cudaStream_t s) {
  CycBFn fn = Cyc::batch(logN);
  if (!fn) return cudaErrorInvalidValue;
  (void)pdl_launch(fn, count, cyc_threads(logN), (size_t)2 * padded_words(1 << logN) * 4, s, jobs);
  return cudaGetLastError();
}
}  // namespace

namespace fpx {

namespace {
bool crt_cl_fill(const PrimeTables* aux, uint32_t P, CrtCl& cc) {
  static const uint32_t kAux[3] = {167772161u, 469762049u, 754974721u};
  if (P < 2) return false;
  for (int i = 0; i < 3; ++i) {
    if (aux[i].p != kAux[i] || aux[i].small_log < kNewtonMaxLog) return false;
    cc.q[i] = dev_tab(aux[i]);
    for (int l = 0; l <= kNewtonMaxLog; ++l) cc.scale_r[i][l] = shoup_const(aux[i].inv_pow2_r[l], aux[i].p);
  }
  cc.g = garner_consts(P);
  cc.P = P;
  cc.pinv = (P & 1u) ? inv_mod_2_32(P) : 0u;
  return true;
}

// One cluster of three CTAs, one per transform prime.
template <typename D>
cudaError_t crt_cl_launch(void (*k)(D), const D& d, cudaStream_t s, unsigned clusters = 1) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(3 * clusters);
  cfg.blockDim = dim3(kNewtonThreads);
  cfg.dynamicSmemBytes = (size_t)kNewtonCrtSmemWords * 4;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 3;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k, d);
  return e != cudaSuccess ? e : cudaGetLastError();
}
}  // namespace

cudaError_t launch_newton_inv_crt(const PrimeTables* aux, uint32_t P, const uint32_t* a, size_t la, uint32_t* c,
                                  size_t K, cudaStream_t s) {
  NewtonCrtD d;
  if (K < 1 || K > (size_t(1) << kNewtonMaxLog) || !crt_cl_fill(aux, P, d.cc)) return cudaErrorInvalidValue;
  d.a = a;
  d.la = (uint32_t)std::min<size_t>(la, K);
  d.c = c;
  d.K = (uint32_t)K;
  return crt_cl_launch(k_newton_inv_crt, d, s);
}

cudaError_t launch_newton_exp_crt(const PrimeTables* aux, uint32_t P, const uint32_t* ap, size_t lap,
                                  const uint32_t* tab, uint32_t* b, uint32_t* c, size_t K, cudaStream_t s) {
  NewtonExpCrtD d;
  if (K < 2 || K > (size_t(1) << kNewtonMaxLog) || !(P & 1u) || !crt_cl_fill(aux, P, d.cc))
    return cudaErrorInvalidValue;
  d.ap = ap;
  d.lap = (uint32_t)std::min<size_t>(lap, K);
  d.tab = tab;
  d.b = b;
  d.c = c;
  d.K = (uint32_t)K;
  return crt_cl_launch(k_newton_exp_crt, d, s);
}

cudaError_t fill_newton_crt_batch(const std::vector<const NewtonJob*>& jobs, void* host) {
  auto* out = static_cast<NewtonCrtJobB*>(host);
  for (size_t i = 0; i < jobs.size(); ++i) {
    const NewtonJob& x = *jobs[i];
    if (x.K < 1 || x.K > (size_t(1) << kNewtonMaxLog) || (x.kind == 1 && (x.K < 2 || !(x.P & 1u))))
      return cudaErrorInvalidValue;
    NewtonCrtJobB j;
    std::memset(&j, 0, sizeof j);
    j.kind = x.kind;
    CrtCl& cc = x.kind == 0 ? j.inv.cc : j.exp.cc;
    if (!crt_cl_fill(x.aux, x.P, cc)) return cudaErrorInvalidValue;
    if (x.kind == 0) {
      j.inv.a = x.a;
      j.inv.la = (uint32_t)std::min<size_t>(x.la, x.K);
      j.inv.c = x.out;
      j.inv.K = (uint32_t)x.K;
    } else {
      j.exp.ap = x.a;
      j.exp.lap = (uint32_t)std::min<size_t>(x.la, x.K);
      j.exp.tab = x.tab;
      j.exp.b = x.out;
      j.exp.c = x.c;
      j.exp.K = (uint32_t)x.K;
    }
    std::memcpy(out + i, &j, sizeof j);
  }
  return cudaSuccess;
}

// Any number of cluster jobs: launches of at most kCrtClustersPerLaunch clusters
// each, the descriptor pointer advanced by the jobs already launched.
constexpr size_t kCrtClustersPerLaunch = 65535;

cudaError_t launch_newton_crt_b(const void* dev, size_t count, cudaStream_t s) {
  const auto* jobs = static_cast<const NewtonCrtJobB*>(dev);
  for (size_t done = 0; done < count;) {
    const size_t n = std::min(count - done, kCrtClustersPerLaunch);
    const cudaError_t e = crt_cl_launch(k_newton_crt_b, jobs + done, s, (unsigned)n);
    if (e != cudaSuccess) return e;
    done += n;
  }
  return cudaSuccess;
}

cudaError_t launch_newton_sqrt_crt(const PrimeTables* aux, uint32_t P, const uint32_t* u, size_t ulen, uint32_t root,
                                   uint32_t root_inv, uint32_t* b, uint32_t* c, size_t K, cudaStream_t s) {
  NewtonSqrtCrtD d;
  if (K < 1 || K > (size_t(1) << kNewtonMaxLog) || !(P & 1u) || !crt_cl_fill(aux, P, d.cc))
    return cudaErrorInvalidValue;
  d.u = u;
  d.ulen = (uint32_t)std::min<size_t>(ulen, K);
  d.b = b;
  d.c = c;
  d.K = (uint32_t)K;
  d.root = root;
  d.root_inv = root_inv;
  return crt_cl_launch(k_newton_sqrt_crt, d, s);
}

}  // namespace fpx
