// field.cuh - modular arithmetic for the B200 transform kernels.
//
// Conventions (the reference's lazy-reduction contract, simd.hpp:12-21 and
// ntt.hpp:19-27, re-derived for 32-bit GPU lanes):
//   * every transform prime satisfies p < 2^30, so 4p < 2^32;
//   * forward (DIF) butterflies keep values in [0, 2p);
//   * inverse (DIT, Harvey-style) butterflies keep values in [0, 4p);
//   * twiddles are multiplied with Shoup's method: a precomputed quotient
//     wq = floor(w * 2^32 / p) turns a*w mod p into one mul.hi and two mul.lo
//     (the reference's Q32 fixed multipliers, simd.hpp:98-147);
//   * products of two variable operands use Montgomery REDC with mul.lo/mul.hi
//     (modint.hpp:88-93), which leaves a factor 2^-32 that callers fold into a
//     constant elsewhere.
#pragma once
#include <cstdint>

namespace fpx_dev {

struct Fp {
  uint32_t p;     // modulus, < 2^30
  uint32_t p2;    // 2p
  uint32_t pinv;  // p^-1 mod 2^32
};

__host__ __device__ inline uint32_t inv_mod_2_32(uint32_t a) {
  uint32_t x = 1;
  for (int i = 0; i < 5; ++i) x *= 2u - a * x;
  return x;
}

__host__ inline Fp make_fp(uint32_t p) { return Fp{p, 2u * p, inv_mod_2_32(p)}; }

// min(x, x - m) over unsigned: subtract m once if x >= m (x < 2m required).
// One DPX add-min instruction on sm_90 and later.
__device__ __forceinline__ uint32_t red(uint32_t x, uint32_t m) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  return __viaddmin_u32(x, 0u - m, x);
#else
  return min(x, x - m);
#endif
}

// a*w mod p in [0, 2p) for any a < 2^32, w < p, wq = floor(w*2^32/p).
__device__ __forceinline__ uint32_t shoup(uint32_t a, uint32_t w, uint32_t wq, uint32_t p) {
  const uint32_t q = __umulhi(a, wq);
  return a * w - q * p;
}
__device__ __forceinline__ uint32_t shoup(uint32_t a, uint2 t, uint32_t p) { return shoup(a, t.x, t.y, p); }

// Montgomery product a*b*2^-32 mod p in (0, 2p) for a*b < p*2^32.
__device__ __forceinline__ uint32_t mont(uint32_t a, uint32_t b, const Fp& f) {
  const uint32_t lo = a * b;
  const uint32_t hi = __umulhi(a, b);
  const uint32_t m = lo * f.pinv;
  return hi - __umulhi(m, f.p) + f.p;
}

// Canonical residue from a lazy value in [0, 4p).
__device__ __forceinline__ uint32_t canon4(uint32_t x, const Fp& f) { return red(red(x, f.p2), f.p); }
__device__ __forceinline__ uint32_t canon2(uint32_t x, const Fp& f) { return red(x, f.p); }

// x mod p for any 32-bit x: Shoup by w = 1 (q1 = floor(2^32/p)) then one subtract.
__device__ __forceinline__ uint32_t reduce_any(uint32_t x, uint32_t q1, const Fp& f) {
  return red(x - __umulhi(x, q1) * f.p, f.p);
}

// Gentleman-Sande (DIF) butterfly, inputs/outputs in [0, 2p).
__device__ __forceinline__ void dif_bf(uint32_t& u, uint32_t& v, uint2 w, const Fp& f) {
  const uint32_t s = u + v;
  const uint32_t d = u - v + f.p2;
  u = red(s, f.p2);
  v = shoup(d, w, f.p);
}
// DIF butterfly with unit twiddle.
__device__ __forceinline__ void dif_bf1(uint32_t& u, uint32_t& v, const Fp& f) {
  const uint32_t s = u + v;
  const uint32_t d = u - v + f.p2;
  u = red(s, f.p2);
  v = red(d, f.p2);
}
// Cooley-Tukey (DIT) butterfly, Harvey's lazy form: inputs/outputs in [0, 4p).
__device__ __forceinline__ void dit_bf(uint32_t& u, uint32_t& v, uint2 w, const Fp& f) {
  const uint32_t a = red(u, f.p2);
  const uint32_t t = shoup(v, w, f.p);
  u = a + t;
  v = a - t + f.p2;
}
__device__ __forceinline__ void dit_bf1(uint32_t& u, uint32_t& v, const Fp& f) {
  const uint32_t a = red(u, f.p2);
  const uint32_t t = red(v, f.p2);
  u = a + t;
  v = a - t + f.p2;
}

}  // namespace fpx_dev
