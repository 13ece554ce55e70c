// fpx/fastpoly.hpp - C++20 drop-in for the reference's polynomial API, backed
// by the B200 library through its C ABI (fpx_b200.h).
//
// Same names, signatures, value semantics and error types as the reference's
// umbrella header include/fastpoly/fastpoly.hpp:
//   fpx::Mont<Mod, Root>, fpx::ModInt<Mod>, fpx::mod998244353 ...   (modint.hpp:57-205)
//   fpx::Poly<M> : std::vector<M>                                    (poly.hpp:16-86)
//   fpx::poly::conv / inv / log / exp / sqrt / pow / divmod / div / mod
//   fpx::NttPlan<M>::get(n)->forward / inverse                       (ntt.hpp:130-192)
//   fpx::poly::domain_error, fpx::ntt_size_error
// A Poly<Mont<p>> hands its Montgomery limbs to the GPU unchanged
// (FPX_REPR_MONTGOMERY); the first and last GPU passes convert.  The O(n) host
// helpers (add, sub, neg, mul_scalar, shift, eval, derivative, integral) are
// plain loops: they are not on the transform path.
//
// Link with fastpoly_b200/libfpx_b200.so.  One process-wide context on device
// FPX_DEVICE (default 0) is created on first use; calls from several threads
// are serialised inside it.
#ifndef FPX_DROPIN_FASTPOLY_HPP
#define FPX_DROPIN_FASTPOLY_HPP

#include <algorithm>
#include <array>
#include <bit>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <istream>
#include <map>
#include <memory>
#include <mutex>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "fpx_b200.h"

namespace fpx {

// ------------------------------------------------------------------ field

namespace detail {
// x^e mod m for 64-bit intermediates (compile-time friendly).
constexpr uint64_t pow_mod(uint64_t x, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  x %= m;
  while (e) {
    if (e & 1) r = r * x % m;
    x = x * x % m;
    e >>= 1;
  }
  return r;
}
}  // namespace detail

/// a^-1 mod 2^32 for odd a: a is its own inverse to 3 bits, and each Newton
/// step x <- x (2 - a x) doubles the correct bits (3, 6, 12, 24, 48).
constexpr uint32_t inv_mod_2_32(uint32_t a) {
  uint32_t x = a;
  for (int bits = 3; bits < 32; bits *= 2) x *= 2u - a * x;
  return x;
}

/// The smallest primitive root of the prime p: the first g whose powers
/// g^((p-1)/q) avoid 1 for every prime q dividing p - 1.
constexpr uint32_t primitive_root(uint32_t p) {
  if (p == 2) return 1;
  std::array<uint32_t, 10> q{};  // distinct prime factors of p - 1 (at most 9 below 2^31)
  size_t nq = 0;
  uint32_t r = p - 1;
  for (uint32_t d = 2; uint64_t(d) * d <= r; d += (d == 2 ? 1 : 2)) {
    if (r % d) continue;
    q[nq++] = d;
    while (r % d == 0) r /= d;
  }
  if (r > 1) q[nq++] = r;
  for (uint32_t g = 2; g < p; ++g) {
    size_t k = 0;
    while (k < nq && detail::pow_mod(g, (p - 1) / q[k], p) != 1) ++k;
    if (k == nq) return g;
  }
  return 0;
}

/// Element of GF(Mod) stored as the Montgomery limb x * 2^32 mod Mod (a single
/// bit for Mod = 2), bit-compatible with the reference's Mont.
template <uint32_t Mod, uint32_t Root = 0>
class Mont {
 public:
  static_assert(Mod < (1u << 31) && Mod >= 2, "modulus must be a prime in [2, 2^31)");
  static constexpr uint32_t mod = Mod;
  static constexpr uint32_t primitive_root = Root != 0 ? Root : fpx::primitive_root(Mod);
  // -Mod^-1 mod 2^32 (0 for Mod = 2, whose limbs are the bits themselves)
  static constexpr uint32_t ninv = Mod == 2 ? 0u : static_cast<uint32_t>(0u - inv_mod_2_32(Mod));
  static constexpr uint32_t one = Mod == 2 ? 1u : static_cast<uint32_t>((uint64_t(1) << 32) % Mod);
  static constexpr uint32_t r2 = static_cast<uint32_t>(uint64_t(one) * one % Mod);
  static constexpr uint32_t inv2 = (Mod + 1) / 2;

  constexpr Mont() : v_(0) {}
  template <class I, class = std::enable_if_t<std::is_integral_v<I> && !std::is_same_v<I, bool>>>
  constexpr Mont(I x) : v_(to_limb(static_cast<uint64_t>(x))) {}

  static constexpr Mont from_int(uint64_t x) { return of_limb(to_limb(x)); }
  static constexpr Mont raw(uint32_t x) { return of_limb(x); }
  /// t * 2^-32 mod Mod for t < Mod * 2^32 (Montgomery reduction), canonical.
  static constexpr uint32_t reduce(uint64_t t) {
    if constexpr (Mod == 2) {
      return static_cast<uint32_t>(t & 1u);
    } else {
      // t + m Mod is divisible by 2^32 for m = (t mod 2^32) (-Mod^-1)
      const uint64_t m = static_cast<uint32_t>(static_cast<uint32_t>(t) * ninv);
      const uint64_t u = (t >> 32) + ((static_cast<uint64_t>(static_cast<uint32_t>(t)) + m * Mod) >> 32);
      return canon(u);
    }
  }
  constexpr uint32_t val() const { return reduce(v_); }
  constexpr uint32_t raw_val() const { return v_; }

  friend constexpr Mont operator+(Mont a, Mont b) { return of_limb(canon(uint64_t(a.v_) + b.v_)); }
  friend constexpr Mont operator-(Mont a, Mont b) { return of_limb(canon(uint64_t(a.v_) + Mod - b.v_)); }
  friend constexpr Mont operator-(Mont a) { return Mont() - a; }
  friend constexpr Mont operator*(Mont a, Mont b) { return of_limb(reduce(uint64_t(a.v_) * b.v_)); }
  friend constexpr Mont operator/(Mont a, Mont b) { return a * b.inv(); }
  constexpr Mont& operator+=(Mont b) { return *this = *this + b; }
  constexpr Mont& operator-=(Mont b) { return *this = *this - b; }
  constexpr Mont& operator*=(Mont b) { return *this = *this * b; }
  constexpr Mont& operator/=(Mont b) { return *this = *this / b; }
  friend constexpr bool operator==(Mont a, Mont b) { return a.v_ == b.v_; }
  friend constexpr bool operator!=(Mont a, Mont b) { return a.v_ != b.v_; }
  constexpr bool is_zero() const { return v_ == 0; }
  constexpr bool operator!() const { return v_ == 0; }
  constexpr explicit operator bool() const { return v_ != 0; }

  /// this^e, scanning the exponent from its top bit down.
  constexpr Mont pow(uint64_t e) const {
    Mont r = from_int(1);
    for (int bit = 63; bit >= 0; --bit) {
      r *= r;
      if ((e >> bit) & 1) r *= *this;
    }
    return r;
  }
  /// Multiplicative inverse by Fermat (0 maps to 0).
  constexpr Mont inv() const {
    if constexpr (Mod == 2) return *this;
    else return pow(Mod - 2);
  }
  /// A square root, the one Tonelli-Shanks gives with the non-residue z found
  /// by counting up from 2 (the reference's choice, which fixes poly::sqrt's
  /// result); false for a non-residue.  For Mod = 3 mod 4 this is
  /// this^((Mod+1)/4), the case s = 1 below.
  bool sqrt(Mont& out) const {
    if constexpr (Mod == 2) {
      out = *this;
      return true;
    } else {
      const Mont unit = from_int(1);
      if (is_zero()) {
        out = *this;
        return true;
      }
      if (pow((Mod - 1) / 2) != unit) return false;  // Euler's criterion
      int s = std::countr_zero(Mod - 1);             // Mod - 1 = q 2^s, q odd
      const uint64_t q = (Mod - 1) >> s;
      Mont z = from_int(2);
      while (z.pow((Mod - 1) / 2) == unit) z += unit;  // the first non-residue
      Mont c = z.pow(q), t = pow(q), root = pow((q + 1) / 2);
      while (t != unit) {
        int i = 1;  // least i with t^(2^i) = 1
        for (Mont sq = t * t; sq != unit; sq *= sq) ++i;
        Mont b = c;
        for (int k = 0; k < s - i - 1; ++k) b *= b;
        root *= b;
        c = b * b;
        t *= c;
        s = i;
      }
      out = root;
      return true;
    }
  }
  std::string str() const { return std::to_string(val()); }

 private:
  static constexpr uint32_t canon(uint64_t x) { return static_cast<uint32_t>(x >= Mod ? x - Mod : x); }
  static constexpr uint32_t to_limb(uint64_t x) { return static_cast<uint32_t>(x % Mod * uint64_t(one) % Mod); }
  static constexpr Mont of_limb(uint32_t v) {
    Mont m;
    m.v_ = v;
    return m;
  }
  uint32_t v_;
};

template <uint32_t M, uint32_t R>
std::ostream& operator<<(std::ostream& os, const Mont<M, R>& a) { return os << a.val(); }
template <uint32_t M, uint32_t R>
std::istream& operator>>(std::istream& is, Mont<M, R>& a) {
  uint64_t x = 0;
  is >> x;
  a = Mont<M, R>::from_int(x);
  return is;
}

using mod998244353 = Mont<998244353u, 3>;
using mod1004535809 = Mont<1004535809u, 3>;
using mod469762049 = Mont<469762049u, 3>;
using mod167772161 = Mont<167772161u, 3>;
using mod754974721 = Mont<754974721u, 11>;
using mod1224736769 = Mont<1224736769u, 3>;
template <uint32_t Mod>
using ModInt = Mont<Mod>;
using mod1000000007 = Mont<1000000007u>;

// ------------------------------------------------------------------ errors

class ntt_size_error : public std::runtime_error {
 public:
  explicit ntt_size_error(const std::string& s) : std::runtime_error(s) {}
};
namespace poly {
class domain_error : public std::runtime_error {
 public:
  explicit domain_error(const std::string& s) : std::runtime_error(s) {}
};
template <class M>
using vec = std::vector<M>;
}  // namespace poly

namespace gpu {

/// The process-wide context (device from FPX_DEVICE, default 0).
inline fpx_ctx* context() {
  static std::once_flag once;
  static fpx_ctx* ctx = nullptr;
  static int status = 0;
  std::call_once(once, [] {
    const char* d = std::getenv("FPX_DEVICE");
    status = fpx_ctx_create(d ? std::atoi(d) : 0, 0, &ctx);
  });
  if (!ctx) throw std::runtime_error("fastpoly_b200: no usable CUDA device (status " + std::to_string(status) + ")");
  return ctx;
}

inline void check(int rc, const char* what) {
  if (rc == FPX_OK) return;
  const std::string msg = std::string(what) + ": " + fpx_last_error_message(context());
  if (rc == FPX_EDOMAIN) throw poly::domain_error(msg);
  if (rc == FPX_ESIZE) throw ntt_size_error(msg);
  if (rc == FPX_ELENGTH) throw std::length_error(msg);
  if (rc == FPX_ENOMEM) throw std::bad_alloc();
  throw std::runtime_error(msg);
}

template <class M>
const uint32_t* limbs(const std::vector<M>& v) {
  static_assert(sizeof(M) == sizeof(uint32_t), "Mont must be a single 32-bit limb");
  return reinterpret_cast<const uint32_t*>(v.data());
}
template <class M>
uint32_t* limbs(std::vector<M>& v) {
  return reinterpret_cast<uint32_t*>(v.data());
}

}  // namespace gpu

// ------------------------------------------------------- scratch memory

/// The reference's scratch statistics (memory.hpp:21-26), here of the GPU
/// context's device pool (one per process rather than per thread).
#ifndef FASTPOLY_SCRATCH_CACHE_BYTES
// The reference's per-thread idle scratch limit (memory.hpp:15-17).  The device
// pool keeps every idle block until release_scratch_memory(), so a warm call of
// any size is served from the cache.
#define FASTPOLY_SCRATCH_CACHE_BYTES (64u * 1024u * 1024u)
#endif

struct ScratchMemoryStats {
  size_t cached_bytes = 0;
  size_t cached_blocks = 0;
  size_t system_allocations = 0;
  size_t cache_hits = 0;
};
inline ScratchMemoryStats scratch_memory_stats() noexcept {
  fpx_pool_stats_t st{};
  try {
    if (fpx_pool_stats(gpu::context(), &st) != FPX_OK) return {};
  } catch (...) {
    return {};
  }
  return ScratchMemoryStats{st.cached_bytes, st.cached_blocks, st.system_allocations, st.cache_hits};
}
/// Frees the idle cached blocks (memory.hpp:252-254); live buffers and plans stay.
inline void release_scratch_memory() noexcept {
  try {
    (void)fpx_release_pool(gpu::context());
  } catch (...) {
  }
}

// ---------------------------------------------------------------- NttPlan

/// GPU transform of one size (the reference's NttPlan<M>, ntt.hpp:86-194):
/// forward is the bit-reversal-free DIF (spectrum in bit-reversed order),
/// inverse the matching DIT scaled by 1/n; both on Montgomery limbs, in place,
/// outputs in [0, Mod).  Requires Mod < 2^30.
template <class M>
class NttPlan {
 public:
  static std::shared_ptr<const NttPlan> get(uint32_t n) {
    check_size(n);
    return std::shared_ptr<const NttPlan>(new NttPlan(n));
  }
  /// One plan per size for the life of the process (ntt.hpp:135).
  static const NttPlan& get_ref(uint32_t n) {
    check_size(n);
    static std::mutex mu;
    static std::map<uint32_t, std::unique_ptr<NttPlan>> plans;
    std::lock_guard<std::mutex> g(mu);
    auto& slot = plans[n];
    if (!slot) slot.reset(new NttPlan(n));
    return *slot;
  }
  uint32_t size() const { return n_; }
  int log_size() const { return std::countr_zero(n_); }
  void forward(uint32_t* a) const { gpu::check(fpx_ntt_forward(gpu::context(), M::mod, a, n_, FPX_REPR_MONTGOMERY), "ntt"); }
  void inverse(uint32_t* a) const { gpu::check(fpx_ntt_inverse(gpu::context(), M::mod, a, n_, FPX_REPR_MONTGOMERY), "ntt"); }
  /// The reference's lazy forward (ntt.hpp:145-148): same permutation and residues
  /// as forward(); the GPU returns them reduced, a valid lazy representative.
  void forward_lazy(uint32_t* a) const { forward(a); }
  /// Forward transform of a live prefix a[0, count), [count, n) taken as zero
  /// (ntt.hpp:150-175): those limbs are overwritten with zeros first.
  void forward_prefix(uint32_t* a, size_t count) const {
    if (count > n_) throw ntt_size_error("NTT input prefix exceeds plan size");
    std::memset(a + count, 0, (n_ - count) * sizeof(uint32_t));
    forward(a);
  }
  /// Inverse whose caller needs only [0, count) (ntt.hpp:181-188); every output
  /// is produced, the rest is valid too.
  void inverse_prefix(uint32_t* a, size_t count) const {
    if (count > n_) throw ntt_size_error("NTT output prefix exceeds plan size");
    inverse(a);
  }
  /// Inverse whose caller needs only the high half [n/2, n) (ntt.hpp:190-191).
  void inverse_highhalf(uint32_t* a) const { inverse(a); }

 private:
  explicit NttPlan(uint32_t n) : n_(n) {}
  static void check_size(uint32_t n) {
    if (n < 2 || (n & (n - 1)) != 0) throw ntt_size_error("NTT size must be a power of two");
    if (n > (uint64_t(1) << fpx_ntt_max_log(M::mod))) throw ntt_size_error("NTT size exceeds 2^v2(mod-1) for this modulus");
  }
  uint32_t n_;
};

// ------------------------------------------------------------------ poly

namespace poly {

inline constexpr size_t naive_threshold = 40;

template <class M>
void trim(vec<M>& a) {
  while (!a.empty() && a.back().is_zero()) a.pop_back();
}

/// Product of a and b truncated to n coefficients (convolution.hpp:145-147).
template <class M>
vec<M> conv(const vec<M>& a, const vec<M>& b, size_t n = SIZE_MAX) {
  if (a.empty() || b.empty() || n == 0) return {};
  const size_t la = std::min(a.size(), n), lb = std::min(b.size(), n);
  if (la > SIZE_MAX - (lb - 1)) throw std::length_error("poly::conv: result length overflows size_t");
  vec<M> r(std::min(la + lb - 1, n));
  size_t got = 0;
  gpu::check(fpx_conv(gpu::context(), M::mod, gpu::limbs(a), a.size(), gpu::limbs(b), b.size(), n, gpu::limbs(r), &got,
                      FPX_REPR_MONTGOMERY),
             "poly::conv");
  r.resize(got);
  return r;
}

#define FPX_SERIES(name, fn)                                                                                   \
  template <class M>                                                                                           \
  vec<M> name(const vec<M>& a, size_t n) {                                                                     \
    vec<M> r(n);                                                                                               \
    gpu::check(fn(gpu::context(), M::mod, gpu::limbs(a), a.size(), n, gpu::limbs(r), FPX_REPR_MONTGOMERY),     \
               "poly::" #name);                                                                                \
    return r;                                                                                                  \
  }
FPX_SERIES(inv, fpx_inv)
FPX_SERIES(log, fpx_log)
FPX_SERIES(exp, fpx_exp)
FPX_SERIES(sqrt, fpx_sqrt)
#undef FPX_SERIES

template <class M>
vec<M> pow(const vec<M>& a, uint64_t k, size_t n) {
  vec<M> r(n);
  gpu::check(fpx_pow(gpu::context(), M::mod, gpu::limbs(a), a.size(), k, n, gpu::limbs(r), FPX_REPR_MONTGOMERY),
             "poly::pow");
  return r;
}

template <class M>
std::pair<vec<M>, vec<M>> divmod(const vec<M>& a, const vec<M>& b) {
  vec<M> q(std::max<size_t>(a.size(), 1)), r(std::max<size_t>(b.size(), 1));
  size_t lq = 0, lr = 0;
  gpu::check(fpx_divmod(gpu::context(), M::mod, gpu::limbs(a), a.size(), gpu::limbs(b), b.size(), gpu::limbs(q), &lq,
                        gpu::limbs(r), &lr, FPX_REPR_MONTGOMERY),
             "poly::divmod");
  q.resize(lq);
  r.resize(lr);
  return {std::move(q), std::move(r)};
}
template <class M>
vec<M> div(const vec<M>& a, const vec<M>& b) { return divmod(a, b).first; }
template <class M>
vec<M> mod(const vec<M>& a, const vec<M>& b) { return divmod(a, b).second; }

// ---- O(n) host helpers (basic.hpp, calculus.hpp); not on the transform path.
template <class M>
vec<M> add(const vec<M>& a, const vec<M>& b) {
  vec<M> r = a.size() >= b.size() ? a : b;
  const vec<M>& s = a.size() >= b.size() ? b : a;
  for (size_t i = 0; i < s.size(); ++i) r[i] += s[i];
  return r;
}
template <class M>
vec<M> sub(const vec<M>& a, const vec<M>& b) {
  vec<M> r = a;
  if (r.size() < b.size()) r.resize(b.size());
  for (size_t i = 0; i < b.size(); ++i) r[i] -= b[i];
  return r;
}
template <class M>
vec<M> neg(vec<M> a) {
  for (auto& x : a) x = -x;
  return a;
}
template <class M>
vec<M> mul_scalar(const vec<M>& a, M c) {
  vec<M> r(a.size());
  for (size_t i = 0; i < a.size(); ++i) r[i] = a[i] * c;
  return r;
}
template <class M>
vec<M> shift(const vec<M>& a, size_t k, size_t n = SIZE_MAX) {
  vec<M> r(std::min(a.size() + k, n), M());
  for (size_t i = 0; i < a.size() && i + k < r.size(); ++i) r[i + k] = a[i];
  return r;
}
template <class M>
M eval(const vec<M>& a, M x) {
  M r;
  for (size_t i = a.size(); i-- > 0;) r = r * x + a[i];
  return r;
}
template <class M>
vec<M> derivative(const vec<M>& a) {
  if (a.size() <= 1) return {};
  vec<M> r(a.size() - 1);
  for (size_t i = 1; i < a.size(); ++i) r[i - 1] = a[i] * M::from_int(i);
  return r;
}
template <class M>
vec<M> inv_series(size_t n) {
  if (n >= M::mod) throw domain_error("poly::inv_series: length must be < mod");
  vec<M> r(n + 1, M());
  if (n == 0) return r;
  r[1] = M::from_int(1);
  for (size_t i = 2; i <= n; ++i) r[i] = -(M::from_int(M::mod / i) * r[M::mod % i]);
  return r;
}
template <class M>
vec<M> integral(const vec<M>& a) {
  if (a.empty()) return {};
  const vec<M> iv = inv_series<M>(a.size());
  vec<M> r(a.size() + 1);
  for (size_t i = 0; i < a.size(); ++i) r[i + 1] = a[i] * iv[i + 1];
  return r;
}

// The reference's three-prime CRT helpers (crt_convolution.hpp:78-227), which its
// own tests call directly.  Products are exact, so every block size gives the same
// values; the GPU picks its own schedule for each product.
namespace detail {

inline constexpr size_t crt_block_size = size_t(1) << 23;
inline constexpr uint64_t crt_aux_primes[3] = {167772161u, 469762049u, 754974721u};

/// Auxiliary primes that make an exact product of `terms`-term operands mod
/// M::mod unique: the first k whose product exceeds terms * (p - 1)^2.
template <class M>
constexpr size_t crt_prime_count(size_t terms) {
  const unsigned __int128 worst = (unsigned __int128)(M::mod - 1) * (M::mod - 1) * terms;
  unsigned __int128 range = 1;
  for (size_t k = 0; k < 2; ++k) {
    range *= crt_aux_primes[k];
    if (worst < range) return k + 1;
  }
  return 3;
}

/// a * b truncated to `out` terms, zero-padded to exactly `out`.
template <class M, size_t BlockSize = crt_block_size>
vec<M> crt_convolution(const vec<M>& a, const vec<M>& b, size_t out) {
  static_assert(BlockSize > 0 && BlockSize <= crt_block_size);
  vec<M> r = conv(a, b, out);
  r.resize(out);
  return r;
}

/// Coefficients [offset, offset + count) of a * b, a read up to offset + count
/// terms and b up to m (offset defaults to m): the Newton middle product.  As in
/// the reference, the window must lie above every coefficient a cyclic product
/// of next_pow2(2m) points would wrap; there it equals the exact product.
template <class M>
vec<M> crt_middle_product(const vec<M>& a, const vec<M>& b, size_t m, size_t count, size_t offset = SIZE_MAX) {
  if (offset == SIZE_MAX) offset = m;
  vec<M> r(count);
  const size_t la = std::min(a.size(), offset + count), lb = std::min(b.size(), m);
  if (la == 0 || lb == 0) return r;
  const vec<M> full = conv(vec<M>(a.begin(), a.begin() + la), vec<M>(b.begin(), b.begin() + lb), offset + count);
  for (size_t i = 0; i < count && offset + i < full.size(); ++i) r[i] = full[offset + i];
  return r;
}

}  // namespace detail

}  // namespace poly

// The SIMD width the reference's kernels are written for (fastpoly/simd.hpp);
// here the 32 lanes of a warp, the unit the GPU kernels are laid out in.
namespace simd {
inline constexpr unsigned lane = 32;
}  // namespace simd

// ----------------------------------------------------------------- batches

namespace gpu {

/// Many fpx::poly operations in one call (fpx_batch_run).  No counterpart in
/// the reference, whose callers loop over the single functions: queue the
/// operations, run() once, then get() each result, which is exactly the single
/// function's result, or throws exactly its exception.  The input vectors must
/// stay alive and unchanged until run() returns.
template <class M>
class Batch {
 public:
  using vec = poly::vec<M>;
  size_t conv(const vec& a, const vec& b, size_t n = SIZE_MAX) { return add(FPX_OP_CONV, a, &b, n, 0); }
  size_t inv(const vec& a, size_t n) { return add(FPX_OP_INV, a, nullptr, n, 0); }
  size_t log(const vec& a, size_t n) { return add(FPX_OP_LOG, a, nullptr, n, 0); }
  size_t exp(const vec& a, size_t n) { return add(FPX_OP_EXP, a, nullptr, n, 0); }
  size_t sqrt(const vec& a, size_t n) { return add(FPX_OP_SQRT, a, nullptr, n, 0); }
  size_t pow(const vec& a, uint64_t k, size_t n) { return add(FPX_OP_POW, a, nullptr, n, k); }
  size_t divmod(const vec& a, const vec& b) { return add(FPX_OP_DIVMOD, a, &b, 0, 0); }
  size_t size() const { return items_.size(); }

  /// Runs every queued operation; per-operation errors are kept for get().
  void run() {
    std::vector<fpx_job> jobs(items_.size());
    for (size_t i = 0; i < items_.size(); ++i) {
      Item& it = items_[i];
      fpx_job& j = jobs[i];
      j = fpx_job{};
      j.op = it.op;
      j.p = M::mod;
      j.a = limbs(*it.a);
      j.la = it.a->size();
      if (it.b) {
        j.b = limbs(*it.b);
        j.lb = it.b->size();
      }
      j.k = it.k;
      j.n = it.n;
      size_t cap = it.n;
      if (it.op == FPX_OP_CONV) {
        const size_t la = std::min(j.la, it.n), lb = std::min(j.lb, it.n);
        cap = la && lb ? (la > SIZE_MAX - lb ? it.n : std::min(la + lb - 1, it.n)) : 0;
      } else if (it.op == FPX_OP_DIVMOD) {
        cap = j.la;
        it.out2.resize(j.lb);
        j.out2 = limbs(it.out2);
      }
      it.out.resize(cap);
      j.out = limbs(it.out);
    }
    const int rc = fpx_batch_run(context(), jobs.data(), jobs.size(), FPX_REPR_MONTGOMERY);
    if (rc != FPX_OK && rc != FPX_EDOMAIN && rc != FPX_ESIZE && rc != FPX_ELENGTH && rc != FPX_EINVAL)
      check(rc, "gpu::Batch::run");
    for (size_t i = 0; i < items_.size(); ++i) {
      Item& it = items_[i];
      it.status = jobs[i].status;
      it.out.resize(it.status == FPX_OK ? jobs[i].out_len : 0);
      if (it.op == FPX_OP_DIVMOD) it.out2.resize(it.status == FPX_OK ? jobs[i].out2_len : 0);
    }
    ran_ = true;
  }

  /// Result of operation h (the quotient for divmod).
  const vec& get(size_t h) const {
    status_of(h);
    return items_[h].out;
  }
  /// Remainder of divmod operation h.
  const vec& remainder(size_t h) const {
    status_of(h);
    return items_[h].out2;
  }

 private:
  struct Item {
    int op;
    const vec* a;
    const vec* b;
    size_t n;
    uint64_t k;
    vec out, out2;
    int status = FPX_OK;
  };
  size_t add(int op, const vec& a, const vec* b, size_t n, uint64_t k) {
    items_.push_back(Item{op, &a, b, n, k, {}, {}, FPX_OK});
    ran_ = false;
    return items_.size() - 1;
  }
  void status_of(size_t h) const {
    if (!ran_) throw std::logic_error("gpu::Batch: run() has not been called");
    const int rc = items_.at(h).status;
    if (rc == FPX_OK) return;
    if (rc == FPX_EDOMAIN) throw poly::domain_error("gpu::Batch: operation " + std::to_string(h));
    if (rc == FPX_ESIZE) throw ntt_size_error("gpu::Batch: operation " + std::to_string(h));
    if (rc == FPX_ELENGTH) throw std::length_error("gpu::Batch: operation " + std::to_string(h));
    throw std::runtime_error("gpu::Batch: operation " + std::to_string(h) + " failed with status " +
                             std::to_string(rc));
  }
  std::vector<Item> items_;
  bool ran_ = false;
};

}  // namespace gpu

// ------------------------------------------------------------------ Poly

template <class M>
class Poly : public std::vector<M> {
 public:
  using base = std::vector<M>;
  using value_type = M;
  Poly() = default;
  Poly(const base& v) : base(v) {}
  Poly(base&& v) : base(std::move(v)) {}
  Poly(std::initializer_list<M> il) : base(il) {}
  explicit Poly(size_t n, M v = M()) : base(n, v) {}
  using base::size;
  using base::operator[];

  size_t degree() const { return this->empty() ? 0 : this->size() - 1; }
  bool is_zero() const {
    for (const auto& x : *this)
      if (!x.is_zero()) return false;
    return true;
  }
  Poly& trim() { poly::trim(*this); return *this; }
  Poly& resize_(size_t n) { this->resize(n); return *this; }
  Poly operator+(const base& b) const { return poly::add<M>(*this, b); }
  Poly operator-(const base& b) const { return poly::sub<M>(*this, b); }
  Poly operator-() const { return poly::neg<M>(*this); }
  Poly operator*(const base& b) const { return poly::conv<M>(*this, b); }
  Poly operator*(M c) const { return poly::mul_scalar<M>(*this, c); }
  Poly operator<<(size_t k) const { return poly::shift<M>(*this, k); }
  // In place, in the existing storage (poly.hpp:47-50): b may be *this itself,
  // and a longer b grows *this to its length.
  Poly& operator+=(const base& b) { return accumulate<false>(b); }
  Poly& operator-=(const base& b) { return accumulate<true>(b); }
  Poly& operator*=(const base& b) { return *this = poly::conv<M>(*this, b); }
  Poly& operator*=(M c) {
    for (auto& x : *this) x *= c;
    return *this;
  }
  Poly mul(const base& b, size_t n) const { return poly::conv<M>(*this, b, n); }
  Poly derivative() const { return poly::derivative<M>(*this); }
  Poly integral() const { return poly::integral<M>(*this); }
  Poly inv(size_t n) const { return poly::inv<M>(*this, n); }
  Poly log(size_t n) const { return poly::log<M>(*this, n); }
  Poly exp(size_t n) const { return poly::exp<M>(*this, n); }
  Poly sqrt(size_t n) const { return poly::sqrt<M>(*this, n); }
  Poly pow(uint64_t k, size_t n) const { return poly::pow<M>(*this, k, n); }
  std::pair<Poly, Poly> divmod(const base& b) const {
    auto r = poly::divmod<M>(*this, b);
    return {Poly(std::move(r.first)), Poly(std::move(r.second))};
  }
  Poly div(const base& b) const { return poly::div<M>(*this, b); }
  Poly mod(const base& b) const { return poly::mod<M>(*this, b); }
  M eval(M x) const { return poly::eval<M>(*this, x); }
  std::vector<uint32_t> to_ints() const {
    std::vector<uint32_t> r(this->size());
    for (size_t i = 0; i < this->size(); ++i) r[i] = (*this)[i].val();
    return r;
  }
  static Poly from_ints(const std::vector<uint32_t>& v) {
    Poly r(v.size());
    for (size_t i = 0; i < v.size(); ++i) r[i] = M::from_int(v[i]);
    return r;
  }
 private:
  template <bool SUB>
  Poly& accumulate(const base& b) {
    const size_t nb = b.size();
    if (nb > this->size()) this->resize(nb);  // never taken when b is *this
    M* x = this->data();
    const M* y = b.data();
    for (size_t i = 0; i < nb; ++i) x[i] = SUB ? x[i] - y[i] : x[i] + y[i];
    return *this;
  }
};

inline const char* simd_backend() { return "cuda-sm_100a"; }

}  // namespace fpx

#endif  // FPX_DROPIN_FASTPOLY_HPP
