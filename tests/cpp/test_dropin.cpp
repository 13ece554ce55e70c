// Drop-in check: reference-style code compiled against include/fpx/fastpoly.hpp
// runs on the GPU library and satisfies the reference's own contracts
// (tests/test_prime_poly.cpp:315-362, tests/test_poly.cpp:160-345), checked
// against O(n^2) definitions written here.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "fpx/fastpoly.hpp"

using namespace fpx;

static int failures = 0;
#define CHECK(c)                                                       \
  do {                                                                 \
    if (!(c)) {                                                        \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);         \
      ++failures;                                                      \
    }                                                                  \
  } while (0)

template <class M>
std::vector<M> naive(const std::vector<M>& a, const std::vector<M>& b, size_t n) {
  if (a.empty() || b.empty() || n == 0) return {};
  std::vector<M> r(std::min(n, a.size() + b.size() - 1));
  for (size_t i = 0; i < a.size(); ++i)
    for (size_t j = 0; j < b.size() && i + j < r.size(); ++j) r[i + j] += a[i] * b[j];
  return r;
}

template <class M>
std::vector<M> rnd(size_t n, std::mt19937_64& g) {
  std::vector<M> a(n);
  for (auto& x : a) x = M::from_int(g() % M::mod);
  return a;
}

template <class M>
void suite(const char* name) {
  std::mt19937_64 g(7);
  for (size_t la : {size_t(1), size_t(39), size_t(41), size_t(300), size_t(5000)}) {
    auto a = rnd<M>(la, g), b = rnd<M>(la + 13, g);
    CHECK(poly::conv(a, b) == naive(a, b, SIZE_MAX));
    CHECK(poly::conv(a, b, la) == naive(a, b, la));
  }
  for (size_t n : {size_t(1), size_t(33), size_t(257), size_t(3000)}) {
    auto a = rnd<M>(n, g);
    a[0] = M::from_int(1);
    auto ia = poly::inv(a, n);
    auto unit = naive(a, ia, n);
    CHECK(unit[0] == M::from_int(1));
    bool zero = true;
    for (size_t i = 1; i < n; ++i) zero = zero && unit[i].is_zero();
    CHECK(zero);
    if (n <= M::mod) {
      auto l = poly::log(a, n);
      CHECK(poly::exp(l, n) == a);
    }
    auto sq = naive(a, a, n);
    auto r = poly::sqrt(sq, n);
    CHECK(naive(r, r, n) == sq);
    auto p3 = poly::pow(a, 3, n);
    CHECK(p3 == naive(naive(a, a, n), a, n));
  }
  // divmod round trip (tests/test_poly.cpp:316-344)
  auto bdiv = rnd<M>(143, g);
  bdiv.back() = M::from_int(1);
  auto q0 = rnd<M>(177, g);
  q0.back() = M::from_int(1);
  auto rem = rnd<M>(141, g);
  poly::trim(rem);
  auto prod = naive(bdiv, q0, SIZE_MAX);
  auto dividend = poly::add(prod, rem);
  auto [q, r] = poly::divmod(dividend, bdiv);
  CHECK(q == q0);
  CHECK(r == rem);
  // errors
  bool threw = false;
  try { (void)poly::inv(std::vector<M>{M(), M::from_int(1)}, 8); } catch (const poly::domain_error&) { threw = true; }
  CHECK(threw);
  // one batch of the same operations: every result equals the single call's
  {
    gpu::Batch<M> batch;
    auto x = rnd<M>(900, g), y = rnd<M>(1300, g), e0 = rnd<M>(700, g), l1 = rnd<M>(600, g);
    x[0] = M::from_int(3);
    e0[0] = M();
    l1[0] = M::from_int(1);
    const auto bad = std::vector<M>{M(), M::from_int(1)};
    const auto sq = naive(x, x, 900);  // batch inputs must outlive run()
    const size_t hc = batch.conv(x, y), ht = batch.conv(x, y, 500), hi = batch.inv(x, 1000);
    const size_t he = batch.exp(e0, 800), hl = batch.log(l1, 600), hq = batch.divmod(y, x);
    const size_t hp = batch.pow(x, 5, 700), hs = batch.sqrt(sq, 900), hb = batch.inv(bad, 8);
    batch.run();
    CHECK(batch.get(hc) == poly::conv(x, y));
    CHECK(batch.get(ht) == poly::conv(x, y, 500));
    CHECK(batch.get(hi) == poly::inv(x, 1000));
    CHECK(batch.get(he) == poly::exp(e0, 800));
    CHECK(batch.get(hl) == poly::log(l1, 600));
    const auto [bq, br] = poly::divmod(y, x);
    CHECK(batch.get(hq) == bq);
    CHECK(batch.remainder(hq) == br);
    CHECK(batch.get(hp) == poly::pow(x, 5, 700));
    CHECK(batch.get(hs) == poly::sqrt(sq, 900));
    bool batch_threw = false;
    try { (void)batch.get(hb); } catch (const poly::domain_error&) { batch_threw = true; }
    CHECK(batch_threw);
  }
  std::printf("  %s ok\n", name);
}

int main() {
  suite<mod998244353>("998244353");
  suite<mod1000000007>("1000000007");
  suite<ModInt<2147483647u>>("2147483647");
  {  // tests/test_prime_poly.cpp:346-360 (Poly method API)
    using M = mod1000000007;
    const Poly<M> a{1, 2, 3}, b{1, 1};
    CHECK(((a + b) - b) == a);
    CHECK((a * (-M(1))) == -a);
    CHECK((a << 2)[2] == a[0]);
    CHECK(a.eval(M(2)) == M(17));
    CHECK(a.integral().derivative() == a);
    CHECK(a.inv(257).size() == 257u);
    auto padded = a;
    padded.resize(257);
    CHECK(a.log(257).exp(257) == padded);
    const auto square = a.mul(a, 257);
    CHECK(square.sqrt(257).mul(square.sqrt(257), 257) == a.pow(2, 257));
    CHECK((a * b).div(b) == a);
    CHECK((a * b).mod(b).empty());
  }
  {  // GPU NttPlan keeps the reference's permutation: constant -> impulse at 0 (test_ntt.cpp:223-235)
    using M = mod998244353;
    const uint32_t n = 64;
    auto plan = NttPlan<M>::get(n);
    std::vector<uint32_t> a(n, M::from_int(5).raw_val());
    plan->forward(a.data());
    int nonzero = 0;
    for (auto x : a) nonzero += x != 0;
    CHECK(nonzero == 1);
    CHECK(a[0] == M::from_int(5ull * n).raw_val());
    plan->inverse(a.data());
    CHECK(a[7] == M::from_int(5).raw_val());
    bool threw = false;
    try { (void)NttPlan<M>::get(1u << 24); } catch (const ntt_size_error&) { threw = true; }
    CHECK(threw);
    // window contracts (tests/test_ntt.cpp:289-336): a prefix forward equals the
    // zero-padded forward, the prefix / high-half inverses give back the window
    std::mt19937_64 g(11);
    const uint32_t m = 1024;
    const auto& big = NttPlan<M>::get_ref(m);
    CHECK(&big == &NttPlan<M>::get_ref(m) && big.log_size() == 10);
    std::vector<uint32_t> x(m), padded(m, 0);
    for (uint32_t i = 0; i < 300; ++i) x[i] = padded[i] = M::from_int(g() % M::mod).raw_val();
    const auto orig = padded;
    for (uint32_t i = 300; i < m; ++i) x[i] = 12345;  // garbage past the prefix
    big.forward_prefix(x.data(), 300);
    big.forward_lazy(padded.data());
    CHECK(x == padded);
    auto lo = x, hi = x;
    big.inverse_prefix(lo.data(), 300);
    big.inverse_highhalf(hi.data());
    bool lo_ok = true, hi_ok = true;
    for (uint32_t i = 0; i < 300; ++i) lo_ok = lo_ok && lo[i] == orig[i];
    CHECK(lo_ok);
    for (uint32_t i = m / 2; i < m; ++i) hi_ok = hi_ok && hi[i] == orig[i];
    CHECK(hi_ok);
    threw = false;
    try { big.forward_prefix(x.data(), m + 1); } catch (const ntt_size_error&) { threw = true; }
    CHECK(threw);
  }
  {  // scratch statistics of the device pool (memory.hpp:21-26, 252-258)
    const auto st = scratch_memory_stats();
    CHECK(st.system_allocations > 0);
    release_scratch_memory();
    CHECK(scratch_memory_stats().cached_bytes == 0);
  }
  std::printf(failures ? "FAILED (%d)\n" : "all drop-in checks passed\n", failures);
  return failures ? 1 : 0;
}
