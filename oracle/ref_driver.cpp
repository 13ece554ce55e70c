// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-callable shim over the UNMODIFIED reference library (xcx0902/fastpoly,
// header-only C++20), compiled from the reference's own headers by
// oracle/Makefile into oracle/_ref/.  It serves two purposes:
//   * pinning the C restatement (oracle/fpx_oracle.c) against the reference
//     itself on the same inputs (tests/golden/make_golden.py writes the
//     reference's outputs that tests/test_oracle_golden.py checks the oracle
//     against) and the GPU tests that call the reference directly;
//   * the timed CPU baseline (bench.py --impl reference / cpu_baseline).
// Nothing here is part of the product library.
//
// Every entry point takes and returns canonical residues; the conversion to the
// reference's Montgomery limbs (Mont::from_int / val, modint.hpp:83-96) happens
// outside the timed region of the fpr_time_* functions.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "fastpoly/fastpoly.hpp"

namespace {

enum { FPR_OK = 0, FPR_EDOMAIN = 1, FPR_ESIZE = 2, FPR_ELENGTH = 3, FPR_EUNSUPPORTED = 5, FPR_EOTHER = 6 };
enum Op { OP_CONV = 0, OP_INV = 1, OP_LOG = 2, OP_EXP = 3, OP_SQRT = 4, OP_POW = 5, OP_DIVMOD = 6,
          OP_NTT_FWD = 7, OP_NTT_INV = 8, OP_CRT64 = 9 };

template <class M>
std::vector<M> load(const uint32_t* v, size_t n) {
  std::vector<M> r(n);
  for (size_t i = 0; i < n; ++i) r[i] = M::from_int(v[i]);
  return r;
}
template <class M>
size_t store(const std::vector<M>& r, uint32_t* out) {
  for (size_t i = 0; i < r.size(); ++i) out[i] = r[i].val();
  return r.size();
}

struct Args {
  const uint32_t* a; size_t la;
  const uint32_t* b; size_t lb;
  size_t n; uint64_t k;
};

// Runs one operation on already-converted inputs; returns outputs in Montgomery form.
template <class M>
struct Runner {
  std::vector<M> a, b;
  size_t n; uint64_t k;
  std::vector<M> r1, r2;
  void run(int op) {
    namespace P = fpx::poly;
    switch (op) {
      case OP_CONV: r1 = (n == SIZE_MAX) ? P::conv(a, b) : P::conv(a, b, n); break;
      case OP_INV: r1 = P::inv(a, n); break;
      case OP_LOG: r1 = P::log(a, n); break;
      case OP_EXP: r1 = P::exp(a, n); break;
      case OP_SQRT: r1 = P::sqrt(a, n); break;
      case OP_POW: r1 = P::pow(a, k, n); break;
      case OP_DIVMOD: { auto qr = P::divmod(a, b); r1 = std::move(qr.first); r2 = std::move(qr.second); break; }
      case OP_CRT64: r1 = P::detail::crt_convolution<M, 64>(a, b, n); break;
      case OP_NTT_FWD:
      case OP_NTT_INV: {
        r1 = a;
        const auto& plan = fpx::NttPlan<M>::get_ref(static_cast<uint32_t>(a.size()));
        auto* p = reinterpret_cast<uint32_t*>(r1.data());
        if (op == OP_NTT_FWD) plan.forward(p); else plan.inverse(p);
        break;
      }
      default: throw std::invalid_argument("op");
    }
  }
};

template <class M>
int dispatch(int op, const Args& x, uint32_t* o1, size_t* l1, uint32_t* o2, size_t* l2,
             int reps, int threads, double* times) {
  try {
    Runner<M> base;
    base.a = load<M>(x.a, x.la);
    base.b = load<M>(x.b, x.lb);
    base.n = x.n; base.k = x.k;
    if (threads <= 1) {
      for (int r = 0; r < reps; ++r) {
        base.r1.clear(); base.r2.clear();
        const auto t0 = std::chrono::steady_clock::now();
        base.run(op);
        const auto t1 = std::chrono::steady_clock::now();
        if (times) times[r] = std::chrono::duration<double>(t1 - t0).count();
      }
    } else {
      // Independent calls on `threads` host threads (the library is thread-safe
      // across calls): whole-machine throughput of the same single-call work.
      std::vector<Runner<M>> work(static_cast<size_t>(threads), base);
      base.run(op);  // warm plans once
      for (int r = 0; r < reps; ++r) {
        std::atomic<int> ready{0};
        std::atomic<bool> go{false};
        std::vector<std::thread> pool;
        std::chrono::steady_clock::time_point t0;
        for (int t = 0; t < threads; ++t)
          pool.emplace_back([&, t] {
            ready.fetch_add(1);
            while (!go.load()) std::this_thread::yield();
            work[static_cast<size_t>(t)].run(op);
          });
        while (ready.load() != threads) std::this_thread::yield();
        t0 = std::chrono::steady_clock::now();
        go.store(true);
        for (auto& th : pool) th.join();
        const auto t1 = std::chrono::steady_clock::now();
        if (times) times[r] = std::chrono::duration<double>(t1 - t0).count();
      }
    }
    if (o1 && l1) *l1 = store(base.r1, o1);
    if (o2 && l2) *l2 = store(base.r2, o2);
    return FPR_OK;
  } catch (const fpx::poly::domain_error&) {
    return FPR_EDOMAIN;
  } catch (const fpx::ntt_size_error&) {
    return FPR_ESIZE;
  } catch (const std::length_error&) {
    return FPR_ELENGTH;
  } catch (...) {
    return FPR_EOTHER;
  }
}

// The reference's own aliases where it defines one (modint.hpp:195-205),
// otherwise ModInt<p> (automatic primitive root, modint.hpp:28-52, 203-204).
#define FPR_MODULI(X)                                  \
  X(998244353u, fpx::mod998244353)                     \
  X(167772161u, fpx::mod167772161)                     \
  X(469762049u, fpx::mod469762049)                     \
  X(754974721u, fpx::mod754974721)                     \
  X(1004535809u, fpx::mod1004535809)                   \
  X(1224736769u, fpx::mod1224736769)                   \
  X(1000000007u, fpx::mod1000000007)                   \
  X(2147483647u, fpx::ModInt<2147483647u>)             \
  X(1073479681u, (fpx::Mont<1073479681u, 11>))         \
  X(2013265921u, (fpx::Mont<2013265921u, 31>))         \
  X(2u, fpx::ModInt<2u>)                               \
  X(3u, fpx::ModInt<3u>)                               \
  X(17u, fpx::ModInt<17u>)                             \
  X(97u, fpx::ModInt<97u>)                             \
  X(193u, fpx::ModInt<193u>)                           \
  X(257u, fpx::ModInt<257u>)                           \
  X(641u, fpx::ModInt<641u>)                           \
  X(100003u, fpx::ModInt<100003u>)

template <class T> struct unparen;
template <class T> struct unparen<void(T)> { using type = T; };

}  // namespace

extern "C" {

// Supported moduli (for tests to enumerate); returns the count, writes up to cap.
size_t fpr_moduli(uint32_t* out, size_t cap) {
  size_t i = 0;
#define X(P, T) if (i < cap) out[i] = P; ++i;
  FPR_MODULI(X)
#undef X
  return i;
}

const char* fpr_simd_backend(void) { return fpx::simd_backend(); }

// Runs `op` `reps` times on `threads` threads (reps >= 1); times[] gets the
// wall time of each repetition (seconds); o1/o2 get the last outputs.
int fpr_run(int op, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb,
            size_t n, uint64_t k, uint32_t* o1, size_t* l1, uint32_t* o2, size_t* l2,
            int reps, int threads, double* times) {
  Args x{a, la, b, lb, n, k};
  if (reps < 1) reps = 1;
  switch (p) {
#define X(P, T) case P: return dispatch<typename unparen<void(T)>::type>(op, x, o1, l1, o2, l2, reps, threads, times);
    FPR_MODULI(X)
#undef X
    default: return FPR_EUNSUPPORTED;
  }
}

}  // extern "C"
