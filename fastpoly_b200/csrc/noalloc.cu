// noalloc.cu - fpx_conv_noalloc: the convolution with no device allocation.
//
// Some callers cannot allocate device memory when they need a product: their
// device memory belongs to a host framework's own allocator (often reserved in
// full when the process starts), or they run in a latency-critical loop where
// cudaMalloc's implicit device synchronisation is not acceptable.  For them this
// entry point runs the same kernels as fpx_conv_device, but the two transform
// buffers and the twiddle tables live in one file-scope static device array,
// g_noalloc_scratch, sized for transforms of up to 2^20 points (about 8.3 MiB).
// Every GPU that loads the library holds that array until the process exits.
//
// The caller passes device pointers for the inputs and the output and a stream;
// the call allocates nothing (no cudaMalloc, no cudaFree, no context, no pool).
// The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (and sets the kernels' shared-memory limits); make that
// first call before any stream capture.  The device is the current one: the
// stream must belong to it, and the address is cached per device for the life
// of the process, so no cudaDeviceReset may come between calls.  All calls
// share the array and it keeps the last call's contents: each call rebuilds the
// table entries its transform size reads, and the transform buffers are fully
// written before they are read.  Calls whose work
// overlaps on the GPU (different streams, or different host threads) race on
// the array and must be serialised by the caller.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "engine.h"
#include "field.cuh"
#include "fpx_b200.h"
#include "kernels.h"

namespace {

constexpr int kMaxLog = 20;                       // largest transform: 2^20 points
constexpr size_t kMaxN = size_t(1) << kMaxLog;
constexpr size_t kSmallWords = size_t(2) << 13;   // 2^13 (value, quotient) pairs
constexpr size_t kLoWords = 2 * 256;                // Bailey lo and mid tables: 256 pairs each
constexpr size_t kHiWords = 2 * ((kMaxN >> 16) > 0 ? (kMaxN >> 16) : 1);
// Layout in 32-bit words: two transform buffers, forward and inverse per-prime
// tables, forward Bailey tables (lo, mid, hi), inverse Bailey tables (lo scaled
// by 2^32 / N, mid, hi).
constexpr size_t kOffT1 = 0;
constexpr size_t kOffT2 = kMaxN;
constexpr size_t kOffFwd = 2 * kMaxN;
constexpr size_t kOffInv = kOffFwd + kSmallWords;
constexpr size_t kOffLoF = kOffInv + kSmallWords;
constexpr size_t kOffMidF = kOffLoF + kLoWords;
constexpr size_t kOffHiF = kOffMidF + kLoWords;
constexpr size_t kOffLoI = kOffHiF + kHiWords;
constexpr size_t kOffMidI = kOffLoI + kLoWords;
constexpr size_t kOffHiI = kOffMidI + kLoWords;
constexpr size_t kWords = kOffHiI + kHiWords;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kWords];

struct Roots {
  uint32_t p, pinv;        // modulus and p^-1 mod 2^32 (Montgomery products)
  uint32_t r1;             // 2^32 mod p: Montgomery form of 1
  uint32_t w[14], wi[14];  // Montgomery forms of the primitive 2^lg-th root and its inverse (lg <= 13)
  uint32_t wN, wNi;        // Montgomery forms of the primitive N-th root and its inverse (two-pass sizes)
  uint32_t inv_scale;      // Montgomery form of 2^32 / N mod p
  uint32_t small;          // one-CTA table entries used: min(N, 2^13)
  uint32_t nhi;            // max(1, N / 65536) for two-pass sizes, 0 for one-CTA sizes (no Bailey tables)
};

// Montgomery arithmetic for the table build: every factor is kept in [0, p).
__device__ uint32_t mmul(uint32_t a, uint32_t b, const Roots& r) {
  return fpx_dev::red(fpx_dev::mont(a, b, fpx_dev::Fp{r.p, 2u * r.p, r.pinv}), r.p);
}
// x^e from the Montgomery form of x; returns the canonical residue.
__device__ uint32_t powm_dev(uint32_t xm, uint32_t e, const Roots& r) {
  uint32_t acc = r.r1;
  for (; e; e >>= 1, xm = mmul(xm, xm, r))
    if (e & 1) acc = mmul(acc, xm, r);
  return mmul(acc, 1u, r);
}
__device__ void put(uint32_t* t, size_t i, uint32_t w, uint32_t p) {
  t[2 * i] = w;
  t[2 * i + 1] = (uint32_t)(((uint64_t)w << 32) / p);
}

// Rebuilds the twiddle tables the transform of N points reads: the first
// min(N, 2^13) entries of the per-prime tables and, for two-pass sizes only,
// the Bailey tables.
__global__ void k_noalloc_tables(Roots r) {
  uint32_t* s = g_noalloc_scratch;
  const uint32_t p = r.p;
  const size_t total = r.small + (r.nhi ? 512 + r.nhi : 0);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    if (i < r.small) {
      if (i == 0) {
        put(s + kOffFwd, 0, 1 % p, p);
        put(s + kOffInv, 0, 1 % p, p);
        continue;
      }
      const uint32_t h = 1u << (31 - __clz((unsigned)i));  // entry h + k is w_{2h}^k
      const int lg = 32 - __clz(h);
      const uint32_t k = (uint32_t)i - h;
      put(s + kOffFwd, i, powm_dev(r.w[lg], k, r), p);
      put(s + kOffInv, i, powm_dev(r.wi[lg], k, r), p);
    } else if (i < r.small + 512) {
      const uint32_t y = (uint32_t)(i - r.small);
      if (y < 256) {  // w_N^y, inverse scaled by 2^32 / N
        put(s + kOffLoF, y, powm_dev(r.wN, y, r), p);
        put(s + kOffLoI, y, mmul(powm_dev(r.wNi, y, r), r.inv_scale, r), p);
      } else {        // w_N^(256 y)
        put(s + kOffMidF, y - 256, powm_dev(r.wN, 256u * (y - 256), r), p);
        put(s + kOffMidI, y - 256, powm_dev(r.wNi, 256u * (y - 256), r), p);
      }
    } else {  // w_N^(65536 x)
      const uint32_t x = (uint32_t)(i - r.small - 512);
      put(s + kOffHiF, x, powm_dev(r.wN, 65536u * x, r), p);
      put(s + kOffHiI, x, powm_dev(r.wNi, 65536u * x, r), p);
    }
  }
}

std::mutex g_setup_mu;
uint32_t* g_addr[64];  // device address of g_noalloc_scratch, per device

// Once per device, with that device current: the array's device address and
// the kernels' shared-memory opt-in.  Returns nullptr on failure.
uint32_t* scratch_address(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> g(g_setup_mu);
  if (!g_addr[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    if (fpx::kernels_init() != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    g_addr[dev] = static_cast<uint32_t*>(ptr);
  }
  return g_addr[dev];
}

}  // namespace

extern "C" int fpx_conv_noalloc(uint32_t p, const uint32_t* d_a, size_t la, const uint32_t* d_b, size_t lb, size_t n,
                                uint32_t* d_out, size_t* out_len, void* stream) {
  if (!out_len) return FPX_EINVAL;
  *out_len = 0;
  if (la == 0 || lb == 0 || n == 0) return FPX_OK;
  // An error already pending from the caller's own work is left pending for the
  // caller and nothing is launched: every error seen below is this call's.
  if (cudaPeekAtLastError() != cudaSuccess) return FPX_ECUDA;
  if (!d_a || !d_b || !d_out) return FPX_EINVAL;
  if (!(p & 1u) || p >= (1u << 30) || !fpx::is_prime(p)) return FPX_EINVAL;
  la = la < n ? la : n;
  lb = lb < n ? lb : n;
  if (la > SIZE_MAX - (lb - 1)) return FPX_ELENGTH;
  const size_t full = la + lb - 1, outn = full < n ? full : n;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if ((la < lb ? la : lb) <= 40) {  // direct product (convolution.hpp:33-95): no scratch at all
    const bool swap = la > lb;
    if (fpx::launch_direct_product(p, swap ? d_b : d_a, swap ? lb : la, swap ? d_a : d_b, swap ? la : lb, 0, outn,
                                   d_out, 0, s) != cudaSuccess)
      return FPX_ECUDA;
    *out_len = outn;
    return FPX_OK;
  }
  int logN = 0;
  while ((size_t(1) << logN) < full) ++logN;
  if (logN > kMaxLog || logN > fpx::v2_of(p)) return FPX_ESIZE;  // beyond the static array / the prime's roots
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FPX_ECUDA;
  uint32_t* base = scratch_address(dev);
  if (!base) return FPX_ECUDA;

  Roots r{};
  r.p = p;
  r.pinv = fpx_dev::inv_mod_2_32(p);
  const uint32_t R = (uint32_t)((uint64_t(1) << 32) % p);
  r.r1 = R;
  auto to_mont = [&](uint32_t x) { return (uint32_t)((uint64_t)x * R % p); };
  const uint32_t g = fpx::primitive_root(p);
  for (int lg = 1; lg <= 13 && lg <= fpx::v2_of(p); ++lg) {
    const uint32_t w = fpx::powm(g, (p - 1) >> lg, p);
    r.w[lg] = to_mont(w);
    r.wi[lg] = to_mont(fpx::invm(w, p));
  }
  const uint32_t N = 1u << logN;
  const uint32_t scale = (uint32_t)((uint64_t)fpx::invm(N % p, p) * R % p);  // undoes the Montgomery pointwise
  r.small = N < (1u << 13) ? N : (1u << 13);
  if (logN > 13) {
    const uint32_t wN = fpx::powm(g, (p - 1) >> logN, p);
    r.wN = to_mont(wN);
    r.wNi = to_mont(fpx::invm(wN, p));
    r.inv_scale = to_mont(scale);
    r.nhi = (N >> 16) > 0 ? (N >> 16) : 1;
  }
  const unsigned blocks = (r.small + (r.nhi ? 512 + r.nhi : 0) + 255) / 256;
  k_noalloc_tables<<<blocks < 64 ? blocks : 64, 256, 0, s>>>(r);
  if (cudaGetLastError() != cudaSuccess) return FPX_ECUDA;

  fpx::PrimeTables pt;
  pt.p = p;
  pt.max_log = fpx::v2_of(p);
  pt.small_log = 13;
  pt.fwd = reinterpret_cast<const fpx::Tw2*>(base + kOffFwd);
  pt.inv = reinterpret_cast<const fpx::Tw2*>(base + kOffInv);
  pt.q1 = (uint32_t)((uint64_t(1) << 32) / p);
  const bool square = d_a == d_b && la == lb;
  cudaError_t e;
  if (logN <= fpx::small_kernel_max_log()) {
    fpx::SmallJob j;
    j.x = fpx::InOp{d_a, (uint32_t)la, 0};
    j.ymode = square ? 3 : 1;
    if (!square) j.y = fpx::InOp{d_b, (uint32_t)lb, 0};
    j.epi.out = d_out;
    j.epi.lo = 0;
    j.epi.hi = (uint32_t)outn;
    j.epi.scale = fpx::Tw2{scale, (uint32_t)(((uint64_t)scale << 32) / p)};
    e = fpx::launch_small(pt, logN, j, s);
  } else {
    fpx::BigTables bt;
    bt.logN = logN;
    bt.logC = 12;
    bt.logR = logN - 12;
    bt.lo_fwd = reinterpret_cast<const fpx::Tw2*>(base + kOffLoF);
    bt.mid_fwd = reinterpret_cast<const fpx::Tw2*>(base + kOffMidF);
    bt.hi_fwd = reinterpret_cast<const fpx::Tw2*>(base + kOffHiF);
    bt.lo_inv_r = reinterpret_cast<const fpx::Tw2*>(base + kOffLoI);
    bt.mid_inv = reinterpret_cast<const fpx::Tw2*>(base + kOffMidI);
    bt.hi_inv = reinterpret_cast<const fpx::Tw2*>(base + kOffHiI);
    uint32_t* t1 = base + kOffT1;
    uint32_t* t2 = base + kOffT2;
    fpx::InOp ins[2] = {fpx::InOp{d_a, (uint32_t)la, 0}, fpx::InOp{d_b, (uint32_t)lb, 0}};
    uint32_t* outs[2] = {t1, t2};
    e = fpx::launch_colfwd(pt, bt, square ? 1 : 2, ins, outs, s);
    if (e == cudaSuccess) e = fpx::launch_rows(pt, bt, t1, square ? nullptr : t2, square ? 3 : 1, nullptr, 1, 1, s);
    fpx::Epi epi;
    epi.out = d_out;
    epi.lo = 0;
    epi.hi = (uint32_t)outn;
    if (e == cudaSuccess) e = fpx::launch_colinv(pt, bt, t1, 1, epi, s);
  }
  if (e != cudaSuccess) return FPX_ECUDA;
  *out_len = outn;
  return FPX_OK;
}
