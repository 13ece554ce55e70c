// peaks.cu - measured 32-bit integer multiply rate, the compute denominator of
// the transform roofline (mulmod count over the INT32 multiply rate).
//
// Every thread runs 8 independent chains of x = mul.hi(x, c1) + x * c2 (one
// mul.hi.u32 and one mad.lo.u32 per step, the two instructions a Shoup or
// Montgomery mulmod is built from); the rate is thread-level multiply
// instructions per second over the whole GPU, timed with CUDA events.
//
// The second probe times the transform's own unit of work: the lazy DIF
// butterfly of the kernels (u + v reduced to [0, 2p), (u - v + 2p) * w by a
// Shoup product: one mul.hi and two mul.lo), 8 independent chains per thread.
// On B200 mul.hi.u32 issues at a quarter and mul.lo / mad.lo at half the warp
// rate on the same pipe, so a butterfly holds that pipe 8 cycles: the rate is
// the compute ceiling of every transform pass.
#include <cstdint>

#include <cuda_runtime.h>

#include "fpx_b200.h"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_imad_rate(uint32_t* sink, uint32_t seed, int iters) {
  uint32_t x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = (threadIdx.x + blockIdx.x * 977u) * (2u * k + 1u) ^ seed;
  const uint32_t c1 = seed | 1u, c2 = seed * 2654435761u + 7u;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = __umulhi(x[k], c1) + x[k] * c2;
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s ^= x[k];
  if (s == 0x9e3779b9u) sink[0] = s;  // keeps the chains live; practically never stores
}

__global__ void __launch_bounds__(256) k_butterfly_rate(uint32_t* sink, uint32_t seed, int iters, uint32_t p) {
  uint32_t u[kChains], v[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) {
    u[k] = ((threadIdx.x + blockIdx.x * 977u) * (2u * k + 1u) ^ seed) % p;
    v[k] = (u[k] * 2654435761u) % p;
  }
  const uint32_t p2 = 2 * p, w = seed % p, wq = (uint32_t)(((uint64_t)w << 32) / p);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
      const uint32_t s = u[k] + v[k];
      const uint32_t d = u[k] - v[k] + p2;
      u[k] = __viaddmin_u32(s, 0u - p2, s);
      v[k] = d * w - __umulhi(d, wq) * p;
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s ^= u[k] + v[k];
  if (s == 0x9e3779b9u) sink[0] = s;
}

// Launches `body(blocks, threads, iters, sink)` once to warm up and once timed.
template <class Body>
int time_probe(int device, double units_per_launch_per_iter, double* per_second, Body body) {
  if (!per_second) return FPX_EINVAL;
  *per_second = 0;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return FPX_EUNSUPPORTED;
  }
  if (device < 0 || device >= n || cudaSetDevice(device) != cudaSuccess) return FPX_EINVAL;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint32_t* sink = nullptr;
  if (cudaMalloc(&sink, 16) != cudaSuccess) return FPX_ENOMEM;
  cudaEvent_t b, e;
  cudaEventCreate(&b);
  cudaEventCreate(&e);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  body(blocks, threads, 64, sink);  // warm-up
  cudaEventRecord(b);
  body(blocks, threads, iters, sink);
  cudaEventRecord(e);
  cudaError_t err = cudaEventSynchronize(e);
  float ms = 0;
  if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, b, e);
  cudaEventDestroy(b);
  cudaEventDestroy(e);
  cudaFree(sink);
  if (err != cudaSuccess || ms <= 0) {
    cudaGetLastError();
    return FPX_ECUDA;
  }
  *per_second = units_per_launch_per_iter * iters * blocks * threads / (ms * 1e-3);
  return FPX_OK;
}

}  // namespace

extern "C" int fpx_measure_butterfly_rate(int device, double* per_second) {
  return time_probe(device, kChains, per_second, [](int blocks, int threads, int iters, uint32_t* sink) {
    k_butterfly_rate<<<blocks, threads>>>(sink, 0x5bd1e995u, iters, 998244353u);
  });
}

extern "C" int fpx_measure_imad_rate(int device, double* per_second) {
  // two multiply instructions per chain step
  return time_probe(device, 2.0 * kChains, per_second, [](int blocks, int threads, int iters, uint32_t* sink) {
    k_imad_rate<<<blocks, threads>>>(sink, 0x5bd1e995u, iters);
  });
}
