// peaks.cu - measured 32-bit integer multiply rate, the compute denominator of
// the transform roofline (mulmod count over the INT32 multiply rate).
//
// Every thread runs 8 independent chains of x = mul.hi(x, c1) + x * c2 (one
// mul.hi.u32 and one mad.lo.u32 per step, the two instructions a Shoup or
// Montgomery mulmod is built from); the rate is thread-level multiply
// instructions per second over the whole GPU, timed with CUDA events.
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

}  // namespace

extern "C" int fpx_measure_imad_rate(int device, double* per_second) {
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
  k_imad_rate<<<blocks, threads>>>(sink, 12345u, 64);  // warm-up
  cudaEventRecord(b);
  k_imad_rate<<<blocks, threads>>>(sink, 0x5bd1e995u, iters);
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
  const double instr = 2.0 * kChains * (double)iters * blocks * threads;
  *per_second = instr / (ms * 1e-3);
  return FPX_OK;
}
