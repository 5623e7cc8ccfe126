// Integer-pipe throughput probe: the denominators of the INT roofline the dense
// kernels are reported against.  No counterpart in the reference.  It is a bench
// instrument, built into its own library (_lib/libde_probe.so), not part of the
// matcher's C ABI:
//
//   int de_int_probe(int op, int trips, void* stream, float* ms, double* lane_ops)
//
// runs op 0 add.u32, 1 lop3.b32, 2 shf (funnel rotate), 3 mad.lo.u32 or 4 popc.b32 as
// 8 independent chains per thread on every SM for `trips` loop trips; *ms is the
// CUDA-event time of the timed launch and *lane_ops the warp-lane operations it
// executed, so lane_ops / (ms * SM clock * SMs) is the op's rate per SM clock.
//
// Each thread runs 8 independent accumulator chains of one instruction class, 16 x 8
// instructions per loop trip, written as inline PTX so the chains are neither folded
// nor merged; the grid fills every SM (8 CTAs of 256 threads each).  The result is
// kept live through a store that never happens for any real input, so the loop
// cannot be removed.  Rates are warp-lane operations per SM clock.

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/doubleeye_b200.h"

namespace {

template <int OP>
__device__ __forceinline__ uint32_t probe_op(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  if constexpr (OP == 0) {
    asm volatile("add.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  } else if constexpr (OP == 1) {
    asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  } else if constexpr (OP == 2) {
    asm volatile("shf.l.wrap.b32 %0, %1, %1, 7;" : "=r"(r) : "r"(a));
  } else if constexpr (OP == 3) {
    asm volatile("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  } else {
    asm volatile("popc.b32 %0, %1;" : "=r"(r) : "r"(a));
  }
  return r;
}

template <int OP>
__global__ void __launch_bounds__(256) k_int_probe(uint32_t* sink, int trips, uint32_t seed) {
  uint32_t a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + threadIdx.x * 8u + uint32_t(i);
  const uint32_t b = seed * 3u + 1u, c = seed ^ 0x9e3779b9u;
  for (int t = 0; t < trips; ++t) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = probe_op<OP>(a[i], b, c);
  }
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) r ^= a[i];
  if (r == seed + 0x7fffffffu && sink) sink[blockIdx.x] = r;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int de_int_probe(int op, int trips, void* stream, float* ms, double* lane_ops) {
  if (op < 0 || op > 4 || trips < 1 || !ms || !lane_ops) return DE_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return DE_ERR_CUDA;
  const int blocks = nsm * 8, threads = 256;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return DE_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return DE_ERR_CUDA; }
  auto launch = [&](int n) {
    switch (op) {
      case 0: k_int_probe<0><<<blocks, threads, 0, s>>>(nullptr, n, 12345u); break;
      case 1: k_int_probe<1><<<blocks, threads, 0, s>>>(nullptr, n, 12345u); break;
      case 2: k_int_probe<2><<<blocks, threads, 0, s>>>(nullptr, n, 12345u); break;
      case 3: k_int_probe<3><<<blocks, threads, 0, s>>>(nullptr, n, 12345u); break;
      default: k_int_probe<4><<<blocks, threads, 0, s>>>(nullptr, n, 12345u); break;
    }
  };
  launch(trips / 8 + 1);                              // warm-up
  cudaEventRecord(e0, s);
  launch(trips);
  cudaEventRecord(e1, s);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return DE_ERR_CUDA;
  *ms = t;
  *lane_ops = double(blocks) * threads * double(trips) * 16.0 * 8.0;
  return DE_OK;
}
