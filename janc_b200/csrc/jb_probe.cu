// Measurement helper: a float64 FMA throughput kernel used to measure the
// FP64 peak of the device the benchmark runs on (the denominator of the
// compute roofline).  Each thread runs 8 independent FMA chains.
#include <cuda_runtime.h>

namespace {
__global__ void k_fp64_fma(int iters, double seed, double* out) {
  double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
  double a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const double b = 0.999999, c = 1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
      a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
  }
  double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 0.1234567) out[blockIdx.x] = s;  // keeps the chains live
}
}  // namespace

extern "C" int jb_probe_fp64_fma(int blocks, int iters, double* scratch, void* stream) {
  if (blocks <= 0 || iters <= 0 || !scratch) return 1;
  k_fp64_fma<<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 1.0, scratch);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
