// ib_peak.cu -- FMA-chain microbenchmark for the FP64 / FP32 roofline denominators.
//
// Every thread runs 8 independent FMA chains (enough ILP to cover the pipe
// latency) for a fixed number of iterations; the result is folded into one
// store so the compiler cannot drop the work.  Timed with CUDA events.
#include <cuda_runtime.h>

#include "../../include/intception_b200.h"

namespace {

template <typename T>
__global__ void ib_fma_chains(T* out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (T)-12345.678) out[blockIdx.x] = s;  // never true for these inputs; keeps the chains live
}

}  // namespace

extern "C" int intception_b200_fma_peak(int fp64, int iters, double* flops_per_second) {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return IB_ERR_NODEVICE;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = nsm * 8;
  void* out = nullptr;
  if (cudaMalloc(&out, blocks * sizeof(double)) != cudaSuccess) return IB_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0);
    if (fp64)
      ib_fma_chains<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
    else
      ib_fma_chains<float><<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;  // first launch is warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return IB_ERR_CUDA;
  const double fmas = (double)blocks * threads * iters * 16.0 * 8.0;
  *flops_per_second = 2.0 * fmas / (best * 1e-3);
  return IB_OK;
}
