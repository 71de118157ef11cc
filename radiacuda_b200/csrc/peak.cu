// peak.cu -- FP64 / FP32 pipe microbenchmarks.
//
// The measured-peaks file of this pool holds HBM copy bandwidth and cuBLAS
// BF16 throughput only; the assembly and field kernels are bound by the FP64
// (or FP32) pipes, so their roofline denominators are measured here: long
// chains of independent fused multiply-adds, 8 chains per thread, enough
// warps to fill every SM.
#include "internal.cuh"

namespace rb {

template <typename T>
__global__ void __launch_bounds__(256) fma_loop_kernel(T *out, int iters, T a, T b)
{
  T x0 = threadIdx.x * T(1e-7), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
  T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-12345.678)) out[0] = s;  // never true; keeps the chains alive
}

}  // namespace rb

using namespace rb;

extern "C" RADB200_API int radb200_measure_fma_peak(int fp64, double *tflops)
{
  int dev = 0, sms = 0;
  RB_CUDA(cudaGetDevice(&dev));
  RB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DBuf o;
  RB_TRY(o.alloc(16));
  const int blocks = sms * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  RB_CUDA(cudaEventCreate(&e0));
  RB_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    RB_CUDA(cudaEventRecord(e0));
    if (fp64) fma_loop_kernel<double><<<blocks, threads>>>(o.as<double>(), iters, 0.999999, 1e-9);
    else fma_loop_kernel<float><<<blocks, threads>>>(o.as<float>(), iters, 0.999999f, 1e-9f);
    RB_TRY(check_launch("fma_loop_kernel"));
    RB_CUDA(cudaEventRecord(e1));
    RB_CUDA(cudaEventSynchronize(e1));
    float ms;
    RB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return 0;
}
