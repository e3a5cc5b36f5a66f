// ov_peak.cu - FMA throughput microbenchmark: the FP32 / FP64 roofline
// denominators of the Biot-Savart kernels, measured on the running GPU.
// Eight independent FMA chains per thread keep the pipes full; the result is
// written so the chains are not eliminated.
#include "openvort_b200.h"
#include "ov_internal.h"

namespace {

template <class T>
__global__ void k_fma(T* out, int iters, T a, T b) {
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
    x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
      x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
  }
  T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (T)-1.2345) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <class T>
bool run(double* tflops) {
  int dev = 0, sms = 0;
  OV_TRY_CUDA(cudaGetDevice(&dev));
  OV_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 256, blocks = sms * 8;
  const int iters = sizeof(T) == 8 ? 1024 : 2048;
  T* out = nullptr;
  OV_TRY_CUDA(cudaMalloc(&out, sizeof(T) * threads * blocks));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  T a = (T)0.999999, b = (T)1e-7;
  k_fma<T><<<blocks, threads>>>(out, iters, a, b);   // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    k_fma<T><<<blocks, threads>>>(out, iters, a, b);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (!ov_cuda_ok(err, "k_fma")) return false;
  double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return true;
}

}  // namespace

extern "C" int ov_measure_fma_peak(int fp64, double* tflops) {
  ov_clear_error();
  if (!tflops) return OV_ERR_INVALID;
  if (ov_init(0) != OV_OK) return ov_last_error();
  bool ok = fp64 ? run<double>(tflops) : run<float>(tflops);
  return ok ? OV_OK : ov_last_error();
}
