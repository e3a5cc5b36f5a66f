// ov_peak.cu - FMA throughput microbenchmark: the FP32 / FP64 roofline
// denominators of the Biot-Savart kernels, measured on the running GPU; and
// the accuracy check of the refined FP64 reciprocal square root and
// reciprocal the direct sum uses.
// Eight independent FMA chains per thread keep the pipes full; the result is
// written so the chains are not eliminated.
#include <string.h>

#include "openvort_b200.h"
#include "ov_internal.h"

static double __longlong_as_double_host(unsigned long long v) {
  double d;
  memcpy(&d, &v, sizeof(d));
  return d;
}

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

// refined reciprocal square root and reciprocal (rsqrt_nr, rcp_nr) against
// IEEE sqrt and division, over x = 2^(e / 64) for e in [-8192, 8192): the
// largest relative differences, in ulps of the IEEE result (atomicMax on the
// bit patterns of non-negative doubles orders them as numbers)
__global__ void k_check_fast_math(unsigned long long* worst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 16384) return;
  const double x = exp2((i - 8192) / 64.0);
  const double a = 1.0 / sqrt(x), b = rsqrt_nr(x);
  const double c = 1.0 / x, d = rcp_nr(x);
  const double ulp_a = a * 0x1p-52, ulp_c = c * 0x1p-52;
  atomicMax(&worst[0], (unsigned long long)__double_as_longlong(fabs(b - a) / ulp_a));
  atomicMax(&worst[1], (unsigned long long)__double_as_longlong(fabs(d - c) / ulp_c));
}

}  // namespace

extern "C" int ov_check_fast_math(double* rsqrt_ulps, double* rcp_ulps) {
  ov_clear_error();
  if (!rsqrt_ulps || !rcp_ulps) return OV_ERR_INVALID;
  if (ov_init(0) != OV_OK) return ov_last_error();
  unsigned long long* d = nullptr;
  unsigned long long h[2] = {0, 0};
  if (!ov_cuda_ok(cudaMalloc(&d, sizeof(h)), "cudaMalloc")) return ov_last_error();
  bool ok = ov_cuda_ok(cudaMemset(d, 0, sizeof(h)), "cudaMemset");
  if (ok) {
    k_check_fast_math<<<64, 256>>>(d);
    OV_LAUNCHED();
    ok = ov_cuda_ok(cudaGetLastError(), "k_check_fast_math") &&
         ov_cuda_ok(cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost), "cudaMemcpy");
  }
  cudaFree(d);
  if (!ok) return ov_last_error();
  *rsqrt_ulps = __longlong_as_double_host(h[0]);
  *rcp_ulps = __longlong_as_double_host(h[1]);
  return OV_OK;
}

extern "C" int ov_measure_fma_peak(int fp64, double* tflops) {
  ov_clear_error();
  if (!tflops) return OV_ERR_INVALID;
  if (ov_init(0) != OV_OK) return ov_last_error();
  bool ok = fp64 ? run<double>(tflops) : run<float>(tflops);
  return ok ? OV_OK : ov_last_error();
}
