// The device's FP64 fused multiply-add rate, measured: the denominator of the
// FP64 roofline the benchmark reports beside the HBM one.  No counterpart in
// the reference, which measures nothing of the machine.
//
// Every thread runs eight independent chains x = x * a + b (one DFMA each,
// two flops), long enough that launch and tail are noise; the grid fills
// every SM many times over.  The chains' results are stored only when a
// runtime flag the host never sets is set, so the compiler keeps them.
#include <string>

#include "pgb200.h"

extern "C" int pgb_internal_fail(int code, const char *msg);

namespace {

constexpr int kChains = 8;

__global__ void k_fma_chains(double *sink, const double a, const double b, const int iters, const int store) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) x[c] = 1e-3 * (threadIdx.x + c);
  for (int n = 0; n < iters; n++) {
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += x[c];
  if (store) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

int cuda_fail(cudaError_t e, const char *what) {
  return pgb_internal_fail(PGB_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

}  // namespace

extern "C" int pgb_fp64_fma_rate(double *tflops) {
  if (!tflops) return pgb_internal_fail(PGB_ERR_ARG, "null argument");
  int dev = 0, sms = 148;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * 16, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // a contraction factor just below one keeps the chains finite and normal
  const double a = 0.999999, b = 1e-7;
  float best = 1e30f;
  for (int rep = 0; rep < 6; rep++) {
    cudaEventRecord(e0);
    k_fma_chains<<<blocks, threads>>>(nullptr, a, b, iters, 0);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) break;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;  // the first is the warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(e, "FP64 rate");
  const double flops = 2.0 * kChains * (double)iters * threads * (double)blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return PGB_OK;
}
