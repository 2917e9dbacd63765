// mpc_peaks.cu -- microbenchmarks of the FP32 FMA pipe and the MUFU (SFU)
// pipe, the denominators of the fused kernels' roofline.  Each thread runs
// eight independent dependency chains so the pipes, not latency, bound the rate.

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/montepath_cuda.h"
#include "mpc_runtime.h"

namespace {

__global__ void __launch_bounds__(256) fma_peak_kernel(float* out, int iters) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-6f, a2 = a0 + 2e-6f, a3 = a0 + 3e-6f;
  float a4 = a0 + 4e-6f, a5 = a0 + 5e-6f, a6 = a0 + 6e-6f, a7 = a0 + 7e-6f;
  const float m = 0.9999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = fmaf(a0, m, c);
      a1 = fmaf(a1, m, c);
      a2 = fmaf(a2, m, c);
      a3 = fmaf(a3, m, c);
      a4 = fmaf(a4, m, c);
      a5 = fmaf(a5, m, c);
      a6 = fmaf(a6, m, c);
      a7 = fmaf(a7, m, c);
    }
  }
  float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains alive
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__global__ void __launch_bounds__(256) mufu_peak_kernel(float* out, int iters) {
  float a0 = -threadIdx.x * 1e-7f, a1 = a0 - 0.1f, a2 = a0 - 0.2f, a3 = a0 - 0.3f;
  float a4 = a0 - 0.4f, a5 = a0 - 0.5f, a6 = a0 - 0.6f, a7 = a0 - 0.7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = ex2_approx(a0) - 1.0f;
      a1 = ex2_approx(a1) - 1.0f;
      a2 = ex2_approx(a2) - 1.0f;
      a3 = ex2_approx(a3) - 1.0f;
      a4 = ex2_approx(a4) - 1.0f;
      a5 = ex2_approx(a5) - 1.0f;
      a6 = ex2_approx(a6) - 1.0f;
      a7 = ex2_approx(a7) - 1.0f;
    }
  }
  float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678f) out[threadIdx.x] = s;
}

}  // namespace

extern "C" int mpc_measure_peaks(mpc_context_t* ctx, double* fp32_tflops, double* sfu_tops) {
  if (!ctx) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  void* d = nullptr;
  int st = mpc::scratch(ctx, "peaks", 4096, &d);
  if (st != MPC_OK) return st;
  const int blocks = ctx->sm_count * 8, threads = 256, iters = 256;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float ms = 0.0f;
  double best_fma = 0.0, best_mufu = 0.0;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0, ctx->stream);
    fma_peak_kernel<<<blocks, threads, 0, ctx->stream>>>(static_cast<float*>(d), iters);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    double flops = 2.0 * 8 * 16 * double(iters) * blocks * threads;
    if (ms > 0) best_fma = std::max(best_fma, flops / (ms * 1e-3) / 1e12);
    cudaEventRecord(e0, ctx->stream);
    mufu_peak_kernel<<<blocks, threads, 0, ctx->stream>>>(static_cast<float*>(d), iters);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    double ops = 8.0 * 16 * double(iters) * blocks * threads;
    if (ms > 0) best_mufu = std::max(best_mufu, ops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return mpc::cuda_fail(ctx, err, "peak microbenchmarks");
  if (fp32_tflops) *fp32_tflops = best_fma;
  if (sfu_tops) *sfu_tops = best_mufu;
  return MPC_OK;
}
