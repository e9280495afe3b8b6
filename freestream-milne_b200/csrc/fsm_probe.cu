// fsm_probe.cu -- device FP32 FMA throughput probe, the denominator of the
// stream kernels' roofline fraction (they are FP32-pipe bound, so the memory-
// copy and tensor-core peaks do not apply).  Each thread runs 8 independent FMA
// chains; the result is written so the work cannot be removed.
#include <cuda_runtime.h>

#include "../../include/fsm.h"

namespace {
__global__ void __launch_bounds__(256) fsm_probe_ffma_kernel(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5,
        x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fmaf(x0, a, b);
      x1 = fmaf(x1, a, b);
      x2 = fmaf(x2, a, b);
      x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b);
      x5 = fmaf(x5, a, b);
      x6 = fmaf(x6, a, b);
      x7 = fmaf(x7, a, b);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}
}  // namespace

extern "C" fsm_status fsm_probe_fp32_tflops(int device, double* tflops) {
  if (!tflops) return FSM_ERR_INVALID_ARG;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return FSM_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return FSM_ERR_CUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  float* out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(float)) != cudaSuccess) return FSM_ERR_OUT_OF_MEMORY;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fsm_probe_ffma_kernel<<<blocks, threads>>>(out, iters / 8, 0.999f, 0.001f);  // warm-up
  cudaEventRecord(e0);
  fsm_probe_ffma_kernel<<<blocks, threads>>>(out, iters, 0.999f, 0.001f);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess || ms <= 0) return FSM_ERR_CUDA;
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return FSM_OK;
}
