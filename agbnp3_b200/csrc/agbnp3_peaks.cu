/*
 * Arithmetic peaks of the current GPU, measured with our own throughput
 * kernels: the denominators of the pair stages' roofline (FP32 FMA, FP64
 * FMA and special-function unit rates).  Each thread runs eight independent
 * dependency chains for a fixed number of iterations over a grid that fills
 * every SM; the rate is operations / CUDA-event time of the second of two
 * launches.
 */
#include <cuda_runtime.h>
#include <stdio.h>

#include "agbnp3_launch.cuh"

#define PK_ITERS 16384
#define PK_THREADS 512

__global__ void __launch_bounds__(PK_THREADS) k_peak_fma32(float *out, float a, float b) {
  float x[8];
#pragma unroll
  for (int c = 0; c < 8; c++) x[c] = 0.01f * (threadIdx.x + c);
  for (int i = 0; i < PK_ITERS; i++) {
#pragma unroll
    for (int c = 0; c < 8; c++) x[c] = fmaf(x[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) s += x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(PK_THREADS) k_peak_fma64(double *out, double a, double b) {
  double x[8];
#pragma unroll
  for (int c = 0; c < 8; c++) x[c] = 0.01 * (threadIdx.x + c);
  for (int i = 0; i < PK_ITERS / 8; i++) {
#pragma unroll
    for (int c = 0; c < 8; c++) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 8; c++) s += x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

/* x <- 2^-x stays in (0, 1]: one ex2.approx per step and chain */
__global__ void __launch_bounds__(PK_THREADS) k_peak_ex2(float *out) {
  float x[8];
#pragma unroll
  for (int c = 0; c < 8; c++) x[c] = 0.01f * (threadIdx.x + c);
  for (int i = 0; i < PK_ITERS / 4; i++) {
#pragma unroll
    for (int c = 0; c < 8; c++) asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(x[c]) : "f"(-x[c]));
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) s += x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

static int sm_count(int device) {
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return -1;
  return n;
}

/* out[0] FP32 flop/s (FMA = 2), out[1] FP64 flop/s, out[2] ex2 op/s,
   out[3] SM clock in MHz reported by the runtime; returns the number of
   values written or -1 */
extern "C" int agbnp3_measure_peaks(int device, double *out, int n) {
  if (!out || n < 4) return -1;
  if (cudaSetDevice(device) != cudaSuccess) return -1;
  int sms = sm_count(device);
  if (sms <= 0) return -1;
  int blocks = sms * (2048 / PK_THREADS);
  size_t nthr = (size_t)blocks * PK_THREADS;
  void *buf = NULL;
  if (cudaMalloc(&buf, nthr * sizeof(double)) != cudaSuccess) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double ops[3] = {2.0 * 8 * PK_ITERS * (double)nthr, 2.0 * 8 * (PK_ITERS / 8) * (double)nthr,
                   8.0 * (PK_ITERS / 4) * (double)nthr};
  int rc = 4;
  for (int k = 0; k < 3 && rc > 0; k++) {
    float ms = 0.f;
    for (int rep = 0; rep < 2; rep++) {
      cudaEventRecord(e0, 0);
      if (k == 0) k_peak_fma32<<<blocks, PK_THREADS>>>((float *)buf, 0.999f, 0.001f);
      if (k == 1) k_peak_fma64<<<blocks, PK_THREADS>>>((double *)buf, 0.999, 0.001);
      if (k == 2) k_peak_ex2<<<blocks, PK_THREADS>>>((float *)buf);
      cudaEventRecord(e1, 0);
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        rc = -1;
        break;
      }
      cudaEventElapsedTime(&ms, e0, e1);
    }
    out[k] = ms > 0.f ? ops[k] / (ms * 1e-3) : 0.0;
  }
  int clk = 0;
  cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, device);
  out[3] = clk / 1000.0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  return rc;
}
