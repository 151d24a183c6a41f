// peaks.cu -- measured issue-rate roofs of the arithmetic pipes the force
// kernels use: FP32 FMA, FP64 FMA, and the MUFU ex2 / rsqrt functions.
//
// Each kernel runs CH independent dependency chains per thread for ITER
// iterations, on 8 blocks of 256 threads per SM, so every scheduler has
// enough independent work to issue back to back.  Rates are work / CUDA-event
// time of one launch after a warm-up launch.
#include <cuda_runtime.h>

#include "../../include/gemsgpu.h"

namespace {

constexpr int PK_BLOCK = 256;
constexpr int PK_BLOCKS_PER_SM = 8;
constexpr int CH = 8;
constexpr int ITER = 4096;

__global__ void __launch_bounds__(PK_BLOCK) k_peak_ffma(float m, float c, float* out) {
  float a[CH];
#pragma unroll
  for (int k = 0; k < CH; k++) a[k] = (float)(threadIdx.x + k);
  for (int it = 0; it < ITER; it++) {
#pragma unroll
    for (int k = 0; k < CH; k++) a[k] = fmaf(a[k], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < CH; k++) s += a[k];
  if (s == -1.2345f) out[0] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(PK_BLOCK) k_peak_dfma(double m, double c, double* out) {
  double a[CH];
#pragma unroll
  for (int k = 0; k < CH; k++) a[k] = (double)(threadIdx.x + k);
  for (int it = 0; it < ITER / 4; it++) {
#pragma unroll
    for (int k = 0; k < CH; k++) a[k] = fma(a[k], m, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < CH; k++) s += a[k];
  if (s == -1.2345) out[0] = s;
}

// y <- 2^(-y/2): stays in (0.7, 1]; the start values come from memory
__global__ void __launch_bounds__(PK_BLOCK) k_peak_ex2(float h, const float* in, float* out) {
  float a[CH];
#pragma unroll
  for (int k = 0; k < CH; k++) a[k] = in[k];
  for (int it = 0; it < ITER / 4; it++) {
#pragma unroll
    for (int k = 0; k < CH; k++) {
      float x = a[k] * h;
      asm volatile("ex2.approx.ftz.f32 %0, %0;" : "+f"(x));
      a[k] = x;
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < CH; k++) s += a[k];
  if (s == -1.2345f) out[0] = s;
}

// y <- 1/sqrt(y + 1): stays in (0.7, 1]
__global__ void __launch_bounds__(PK_BLOCK) k_peak_rsqrt(float one, float* out) {
  float a[CH];
#pragma unroll
  for (int k = 0; k < CH; k++) a[k] = 0.5f + 0.01f * (float)k;
  for (int it = 0; it < ITER / 4; it++) {
#pragma unroll
    for (int k = 0; k < CH; k++) a[k] = rsqrtf(a[k] + one);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < CH; k++) s += a[k];
  if (s == -1.2345f) out[0] = s;
}

template <class F>
cudaError_t time_launch(cudaStream_t st, F launch, float* ms) {
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  launch();  // warm-up
  cudaEventRecord(e0, st);
  launch();
  cudaEventRecord(e1, st);
  e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return e;
}

}  // namespace

extern "C" int gemsgpu_measure_peaks(int device, double* out) {
  if (!out) return GEMSGPU_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return GEMSGPU_ERR_CUDA;
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return GEMSGPU_ERR_CUDA;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GEMSGPU_ERR_CUDA;
  double* sink = nullptr;
  if (cudaMalloc(&sink, 64) != cudaSuccess) {
    cudaStreamDestroy(st);
    return GEMSGPU_ERR_OOM;
  }
  float* fs = reinterpret_cast<float*>(sink);
  cudaMemsetAsync(sink, 0, 64, st);
  const int grid = nsm * PK_BLOCKS_PER_SM;
  const double threads = (double)grid * PK_BLOCK;
  float ms[4] = {0, 0, 0, 0};
  cudaError_t e = time_launch(st, [&] { k_peak_ffma<<<grid, PK_BLOCK, 0, st>>>(1.0000001f, 1e-7f, fs); }, &ms[0]);
  if (e == cudaSuccess)
    e = time_launch(st, [&] { k_peak_dfma<<<grid, PK_BLOCK, 0, st>>>(1.0000000001, 1e-9, sink); }, &ms[1]);
  if (e == cudaSuccess) e = time_launch(st, [&] { k_peak_ex2<<<grid, PK_BLOCK, 0, st>>>(-0.5f, fs + 8, fs); }, &ms[2]);
  if (e == cudaSuccess) e = time_launch(st, [&] { k_peak_rsqrt<<<grid, PK_BLOCK, 0, st>>>(1.0f, fs); }, &ms[3]);
  cudaFree(sink);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) return GEMSGPU_ERR_CUDA;
  out[0] = threads * ITER * CH * 2.0 / (ms[0] * 1e-3) * 1e-12;        // FP32 TFLOP/s (FMA = 2)
  out[1] = threads * (ITER / 4) * CH * 2.0 / (ms[1] * 1e-3) * 1e-12;  // FP64 TFLOP/s
  out[2] = threads * (ITER / 4) * CH / (ms[2] * 1e-3) * 1e-9;         // ex2 Gop/s
  out[3] = threads * (ITER / 4) * CH / (ms[3] * 1e-3) * 1e-9;         // rsqrt Gop/s
  return GEMSGPU_OK;
}
