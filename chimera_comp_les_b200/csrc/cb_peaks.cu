// Arithmetic-pipe peaks of the GPU the library runs on: the ceiling of the
// compute roofline for the stage kernels (a stencil, no tensor cores).
//
// Every thread runs CH independent fused multiply-add chains (fma.rn in
// inline PTX, so the count does not depend on the compiler's contraction
// flags) over enough resident warps to keep the FP64 or FP32 pipe issuing
// every cycle; the rate is 2 flops per FMA.  A plain add or multiply issues
// on the same pipe at the same rate as an FMA, so code built without FMA
// contraction (the FP64 parity form) tops out at half this flop rate.
#include <cuda_runtime.h>

#include "../../include/chimera_b200.h"

namespace {

constexpr int PK_CH = 8;       // independent chains per thread
constexpr int PK_THREADS = 256;

__global__ void __launch_bounds__(PK_THREADS) fma64_kernel(double *out, int iters, double b, double c) {
  double a[PK_CH];
#pragma unroll
  for (int i = 0; i < PK_CH; i++) a[i] = 1e-3 * threadIdx.x + i;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < PK_CH; i++) asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(a[i]) : "d"(b), "d"(c));
  }
  double s = 0.;
#pragma unroll
  for (int i = 0; i < PK_CH; i++) s += a[i];
  if (s == -1.0) out[blockIdx.x] = s;  // never true: keeps the chains live
}

__global__ void __launch_bounds__(PK_THREADS) fma32_kernel(float *out, int iters, float b, float c) {
  float a[PK_CH];
#pragma unroll
  for (int i = 0; i < PK_CH; i++) a[i] = 1e-3f * threadIdx.x + i;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < PK_CH; i++) asm volatile("fma.rn.f32 %0, %0, %1, %2;" : "+f"(a[i]) : "f"(b), "f"(c));
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < PK_CH; i++) s += a[i];
  if (s == -1.0f) out[blockIdx.x] = s;
}

// Best of `reps` timed launches after one warm-up, in flop/s.
template <typename K, typename T>
cudaError_t time_fma(K kern, T *out, int blocks, int iters, T b, T c, cudaStream_t s, double *flops) {
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  if ((e = cudaEventCreate(&e1)) != cudaSuccess) { cudaEventDestroy(e0); return e; }
  kern<<<blocks, PK_THREADS, 0, s>>>(out, iters, b, c);
  float best = 0.f;
  for (int r = 0; r < 3 && (e = cudaGetLastError()) == cudaSuccess; r++) {
    cudaEventRecord(e0, s);
    kern<<<blocks, PK_THREADS, 0, s>>>(out, iters, b, c);
    cudaEventRecord(e1, s);
    if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r == 0 || ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e == cudaSuccess) *flops = 2.0 * PK_CH * (double)iters * blocks * PK_THREADS / (best * 1e-3);
  return e;
}

}  // namespace

extern "C" int cb_pipe_peaks(int device, double *fp64_tflops, double *fp32_tflops) {
  if (!fp64_tflops || !fp32_tflops) return CB_E_ARG;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return CB_E_CUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8;  // 8 x 256 threads per SM: 64 warps, the SM's limit
  cudaStream_t s = nullptr;
  void *out = nullptr;
  double f64 = 0., f32 = 0.;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&out, (size_t)blocks * sizeof(double));
  // b slightly below 1 and a small c keep every chain finite and normal
  if (e == cudaSuccess)
    e = time_fma(fma64_kernel, static_cast<double *>(out), blocks, 16384, 0.9999999, 1e-7, s, &f64);
  if (e == cudaSuccess)
    e = time_fma(fma32_kernel, static_cast<float *>(out), blocks, 65536, 0.9999999f, 1e-7f, s, &f32);
  if (out) cudaFree(out);
  if (s) cudaStreamDestroy(s);
  cudaSetDevice(prev);
  if (e != cudaSuccess) return CB_E_CUDA;
  *fp64_tflops = f64 * 1e-12;
  *fp32_tflops = f32 * 1e-12;
  return CB_OK;
}
