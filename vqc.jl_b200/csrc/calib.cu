// Measured peaks of the device's FMA pipes: the compute roofline of the tile
// passes (no counterpart in the reference, which runs on the host).
//
// The reverse sweep of the FP32 tile engine is bound by the FMA pipe, not by
// HBM, so its roofline denominator is the rate at which this device retires
// fused multiply-adds.  A calibration kernel runs independent FMA chains on
// every SM (eight chains per thread, 2048 threads per SM) and is timed with
// CUDA events; the result is reported as TFLOP/s (two flops per FMA lane).
//   kind 0: packed two-lane FP32 (fma.rn.f32x2, the tile engine's FP32 body)
//   kind 1: scalar FP32 (fma.rn.f32)
//   kind 2: FP64 (fma.rn.f64, the FP64 tile body)
#include <algorithm>

#include "common.cuh"

namespace vqc {
namespace {

constexpr int kCalibChains = 8;
constexpr int kCalibThreads = 256;
constexpr int kCalibBlocksPerSM = 8;

__global__ void __launch_bounds__(kCalibThreads) k_fma_f32x2(int iters, float seed, float* out) {
  unsigned long long a[kCalibChains];
  const float s = seed + threadIdx.x * 1e-7f;
  const unsigned long long m = (unsigned long long)__float_as_uint(0.999999f) * 0x100000001ull;
  const unsigned long long c = (unsigned long long)__float_as_uint(1e-7f) * 0x100000001ull;
#pragma unroll
  for (int k = 0; k < kCalibChains; ++k) a[k] = (unsigned long long)__float_as_uint(s + k) * 0x100000001ull;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kCalibChains; ++k) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[k]) : "l"(m), "l"(c));
  }
  float t = 0.f;
#pragma unroll
  for (int k = 0; k < kCalibChains; ++k) t += __uint_as_float((unsigned)a[k]) + __uint_as_float((unsigned)(a[k] >> 32));
  if (t == 1234.5f) out[threadIdx.x] = t;  // never true: keeps the chains live
}

__global__ void __launch_bounds__(kCalibThreads) k_fma_f32(int iters, float seed, float* out) {
  float a[kCalibChains];
#pragma unroll
  for (int k = 0; k < kCalibChains; ++k) a[k] = seed + k + threadIdx.x * 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kCalibChains; ++k)
      asm volatile("fma.rn.f32 %0, %0, %1, %2;" : "+f"(a[k]) : "f"(0.999999f), "f"(1e-7f));
  }
  float t = 0.f;
#pragma unroll
  for (int k = 0; k < kCalibChains; ++k) t += a[k];
  if (t == 1234.5f) out[threadIdx.x] = t;
}

__global__ void __launch_bounds__(kCalibThreads) k_fma_f64(int iters, double seed, double* out) {
  double a[kCalibChains];
#pragma unroll
  for (int k = 0; k < kCalibChains; ++k) a[k] = seed + k + threadIdx.x * 1e-12;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kCalibChains; ++k)
      asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(a[k]) : "d"(0.999999999), "d"(1e-12));
  }
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < kCalibChains; ++k) t += a[k];
  if (t == 1234.5) out[threadIdx.x] = t;
}

// One launch of `iters` loop trips; returns its device time in ms.
int calib_launch(int kind, int blocks, int iters, cudaStream_t st, void* out, float* ms) {
  cudaEvent_t a, b;
  VQC_CK(cudaEventCreate(&a));
  VQC_CK(cudaEventCreate(&b));
  VQC_CK(cudaEventRecord(a, st));
  if (kind == 0)
    k_fma_f32x2<<<blocks, kCalibThreads, 0, st>>>(iters, 1.0f, (float*)out);
  else if (kind == 1)
    k_fma_f32<<<blocks, kCalibThreads, 0, st>>>(iters, 1.0f, (float*)out);
  else
    k_fma_f64<<<blocks, kCalibThreads, 0, st>>>(iters, 1.0, (double*)out);
  VQC_CK(cudaGetLastError());
  VQC_CK(cudaEventRecord(b, st));
  VQC_CK(cudaEventSynchronize(b));
  VQC_CK(cudaEventElapsedTime(ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return VQC_OK;
}

}  // namespace
}  // namespace vqc

using namespace vqc;

extern "C" int vqc_fma_peak(int device, int kind, double* tflops) {
  if (!tflops || kind < 0 || kind > 2) return fail(VQC_ERR_ARG, "vqc_fma_peak: kind must be 0, 1 or 2");
  int ndev = 0;
  VQC_CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(VQC_ERR_ARG, "vqc_fma_peak: no such device");
  VQC_CK(cudaSetDevice(device));
  cudaStream_t st;
  VQC_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  void* out = nullptr;
  int rc = VQC_OK;
  const int blocks = device_info(device).sms * kCalibBlocksPerSM;
  // lanes per FMA instruction: 2 for the packed form
  const double lanes = kind == 0 ? 2.0 : 1.0;
  double best = 0;
  if (cudaMalloc(&out, kCalibThreads * sizeof(double)) != cudaSuccess) {
    cudaStreamDestroy(st);
    return fail(VQC_ERR_OOM, "vqc_fma_peak: scratch allocation failed");
  }
  float ms = 0;
  int iters = 1024;
  // grow the loop until one launch takes about 20 ms, then keep the best of three
  for (int k = 0; k < 12 && rc == VQC_OK; ++k) {
    rc = calib_launch(kind, blocks, iters, st, out, &ms);
    if (rc || ms > 10.f) break;
    iters *= 2;
  }
  for (int r = 0; r < 3 && rc == VQC_OK; ++r) {
    rc = calib_launch(kind, blocks, iters, st, out, &ms);
    if (rc == VQC_OK && ms > 0) {
      const double fmas = (double)blocks * kCalibThreads * kCalibChains * (double)iters * lanes;
      best = std::max(best, 2.0 * fmas / (ms * 1e-3) / 1e12);
    }
  }
  cudaFree(out);
  cudaStreamDestroy(st);
  if (rc) return rc;
  *tflops = best;
  return VQC_OK;
}
