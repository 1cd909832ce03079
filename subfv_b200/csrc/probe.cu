// FP64 issue-rate probe: the denominator of the FP64 fraction reported for the kernels
// that are bound by FP64 arithmetic rather than by HBM (geometry, nodal solvers). No
// counterpart in the reference. Every thread runs eight independent chains of fused
// multiply-adds (fma.rn.f64), enough instruction-level parallelism to keep the FP64
// pipes busy at full occupancy; the result is written so the chains are not removed.
#include "../../include/subfv.h"
#include "common.cuh"

using namespace subfv;

namespace {

constexpr int kChains = 8;
constexpr int kProbeThreads = 256;
constexpr int kProbeBlocksPerSm = 8;

__global__ void __launch_bounds__(kProbeThreads) k_fp64_fma(double* __restrict__ out, int iters, double a,
                                                            double b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = 1e-3 * (double)(t + k);
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s = s + x[k];
  out[t] = s;
}

}  // namespace

extern "C" int subfv_probe_fp64_fma(int iters, double* tflops, double* ms) {
  if (iters < 1 || iters > (1 << 20) || !tflops) {
    set_error("subfv_probe_fp64_fma: iters must be in [1, 2^20]");
    return -2;
  }
  int dev = 0, sms = 0;
  SUBFV_CUDA(cudaGetDevice(&dev));
  SUBFV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * kProbeBlocksPerSm;
  const long threads = (long)blocks * kProbeThreads;
  double* out = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = 0;
  float t_ms = 0.f;
  if (cudaMalloc(&out, threads * sizeof(double)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    set_error("subfv_probe_fp64_fma: CUDA setup failed");
    rc = -1;
  } else {
    const double a = 0.9999999, b = 1e-7;
    k_fp64_fma<<<blocks, kProbeThreads, 0, s>>>(out, iters, a, b);  // warm-up
    cudaEventRecord(e0, s);
    k_fp64_fma<<<blocks, kProbeThreads, 0, s>>>(out, iters, a, b);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t_ms, e0, e1) != cudaSuccess ||
        cudaGetLastError() != cudaSuccess || !(t_ms > 0.f)) {
      set_error("subfv_probe_fp64_fma: kernel or timing failed");
      rc = -1;
    }
  }
  if (rc == 0) {
    const double flops = 2.0 * kChains * (double)iters * (double)threads;
    *tflops = flops / (t_ms * 1e-3) / 1e12;
    if (ms) *ms = t_ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (out) cudaFree(out);
  return rc;
}

// Checks div3 / div6 (common.cuh) against CUDA's double division on n inputs: counts
// the inputs whose quotients differ in any bit. No counterpart in the reference.
namespace {
__global__ void k_div_const(const double* __restrict__ x, int n, unsigned long long* __restrict__ bad) {
  unsigned long long nb = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = x[i];
    if (__double_as_longlong(div3(v)) != __double_as_longlong(v / 3.0)) ++nb;
    if (__double_as_longlong(div6(v)) != __double_as_longlong(v / 6.0)) ++nb;
  }
  if (nb) atomicAdd(bad, nb);
}
}  // namespace

extern "C" int subfv_probe_div_const(const double* x, int64_t n, int64_t* mismatches) {
  if (!x || n < 0 || !mismatches) {
    set_error("subfv_probe_div_const: bad argument");
    return -2;
  }
  const int64_t chunk = 1 << 24;
  double* d = nullptr;
  unsigned long long* bad = nullptr;
  int rc = 0;
  if (cudaMalloc(&d, chunk * sizeof(double)) != cudaSuccess || cudaMalloc(&bad, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemset(bad, 0, sizeof(unsigned long long)) != cudaSuccess) {
    set_error("subfv_probe_div_const: CUDA setup failed");
    rc = -1;
  }
  for (int64_t o = 0; rc == 0 && o < n; o += chunk) {
    const int m = (int)(n - o < chunk ? n - o : chunk);
    if (cudaMemcpy(d, x + o, m * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("subfv_probe_div_const: copy failed");
      rc = -1;
      break;
    }
    k_div_const<<<592, 256>>>(d, m, bad);
    if (cudaGetLastError() != cudaSuccess) {
      set_error("subfv_probe_div_const: launch failed");
      rc = -1;
    }
  }
  unsigned long long h = 0;
  if (rc == 0 && (cudaMemcpy(&h, bad, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)) {
    set_error("subfv_probe_div_const: copy back failed");
    rc = -1;
  }
  if (rc == 0) *mismatches = (int64_t)h;
  if (d) cudaFree(d);
  if (bad) cudaFree(bad);
  return rc;
}
