// Peak-rate probes of this GPU: the denominators of the solve kernel's roofline.
//
// The solve kernels are a serial ODE with a small state: no HBM stream and no contraction,
// so neither the copy bandwidth nor the tensor-core rate bounds them.  What bounds them is
// the issue of FP32 (or FP64) arithmetic and shared-memory traffic.  These kernels measure
// those rates on the device at hand, with CUDA events, so that a roofline fraction is
// against a measured figure and not a formula.
//
//   fma_probe<float|double>  every thread runs kChains independent FMA chains: issue-bound
//                            FMA throughput (2 flop per FMA)
//   smem_probe               every thread reads and writes 16-byte words of shared memory
//                            at conflict-free addresses: shared-memory bandwidth
#include <cuda_runtime.h>

#include <algorithm>

#include "mcs_internal.h"

namespace mcs {
namespace {

constexpr int kChains = 8;
constexpr int kProbeThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kProbeThreads) fma_probe(T* out, int iters, T a, T b) {
  T acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) acc[c] = T(threadIdx.x + c);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int r = 0; r < 16; r++)
#pragma unroll
      for (int c = 0; c < kChains; c++) acc[c] = fma(acc[c], a, b);
  }
  T s = T(0);
#pragma unroll
  for (int c = 0; c < kChains; c++) s += acc[c];
  // a store the compiler cannot drop; a, b keep the values bounded (|a| < 1)
  if (s == T(-12345)) out[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kProbeThreads) smem_probe(float* out, int iters) {
  __shared__ float4 buf[kProbeThreads * 4];
  const int t = threadIdx.x;
#pragma unroll
  for (int k = 0; k < 4; k++) buf[t + k * kProbeThreads] = make_float4(t, k, 0.f, 1.f);
  __syncthreads();
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const unsigned base = (unsigned)__cvta_generic_to_shared(buf);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      // consecutive threads touch consecutive 16-byte words: no bank conflicts.  The
      // accesses are volatile PTX so that the compiler keeps every one of them (a thread
      // only touches its own words, which it could otherwise keep in registers).
      const unsigned a = base + 16u * (unsigned)(t + ((k + i) & 3) * kProbeThreads);
      float4 v;
      asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                   : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                   : "r"(a));
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
      asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.y), "f"(v.z),
                   "f"(v.w), "f"(v.x)
                   : "memory");
    }
  }
  if (acc.x == -12345.f) out[blockIdx.x] = acc.y + acc.z + acc.w;
}

// Best of `reps` timed launches (after one untimed) in milliseconds.
template <typename Launch>
int time_best(cudaStream_t st, int reps, Launch launch, float* best_ms) {
  cudaEvent_t e0, e1;
  MCS_CUDA_RET(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(MCS_ERR_CUDA, "event creation failed");
  }
  float best = 1e30f;
  cudaError_t e = cudaSuccess;
  for (int r = -1; r < reps && e == cudaSuccess; r++) {
    e = cudaEventRecord(e0, st);
    if (e == cudaSuccess) launch();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && r >= 0) best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return fail(MCS_ERR_CUDA, "peak probe failed: %s", cudaGetErrorString(e));
  *best_ms = best;
  return MCS_OK;
}

}  // namespace

int measure_peaks(cudaStream_t st, int sms, void* scratch, double* fp32_tflops,
                  double* fp64_tflops, double* smem_tbps) {
  const int blocks = sms * 8;  // 8 blocks of 256 threads: every SM fully occupied
  int rc;
  float ms = 0.f;
  const int it32 = 4096, it64 = 1024, its = 8192;
  float* o32 = static_cast<float*>(scratch);
  double* o64 = static_cast<double*>(scratch);
  rc = time_best(st, 3, [&] { fma_probe<float><<<blocks, kProbeThreads, 0, st>>>(o32, it32, 0.999f, 0.001f); }, &ms);
  if (rc) return rc;
  *fp32_tflops = 2.0 * kChains * 16 * (double)it32 * blocks * kProbeThreads / (ms * 1e-3) / 1e12;
  rc = time_best(st, 3, [&] { fma_probe<double><<<blocks, kProbeThreads, 0, st>>>(o64, it64, 0.999, 0.001); }, &ms);
  if (rc) return rc;
  *fp64_tflops = 2.0 * kChains * 16 * (double)it64 * blocks * kProbeThreads / (ms * 1e-3) / 1e12;
  rc = time_best(st, 3, [&] { smem_probe<<<blocks, kProbeThreads, 0, st>>>(o32, its); }, &ms);
  if (rc) return rc;
  // per iteration and thread: 4 loads and 4 stores of 16 bytes
  *smem_tbps = 128.0 * (double)its * blocks * kProbeThreads / (ms * 1e-3) / 1e12;
  return MCS_OK;
}

}  // namespace mcs
