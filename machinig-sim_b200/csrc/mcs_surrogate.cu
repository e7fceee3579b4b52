// The learned surrogate: an MLP 20 -> 256 -> 256 -> 256 -> 2 (SiLU) trained with a
// Gaussian negative log-likelihood on log critical depths the time-domain solver
// produced.  Weights and activations are BF16 and every product accumulates in FP32; the
// Adam state and master weights are FP32.  Both run on the 5th-generation tensor cores
// (tcgen05.mma with the accumulator in tensor memory): training (forward, backward, Adam)
// through one GEMM kernel with strided operands, inference in one fused kernel.
//
// Layers are padded to tensor-core shapes: the 20 inputs to 32, the 2 outputs to 16;
// padded weights start at zero and get zero gradients, so they stay zero.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "mcs_internal.h"

namespace mcs {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kIn = MCS_FEATURES;
constexpr int kInPad = 32;
constexpr int kHid = 256;
constexpr int kOutPad = 16;
constexpr int kLayers = 4;
constexpr int kK[kLayers] = {kInPad, kHid, kHid, kHid};
constexpr int kN[kLayers] = {kHid, kHid, kHid, kOutPad};
constexpr float kSMin = -7.f, kSMax = 5.f;  // range of the predicted log sigma

// offsets of the parameter blob (floats)
struct Layout {
  size_t mean = 0, stdv = kIn, W[kLayers], b[kLayers], total;
  Layout() {
    size_t o = 2 * kIn;
    for (int l = 0; l < kLayers; l++) {
      W[l] = o;
      o += (size_t)kK[l] * kN[l];
      b[l] = o;
      o += kN[l];
    }
    total = o;
  }
};
const Layout kLay;

// ---------------------------------------------------------------- kernels
__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + __expf(-z)); }

// z = C + bias (kept for the backward pass); out = BF16(silu(z)) or, for the last layer,
// the FP32 z itself
__global__ void bias_act(const float* __restrict__ C, const float* __restrict__ bias, int M,
                         int N, float* __restrict__ z, bf16* __restrict__ out, int act) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)M * N) return;
  const float v = C[i] + bias[i % N];
  if (z) z[i] = v;
  if (out) out[i] = __float2bfloat16(act ? v * sigmoid(v) : v);
}

// Gaussian NLL of y under N(mu, exp(s)^2) with (mu, s) = out[:, 0:2]; writes d loss / d out
// (divided by the batch) in FP32 and BF16 and adds the summed loss to *loss.
__global__ void nll_loss(const float* __restrict__ out, const float* __restrict__ y, int B,
                         float* __restrict__ dout, bf16* __restrict__ doutb,
                         float* __restrict__ loss) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (b < B) {
    const float mu = out[(long)b * kOutPad], s_raw = out[(long)b * kOutPad + 1];
    const float s = fminf(fmaxf(s_raw, kSMin), kSMax);
    const float r = y[b] - mu, iv = __expf(-2.f * s);
    l = s + 0.5f * r * r * iv;
    const float inB = 1.f / (float)B;
    const float dmu = -r * iv * inB;
    const float ds = (s_raw > kSMin && s_raw < kSMax) ? (1.f - r * r * iv) * inB : 0.f;
    for (int c = 0; c < kOutPad; c++) {
      const float d = c == 0 ? dmu : (c == 1 ? ds : 0.f);
      dout[(long)b * kOutPad + c] = d;
      doutb[(long)b * kOutPad + c] = __float2bfloat16(d);
    }
  }
  // warp, then block reduction of the loss
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += part[w];
    atomicAdd(loss, s);
  }
}

// dz = dh * silu'(z) in FP32 and BF16
__global__ void silu_back(const float* __restrict__ dh, const float* __restrict__ z, long n,
                          float* __restrict__ dz, bf16* __restrict__ dzb) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = z[i], sg = sigmoid(v);
  const float d = dh[i] * sg * (1.f + v * (1.f - sg));
  dz[i] = d;
  dzb[i] = __float2bfloat16(d);
}

// db[c] = sum over rows of dz[:, c]
__global__ void col_sum(const float* __restrict__ dz, int M, int N, float* __restrict__ db) {
  const int c = blockIdx.x;
  float s = 0.f;
  for (int r = threadIdx.x; r < M; r += blockDim.x) s += dz[(long)r * N + c];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
    db[c] = t;
  }
}

// Adam on the trainable part of the parameter blob (bias-corrected)
__global__ void adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                     const float* __restrict__ g, long n, float lr, float b1, float b2, float eps,
                     float c1, float c2) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void to_bf16(const float* __restrict__ x, long n, bf16* __restrict__ y) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}

// rows idx[off + b] (or off + b without idx) of the raw features, normalised, BF16, padded
__global__ void gather_rows(const float* __restrict__ X, const int32_t* __restrict__ idx,
                            long off, int B, long n, const float* __restrict__ mean,
                            const float* __restrict__ stdv, const float* __restrict__ y,
                            bf16* __restrict__ xb, float* __restrict__ yb) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)B * kInPad) return;
  const int b = (int)(i / kInPad), c = (int)(i % kInPad);
  const long row = idx ? (long)idx[off + b] : off + b;
  float v = 0.f;
  if (c < kIn && row < n) v = (X[row * kIn + c] - mean[c]) / stdv[c];
  xb[i] = __float2bfloat16(v);
  if (c == 0 && yb) yb[b] = row < n ? y[row] : 0.f;
}



// ------------------------------------------------ inference on the 5th-generation tensor cores
// One CTA of 4 warps owns a tile of 128 rows and runs all four layers on it:
//   * the activation tile A[128 x K] (BF16) stays in shared memory, and each layer's output
//     is written back over it as the next layer's input;
//   * a layer's weights, kept in global memory as W^T[N x K] in the operand layout below,
//     are copied into a shared-memory buffer (at most 256 x 256 BF16 = 128 KB);
//   * one thread issues tcgen05.mma (M = 128, N = 256 or 16, K = 16 per instruction,
//     kind::f16 with BF16 operands and an FP32 accumulator in tensor memory) and commits
//     to an mbarrier;
//   * the four warps read their 32 accumulator lanes back with tcgen05.ld, add the bias,
//     apply SiLU and store BF16 (or, after the last layer, write mu, sigma and the guide).
// Operand layout in shared memory (K-major, no swizzle): element (row, k) of an R-row
// operand sits at ((k / 8) * R + row) * 8 + k % 8, so a core matrix of 8 rows x 16 bytes is
// contiguous, 8-row groups are 128 bytes apart (stride byte offset) and the two 8-element
// halves of one K = 16 step are R * 16 bytes apart (leading byte offset).
constexpr int kTcRows = 128;
constexpr int kTcThreads = 128;
constexpr int kTcCols = 256;                          // tensor-memory columns (N <= 256)
constexpr int kTcSmemA = kTcRows * kHid * 2;          // 64 KB
constexpr int kTcSmemW = kHid * kHid * 2;             // 128 KB
constexpr int kTcConst = 2 * kIn + 3 * kHid + kOutPad;  // mean, std, b0..b3 (floats)
constexpr int kTcSmem = kTcSmemA + kTcSmemW + kTcConst * 4 + 16;
constexpr long long kTcWaitCycles = 4000000000LL;     // ~2 s at 2 GHz: an MMA takes microseconds

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// shared-memory matrix descriptor: start, leading and stride byte offsets (16-byte units),
// descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major
__host__ __device__ constexpr uint32_t instr_desc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kTcRows >> 4) << 24);
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// bounded wait for the mbarrier phase `parity` to complete
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kTcWaitCycles) return false;
  }
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16(lo)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16(hi)) << 16);
}

// layer shapes and bias offsets of the parameter blob, usable in device code
__host__ __device__ constexpr int layer_k(int l) { return l == 0 ? kInPad : kHid; }
__host__ __device__ constexpr int layer_n(int l) { return l == kLayers - 1 ? kOutPad : kHid; }
__host__ __device__ constexpr int bias_off(int l) {
  return l == 0 ? 2 * kIn + kInPad * kHid
                : bias_off(l - 1) + layer_n(l - 1) + layer_k(l) * layer_n(l);
}
static_assert(bias_off(0) == 8232 && bias_off(3) == 144168, "parameter blob layout");

struct TcWeights {
  const bf16* w[kLayers];  // W^T of each layer in the operand layout
};

__global__ void __launch_bounds__(kTcThreads, 1)
    mlp_infer_tc(const float* __restrict__ X, long n, const float* __restrict__ params,
                 TcWeights tw, float* __restrict__ mu, float* __restrict__ sigma,
                 float2* __restrict__ guide, float z, float hw_min, float hw_max,
                 float hw_direct, int spec, float skip_top, float log_amax,
                 int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  bf16* A = reinterpret_cast<bf16*>(smem);
  bf16* W = reinterpret_cast<bf16*>(smem + kTcSmemA);
  float* cst = reinterpret_cast<float*>(smem + kTcSmemA + kTcSmemW);
  uint64_t* bar = reinterpret_cast<uint64_t*>(cst + kTcConst);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const float* mean = cst;
  const float* stdv = cst + kIn;
  const float* bias[kLayers] = {cst + 2 * kIn, cst + 2 * kIn + kHid, cst + 2 * kIn + 2 * kHid,
                                cst + 2 * kIn + 3 * kHid};
  for (int i = tid; i < 2 * kIn; i += kTcThreads) cst[i] = params[i];
  for (int l = 0; l < kLayers; l++)
    for (int i = tid; i < layer_n(l); i += kTcThreads)
      cst[2 * kIn + l * kHid + i] = params[bias_off(l) + i];
  const uint32_t bar_a = smem_addr(bar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
  const uint32_t a_base = smem_addr(A), w_base = smem_addr(W);
  uint32_t phase = 0;
  bool ok = true;
  for (long tile = blockIdx.x; ok && tile * kTcRows < n; tile += gridDim.x) {
    const long row = tile * kTcRows + tid;
    // normalised features of this thread's row -> K chunks 0..3 of A (inputs 20..31 are 0)
    {
      float v[kInPad];
#pragma unroll
      for (int c = 0; c < kInPad; c++) v[c] = 0.f;
      if (row < n) {
#pragma unroll
        for (int c = 0; c < kIn; c++) v[c] = (X[row * kIn + c] - mean[c]) / stdv[c];
      }
#pragma unroll
      for (int kc = 0; kc < kInPad / 8; kc++) {
        uint4 q;
        q.x = pack_bf16(v[8 * kc + 0], v[8 * kc + 1]);
        q.y = pack_bf16(v[8 * kc + 2], v[8 * kc + 3]);
        q.z = pack_bf16(v[8 * kc + 4], v[8 * kc + 5]);
        q.w = pack_bf16(v[8 * kc + 6], v[8 * kc + 7]);
        *reinterpret_cast<uint4*>(A + ((size_t)kc * kTcRows + tid) * 8) = q;
      }
    }
#pragma unroll 1
    for (int l = 0; l < kLayers; l++) {
      const int K = layer_k(l), N = layer_n(l);
      {  // this layer's W^T: a contiguous copy, 16 bytes per thread and step
        const uint4* src = reinterpret_cast<const uint4*>(tw.w[l]);
        uint4* dst = reinterpret_cast<uint4*>(W);
        const int nvec = K * N / 8;
        for (int i = tid; i < nvec; i += kTcThreads) dst[i] = src[i];
      }
      // make the generic-proxy stores visible to the tensor core, and order the previous
      // layer's tensor-memory reads before the new MMAs
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t idesc = instr_desc(N);
        for (int ks = 0; ks < K / 16; ks++) {
          const uint64_t ad = smem_desc(a_base + ks * 2 * (kTcRows * 16), kTcRows * 16, 128);
          const uint64_t bd = smem_desc(w_base + ks * 2 * (N * 16), N * 16, 128);
          const uint32_t acc = ks > 0 ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
              : "memory");
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                bar_a)
            : "memory");
      }
      ok = mbar_wait(bar_a, phase);
      phase ^= 1u;
      ok = __syncthreads_and(ok) != 0;  // one decision for the whole block
      tc_fence_after();
      if (!ok) break;
      const float* b = bias[l];
      if (l < kLayers - 1) {
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 16) {
          uint32_t r[16];
          tmem_ld16(lane_base + (uint32_t)c0, r);
          float h[16];
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const float v = __uint_as_float(r[j]) + b[c0 + j];
            h[j] = v * sigmoid(v);
          }
#pragma unroll
          for (int half = 0; half < 2; half++) {
            uint4 q;
            q.x = pack_bf16(h[8 * half + 0], h[8 * half + 1]);
            q.y = pack_bf16(h[8 * half + 2], h[8 * half + 3]);
            q.z = pack_bf16(h[8 * half + 4], h[8 * half + 5]);
            q.w = pack_bf16(h[8 * half + 6], h[8 * half + 7]);
            *reinterpret_cast<uint4*>(A + ((size_t)(c0 / 8 + half) * kTcRows + tid) * 8) = q;
          }
        }
      } else {
        uint32_t r[16];
        tmem_ld16(lane_base, r);
        if (row < n) {
          const float m = __uint_as_float(r[0]) + b[0];
          const float sv = expf(fminf(fmaxf(__uint_as_float(r[1]) + b[1], kSMin), kSMax));
          if (mu) mu[row] = m;
          if (sigma) sigma[row] = sv;
          if (guide) {
            const float w = z * sv;
            float gy = w > hw_direct ? -1.f : fminf(fmaxf(w, hw_min), hw_max);
            // the speculating guide: -2 marks a point that skips its first trial at a_max
            // (predicted stable there with a probability below skip_top)
            if (spec) gy = (skip_top > 0.f && normcdff((m - log_amax) / sv) < skip_top) ? -2.f : -1.f;
            guide[row] = make_float2(m, gy);
          }
        }
      }
    }
  }
  if (!ok) {
    // an MMA did not complete in time: wait once more (bounded) for it before the tensor
    // memory is released
    mbar_wait(bar_a, phase ^ 1u);
    if (tid == 0) atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcCols)
                 : "memory");
}

// ------------------------------------------------ training GEMMs on the tensor cores
// C[M x N] (+)= A[M x K] B[K x N] with A(m, k) = A[m*sAm + k*sAk] and B(k, n) = B[k*sBk +
// n*sBn] (the strides express the transposes of the backward pass), BF16 operands and an
// FP32 accumulator in tensor memory.  One CTA of 4 warps owns a 128-row x nt-column tile of
// C (nt = 16 ... 256, a multiple of 16) and runs over K in chunks of 64: the threads copy
// the chunk's A rows and B columns into a shared-memory stage in the K-major operand layout
// of mlp_infer_tc (rows past M, columns past N and k past K are zero), one thread issues
// the chunk's tcgen05.mma (K = 16 each) and commits them to the stage's mbarrier.  Two
// stages: the copy of the next chunk overlaps the MMAs of the current one, and a stage is
// refilled only after its mbarrier says the MMAs that read it are done.  The four warps
// read their 32 accumulator rows back with tcgen05.ld.  Every wait is bounded; a timeout
// sets *err and the kernel drains its MMAs (bounded) before it frees the tensor memory.
constexpr int kGtKc = 64;                                  // K per stage
constexpr int kGtStageA = kTcRows * kGtKc * 2;             // 16 KB
constexpr int kGtStageB = kTcCols * kGtKc * 2;             // 32 KB at nt = 256
constexpr int kGtSmem = 2 * (kGtStageA + kGtStageB) + 64;  // stages + 2 mbarriers + TMEM slot

// One operand chunk: rows [r0, r0 + R) of an operand X(r, k) = X[r*sr + k*sk] with r < rmax
// and k in [k0, k0 + kc) with k < kmax (zero elsewhere), into dst in the K-major operand
// layout (element (r, k) at ((k / 8) * R + r) * 8 + k % 8: the 8 k of a row and group are
// 16 contiguous bytes).  The work item of a thread is an 8-k group:
//   * k contiguous in X (sk == 1): one 16-byte load and one 16-byte store per (row, group);
//   * rows contiguous (sr == 1): an 8-row x 8-k block, eight 16-byte loads along the rows,
//     transposed in registers into eight 16-byte stores;
//   * otherwise, or where a vector would leave the bounds or its 16-byte alignment,
//     element by element.
__device__ __forceinline__ uint16_t bf_at(const bf16* p, long i) {
  return __bfloat16_as_ushort(p[i]);
}

__device__ __forceinline__ void stage_operand(const bf16* __restrict__ X, long sr, long sk,
                                              int r0, int rmax, int k0, int kmax, int R,
                                              int kc, uint16_t* __restrict__ dst, int tid) {
  const int groups = kc / 8;
  const bool base16 = (reinterpret_cast<uintptr_t>(X) & 15u) == 0;
  if (sk == 1) {
    // all of a thread's loads (at most 16: 256 rows x 8 groups over 128 threads) are issued
    // before its stores
    constexpr int kItems = kTcCols * (kGtKc / 8) / kTcThreads;
    const bool vec = base16 && (sr % 8) == 0;
    const int items = R * groups;
    uint4 q[kItems];
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      const int e = tid + it * kTcThreads;
      q[it] = make_uint4(0u, 0u, 0u, 0u);
      const int r = e / groups, g = e - r * groups;
      const int gr = r0 + r, gk = k0 + 8 * g;
      if (e < items && gr < rmax) {
        if (vec && gk + 8 <= kmax) {
          q[it] = *reinterpret_cast<const uint4*>(X + gr * sr + gk);
        } else {
          uint16_t v[8];
#pragma unroll
          for (int j = 0; j < 8; j++) v[j] = gk + j < kmax ? bf_at(X, gr * sr + gk + j) : 0;
          q[it].x = v[0] | ((uint32_t)v[1] << 16);
          q[it].y = v[2] | ((uint32_t)v[3] << 16);
          q[it].z = v[4] | ((uint32_t)v[5] << 16);
          q[it].w = v[6] | ((uint32_t)v[7] << 16);
        }
      }
    }
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      const int e = tid + it * kTcThreads;
      const int r = e / groups, g = e - r * groups;
      if (e < items) *reinterpret_cast<uint4*>(dst + ((size_t)g * R + r) * 8) = q[it];
    }
  } else {
    const bool vec = base16 && sr == 1 && (sk % 8) == 0;
    const int rb = R / 8;  // 8-row blocks
    for (int e = tid; e < rb * groups; e += kTcThreads) {
      const int b = e % rb, g = e / rb;  // neighbouring threads: neighbouring row blocks
      const int gr = r0 + 8 * b, gk = k0 + 8 * g;
      uint16_t v[8][8];  // v[j][i]: row gr + i, k gk + j
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const bool kin = gk + j < kmax;
        if (vec && kin && gr + 8 <= rmax) {
          const uint4 q = *reinterpret_cast<const uint4*>(X + gr + (long)(gk + j) * sk);
          const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
          for (int i = 0; i < 4; i++) {
            v[j][2 * i] = (uint16_t)(w[i] & 0xFFFFu);
            v[j][2 * i + 1] = (uint16_t)(w[i] >> 16);
          }
        } else {
#pragma unroll
          for (int i = 0; i < 8; i++)
            v[j][i] = (kin && gr + i < rmax) ? bf_at(X, (long)(gr + i) * sr + (long)(gk + j) * sk)
                                             : (uint16_t)0;
        }
      }
#pragma unroll
      for (int i = 0; i < 8; i++) {
        uint4 q;
        q.x = v[0][i] | ((uint32_t)v[1][i] << 16);
        q.y = v[2][i] | ((uint32_t)v[3][i] << 16);
        q.z = v[4][i] | ((uint32_t)v[5][i] << 16);
        q.w = v[6][i] | ((uint32_t)v[7][i] << 16);
        *reinterpret_cast<uint4*>(dst + ((size_t)g * R + 8 * b + i) * 8) = q;
      }
    }
  }
}

__global__ void __launch_bounds__(kTcThreads, 1)
    gemm_tc(const bf16* __restrict__ A, long sAm, long sAk, const bf16* __restrict__ B,
            long sBk, long sBn, float* __restrict__ C, long ldc, int M, int N, int K, int nt,
            int tcols, int accumulate, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint16_t* sa[2] = {reinterpret_cast<uint16_t*>(smem),
                     reinterpret_cast<uint16_t*>(smem + kGtStageA + kGtStageB)};
  uint16_t* sb[2] = {reinterpret_cast<uint16_t*>(smem + kGtStageA),
                     reinterpret_cast<uint16_t*>(smem + 2 * kGtStageA + kGtStageB)};
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * (kGtStageA + kGtStageB));
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.y * kTcRows, n0 = blockIdx.x * nt;
  const uint32_t bar_a[2] = {smem_addr(bar), smem_addr(bar + 1)};
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a[0]) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a[1]) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = instr_desc(nt);
  const int chunks = (K + kGtKc - 1) / kGtKc;
  bool ok = true;
  int issued = 0;  // chunks whose MMAs were committed
  for (int c = 0; c < chunks; c++) {
    const int s = c & 1;
    if (c >= 2) {  // the MMAs of chunk c - 2 read this stage
      ok = mbar_wait(bar_a[s], (uint32_t)(((c - 2) >> 1) & 1));
      ok = __syncthreads_and(ok) != 0;
      if (!ok) break;
    }
    const int k0 = c * kGtKc;
    const int kc = min(kGtKc, ((K - k0 + 15) / 16) * 16);  // a multiple of 16, zero past K
    stage_operand(A, sAm, sAk, m0, M, k0, K, kTcRows, kc, sa[s], tid);
    stage_operand(B, sBn, sBk, n0, N, k0, K, nt, kc, sb[s], tid);
    // the generic-proxy stores become visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_addr(sa[s]), b0 = smem_addr(sb[s]);
      for (int ks = 0; ks < kc / 16; ks++) {
        const uint64_t ad = smem_desc(a0 + ks * 2 * (kTcRows * 16), kTcRows * 16, 128);
        const uint64_t bd = smem_desc(b0 + ks * 2 * (nt * 16), nt * 16, 128);
        const uint32_t accum = (c > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(accum)
            : "memory");
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              bar_a[s])
          : "memory");
    }
    issued = c + 1;
  }
  // the last commit covers every MMA this thread issued before it; the other stage's
  // last commit has then arrived as well
  if (ok && issued > 0) {
    const int c = issued - 1;
    ok = mbar_wait(bar_a[c & 1], (uint32_t)((c >> 1) & 1));
    if (ok && c >= 1) ok = mbar_wait(bar_a[(c - 1) & 1], (uint32_t)(((c - 1) >> 1) & 1));
    ok = __syncthreads_and(ok) != 0;
  }
  tc_fence_after();
  if (ok && issued > 0) {
    const int r = m0 + warp * 32 + (tid & 31);
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    const bool vec_c = (reinterpret_cast<uintptr_t>(C) & 15u) == 0 && (ldc % 4) == 0;
#pragma unroll 1
    for (int c0 = 0; c0 < nt; c0 += 16) {
      uint32_t v[16];
      tmem_ld16(lane_base + (uint32_t)c0, v);
      if (r < M) {
        float* o = C + (long)r * ldc + n0 + c0;
        if (vec_c && n0 + c0 + 16 <= N) {  // four 16-byte stores along the row
#pragma unroll
          for (int j = 0; j < 4; j++) {
            float4 w = make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                   __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]));
            float4* p4 = reinterpret_cast<float4*>(o) + j;
            if (accumulate) {
              const float4 c = *p4;
              w.x += c.x;
              w.y += c.y;
              w.z += c.z;
              w.w += c.w;
            }
            *p4 = w;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; j++) {
            if (n0 + c0 + j < N)
              o[j] = accumulate ? o[j] + __uint_as_float(v[j]) : __uint_as_float(v[j]);
          }
        }
      }
    }
  } else if (issued > 0) {
    // a wait gave up: wait once more (bounded) for the MMAs in flight before the tensor
    // memory is released, and report it
    const int c = issued - 1;
    mbar_wait(bar_a[c & 1], (uint32_t)((c >> 1) & 1));
    if (c >= 1) mbar_wait(bar_a[(c - 1) & 1], (uint32_t)(((c - 1) >> 1) & 1));
    if (tid == 0) atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tcols)
                 : "memory");
}

// W[K x N] (FP32, row-major) -> BF16 W^T[N x K] in the operand layout of mlp_infer_tc
__global__ void to_bf16_operand(const float* __restrict__ Wf, int K, int N, bf16* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)K * N) return;
  const int k = (int)(i / N), nn = (int)(i % N);
  out[((long)(k / 8) * N + nn) * 8 + (k % 8)] = __float2bfloat16(Wf[i]);
}

inline int blocks(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace
}  // namespace mcs

using namespace mcs;

namespace mcs {
namespace {
// Activations (and gradients) of one batch of up to `cap` rows.
struct Acts {
  int cap = 0;
  bf16* xb = nullptr;
  float* yb = nullptr;
  float* z[kLayers] = {};
  bf16* a[kLayers] = {};
  float* C = nullptr;   // GEMM output
  float* dz = nullptr;  // FP32 d loss / d z
  bf16* dzb = nullptr;
  float* dh = nullptr;
};
}  // namespace
}  // namespace mcs

struct mcs_surrogate {
  mcs_ctx* ctx = nullptr;
  uint64_t seed = 0;
  bool trained = false;
  float* params = nullptr;  // FP32 blob on the device
  float* grad = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  bf16* Wb[kLayers] = {};
  bf16* Wt[kLayers] = {};  // W^T in the tensor-core operand layout (inference)
  int* err = nullptr;      // set by an inference kernel whose MMA wait timed out
  int sms = 0;
  long step = 0;
  Acts tr;   // training and gradients
  float* loss = nullptr;
  std::atomic<int> plans{0};  // guided plans holding this surrogate
  std::mutex mu;
};

namespace mcs {

namespace {

template <typename T>
int dalloc(T** p, size_t count) {
  *p = nullptr;
  const cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? MCS_ERR_NOMEM : MCS_ERR_CUDA,
                "cudaMalloc failed: %s", cudaGetErrorString(e));
  }
  return MCS_OK;
}

void free_acts(Acts& s) {
  cudaFree(s.xb);
  cudaFree(s.yb);
  for (int l = 0; l < kLayers; l++) {
    cudaFree(s.z[l]);
    cudaFree(s.a[l]);
  }
  cudaFree(s.C);
  cudaFree(s.dz);
  cudaFree(s.dzb);
  cudaFree(s.dh);
  s = Acts();
}

int ensure_acts(Acts& s, int rows) {
  if (rows <= s.cap) return MCS_OK;
  free_acts(s);
  int rc;
  const size_t r = (size_t)rows;
  if ((rc = dalloc(&s.xb, r * kInPad)) || (rc = dalloc(&s.yb, r)) ||
      (rc = dalloc(&s.C, r * kHid)) || (rc = dalloc(&s.dz, r * kHid)) ||
      (rc = dalloc(&s.dzb, r * kHid)) || (rc = dalloc(&s.dh, r * kHid))) {
    free_acts(s);
    return rc;
  }
  for (int l = 0; l < kLayers; l++)
    if ((rc = dalloc(&s.z[l], r * kN[l])) || (rc = dalloc(&s.a[l], r * kN[l]))) {
      free_acts(s);
      return rc;
    }
  s.cap = rows;
  return MCS_OK;
}

// xorshift-free reproducible normal draws for the initialisation (SplitMix64 + Box-Muller)
struct Rng {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

void init_host(std::vector<float>& p, uint64_t seed) {
  p.assign(kLay.total, 0.f);
  for (int c = 0; c < kIn; c++) p[kLay.stdv + c] = 1.f;
  Rng rng{seed ^ 0xC0FFEEULL};
  const int fan_in[kLayers] = {kIn, kHid, kHid, kHid};
  for (int l = 0; l < kLayers; l++) {
    const int K = kK[l], N = kN[l];
    const int kreal = l == 0 ? kIn : K, nreal = l == kLayers - 1 ? 2 : N;
    const double lim = std::sqrt(6.0 / fan_in[l]) * (l == kLayers - 1 ? 0.1 : 1.0);
    for (int k = 0; k < kreal; k++)
      for (int n = 0; n < nreal; n++)
        p[kLay.W[l] + (size_t)k * N + n] = (float)((2 * rng.uniform() - 1) * lim);
  }
}

int upload_params(mcs_surrogate* s, const float* host) {
  MCS_CUDA_RET(cudaMemcpy(s->params, host, kLay.total * sizeof(float), cudaMemcpyHostToDevice));
  MCS_CUDA_RET(cudaMemset(s->m, 0, kLay.total * sizeof(float)));
  MCS_CUDA_RET(cudaMemset(s->v, 0, kLay.total * sizeof(float)));
  s->step = 0;
  return MCS_OK;
}

int cast_weights(mcs_surrogate* s, cudaStream_t st) {
  for (int l = 0; l < kLayers; l++) {
    const long n = (long)kK[l] * kN[l];
    to_bf16<<<blocks(n, 256), 256, 0, st>>>(s->params + kLay.W[l], n, s->Wb[l]);
    to_bf16_operand<<<blocks(n, 256), 256, 0, st>>>(s->params + kLay.W[l], kK[l], kN[l],
                                                    s->Wt[l]);
  }
  MCS_CUDA_RET(cudaGetLastError());
  return MCS_OK;
}

// The tile width: the widest of 256 ... 16 columns (an MMA's N) that still gives the grid
// 256 CTAs (two per SM fit in shared and tensor memory), so that the staging loads of
// many CTAs are in flight at once and the small weight-gradient GEMMs (M = 32 or 256 over
// K = the batch) spread over the SMs.
void gemm(cudaStream_t st, int* err, const bf16* A, long sAm, long sAk, const bf16* B,
          long sBk, long sBn, float* C, long ldc, int M, int N, int K, bool accumulate) {
  if (M <= 0 || N <= 0 || K <= 0) return;  // nothing to multiply (never an empty grid)
  int nt = std::min(kTcCols, ((N + 15) / 16) * 16);
  const int mt = (M + kTcRows - 1) / kTcRows;
  while (nt > 16 && (long)mt * ((N + nt - 1) / nt) < 256) nt /= 2;
  nt = std::max(16, (nt / 16) * 16);
  int tcols = 32;
  while (tcols < nt) tcols <<= 1;
  const dim3 grid((unsigned)((N + nt - 1) / nt), (unsigned)mt);
  gemm_tc<<<grid, kTcThreads, kGtSmem, st>>>(A, sAm, sAk, B, sBk, sBn, C, ldc, M, N, K, nt,
                                             tcols, accumulate ? 1 : 0, err);
}

// forward of rows already in A.xb; final FP32 output in A.z[3]
void forward(mcs_surrogate* s, Acts& A, int rows, cudaStream_t st) {
  const bf16* x = A.xb;
  for (int l = 0; l < kLayers; l++) {
    const int K = kK[l], N = kN[l];
    gemm(st, s->err, x, K, 1, s->Wb[l], N, 1, A.C, N, rows, N, K, false);
    const long n = (long)rows * N;
    const bool last = l == kLayers - 1;
    bias_act<<<blocks(n, 256), 256, 0, st>>>(A.C, s->params + kLay.b[l], rows, N, A.z[l],
                                             last ? nullptr : A.a[l], last ? 0 : 1);
    x = A.a[l];
  }
}

// backward from the loss gradient in A.dz / A.dzb ([rows x kOutPad]) into s->grad
void backward(mcs_surrogate* s, Acts& A, int rows, cudaStream_t st) {
  for (int l = kLayers - 1; l >= 0; l--) {
    const int K = kK[l], N = kN[l];
    const bf16* ain = l == 0 ? A.xb : A.a[l - 1];
    // dW = a_in^T dz ; db = colsum(dz)
    gemm(st, s->err, ain, 1, K, A.dzb, N, 1, s->grad + kLay.W[l], N, K, N, rows, false);
    col_sum<<<N, 256, 0, st>>>(A.dz, rows, N, s->grad + kLay.b[l]);
    if (l > 0) {
      // dh = dz W^T ; dz_prev = dh * silu'(z_prev)
      gemm(st, s->err, A.dzb, N, 1, s->Wb[l], 1, N, A.dh, K, rows, K, N, false);
      const long n = (long)rows * K;
      silu_back<<<blocks(n, 256), 256, 0, st>>>(A.dh, A.z[l - 1], n, A.dz, A.dzb);
    }
  }
}

// loss (summed, on the device) and its gradient for rows already gathered
void loss_grad(mcs_surrogate* s, Acts& A, int rows, cudaStream_t st) {
  forward(s, A, rows, st);
  nll_loss<<<blocks(rows, 256), 256, 0, st>>>(A.z[kLayers - 1], A.yb, rows, A.dz, A.dzb,
                                              s->loss);
  backward(s, A, rows, st);
}

}  // namespace

// ---- internal entry points used by the guided solve (mcs_api.cu) ----
// Allocates the inference buffers once (before any stream capture that uses them).
// Sets up what inference needs before any stream capture that uses it.
int surrogate_reserve(mcs_surrogate* s) {
  MCS_CUDA_RET(cudaFuncSetAttribute(mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kTcSmem));
  MCS_CUDA_RET(cudaFuncSetAttribute(gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kGtSmem));
  return MCS_OK;
}

// mu, sigma and the guide of n rows of raw features on the device (tcgen05 kernel).  Rows
// a timed-out kernel did not reach keep a NaN guide, which sends them to the plain
// bisection.
int surrogate_predict_device(mcs_surrogate* s, const float* dX, long n, float* d_mu,
                             float* d_sigma, float2* d_guide, const mcs_guide_opts* g,
                             cudaStream_t st, double a_max) {
  if (n <= 0) return MCS_OK;
  int rc = surrogate_reserve(s);
  if (rc) return rc;
  if (d_guide) MCS_CUDA_RET(cudaMemsetAsync(d_guide, 0xFF, sizeof(float2) * n, st));
  TcWeights tw;
  for (int l = 0; l < kLayers; l++) tw.w[l] = s->Wt[l];
  const long tiles = (n + kTcRows - 1) / kTcRows;
  const int grid = (int)std::min<long>(tiles, std::max(1, s->sms));
  mlp_infer_tc<<<grid, kTcThreads, kTcSmem, st>>>(
      dX, n, s->params, tw, d_mu, d_sigma, d_guide, g ? g->z : 0.f, g ? g->hw_min : 0.f,
      g ? g->hw_max : 0.f, g ? g->hw_direct : 0.f,
      g && g->mode == MCS_GUIDE_SPECULATE ? 1 : 0, g ? g->skip_top : 0.f,
      a_max > 0.0 ? (float)std::log(a_max) : 0.f, s->err);
  MCS_CUDA_RET(cudaGetLastError());
  return MCS_OK;
}

// Reports (and clears) a timed-out inference; call after the stream has been synchronised.
int surrogate_check(mcs_surrogate* s) {
  int e = 0;
  MCS_CUDA_RET(cudaMemcpy(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    cudaMemset(s->err, 0, sizeof(int));
    return fail(MCS_ERR_CUDA, "surrogate: a tensor-core wait timed out");
  }
  return MCS_OK;
}

mcs_ctx* surrogate_ctx(mcs_surrogate* s) { return s->ctx; }
std::mutex& surrogate_mutex(mcs_surrogate* s) { return s->mu; }
void surrogate_hold(mcs_surrogate* s, int delta) { s->plans += delta; }

}  // namespace mcs

extern "C" {

void mcs_default_train_opts(mcs_train_opts* o) {
  if (!o) return;
  o->epochs = 20;
  o->batch = 4096;
  o->lr = 1e-3f;
  o->beta1 = 0.9f;
  o->beta2 = 0.999f;
  o->eps = 1e-8f;
  o->seed = 1;
  o->warm = 0;
  o->keep_best = 1;
}

void mcs_default_guide_opts(mcs_guide_opts* o) {
  if (!o) return;
  o->z = 2.0f;
  o->hw_min = 0.13976194f;  // log(1.15)
  o->hw_max = 0.40546511f;  // log(1.5)
  o->hw_direct = 0.69314718f;  // log(2)
  o->refine = 3;
  o->mode = MCS_GUIDE_SPECULATE;
  o->levels = 8;
  o->skip_top = 0.f;
}

int mcs_surrogate_create(mcs_ctx* ctx, uint64_t seed, mcs_surrogate** out) {
  if (!ctx || !out) return fail(MCS_ERR_ARG, "NULL ctx or surrogate pointer");
  *out = nullptr;
  MCS_CUDA_RET(cudaSetDevice(ctx_device(ctx)));
  mcs_surrogate* s = new mcs_surrogate();
  s->ctx = ctx;
  s->seed = seed;
  int rc;
  if ((rc = dalloc(&s->params, kLay.total)) || (rc = dalloc(&s->grad, kLay.total)) ||
      (rc = dalloc(&s->m, kLay.total)) || (rc = dalloc(&s->v, kLay.total)) ||
      (rc = dalloc(&s->loss, 1))) {
    mcs_surrogate_destroy(s);
    return rc;
  }
  for (int l = 0; l < kLayers; l++)
    if ((rc = dalloc(&s->Wb[l], (size_t)kK[l] * kN[l])) ||
        (rc = dalloc(&s->Wt[l], (size_t)kK[l] * kN[l]))) {
      mcs_surrogate_destroy(s);
      return rc;
    }
  if ((rc = dalloc(&s->err, 1)) || (rc = surrogate_reserve(s))) {
    mcs_surrogate_destroy(s);
    return rc;
  }
  cudaMemset(s->err, 0, sizeof(int));
  cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, ctx_device(ctx));
  std::vector<float> p;
  init_host(p, seed);
  if ((rc = upload_params(s, p.data())) || (rc = cast_weights(s, ctx_stream(ctx))) ||
      (rc = cudaStreamSynchronize(ctx_stream(ctx)) == cudaSuccess ? 0
                                                                  : fail(MCS_ERR_CUDA, "init failed"))) {
    mcs_surrogate_destroy(s);
    return rc;
  }
  *out = s;
  return MCS_OK;
}

int mcs_surrogate_destroy(mcs_surrogate* s) {
  if (!s) return MCS_OK;
  if (s->plans.load() > 0)
    return fail(MCS_ERR_STATE, "%d guided plan(s) still use this surrogate", s->plans.load());
  cudaSetDevice(ctx_device(s->ctx));
  cudaStreamSynchronize(ctx_stream(s->ctx));
  free_acts(s->tr);
  cudaFree(s->params);
  cudaFree(s->grad);
  cudaFree(s->m);
  cudaFree(s->v);
  cudaFree(s->loss);
  for (int l = 0; l < kLayers; l++) {
    cudaFree(s->Wb[l]);
    cudaFree(s->Wt[l]);
  }
  cudaFree(s->err);
  delete s;
  return MCS_OK;
}

int mcs_surrogate_get_params(mcs_surrogate* s, float* out, size_t* n) {
  if (!s || !n) return fail(MCS_ERR_ARG, "NULL surrogate or size");
  if (!out) {
    *n = kLay.total;
    return MCS_OK;
  }
  if (*n < kLay.total) return fail(MCS_ERR_ARG, "buffer holds %zu floats, %zu needed", *n, kLay.total);
  std::lock_guard<std::mutex> lk(s->mu);
  MCS_CUDA_RET(cudaSetDevice(ctx_device(s->ctx)));
  MCS_CUDA_RET(cudaStreamSynchronize(ctx_stream(s->ctx)));
  MCS_CUDA_RET(cudaMemcpy(out, s->params, kLay.total * sizeof(float), cudaMemcpyDeviceToHost));
  *n = kLay.total;
  return MCS_OK;
}

int mcs_surrogate_set_params(mcs_surrogate* s, const float* in, size_t n) {
  if (!s || !in) return fail(MCS_ERR_ARG, "NULL surrogate or parameters");
  if (n != kLay.total) return fail(MCS_ERR_ARG, "expected %zu floats, got %zu", kLay.total, n);
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(in[i])) return fail(MCS_ERR_ARG, "parameter %zu is not finite", i);
  for (int c = 0; c < kIn; c++)
    if (!(in[kLay.stdv + c] > 0)) return fail(MCS_ERR_ARG, "feature scale %d must be > 0", c);
  std::lock_guard<std::mutex> lk(s->mu);
  MCS_CUDA_RET(cudaSetDevice(ctx_device(s->ctx)));
  cudaStreamSynchronize(ctx_stream(s->ctx));
  int rc = upload_params(s, in);
  if (!rc) rc = cast_weights(s, ctx_stream(s->ctx));
  if (!rc) MCS_CUDA_RET(cudaStreamSynchronize(ctx_stream(s->ctx)));
  s->trained = true;
  return rc;
}

int mcs_surrogate_grad(mcs_surrogate* s, const float* X, const float* y, size_t n, float* loss,
                       float* grad) {
  if (!s || !X || !y || !loss || !grad || n == 0 || n > (1u << 20))
    return fail(MCS_ERR_ARG, "bad arguments to mcs_surrogate_grad");
  std::lock_guard<std::mutex> lk(s->mu);
  MCS_CUDA_RET(cudaSetDevice(ctx_device(s->ctx)));
  int rc = ensure_acts(s->tr, (int)n);
  if (rc) return rc;
  float *dX = nullptr, *dy = nullptr;
  if ((rc = dalloc(&dX, n * kIn)) || (rc = dalloc(&dy, n))) {
    cudaFree(dX);
    return rc;
  }
  cudaStream_t st = ctx_stream(s->ctx);
  cudaMemcpyAsync(dX, X, n * kIn * sizeof(float), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dy, y, n * sizeof(float), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(s->loss, 0, sizeof(float), st);
  cudaMemsetAsync(s->grad, 0, kLay.total * sizeof(float), st);
  gather_rows<<<blocks((long)n * kInPad, 256), 256, 0, st>>>(
      dX, nullptr, 0, (int)n, (long)n, s->params + kLay.mean, s->params + kLay.stdv, dy,
      s->tr.xb, s->tr.yb);
  loss_grad(s, s->tr, (int)n, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess)
    e = cudaMemcpy(grad, s->grad, kLay.total * sizeof(float), cudaMemcpyDeviceToHost);
  float ls = 0.f;
  if (e == cudaSuccess) e = cudaMemcpy(&ls, s->loss, sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dX);
  cudaFree(dy);
  if (e != cudaSuccess) return fail(MCS_ERR_CUDA, "gradient failed: %s", cudaGetErrorString(e));
  rc = surrogate_check(s);
  if (rc) return rc;
  *loss = ls / (float)n;
  return MCS_OK;
}

int mcs_surrogate_train(mcs_surrogate* s, const float* X, const float* y, size_t n,
                        const float* Xv, const float* yv, size_t nv, const mcs_train_opts* o,
                        float* train_loss, float* val_loss) {
  if (!s || !X || !y || !o || n == 0) return fail(MCS_ERR_ARG, "bad arguments to train");
  if (o->batch < 16 || o->batch > 65536 || o->epochs < 1 || !(o->lr > 0))
    return fail(MCS_ERR_ARG, "train options out of range");
  if (nv && (!Xv || !yv)) return fail(MCS_ERR_ARG, "validation arrays missing");
  if (n > (size_t)INT32_MAX || nv > (size_t)INT32_MAX) return fail(MCS_ERR_ARG, "too many rows");
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(y[i])) return fail(MCS_ERR_ARG, "target %zu is not finite", i);
  std::lock_guard<std::mutex> lk(s->mu);
  MCS_CUDA_RET(cudaSetDevice(ctx_device(s->ctx)));
  int rc = MCS_OK;
  if (!o->warm) {
    // feature normalisation from the training set, fresh weights and Adam state
    std::vector<double> mean(kIn, 0.0), var(kIn, 0.0);
    for (size_t i = 0; i < n; i++)
      for (int c = 0; c < kIn; c++) mean[c] += X[i * kIn + c];
    for (int c = 0; c < kIn; c++) mean[c] /= (double)n;
    for (size_t i = 0; i < n; i++)
      for (int c = 0; c < kIn; c++) {
        const double d = X[i * kIn + c] - mean[c];
        var[c] += d * d;
      }
    std::vector<float> p;
    init_host(p, s->seed);
    for (int c = 0; c < kIn; c++) {
      p[kLay.mean + c] = (float)mean[c];
      p[kLay.stdv + c] = (float)std::max(1e-6, std::sqrt(var[c] / (double)n));
    }
    cudaStreamSynchronize(ctx_stream(s->ctx));
    rc = upload_params(s, p.data());
    if (!rc) rc = cast_weights(s, ctx_stream(s->ctx));
  }
  const int B = o->batch;
  const bool keep = o->keep_best && nv > 0 && val_loss != nullptr;
  if (!rc) rc = ensure_acts(s->tr, B);
  float *dX = nullptr, *dy = nullptr, *dXv = nullptr, *dyv = nullptr, *best = nullptr;
  int32_t* dperm = nullptr;
  if (!rc && ((rc = dalloc(&dX, n * kIn)) || (rc = dalloc(&dy, n)) ||
              (rc = dalloc(&dperm, n)) || (rc = dalloc(&dXv, std::max<size_t>(nv, 1) * kIn)) ||
              (rc = dalloc(&dyv, std::max<size_t>(nv, 1))) ||
              (keep && (rc = dalloc(&best, kLay.total))))) {
  }
  auto cleanup = [&]() {
    cudaFree(dX);
    cudaFree(dy);
    cudaFree(dperm);
    cudaFree(dXv);
    cudaFree(dyv);
    cudaFree(best);
  };
  if (rc) {
    cleanup();
    return rc;
  }
  cudaStream_t st = ctx_stream(s->ctx);
  cudaStreamSynchronize(st);
  cudaMemcpy(dX, X, n * kIn * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(dy, y, n * sizeof(float), cudaMemcpyHostToDevice);
  if (nv) {
    cudaMemcpy(dXv, Xv, nv * kIn * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dyv, yv, nv * sizeof(float), cudaMemcpyHostToDevice);
  }
  Acts& A = s->tr;
  // the shuffle stream continues across warm-started calls
  Rng rng{s->seed * 0x2545F4914F6CDD1DULL + 7 + (uint64_t)s->step * 0x9E3779B97F4A7C15ULL};
  float best_loss = INFINITY;
  std::vector<int32_t> perm(n);
  const long steps = (long)(n / (size_t)B);
  const long trainable = (long)(kLay.total - kLay.W[0]);
  for (int ep = 0; ep < o->epochs && !rc; ep++) {
    for (size_t i = 0; i < n; i++) perm[i] = (int32_t)i;
    for (size_t i = n - 1; i > 0; i--) std::swap(perm[i], perm[rng.next() % (i + 1)]);
    cudaMemcpyAsync(dperm, perm.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(s->loss, 0, sizeof(float), st);
    for (long k = 0; k < std::max<long>(steps, 1); k++) {
      const int rows = steps ? B : (int)n;
      gather_rows<<<blocks((long)rows * kInPad, 256), 256, 0, st>>>(
          dX, dperm, k * (long)B, rows, (long)n, s->params + kLay.mean, s->params + kLay.stdv, dy,
          A.xb, A.yb);
      loss_grad(s, A, rows, st);
      s->step++;
      const float c1 = 1.f - std::pow(o->beta1, (float)s->step);
      const float c2 = 1.f - std::pow(o->beta2, (float)s->step);
      adam<<<blocks(trainable, 256), 256, 0, st>>>(s->params + kLay.W[0], s->m + kLay.W[0],
                                                   s->v + kLay.W[0], s->grad + kLay.W[0],
                                                   trainable, o->lr, o->beta1, o->beta2, o->eps,
                                                   c1, c2);
      rc = cast_weights(s, st);
      if (rc) break;
    }
    float ls = 0.f;
    cudaError_t e = cudaMemcpyAsync(&ls, s->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // (the host permutation is reused)
    if (e != cudaSuccess) {
      rc = fail(MCS_ERR_CUDA, "training failed: %s", cudaGetErrorString(e));
      break;
    }
    if (train_loss) train_loss[ep] = ls / (float)(steps ? steps * B : (long)n);
    if (val_loss && nv) {
      cudaMemsetAsync(s->loss, 0, sizeof(float), st);
      for (size_t off = 0; off < nv; off += (size_t)B) {
        const int rows = (int)std::min<size_t>((size_t)B, nv - off);
        gather_rows<<<blocks((long)rows * kInPad, 256), 256, 0, st>>>(
            dXv, nullptr, (long)off, rows, (long)nv, s->params + kLay.mean,
            s->params + kLay.stdv, dyv, A.xb, A.yb);
        forward(s, A, rows, st);
        nll_loss<<<blocks(rows, 256), 256, 0, st>>>(A.z[kLayers - 1], A.yb, rows, A.dz, A.dzb,
                                                    s->loss);
      }
      e = cudaMemcpyAsync(&ls, s->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) {
        rc = fail(MCS_ERR_CUDA, "validation failed: %s", cudaGetErrorString(e));
        break;
      }
      val_loss[ep] = ls / (float)nv;
      if (keep && val_loss[ep] < best_loss) {
        best_loss = val_loss[ep];
        cudaMemcpyAsync(best, s->params, kLay.total * sizeof(float), cudaMemcpyDeviceToDevice,
                        st);
      }
    }
  }
  if (!rc && keep && best_loss < INFINITY) {
    cudaMemcpyAsync(s->params, best, kLay.total * sizeof(float), cudaMemcpyDeviceToDevice, st);
    rc = cast_weights(s, st);
  }
  cudaStreamSynchronize(st);
  cleanup();
  if (!rc) rc = surrogate_check(s);  // a training GEMM whose tensor-core wait timed out
  if (!rc) s->trained = true;
  return rc;
}

int mcs_surrogate_predict(mcs_surrogate* s, const float* X, size_t n, float* mu, float* sigma) {
  if (!s || (n && (!X || !mu || !sigma))) return fail(MCS_ERR_ARG, "bad arguments to predict");
  if (n == 0) return MCS_OK;
  std::lock_guard<std::mutex> lk(s->mu);
  MCS_CUDA_RET(cudaSetDevice(ctx_device(s->ctx)));
  float *dX = nullptr, *dmu = nullptr, *dsg = nullptr;
  int rc;
  if ((rc = dalloc(&dX, n * kIn)) || (rc = dalloc(&dmu, n)) || (rc = dalloc(&dsg, n))) {
    cudaFree(dX);
    cudaFree(dmu);
    return rc;
  }
  cudaStream_t st = ctx_stream(s->ctx);
  cudaMemcpyAsync(dX, X, n * kIn * sizeof(float), cudaMemcpyHostToDevice, st);
  rc = surrogate_predict_device(s, dX, (long)n, dmu, dsg, nullptr, nullptr, st, 0.0);
  cudaError_t e = cudaStreamSynchronize(st);
  if (!rc && e == cudaSuccess) rc = surrogate_check(s);
  if (!rc && e == cudaSuccess) e = cudaMemcpy(mu, dmu, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (!rc && e == cudaSuccess)
    e = cudaMemcpy(sigma, dsg, n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dX);
  cudaFree(dmu);
  cudaFree(dsg);
  if (!rc && e != cudaSuccess) rc = fail(MCS_ERR_CUDA, "predict failed: %s", cudaGetErrorString(e));
  return rc;
}

}  // extern "C"
