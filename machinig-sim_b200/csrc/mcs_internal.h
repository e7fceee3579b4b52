// Internal types shared by the host preparation (mcs_api.cu) and the sm_100a kernels
// (mcs_kernels.cu).  Not part of the C ABI.
#pragma once

#include <cstdint>

#include "../../include/mcs.h"

#include <cuda_runtime.h>

#include <mutex>

namespace mcs {

// Records a message for mcs_last_error() (per thread) and returns code.
int fail(int code, const char* fmt, ...);

#define MCS_CUDA_RET(call)                                                                \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return ::mcs::fail(MCS_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
  } while (0)

int ctx_device(mcs_ctx* ctx);
cudaStream_t ctx_stream(mcs_ctx* ctx);

constexpr int kMaxTeeth = MCS_MAX_TEETH;
constexpr int kMaxModes = MCS_MAX_MODES;
constexpr int kMaxSlots = 2;          // slices per lane: nz <= 64
constexpr int kWarp = 32;
constexpr int kMaxSmemPerWarp = 227 * 1024;

// Per-point constants, derived on the host in FP64 exactly as CuttingEngine.configure
// derives them (src/cutting.js:39-82), plus the engagement window of the static arc map
// chatterAt builds (src/stabtd.js:17).  One record per (setup, speed, modal) point.
struct alignas(16) PointParams {
  double omega;      // spindle angular speed [rad/s]
  double dphi;       // rotation per step [rad]
  double dt;         // step [s]
  double R, tanB;    // radius [mm], tan(helix)
  double flute_len;  // [mm] (chatterAt raises it to ap + 1 per trial)
  double Ci;         // process-damping coefficient [N/m], 0 when linear
  double phi_lo;     // engaged angles [phi_lo, phi_hi): bins b0..b1 of the arc map
  double phi_hi;
  double fz, hmax;   // feed per tooth, chip-thickness cap [mm]
  double Ktc, Krc, Kte, Kre;
  double mc;         // size-effect exponent, 0 when linear
  double dR[kMaxTeeth];                 // runout offset of each tooth [mm]
  double mk[2][kMaxModes];              // modal stiffness [N/m] (x, y); 0 when padded
  double mcd[2][kMaxModes];             // modal damping [N s/m]
  double ma[2][kMaxModes];              // dt / modal mass
  int32_t N, spt, spr, decim;
  int32_t nsteps;                       // spt * N * revs
  int32_t type;                         // mcs_tool_type
  int32_t slices_override;              // > 0: equal slices
  int32_t excl_zero;                    // arc map starts at bin 0: phi == 0 is not in cut
  int32_t lpad;                         // ring row pitch (floats)
  int32_t nz_max;                       // slices at the deepest trial of the point
  int32_t ts_c0;                        // first tooth sample inside the index window
  int32_t ts_n;                         // tooth samples in the window (<= 24)
  int32_t hist_h0;                      // first history sample inside the window
  int32_t hist_m;                       // history samples in the window
  int32_t smem_bytes;                   // table + ring + sample/result area (warp_smem)
  int32_t empty;                        // arc covers no bin
  int32_t ring_rows;                    // ring rows: nz_max, or 32 if larger and groups > 1
  int32_t groups;                       // trials one warp may run together (1 or kMaxGroups)
};

// Shared memory of one warp: the sin/cos table of the revolution's positions (float2 or
// double2 by integration precision) followed by the surface ring (always float: the
// reference stores the surface in a Float32Array).
__host__ __device__ inline int table_bytes(int spr, bool fp64) {
  return (spr * (fp64 ? 16 : 8) + 15) & ~15;
}

// After the table and the ring: per trial group, its once-per-tooth samples (float2) and
// its result record.  A warp runs up to kMaxGroups trials of one point together in lane
// groups (speculative bisection levels).
constexpr int kMaxGroups = 16;
constexpr int kToothSamples = 24;
constexpr int kTrialOutBytes = 48;
__host__ __device__ inline int extra_offset(int spr, bool fp64, int ring_rows, int lpad) {
  return (table_bytes(spr, fp64) + 4 * ring_rows * lpad + 15) & ~15;
}
__host__ __device__ inline int warp_smem(int spr, bool fp64, int ring_rows, int lpad,
                                         int groups) {
  return extra_offset(spr, fp64, ring_rows, lpad) + groups * (kToothSamples * 8 + kTrialOutBytes);
}

// Multi-warp solve (several warps share one point's bisection, one trial per warp): the
// table once, then a surface ring and a result record per warp.
constexpr int kCoopMaxWarpsHost = 8;
constexpr int kCoopSmemLimit = kMaxSmemPerWarp - 1024;  // dynamic bytes; static words beside
__host__ __device__ inline int coop_ring_bytes(int ring_rows, int lpad) {
  return (4 * ring_rows * lpad + 15) & ~15;
}
__host__ __device__ inline int coop_smem(int spr, bool fp64, int ring_rows, int lpad, int warps) {
  return table_bytes(spr, fp64) + warps * (coop_ring_bytes(ring_rows, lpad) + kTrialOutBytes);
}

// Options the kernels read (mcs_opts reduced to what the device needs).
struct DevOpts {
  double a_min, a_max, chatter_idx;
  int32_t iters, pad;
};

// Surrogate guidance of the solve kernel (all NULL: the plain algorithm).
struct GuideArgs {
  const float2* guide = nullptr;  // per point (mu, hw) of the log depth; hw < 0: no guess
  const float* sigma = nullptr;   // per point predicted sigma (reported only)
  mcs_guide_info* info = nullptr; // per point path taken
  float hw_min = 0.f;             // half-width the refinement count is calibrated on
  int refine = 0;                 // halvings of a hw_min bracket
  int mode = 0;                   // MCS_GUIDE_SPECULATE or MCS_GUIDE_BRACKET
  int levels = 0;                 // speculate: bisection levels
};

// One chatterAt trial of the batch kernel.
struct TrialItem {
  int32_t point;   // index into the PointParams array
  int32_t out;     // index into the caller's result array
  double ap;
};

// Launch shapes (template parameters) the kernels are instantiated for.
struct KernelShape {
  int slots;  // 1 or 2
  int modes;  // 1..4
  int fp64;   // 0: FP32 force law and modal integration, 1: FP64
  int nl;     // 1: size effect and/or process damping present
  int grouped = 0;  // 1: points may run several trials per warp in lane groups
  int coop = 0;     // > 0: solve with this many warps per point (multi-warp bisection)
  int dense = 0;    // 1: the FP64 linear solve held to more resident warps per SM
};

// Host launchers (mcs_kernels.cu).  chained = 1: a programmatic dependent launch behind the
// previous kernel of the stream (the previous bucket of a plan), which it may overlap once
// all of that kernel's blocks are resident, and whose completion its own completion
// implies.
// mcs_kernels.cu is built once per integration precision, into k32 and k64.
#define MCS_KERNEL_API                                                                      \
  int launch_solve(const KernelShape& shape, int grid, int smem, cudaStream_t stream,     \
                   const PointParams* pts, const int32_t* order, int n, DevOpts opts,      \
                   mcs_result* out, unsigned int* queue, const volatile int* cancel,       \
                   unsigned int* progress, const GuideArgs& guide, int priority,           \
                   bool chained);                                                          \
  int launch_trials(const KernelShape& shape, int grid, int smem, cudaStream_t stream,    \
                    const PointParams* pts, const TrialItem* items, int n,                 \
                    double chatter_idx, mcs_trial_result* out, unsigned int* queue,        \
                    int priority, bool chained);                                           \
  int occupancy_solve(const KernelShape& shape, int smem, int* blocks_per_sm);            \
  int occupancy_trials(const KernelShape& shape, int smem, int* blocks_per_sm);           \
  int set_smem_limits();
namespace k32 {
MCS_KERNEL_API
}
namespace k64 {
MCS_KERNEL_API
}
#undef MCS_KERNEL_API
inline int launch_solve(const KernelShape& shape, int grid, int smem, cudaStream_t stream,
                        const PointParams* pts, const int32_t* order, int n, DevOpts opts,
                        mcs_result* out, unsigned int* queue, const volatile int* cancel,
                        unsigned int* progress, const GuideArgs& guide = GuideArgs(),
                        int priority = 0, bool chained = false) {
  return (shape.fp64 ? k64::launch_solve : k32::launch_solve)(
      shape, grid, smem, stream, pts, order, n, opts, out, queue, cancel, progress, guide,
      priority, chained);
}
inline int launch_trials(const KernelShape& shape, int grid, int smem, cudaStream_t stream,
                         const PointParams* pts, const TrialItem* items, int n,
                         double chatter_idx, mcs_trial_result* out, unsigned int* queue,
                         int priority = 0, bool chained = false) {
  return (shape.fp64 ? k64::launch_trials : k32::launch_trials)(
      shape, grid, smem, stream, pts, items, n, chatter_idx, out, queue, priority, chained);
}
inline int occupancy_solve(const KernelShape& shape, int smem, int* blocks_per_sm) {
  return (shape.fp64 ? k64::occupancy_solve : k32::occupancy_solve)(shape, smem, blocks_per_sm);
}
inline int occupancy_trials(const KernelShape& shape, int smem, int* blocks_per_sm) {
  return (shape.fp64 ? k64::occupancy_trials : k32::occupancy_trials)(shape, smem,
                                                                      blocks_per_sm);
}
inline int set_smem_limits() {
  const int rc = k32::set_smem_limits();
  return rc ? rc : k64::set_smem_limits();
}
// surrogate (mcs_surrogate.cu)
int surrogate_predict_device(mcs_surrogate* s, const float* dX, long n, float* d_mu,
                             float* d_sigma, float2* d_guide, const mcs_guide_opts* g,
                             cudaStream_t st, double a_max);
int surrogate_reserve(mcs_surrogate* s);
// after a synchronise: MCS_ERR_CUDA if an inference kernel timed out waiting for its MMAs
int surrogate_check(mcs_surrogate* s);
mcs_ctx* surrogate_ctx(mcs_surrogate* s);
std::mutex& surrogate_mutex(mcs_surrogate* s);
// guided plans that hold the surrogate (it cannot be destroyed while any do)
void surrogate_hold(mcs_surrogate* s, int delta);
// peak-rate probes (mcs_probe.cu); scratch: a device buffer of at least 16 KB
int measure_peaks(cudaStream_t st, int sms, void* scratch, double* fp32_tflops,
                  double* fp64_tflops, double* smem_tbps);
int launch_lobes(cudaStream_t stream, const mcs_modal* modals, const mcs_lobe_query* qs, int n_q,
                 const double* rpm, int n_rpm, double* out, const int* q_begin = nullptr,
                 const int* q_count = nullptr);

}  // namespace mcs
