// sm_100a kernels of the time-domain chatter stability path.
//
// One warp simulates one cut (a chatterAt trial, src/stabtd.js:14-22) and, in the solve
// kernel, runs the whole bisection of timeDomainLimit (src/stabtd.js:24-32) for one
// (setup, speed) point.  Warps take points from an atomic work queue (persistent launch).
//
// Work layout inside a warp (the run() loop of src/cutting.js:168-293):
//   * lane l owns axial slices l and l + 32 (SLOTS = 1 or 2 -> nz <= 64); the slice
//     geometry (cutting.js:98-124) lives in registers for the whole trial;
//   * per step the N teeth are visited in turn; a tooth whose slices are all outside
//     the engaged arc is skipped by the whole warp (vote), otherwise every lane whose
//     slice is in cut evaluates the force law (cutting.js:181-207) in FP32;
//   * Fx, Fy are summed with a butterfly of shuffles, so every lane holds the total and
//     runs the modal update (semi-implicit Euler, cutting.js:246-255) redundantly;
//   * the once-per-tooth samples of the chatter-index window sit one per lane, and the
//     decimated-history statistics are accumulated in FP64 (cutting.js:265-292,299-318).
//
// The delayed surface: the reference keeps surf[slice][position] for a whole revolution
// (cutting.js:62-68).  With the static arc map of chatterAt a (slice, position) cell has
// a fixed angle phi = position*dphi - lag(slice) (mod 2pi), so only the cells whose angle
// lies in the engaged bins are ever read in cut; all other cells are written and never
// read.  The ring therefore holds, per slice, only the positions of the engaged window
// (length <= (phi_hi - phi_lo)/dphi + 2), in shared memory next to a sin/cos table of the
// revolution's positions.  Whether a cell is in cut is an integer window test, so the
// engagement pattern is the one the reference's bin lookup gives (up to angles within
// ~1e-15 rad of a bin edge).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "mcs_internal.h"

namespace mcs {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr float kLog2HRef = -4.321928094887363f;  // log2(H_REF = 0.05 mm), cutting.js:18
constexpr float kHMin = 0.002f;                    // cutting.js:19

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__host__ __device__ __forceinline__ int table_bytes(int spr) { return (spr * 8 + 15) & ~15; }

struct TrialOut {
  double index, once, amp;
  unsigned long long engaged, evals;
  int status;
};

// sin/cos of every position of one revolution: theta(p) = p * dphi.
__device__ __forceinline__ void build_table(const PointParams* __restrict__ P, float2* table,
                                            int lane) {
  const int spr = P->spr;
  const double dphi = P->dphi;
  for (int p = lane; p < spr; p += kWarp) {
    double s, c;
    sincos(p * dphi, &s, &c);
    table[p] = make_float2((float)s, (float)c);
  }
  __syncwarp();
}

// One chatterAt trial at depth ap: configure + setEngagement + kick + run + chatterIndex.
template <int SLOTS, int NM>
__device__ TrialOut simulate_trial(const PointParams* __restrict__ P, double ap,
                                   const float2* __restrict__ table, float* __restrict__ ring,
                                   int lane) {
  TrialOut res;
  const int N = P->N, spt = P->spt, spr = P->spr, lpad = P->lpad;

  // ---- slices of this trial (stabtd.js:16-18 -> cutting.js:63-64, 98-124), FP64 ----
  int nz;
  double dz;
  if (P->slices_override > 0) {
    nz = ap > 0 ? P->slices_override : 0;
    dz = ap / P->slices_override;
  } else {
    const double flute = fmax(P->flute_len, ap + 1.0);
    dz = fmax(0.25, flute / 48.0);
    const int maxs = (int)ceil(flute / dz);
    nz = ap > 0 ? min(maxs, (int)ceil(ap / dz)) : 0;
  }
  // process damping per slice, Ci*b/V_c (cutting.js:155-156,203)
  const double pdK = P->Ci != 0.0 ? P->Ci * dz * 1e-3 / (P->omega * 1e-3) : 0.0;

  float sL[SLOTS], cL[SLOTS], ktb[SLOTS], kteb[SLOTS], krb[SLOTS], kreb[SLOTS], pdc[SLOTS],
      fzk[SLOTS];
  int p0[SLOTS], len[SLOTS], base[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; s++) {
    const int k = lane + kWarp * s;
    sL[s] = cL[s] = ktb[s] = kteb[s] = krb[s] = kreb[s] = pdc[s] = fzk[s] = 0.f;
    p0[s] = 0;
    len[s] = 0;
    base[s] = k * lpad;
    if (k < nz && !P->empty) {
      const double b = fmin(dz, ap - k * dz);
      const double zr = k * dz + 0.5 * b;
      double r = P->R, kap = 1.0;
      if (P->type == MCS_TOOL_BALL && zr < P->R) {
        const double d = P->R - zr;
        r = sqrt(fmax(1e-6, P->R * P->R - d * d));
        kap = r / P->R;
      }
      const double lag = zr * P->tanB / P->R;
      double sl, cl;
      sincos(lag, &sl, &cl);
      sL[s] = (float)sl;
      cL[s] = (float)cl;
      // positions p whose angle p*dphi - lag (mod 2pi) falls in [phi_lo, phi_hi)
      const double u = (P->phi_lo + lag) / P->dphi;
      const double w = (P->phi_hi + lag) / P->dphi;
      double cu = ceil(u);
      double L = ceil(w) - cu;
      if (P->excl_zero && u == cu) {  // phi == 0 has sin(phi) <= 0: out of cut
        cu += 1.0;
        L -= 1.0;
      }
      long long pc = (long long)cu % spr;
      if (pc < 0) pc += spr;
      p0[s] = (int)pc;
      len[s] = (int)fmin(fmax(L, 0.0), (double)lpad);
      ktb[s] = (float)(P->Ktc * b);
      kteb[s] = (float)(P->Kte * b);
      krb[s] = (float)(P->Krc * b);
      kreb[s] = (float)(P->Kre * b);
      pdc[s] = (float)(pdK * (b / dz) / r);
      fzk[s] = (float)((double)P->fz * kap);
    }
  }
  // a fresh engine's surface is all zeros (cutting.js:68)
  for (int i = lane; i < nz * lpad; i += kWarp) ring[i] = 0.f;
  __syncwarp();

  float dRr[kMaxTeeth];
#pragma unroll
  for (int i = 0; i < kMaxTeeth; i++) dRr[i] = P->dR[i];
  float mk[2][NM], mcd[2][NM], ma[2][NM], q[2][NM], v[2][NM];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int j = 0; j < NM; j++) {
      mk[a][j] = P->mk[a][j];
      mcd[a][j] = P->mcd[a][j];
      ma[a][j] = P->ma[a][j];
      q[a][j] = 0.f;
      v[a][j] = 0.f;
    }
  // the kick e.vx = 0.01 m/s goes into the first x mode at the first run (cutting.js:164)
  v[0][0] = 0.01f;
  float x = 0.f, y = 0.f, vxs = 0.01f, vys = 0.f;

  const float hmax = P->hmax, mc = P->mc, dtf = P->dtf;
  const bool size_effect = mc != 0.f;
  const bool pd = pdK != 0.0;
  const int nsteps = P->nsteps, decim = P->decim, ts_c0 = P->ts_c0, h0 = P->hist_h0;
  int pr = 0, phc = 0, dcnt = 0, tcount = 0, hcount = 0, eng = 0;
  float tsx = 0.f, tsy = 0.f;
  double sx = 0.0, sy = 0.0, sxx = 0.0, syy = 0.0, shx = 0.0, shy = 0.0;

  for (int step = 0; step < nsteps; step++) {
    const float xm = x * 1e3f, ym = y * 1e3f;  // tool position [mm]
    float Fx = 0.f, Fy = 0.f;
    int p = pr;  // position of tooth i: pr + i*spt (mod spr)
#pragma unroll
    for (int i = 0; i < kMaxTeeth; i++) {
      if (i >= N) break;
      int jj[SLOTS];
      bool act[SLOTS];
      bool any = false;
#pragma unroll
      for (int s = 0; s < SLOTS; s++) {
        int j = p - p0[s];
        if (j < 0) j += spr;
        jj[s] = j;
        act[s] = j < len[s];
        any |= act[s];
      }
      if (__any_sync(kFull, any)) {
        const float2 sc = table[p];  // sin, cos of p*dphi (same address for all lanes)
#pragma unroll
        for (int s = 0; s < SLOTS; s++) {
          if (act[s]) {
            // phi = p*dphi - lag: rotate the table entry by the slice's helix lag
            const float sn = fmaf(sc.x, cL[s], -sc.y * sL[s]);
            const float cs = fmaf(sc.y, cL[s], sc.x * sL[s]);
            // feed u = [1, 0]: edge normal n = (sin phi, cos phi), tangent t = (cos, -sin)
            const float rn = fmaf(xm, sn, fmaf(ym, cs, dRr[i]));
            float* cell = ring + base[s] + jj[s];
            const float prev = *cell;
            const float feedH = fzk[s] * sn;
            float h = (feedH + rn) - prev;
            if (h <= 0.f) {
              *cell = prev - feedH;  // out of cut: the old surface survives one more feed
            } else {
              *cell = rn;
              h = fminf(h, hmax);
              float kse = h;  // se * h
              if (size_effect)
                kse = h * exp2f(mc * (kLog2HRef - __log2f(fmaxf(h, kHMin))));
              const float Ft = fmaf(ktb[s], kse, kteb[s]);
              float Fr = fmaf(krb[s], kse, kreb[s]);
              if (pd) Fr = fmaf(pdc[s], fmaf(vxs, sn, vys * cs), Fr);
              Fx = fmaf(-Ft, cs, fmaf(-Fr, sn, Fx));
              Fy = fmaf(Ft, sn, fmaf(-Fr, cs, Fy));
              eng++;
            }
          }
        }
      }
      p += spt;
      if (p >= spr) p -= spr;
    }
    Fx = warp_sum(Fx);
    Fy = warp_sum(Fy);
    // modal integration, semi-implicit Euler; padded modes have k = c = dt/m = 0
    float xs = 0.f, ys = 0.f, vxa = 0.f, vya = 0.f;
#pragma unroll
    for (int j = 0; j < NM; j++) {
      v[0][j] = fmaf(fmaf(-mcd[0][j], v[0][j], fmaf(-mk[0][j], q[0][j], Fx)), ma[0][j], v[0][j]);
      q[0][j] = fmaf(v[0][j], dtf, q[0][j]);
      xs += q[0][j];
      vxa += v[0][j];
      v[1][j] = fmaf(fmaf(-mcd[1][j], v[1][j], fmaf(-mk[1][j], q[1][j], Fy)), ma[1][j], v[1][j]);
      q[1][j] = fmaf(v[1][j], dtf, q[1][j]);
      ys += q[1][j];
      vya += v[1][j];
    }
    x = xs;
    y = ys;
    vxs = vxa;
    vys = vya;
    if (++pr == spr) pr = 0;
    if (++phc == spt) {  // once-per-tooth sample (cutting.js:266-268)
      phc = 0;
      if (tcount - ts_c0 == lane) {
        tsx = x;
        tsy = y;
      }
      tcount++;
    }
    if (++dcnt == decim) {  // decimated history (cutting.js:288-292), FP64 window sums
      dcnt = 0;
      if (hcount >= h0) {
        const double hx = (double)(x * 1e6f), hy = (double)(y * 1e6f);
        if (hcount == h0) {
          shx = hx;
          shy = hy;
        }
        const double dx = hx - shx, dy = hy - shy;
        sx += dx;
        sy += dy;
        sxx = fma(dx, dx, sxx);
        syy = fma(dy, dy, syy);
      }
      hcount++;
    }
  }

  // ---- chatterIndex (cutting.js:299-318) in FP64 ----
  res.engaged = (unsigned long long)__reduce_add_sync(kFull, (unsigned)eng);
  res.evals = (unsigned long long)nsteps * (unsigned long long)(N * nz);
  const int n = P->ts_n;
  if (n < 8) {
    res.index = 0.0;
    res.once = 0.0;
    res.amp = 0.0;
  } else {
    const bool mine = lane < n;
    const double tx = mine ? (double)tsx : 0.0, ty = mine ? (double)tsy : 0.0;
    const double mx = warp_sum(tx) / n, my = warp_sum(ty) / n;
    const double ex = mine ? (double)tsx - mx : 0.0, ey = mine ? (double)tsy - my : 0.0;
    const double vv = warp_sum(ex * ex + ey * ey);
    const double once = sqrt(vv / n) * 1e6;
    const double md = P->hist_m ? (double)P->hist_m : 1.0;
    const double w = fmax(0.0, (sxx - sx * sx / md) + (syy - sy * sy / md));
    const double amp = sqrt(w / md);
    res.once = once;
    res.amp = amp;
    res.index = once / (amp + 0.05);
  }
  res.status = (isfinite(x) && isfinite(y) && isfinite(res.index)) ? MCS_OK : MCS_ERR_DIVERGED;
  return res;
}

__device__ __forceinline__ bool read_cancel(const volatile int* cancel, int lane) {
  int c = 0;
  if (cancel != nullptr && lane == 0) c = *cancel;
  return __shfl_sync(kFull, c, 0) != 0;
}

// Persistent solve: each warp takes points from the queue and runs timeDomainLimit.
template <int SLOTS, int NM>
__global__ void __launch_bounds__(kWarp) solve_kernel(const PointParams* __restrict__ pts,
                                                      const int32_t* __restrict__ order, int n,
                                                      DevOpts o, mcs_result* __restrict__ out,
                                                      unsigned int* __restrict__ queue,
                                                      const volatile int* cancel,
                                                      unsigned int* progress) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x;
  for (;;) {
    unsigned int w = 0;
    if (lane == 0) w = atomicAdd(queue, 1u);
    w = __shfl_sync(kFull, w, 0);
    if (w >= (unsigned)n) break;
    const int pi = order[w];
    const PointParams* P = pts + pi;
    float2* table = reinterpret_cast<float2*>(smem);
    float* ring = reinterpret_cast<float*>(smem + table_bytes(P->spr));
    mcs_result r;
    r.status = MCS_OK;
    r.trials = 0;
    r.evals = 0;
    r.engaged = 0;
    r.steps_per_tooth = P->spt;
    r.open = 0;
    r.alim = r.lo = r.hi = 0.0;
    if (read_cancel(cancel, lane)) {
      r.status = MCS_ERR_CANCELLED;
    } else {
      build_table(P, table, lane);
      auto chatter = [&](double ap, bool& ok) -> bool {
        const TrialOut t = simulate_trial<SLOTS, NM>(P, ap, table, ring, lane);
        r.trials++;
        r.evals += t.evals;
        r.engaged += t.engaged;
        if (t.status != MCS_OK) r.status = t.status;
        ok = t.status == MCS_OK;
        return t.index > o.chatter_idx;
      };
      bool ok = true;
      if (!chatter(o.a_max, ok)) {
        r.alim = o.a_max;
        r.lo = o.a_max;
        r.hi = INFINITY;
        r.open = 1;
      } else {
        double lo = o.a_min, hi = o.a_max;
        for (int it = 0; it < o.iters; it++) {
          if (read_cancel(cancel, lane)) {
            r.status = MCS_ERR_CANCELLED;
            break;
          }
          const double m = sqrt(lo * hi);
          if (chatter(m, ok))
            hi = m;
          else
            lo = m;
        }
        r.alim = sqrt(lo * hi);
        r.lo = lo;
        r.hi = hi;
      }
    }
    if (lane == 0) {
      out[pi] = r;
      if (progress != nullptr) atomicAdd(progress, 1u);
    }
    __syncwarp();
  }
}

// Batch of independent chatterAt trials (decision replay at given depths).
template <int SLOTS, int NM>
__global__ void __launch_bounds__(kWarp) trials_kernel(const PointParams* __restrict__ pts,
                                                       const TrialItem* __restrict__ items,
                                                       int n, double chatter_idx,
                                                       mcs_trial_result* __restrict__ out,
                                                       unsigned int* __restrict__ queue) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x;
  for (;;) {
    unsigned int w = 0;
    if (lane == 0) w = atomicAdd(queue, 1u);
    w = __shfl_sync(kFull, w, 0);
    if (w >= (unsigned)n) break;
    const TrialItem it = items[w];
    const PointParams* P = pts + it.point;
    float2* table = reinterpret_cast<float2*>(smem);
    float* ring = reinterpret_cast<float*>(smem + table_bytes(P->spr));
    build_table(P, table, lane);
    const TrialOut t = simulate_trial<SLOTS, NM>(P, it.ap, table, ring, lane);
    if (lane == 0) {
      mcs_trial_result r;
      r.index = t.index;
      r.once = t.once;
      r.amp = t.amp;
      r.chatter = t.index > chatter_idx ? 1 : 0;
      r.status = t.status;
      out[it.out] = r;
    }
    __syncwarp();
  }
}

template <int SLOTS, int NM>
void* solve_fn() {
  return reinterpret_cast<void*>(&solve_kernel<SLOTS, NM>);
}
template <int SLOTS, int NM>
void* trials_fn() {
  return reinterpret_cast<void*>(&trials_kernel<SLOTS, NM>);
}

void* pick(bool solve, const KernelShape& s) {
#define MCS_PICK(SL, NMV)                                      \
  if (s.slots == SL && s.modes == NMV)                         \
    return solve ? solve_fn<SL, NMV>() : trials_fn<SL, NMV>();
  MCS_PICK(1, 1)
  MCS_PICK(1, 2)
  MCS_PICK(1, 3)
  MCS_PICK(1, 4)
  MCS_PICK(2, 1)
  MCS_PICK(2, 2)
  MCS_PICK(2, 3)
  MCS_PICK(2, 4)
#undef MCS_PICK
  return nullptr;
}

}  // namespace

int set_smem_limits() {
  for (int sl = 1; sl <= kMaxSlots; sl++)
    for (int nm = 1; nm <= kMaxModes; nm++)
      for (int k = 0; k < 2; k++) {
        void* f = pick(k == 0, KernelShape{sl, nm});
        cudaError_t e =
            cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemPerWarp);
        if (e != cudaSuccess) return (int)e;
        e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return (int)e;
      }
  return 0;
}

int occupancy_solve(const KernelShape& shape, int smem, int* blocks_per_sm) {
  void* f = pick(true, shape);
  if (!f) return (int)cudaErrorInvalidValue;
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, kWarp, smem);
}

int occupancy_trials(const KernelShape& shape, int smem, int* blocks_per_sm) {
  void* f = pick(false, shape);
  if (!f) return (int)cudaErrorInvalidValue;
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, kWarp, smem);
}

int launch_solve(const KernelShape& shape, int grid, int smem, cudaStream_t stream,
                 const PointParams* pts, const int32_t* order, int n, DevOpts opts,
                 mcs_result* out, unsigned int* queue, const volatile int* cancel,
                 unsigned int* progress) {
  void* f = pick(true, shape);
  if (!f) return (int)cudaErrorInvalidValue;
  void* args[] = {&pts, &order, &n, &opts, &out, &queue, &cancel, &progress};
  return (int)cudaLaunchKernel(f, dim3(grid), dim3(kWarp), args, (size_t)smem, stream);
}

int launch_trials(const KernelShape& shape, int grid, int smem, cudaStream_t stream,
                  const PointParams* pts, const TrialItem* items, int n, double chatter_idx,
                  mcs_trial_result* out, unsigned int* queue) {
  void* f = pick(false, shape);
  if (!f) return (int)cudaErrorInvalidValue;
  void* args[] = {&pts, &items, &n, &chatter_idx, &out, &queue};
  return (int)cudaLaunchKernel(f, dim3(grid), dim3(kWarp), args, (size_t)smem, stream);
}

}  // namespace mcs
